/*
 * fa_oracle.h — CPU oracle for the batched Atari 2600 core.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * CPU emulator path (RPP1011/fast-atari-rs):
 *   src/cpu.rs           Cpu, Status, reset, step       (oracle/cpu_step.h)
 *   src/atari.rs:9-105   Action, BankScheme::detect
 *   src/atari.rs:384-620 HeadlessBus, HeadlessAtari
 *   src/headless_tia.rs  HeadlessTia
 *   src/pia.rs           Pia
 * It is the checker for the CUDA path and the timed CPU baseline; only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load it.
 *
 * Parity pinning: instruction level by the reference's own known-answer tests
 * (tests/cycle_counts.rs, restated in tests/test_oracle_kat.py); frame level by
 * this restatement only (the reference is Rust and no Rust toolchain exists
 * here), frozen as self-generated regression vectors under tests/golden/.
 */
#ifndef FA_ORACLE_H
#define FA_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/fast_atari.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_atari orc_atari;

/* 6502 registers for the flat-memory known-answer runner. */
typedef struct orc_regs {
    uint16_t pc;
    uint8_t  sp, a, x, y, p, _pad;
    uint64_t cycles;
} orc_regs;

/* The oracle's counterpart of fa_rom_set_scheme: the scheme of one ROM image
 * (by its bytes) for every later orc_create / orc_rcreate / orc_reset_state /
 * orc_run_batch given the same bytes; scheme < 0 removes the record.  E0 and
 * 3F are restated from the published behaviour of those carts (the reference
 * has neither).  Returns 0, or -1 for a length the scheme cannot hold.  Not
 * thread-safe: register before running. */
int orc_rom_set_scheme(const uint8_t* rom, size_t rom_len, int scheme);

/* HeadlessAtari::new (src/atari.rs:562-569).  Returns NULL for ROM lengths the
 * reference cannot construct (it panics on those). */
orc_atari* orc_create(const uint8_t* rom, size_t rom_len);
orc_atari* orc_clone(const orc_atari* e);
void       orc_destroy(orc_atari* e);

/* HeadlessAtari::set_action (src/atari.rs:571-582); index > 17 is NOOP. */
void     orc_set_action(orc_atari* e, unsigned action);
/* HeadlessAtari::run_frame (src/atari.rs:584-598); returns frame cycles. */
uint64_t orc_run_frame(orc_atari* e);
/* HeadlessAtari::ram (src/atari.rs:617-619): 128 bytes. */
void     orc_ram(const orc_atari* e, uint8_t* out128);
/* Number of instructions executed since creation (work-unit counter). */
uint64_t orc_instructions(const orc_atari* e);

/* AtariStateGpu::from_headless (src/cuda_env.rs:43-93) plus the extension. */
void orc_get_state(const orc_atari* e, fa_state* out);
/* Inverse: rebuild the emulator (incl. its flat memory) from a state. */
void orc_set_state(orc_atari* e, const fa_state* in);

/* BatchAtariGpu::reset for one instance (src/cuda_env.rs:134-139):
 * new(rom) + run_frame(); frame_no is 0 afterwards. */
int orc_reset_state(const uint8_t* rom, size_t rom_len, fa_state* out);

/*
 * Run n instances for k frames each from `states` (in/out), actions
 * frame-major (actions[f*n + i]).  Before each frame, an instance whose
 * frame_no >= episode_frames (when nonzero) is restored to *snapshot.
 * obs (n*128, may be NULL) receives the final RAM.  Work is split over
 * nthreads pthreads (pinned to cores when pin != 0).  Returns total guest
 * instructions executed, or (uint64_t)-1 on error.
 */
uint64_t orc_run_batch(const uint8_t* rom, size_t rom_len, size_t n, int k,
                       fa_state* states, const uint8_t* actions,
                       const fa_state* snapshot, uint32_t episode_frames,
                       uint8_t* obs, int nthreads, int pin);

/* Same, recording every frame's RAM into ram_trace[(f*n + i)*128]. */
uint64_t orc_run_batch_trace(const uint8_t* rom, size_t rom_len, size_t n, int k,
                             fa_state* states, const uint8_t* actions,
                             const fa_state* snapshot, uint32_t episode_frames,
                             uint8_t* ram_trace, int nthreads);

/*
 * Known-answer runner on FlatMemory (src/cpu.rs:69-90): reset from
 * $FFFC/$FFFD of mem64k, then execute nsteps instructions, writing each
 * instruction's cycle count to cycles_out[i].  mem64k is updated in place.
 * Returns the number of steps run before an illegal opcode (== nsteps when
 * none).
 */
int orc_flat_run(uint8_t* mem64k, int nsteps, uint8_t* cycles_out, orc_regs* regs);

/* Same, starting from caller-provided registers instead of a reset. */
int orc_flat_run_from(uint8_t* mem64k, int nsteps, uint8_t* cycles_out, orc_regs* regs);

/* sizeof(fa_state) as compiled into the oracle (ABI check). */
size_t orc_state_size(void);

/* Test switch: 0 skips the headless bus's phantom reads and read-modify-
 * write's first write (their cycles still count), as a core without them
 * would; 1 (the default) issues them as the reference does. */
void orc_set_phantoms(int on);

/* Atari::render: RGBA (4 bytes per pixel) of `pixels` palette indices. */
void orc_rgba(const uint8_t* fb, size_t pixels, uint8_t* out);

/* ---- rendering console (src/tia.rs, src/atari.rs:107-306): one bus access per
 * CPU cycle, three TIA clocks and one PIA clock per access, 160 x 192 palette
 * index framebuffer. */
typedef struct orc_ratari orc_ratari;
orc_ratari*    orc_rcreate(const uint8_t* rom, size_t rom_len);   /* Atari::new */
orc_ratari*    orc_rclone(const orc_ratari* e);
void           orc_rdestroy(orc_ratari* e);
void           orc_rset_action(orc_ratari* e, unsigned action);
uint64_t       orc_rrun_frame(orc_ratari* e);
const uint8_t* orc_rframebuffer(const orc_ratari* e);
void           orc_rram(const orc_ratari* e, uint8_t* out128);
void           orc_rregs(const orc_ratari* e, uint32_t* out8);
unsigned       orc_rmapper(const orc_ratari* e);
size_t         orc_rtia_size(void);
void           orc_rtia_copy(const orc_ratari* e, void* out);
/* k frames on each of n rendering consoles (actions [k][n]), nthreads threads. */
uint64_t       orc_rrun_batch(orc_ratari** cs, size_t n, int k, const uint8_t* actions, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
