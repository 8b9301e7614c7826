/*
 * fast_atari.h — C ABI of the B200 batched Atari 2600 emulator core.
 *
 * This is the drop-in boundary for the reference's `BatchAtariGpu`
 * (src/cuda_env.rs:99-191 of RPP1011/fast-atari-rs).  Every entry point is
 * plain C: pointers, sizes and int status codes, no CUDA or torch types in the
 * signatures (streams are passed as `void*`, i.e. a `cudaStream_t`).
 *
 * Conventions
 *   - Return value 0 (FA_OK) on success, a negative FA_ERR_* code on failure;
 *     fa_last_error() returns a thread-local text for the last failure.
 *   - Host buffers are borrowed for the duration of the call and copied.
 *   - Every call on a handle is synchronous unless its name ends in `_async`
 *     (those enqueue on the given stream and return immediately).
 *   - A handle is used by one caller thread at a time (the reference's
 *     `&mut self` discipline).
 */
#ifndef FAST_ATARI_H
#define FAST_ATARI_H

#include <stddef.h>   /* size_t, offsetof */
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- errors */
#define FA_OK               0
#define FA_ERR_INVALID     -1   /* bad argument (null pointer, size mismatch, k < 1) */
#define FA_ERR_BAD_ROM     -2   /* ROM length the reference cannot construct */
#define FA_ERR_CUDA        -3   /* a CUDA runtime call failed */
#define FA_ERR_NO_DEVICE   -4   /* no CUDA device, or the kernels are missing */
#define FA_ERR_KERNEL      -5   /* a device-side bounded wait gave up (error word set) */
#define FA_ERR_CAPACITY    -6   /* request exceeds a configured capacity or budget */

/* ------------------------------------------------ per-instance run status */
/* Halting bits: the instance stops executing until reset or fa_set_states. */
#define FA_STATUS_ILLEGAL_OPCODE  0x1u   /* reference panics (src/cpu.rs:1139-1141) */
#define FA_STATUS_VSYNC_BUDGET    0x2u   /* VSYNC held for > FA_VSYNC_BUDGET cycles;
                                            the reference loops forever (src/atari.rs:588-590) */
#define FA_STATUS_NOT_RESET       0x4u   /* created but never reset; the reference
                                            panics when stepping such a state */
#define FA_STATUS_HALT_MASK       0x7u
/* Informational, sticky: a frame ended on the 100,000-cycle cap (src/atari.rs:594). */
#define FA_STATUS_CYCLE_CAP       0x100u

#define FA_FRAME_CYCLE_CAP   100000u
#define FA_VSYNC_BUDGET      2000000u

/* Bank-switching schemes (src/atari.rs:83-105). */
#define FA_SCHEME_FIXED 0
#define FA_SCHEME_F8    1
#define FA_SCHEME_F6    2
#define FA_SCHEME_F4    3
/* Schemes the reference does not have (its BankScheme::detect picks by size
 * alone, so these carts run as F8 there and crash or misbehave).  E0 and 3F
 * are never picked by size: register them per ROM with fa_rom_set_scheme. */
#define FA_SCHEME_E0    4   /* Parker Brothers, 8K: four 1K windows; any access to
                               $1FE0-$1FE7 / $1FE8-$1FEF / $1FF0-$1FF7 maps 1K slice
                               (addr & 7) into window 0 / 1 / 2; window 3 holds
                               slice 7.  Power-on windows: slices 4, 5, 6, 7. */
#define FA_SCHEME_3F    5   /* Tigervision, 2K multiples up to 32K: $1000-$17FF is a
                               switchable 2K bank, $1800-$1FFF the last 2K; a write
                               of v to $0000-$003F selects bank v mod (len / 2K) and
                               also reaches the TIA.  Power-on bank: 0. */
#define FA_SCHEME_DPC   6   /* Activision's DPC (Pitfall II): 8K of program in two 4K
                               banks ($1FF8 / $1FF9 select bank 0 / 1, any access;
                               power-on bank 1), 2K of display data read through 8
                               data fetchers, an 8-bit random number generator and 3
                               music channels.  Reads of $1000-$103F and writes of
                               $1040-$107F reach the DPC registers (fa_state's dpc_*
                               fields).  Unlike E0 and 3F, picked by size: 10240
                               bytes (program + display data) or 10495 (with the 255
                               bytes that dumps of the cart carry after them, ignored),
                               lengths the reference cannot construct. */
#define FA_SCHEME_FE    7   /* Activision FE, 8K: two 4K banks at $1000-$1FFF.  Every
                               bus access (phantom ones included) to $01FE arms the
                               cart; the next access then selects the bank by bit 5
                               of its data (set: bank 0, clear: bank 1), as JSR and
                               RTS with the stack at $01FE/$01FF do on these carts.
                               Power-on bank: 1.  Registered per ROM, like E0. */
#define FA_SCHEME_AUTO  (-1)

#define FA_RAM_BYTES 128
#define FA_NUM_ACTIONS 18

/*
 * Full per-instance state, array-of-structs, as returned by fa_get_states.
 * Bytes [0, 221) have exactly the layout of the reference's `AtariStateGpu`
 * (src/cuda_env.rs:10-38, repr(C)); the tail adds what the reference GPU state
 * lacks: the CPU cycle counter (`Cpu::cycles`, src/cpu.rs:104), a frame
 * counter and the run status word.
 */
typedef struct fa_state {
    uint8_t  a, x, y, sp;
    uint16_t pc;
    uint8_t  status;
    uint8_t  _pad0;
    uint8_t  ram[FA_RAM_BYTES];
    uint8_t  port_a_output, port_a_ddr, port_a_input;
    uint8_t  port_b_output, port_b_ddr, port_b_input;
    uint16_t timer_value, timer_prescaler, timer_prescaler_select;
    uint8_t  timer_underflow, _pad1, _pad2, _pad3;
    uint16_t tia_clock, tia_scanline;
    uint8_t  tia_wsync, tia_frame_complete, tia_vsync, tia_vblank;
    uint8_t  cxm0p, cxm1p, cxp0fb, cxp1fb, cxm0fb, cxm1fb, cxblpf, cxppmm;
    uint8_t  inpt4, inpt5, paddle0, paddle1;
    uint16_t paddle_counter;
    uint8_t  paddle_dumped, _pad4;
    uint16_t pos_p0, pos_p1, pos_m0, pos_m1, pos_bl;
    uint8_t  hmp0, hmp1, hmm0, hmm1, hmbl, _pad5;
    uint8_t  grp0, grp1, grp0_old, grp1_old;
    uint8_t  enam0, enam1, enabl, enabl_old;
    uint8_t  vdelp0, vdelp1, vdelbl;
    uint8_t  resmp0, resmp1, nusiz0, nusiz1;
    uint8_t  colup0, colup1, colupf, colubk;
    uint8_t  ctrlpf, refp0, refp1;
    uint8_t  pf0, pf1, pf2;
    uint8_t  bank, scheme;
    uint8_t  _pad_end[2];
    /* ---- extension beyond the reference layout ---- */
    /* E0, 3F, DPC and FE bank state, 16 bits little-endian: E0 = slice of
     * window 0 | window 1 << 4 | window 2 << 8; 3F = the 2K bank at $1000; DPC
     * = the 4K program bank; FE = the 4K bank | 0x100 while the last access
     * was to $01FE.  0 for the reference's schemes, whose bank is `bank`. */
    uint8_t  mapper[2];
    uint8_t  _pad_ext;
    uint64_t cycles;      /* Cpu::cycles: executed instruction cycles, never reset */
    uint32_t frame_no;    /* frames run since the last reset (episode counter) */
    uint32_t run_status;  /* FA_STATUS_* bits */
    /* DPC registers (FA_SCHEME_DPC; 0 for every other scheme, whose
     * fa_set_states does not take them).  Fetcher k has
     * an 11-bit counter, top and bottom registers and a flag (bit k of
     * dpc_flags: the flag reads $FF).  dpc_music bit m: fetcher 5 + m is a
     * music channel.  dpc_osc: the music oscillator's clock count when the
     * fetchers were last brought up to date (it counts 20,000 per second of
     * Cpu::cycles at 3,579,545 / 3 cycles per second). */
    uint16_t dpc_counter[8];
    uint8_t  dpc_top[8];
    uint8_t  dpc_bottom[8];
    uint8_t  dpc_flags, dpc_music, dpc_random, _pad_dpc;
    uint32_t dpc_osc;
} fa_state;

#define FA_STATE_REF_BYTES 221   /* prefix shared with the reference AtariStateGpu */
#define FA_STATE_BYTES     280

#ifdef __cplusplus
#define FA_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define FA_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
FA_STATIC_ASSERT(sizeof(fa_state) == FA_STATE_BYTES, "fa_state size");
FA_STATIC_ASSERT(offsetof(fa_state, ram) == 8, "ram offset");
FA_STATIC_ASSERT(offsetof(fa_state, timer_value) == 142, "timer offset");
FA_STATIC_ASSERT(offsetof(fa_state, tia_clock) == 152, "tia offset");
FA_STATIC_ASSERT(offsetof(fa_state, paddle_counter) == 172, "paddle offset");
FA_STATIC_ASSERT(offsetof(fa_state, pos_p0) == 176, "pos offset");
FA_STATIC_ASSERT(offsetof(fa_state, bank) == 217, "bank offset");
FA_STATIC_ASSERT(offsetof(fa_state, cycles) == 224, "cycles offset");
FA_STATIC_ASSERT(offsetof(fa_state, run_status) == 236, "status offset");
FA_STATIC_ASSERT(offsetof(fa_state, dpc_counter) == 240, "dpc offset");
FA_STATIC_ASSERT(offsetof(fa_state, dpc_osc) == 276, "dpc oscillator offset");

/* Opaque handle: one ROM, n instances, resident in HBM (`BatchAtariGpu`). */
typedef struct fa_handle fa_handle;

/* Text of the last error on this thread ("" if none). */
const char* fa_last_error(void);

/* Library version string. */
const char* fa_version(void);

/* Number of CUDA devices visible (0 when none); never fails. */
int fa_device_count(void);

/* Make `device` current on the calling thread for handles and pools created
 * afterwards (the library links its own CUDA runtime, so another runtime's
 * current device does not carry over). */
int fa_set_device(int device);

/* Bound, in nanoseconds, of the device-side wait for the ROM images that a
 * launch stages into shared memory (2,000,000,000 = 2 s by default;
 * 0..10,000,000,000 accepted, process-wide, for launches enqueued after the
 * call).  A wait that gives up leaves every instance of its CTA untouched,
 * sets bit 0x1 of the launch's device error word, and the call returns
 * FA_ERR_KERNEL (fa_last_error names the word).  0 gives up at once, which lets a test exercise that
 * path without a fault.  No counterpart in the reference, which has no
 * device-side waits. */
int fa_set_wait_limit_ns(uint64_t ns);
uint64_t fa_wait_limit_ns_get(void);

/*
 * ROM schemes.  No counterpart in the reference, which picks a scheme from
 * the ROM length alone (src/atari.rs:96-105).  fa_rom_set_scheme records,
 * process-wide, the scheme of one ROM image (identified by its bytes); every
 * entry point that is later given the same bytes (fa_create, fa_pool_add_cart,
 * fa_server_create, fa_render_create, fa_autotune) uses it instead of the
 * size rule.  FA_SCHEME_AUTO removes the record.  The length must suit the
 * scheme: E0 and FE exactly 8192; 3F a multiple of 2048 up to 32768; DPC
 * 10240 or 10495; the reference's
 * schemes the lengths fa_create accepts for them.  FA_ERR_BAD_ROM otherwise.
 */
int fa_rom_set_scheme(const uint8_t* rom, size_t rom_len, int scheme);

/* The scheme the entry points will use for these bytes (a registered one,
 * else DPC for 10240 or 10495 bytes, else the size rule), or FA_ERR_BAD_ROM
 * for a length that cannot be built. */
int fa_rom_scheme(const uint8_t* rom, size_t rom_len);

/* A guess from the ROM's code, for a caller deciding what to register; never
 * applied by itself.  It counts absolute and indexed loads and stores aimed at
 * the E0 hotspots $1FE0-$1FF7, zero-page stores to $3F (STA/STX/STY $3F), and
 * accesses to the hotspots of the scheme the size rule gives (F8 $1FF8-$1FF9,
 * F6 $1FF6-$1FF9, F4 $1FF4-$1FFB).  An 8K image with at least three E0
 * accesses, over eight times the size-rule ones, and a reset vector in
 * $1C00-$1FFF is E0; at least three $3F stores, over eight times the size-rule
 * accesses, and a reset vector in $1800-$1FFF make a 2K-multiple image 3F;
 * an 8K image with no access to the F8 hotspots, at least six JSRs into
 * $Dxxx and six into $Fxxx (FE carts call across their banks that way) and
 * a reset vector in one of those ranges is FE; a DPC length is DPC; anything
 * else gets the size rule.  On random bytes it picks E0, 3F or FE for a few
 * percent of 8K images. */
int fa_rom_guess_scheme(const uint8_t* rom, size_t rom_len);

/*
 * BatchAtariGpu::new (src/cuda_env.rs:112-126).  Uploads the ROM and allocates
 * SoA state for n instances on the current device.  The ROM length must be one
 * the reference can construct: 1..4096 (Fixed, mirrored into the 4K window),
 * 8192 (F8), 16384 (F6) or >= 32768 (F4, first 32 KiB used); or, for bytes
 * registered with fa_rom_set_scheme, one the registered scheme holds.
 * Instances start zeroed, as in the reference; call fa_reset before stepping.
 */
int fa_create(const uint8_t* rom, size_t rom_len, size_t n, fa_handle** out);

/* Drop (frees every device buffer of the handle). NULL is ignored. */
void fa_destroy(fa_handle* h);

/* BatchAtariGpu::num_envs (src/cuda_env.rs:190). */
size_t fa_num_envs(const fa_handle* h);

/*
 * BatchAtariGpu::set_sorted (src/cuda_env.rs:129).  sorted != 0 groups the
 * lanes of a warp by program counter with __match_any_sync and runs every
 * group once per round (FA_SCHED_MATCH); 0 runs every lane's own instruction
 * stream (FA_SCHED_LANE).  A new handle starts with FA_SCHED_PC, the
 * convergence policy (see fa_set_launch); results never depend on the policy.
 */
int fa_set_sorted(fa_handle* h, int sorted);

/*
 * BatchAtariGpu::reset (src/cuda_env.rs:131-142): every instance becomes
 * HeadlessAtari::new(rom) followed by one run_frame().  Computed on the device
 * once and broadcast.  obs_out (n*128 bytes, may be NULL) receives the RAM.
 */
int fa_reset(fa_handle* h, uint8_t* obs_out);

/*
 * BatchAtariGpu::step (src/cuda_env.rs:144-161): apply actions[i] (0..17, other
 * values act as NOOP like Action::from_index) to instance i and run one frame.
 * obs_out (n*128 bytes, may be NULL) receives each instance's RAM.
 */
int fa_step(fa_handle* h, const uint8_t* actions, uint8_t* obs_out);

/*
 * BatchAtariGpu::step_multi (src/cuda_env.rs:166-184): k frames in one launch,
 * actions frame-major (actions[f*n + i]); obs_out gets the last frame's RAM.
 */
int fa_step_multi(fa_handle* h, const uint8_t* actions, int k, uint8_t* obs_out);

/*
 * Device-pointer variant of step_multi, enqueued on `stream` (a cudaStream_t,
 * NULL = the handle's own stream).  d_actions holds k*n bytes and d_obs n*128
 * bytes of device memory (d_obs may be NULL).  Returns without synchronising.
 */
int fa_step_multi_async(fa_handle* h, const uint8_t* d_actions, int k,
                        uint8_t* d_obs, void* stream);

/* Wait for all work enqueued on the handle's stream; reports kernel errors. */
int fa_synchronize(fa_handle* h);

/* BatchAtariGpu::download_states (src/cuda_env.rs:186-188), extended layout. */
int fa_get_states(fa_handle* h, fa_state* out);

/* Upload full states for all n instances (checkpoint restore). */
int fa_set_states(fa_handle* h, const fa_state* in);

/* Copy instance idx's 128-byte RAM (HeadlessAtari::ram, src/atari.rs:617). */
int fa_get_ram(fa_handle* h, size_t idx, uint8_t* out128);

/* Copy every instance's run-status word (n entries). */
int fa_get_status(fa_handle* h, uint32_t* out);

/*
 * Periodic episode reset: before each frame, an instance whose frame_no has
 * reached episode_frames is restored to the post-reset snapshot (frame_no 0).
 * 0 disables it.  Phase offsets are set through fa_set_frame_numbers.
 */
int fa_set_episode_frames(fa_handle* h, uint32_t episode_frames);

/* Overwrite every instance's frame_no (n entries). */
int fa_set_frame_numbers(fa_handle* h, const uint32_t* frame_no);

/* Lane scheduling policies inside a warp (fa_set_launch `sched`). */
#define FA_SCHED_LANE  0   /* each lane runs its own instruction stream */
#define FA_SCHED_PC    1   /* lanes at the (bank, pc) of the lane furthest behind run together;
                              "behind" by (frame, bank-switch hotspot accesses this frame, pc) */
#define FA_SCHED_LINE  2   /* as FA_SCHED_PC, behind by (frame, scanline, pc) */
#define FA_SCHED_MATCH 3   /* __match_any_sync groups by pc, every group each round */

/*
 * Launch shape of the handle (no reference counterpart; the reference uses a
 * fixed 128-thread block, src/cuda_env.rs:147).  block in {64,128,256,512};
 * persistent != 0 sizes the grid to the SMs and feeds CTAs from a device work
 * queue instead of one CTA per 'block' instances.
 */
int fa_set_launch(fa_handle* h, int block, int sched, int persistent);
int fa_get_launch(const fa_handle* h, int* block, int* sched, int* persistent);

/* Persistent form only: warps per CTA (0 = as many as shared memory fits;
 * else 2, 4, 8, 16, 24, 28 or 32).  Fewer warps raise the register budget per
 * thread (65536 / (32 x warps)). */
int fa_set_cta_warps(fa_handle* h, int warps);

/* Guest (6502) instructions executed by the handle's last synchronous call. */
unsigned long long fa_last_instructions(const fa_handle* h);

/* Lane slots the warp scheduler offered in that call (scheduler rounds x 32);
 * instructions / lane slots is the SIMT lane efficiency of the emulation. */
unsigned long long fa_last_lane_slots(const fa_handle* h);

/* The post-reset snapshot every instance starts from (after fa_reset). */
int fa_get_snapshot(fa_handle* h, fa_state* out);

/* Device pointer to the SoA state rows (FA layout, for zero-copy readers);
 * *stride_words receives the row stride in 32-bit words. */
void* fa_device_state(fa_handle* h, uint32_t* stride_words);

/* ------------------------------------------------------------------ pools
 * The batched form (no reference counterpart: the reference steps one ROM per
 * BatchAtariGpu).  A pool holds up to 16 carts, each with its own instance
 * set, and steps all of them in ONE launch whose persistent CTAs pull work
 * units (up to `block` instances of one cart) from a device queue, heaviest
 * cart first.  Actions and observations are passed per cart: actions[g] is
 * k * n_g bytes frame-major, obs[g] is n_g * 128 bytes (or NULL).
 */
typedef struct fa_pool fa_pool;
typedef struct fa_graph fa_graph;

int  fa_pool_create(fa_pool** out);
void fa_pool_destroy(fa_pool* p);
/* Add a cart with n instances, reset on the device; *group gets its index. */
int  fa_pool_add_cart(fa_pool* p, const uint8_t* rom, size_t rom_len, size_t n, int* group);
int  fa_pool_num_groups(const fa_pool* p);
/* The handle owning group g's instances (get/set states, status, episode
 * settings apply to it); owned by the pool. */
fa_handle* fa_pool_group(fa_pool* p, int group);
/* Per-cart warp policy and relative cost of one of its units (queue order). */
int  fa_pool_set_group(fa_pool* p, int group, int sched, float weight);
int  fa_pool_set_launch(fa_pool* p, int block, int persistent);
int  fa_pool_set_cta_warps(fa_pool* p, int warps);
/* Synchronous steps from host buffers: batched (one launch for all carts)
 * and plain (one launch per frame per cart, the reference's form). */
int  fa_pool_step(fa_pool* p, const uint8_t* const* actions, int k, uint8_t* const* obs);
int  fa_pool_step_plain(fa_pool* p, const uint8_t* const* actions, int k, uint8_t* const* obs);
/* Same from device buffers, enqueued on `stream` (NULL: the pool's stream). */
int  fa_pool_step_async(fa_pool* p, const uint8_t* const* d_actions, int k, uint8_t* const* d_obs,
                        void* stream);
int  fa_pool_step_plain_async(fa_pool* p, const uint8_t* const* d_actions, int k,
                              uint8_t* const* d_obs, void* stream);
int  fa_pool_synchronize(fa_pool* p);
/* Zero the instruction / lane-slot counters (read after a synchronize). */
int  fa_pool_reset_counters(fa_pool* p);
/* Diagnostics (no counterpart in the reference): with a device buffer of
 * cap x 3 unsigned 64-bit words set, every batched launch of the pool
 * records, for each work unit (32 instances of one cart, in launch order:
 * carts by decreasing queue weight), its start and end in device
 * nanoseconds (%globaltimer) and smid << 32 | warp << 16 | group.  NULL
 * (with cap 0) stops the records. */
int  fa_pool_set_trace(fa_pool* p, unsigned long long* d_trace, uint32_t cap);
/* Placement of the persistent launch's first wave (off by default; no
 * counterpart in the reference): with one CTA per SM, 1 spreads the work
 * units over the SMs' four warp schedulers so that each scheduler's summed
 * cost (the cart's weight from fa_pool_set_group, per instance-frame) is as
 * even as longest-processing-time-first makes it; 0 places unit
 * warp * grid + cta as the queue order gives them.  Results do not depend
 * on it. */
int  fa_pool_set_balance(fa_pool* p, int on);
unsigned long long fa_pool_last_instructions(const fa_pool* p);
unsigned long long fa_pool_last_lane_slots(const fa_pool* p);
/* The pool's own stream (a cudaStream_t). */
void* fa_pool_stream(fa_pool* p);
/*
 * Capture `calls` consecutive batched steps of k frames into a CUDA graph.
 * d_actions[g] holds calls * k * n_g bytes (call c uses the slice starting at
 * c * k * n_g); d_obs[g] (or NULL) receives each call's RAM.  The graph
 * replays against the pool's current state.
 */
int  fa_pool_graph_create(fa_pool* p, const uint8_t* const* d_actions, int k, int calls,
                          uint8_t* const* d_obs, fa_graph** out);
int  fa_graph_launch(fa_graph* g, void* stream);
void fa_graph_destroy(fa_graph* g);

/* Observation bytes -> f32 in [0, 1] (b / 255, IEEE single division), on the
 * device: BatchAtariGpuEnv's RAM observation (src/rl4burn_env.rs:320-322)
 * written into a caller buffer of `count` floats, enqueued on `stream`. */
int fa_obs_to_unit_f32(const uint8_t* d_obs, float* d_out, size_t count, void* stream);

/*
 * Reward and termination from RAM.  No counterpart in the reference, which
 * returns reward 0 and never terminates (src/atari.rs:348,
 * src/rl4burn_env.rs:123); where a game keeps its score and lives is per-game
 * knowledge the caller supplies.  Offsets are RAM offsets 0..127 ($80 + offset).
 */
typedef struct fa_reward_spec {
    uint8_t score_addr[4];   /* score bytes, most significant first */
    uint8_t score_bytes;     /* 0..4 (0: no score, reward 0) */
    uint8_t score_bcd;       /* 1: two decimal digits per byte (high nibble first); 0: binary */
    uint8_t lives_addr;      /* lives = (ram[lives_addr] & lives_mask) >> lives_shift */
    uint8_t lives_mask;      /* 0: no lives counter */
    uint8_t lives_shift;
    uint8_t terminal_addr;   /* terminal when (ram[terminal_addr] & terminal_mask) == terminal_value */
    uint8_t terminal_mask;   /* 0: no terminal test */
    uint8_t terminal_value;
} fa_reward_spec;

#define FA_EPISODE_TERMINAL  0x1u   /* the terminal test holds */
#define FA_EPISODE_LIFE_LOST 0x2u   /* the lives counter went down */

/*
 * For n observation rows (128 bytes each, as fa_step writes them) on the
 * device: reward[i] = score - d_score[i] as float, flags[i] = FA_EPISODE_*,
 * then d_score[i] = score and d_lives[i] = lives.  With init != 0 only the
 * scores and lives are recorded (reward 0, no life lost), as after a reset.
 * d_score / d_lives persist between calls (n int32 each, caller-owned);
 * d_reward (n floats) and d_flags (n bytes) may be null.  Enqueued on stream.
 */
int fa_obs_reward(const uint8_t* d_obs, size_t n, const fa_reward_spec* spec, int init, int32_t* d_score,
                  int32_t* d_lives, float* d_reward, uint8_t* d_flags, void* stream);

/* ---------------------------------------------------------------- autotuning
 * Project-written tuner (no reference counterpart; the reference hard-codes
 * 128-thread blocks and a manual set_sorted).  For one ROM and n instances it
 * times, on the current device, the warp policy, then the launch shape
 * (persistent CTAs of 8..32 warps = register caps of 256..64 per thread, or
 * the plain form with 64..512-thread CTAs), then the frames per launch K, and
 * returns the fastest record.  All configurations give identical results.
 */
typedef struct fa_tuning {
    int   block;                  /* CTA size of the plain form */
    int   persistent;             /* 1: persistent form */
    int   cta_warps;              /* persistent form: warps per CTA (0 = auto) */
    int   sched;                  /* FA_SCHED_* */
    int   k;                      /* frames per launch */
    float frames_per_s;           /* measured */
    float ns_per_instance_frame;  /* measured cost; a pool's queue weight */
} fa_tuning;

int fa_autotune(const uint8_t* rom, size_t rom_len, size_t n, fa_tuning* best,
                fa_tuning* table, int table_cap, int* table_len);

/* ------------------------------------------------------------------ serving
 * Continuous-batching server (no reference counterpart: BatchAtariGpu,
 * src/cuda_env.rs:99-191, serves one caller with one synchronous step per
 * call).  A server holds up to 16 carts and any number of sessions; a session
 * is one client's instance set of one cart, resident in HBM between requests.
 * A step request names a session, a batch size n, a frame count k and k*n
 * actions (frame-major), and steps instances [0, n) of the session k frames;
 * if n exceeds the instances the session holds, the new ones are admitted
 * first, each starting from the cart's post-reset snapshot (BatchAtariGpu::
 * reset, src/cuda_env.rs:131-142).  Admission is charged against a budget of
 * state bytes (whole 256-instance blocks of 68,608 bytes); when the budget is
 * spent, admissions wait in FIFO order until a session is closed.  A
 * session's requests run one at a time in submission order; requests of
 * different sessions are batched into shared launches whenever they are
 * ready, with up to max_inflight batches on the GPU at once.  Every result is
 * identical to stepping the same session alone.  All calls are thread-safe.
 */
#define FA_ERR_TIMEOUT     -7   /* fa_server_wait: the request was not done in time */

#define FA_SERVE_BATCHED 0   /* continuous batching (fa_serve launches, batches overlap) */
#define FA_SERVE_PLAIN   1   /* FIFO of static batches, one on the GPU at a time, one
                                launch per frame per cart (the reference's per-frame form) */

typedef struct fa_server fa_server;

typedef struct fa_server_config {
    size_t state_budget_bytes;   /* resident state admitted at most (0 = 64 GiB) */
    int    mode;                 /* FA_SERVE_BATCHED or FA_SERVE_PLAIN */
    int    block;                /* CTA size, 128, 256 or 512 (0 = 512 batched, 128 plain) */
    int    max_inflight;         /* batches on the GPU at once, 1..64 (0 = 32; plain: 1) */
    int    sched;                /* FA_SCHED_* warp policy (a NULL config: FA_SCHED_PC) */
} fa_server_config;

typedef struct fa_request_info {
    int    status;               /* FA_OK or an FA_ERR_* code */
    int    waited_admission;     /* 1 if its admission waited for budget */
    unsigned batch_requests;     /* requests in the launch batch it ran in */
    double latency_ms;           /* submit -> observations in the caller's buffer */
    double queue_ms;             /* submit -> dispatch to the GPU */
    double session_wait_ms;      /* of queue_ms: waiting for the same session's earlier
                                    requests (an actor steps after it sees its observations) */
    double service_ms;           /* dispatch -> done: the GPU work of its batch and the
                                    completion signal */
} fa_request_info;

typedef struct fa_server_stats {
    unsigned long long requests_submitted, requests_done, requests_failed;
    unsigned long long instance_frames;       /* sum of n * k over completed requests */
    unsigned long long dispatches;            /* batches sent to the GPU */
    unsigned long long dispatched_requests;
    unsigned long long launches;              /* kernel launches */
    unsigned long long admission_waits;       /* requests whose admission waited */
    unsigned long long guest_instructions;    /* 6502 instructions executed */
    unsigned long long lane_slots;            /* warp lane slots offered */
    long long sessions_open;
    size_t state_bytes_in_use, state_bytes_peak, state_budget_bytes;
} fa_server_stats;

/* Create a server on the current device for ncarts ROMs (each checked and
 * reset as by fa_create + fa_reset); cfg may be NULL (defaults).  Starts the
 * engine thread. */
int  fa_server_create(const uint8_t* const* roms, const size_t* rom_lens, int ncarts,
                      const fa_server_config* cfg, fa_server** out);
/* Stop the engine after the work on the GPU finishes (requests still waiting
 * for admission fail with FA_ERR_CAPACITY) and free everything. */
void fa_server_destroy(fa_server* s);
/* Open an empty session of cart `cart` (instances are admitted by requests). */
int  fa_server_open(fa_server* s, int cart, int64_t* session);
/* Close a session: its queued requests still run, then its state is freed. */
int  fa_server_close(fa_server* s, int64_t session);
/* Queue a step request; actions (k*n bytes) are copied, obs (n*128 bytes, or
 * NULL) is written before the request completes and must stay valid until
 * fa_server_wait returns for the ticket.  n larger than the whole budget
 * fails with FA_ERR_CAPACITY. */
int  fa_server_submit(fa_server* s, int64_t session, const uint8_t* actions, uint32_t n, int k,
                      uint8_t* obs, uint64_t* ticket);
/* Wait for a ticket (timeout_ms < 0: no limit; FA_ERR_TIMEOUT on expiry, the
 * ticket stays valid).  Each ticket is waited for until it completes, once. */
int  fa_server_wait(fa_server* s, uint64_t ticket, int timeout_ms, fa_request_info* info);
/* Submit and wait. */
int  fa_server_step(fa_server* s, int64_t session, const uint8_t* actions, uint32_t n, int k,
                    uint8_t* obs, fa_request_info* info);
/* Instances the session holds (the largest n of its requests so far). */
int  fa_server_session_size(fa_server* s, int64_t session, uint32_t* size);
/* Full states of instances [first, first+count) of a session, after its
 * queued requests complete (fa_state layout, as fa_get_states). */
int  fa_server_get_states(fa_server* s, int64_t session, uint32_t first, uint32_t count, fa_state* out);
int  fa_server_stats_get(fa_server* s, fa_server_stats* out);

/* Simulated actor clients.  `requests` step requests arrive as a Poisson
 * process at `offered_frames_per_s` instance-frames per second (0: all at
 * once, the saturation throughput); each picks one of `clients` clients and
 * one of the server's carts uniformly, a batch size lognormal(batch_median,
 * batch_sigma) clipped to [batch_min, batch_max] and k uniform in
 * [k_min, k_max], with actions uniform over the 18 joystick actions.  The
 * trace depends only on the configuration (seed included), not on timing.
 * Every (client, cart) is a session opened for the run and closed after it.
 * records (NULL or `requests` entries, in arrival order) receives each
 * request's shape and the parts of its latency. */
typedef struct fa_loadgen_config {
    int      clients;
    int      requests;
    double   offered_frames_per_s;
    uint64_t seed;
    uint32_t batch_median, batch_min, batch_max;
    double   batch_sigma;
    int      k_min, k_max;
} fa_loadgen_config;

typedef struct fa_loadgen_result {
    unsigned long long requests, admission_waits;
    double instances;              /* sum of n over the requests */
    double instance_frames;        /* sum of n * k */
    double elapsed_s;              /* first arrival -> last completion */
    double frames_per_s;           /* instance_frames / elapsed_s */
    double steady_frames_per_s;    /* completion rate between the 10th and 60th
                                      percentile of completion times */
    double offered_frames_per_s;
    double arrival_window_s;       /* last arrival time */
    double p50_ms, p90_ms, p99_ms, max_ms, mean_ms;
    double mean_queue_ms;          /* submit -> dispatch */
    double mean_batch_requests;    /* requests per launch batch, averaged over requests */
    int    errors;
} fa_loadgen_result;

typedef struct fa_loadgen_record {
    uint32_t cart, n, k, batch_requests;
    double   arrival_s;            /* submit time from the run's start */
    double   latency_ms;           /* = session_wait_ms + dispatch_ms + service_ms */
    double   session_wait_ms;      /* the same session's earlier requests still running */
    double   dispatch_ms;          /* ready -> dispatched: launch slots and state admission */
    double   service_ms;           /* dispatched -> done */
} fa_loadgen_record;

int fa_server_loadgen(fa_server* s, const fa_loadgen_config* cfg, fa_loadgen_result* out,
                      fa_loadgen_record* records);

/* ------------------------------------------------------------ rendering
 * The reference's rendering console (Atari, src/atari.rs:107-306, with the
 * pixel-accurate Tia of src/tia.rs): every CPU bus access ticks the TIA three
 * times and the PIA once, writes land on the third TIA clock of their cycle,
 * and each TIA clock inside the visible window renders one pixel of a
 * 160 x 192 framebuffer of NTSC palette indices (Atari::framebuffer).  One
 * console per GPU thread, as the headless core; framebuffers stay on the
 * device between calls (FA_FB_BYTES = 30,720 bytes per console).  The
 * reference renders one console per call on the CPU; the batched form and
 * this API have no counterpart there.
 */
#define FA_FB_WIDTH  160
#define FA_FB_HEIGHT 192
typedef struct fa_render fa_render;
/* n rendering consoles of one ROM on the current device (lengths as fa_create;
 * DPC and FE carts, FA_ERR_BAD_ROM: they run on the headless console only). */
int  fa_render_create(const uint8_t* rom, size_t rom_len, size_t n, fa_render** out);
void fa_render_destroy(fa_render* r);
size_t fa_render_num_envs(const fa_render* r);
/* CTA size in warps (4, 8 or 16; 16 by default) and warp policy (FA_SCHED_*). */
int  fa_render_set_launch(fa_render* r, int cta_warps, int sched);
/* Every console becomes Atari::new(rom) followed by one run_frame() without
 * an action.  fb_out (n * 160 * 192 bytes) and ram_out (n * 128) may be NULL. */
int  fa_render_reset(fa_render* r, uint8_t* fb_out, uint8_t* ram_out);
/* k frames per console (actions frame-major, k * n bytes, set_action before
 * each frame); fb_out receives the framebuffers after the last frame,
 * ram_out the RAM (either may be NULL). */
int  fa_render_step_multi(fa_render* r, const uint8_t* actions, int k, uint8_t* fb_out, uint8_t* ram_out);
/* Device-buffer variant on `stream` (NULL: the handle's stream); d_obs
 * (n * 128, 16-byte aligned, or NULL) receives the RAM. */
int  fa_render_step_multi_async(fa_render* r, const uint8_t* d_actions, int k, uint8_t* d_obs, void* stream);
int  fa_render_synchronize(fa_render* r);
/* The device framebuffers (n * FA_FB_WIDTH * FA_FB_HEIGHT bytes, console-major). */
uint8_t* fa_render_device_framebuffers(fa_render* r);
int  fa_render_get_framebuffers(fa_render* r, uint8_t* out);
/* CPU, RAM, PIA and TIA register state (fa_state layout; cycles, frame_no, run_status). */
int  fa_render_get_states(fa_render* r, fa_state* out);
unsigned long long fa_render_last_instructions(const fa_render* r);
/* Atari::render (src/atari.rs:356-369): consoles [first, first + count) as
 * RGBA, 160 x 192 x 4 bytes each (R, G, B from ntsc_palette,
 * src/atari.rs:624-645, then 255), converted on the device.  The _async form
 * writes into a device buffer (16-byte aligned) on `stream` (NULL: the
 * handle's); fa_render_get_rgba converts a chunk at a time on the device and
 * copies each into the host buffer. */
int  fa_render_rgba_async(fa_render* r, size_t first, size_t count, uint8_t* d_rgba, void* stream);
int  fa_render_get_rgba(fa_render* r, size_t first, size_t count, uint8_t* rgba_out);
/* ntsc_palette (src/atari.rs:624-645) of one palette index, packed as
 * R | G << 8 | B << 16 | 255 << 24. */
uint32_t fa_palette_rgba(uint8_t index);

/* -------------------------------------------------- no-allocation stepping
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (device memory owned by another allocator, or a stepping loop that must not
 * trigger cudaMalloc's implicit device synchronisation): runs `calls`
 * consecutive batched steps of k frames over caller-owned buffers and
 * allocates nothing.
 *   d_rom_image  nbanks * 4096 bytes, 16-byte aligned (Fixed carts as their
 *                mirrored 4 KiB window, banked carts as-is)
 *   scheme       FA_SCHEME_FIXED, _F8, _F6 or _F4 (E0, 3F, DPC and FE are not taken here)
 *   d_state      the FA SoA state rows (fa_device_state layout), stride >= n,
 *                of instances created for the same scheme (rows of another
 *                scheme keep bank numbers this one does not have, and step
 *                wrongly)
 *   d_actions    calls * k * n bytes; call c uses the slice at c * k * n
 *   d_obs        n * 128 bytes (16-byte aligned) or NULL; gets each call's RAM
 * The kernel's scratch (one work-queue counter per call, error word,
 * counters) is a fixed array compiled into the library, present on every GPU
 * that loads it: calls is limited to 1..1024 (FA_ERR_CAPACITY beyond).  The
 * first call on a device looks up that array's device address, so make it
 * before any stream capture.  Every call shares the array: calls that overlap
 * on the GPU (other streams, other threads) race and must not be issued.
 * No periodic episode reset is applied here (a handle's
 * fa_set_episode_frames does not carry over to its rows).  Each call waits
 * on the host until its steps on `stream` finish (it synchronises that
 * stream only) and reports device-side errors.
 */
int fa_step_static(const uint8_t* d_rom_image, int scheme, uint32_t* d_state, uint32_t stride,
                   uint32_t n, const uint8_t* d_actions, int k, int calls, uint8_t* d_obs,
                   int sched, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FAST_ATARI_H */
