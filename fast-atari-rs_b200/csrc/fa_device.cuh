// fa_device.cuh — the per-thread Atari 2600 emulator for sm_100a.
//
// One thread emulates one console.  Its hot state lives in registers; its
// 128-byte PIA RAM and the TIA registers that change only on a write live in
// shared memory, interleaved by thread in 32-bit words (byte o of thread t is
// at word (o/4)*BLOCK + t), so lanes touching any offsets hit bank t%32 and
// never conflict.  ROM banks sit in shared memory, staged once per block.
//
// Semantics are those of the reference CPU emulator (RPP1011/fast-atari-rs):
//   src/cpu.rs            6502 step, including every phantom access whose
//                         side effect is visible on the Atari bus
//   src/atari.rs:460-552  HeadlessBus read/write decode and bank hotspots
//   src/atari.rs:584-614  run_frame / run_one_cycle
//   src/headless_tia.rs   HeadlessTia
//   src/pia.rs            Pia
// The instruction decoder is organised by the 6502 opcode bit fields
// (aaa bbb cc) instead of one 151-way switch: lanes executing different
// opcodes that share an addressing mode or an ALU operation share code.
#pragma once
#include <stdint.h>

#include "fa_internal.h"
#include "fa_layout.h"

namespace fa {

enum : uint32_t { F_C = 1, F_Z = 2, F_I = 4, F_D = 8, F_B = 16, F_U = 32, F_V = 64, F_N = 128 };

// Action -> (SWCHA | INPT4<<8 | paddle0<<16), src/atari.rs:34-81,571-582.
constexpr uint32_t act_word(int up, int down, int left, int right, int fire)
{
    return (0xFFu & ~(up ? 0x10u : 0u) & ~(down ? 0x20u : 0u) & ~(left ? 0x40u : 0u) & ~(right ? 0x80u : 0u))
         | ((fire ? 0u : 1u) << 8) | ((left ? 200u : right ? 50u : 128u) << 16);
}

// Action::decode order (src/atari.rs:59-80): up, down, left, right, fire.
static __constant__ uint32_t c_action_table[18] = {
    act_word(0, 0, 0, 0, 0), act_word(0, 0, 0, 0, 1), act_word(1, 0, 0, 0, 0), act_word(0, 0, 0, 1, 0),
    act_word(0, 0, 1, 0, 0), act_word(0, 1, 0, 0, 0), act_word(1, 0, 0, 1, 0), act_word(1, 0, 1, 0, 0),
    act_word(0, 1, 0, 1, 0), act_word(0, 1, 1, 0, 0), act_word(1, 0, 0, 0, 1), act_word(0, 0, 0, 1, 1),
    act_word(0, 0, 1, 0, 1), act_word(0, 1, 0, 0, 1), act_word(1, 0, 0, 1, 1), act_word(1, 0, 1, 0, 1),
    act_word(0, 1, 0, 1, 1), act_word(0, 1, 1, 0, 1),
};

// Bit op of word op>>5 is set for the 151 legal opcodes (src/cpu.rs:253-1141).
static __constant__ uint32_t c_legal[8] = {
    0x63636763u, 0x63637773u, 0x63637763u, 0x63637763u,
    0x27737572u, 0x77737777u, 0x63637773u, 0x63637773u,
};

// Packed TIA flag word (Emu::tw).
enum : uint32_t { TW_WSYNC = 1u << 16, TW_FCOMP = 1u << 17, TW_PDUMP = 1u << 18 };

template <int BLOCK>
__device__ __forceinline__ uint32_t priv_off(uint32_t o) { return (o & ~3u) * BLOCK + (o & 3u); }

__device__ __forceinline__ uint32_t mod160(int v)
{
    int r = v % 160;
    return (uint32_t)(r < 0 ? r + 160 : r);
}

// Byte o (>= 128) of an instance's private bytes, in its HBM state rows:
// `col` is the instance's column base, stride4 the row stride in bytes.
__device__ __forceinline__ uint32_t cold_off(uint32_t o, uint32_t stride4) { return (o >> 2) * stride4 + (o & 3u); }

// TIA or PIA register read (HeadlessTia::read, src/headless_tia.rs:205-223;
// Pia::read I/O half, src/pia.rs:169-199).  Bit 8 of the result asks the
// caller to clear the timer underflow flag (an INTIM read).
static __device__ __noinline__ uint32_t io_read(uint32_t a, uint32_t pcnt, uint32_t pins, uint32_t pads,
                                         uint32_t ports, uint32_t timer, const uint8_t* col, uint32_t stride4)
{
    if (a & 0x80u) {                                                 // PIA: (a & 0x280) == 0x280
        switch (a & 7u) {
        case 0: return ((pins & ~(ports >> 8)) | (ports & (ports >> 8))) & 0xFFu;
        case 1: return (ports >> 8) & 0xFFu;
        case 2: return (((pins >> 8) & ~(ports >> 24)) | ((ports >> 16) & (ports >> 24))) & 0xFFu;
        case 3: return ports >> 24;
        case 4: return (timer & 0xFFu) | 0x100u;
        case 5: return (timer >> 16) ? 0x80u : 0u;
        default: return 0u;
        }
    }
    const uint32_t r = a & 0x0Fu;
    if (r < 8u) return col[cold_off(PB_CX + r, stride4)];
    switch (r) {
    case 0x8: return pcnt >= (pads & 0xFFu) ? 0x80u : 0u;
    case 0x9: return pcnt >= (pads >> 8) ? 0x80u : 0u;
    case 0xA: case 0xB: return 0x80u;
    case 0xC: return (pins >> 16) & 1u ? 0x80u : 0u;
    case 0xD: return (pins >> 17) & 1u ? 0x80u : 0u;
    default: return 0u;
    }
}

// HeadlessTia::write (src/headless_tia.rs:225-298).  tw is the packed flag
// word, lw = scanline | paddle_counter<<16; both come back updated.  The
// write-only registers live in the instance's HBM rows (col, stride4).
static __device__ __noinline__ uint2 tia_write_io(uint32_t a, uint32_t v, uint32_t clock, uint32_t tw, uint32_t lw,
                                           uint8_t* col, uint32_t stride4)
{
    auto stp = [&](uint32_t o, uint32_t val) { col[cold_off(o, stride4)] = (uint8_t)val; };
    auto ldp = [&](uint32_t o) -> uint32_t { return col[cold_off(o, stride4)]; };
    auto stp16 = [&](uint32_t o, uint32_t val) { *(uint16_t*)(col + cold_off(o, stride4)) = (uint16_t)val; };
    auto ldp16 = [&](uint32_t o) -> uint32_t { return *(const uint16_t*)(col + cold_off(o, stride4)); };
    const uint32_t r = a & 0x3Fu;
    switch (r) {
    case 0x00:                                                        // VSYNC rising edge starts a frame
        if (!(tw & 2u) && (v & 2u)) { lw &= 0xFFFF0000u; tw |= TW_FCOMP; }
        tw = (tw & ~0xFFu) | v;
        break;
    case 0x01:                                                        // VBLANK bit 7 dumps the paddles
        if (v & 0x80u) { lw &= 0xFFFFu; tw |= TW_PDUMP; } else tw &= ~TW_PDUMP;
        tw = (tw & ~0xFF00u) | (v << 8);
        break;
    case 0x02: tw |= TW_WSYNC; break;
    case 0x04: stp(PB_NUSIZ0, v); break;
    case 0x05: stp(PB_NUSIZ1, v); break;
    case 0x06: case 0x07: case 0x08: case 0x09: stp(PB_COLUP0 + (r - 0x06u), v); break;
    case 0x0A: stp(PB_CTRLPF, v); break;
    case 0x0B: stp(PB_REFP0, (v >> 3) & 1u); break;
    case 0x0C: stp(PB_REFP1, (v >> 3) & 1u); break;
    case 0x0D: case 0x0E: case 0x0F: stp(PB_PF0 + (r - 0x0Du), v); break;
    case 0x10: case 0x11: case 0x12: case 0x13: case 0x14:
        // RESPx: (clock as i16 - 68 + 5).rem_euclid(160)
        stp16(PB_POS + 2u * (r - 0x10u), mod160((int16_t)(uint16_t)(clock - 63u)));
        break;
    case 0x1B: stp(PB_GRP0_OLD, ldp(PB_GRP0)); stp(PB_GRP0, v); break;
    case 0x1C:
        stp(PB_GRP1_OLD, ldp(PB_GRP1)); stp(PB_GRP1, v);
        stp(PB_ENABL_OLD, ldp(PB_ENABL)); break;
    case 0x1D: case 0x1E: case 0x1F: stp(PB_ENAM0 + (r - 0x1Du), (v >> 1) & 1u); break;
    case 0x20: case 0x21: case 0x22: case 0x23: case 0x24: stp(PB_HM + (r - 0x20u), v); break;
    case 0x25: case 0x26: case 0x27: stp(PB_VDELP0 + (r - 0x25u), v & 1u); break;
    case 0x28: case 0x29: stp(PB_RESMP0 + (r - 0x28u), (v >> 1) & 1u); break;
    case 0x2A:                                                        // HMOVE
        for (uint32_t k = 0; k < 5u; k++) {
            int off = ((int)(int8_t)(uint8_t)ldp(PB_HM + k)) >> 4;
            int16_t d = (int16_t)(uint16_t)(ldp16(PB_POS + 2u * k) - (uint32_t)off);
            stp16(PB_POS + 2u * k, mod160(d));
        }
        break;
    case 0x2B: for (uint32_t k = 0; k < 5u; k++) stp(PB_HM + k, 0); break;
    case 0x2C: for (uint32_t k = 0; k < 8u; k++) stp(PB_CX + k, 0); break;
    default: break;
    }
    return make_uint2(tw, lw);
}

// Pia::write, I/O half (src/pia.rs:202-228).  Returns (ports, timer value,
// prescaler, select | underflow<<16).
static __device__ __noinline__ uint4 pia_write_io(uint32_t a, uint32_t v, uint32_t ports, uint32_t tv, uint32_t ps,
                                           uint32_t sel_uf)
{
    if (a & 0x10u) {
        const uint32_t sel = 1u << ((0xA630u >> (4u * (a & 3u))) & 0xFu);   // 1, 8, 64, 1024
        return make_uint4(ports, v, sel, sel);
    }
    const uint32_t sh = 8u * (a & 3u);                                 // pa_out pa_ddr pb_out pb_ddr
    return make_uint4((ports & ~(0xFFu << sh)) | (v << sh), tv, ps, sel_uf);
}

template <int BLOCK>
struct Emu {
    // ---- placement
    uint8_t* pv;             // this thread's RAM (shared memory, interleaved by thread)
    const FaGroup* G;        // the instance's group (HBM state rows, stride)
    uint32_t i;              // the instance's index in its group
    const uint8_t* rom;      // shared-memory ROM image, nbanks * 4 KiB
    uint32_t hot_lo, nbanks;
    // ---- CPU (src/cpu.rs:96-105)
    uint32_t a, x, y, sp, p, pc;
    uint32_t bank;           // bank index (bits 0-2) | hotspot accesses this frame << 3,
                             // saturating at 511: the count is a scheduling key only
    uint32_t cyc_acc;         // instruction cycles not yet added to Cpu::cycles in HBM
    // ---- PIA (src/pia.rs:26-44): timer unpacked (ticked every instruction),
    //      ports and input pins packed (touched only by I/O accesses)
    uint32_t tv, ps, sel, uf;
    uint32_t ports;          // pa_out | pa_ddr<<8 | pb_out<<16 | pb_ddr<<24
    uint32_t pins;           // pa_in | pb_in<<8 | inpt4<<16 | inpt5<<17
    uint32_t pads;           // paddle0 | paddle1<<8
    // ---- TIA (src/headless_tia.rs:16-45): beam position unpacked, flags packed
    uint32_t clock, scanline, pcnt;
    uint32_t tw;             // vsync | vblank<<8 | wsync<<16 | frame_complete<<17 | paddle_dumped<<18
    // ---- run bookkeeping
    uint32_t instr;           // instructions executed in this launch (statistics)

    // The instance's HBM rows.  Cpu::cycles, the frame counter and the run
    // status stay there and change only at frame boundaries.
    __device__ __forceinline__ uint32_t* column() const { return G->state + i; }
    __device__ __forceinline__ uint32_t& row(uint32_t w) const { return column()[(size_t)w * G->stride]; }
    __device__ __forceinline__ void fold_cycles()
    {
        uint32_t& lo = row(R_CYC_LO);
        const uint32_t v = lo + cyc_acc;
        if (v < cyc_acc) row(R_CYC_HI) += 1u;
        lo = v;
        cyc_acc = 0;
    }
    __device__ __forceinline__ void set_status(uint32_t bits) { row(R_STATUS) |= bits; }

    __device__ __forceinline__ bool vsync_on() const { return (tw & 2u) != 0; }
    __device__ __forceinline__ bool wsync() const { return (tw & TW_WSYNC) != 0; }

    // ------------------------------------------------------------ private bytes
    __device__ __forceinline__ uint32_t poff(uint32_t o) const { return priv_off<BLOCK>(o); }
    __device__ __forceinline__ uint32_t ldp(uint32_t o) const { return pv[poff(o)]; }
    __device__ __forceinline__ void stp(uint32_t o, uint32_t v) { pv[poff(o)] = (uint8_t)v; }
    __device__ __forceinline__ uint32_t ldp16(uint32_t o) const { return *(const uint16_t*)(pv + poff(o)); }
    __device__ __forceinline__ void stp16(uint32_t o, uint32_t v) { *(uint16_t*)(pv + poff(o)) = (uint16_t)v; }

    // ------------------------------------------------------------ flags
    __device__ __forceinline__ void nz(uint32_t v) { p = (p & ~(F_N | F_Z)) | (v & F_N) | (v ? 0u : F_Z); }
    __device__ __forceinline__ void setc(bool c) { p = (p & ~F_C) | (c ? F_C : 0u); }

    // ------------------------------------------------------------ bank switching
    // A hotspot access selects its bank (src/atari.rs:460-492) and counts one
    // more bank-switch point passed this frame in bank's upper bits.
    __device__ __forceinline__ void bsw(uint32_t a13)
    {
        uint32_t d = a13 - hot_lo;
        if (d < nbanks) bank = (bank < (511u << 3) ? ((bank + 8u) & ~7u) : (bank & ~7u)) | d;
    }

    // ------------------------------------------------------------ TIA (headless_tia.rs)
    __device__ __forceinline__ void end_scanline()                   // :183-198
    {
        clock = (clock - 228u) & 0xFFFFu;
        scanline = (scanline + 1u) & 0xFFFFu;
        tw &= ~TW_WSYNC;
        if (!(tw & TW_PDUMP) && pcnt < 256u) pcnt++;
        if (scanline >= 262u) { scanline = 0; tw |= TW_FCOMP; }
    }
    __device__ __forceinline__ void tia_tick(uint32_t n)            // :153-158
    {
        clock = (clock + 3u * n) & 0xFFFFu;
        if (clock >= 228u) end_scanline();
    }
    __device__ __forceinline__ uint32_t tia_skip()                   // :163-180
    {
        uint32_t rem = clock >= 228u ? 0u : 228u - clock;
        uint32_t c = (rem + 2u) / 3u;
        if (c) { clock = 228u; end_scanline(); }
        return c;
    }

    // ------------------------------------------------------------ PIA timer (pia.rs:107-166)
    __device__ __forceinline__ void pia_tick(uint32_t n)
    {
        if (n == 0) return;
        if (tv == 0 && uf) { tv = (0xFFu - (n - 1u)) & 0xFFu; return; }
        uint32_t rem = n;
        if (ps > 0) {
            if (rem < ps) { ps -= rem; return; }
            rem -= ps;
            ps = 0;
            if (tv == 0) {
                uf = 1;
                tv = rem ? ((0xFFu - (rem - 1u)) & 0xFFu) : 0xFFu;
                return;
            }
            tv -= 1u;
        }
        if (rem == 0) { ps = sel; return; }
        uint32_t full, left;
        if ((sel & (sel - 1u)) == 0) {                    // 1, 8, 64, 1024
            uint32_t sh = __ffs(sel) - 1u;
            full = rem >> sh;
            left = rem & (sel - 1u);
        } else {
            full = rem / sel;
            left = rem % sel;
        }
        if (full >= tv) {
            rem = (rem - ((tv * sel) & 0xFFFFu)) & 0xFFFFu;   // u16 arithmetic as in the reference
            uf = 1;
            tv = rem ? ((0xFFu - (rem - 1u)) & 0xFFu) : 0xFFu;
        } else {
            tv -= full;
            ps = sel - left;
        }
    }

    // ------------------------------------------------------------ bus (atari.rs:497-552)
    // ROM, RAM and hotspots are handled inline; TIA and PIA registers go
    // through one out-of-line copy of their decoders (io_read / tia_write_io /
    // pia_write_io), which keeps the interpreter's code small enough to stay
    // resident in the instruction cache.
    __device__ __forceinline__ uint32_t io(uint32_t a)               // TIA or PIA register read
    {
        uint32_t r = io_read(a, pcnt, pins, pads, ports, tv | (uf << 16), (const uint8_t*)column(), G->stride * 4u);
        if (r & 0x100u) uf = 0;                                     // INTIM read clears the flag
        return r & 0xFFu;
    }
    __device__ __forceinline__ void io_write(uint32_t a, uint32_t v)  // TIA or PIA register write
    {
        if (a & 0x200u) {
            uint4 r = pia_write_io(a, v, ports, tv, ps, sel | (uf << 16));
            ports = r.x; tv = r.y; ps = r.z; sel = r.w & 0xFFFFu; uf = r.w >> 16;
        } else {
            uint2 r = tia_write_io(a, v, clock, tw, scanline | (pcnt << 16), (uint8_t*)column(), G->stride * 4u);
            tw = r.x; scanline = r.y & 0xFFFFu; pcnt = r.y >> 16;
        }
    }
    __device__ __forceinline__ uint32_t read_low(uint32_t a)         // a < 0x1000
    {
        if ((a & 0x80u) && (a & 0x280u) != 0x280u)                  // RAM and its mirrors
            return a < 0x200u ? ldp(a & 0x7Fu) : 0u;                // other mirrors read the never-written flat array
        return io(a);
    }
    __device__ __forceinline__ uint32_t read(uint32_t addr)
    {
        uint32_t a = addr & 0x1FFFu;
        if (a & 0x1000u) { bsw(a); return rom[((bank & 7u) << 12) | (a & 0xFFFu)]; }
        return read_low(a);
    }
    __device__ __forceinline__ void write(uint32_t addr, uint32_t v)
    {
        uint32_t a = addr & 0x1FFFu;
        if (a & 0x1000u) { bsw(a); return; }
        if ((a & 0x280u) == 0x080u) { stp(a & 0x7Fu, v); return; }
        io_write(a, v);
    }
    // A phantom read: only its side effects (hotspot, INTIM) matter.
    __device__ __forceinline__ void dummy(uint32_t addr)
    {
        uint32_t a = addr & 0x1FFFu;
        if (a & 0x1000u) bsw(a);
        else if ((a & 0x287u) == 0x284u) uf = 0;
    }
    __device__ __forceinline__ uint32_t zp_read(uint32_t z) { return (z & 0x80u) ? ldp(z & 0x7Fu) : io(z); }
    __device__ __forceinline__ uint32_t fetch() { uint32_t v = read(pc); pc = (pc + 1u) & 0xFFFFu; return v; }
    __device__ __forceinline__ void push(uint32_t v)
    {
        if (sp & 0x80u) stp(sp & 0x7Fu, v); else io_write(0x100u | sp, v);
        sp = (sp - 1u) & 0xFFu;
    }
    __device__ __forceinline__ uint32_t pull()
    {
        sp = (sp + 1u) & 0xFFu;
        return (sp & 0x80u) ? ldp(sp & 0x7Fu) : io(0x100u | sp);
    }
    // Read-modify-write's two writes; a RAM target only needs the second.
    __device__ __forceinline__ void rmw_store(uint32_t ea, uint32_t oldv, uint32_t newv)
    {
        uint32_t a = ea & 0x1FFFu;
        if ((a & 0x1280u) == 0x080u) { stp(a & 0x7Fu, newv); return; }
        write(ea, oldv);
        write(ea, newv);
    }

    // ------------------------------------------------------------ ALU (cpu.rs:153-241)
    __device__ __forceinline__ void adc(uint32_t v)
    {
        uint32_t c = p & F_C;
        if (p & F_D) {
            uint32_t lo = (a & 0xFu) + (v & 0xFu) + c;
            if (lo > 9u) lo += 6u;
            uint32_t hi = (a >> 4) + (v >> 4) + (lo > 0xFu ? 1u : 0u);
            uint32_t bin = (a + v + c) & 0xFFu;
            uint32_t res = ((hi << 4) | (lo & 0xFu)) & 0xFFu;
            p &= ~(F_Z | F_N | F_V | F_C);
            p |= bin ? 0u : F_Z;
            p |= (hi & 8u) ? F_N : 0u;
            p |= (~(a ^ v) & (a ^ res) & 0x80u) ? F_V : 0u;
            if (hi > 9u) hi += 6u;
            p |= hi > 0xFu ? F_C : 0u;
            a = ((hi & 0xFu) << 4) | (lo & 0xFu);
        } else {
            uint32_t s = a + v + c;
            uint32_t r = s & 0xFFu;
            p = (p & ~(F_V | F_C)) | (s >> 8) | ((~(a ^ v) & (a ^ r) & 0x80u) ? F_V : 0u);
            a = r;
            nz(a);
        }
    }
    __device__ __forceinline__ void sbc(uint32_t v)
    {
        uint32_t b = (p & F_C) ^ 1u;
        int bin = (int)a - (int)v - (int)b;
        uint32_t r = (uint32_t)bin & 0xFFu;
        if (p & F_D) {
            uint32_t lo = ((a & 0xFu) - (v & 0xFu) - b) & 0xFFu;
            uint32_t lob = 0;
            if (lo & 0x80u) { lo = (lo - 6u) & 0xFFu; lob = 1; }
            uint32_t hi = ((a >> 4) - (v >> 4) - lob) & 0xFFu;
            if (hi & 0x80u) hi = (hi - 6u) & 0xFFu;
            p &= ~(F_Z | F_N | F_V | F_C);
            p |= bin >= 0 ? F_C : 0u;
            p |= r ? 0u : F_Z;
            p |= r & F_N;
            p |= ((a ^ v) & (a ^ r) & 0x80u) ? F_V : 0u;
            a = ((hi & 0xFu) << 4) | (lo & 0xFu);
        } else {
            p = (p & ~(F_V | F_C)) | (bin >= 0 ? F_C : 0u) | (((a ^ v) & (a ^ r) & 0x80u) ? F_V : 0u);
            a = r;
            nz(a);
        }
    }
    __device__ __forceinline__ void cmp(uint32_t reg, uint32_t v)
    {
        setc(reg >= v);
        nz((reg - v) & 0xFFu);
    }
    __device__ __forceinline__ void bit(uint32_t v)
    {
        p = (p & ~(F_Z | F_V | F_N)) | ((a & v) ? 0u : F_Z) | (v & (F_V | F_N));
    }
    // Shift/rotate/INC/DEC by the aaa field of a cc=10 opcode.
    __device__ __forceinline__ uint32_t shift_op(uint32_t aaa, uint32_t v)
    {
        uint32_t r;
        switch (aaa) {
        case 0: setc(v & 0x80u); r = (v << 1) & 0xFFu; break;                       // ASL
        case 1: r = ((v << 1) | (p & F_C)) & 0xFFu; setc(v & 0x80u); break;         // ROL
        case 2: setc(v & 1u); r = v >> 1; break;                                    // LSR
        case 3: r = (v >> 1) | ((p & F_C) << 7); setc(v & 1u); break;               // ROR
        case 6: r = (v - 1u) & 0xFFu; break;                                        // DEC
        default: r = (v + 1u) & 0xFFu; break;                                       // INC
        }
        nz(r);
        return r;
    }

    // ------------------------------------------------------------ instruction groups
    // The opcode (at pc0) and the byte after it (b1: the operand, or the
    // phantom read every 1-byte instruction makes at pc0+1) are read by
    // step() for every legal opcode, in that order, as the reference does on
    // cycles 1 and 2.  b2 is the byte at pc0+2 for the 3-byte forms, read on
    // cycle 3 (JSR reads its high byte later and fetches it itself).

    // cc = 01: ORA AND EOR ADC STA LDA CMP SBC x 8 addressing modes.
    __device__ __forceinline__ uint32_t group1(uint32_t pc0, uint32_t aaa, uint32_t bbb, uint32_t b1, uint32_t b2)
    {
        const bool st = aaa == 4u;
        uint32_t ea, cyc, v;
        switch (bbb) {
        case 0: {                                                   // (zp,X)
            const uint32_t z = (b1 + x) & 0xFFu;
            const uint32_t lo = zp_read(z);
            ea = (zp_read((z + 1u) & 0xFFu) << 8) | lo;
            cyc = 6;
            break;
        }
        case 1: ea = b1; cyc = 3; break;                            // zp
        case 2: v = b1; cyc = 2; pc = (pc0 + 2u) & 0xFFFFu; goto operate;   // #imm ($89 is illegal)
        case 3: ea = (b2 << 8) | b1; cyc = 4; break;                // abs
        case 4: {                                                   // (zp),Y
            const uint32_t lo = zp_read(b1);
            const uint32_t base = (zp_read((b1 + 1u) & 0xFFu) << 8) | lo;
            ea = (base + y) & 0xFFFFu;
            cyc = 5;
            if (st || ((base ^ ea) & 0xFF00u)) { dummy((base & 0xFF00u) | (ea & 0xFFu)); cyc = 6; }
            break;
        }
        case 5: ea = (b1 + x) & 0xFFu; cyc = 4; break;             // zp,X
        default: {                                                  // abs,Y / abs,X
            const uint32_t base = (b2 << 8) | b1;
            ea = (base + (bbb == 6u ? y : x)) & 0xFFFFu;
            cyc = 4;
            if (st || ((base ^ ea) & 0xFF00u)) { dummy((base & 0xFF00u) | (ea & 0xFFu)); cyc = 5; }
            break;
        }
        }
        pc = (pc0 + ((bbb == 3u || bbb >= 6u) ? 3u : 2u)) & 0xFFFFu;
        if (st) { write(ea, a); return cyc; }
        v = read(ea);
    operate:
        switch (aaa) {
        case 0: a |= v; nz(a); break;
        case 1: a &= v; nz(a); break;
        case 2: a ^= v; nz(a); break;
        case 3: adc(v); break;
        case 5: a = v; nz(a); break;
        case 6: cmp(a, v); break;
        default: sbc(v); break;
        }
        return cyc;
    }

    // cc = 10: ASL ROL LSR ROR STX LDX DEC INC, plus TXA TAX DEX NOP TXS TSX.
    __device__ __forceinline__ uint32_t group2(uint32_t pc0, uint32_t aaa, uint32_t bbb, uint32_t b1, uint32_t b2)
    {
        uint32_t ea, cyc;
        switch (bbb) {
        case 0:                                                     // LDX #imm
            x = b1; nz(x); pc = (pc0 + 2u) & 0xFFFFu; return 2;
        case 2:                                                     // accumulator / implied
            pc = (pc0 + 1u) & 0xFFFFu;
            switch (aaa) {
            case 4: a = x; nz(a); break;                            // TXA
            case 5: x = a; nz(x); break;                            // TAX
            case 6: x = (x - 1u) & 0xFFu; nz(x); break;             // DEX
            case 7: break;                                          // NOP
            default: a = shift_op(aaa, a); break;
            }
            return 2;
        case 6:                                                     // TXS / TSX
            pc = (pc0 + 1u) & 0xFFFFu;
            if (aaa == 4u) sp = x; else { x = sp; nz(x); }
            return 2;
        case 1: ea = b1; cyc = 3; pc = (pc0 + 2u) & 0xFFFFu; break; // zp
        case 3: ea = (b2 << 8) | b1; cyc = 4; pc = (pc0 + 3u) & 0xFFFFu; break;
        case 5:                                                     // zp,X (zp,Y for STX/LDX)
            ea = (b1 + ((aaa == 4u || aaa == 5u) ? y : x)) & 0xFFu; cyc = 4; pc = (pc0 + 2u) & 0xFFFFu; break;
        default: {                                                  // abs,X (abs,Y for LDX)
            pc = (pc0 + 3u) & 0xFFFFu;
            const uint32_t base = (b2 << 8) | b1;
            if (aaa == 5u) {
                ea = (base + y) & 0xFFFFu; cyc = 4;
                if ((base ^ ea) & 0xFF00u) { dummy((base & 0xFF00u) | (ea & 0xFFu)); cyc = 5; }
                x = read(ea); nz(x); return cyc;
            }
            ea = (base + x) & 0xFFFFu;
            dummy((base & 0xFF00u) | (ea & 0xFFu));
            const uint32_t v = read(ea);
            rmw_store(ea, v, shift_op(aaa, v));
            return 7;
        }
        }
        if (aaa == 4u) { write(ea, x); return cyc; }
        if (aaa == 5u) { x = read(ea); nz(x); return cyc; }
        const uint32_t v = read(ea);
        rmw_store(ea, v, shift_op(aaa, v));
        return cyc + 2u;
    }

    // cc = 00: control flow, stack, flags, BIT/STY/LDY/CPY/CPX.
    __device__ __forceinline__ uint32_t group0(uint32_t pc0, uint32_t aaa, uint32_t bbb, uint32_t b1, uint32_t b2)
    {
        switch (bbb) {
        case 4: {                                                   // branches
            pc = (pc0 + 2u) & 0xFFFFu;
            const uint32_t pos = (0x1067u >> (4u * (aaa >> 1))) & 0xFu;    // N V C Z
            if (((p >> pos) & 1u) != (aaa & 1u)) return 2;
            dummy(pc);
            const uint32_t npc = (pc + (uint32_t)(int32_t)(int8_t)(uint8_t)b1) & 0xFFFFu;
            uint32_t cyc = 3;
            if ((pc ^ npc) & 0xFF00u) { dummy((pc & 0xFF00u) | (npc & 0xFFu)); cyc = 4; }
            pc = npc;
            return cyc;
        }
        case 6:                                                     // flags, TYA
            pc = (pc0 + 1u) & 0xFFFFu;
            switch (aaa) {
            case 0: p &= ~F_C; break;
            case 1: p |= F_C; break;
            case 2: p &= ~F_I; break;
            case 3: p |= F_I; break;
            case 4: a = y; nz(a); break;
            case 5: p &= ~F_V; break;
            case 6: p &= ~F_D; break;
            default: p |= F_D; break;
            }
            return 2;
        case 2:                                                     // stack, DEY TAY INY INX
            pc = (pc0 + 1u) & 0xFFFFu;
            switch (aaa) {
            case 0: push(p | F_B | F_U); return 3;                  // PHP
            case 1: p = pull() & ~(F_B | F_U); return 4;            // PLP
            case 2: push(a); return 3;                              // PHA
            case 3: a = pull(); nz(a); return 4;                    // PLA
            case 4: y = (y - 1u) & 0xFFu; nz(y); return 2;          // DEY
            case 5: y = a; nz(y); return 2;                         // TAY
            case 6: y = (y + 1u) & 0xFFu; nz(y); return 2;          // INY
            default: x = (x + 1u) & 0xFFu; nz(x); return 2;         // INX
            }
        case 0:
            switch (aaa) {
            case 0: {                                               // BRK (b1 is the padding byte)
                pc = (pc0 + 2u) & 0xFFFFu;
                push(pc >> 8); push(pc & 0xFFu); push(p | F_B | F_U);
                p |= F_I;
                const uint32_t lo = read(0xFFFEu);
                pc = (read(0xFFFFu) << 8) | lo;
                return 7;
            }
            case 1: {                                               // JSR: pushes before the high byte
                pc = (pc0 + 2u) & 0xFFFFu;
                push(pc >> 8); push(pc & 0xFFu);
                pc = (read(pc) << 8) | b1;
                return 6;
            }
            case 2: {                                               // RTI
                p = pull() & ~(F_B | F_U);
                const uint32_t lo = pull();
                pc = (pull() << 8) | lo;
                return 6;
            }
            case 3: {                                               // RTS
                const uint32_t lo = pull();
                const uint32_t ra = (pull() << 8) | lo;
                dummy(ra);
                pc = (ra + 1u) & 0xFFFFu;
                return 6;
            }
            case 5: y = b1; nz(y); break;                           // LDY #
            case 6: cmp(y, b1); break;                              // CPY #
            default: cmp(x, b1); break;                             // CPX #
            }
            pc = (pc0 + 2u) & 0xFFFFu;
            return 2;
        case 3:                                                     // absolute
            pc = (pc0 + 3u) & 0xFFFFu;
            if (aaa == 2u) { pc = (b2 << 8) | b1; return 3; }       // JMP
            if (aaa == 3u) {                                        // JMP (ind), page-wrap bug
                const uint32_t ptr = (b2 << 8) | b1;
                const uint32_t tlo = read(ptr);
                pc = (read((ptr & 0xFF00u) | ((ptr + 1u) & 0xFFu)) << 8) | tlo;
                return 5;
            }
            return mem0(aaa, (b2 << 8) | b1, 4);
        case 1:                                                     // zp: BIT STY LDY CPY CPX
            pc = (pc0 + 2u) & 0xFFFFu;
            return mem0(aaa, b1, 3);
        case 5:                                                     // zp,X: STY LDY
            pc = (pc0 + 2u) & 0xFFFFu;
            return mem0(aaa, (b1 + x) & 0xFFu, 4);
        default: {                                                  // abs,X: LDY
            pc = (pc0 + 3u) & 0xFFFFu;
            const uint32_t base = (b2 << 8) | b1;
            const uint32_t ea = (base + x) & 0xFFFFu;
            uint32_t cyc = 4;
            if ((base ^ ea) & 0xFF00u) { dummy((base & 0xFF00u) | (ea & 0xFFu)); cyc = 5; }
            y = read(ea); nz(y);
            return cyc;
        }
        }
    }
    __device__ __forceinline__ uint32_t mem0(uint32_t aaa, uint32_t ea, uint32_t cyc)
    {
        if (aaa == 4u) { write(ea, y); return cyc; }                // STY
        const uint32_t v = read(ea);
        switch (aaa) {
        case 1: bit(v); break;
        case 5: y = v; nz(y); break;
        case 6: cmp(y, v); break;
        default: cmp(x, v); break;
        }
        return cyc;
    }

    // One instruction; returns its cycle count, or 0 for an illegal opcode
    // (pc is then past the opcode and nothing else changed: the reference
    // panics right after the opcode fetch, src/cpu.rs:1139-1141).
    __device__ __forceinline__ uint32_t step()
    {
        const uint32_t pc0 = pc;
        const uint32_t a0 = pc0 & 0x1FFFu;
        uint32_t op, b1, b2 = 0;
        if (a0 >= 0x1000u && a0 + 2u < hot_lo) {
            // Fast path: the three bytes at pc0 lie in the current bank and
            // below every hotspot, so reading them has no side effect.
            const uint8_t* q = rom + ((bank & 7u) << 12) + (a0 & 0xFFFu);
            op = q[0];
            if (!((c_legal[op >> 5] >> (op & 31u)) & 1u)) { pc = (pc0 + 1u) & 0xFFFFu; return 0; }
            b1 = q[1];
            b2 = q[2];
        } else {
            op = read(pc0);
            if (!((c_legal[op >> 5] >> (op & 31u)) & 1u)) { pc = (pc0 + 1u) & 0xFFFFu; return 0; }
            b1 = read((pc0 + 1u) & 0xFFFFu);
            const uint32_t bb = (op >> 2) & 7u;
            if (bb == 3u || bb == 7u || (bb == 6u && (op & 3u) == 1u)) b2 = read((pc0 + 2u) & 0xFFFFu);
        }
        const uint32_t aaa = op >> 5, bbb = (op >> 2) & 7u, cc = op & 3u;
        if (cc == 1u) return group1(pc0, aaa, bbb, b1, b2);
        if (cc == 2u) return group2(pc0, aaa, bbb, b1, b2);
        return group0(pc0, aaa, bbb, b1, b2);
    }

    // HeadlessAtari::set_action (src/atari.rs:571-582).
    __device__ __forceinline__ void apply_action(uint32_t act)
    {
        uint32_t t = c_action_table[act < 18u ? act : 0u];
        pins = (pins & ~0x100FFu) | (t & 0xFFu) | (((t >> 8) & 1u) << 16);
        pads = (pads & ~0xFFu) | ((t >> 16) & 0xFFu);
    }

    // ------------------------------------------------------------ state movement
    __device__ __forceinline__ void load_hot(const uint32_t* col, uint32_t stride)
    {
        uint32_t w;
        w = col[R_AXYS * stride];  a = w & 0xFF; x = (w >> 8) & 0xFF; y = (w >> 16) & 0xFF; sp = w >> 24;
        w = col[R_PC * stride];    pc = w & 0xFFFF; p = (w >> 16) & 0xFF; bank = w >> 24;
        cyc_acc = 0;
        const uint32_t p0 = col[R_PIA0 * stride];                  // pa_out pa_ddr pa_in pb_out
        const uint32_t p1 = col[R_PIA1 * stride];                  // pb_ddr pb_in uf pdump
        ports = (p0 & 0xFFFFu) | ((p0 >> 24) << 16) | ((p1 & 0xFFu) << 24);
        uf = (p1 >> 16) & 0xFF;
        w = col[R_TIMER * stride]; tv = w & 0xFFFF; ps = w >> 16;
        w = col[R_SELPC * stride]; sel = w & 0xFFFF; pcnt = w >> 16;
        w = col[R_TIA0 * stride];  clock = w & 0xFFFF; scanline = w >> 16;
        w = col[R_TIA1 * stride];                                   // wsync fcomp vsync vblank
        tw = ((w >> 16) & 0xFFFFu) | ((w & 1u) << 16) | (((w >> 8) & 1u) << 17) | (((p1 >> 24) & 1u) << 18);
        w = col[R_TIA2 * stride];                                   // inpt4 inpt5 pad0 pad1
        pins = ((p0 >> 16) & 0xFFu) | (((p1 >> 8) & 0xFFu) << 8) | ((w & 1u) << 16) | (((w >> 8) & 1u) << 17);
        pads = w >> 16;
    }
    __device__ __forceinline__ void store_hot(uint32_t* col, uint32_t stride) const
    {
        col[R_AXYS * stride] = a | (x << 8) | (y << 16) | (sp << 24);
        col[R_PC * stride] = pc | (p << 16) | ((bank & 7u) << 24);
        col[R_PIA0 * stride] = (ports & 0xFFFFu) | ((pins & 0xFFu) << 16) | (((ports >> 16) & 0xFFu) << 24);
        col[R_PIA1 * stride] = (ports >> 24) | (((pins >> 8) & 0xFFu) << 8) | (uf << 16) | (((tw >> 18) & 1u) << 24);
        col[R_TIMER * stride] = tv | (ps << 16);
        col[R_SELPC * stride] = sel | (pcnt << 16);
        col[R_TIA0 * stride] = clock | (scanline << 16);
        col[R_TIA1 * stride] = ((tw >> 16) & 1u) | (((tw >> 17) & 1u) << 8) | ((tw & 0xFFFFu) << 16);
        col[R_TIA2 * stride] = ((pins >> 16) & 1u) | (((pins >> 17) & 1u) << 8) | (pads << 16);
    }
    // RAM words from the HBM rows into shared memory and back.
    __device__ __forceinline__ void load_ram(const uint32_t* c, uint32_t stride)
    {
        uint32_t* w = (uint32_t*)pv;
#pragma unroll 4
        for (uint32_t k = 0; k < FA_SMEM_WORDS; k++) w[k * BLOCK] = c[k * stride];
    }
    __device__ __forceinline__ void store_ram(uint32_t* c, uint32_t stride) const
    {
        const uint32_t* w = (const uint32_t*)pv;
#pragma unroll 4
        for (uint32_t k = 0; k < FA_SMEM_WORDS; k++) c[k * stride] = w[k * BLOCK];
    }
};

}  // namespace fa
