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
enum : uint32_t { TW_WSYNC = 1u << 16, TW_FCOMP = 1u << 17, TW_PDUMP = 1u << 18,
                  // rendering console only
                  TW_HMOVE = 1u << 19, TW_LATCH = 1u << 20, TW_L4 = 1u << 21, TW_L5 = 1u << 22 };

// NUSIZ copy offsets as a mask over {0, 16, 32, 64} (tia.rs:440-450, 480-488).
static __constant__ uint32_t c_copies[8] = { 0x1, 0x3, 0x5, 0x7, 0x9, 0x1, 0xD, 0x1 };


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
// Pia::read I/O half, src/pia.rs:169-199), INTIM apart (pia_intim_io):
// sel_uf carries the timer's underflow flag in bits 16 and up.
static __device__ __noinline__ uint32_t io_read(uint32_t a, uint32_t pcnt, uint32_t pins, uint32_t pads,
                                         uint32_t ports, uint32_t sel_uf, const uint8_t* col, uint32_t stride4)
{
    if (a & 0x80u) {                                                 // PIA: (a & 0x280) == 0x280
        switch (a & 7u) {
        case 0: return ((pins & ~(ports >> 8)) | (ports & (ports >> 8))) & 0xFFu;
        case 1: return (ports >> 8) & 0xFFu;
        case 2: return (((pins >> 8) & ~(ports >> 24)) | ((ports >> 16) & (ports >> 24))) & 0xFFu;
        case 3: return ports >> 24;
        case 5: return (sel_uf >> 16) ? 0x80u : 0u;
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

// ---------------------------------------------------------------- rendering console
// The pixel-accurate Tia (src/tia.rs) and the per-cycle Pia::tick
// (src/pia.rs:80-103) of the reference's rendering console, as out-of-line
// functions on the state they touch.  The registers of the TIA are the
// console's private bytes in shared memory (PB_* graphics registers, RB_*
// extras), interleaved by lane in 32-lane slabs; the framebuffer is HBM.
struct RState {
    uint32_t clock, scanline, tw, pcnt, vtop;   // beam, TIA flags, paddle counter, visible_top | vblank_top << 16
    uint32_t rx;                                // the current line's pixels are drawn up to this clock
    uint32_t sc;                                // the framebuffer sector (32 pixels) whose pixels the sector buffer holds
    uint32_t zr;                                // rows written since the clear point | R_ZPEND (rows after them not yet zeroed)
    uint32_t tv, ps, sel, uf;                   // PIA timer
};
constexpr uint32_t R_ZPEND = 0x100u;

static __device__ __forceinline__ uint32_t rp8(const uint8_t* pv, uint32_t o) { return pv[(o & ~3u) * 32u + (o & 3u)]; }
static __device__ __forceinline__ void wp8(uint8_t* pv, uint32_t o, uint32_t v) { pv[(o & ~3u) * 32u + (o & 3u)] = (uint8_t)v; }
static __device__ __forceinline__ uint32_t rp16(const uint8_t* pv, uint32_t o) { return *(const uint16_t*)(pv + (o & ~3u) * 32u + (o & 3u)); }
static __device__ __forceinline__ void wp16(uint8_t* pv, uint32_t o, uint32_t v) { *(uint16_t*)(pv + (o & ~3u) * 32u + (o & 3u)) = (uint16_t)v; }

// ---- framebuffer writes through a one-sector buffer
// Pixels of a line are drawn left to right, so a console stages the 32
// pixels of the framebuffer sector it is drawing (8 words after its private
// bytes in its shared-memory slab) and writes each sector whole, with two
// 16-byte stores, when the drawing moves past it: every sector of a visible
// row is written once, with zeros where nothing was drawn.  The reference
// clears the framebuffer where the visible area starts (tia.rs:349-351);
// here the rows are written as the beam completes them, and the rows the
// frame has not reached are zeroed when the framebuffer can next be seen
// (VSYNC, the end of a frame, the end of a call).
static __device__ __forceinline__ uint32_t* r_sbuf(uint8_t* pv, uint32_t k)
{
    return (uint32_t*)(pv + (FA_RPRIV_BYTES + 4u * k) * 32u);
}
static __device__ __forceinline__ void r_sec_write(uint8_t* pv, uint8_t* fbp, uint32_t sc)
{
    uint4* d = (uint4*)(fbp + (size_t)sc * 32u);
    d[0] = make_uint4(*r_sbuf(pv, 0), *r_sbuf(pv, 1), *r_sbuf(pv, 2), *r_sbuf(pv, 3));
    d[1] = make_uint4(*r_sbuf(pv, 4), *r_sbuf(pv, 5), *r_sbuf(pv, 6), *r_sbuf(pv, 7));
}
static __device__ __forceinline__ void r_sec_clear(uint8_t* pv)
{
#pragma unroll
    for (uint32_t k = 0; k < 8u; k++) *r_sbuf(pv, k) = 0u;
}
static __device__ __forceinline__ void r_zero_sectors(uint8_t* fbp, uint32_t from, uint32_t to)   // [from, to)
{
    uint4* d = (uint4*)fbp;
    for (uint32_t q = 2u * from; q < 2u * to; q++) d[q] = make_uint4(0u, 0u, 0u, 0u);
}
// The buffer moves on to sector t: the sector it held is written, the ones
// skipped between become zeros.
static __device__ void r_seek(uint32_t& sc, uint8_t* pv, uint8_t* fbp, uint32_t t)
{
    r_sec_write(pv, fbp, sc);
    if (t > sc) {
        r_zero_sectors(fbp, sc + 1u, t);
        r_sec_clear(pv);
    } else {                                                         // not reached by drawing order; kept exact
        const uint4* q = (const uint4*)(fbp + (size_t)t * 32u);
        const uint4 u0 = q[0], u1 = q[1];
        *r_sbuf(pv, 0) = u0.x; *r_sbuf(pv, 1) = u0.y; *r_sbuf(pv, 2) = u0.z; *r_sbuf(pv, 3) = u0.w;
        *r_sbuf(pv, 4) = u1.x; *r_sbuf(pv, 5) = u1.y; *r_sbuf(pv, 6) = u1.z; *r_sbuf(pv, 7) = u1.w;
    }
    sc = t;
}

// Bits 0..7 of b, each repeated over two bits.
static __device__ __forceinline__ uint32_t r_spread2(uint32_t b)
{
    uint32_t t = (b | (b << 4)) & 0x0F0Fu;
    t = (t | (t << 2)) & 0x3333u;
    t = (t | (t << 1)) & 0x5555u;
    return t * 3u;
}

// Bits 0..7 of b, each repeated over four bits.
static __device__ __forceinline__ uint32_t r_spread4(uint32_t b)
{
    uint32_t t = (b & 0x0Fu) | ((b & 0xF0u) << 12);
    t = (t | (t << 6)) & 0x03030303u;
    t = (t | (t << 3)) & 0x11111111u;
    return t * 0xFu;
}

// Bits 0..3 of n moved to bits 0, 4, 8, 12.
static __device__ __forceinline__ uint32_t r_nib(uint32_t n)
{
    const uint32_t t = (n | (n << 6)) & 0x303u;
    return (t | (t << 3)) & 0x1111u;
}

// Bits 0..3 of n as byte masks.
static __device__ __forceinline__ uint32_t r_bytes(uint32_t n)
{
    return (((n & 0xFu) * 0x00204081u) & 0x01010101u) * 0xFFu;
}

// Pixels [X, X + 32) of the 160-pixel line covered by an object of len <= 32
// pixels starting at pixel s < 160, whose graphics g hold pixel d from its
// left edge in bit d: bit i = pixel X + i.  An object wraps from pixel 159
// to pixel 0, as the position arithmetic of tia.rs:406-507 does mod 160.
static __device__ __forceinline__ uint32_t r_place(uint32_t g, uint32_t len, uint32_t s, uint32_t X)
{
    const uint32_t i0 = s >= X ? s - X : s + 160u - X;
    if (i0 < 32u) return g << i0;
    const uint32_t d0 = 160u - i0;
    return d0 < len ? g >> d0 : 0u;
}

static __device__ __forceinline__ uint32_t r_copies(uint32_t g, uint32_t len, uint32_t pos, uint32_t copies, uint32_t X)
{
    uint32_t m = r_place(g, len, pos, X);
#pragma unroll
    for (uint32_t c = 1; c < 4u; c++)
        if ((copies >> c) & 1u) {
            uint32_t st = pos + (8u << c);                            // copies at +16, +32, +64
            if (st >= 160u) st -= 160u;
            m |= r_place(g, len, st, X);
        }
    return m;
}

// Player n over pixels [X, X + 32) (tia.rs:423-465): NUSIZ copies and
// widths, REFP reflection, VDELP's old graphics.
static __device__ __forceinline__ uint32_t r_player_mask(const uint8_t* pv, uint32_t n, uint32_t X)
{
    const uint32_t grp = rp8(pv, n ? (rp8(pv, PB_VDELP1) ? PB_GRP1_OLD : PB_GRP1) : (rp8(pv, PB_VDELP0) ? PB_GRP0_OLD : PB_GRP0));
    if (grp == 0) return 0;
    const uint32_t mode = rp8(pv, n ? PB_NUSIZ1 : PB_NUSIZ0) & 7u;
    const uint32_t g8 = rp8(pv, n ? PB_REFP1 : PB_REFP0) ? grp : __brev(grp) >> 24;
    const uint32_t g = mode == 5u ? r_spread2(g8) : mode == 7u ? r_spread4(g8) : g8;
    const uint32_t len = mode == 5u ? 16u : mode == 7u ? 32u : 8u;
    return r_copies(g, len, rp16(pv, PB_POS + 2u * n), c_copies[mode], X);
}

// Missile n over pixels [X, X + 32) (tia.rs:468-497).
static __device__ __forceinline__ uint32_t r_missile_mask(const uint8_t* pv, uint32_t n, uint32_t X)
{
    if (!rp8(pv, n ? PB_ENAM1 : PB_ENAM0) || rp8(pv, n ? PB_RESMP1 : PB_RESMP0)) return 0;
    const uint32_t nusiz = rp8(pv, n ? PB_NUSIZ1 : PB_NUSIZ0);
    const uint32_t len = 1u << ((nusiz >> 4) & 3u);
    return r_copies((1u << len) - 1u, len, rp16(pv, PB_POS + 4u + 2u * n), c_copies[nusiz & 7u], X);
}

// Pixels [x0, x1) of visible line `vis` with the TIA registers as they are:
// Tia::tick's pixel stage (tia.rs:311-346) with compute_pixel (tia.rs:375-403)
// and the object tests (tia.rs:406-507), over a span in which no register
// changes.  Each object is a bit mask over 32 pixels at a time; the
// collision latches are the masks' intersections, and the priority of
// compute_pixel is the order in which the colors are laid down.  Each
// 32-pixel chunk is one framebuffer sector: its pixels go into the sector
// buffer four to a word, and the buffer is written out when the drawing
// moves to another sector (r_seek).
static __device__ __noinline__ RState r_span(RState s, uint8_t* pv, uint8_t* fbp, uint32_t vis, uint32_t x0, uint32_t x1)
{
    const uint32_t ctrlpf = rp8(pv, PB_CTRLPF);
    const uint32_t pfw = (rp8(pv, PB_PF0) >> 4) | (__brev(rp8(pv, PB_PF1)) >> 24 << 4) | (rp8(pv, PB_PF2) << 12);
    const uint32_t pfr = (ctrlpf & 1u) ? __brev(pfw) >> 12 : pfw;    // the right half, reflected or repeated
    const uint64_t line = (uint64_t)pfw | ((uint64_t)pfr << 20);     // bit g = playfield pixels 4g..4g+3
    const bool ben = rp8(pv, rp8(pv, PB_VDELBL) ? PB_ENABL_OLD : PB_ENABL) != 0;
    const uint32_t blen = 1u << ((ctrlpf >> 4) & 3u);
    uint32_t cx = 0;                                                 // bit 2r: 0x80 of CXr, bit 2r+1: 0x40
    for (uint32_t X = x0 & ~31u; X < x1; X += 32u) {
        const uint32_t lo = x0 > X ? x0 - X : 0u, hi = x1 < X + 32u ? x1 - X : 32u;
        const uint32_t in = (hi >= 32u ? 0xFFFFFFFFu : (1u << hi) - 1u) & ~((1u << lo) - 1u);
        const uint32_t pf = r_spread4((uint32_t)(line >> (X >> 2)) & 0xFFu) & in;
        const uint32_t p0 = r_player_mask(pv, 0, X) & in, p1 = r_player_mask(pv, 1, X) & in;
        const uint32_t m0 = r_missile_mask(pv, 0, X) & in, m1 = r_missile_mask(pv, 1, X) & in;
        const uint32_t bl = ben ? r_place((1u << blen) - 1u, blen, rp16(pv, PB_POS + 8u), X) & in : 0u;
        cx |= ((m0 & p1) ? 0x1u : 0u) | ((m0 & p0) ? 0x2u : 0u) | ((m1 & p0) ? 0x4u : 0u) | ((m1 & p1) ? 0x8u : 0u)
            | ((p0 & pf) ? 0x10u : 0u) | ((p0 & bl) ? 0x20u : 0u) | ((p1 & pf) ? 0x40u : 0u) | ((p1 & bl) ? 0x80u : 0u)
            | ((m0 & pf) ? 0x100u : 0u) | ((m0 & bl) ? 0x200u : 0u) | ((m1 & pf) ? 0x400u : 0u) | ((m1 & bl) ? 0x800u : 0u)
            | ((bl & pf) ? 0x1000u : 0u) | ((p0 & p1) ? 0x4000u : 0u) | ((m0 & m1) ? 0x8000u : 0u);
        uint32_t A = p0 | m0, B = p1 | m1, F = pf | bl;
        if ((s.tw & TW_HMOVE) && X == 0u) { A &= ~0xFFu; B &= ~0xFFu; F &= ~0xFFu; }   // HMOVE comb: background
        // compute_pixel's choice as a 2-bit index per pixel, for all 32 at once:
        // 0 background, 1 playfield/ball, 2 player 1, 3 player 0.
        const uint32_t I1 = (ctrlpf & 4u) ? (A | B) & ~F : A | B;    // playfield priority: F wins
        const uint32_t I0 = (ctrlpf & 4u) ? F | A : A | (F & ~B);
        const uint32_t c0 = rp8(pv, PB_COLUP0), c1 = rp8(pv, PB_COLUP1), cbk = rp8(pv, PB_COLUBK);
        const uint32_t cpf = rp8(pv, PB_COLUPF);
        const uint32_t tl = cbk | (((ctrlpf & 2u) ? c0 : cpf) << 8) | (c1 << 16) | (c0 << 24);   // x < 80 (score mode)
        const uint32_t tr = cbk | (((ctrlpf & 2u) ? c1 : cpf) << 8) | (c1 << 16) | (c0 << 24);
        const uint32_t t = vis * (FA_FB_W / 32u) + (X >> 5);            // the chunk is one framebuffer sector
        if (t != s.sc) r_seek(s.sc, pv, fbp, t);
        for (uint32_t q = lo >> 2; q < (hi + 3u) >> 2; q++) {
            const uint32_t x = X + 4u * q;
            // Four pixels' indices as a byte-permute selector, one nibble each.
            const uint32_t sel = r_nib((I0 >> (4u * q)) & 0xFu) | (r_nib((I1 >> (4u * q)) & 0xFu) << 1);
            const uint32_t w = __byte_perm(x < 80u ? tl : tr, 0u, sel);
            const uint32_t wl = lo > 4u * q ? lo - 4u * q : 0u, wh = hi < 4u * q + 4u ? hi - 4u * q : 4u;
            const uint32_t pm = ((1u << wh) - 1u) & ~((1u << wl) - 1u);
            uint32_t* bp = r_sbuf(pv, q);
            if (pm == 0xFu) {
                *bp = w;
            } else {
                const uint32_t bm = r_bytes(pm);
                *bp = (*bp & ~bm) | (w & bm);
            }
        }
    }
    if (cx) {                                                        // collision latches (tia.rs:329-343)
#pragma unroll
        for (uint32_t r = 0; r < 8u; r++) {
            const uint32_t b = (((cx >> (2u * r)) & 1u) ? 0x80u : 0u) | (((cx >> (2u * r + 1u)) & 1u) ? 0x40u : 0u);
            if (b) wp8(pv, PB_CX + r, rp8(pv, PB_CX + r) | b);
        }
    }
    return s;
}

// The pixels of the current line from clock s.rx up to clock `upto`, with
// the registers as they are: pixels are drawn only when something that
// affects them is about to change (a register write, a delayed playfield
// write, a collision read, the end of the line or of the call).
static __device__ __forceinline__ void r_pending(RState& s, uint8_t* pv, uint8_t* fbp, uint32_t upto)
{
    const uint32_t from = s.rx > 68u ? s.rx : 68u;
    s.rx = upto;
    if (upto <= from || (s.tw & 0x200u)) return;
    const uint32_t vis = (s.scanline - (s.vtop & 0xFFFFu)) & 0xFFFFu;
    if (vis < FA_FB_H) s = r_span(s, pv, fbp, vis, from - 68u, upto - 68u);
}

// The framebuffer as the reference would show it now (the pixels up to the
// beam are already drawn): the beam's row as far as drawn, with zeros after,
// and, once after each clear point, zeros in the rows the beam has not reached.
static __device__ __forceinline__ void r_observe(RState& s, uint8_t* pv, uint8_t* fbp)
{
    const uint32_t vis = (s.scanline - (s.vtop & 0xFFFFu)) & 0xFFFFu;
    constexpr uint32_t SPR = FA_FB_W / 32u, NSEC = FA_FB_H * SPR;   // sectors per row, in all
    if (vis < FA_FB_H) {
        r_sec_write(pv, fbp, s.sc);
        r_zero_sectors(fbp, s.sc + 1u, (vis + 1u) * SPR);
        if (s.zr & R_ZPEND) r_zero_sectors(fbp, (vis + 1u) * SPR, NSEC);
    } else if (s.zr & R_ZPEND) {
        r_zero_sectors(fbp, (s.zr & 0xFFu) * SPR, NSEC);
    }
    s.zr &= ~R_ZPEND;
}

// n TIA clocks, exactly as n calls of Tia::tick (tia.rs:271-372), advanced a
// line at a time: between register writes nothing but the pixels, the
// collision latches and the beam changes from one clock to the next (the
// input latches are idempotent, the resizer's candidate is the scanline
// itself, and a delayed playfield write fires on the first clock after it).
static __device__ __forceinline__ void r_advance(RState& s, uint32_t n, uint32_t pins, uint8_t* pv, uint8_t* fbp)
{
    if (n == 0) return;
    const uint32_t dlen = rp8(pv, RB_DLEN);
    if (dlen) {                                                      // every pending write has one clock left
        r_pending(s, pv, fbp, s.clock);
        for (uint32_t i = 0; i < dlen; i++) {
            const uint32_t reg = rp8(pv, RB_DQ + 3u * i + 1u), val = rp8(pv, RB_DQ + 3u * i + 2u);
            wp8(pv, reg == 0x0Du ? PB_PF0 : reg == 0x0Eu ? PB_PF1 : PB_PF2, val);
        }
        wp8(pv, RB_DLEN, 0u);
    }
    if (s.tw & TW_LATCH) {
        if (!(pins & 0x10000u)) s.tw &= ~TW_L4;
        if (!(pins & 0x20000u)) s.tw &= ~TW_L5;
    }
    while (n) {
        if (!(s.tw & 0x200u) && s.scanline >= 23u && s.scanline < (s.vtop >> 16))
            s.vtop = (s.vtop & 0xFFFFu) | (s.scanline << 16);
        const uint32_t seg = n < 228u - s.clock ? n : 228u - s.clock;
        s.clock += seg;
        n -= seg;
        if (s.clock >= 228u) {
            r_pending(s, pv, fbp, 228u);
            const uint32_t vis = (s.scanline - (s.vtop & 0xFFFFu)) & 0xFFFFu;
            if (vis < FA_FB_H) {                                     // the row is complete: written whole
                r_seek(s.sc, pv, fbp, (vis + 1u) * (FA_FB_W / 32u));
                s.zr = (s.zr & R_ZPEND) | (vis + 1u);
            }
            s.clock = 0;
            s.rx = 0;
            s.scanline = (s.scanline + 1u) & 0xFFFFu;
            s.tw &= ~(TW_WSYNC | TW_HMOVE);
            if (s.scanline == (s.vtop & 0xFFFFu)) {                  // framebuffer cleared (tia.rs:349-351)
                s.sc = 0;
                r_sec_clear(pv);
                s.zr = R_ZPEND;
            }
            if (!(s.tw & TW_PDUMP) && s.pcnt < 256u) s.pcnt++;
            if (s.scanline >= 262u) { s.scanline = 0; s.tw |= TW_FCOMP; }
        }
    }
}

// The pending pixels of the current line, up to the beam, then the
// framebuffer as it can be seen now.
static __device__ __noinline__ RState render_observe(RState s, uint8_t* pv, uint8_t* fbp)
{
    r_pending(s, pv, fbp, s.clock);
    r_observe(s, pv, fbp);
    return s;
}

static __device__ __forceinline__ void r_pia_tick(RState& s)     // pia.rs:80-103
{
    if (s.tv == 0 && s.uf) { s.tv = 0xFFu; return; }
    s.ps = (s.ps - 1u) & 0xFFFFu;
    if (s.ps == 0) {
        s.ps = s.uf ? 1u : s.sel;
        if (s.tv == 0) { s.uf = 1; s.tv = 0xFFu; } else s.tv -= 1u;
    }
}

// m calls of Pia::tick (pia.rs:80-103), a prescaler period at a time.
static __device__ __forceinline__ void r_pia_ticks(RState& s, uint32_t m)
{
    while (m) {
        if (s.ps == 0 || (s.uf && s.tv == 0)) { r_pia_tick(s); m--; continue; }
        if (s.uf && s.ps == 1u) { s.tv = (s.tv - m) & 0xFFu; return; }   // after underflow: one count per tick
        if (m < s.ps) { s.ps -= m; return; }
        m -= s.ps;                                                   // the tick that empties the prescaler
        s.ps = s.uf ? 1u : s.sel;
        if (s.tv == 0) { s.uf = 1; s.tv = 0xFFu; } else s.tv -= 1u;
    }
}

// n CPU cycles of the rendering console: three TIA clocks and one PIA clock
// each (the TIA and the PIA do not interact, so each is advanced in bulk).
static __device__ __noinline__ RState render_cycles(RState s, uint32_t n, uint32_t pins, uint8_t* pv, uint8_t* fbp)
{
    r_advance(s, 3u * n, pins, pv, fbp);
    r_pia_ticks(s, n);
    return s;
}

// n TIA clocks alone (the clocks around a PIA write, src/atari.rs:207-222).
static __device__ __noinline__ RState render_tia_ticks(RState s, uint32_t n, uint32_t pins, uint8_t* pv, uint8_t* fbp)
{
    r_advance(s, n, pins, pv, fbp);
    return s;
}

static __device__ __forceinline__ uint32_t r_resp_player(uint32_t clk)       // tia.rs:512-520
{
    const uint32_t dc = (clk + (clk < 68u ? 3u : 4u) + 156u) % 228u;
    return dc >= 68u ? dc - 68u : dc + 160u - 68u;
}

static __device__ __forceinline__ void r_resize_commit(RState& s, uint8_t* pv)  // tia.rs:247-268
{
    const uint32_t vbt = s.vtop >> 16, top = s.vtop & 0xFFFFu;
    if (vbt > 262u) return;
    const uint32_t clamped = vbt < 23u ? 23u : vbt > 32u ? 32u : vbt;
    const uint32_t cand = clamped < top ? clamped : top;
    uint32_t ntop = top;
    const uint32_t ptop = rp16(pv, RB_PTOP), pfr = rp8(pv, RB_PFRAMES);
    if (cand != ptop) { wp16(pv, RB_PTOP, cand); wp8(pv, RB_PFRAMES, 3u); }
    else if (pfr > 0) { wp8(pv, RB_PFRAMES, pfr - 1u); if (pfr == 1u) ntop = ptop; }
    s.vtop = ntop | (ntop << 16);
}

// Tia::write (tia.rs:570-674) of register a & 0x3F.
// Registers whose write can change a pixel or a collision latch from the
// next clock on: VSYNC, VBLANK, NUSIZx-REFPx, RESPx-RESBL, GRPx-ENABL,
// VDELx-RESMPx, HMOVE and CXCLR.  The playfield registers reach the pixels
// through the delayed-write queue (flushed when it fires); WSYNC, RSYNC,
// audio, HMxx and HMCLR never do.
constexpr uint64_t R_PIXEL_REGS = 0x17E0F81F1FF3ull;

static __device__ __forceinline__ void r_write(uint32_t a, uint32_t v, RState& s, uint8_t* pv, uint8_t* fbp)
{
    if ((R_PIXEL_REGS >> (a & 0x3Fu)) & 1u) r_pending(s, pv, fbp, s.clock);   // the pixels drawn before the write
    switch (a & 0x3Fu) {
    case 0x00:
        if (!(s.tw & 2u) && (v & 2u)) { r_observe(s, pv, fbp); r_resize_commit(s, pv); s.scanline = 0; s.tw |= TW_FCOMP; }
        s.tw = (s.tw & ~0xFFu) | v;
        break;
    case 0x01:
        if (v & 0x40u) s.tw |= TW_LATCH | TW_L4 | TW_L5;
        else s.tw &= ~TW_LATCH;
        if (v & 0x80u) { s.pcnt = 0; s.tw |= TW_PDUMP; }
        else s.tw &= ~TW_PDUMP;
        s.tw = (s.tw & ~0xFF00u) | (v << 8);
        break;
    case 0x02: s.tw |= TW_WSYNC; break;
    case 0x04: wp8(pv, PB_NUSIZ0, v); break;
    case 0x05: wp8(pv, PB_NUSIZ1, v); break;
    case 0x06: wp8(pv, PB_COLUP0, v); break;
    case 0x07: wp8(pv, PB_COLUP1, v); break;
    case 0x08: wp8(pv, PB_COLUPF, v); break;
    case 0x09: wp8(pv, PB_COLUBK, v); break;
    case 0x0A: wp8(pv, PB_CTRLPF, v); break;
    case 0x0B: wp8(pv, PB_REFP0, (v & 8u) ? 1u : 0u); break;
    case 0x0C: wp8(pv, PB_REFP1, (v & 8u) ? 1u : 0u); break;
    case 0x0D: case 0x0E: case 0x0F: {                              // written after one TIA clock
        const uint32_t n = rp8(pv, RB_DLEN);
        if (n < 4u) {
            wp8(pv, RB_DQ + 3u * n, 1u);
            wp8(pv, RB_DQ + 3u * n + 1u, a & 0x3Fu);
            wp8(pv, RB_DQ + 3u * n + 2u, v);
            wp8(pv, RB_DLEN, n + 1u);
        } else {                                                    // queue full: written now
            r_pending(s, pv, fbp, s.clock);
            wp8(pv, (a & 0x3Fu) == 0x0Du ? PB_PF0 : (a & 0x3Fu) == 0x0Eu ? PB_PF1 : PB_PF2, v);
        }
        break;
    }
    case 0x10: wp16(pv, PB_POS + 0u, r_resp_player(s.clock)); break;
    case 0x11: wp16(pv, PB_POS + 2u, r_resp_player(s.clock)); break;
    case 0x12: wp16(pv, PB_POS + 4u, mod160((int)s.clock - 68 + 5)); break;
    case 0x13: wp16(pv, PB_POS + 6u, mod160((int)s.clock - 68 + 5)); break;
    case 0x14: wp16(pv, PB_POS + 8u, mod160((int)s.clock - 68 + 5)); break;
    case 0x1B: wp8(pv, PB_GRP0_OLD, rp8(pv, PB_GRP0)); wp8(pv, PB_GRP0, v); break;
    case 0x1C: wp8(pv, PB_GRP1_OLD, rp8(pv, PB_GRP1)); wp8(pv, PB_GRP1, v); wp8(pv, PB_ENABL_OLD, rp8(pv, PB_ENABL)); break;
    case 0x1D: wp8(pv, PB_ENAM0, (v & 2u) ? 1u : 0u); break;
    case 0x1E: wp8(pv, PB_ENAM1, (v & 2u) ? 1u : 0u); break;
    case 0x1F: wp8(pv, PB_ENABL, (v & 2u) ? 1u : 0u); break;
    case 0x20: case 0x21: case 0x22: case 0x23: case 0x24: wp8(pv, PB_HM + ((a & 0x3Fu) - 0x20u), v); break;
    case 0x25: wp8(pv, PB_VDELP0, v & 1u); break;
    case 0x26: wp8(pv, PB_VDELP1, v & 1u); break;
    case 0x27: wp8(pv, PB_VDELBL, v & 1u); break;
    case 0x28: wp8(pv, PB_RESMP0, (v & 2u) ? 1u : 0u); break;
    case 0x29: wp8(pv, PB_RESMP1, (v & 2u) ? 1u : 0u); break;
    case 0x2A:                                                      // HMOVE
        for (uint32_t o = 0; o < 5u; o++) {
            const int hm = (int)(int8_t)(uint8_t)rp8(pv, PB_HM + o) >> 4;
            wp16(pv, PB_POS + 2u * o, mod160((int)rp16(pv, PB_POS + 2u * o) - hm));
        }
        s.tw |= TW_HMOVE;
        break;
    case 0x2B: for (uint32_t o = 0; o < 5u; o++) wp8(pv, PB_HM + o, 0u); break;
    case 0x2C: for (uint32_t o = 0; o < 8u; o++) wp8(pv, PB_CX + o, 0u); break;
    default: break;                                                 // RSYNC, audio
    }
}

// `owed` whole CPU cycles, then Bus::write of a TIA register
// (src/atari.rs:207-222): two TIA clocks, the write, one TIA clock and the
// PIA clock.  One call per write: the cycles before it ride along.
static __device__ __noinline__ RState render_write_cycle(uint32_t a, uint32_t v, uint32_t owed, RState s, uint32_t pins,
                                                         uint8_t* pv, uint8_t* fbp)
{
    if (owed) {
        r_advance(s, 3u * owed, pins, pv, fbp);
        r_pia_ticks(s, owed);
    }
    r_advance(s, 2u, pins, pv, fbp);
    r_write(a, v, s, pv, fbp);
    r_advance(s, 1u, pins, pv, fbp);
    r_pia_tick(s);
    return s;
}

// Tia::read (tia.rs:533-566) or Pia::read of an I/O register (pia.rs:169-199);
// .y = 1 when the read clears the timer's underflow flag (INTIM).
static __device__ __forceinline__ uint2 r_read_value(uint32_t a, const RState& s, uint32_t pins, uint32_t pads,
                                                     uint32_t ports, const uint8_t* pv)
{
    if ((a & 0x1080u) == 0) {
        const uint32_t r = a & 0x0Fu;
        if (r < 8u) return make_uint2(rp8(pv, PB_CX + r), 0u);
        switch (r) {
        case 0x8: return make_uint2(s.pcnt >= (pads & 0xFFu) ? 0x80u : 0u, 0u);
        case 0x9: return make_uint2(s.pcnt >= ((pads >> 8) & 0xFFu) ? 0x80u : 0u, 0u);
        case 0xA: case 0xB: return make_uint2(0x80u, 0u);
        case 0xC: return make_uint2((s.tw & TW_LATCH) ? ((s.tw & TW_L4) ? 0x80u : 0u) : ((pins & 0x10000u) ? 0x80u : 0u), 0u);
        case 0xD: return make_uint2((s.tw & TW_LATCH) ? ((s.tw & TW_L5) ? 0x80u : 0u) : ((pins & 0x20000u) ? 0x80u : 0u), 0u);
        default: return make_uint2(0u, 0u);
        }
    }
    switch (a & 7u) {
    case 0: { const uint32_t ddr = (ports >> 8) & 0xFFu; return make_uint2(((pins & 0xFFu) & ~ddr) | (ports & ddr & 0xFFu), 0u); }
    case 1: return make_uint2((ports >> 8) & 0xFFu, 0u);
    case 2: { const uint32_t ddr = ports >> 24; return make_uint2((((pins >> 8) & 0xFFu) & ~ddr) | ((ports >> 16) & ddr & 0xFFu), 0u); }
    case 3: return make_uint2(ports >> 24, 0u);
    case 4: return make_uint2(s.tv & 0xFFu, 1u);
    case 5: return make_uint2(s.uf ? 0x80u : 0u, 0u);
    default: return make_uint2(0u, 0u);
    }
}

struct RRead {
    RState s;
    uint32_t v;
};

// `owed` whole CPU cycles, then the read of a TIA or PIA register in its own
// cycle (Bus::read, src/atari.rs:195-205): collisions drawn up to the beam,
// the value, then three TIA clocks and the PIA clock.  One call per read.
static __device__ __noinline__ RRead render_io_read(uint32_t a, uint32_t owed, RState s, uint32_t pins, uint32_t pads,
                                                    uint32_t ports, uint8_t* pv, uint8_t* fbp)
{
    if (owed) {
        r_advance(s, 3u * owed, pins, pv, fbp);
        r_pia_ticks(s, owed);
    }
    if ((a & 0x1080u) == 0 && (a & 0x0Fu) < 8u) r_pending(s, pv, fbp, s.clock);   // collisions so far
    const uint2 r = r_read_value(a, s, pins, pads, ports, pv);
    if (r.y) s.uf = 0;                                               // INTIM read clears the flag
    r_advance(s, 3u, pins, pv, fbp);
    r_pia_tick(s);
    RRead out;
    out.s = s;
    out.v = r.x;
    return out;
}

// ---------------------------------------------------------------- DPC (Pitfall II)
// The DPC chip of FA_SCHEME_DPC carts (no counterpart in the reference),
// with the semantics the oracle's DPC section fixes: 8 data fetchers (11-bit
// counter, top, bottom, flag), an 8-bit random number generator and 3 music
// channels clocked at 20 kHz of Cpu::cycles.  The registers stay in their
// HBM rows (R_DPC_*) and are changed there in place, one access at a time:
// a read of $1000-$103F (wr 0; returns the value) or a write of v to
// $1040-$107F (wr 1).  cyc_acc: the instruction cycles not yet added to the
// rows' Cpu::cycles (none of the accessing instruction's).  `disp` is the
// 2K of display data.  One out-of-line copy for every access site.
static __device__ __forceinline__ uint32_t dpc_byte(uint32_t w, uint32_t k) { return (w >> ((k & 3u) * 8u)) & 0xFFu; }

static __device__ __noinline__ uint32_t dpc_io(uint32_t a, uint32_t v, uint32_t wr, uint32_t* col, uint32_t S,
                                               const uint8_t* disp, uint32_t cyc_acc)
{
    const uint32_t misc = col[(size_t)R_DPC_MISC * S];
    uint32_t flags = misc & 0xFFu, music = (misc >> 8) & 7u, rnd = (misc >> 16) & 0xFFu;
    // The music channels up to the instruction's start: one clock of the
    // oscillator counts a channel's low byte down, the clock after 0 reloads
    // top; the flag is set while the low byte is above bottom.
    const unsigned long long t =
        (((unsigned long long)col[(size_t)R_CYC_HI * S] << 32) | col[(size_t)R_CYC_LO * S]) + cyc_acc;
    const uint32_t now = (uint32_t)((t / 3579545ull) * 60000ull + ((t % 3579545ull) * 60000ull) / 3579545ull);
    const uint32_t clocks = now - col[(size_t)R_DPC_OSC * S];
    col[(size_t)R_DPC_OSC * S] = now;
    if (clocks && music) {
#pragma unroll 1
        for (uint32_t f = 5u; f < 8u; f++) {
            if (!((music >> (f - 5u)) & 1u)) continue;
            uint32_t& cw = col[(size_t)(R_DPC_CNT + (f >> 1)) * S];
            const uint32_t sh = (f & 1u) * 16u, cnt = (cw >> sh) & 0x7FFu;
            const uint32_t top = dpc_byte(col[(size_t)(R_DPC_TOP + (f >> 2)) * S], f);
            const uint32_t bot = dpc_byte(col[(size_t)(R_DPC_BOT + (f >> 2)) * S], f);
            uint32_t low = cnt & 0xFFu;
            low = clocks <= low ? low - clocks : top - (clocks - low - 1u) % (top + 1u);
            cw = (cw & ~(0xFFFFu << sh)) | (((cnt & 0x700u) | low) << sh);
            flags = low > bot ? flags | (1u << f) : flags & ~(1u << f);
        }
    }
    const uint32_t k = a & 7u, f = (a >> 3) & 7u, sh = (k & 1u) * 16u;
    uint32_t& cw = col[(size_t)(R_DPC_CNT + (k >> 1)) * S];
    uint32_t& tw = col[(size_t)(R_DPC_TOP + (k >> 2)) * S];
    uint32_t& bw = col[(size_t)(R_DPC_BOT + (k >> 2)) * S];
    uint32_t cnt = (cw >> sh) & 0x7FFu, out = 0u;
    if (!wr) {
        const bool mus = k >= 5u && ((music >> (k - 5u)) & 1u);
        // The generator shifts left, taking in the XNOR of bits 7, 5, 4, 3.
        rnd = ((rnd << 1) | (~((rnd >> 7) ^ (rnd >> 5) ^ (rnd >> 4) ^ (rnd >> 3)) & 1u)) & 0xFFu;
        if (!mus) {
            const uint32_t low = cnt & 0xFFu;
            if (low == dpc_byte(tw, k)) flags |= 1u << k;
            else if (low == dpc_byte(bw, k)) flags &= ~(1u << k);
        }
        const uint32_t flag = ((flags >> k) & 1u) ? 0xFFu : 0u, data = disp[2047u - cnt];
        switch (f) {
        case 0:
            if (k < 4u) out = rnd;
            else
                for (uint32_t m = 0; m < 3u; m++) out += (((music & (flags >> 5)) >> m) & 1u) ? 4u + m : 0u;
            break;
        case 1: out = data; break;
        case 2: out = data & flag; break;
        case 7: out = flag; break;
        default: break;
        }
        if (!mus) cw = (cw & ~(0xFFFFu << sh)) | (((cnt - 1u) & 0x7FFu) << sh);
    } else {
        const uint32_t bs = (k & 3u) * 8u;
        switch (f) {
        case 0: tw = (tw & ~(0xFFu << bs)) | (v << bs); flags &= ~(1u << k); break;
        case 1: bw = (bw & ~(0xFFu << bs)) | (v << bs); break;
        case 2: cw = (cw & ~(0xFFFFu << sh)) | (((cnt & 0x700u) | v) << sh); break;
        case 3:
            cw = (cw & ~(0xFFFFu << sh)) | ((((v & 7u) << 8) | (cnt & 0xFFu)) << sh);
            if (k >= 5u) music = (music & ~(1u << (k - 5u))) | (((v >> 4) & 1u) << (k - 5u));
            break;
        case 6: rnd = 1u; break;
        default: break;
        }
    }
    col[(size_t)R_DPC_MISC * S] = flags | (music << 8) | (rnd << 16);
    return out;
}

// ---------------------------------------------------------------- PIA timer (pia.rs:107-166)
// Pia::tick_n on the unpacked timer: value, prescaler, interval, underflow.
static __device__ __forceinline__ void pia_tick_n(uint32_t& tv, uint32_t& ps, uint32_t sel, uint32_t& uf, uint32_t n)
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

// Headless timer bookkeeping (Emu::pia_count).  The window of a timer state
// is the run of cycles over which tick_n only counts.  With tv >= 1 it ends
// at the decrement that brings tv to zero: ps (a prescaler of 0, just after
// an underflow, counts as a whole interval: tick_n then decrements after sel
// cycles) plus tv - 1 intervals.  With tv = 0, no underflow flag and a
// prescaler left, it ends when the prescaler runs out (that decrement
// underflows).  Any other state, an interval that is not one of 1, 8, 64,
// 1024, or a prescaler above the interval (states only an upload makes)
// have no window: 0, every call exact.
static __device__ __forceinline__ uint32_t pia_span_of(uint32_t tv, uint32_t ps, uint32_t sel, uint32_t uf)
{
    if (sel == 0u || (sel & (sel - 1u)) != 0u || sel > 1024u || ps > sel) return 0u;
    if (tv == 0u) return uf ? 0u : ps;
    return (ps ? ps : sel) + ((tv - 1u) << (__ffs(sel) - 1u));
}
// (tv, ps) with the counted cycles (the window less tlim) applied: fewer
// cycles than the window, so tick_n's counting branches alone apply.
static __device__ __forceinline__ uint2 pia_now_of(uint32_t tv, uint32_t ps, uint32_t sel, uint32_t uf, uint32_t tlim)
{
    const uint32_t e = pia_span_of(tv, ps, sel, uf) - tlim;
    if (e == 0u) return make_uint2(tv, ps);
    const uint32_t p0 = ps ? ps : sel;
    if (e < p0) return make_uint2(tv, p0 - e);
    const uint32_t k = e - p0;
    return make_uint2(tv - 1u - (k >> (__ffs(sel) - 1u)), sel - (k & (sel - 1u)));
}
// An INTIM read (pia.rs:187-190): the counted cycles settled, the underflow
// flag cleared (tv = 0 with a prescaler left may gain a window by it).
// Packed (tv | ps << 16, sel | uf << 16, tlim); the value read is tv & 0xFF.
static __device__ __noinline__ uint4 pia_intim_io(uint32_t tv_ps, uint32_t sel_uf, uint32_t tlim)
{
    const uint32_t sel = sel_uf & 0xFFFFu;
    const uint2 t = pia_now_of(tv_ps & 0xFFFFu, tv_ps >> 16, sel, sel_uf >> 16, tlim);
    return make_uint4(t.x | (t.y << 16), sel, pia_span_of(t.x, t.y, sel, 0u), 0u);
}
// Pia::write of an I/O register by the headless core (src/pia.rs:202-228):
// (ports, tv | ps << 16, sel | uf << 16, tlim) after it.  A port write
// leaves the timer and its counting alone; a timer write replaces value,
// prescaler, interval and flag, so the cycles counted so far no longer
// matter.
static __device__ __noinline__ uint4 pia_store_io(uint32_t a, uint32_t v, uint32_t ports, uint32_t tp, uint32_t su,
                                                  uint32_t tlim)
{
    if (a & 0x10u) {
        const uint32_t sel = 1u << ((0xA630u >> (4u * (a & 3u))) & 0xFu);   // 1, 8, 64, 1024
        return make_uint4(ports, v | (sel << 16), sel, pia_span_of(v, sel, sel, 0u));
    }
    const uint32_t sh = 8u * (a & 3u);                                 // pa_out pa_ddr pb_out pb_ddr
    return make_uint4((ports & ~(0xFFu << sh)) | (v << sh), tp, su, tlim);
}
// Packed (tv | ps << 16, sel | uf << 16, tlim) after settling and one exact
// call of n cycles.
static __device__ __noinline__ uint4 pia_sync_io(uint32_t tv_ps, uint32_t sel_uf, uint32_t tlim, uint32_t n)
{
    const uint32_t sel = sel_uf & 0xFFFFu;
    uint32_t uf = sel_uf >> 16;
    const uint2 t = pia_now_of(tv_ps & 0xFFFFu, tv_ps >> 16, sel, uf, tlim);
    uint32_t tv = t.x, ps = t.y;
    pia_tick_n(tv, ps, sel, uf, n);
    return make_uint4(tv | (ps << 16), sel | (uf << 16), pia_span_of(tv, ps, sel, uf), 0u);
}

// SLICED: the core of E0 and 3F carts (with DPC, of DPC carts alone; with
// FE, of FE carts alone).  The DPC and FE cores are their own builds so that
// the E0 / 3F core carries none of their bus decode.  The FE core issues
// every bus access the reference CPU makes, phantom ones included: any of
// them can select an FE cart's bank.
template <int BLOCK, bool RENDER = false, bool SLICED = false, bool DPC = false, bool FE = false>
struct Emu {
    static_assert(!DPC || (SLICED && !RENDER), "the DPC core is a headless sliced core");
    static_assert(!FE || (SLICED && !RENDER && !DPC), "the FE core is a headless sliced core");
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
    uint32_t slices;         // SLICED (E0, 3F carts): the 1K ROM slice of window k in byte k
    uint32_t cyc_acc;         // instruction cycles not yet added to Cpu::cycles in HBM
    // ---- PIA (src/pia.rs:26-44): timer unpacked, ports and input pins packed
    //      (touched only by I/O accesses)
    uint32_t tp;             // timer value | prescaler << 16 (the R_TIMER row word)
    uint32_t su;             // interval (1, 8, 64, 1024) | underflow flag << 16
    uint32_t tlim;           // headless: cycles the timer may still count before an exact tick
                             // (tp lags by pia_span() - tlim counted cycles; see pia_count)
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
    // Sliced carts.  The ROM byte at a (A12 set): window (a >> 10) & 3 holds
    // slice `slices` byte k.
    __device__ __forceinline__ uint32_t srom(uint32_t a) const
    {
        return (((slices >> ((a >> 7) & 0x18u)) & 0x1Fu) << 10) | (a & 0x3FFu);
    }
    __device__ __forceinline__ void sbump() { bank = bank < (511u << 3) ? bank + 8u : bank; }
    // E0: any access to $1FE0-$1FF7 maps slice (a & 7) into window (a - $1FE0) >> 3.
    // DPC core: any access to $1FF8 / $1FF9 maps program bank 0 / 1 (slices 4b..4b+3).
    __device__ __forceinline__ void e0_hot(uint32_t a13)
    {
        if constexpr (DPC) {
            if ((a13 | 1u) == 0x1FF9u) {
                slices = (a13 & 1u) * 0x04040404u + 0x03020100u;
                sbump();
            }
        } else {
            const uint32_t d = a13 - 0x1FE0u;
            if (d < 24u && fa_map_kind(hot_lo) == FA_MAP_E0) {
                const uint32_t sh = (d >> 3) * 8u;
                slices = (slices & ~(0xFFu << sh)) | ((a13 & 7u) << sh);
                sbump();
            }
        }
    }
    // The bank state (fa_state::mapper) to and from `slices`, for this core's
    // schemes only (fa_slices_from_mapper / fa_mapper_from_slices decode all
    // of them; a core carries only its own).
    __device__ __forceinline__ uint32_t slices_of(uint32_t m) const
    {
        if constexpr (DPC || FE) return fa_slices_4k_bank(m, FE);
        else return fa_slices_e0_3f(hot_lo, m);
    }
    __device__ __forceinline__ uint32_t mapper_of(uint32_t s) const
    {
        if constexpr (DPC || FE) return fa_mapper_4k_bank(s, FE);
        else return fa_mapper_e0_3f(hot_lo, s);
    }
    // FE core: the access after one to $01FE selects the 4K bank by bit 5 of
    // its data (set: bank 0, clear: bank 1); bit 7 of `slices` marks that the
    // last access was to $01FE.  v is the byte the access read or wrote.
    __device__ __forceinline__ void fe_note(uint32_t a13, uint32_t v)
    {
        if (slices & 0x80u) {
            slices = ((v & 0x20u) ? 0u : 0x04040404u) + 0x03020100u;
            sbump();
        }
        if (a13 == 0x01FEu) slices |= 0x80u;
    }
    // DPC core: reads of $1000-$103F and writes of $1040-$107F reach the registers.
    __device__ __forceinline__ uint32_t dpc(uint32_t a13, uint32_t v, uint32_t wr)
    {
        return dpc_io(a13, v, wr, column(), G->stride, rom + 8192u, cyc_acc);
    }
    // 3F: a write of v to $0000-$003F maps 2K bank v mod n at $1000-$17FF.
    __device__ __forceinline__ void f3_write(uint32_t a13, uint32_t v)
    {
        if (a13 < 0x40u && fa_map_kind(hot_lo) == FA_MAP_3F) {
            const uint32_t b = v % (hot_lo & 0xFFu);
            slices = (slices & 0xFFFF0000u) | (2u * b) | ((2u * b + 1u) << 8);
            sbump();
        }
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
        uint32_t tv = tp & 0xFFFFu, ps = tp >> 16, uf = su >> 16;
        pia_tick_n(tv, ps, su & 0xFFFFu, uf, n);
        tp = tv | (ps << 16);
        su = (su & 0xFFFFu) | (uf << 16);
    }

    // Headless consoles tick the timer once per instruction, with the
    // instruction's cycles (atari.rs:497-552).  Until a call makes the
    // decrement that brings the value to zero, or is made with the value at
    // zero, Pia::tick_n only counts, and consecutive calls add up: tick_n(a)
    // then tick_n(b) leaves what tick_n(a + b) leaves.  So an instruction
    // only takes its cycles off tlim, the cycles left before such a call;
    // the call that reaches it runs exactly through pia_tick, and the
    // counted cycles are folded into tp (pia_settle) before INTIM is
    // read, a PIA register is written or the state is stored.
    __device__ __forceinline__ uint32_t pia_span() const { return pia_span_of(tp & 0xFFFFu, tp >> 16, su & 0xFFFFu, su >> 16); }
    __device__ __forceinline__ uint2 pia_now() const { return pia_now_of(tp & 0xFFFFu, tp >> 16, su & 0xFFFFu, su >> 16, tlim); }
    // Fold the counted cycles in, run one exact call of n cycles (none for
    // n = 0), and open the next window: one out-of-line copy.
    __device__ __forceinline__ void pia_sync(uint32_t n)
    {
        const uint4 r = pia_sync_io(tp, su, tlim, n);
        tp = r.x;
        su = r.y;
        tlim = r.z;
    }
    __device__ __forceinline__ void pia_settle() { pia_sync(0u); }
    // An INTIM read: the counted cycles settled, the underflow flag cleared.
    __device__ __forceinline__ void pia_intim()
    {
        const uint4 r = pia_intim_io(tp, su, tlim);
        tp = r.x; su = r.y; tlim = r.z;
    }
    __device__ __forceinline__ void pia_count(uint32_t n)
    {
        if (n < tlim) { tlim -= n; return; }
        // The call reaches the end of the window.  tick_n then underflows: uf
        // set, prescaler 0, and the o cycles past the window counted one per
        // cycle from $FF ($FF itself when o is 0).  That holds whatever the
        // state at the call when o > 0.  When o is 0 it needs a window that
        // began at tv = 0, or tv >= 2 at the call (with tv 1 and a prescaler
        // left, the call only empties the prescaler), which tlim > sel
        // guarantees.  Anything else runs exactly.
        const uint32_t sel = su & 0xFFFFu;
        if (tlim != 0u && (n > tlim || tlim > sel || (tp & 0xFFFFu) == 0u)) {
            const uint32_t o = n - tlim;
            const uint32_t tv = o ? (0u - o) & 0xFFu : 0xFFu;
            tp = tv;
            su = sel | 0x10000u;
            tlim = tv << (__ffs(sel) - 1u);
            return;
        }
        pia_sync(n);
    }

    // ------------------------------------------------------------ bus
    // Every access carries j, its cycle within the instruction: the
    // reference's CPU makes exactly one bus access per cycle (src/cpu.rs).
    // The headless console (atari.rs:497-552) ignores j: it ticks the TIA and
    // PIA once per instruction, after it.  The rendering console (RENDER,
    // atari.rs:195-222) ticks them up to cycle j before any access that
    // reaches a TIA or PIA register, whose state depends on the beam, and
    // gives writes the Bus's timing (two TIA clocks, the write, one TIA clock
    // and the PIA clock); accesses to ROM and RAM do not depend on the beam
    // and are ticked with the rest of the instruction.
    // Headless: ROM, RAM and hotspots are handled inline; TIA and PIA
    // registers go through one out-of-line copy of their decoders (io_read /
    // tia_write_io / pia_write_io), which keeps the interpreter's code small
    // enough to stay resident in the instruction cache.
    __device__ __forceinline__ uint32_t io(uint32_t a, uint32_t j)   // TIA or PIA register read
    {
        if constexpr (RENDER) {
            const uint32_t d = j - done;                              // cycles owed before this one
            const RRead r = render_io_read(a, (int32_t)d > 0 ? d : 0u, rpack(), pins, pads, ports, pv, fbp);
            runpack(r.s);
            done = j + 1u;
            return r.v;
        } else {
            if ((a & 0x87u) == 0x84u) {                             // INTIM: settles and clears the flag
                pia_intim();
                return tp & 0xFFu;
            }
            return io_read(a, pcnt, pins, pads, ports, su, (const uint8_t*)column(), G->stride * 4u);
        }
    }
    __device__ __forceinline__ void io_write(uint32_t a, uint32_t v, uint32_t j)  // TIA or PIA register write
    {
        if constexpr (SLICED) f3_write(a, v);                       // the write still reaches the TIA
        if constexpr (RENDER) {
            if ((a & 0x1080u) != 0) {                                 // PIA register: rare, the general path
                rsync(j);
                r_write_cycle(a, v);
            } else {
                const uint32_t d = j - done;
                runpack(render_write_cycle(a, v, (int32_t)d > 0 ? d : 0u, rpack(), pins, pv, fbp));
            }
            done = j + 1u;
        } else if (a & 0x200u) {
            const uint4 r = pia_store_io(a, v, ports, tp, su, tlim);
            ports = r.x; tp = r.y; su = r.z; tlim = r.w;
        } else {
            uint2 r = tia_write_io(a, v, clock, tw, scanline | (pcnt << 16), (uint8_t*)column(), G->stride * 4u);
            tw = r.x; scanline = r.y & 0xFFFFu; pcnt = r.y >> 16;
        }
    }
    __device__ __forceinline__ uint32_t read_low(uint32_t a, uint32_t j)   // a < 0x1000
    {
        if ((a & 0x80u) && (a & 0x280u) != 0x280u) {                // RAM and its mirrors
            if constexpr (RENDER) return ldp(a & 0x7Fu);           // the rendering bus reads PIA RAM at every mirror
            else return a < 0x200u ? ldp(a & 0x7Fu) : 0u;           // other mirrors read the never-written flat array
        }
        return io(a, j);
    }
    __device__ __forceinline__ uint32_t read(uint32_t addr, uint32_t j)
    {
        uint32_t a = addr & 0x1FFFu;
        if (a & 0x1000u) {
            if constexpr (SLICED) {
                if constexpr (DPC) {
                    if (a < 0x1040u) return dpc(a, 0u, 0u);
                }
                e0_hot(a);
                if constexpr (FE) {
                    const uint32_t v = rom[srom(a)];
                    fe_note(a, v);
                    return v;
                }
                return rom[srom(a)];
            } else {
                bsw(a);
                return rom[((bank & 7u) << 12) | (a & 0xFFFu)];
            }
        }
        if constexpr (FE) {
            const uint32_t v = read_low(a, j);
            fe_note(a, v);
            return v;
        }
        return read_low(a, j);
    }
    __device__ __forceinline__ void write(uint32_t addr, uint32_t v, uint32_t j)
    {
        uint32_t a = addr & 0x1FFFu;
        if constexpr (FE) fe_note(a, v);
        if (a & 0x1000u) {
            if constexpr (SLICED) {
                if constexpr (DPC) {
                    if (a - 0x1040u < 0x40u) (void)dpc(a, v, 1u);
                }
                e0_hot(a);
            } else {
                bsw(a);
            }
            return;
        }
        if ((a & 0x280u) == 0x080u) { stp(a & 0x7Fu, v); return; }
        io_write(a, v, j);
    }
    // A phantom read: only its side effects (hotspot, INTIM) matter; in the FE
    // core its value too.
    __device__ __forceinline__ void dummy(uint32_t addr, uint32_t j)
    {
        if constexpr (FE) {
            (void)read(addr, j);
            return;
        }
        uint32_t a = addr & 0x1FFFu;
        if (a & 0x1000u) {
            if constexpr (SLICED) {
                if constexpr (DPC) {
                    if (a < 0x1040u) (void)dpc(a, 0u, 0u);
                }
                e0_hot(a);
            } else {
                bsw(a);
            }
        } else if ((a & 0x287u) == 0x284u) {
            if constexpr (RENDER) (void)io(a, j);
            else pia_intim();
        }
    }
    __device__ __forceinline__ uint32_t zp_read(uint32_t z, uint32_t j)
    {
        if constexpr (FE) {
            const uint32_t v = (z & 0x80u) ? ldp(z & 0x7Fu) : io(z, j);
            fe_note(z, v);
            return v;
        }
        return (z & 0x80u) ? ldp(z & 0x7Fu) : io(z, j);
    }
    __device__ __forceinline__ void push(uint32_t v, uint32_t j)
    {
        if constexpr (FE) fe_note(0x100u | sp, v);
        if (sp & 0x80u) stp(sp & 0x7Fu, v); else io_write(0x100u | sp, v, j);
        sp = (sp - 1u) & 0xFFu;
    }
    __device__ __forceinline__ uint32_t pull(uint32_t j)
    {
        sp = (sp + 1u) & 0xFFu;
        if constexpr (FE) {
            const uint32_t v = (sp & 0x80u) ? ldp(sp & 0x7Fu)
                                            : io_read(0x100u | sp, pcnt, pins, pads, ports, su, (const uint8_t*)column(),
                                                      G->stride * 4u);
            fe_note(0x100u | sp, v);
            return v;
        }
        if (sp & 0x80u) return ldp(sp & 0x7Fu);
        if constexpr (RENDER) return io(0x100u | sp, j);
        else return io_read(0x100u | sp, pcnt, pins, pads, ports, su, (const uint8_t*)column(), G->stride * 4u);  // TIA
    }
    // Read-modify-write's two writes, on cycles j and j+1; a RAM target only
    // needs the second.
    __device__ __forceinline__ void rmw_store(uint32_t ea, uint32_t oldv, uint32_t newv, uint32_t j)
    {
        uint32_t a = ea & 0x1FFFu;
        if constexpr (!FE) {                                          // FE: the first write is an access too
            if ((a & 0x1280u) == 0x080u) { stp(a & 0x7Fu, newv); return; }
        }
#pragma unroll 1
        for (uint32_t m = 0; m < 2u; m++) write(ea, m ? newv : oldv, j + m);
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
        uint32_t ea, cyc, v, base = 0;
        bool indexed = false;                                       // (zp),Y, abs,Y, abs,X: a page may be crossed
        switch (bbb) {
        case 0: case 4: {
            // (zp,X): the pointer at zp b1 + X, read on cycles 3-4; (zp),Y: at
            // zp b1, on cycles 2-3.  One zero-page read loop for both.
            const uint32_t z = bbb == 0u ? (b1 + x) & 0xFFu : b1, j0 = bbb == 0u ? 3u : 2u;
            if constexpr (FE) {
                if (bbb == 0u) dummy(b1, 2);                        // the base, before X is added
            }
            uint32_t ptr = 0;
#pragma unroll 1
            for (uint32_t m = 0; m < 2u; m++) ptr |= zp_read((z + m) & 0xFFu, j0 + m) << (8u * m);
            if (bbb == 0u) { ea = ptr; cyc = 6; }
            else { base = ptr; ea = (ptr + y) & 0xFFFFu; cyc = 5; indexed = true; }
            break;
        }
        case 1: ea = b1; cyc = 3; break;                            // zp
        case 2: v = b1; cyc = 2; pc = (pc0 + 2u) & 0xFFFFu; goto operate;   // #imm ($89 is illegal)
        case 3: ea = (b2 << 8) | b1; cyc = 4; break;                // abs
        case 5:                                                     // zp,X
            ea = (b1 + x) & 0xFFu; cyc = 4;
            if constexpr (FE) dummy(b1, 2);                         // the base, before X is added
            break;
        default:                                                    // abs,Y / abs,X
            base = (b2 << 8) | b1;
            ea = (base + (bbb == 6u ? y : x)) & 0xFFFFu;
            cyc = 4;
            indexed = true;
            break;
        }
        // The fix-up read at the unfixed address (every store, or a page crossed).
        if (indexed && (st || ((base ^ ea) & 0xFF00u))) { dummy((base & 0xFF00u) | (ea & 0xFFu), cyc - 1u); cyc++; }
        pc = (pc0 + ((bbb == 3u || bbb >= 6u) ? 3u : 2u)) & 0xFFFFu;
        if (st) { write(ea, a, cyc - 1u); return cyc; }
        v = read(ea, cyc - 1u);
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
            ea = (b1 + ((aaa == 4u || aaa == 5u) ? y : x)) & 0xFFu; cyc = 4; pc = (pc0 + 2u) & 0xFFFFu;
            if constexpr (FE) dummy(b1, 2);                         // the base, before the index is added
            break;
        default: {                                                  // abs,X (abs,Y for LDX)
            pc = (pc0 + 3u) & 0xFFFFu;
            const uint32_t base = (b2 << 8) | b1;
            ea = (base + (aaa == 5u ? y : x)) & 0xFFFFu;
            cyc = 4;
            // LDX reads the unfixed address only when a page is crossed; the
            // read-modify-write forms always do, and take 7 cycles.
            if (aaa != 5u || ((base ^ ea) & 0xFF00u)) { dummy((base & 0xFF00u) | (ea & 0xFFu), 3); cyc = 5; }
            break;
        }
        }
        if (aaa == 4u) { write(ea, x, cyc - 1u); return cyc; }
        if (aaa == 5u) { x = read(ea, cyc - 1u); nz(x); return cyc; }
        const uint32_t v = read(ea, cyc - 1u);
        rmw_store(ea, v, shift_op(aaa, v), cyc);
        return cyc + 2u;
    }

    // cc = 00: control flow, stack, flags, BIT/STY/LDY/CPY/CPX.
    // Bus-access sites are shared between the instructions of a group (one
    // read and one write site for the memory forms, one push loop, one pull
    // loop, one read loop for the new pc's bytes): every site is inlined code,
    // and the interpreter's size decides how well it stays in the
    // instruction cache.
    __device__ __forceinline__ uint32_t group0(uint32_t pc0, uint32_t aaa, uint32_t bbb, uint32_t b1, uint32_t b2)
    {
        uint32_t ea, cyc, vb, vn, vs, vj, vv;
        switch (bbb) {
        case 4: {                                                   // branches
            pc = (pc0 + 2u) & 0xFFFFu;
            const uint32_t pos = (0x1067u >> (4u * (aaa >> 1))) & 0xFu;    // N V C Z
            if (((p >> pos) & 1u) != (aaa & 1u)) return 2;
            dummy(pc, 2);
            const uint32_t npc = (pc + (uint32_t)(int32_t)(int8_t)(uint8_t)b1) & 0xFFFFu;
            uint32_t bc = 3;
            if ((pc ^ npc) & 0xFF00u) { dummy((pc & 0xFF00u) | (npc & 0xFFu), 3); bc = 4; }
            pc = npc;
            return bc;
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
            case 4: y = (y - 1u) & 0xFFu; nz(y); return 2;          // DEY
            case 5: y = a; nz(y); return 2;                         // TAY
            case 6: y = (y + 1u) & 0xFFu; nz(y); return 2;          // INY
            case 7: x = (x + 1u) & 0xFFu; nz(x); return 2;          // INX
            default: break;
            }
            if (aaa & 1u) {                                         // PLP, PLA
                if constexpr (FE) dummy(0x100u | sp, 2);            // the stack, before the pull
                const uint32_t v = pull(3);
                if (aaa == 1u) p = v & ~(F_B | F_U);
                else { a = v; nz(a); }
                return 4;
            }
            push(aaa == 0u ? (p | F_B | F_U) : a, 2);               // PHP, PHA
            return 3;
        case 0:
            if (aaa < 2u) {                                         // BRK (b1 is the padding byte), JSR
                const bool brk = aaa == 0u;
                pc = (pc0 + 2u) & 0xFFFFu;
                // BRK pushes pch, pcl, p on cycles 2-4; JSR pushes pch, pcl on
                // cycles 3-4, before it reads the high byte.
                const uint32_t n = brk ? 3u : 2u, j0 = brk ? 2u : 3u;
                const uint32_t w = brk ? (pc << 8) | p | F_B | F_U : pc;
                if constexpr (FE) {
                    if (!brk) dummy(0x100u | sp, 2);                // JSR reads the stack before its pushes
                }
#pragma unroll 1
                for (uint32_t k = 0; k < n; k++) push((w >> (8u * (n - 1u - k))) & 0xFFu, j0 + k);
                if (brk) p |= F_I;
                // BRK: the vector at $FFFE-$FFFF on cycles 5-6; JSR: the high
                // byte at pc on cycle 5.
                vb = brk ? 0xFFFEu : pc; vn = brk ? 2u : 1u; vs = brk ? 0u : 8u; vj = 5u; vv = brk ? 0u : b1;
                cyc = brk ? 7u : 6u;
                goto vector;
            }
            if (aaa < 4u) {                                         // RTI (p, pcl, pch), RTS (pcl, pch)
                const bool rti = aaa == 2u;
                const uint32_t n = rti ? 3u : 2u;
                if constexpr (FE) dummy(0x100u | sp, 2);                // the stack, before the pulls
                uint32_t w = 0;
#pragma unroll 1
                for (uint32_t k = 0; k < n; k++) w |= pull(3u + k) << (8u * k);
                if (rti) {
                    p = w & 0xFFu & ~(F_B | F_U);
                    pc = w >> 8;
                } else {
                    dummy(w, 5);
                    pc = (w + 1u) & 0xFFFFu;
                }
                return 6;
            }
            switch (aaa) {
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
                vb = (b2 << 8) | b1; vn = 2u; vs = 0u; vj = 3u; vv = 0u; cyc = 5u;
                goto vector;
            }
            ea = (b2 << 8) | b1; cyc = 4;
            break;
        case 1:                                                     // zp: BIT STY LDY CPY CPX
            pc = (pc0 + 2u) & 0xFFFFu;
            ea = b1; cyc = 3;
            break;
        case 5:                                                     // zp,X: STY LDY
            pc = (pc0 + 2u) & 0xFFFFu;
            ea = (b1 + x) & 0xFFu; cyc = 4;
            if constexpr (FE) dummy(b1, 2);                         // the base, before X is added
            break;
        default: {                                                  // abs,X: LDY
            pc = (pc0 + 3u) & 0xFFFFu;
            const uint32_t base = (b2 << 8) | b1;
            ea = (base + x) & 0xFFFFu;
            cyc = 4;
            if ((base ^ ea) & 0xFF00u) { dummy((base & 0xFF00u) | (ea & 0xFFu), 3); cyc = 5; }
            break;
        }
        }
        return mem0(aaa, ea, cyc);
    vector:                                                         // vn bytes from vb on, within its page
#pragma unroll 1
        for (uint32_t m = 0; m < vn; m++) vv |= read((vb & 0xFF00u) | ((vb + m) & 0xFFu), vj + m) << (vs + 8u * m);
        pc = vv;
        return cyc;
    }
    __device__ __forceinline__ uint32_t mem0(uint32_t aaa, uint32_t ea, uint32_t cyc)
    {
        if (aaa == 4u) { write(ea, y, cyc - 1u); return cyc; }      // STY
        const uint32_t v = read(ea, cyc - 1u);
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
        // Fast path: the three bytes at pc0 lie in the current bank (SLICED:
        // in one window) and clear of every hotspot (and, DPC, of its read
        // registers at $1000-$103F), so reading them has no side effect.
        if (DPC      ? (a0 >= 0x1040u && (a0 & 0x3FFu) <= 0x3FDu && (a0 + 2u < 0x1FF8u || a0 > 0x1FF9u))
            : FE     ? (a0 >= 0x1000u && (a0 & 0x3FFu) <= 0x3FDu && !(slices & 0x80u))     // not armed by $01FE
            : SLICED ? (a0 >= 0x1000u && (a0 & 0x3FFu) <= 0x3FDu && (a0 + 2u < 0x1FE0u || a0 > 0x1FF7u))
                     : (a0 >= 0x1000u && a0 + 2u < hot_lo)) {
            const uint8_t* q = SLICED ? rom + srom(a0) : rom + ((bank & 7u) << 12) + (a0 & 0xFFFu);
            op = q[0];
            if (!((c_legal[op >> 5] >> (op & 31u)) & 1u)) { pc = (pc0 + 1u) & 0xFFFFu; return 0; }
            b1 = q[1];
            b2 = q[2];
        } else {
            // The opcode, then its operand bytes, through one bus-read site.
            uint32_t n = 2u, w = 0u;
            op = 0u;
#pragma unroll 1
            for (uint32_t k = 0; k < n; k++) {
                const uint32_t v = read((pc0 + k) & 0xFFFFu, k);
                if (k == 0u) {
                    op = v;
                    if (!((c_legal[op >> 5] >> (op & 31u)) & 1u)) { pc = (pc0 + 1u) & 0xFFFFu; return 0; }
                    const uint32_t bb = (op >> 2) & 7u;
                    if (bb == 3u || bb == 7u || (bb == 6u && (op & 3u) == 1u)) n = 3u;
                } else {
                    w |= v << (8u * (k - 1u));
                }
            }
            b1 = w & 0xFFu;
            b2 = w >> 8;
        }
        const uint32_t aaa = op >> 5, bbb = (op >> 2) & 7u, cc = op & 3u;
        if (cc == 1u) return group1(pc0, aaa, bbb, b1, b2);
        if (cc == 2u) return group2(pc0, aaa, bbb, b1, b2);
        return group0(pc0, aaa, bbb, b1, b2);
    }

    // ------------------------------------------------------------ rendering console
    // Used only by RENDER instantiations.  The pixel-accurate Tia of the
    // reference's rendering console (src/tia.rs) and Pia::tick run out of
    // line (render_cycles / render_tia_ticks / render_io_read / render_write_cycle,
    // below), on the state they touch passed by value: one copy of the pixel
    // pipeline however many bus-access sites the interpreter has.
    uint32_t done;            // cycle of the current instruction the TIA and PIA have reached (0 - lag at its start)
    uint32_t lag;             // CPU cycles of earlier instructions not yet given to the TIA and PIA
    uint32_t vtop;            // visible_top | vblank_top << 16
    uint8_t* fbp;             // this instance's framebuffer, 160 x 192 palette indices
    uint32_t sc, zr;          // framebuffer sector in the sector buffer; rows written since the clear point | R_ZPEND
    uint32_t rx;              // the current line's pixels are drawn up to this TIA clock

    __device__ __forceinline__ RState rpack() const
    {
        RState r;
        r.clock = clock; r.scanline = scanline; r.tw = tw; r.pcnt = pcnt; r.vtop = vtop;
        r.sc = sc; r.zr = zr; r.tv = tp & 0xFFFFu; r.ps = tp >> 16; r.sel = su & 0xFFFFu; r.uf = su >> 16;
        r.rx = rx;
        return r;
    }
    __device__ __forceinline__ void runpack(const RState& r)
    {
        clock = r.clock; scanline = r.scanline; tw = r.tw; pcnt = r.pcnt; vtop = r.vtop;
        sc = r.sc; zr = r.zr; tp = r.tv | (r.ps << 16); su = r.sel | (r.uf << 16);
        rx = r.rx;
    }
    // The TIA and the PIA up to cycle j of the current instruction.  They are
    // advanced only before an access that observes or changes them: the
    // cycles of instructions that touch only ROM and RAM are owed (lag) and
    // given in one piece.
    __device__ __forceinline__ void rsync(uint32_t j)
    {
        const uint32_t d = j - done;
        if ((int32_t)d > 0) { runpack(render_cycles(rpack(), d, pins, pv, fbp)); done = j; }
    }
    __device__ __forceinline__ void rcycles(uint32_t n) { runpack(render_cycles(rpack(), n, pins, pv, fbp)); }
    __device__ __forceinline__ void settle()
    {
        if (lag) { runpack(render_cycles(rpack(), lag, pins, pv, fbp)); lag = 0; }
    }
    // Bus::write of a PIA register (src/atari.rs:207-222): two TIA clocks, the
    // write, one TIA clock, the PIA clock.
    __device__ __forceinline__ void r_write_cycle(uint32_t a, uint32_t v)
    {
        RState r = render_tia_ticks(rpack(), 2u, pins, pv, fbp);
        const uint4 q = pia_write_io(a, v, ports, r.tv, r.ps, r.sel | (r.uf << 16));
        ports = q.x; r.tv = q.y; r.ps = q.z; r.sel = q.w & 0xFFFFu; r.uf = q.w >> 16;
        r = render_tia_ticks(r, 1u, pins, pv, fbp);
        runpack(r);
        pia_tick1();
    }
    __device__ __forceinline__ void pia_tick1()                      // pia.rs:80-103
    {
        uint32_t tv = tp & 0xFFFFu, ps = tp >> 16, uf = su >> 16;
        if (tv == 0 && uf) {
            tv = 0xFFu;
        } else {
            ps = (ps - 1u) & 0xFFFFu;
            if (ps == 0) {
                ps = uf ? 1u : (su & 0xFFFFu);
                if (tv == 0) { uf = 1; tv = 0xFFu; } else tv -= 1u;
            }
        }
        tp = tv | (ps << 16);
        su = (su & 0xFFFFu) | (uf << 16);
    }
    // The owed cycles, the pixels up to the beam, and the framebuffer as it
    // can be seen now (the end of a frame or of a call).
    __device__ __forceinline__ void fb_observe()
    {
        settle();
        runpack(render_observe(rpack(), pv, fbp));
    }
    // The sector buffer at the start of a call: the sector where the beam's
    // row has been drawn to, as the last call left it in the framebuffer.
    __device__ __forceinline__ void fb_resume()
    {
        const uint32_t vis = (scanline - (vtop & 0xFFFFu)) & 0xFFFFu;
        zr = vis < FA_FB_H ? vis : FA_FB_H;
        if (vis < FA_FB_H) {
            const uint32_t x = (rx > 68u ? rx : 68u) - 68u;
            sc = vis * (FA_FB_W / 32u) + ((x >> 5) < 4u ? (x >> 5) : 4u);
            const uint4* q = (const uint4*)(fbp + (size_t)sc * 32u);
            const uint4 u0 = q[0], u1 = q[1];
            *r_sbuf(pv, 0) = u0.x; *r_sbuf(pv, 1) = u0.y; *r_sbuf(pv, 2) = u0.z; *r_sbuf(pv, 3) = u0.w;
            *r_sbuf(pv, 4) = u1.x; *r_sbuf(pv, 5) = u1.y; *r_sbuf(pv, 6) = u1.z; *r_sbuf(pv, 7) = u1.w;
        } else {
            sc = 0;
            r_sec_clear(pv);
        }
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
        tp = col[R_TIMER * stride];
        w = col[R_SELPC * stride]; su = (w & 0xFFFFu) | (((p1 >> 16) & 0xFFu) << 16); pcnt = w >> 16;
        tlim = RENDER ? 0u : pia_span();
        w = col[R_TIA0 * stride];  clock = w & 0xFFFF; scanline = w >> 16;
        w = col[R_TIA1 * stride];                                   // wsync fcomp vsync vblank
        tw = ((w >> 16) & 0xFFFFu) | ((w & 1u) << 16) | (((w >> 8) & 1u) << 17) | (((p1 >> 24) & 1u) << 18);
        if constexpr (SLICED) slices = slices_of(fa_tia1_mapper(w));
        w = col[R_TIA2 * stride];                                   // inpt4 inpt5 pad0 pad1
        pins = ((p0 >> 16) & 0xFFu) | (((p1 >> 8) & 0xFFu) << 8) | ((w & 1u) << 16) | (((w >> 8) & 1u) << 17);
        pads = w >> 16;
    }
    __device__ __forceinline__ void store_hot(uint32_t* col, uint32_t stride) const
    {
        col[R_AXYS * stride] = a | (x << 8) | (y << 16) | (sp << 24);
        col[R_PC * stride] = pc | (p << 16) | ((bank & 7u) << 24);
        col[R_PIA0 * stride] = (ports & 0xFFFFu) | ((pins & 0xFFu) << 16) | (((ports >> 16) & 0xFFu) << 24);
        col[R_PIA1 * stride] = (ports >> 24) | (((pins >> 8) & 0xFFu) << 8) | ((su >> 16) << 16) | (((tw >> 18) & 1u) << 24);
        const uint2 t = RENDER ? make_uint2(tp & 0xFFFFu, tp >> 16) : pia_now();
        col[R_TIMER * stride] = t.x | (t.y << 16);
        col[R_SELPC * stride] = (su & 0xFFFFu) | (pcnt << 16);
        col[R_TIA0 * stride] = clock | (scanline << 16);
        uint32_t t1 = ((tw >> 16) & 1u) | (((tw >> 17) & 1u) << 8) | ((tw & 0xFFFFu) << 16);
        if constexpr (SLICED) t1 |= fa_mapper_tia1(mapper_of(slices));
        col[R_TIA1 * stride] = t1;
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
