/*
 * fa_oracle.c — CPU oracle: plain-C restatement of the reference HeadlessAtari.
 *
 * TEST INFRASTRUCTURE ONLY (see fa_oracle.h).  Each function cites the
 * reference file:line it restates.  The structure deliberately follows the
 * reference (flat 8 KiB bus array, 4 KiB bank memcpy, per-instruction bulk
 * TIA/PIA advance) so that it checks the CUDA path, which is organised very
 * differently, and so that its timing is representative of the reference's
 * CPU emulator.
 */
#define _GNU_SOURCE
#include "fa_oracle.h"

#include <pthread.h>
#include <sched.h>
#include <stdlib.h>
#include <string.h>

enum { F_C = 1, F_Z = 2, F_I = 4, F_D = 8, F_B = 16, F_U = 32, F_V = 64, F_N = 128 };

/* ------------------------------------------------------------ CPU (cpu.rs) */
typedef struct orc_cpu {          /* Cpu, src/cpu.rs:96-105 */
    uint16_t pc;
    uint8_t  sp, a, x, y, p;
    uint64_t cycles;
} orc_cpu;

static inline void orc_setf(orc_cpu* c, uint8_t f, int on)       /* Status::set :42 */
{
    if (on) c->p |= f; else c->p &= (uint8_t)~f;
}
static inline void orc_zn(orc_cpu* c, uint8_t v)                 /* Status::set_zn :48 */
{
    orc_setf(c, F_Z, v == 0);
    orc_setf(c, F_N, (v & 0x80) != 0);
}

static void orc_adc(orc_cpu* c, uint8_t v)                        /* cpu.rs:153-175 */
{
    uint8_t carry = (c->p & F_C) ? 1 : 0;
    if (c->p & F_D) {
        uint8_t lo = (uint8_t)((c->a & 0x0F) + (v & 0x0F) + carry);
        if (lo > 9) lo = (uint8_t)(lo + 6);
        uint8_t hi = (uint8_t)((c->a >> 4) + (v >> 4) + (lo > 0x0F ? 1 : 0));
        uint16_t bin = (uint16_t)(c->a + v + carry);
        orc_setf(c, F_Z, (uint8_t)bin == 0);
        orc_setf(c, F_N, (hi & 0x08) != 0);
        orc_setf(c, F_V, ((uint8_t)(~(c->a ^ v)) & (uint8_t)(c->a ^ (uint8_t)((hi << 4) | (lo & 0x0F))) & 0x80) != 0);
        if (hi > 9) hi = (uint8_t)(hi + 6);
        orc_setf(c, F_C, hi > 0x0F);
        c->a = (uint8_t)(((hi & 0x0F) << 4) | (lo & 0x0F));
    } else {
        uint16_t s = (uint16_t)(c->a + v + carry);
        uint8_t r = (uint8_t)s;
        orc_setf(c, F_C, s > 0xFF);
        orc_setf(c, F_V, ((uint8_t)(~(c->a ^ v)) & (uint8_t)(c->a ^ r) & 0x80) != 0);
        c->a = r;
        orc_zn(c, c->a);
    }
}

static void orc_sbc(orc_cpu* c, uint8_t v)                        /* cpu.rs:178-200 */
{
    uint8_t borrow = (c->p & F_C) ? 0 : 1;
    if (c->p & F_D) {
        uint8_t lo = (uint8_t)((c->a & 0x0F) - (v & 0x0F) - borrow);
        uint8_t lob = 0;
        if ((int8_t)lo < 0) { lo = (uint8_t)(lo - 6); lob = 1; }
        uint8_t hi = (uint8_t)((c->a >> 4) - (v >> 4) - lob);
        if ((int8_t)hi < 0) hi = (uint8_t)(hi - 6);
        int16_t bin = (int16_t)((int16_t)c->a - (int16_t)v - (int16_t)borrow);
        orc_setf(c, F_C, bin >= 0);
        orc_setf(c, F_Z, (uint8_t)bin == 0);
        orc_setf(c, F_N, ((uint8_t)bin & 0x80) != 0);
        orc_setf(c, F_V, ((c->a ^ v) & (c->a ^ (uint8_t)bin) & 0x80) != 0);
        c->a = (uint8_t)(((hi & 0x0F) << 4) | (lo & 0x0F));
    } else {
        uint8_t d1 = (uint8_t)(c->a - v);
        int b1 = v > c->a;
        uint8_t d2 = (uint8_t)(d1 - borrow);
        int b2 = borrow > d1;
        orc_setf(c, F_C, !(b1 || b2));
        orc_setf(c, F_V, ((c->a ^ v) & (c->a ^ d2) & 0x80) != 0);
        c->a = d2;
        orc_zn(c, c->a);
    }
}

static inline void orc_compare(orc_cpu* c, uint8_t reg, uint8_t v) /* cpu.rs:203-207 */
{
    orc_setf(c, F_C, reg >= v);
    orc_zn(c, (uint8_t)(reg - v));
}
static inline uint8_t orc_asl(orc_cpu* c, uint8_t v)               /* cpu.rs:210-215 */
{
    orc_setf(c, F_C, (v & 0x80) != 0);
    uint8_t r = (uint8_t)(v << 1); orc_zn(c, r); return r;
}
static inline uint8_t orc_lsr(orc_cpu* c, uint8_t v)               /* cpu.rs:218-223 */
{
    orc_setf(c, F_C, (v & 0x01) != 0);
    uint8_t r = (uint8_t)(v >> 1); orc_zn(c, r); return r;
}
static inline uint8_t orc_rol(orc_cpu* c, uint8_t v)               /* cpu.rs:226-232 */
{
    uint8_t oc = (c->p & F_C) ? 1 : 0;
    orc_setf(c, F_C, (v & 0x80) != 0);
    uint8_t r = (uint8_t)((v << 1) | oc); orc_zn(c, r); return r;
}
static inline uint8_t orc_ror(orc_cpu* c, uint8_t v)               /* cpu.rs:235-241 */
{
    uint8_t oc = (c->p & F_C) ? 1 : 0;
    orc_setf(c, F_C, (v & 0x01) != 0);
    uint8_t r = (uint8_t)((v >> 1) | (oc << 7)); orc_zn(c, r); return r;
}

/* The per-opcode operation of the read-type instructions (the inner matches
 * of cpu.rs:342-354, 371-390, 427-436, 573-590, 668-677, 758-767, 812-820,
 * 869-877). */
static void orc_read_op(orc_cpu* c, uint8_t op, uint8_t v)
{
    switch (op) {
    case 0xA9: case 0xA5: case 0xB5: case 0xAD: case 0xBD: case 0xB9: case 0xA1: case 0xB1:
        c->a = v; orc_zn(c, c->a); break;                                      /* LDA */
    case 0xA2: case 0xA6: case 0xAE:
        c->x = v; orc_zn(c, c->x); break;                                      /* LDX */
    case 0xA0: case 0xA4: case 0xB4: case 0xAC: case 0xBC:
        c->y = v; orc_zn(c, c->y); break;                                      /* LDY */
    case 0x69: case 0x65: case 0x75: case 0x6D: case 0x7D: case 0x79: case 0x61: case 0x71:
        orc_adc(c, v); break;
    case 0xE9: case 0xE5: case 0xF5: case 0xED: case 0xFD: case 0xF9: case 0xE1: case 0xF1:
        orc_sbc(c, v); break;
    case 0x29: case 0x25: case 0x35: case 0x2D: case 0x3D: case 0x39: case 0x21: case 0x31:
        c->a &= v; orc_zn(c, c->a); break;                                     /* AND */
    case 0x09: case 0x05: case 0x15: case 0x0D: case 0x1D: case 0x19: case 0x01: case 0x11:
        c->a |= v; orc_zn(c, c->a); break;                                     /* ORA */
    case 0x49: case 0x45: case 0x55: case 0x4D: case 0x5D: case 0x59: case 0x41: case 0x51:
        c->a ^= v; orc_zn(c, c->a); break;                                     /* EOR */
    case 0xC9: case 0xC5: case 0xD5: case 0xCD: case 0xDD: case 0xD9: case 0xC1: case 0xD1:
        orc_compare(c, c->a, v); break;                                        /* CMP */
    case 0xE0: case 0xE4: case 0xEC:
        orc_compare(c, c->x, v); break;                                        /* CPX */
    case 0xC0: case 0xC4: case 0xCC:
        orc_compare(c, c->y, v); break;                                        /* CPY */
    case 0x24: case 0x2C:                                                      /* BIT */
        orc_setf(c, F_Z, (c->a & v) == 0);
        orc_setf(c, F_V, (v & 0x40) != 0);
        orc_setf(c, F_N, (v & 0x80) != 0);
        break;
    default: break;
    }
}

static inline uint8_t orc_store_val(const orc_cpu* c, uint8_t op)
{
    switch (op) {
    case 0x86: case 0x8E: case 0x96: return c->x;                              /* STX */
    case 0x84: case 0x8C: case 0x94: return c->y;                              /* STY */
    default: return c->a;                                                      /* STA */
    }
}

static uint8_t orc_rmw(orc_cpu* c, uint8_t op, uint8_t v)
{
    switch (op) {
    case 0x06: case 0x16: case 0x0E: case 0x1E: return orc_asl(c, v);
    case 0x46: case 0x56: case 0x4E: case 0x5E: return orc_lsr(c, v);
    case 0x26: case 0x36: case 0x2E: case 0x3E: return orc_rol(c, v);
    case 0x66: case 0x76: case 0x6E: case 0x7E: return orc_ror(c, v);
    case 0xE6: case 0xF6: case 0xEE: case 0xFE: { uint8_t r = (uint8_t)(v + 1); orc_zn(c, r); return r; }
    default:                                    { uint8_t r = (uint8_t)(v - 1); orc_zn(c, r); return r; }
    }
}

/* ----------------------------------------------- HeadlessTia (headless_tia.rs) */
typedef struct orc_tia {          /* HeadlessTia, headless_tia.rs:16-88 */
    uint16_t clock, scanline;
    uint8_t  wsync, frame_complete, vsync, vblank;
    uint8_t  cx[8];               /* cxm0p cxm1p cxp0fb cxp1fb cxm0fb cxm1fb cxblpf cxppmm */
    uint8_t  inpt4, inpt5, paddle0, paddle1;
    uint16_t paddle_counter;
    uint8_t  paddle_dumped;
    uint16_t pos[5];              /* p0 p1 m0 m1 bl */
    uint8_t  hm[5];               /* hmp0 hmp1 hmm0 hmm1 hmbl */
    uint8_t  grp0, grp1, grp0_old, grp1_old;
    uint8_t  enam0, enam1, enabl, enabl_old;
    uint8_t  vdelp0, vdelp1, vdelbl, resmp0, resmp1;
    uint8_t  nusiz0, nusiz1, colup0, colup1, colupf, colubk, ctrlpf, refp0, refp1;
    uint8_t  pf0, pf1, pf2;
} orc_tia;

static void orc_tia_default(orc_tia* t)                            /* headless_tia.rs:90-118 */
{
    memset(t, 0, sizeof(*t));
    t->inpt4 = 1;
    t->inpt5 = 1;
}

static void orc_tia_end_scanline(orc_tia* t)                       /* headless_tia.rs:183-198 */
{
    t->clock = (uint16_t)(t->clock - 228);
    t->scanline++;
    t->wsync = 0;
    if (!t->paddle_dumped && t->paddle_counter < 256) t->paddle_counter++;
    if (t->scanline >= 262) {                                      /* SCANLINES_PER_FRAME */
        t->scanline = 0;
        if (!t->frame_complete) t->frame_complete = 1;
    }
}

static inline void orc_tia_tick_n(orc_tia* t, uint8_t n)           /* headless_tia.rs:153-158 */
{
    t->clock = (uint16_t)(t->clock + n * 3);
    if (t->clock >= 228) orc_tia_end_scanline(t);
}

static uint16_t orc_tia_skip_to_scanline_end(orc_tia* t)           /* headless_tia.rs:163-180 */
{
    uint16_t rem = t->clock >= 228 ? 0 : (uint16_t)(228 - t->clock);
    uint16_t cpu = (uint16_t)((rem + 2) / 3);
    if (cpu > 0) {
        t->clock = 228;
        orc_tia_end_scanline(t);
    }
    return cpu;
}

static uint16_t orc_hmove(uint16_t pos, uint8_t hm)                /* headless_tia.rs:200-203 */
{
    int16_t off = (int16_t)(((int8_t)hm) >> 4);                    /* arithmetic shift of i8 */
    int r = (int16_t)((int16_t)pos - off) % 160;                   /* i16 wrapping, rem_euclid */
    if (r < 0) r += 160;
    return (uint16_t)r;
}

static uint8_t orc_tia_read(const orc_tia* t, uint16_t addr)       /* headless_tia.rs:205-223 */
{
    switch (addr & 0x0F) {
    case 0x00: case 0x01: case 0x02: case 0x03:
    case 0x04: case 0x05: case 0x06: case 0x07: return t->cx[addr & 7];
    case 0x08: return t->paddle_counter >= t->paddle0 ? 0x80 : 0x00;
    case 0x09: return t->paddle_counter >= t->paddle1 ? 0x80 : 0x00;
    case 0x0A: case 0x0B: return 0x80;
    case 0x0C: return t->inpt4 ? 0x80 : 0x00;
    case 0x0D: return t->inpt5 ? 0x80 : 0x00;
    default: return 0;
    }
}

static uint16_t orc_resp_pos(const orc_tia* t)                     /* headless_tia.rs:257-261 */
{
    int r = (int16_t)((int16_t)t->clock - 68 + 5) % 160;          /* i16, rem_euclid */
    if (r < 0) r += 160;
    return (uint16_t)r;
}

static void orc_tia_write(orc_tia* t, uint16_t addr, uint8_t v)    /* headless_tia.rs:225-298 */
{
    switch (addr & 0x3F) {
    case 0x00:
        if (!(t->vsync & 0x02) && (v & 0x02)) { t->scanline = 0; t->frame_complete = 1; }
        t->vsync = v; break;
    case 0x01:
        if (v & 0x80) { t->paddle_counter = 0; t->paddle_dumped = 1; }
        else if (t->paddle_dumped) t->paddle_dumped = 0;
        t->vblank = v; break;
    case 0x02: t->wsync = 1; break;
    case 0x04: t->nusiz0 = v; break;
    case 0x05: t->nusiz1 = v; break;
    case 0x06: t->colup0 = v; break;
    case 0x07: t->colup1 = v; break;
    case 0x08: t->colupf = v; break;
    case 0x09: t->colubk = v; break;
    case 0x0A: t->ctrlpf = v; break;
    case 0x0B: t->refp0 = (v & 0x08) != 0; break;
    case 0x0C: t->refp1 = (v & 0x08) != 0; break;
    case 0x0D: t->pf0 = v; break;
    case 0x0E: t->pf1 = v; break;
    case 0x0F: t->pf2 = v; break;
    case 0x10: case 0x11: case 0x12: case 0x13: case 0x14:
        t->pos[(addr & 0x3F) - 0x10] = orc_resp_pos(t); break;
    case 0x1B: t->grp0_old = t->grp0; t->grp0 = v; break;
    case 0x1C: t->grp1_old = t->grp1; t->grp1 = v; t->enabl_old = t->enabl; break;
    case 0x1D: t->enam0 = (v & 0x02) != 0; break;
    case 0x1E: t->enam1 = (v & 0x02) != 0; break;
    case 0x1F: t->enabl = (v & 0x02) != 0; break;
    case 0x20: case 0x21: case 0x22: case 0x23: case 0x24:
        t->hm[(addr & 0x3F) - 0x20] = v; break;
    case 0x25: t->vdelp0 = (v & 0x01) != 0; break;
    case 0x26: t->vdelp1 = (v & 0x01) != 0; break;
    case 0x27: t->vdelbl = (v & 0x01) != 0; break;
    case 0x28: t->resmp0 = (v & 0x02) != 0; break;
    case 0x29: t->resmp1 = (v & 0x02) != 0; break;
    case 0x2A:
        for (int i = 0; i < 5; i++) t->pos[i] = orc_hmove(t->pos[i], t->hm[i]);
        break;
    case 0x2B: memset(t->hm, 0, sizeof(t->hm)); break;
    case 0x2C: memset(t->cx, 0, sizeof(t->cx)); break;
    default: break;                                                /* 0x03, audio, unused */
    }
}

/* ---------------------------------------------------------------- Pia (pia.rs) */
typedef struct orc_pia {          /* Pia, pia.rs:26-44 */
    uint8_t  ram[128];
    uint8_t  pa_out, pa_ddr, pa_in, pb_out, pb_ddr, pb_in;
    uint16_t timer_value, timer_prescaler, timer_select;
    uint8_t  timer_underflow;
} orc_pia;

static void orc_pia_default(orc_pia* p)                            /* pia.rs:46-62 */
{
    memset(p, 0, sizeof(*p));
    p->pa_in = 0xFF;
    p->pb_in = 0x3F;
    p->timer_prescaler = 1;
    p->timer_select = 1;
}

static void orc_pia_tick_n(orc_pia* p, uint16_t n)                 /* pia.rs:107-166 */
{
    if (n == 0) return;
    if (p->timer_value == 0 && p->timer_underflow) {
        p->timer_value = (uint16_t)((uint16_t)(0xFF - (n - 1)) & 0xFF);
        return;
    }
    uint16_t rem = n;
    if (p->timer_prescaler > 0) {
        if (rem < p->timer_prescaler) { p->timer_prescaler = (uint16_t)(p->timer_prescaler - rem); return; }
        rem = (uint16_t)(rem - p->timer_prescaler);
        p->timer_prescaler = 0;
        if (p->timer_value == 0) {
            p->timer_underflow = 1;
            p->timer_value = 0xFF;
            if (rem > 0) p->timer_value = (uint16_t)((uint16_t)(0xFF - (rem - 1)) & 0xFF);
            return;
        }
        p->timer_value--;
    }
    if (rem == 0) { p->timer_prescaler = p->timer_select; return; }
    uint16_t ps = p->timer_select;
    uint16_t full = (uint16_t)(rem / ps);
    uint16_t left = (uint16_t)(rem % ps);
    if (full >= p->timer_value) {
        uint16_t to_zero = (uint16_t)(p->timer_value * ps);        /* u16 arithmetic as in Rust */
        rem = (uint16_t)(rem - to_zero);
        p->timer_underflow = 1;
        p->timer_value = 0xFF;
        if (rem > 0) p->timer_value = (uint16_t)((uint16_t)(0xFF - (rem - 1)) & 0xFF);
    } else {
        p->timer_value = (uint16_t)(p->timer_value - full);
        p->timer_prescaler = (uint16_t)(ps - left);
    }
}

static uint8_t orc_pia_read(orc_pia* p, uint16_t addr)             /* pia.rs:169-199 */
{
    if (!(addr & 0x200)) return p->ram[addr & 0x7F];
    switch (addr & 0x07) {
    case 0x00: return (uint8_t)((p->pa_in & ~p->pa_ddr) | (p->pa_out & p->pa_ddr));
    case 0x01: return p->pa_ddr;
    case 0x02: return (uint8_t)((p->pb_in & ~p->pb_ddr) | (p->pb_out & p->pb_ddr));
    case 0x03: return p->pb_ddr;
    case 0x04: p->timer_underflow = 0; return (uint8_t)p->timer_value;
    case 0x05: return p->timer_underflow ? 0x80 : 0x00;
    default: return 0;
    }
}

static void orc_pia_write(orc_pia* p, uint16_t addr, uint8_t v)    /* pia.rs:202-228 */
{
    static const uint16_t sel[4] = { 1, 8, 64, 1024 };
    if (!(addr & 0x200)) { p->ram[addr & 0x7F] = v; return; }
    if (addr & 0x10) {
        p->timer_value = v;
        p->timer_underflow = 0;
        p->timer_select = sel[addr & 3];
        p->timer_prescaler = p->timer_select;
        return;
    }
    switch (addr & 0x03) {
    case 0: p->pa_out = v; break;
    case 1: p->pa_ddr = v; break;
    case 2: p->pb_out = v; break;
    default: p->pb_ddr = v; break;
    }
}

/* ------------------------------------------------- DPC (Pitfall II's cartridge chip)
 * The reference has no DPC cart (its size rule cannot construct one).  This is
 * the chip as its published descriptions give it (Activision's US patent
 * 4,644,495 and the community's cartridge documentation), with the choices
 * they leave open fixed here and in the device core alike:
 *   - a read of $1000-$103F: fetcher k = a & 7, function f = (a >> 3) & 7.
 *     The music channels are first brought up to the instruction's start
 *     (Cpu::cycles), the random number generator steps, and a fetcher that is
 *     not a music channel updates its flag (set when the counter's low byte
 *     equals top, else cleared when it equals bottom).  f 0 reads the random
 *     number (k < 4) or the music amplitude (k >= 4); f 1 the display byte at
 *     the counter; f 2 that byte ANDed with the flag; f 7 the flag; the rest
 *     0.  Then the counter counts down (11 bits), unless the fetcher is a
 *     music channel.
 *   - a write of $1040-$107F (same k and f): music brought up to date, then
 *     f 0 top (and the flag cleared), f 1 bottom, f 2 counter low byte, f 3
 *     counter bits 8-10 (and, for fetchers 5-7, music mode from bit 4), f 6
 *     the random number reset to 1; the rest nothing.
 *   - display data: the 2K after the 8K of program, addressed downward from
 *     its end (counter c reads byte 2047 - c), as dumps of the cart hold it.
 *   - music: the oscillator counts 20,000 clocks per second of CPU cycles
 *     (3,579,545 / 3 per second), exactly: clock(t) = floor(t * 60000 /
 *     3579545).  Each clock counts a music channel's low byte down by one;
 *     the clock after 0 reloads top.  After an update that counted clocks,
 *     a channel's flag is set while its low byte is above bottom.  The
 *     amplitude is 4, 5 and 6 for channels 5, 6 and 7 whose flag is set,
 *     summed.
 *   - the random number generator shifts left, taking in the XNOR of bits 7,
 *     5, 4 and 3; power-on value 1. */
typedef struct orc_dpc {
    uint16_t counter[8];
    uint8_t  top[8], bottom[8];
    uint8_t  flags, music, random;
    uint32_t osc;
} orc_dpc;

/* ------------------------------------------------- HeadlessBus + HeadlessAtari */
struct orc_atari {
    orc_cpu  cpu;
    orc_tia  tia;
    orc_pia  pia;
    uint8_t  mem[8192];           /* HeadlessBus::mem, atari.rs:402 */
    uint8_t* rom;
    size_t   rom_len;
    int      bank;
    int      scheme;
    int      slice[4];            /* E0 / 3F / DPC: the 1K ROM slice in each 1K window of $1000-$1FFF */
    orc_dpc  dpc;                 /* DPC registers (FA_SCHEME_DPC) */
    int      fe_pend;             /* FE: the last bus access was to $01FE */
    uint32_t frame_no;
    uint32_t run_status;
    uint64_t instructions;
};

static int orc_detect(size_t len)                                  /* atari.rs:96-105 */
{
    if (len <= 4096) return FA_SCHEME_FIXED;
    if (len <= 8192) return FA_SCHEME_F8;
    if (len <= 16384) return FA_SCHEME_F6;
    return FA_SCHEME_F4;
}

/* Lengths for which HeadlessBus::new does not panic: the power-on bank's
 * slice rom[bank*4096 .. bank*4096+4096] must exist (atari.rs:412-448), and
 * the Fixed mirror i % rom_len needs rom_len > 0. */
static int orc_rom_len_ok(size_t len)
{
    if (len == 0) return 0;
    switch (orc_detect(len)) {
    case FA_SCHEME_FIXED: return 1;
    case FA_SCHEME_F8: return len >= 8192;
    case FA_SCHEME_F6: return len >= 16384;
    default: return len >= 32768;
    }
}

/* Schemes registered per ROM image, as the library's fa_rom_set_scheme does:
 * keyed by FNV-1a of the bytes and the length.  E0 and 3F are never picked by
 * size (the reference has neither). */
#define ORC_MAX_SCHEMES 64
static struct { uint64_t h; size_t len; int scheme; } g_orc_reg[ORC_MAX_SCHEMES];
static int g_orc_nreg;

static uint64_t orc_rom_hash(const uint8_t* rom, size_t len)
{
    uint64_t h = 0xCBF29CE484222325ull;
    for (size_t i = 0; i < len; i++) h = (h ^ rom[i]) * 0x100000001B3ull;
    return h;
}

static int orc_dpc_len(size_t len) { return len == 10240 || len == 10495; }

static int orc_scheme_len_ok(int scheme, size_t len)
{
    if (scheme == FA_SCHEME_E0 || scheme == FA_SCHEME_FE) return len == 8192;
    if (scheme == FA_SCHEME_DPC) return orc_dpc_len(len);
    if (scheme == FA_SCHEME_3F) return len >= 2048 && len <= 32768 && len % 2048 == 0;
    return orc_rom_len_ok(len) && orc_detect(len) == scheme;
}

int orc_rom_set_scheme(const uint8_t* rom, size_t len, int scheme)
{
    if (!rom || len == 0) return -1;
    if (scheme >= 0 && !orc_scheme_len_ok(scheme, len)) return -1;
    const uint64_t h = orc_rom_hash(rom, len);
    for (int i = 0; i < g_orc_nreg; i++)
        if (g_orc_reg[i].h == h && g_orc_reg[i].len == len) { g_orc_reg[i] = g_orc_reg[--g_orc_nreg]; break; }
    if (scheme < 0) return 0;
    if (g_orc_nreg == ORC_MAX_SCHEMES) return -1;
    g_orc_reg[g_orc_nreg].h = h;
    g_orc_reg[g_orc_nreg].len = len;
    g_orc_reg[g_orc_nreg].scheme = scheme;
    g_orc_nreg++;
    return 0;
}

/* The scheme of a ROM image: registered, else the size rule; -1 when the
 * reference could not construct it. */
static int orc_scheme_for(const uint8_t* rom, size_t len)
{
    if (!rom || len == 0) return -1;
    const uint64_t h = orc_rom_hash(rom, len);
    for (int i = 0; i < g_orc_nreg; i++)
        if (g_orc_reg[i].h == h && g_orc_reg[i].len == len) return g_orc_reg[i].scheme;
    if (orc_dpc_len(len)) return FA_SCHEME_DPC;
    return orc_rom_len_ok(len) ? orc_detect(len) : -1;
}

static int orc_sliced(int scheme)
{
    return scheme == FA_SCHEME_E0 || scheme == FA_SCHEME_3F || scheme == FA_SCHEME_DPC || scheme == FA_SCHEME_FE;
}

/* Power-on windows of the sliced schemes: E0 slices 4, 5, 6, 7; 3F 2K bank 0
 * under the last 2K. */
static void orc_power_on_slices(int scheme, size_t len, int* slice)
{
    if (scheme == FA_SCHEME_E0 || scheme == FA_SCHEME_DPC || scheme == FA_SCHEME_FE) {
        slice[0] = 4; slice[1] = 5; slice[2] = 6; slice[3] = 7;
        return;
    }
    const int l = (int)(len / 2048) - 1;
    slice[0] = 0; slice[1] = 1; slice[2] = 2 * l; slice[3] = 2 * l + 1;
}

static unsigned orc_mapper_of(int scheme, const int* slice)
{
    if (scheme == FA_SCHEME_E0) return (unsigned)(slice[0] | slice[1] << 4 | slice[2] << 8);
    if (scheme == FA_SCHEME_3F) return (unsigned)(slice[0] / 2);
    if (scheme == FA_SCHEME_DPC || scheme == FA_SCHEME_FE) return (unsigned)(slice[0] / 4);
    return 0;
}

static void orc_slices_of(int scheme, size_t len, unsigned m, int* slice)
{
    orc_power_on_slices(scheme, len, slice);
    if (scheme == FA_SCHEME_E0) { slice[0] = m & 7; slice[1] = (m >> 4) & 7; slice[2] = (m >> 8) & 7; }
    else if (scheme == FA_SCHEME_3F) { const int b = (int)((m & 0xFF) % (len / 2048)); slice[0] = 2 * b; slice[1] = 2 * b + 1; }
    else if (scheme == FA_SCHEME_DPC || scheme == FA_SCHEME_FE) for (int w = 0; w < 4; w++) slice[w] = 4 * (int)(m & 1) + w;
}

static void orc_load_window(orc_atari* e, int w)
{
    memcpy(&e->mem[0x1000 + 1024 * w], &e->rom[(size_t)e->slice[w] * 1024], 1024);
}

static void orc_load_bank(orc_atari* e, int bank)                  /* atari.rs:433-449 */
{
    if (orc_sliced(e->scheme)) {
        for (int w = 0; w < 4; w++) orc_load_window(e, w);
        return;
    }
    if (e->scheme == FA_SCHEME_FIXED) {
        for (int i = 0; i < 4096; i++) e->mem[0x1000 + i] = e->rom[(size_t)i % e->rom_len];
        return;
    }
    memcpy(&e->mem[0x1000], &e->rom[(size_t)bank * 4096], 4096);
}

static void orc_sync_ram_to_mem(orc_atari* e)                      /* atari.rs:454-457 */
{
    memcpy(&e->mem[0x80], e->pia.ram, 128);
    memcpy(&e->mem[0x180], e->pia.ram, 128);
}

static inline void orc_check_bankswitch(orc_atari* e, uint16_t addr) /* atari.rs:460-492 */
{
    uint16_t a = addr & 0x1FFF;
    int nb;
    switch (e->scheme) {
    case FA_SCHEME_F8: if (a < 0x1FF8 || a > 0x1FF9) return; nb = a - 0x1FF8; break;
    case FA_SCHEME_F6: if (a < 0x1FF6 || a > 0x1FF9) return; nb = a - 0x1FF6; break;
    case FA_SCHEME_F4: if (a < 0x1FF4 || a > 0x1FFB) return; nb = a - 0x1FF4; break;
    case FA_SCHEME_E0:                       /* $1FE0-$1FF7: slice a & 7 into window (a - $1FE0) / 8 */
        if (a >= 0x1FE0 && a <= 0x1FF7) {
            const int w = (a - 0x1FE0) >> 3;
            e->slice[w] = a & 7;
            orc_load_window(e, w);
        }
        return;
    case FA_SCHEME_DPC:                      /* $1FF8 / $1FF9: program bank 0 / 1 */
        if (a == 0x1FF8 || a == 0x1FF9)
            for (int w = 0; w < 4; w++) {
                e->slice[w] = 4 * (a - 0x1FF8) + w;
                orc_load_window(e, w);
            }
        return;
    default: return;
    }
    if (nb != e->bank) {
        e->bank = nb;
        orc_load_bank(e, nb);
    }
}

/* The oscillator's clock count at CPU cycle t: floor(t * 60000 / 3579545)
 * without overflowing 64 bits, modulo 2^32. */
static uint32_t orc_dpc_clock_at(uint64_t t)
{
    return (uint32_t)((t / 3579545u) * 60000u + ((t % 3579545u) * 60000u) / 3579545u);
}

/* A music channel's low byte after k oscillator clocks. */
static uint32_t orc_dpc_count_down(uint32_t low, uint32_t top, uint32_t k)
{
    if (k <= low) return low - k;
    k -= low + 1;                                    /* the clock that leaves 0 reloads top */
    return top - k % (top + 1);
}

static void orc_dpc_update(orc_atari* e)
{
    orc_dpc* d = &e->dpc;
    const uint32_t now = orc_dpc_clock_at(e->cpu.cycles);
    const uint32_t k = now - d->osc;
    d->osc = now;
    if (k == 0) return;
    for (int m = 0; m < 3; m++) {
        if (!((d->music >> m) & 1)) continue;
        const int f = 5 + m;
        const uint32_t low = orc_dpc_count_down(d->counter[f] & 0xFFu, d->top[f], k);
        d->counter[f] = (uint16_t)((d->counter[f] & 0x700u) | low);
        if (low > d->bottom[f]) d->flags |= (uint8_t)(1u << f);
        else d->flags &= (uint8_t)~(1u << f);
    }
}

static uint8_t orc_dpc_next_random(uint8_t r)
{
    const unsigned x = (unsigned)(r >> 7) ^ (unsigned)(r >> 5) ^ (unsigned)(r >> 4) ^ (unsigned)(r >> 3);
    return (uint8_t)((r << 1) | (~x & 1u));
}

static uint8_t orc_dpc_read(orc_atari* e, uint16_t a)
{
    orc_dpc* d = &e->dpc;
    const int k = a & 7, f = (a >> 3) & 7;
    const int music = k >= 5 && ((d->music >> (k - 5)) & 1);
    orc_dpc_update(e);
    d->random = orc_dpc_next_random(d->random);
    if (!music) {
        const unsigned low = d->counter[k] & 0xFFu;
        if (low == d->top[k]) d->flags |= (uint8_t)(1u << k);
        else if (low == d->bottom[k]) d->flags &= (uint8_t)~(1u << k);
    }
    const uint8_t flag = ((d->flags >> k) & 1) ? 0xFF : 0x00;
    const uint8_t data = e->rom[8192 + 2047 - d->counter[k]];
    uint8_t v = 0;
    switch (f) {
    case 0:
        if (k < 4) v = d->random;
        else
            for (int m = 0; m < 3; m++)
                if (((d->music >> m) & 1) && ((d->flags >> (5 + m)) & 1)) v = (uint8_t)(v + 4 + m);
        break;
    case 1: v = data; break;
    case 2: v = data & flag; break;
    case 7: v = flag; break;
    default: break;
    }
    if (!music) d->counter[k] = (uint16_t)((d->counter[k] - 1u) & 0x7FFu);
    return v;
}

static void orc_dpc_write(orc_atari* e, uint16_t a, uint8_t v)
{
    orc_dpc* d = &e->dpc;
    const int k = a & 7, f = (a >> 3) & 7;
    orc_dpc_update(e);
    switch (f) {
    case 0: d->top[k] = v; d->flags &= (uint8_t)~(1u << k); break;
    case 1: d->bottom[k] = v; break;
    case 2: d->counter[k] = (uint16_t)((d->counter[k] & 0x700u) | v); break;
    case 3:
        d->counter[k] = (uint16_t)(((v & 7u) << 8) | (d->counter[k] & 0xFFu));
        if (k >= 5) d->music = (uint8_t)((d->music & ~(1u << (k - 5))) | (((v >> 4) & 1u) << (k - 5)));
        break;
    case 6: d->random = 1; break;
    default: break;
    }
}

/* FE (Activision): an access after one to $01FE selects the 4K bank by bit 5
 * of its data (set: bank 0, clear: bank 1); the access itself is served from
 * the mapping before the switch.  The reference has no FE cart: this is the
 * published behaviour of these carts, for every access the reference CPU
 * makes (phantom ones included). */
static inline void orc_fe_note(orc_atari* e, uint16_t a13, uint8_t v)
{
    if (e->fe_pend) {
        const int b = (v & 0x20) ? 0 : 1;
        for (int w = 0; w < 4; w++) {
            e->slice[w] = 4 * b + w;
            orc_load_window(e, w);
        }
    }
    e->fe_pend = a13 == 0x01FE;
}

static inline uint8_t orc_bus_read_value(orc_atari* e, uint16_t addr);

static inline uint8_t orc_bus_read(orc_atari* e, uint16_t addr)
{
    const uint8_t v = orc_bus_read_value(e, addr);
    if (e->scheme == FA_SCHEME_FE) orc_fe_note(e, (uint16_t)(addr & 0x1FFF), v);
    return v;
}

static inline uint8_t orc_bus_read_value(orc_atari* e, uint16_t addr) /* atari.rs:497-520 */
{
    uint16_t a = addr & 0x1FFF;
    if (e->scheme == FA_SCHEME_DPC && (a & 0x1FC0) == 0x1000) return orc_dpc_read(e, a);
    if ((a & 0x1080) != 0 && (a & 0x1280) != 0x0280) {
        if ((a & 0x1000) && e->scheme != FA_SCHEME_FIXED) orc_check_bankswitch(e, addr);
        return e->mem[a];
    }
    if ((a & 0x1280) == 0x0280) return orc_pia_read(&e->pia, a);
    if ((a & 0x1080) == 0) return orc_tia_read(&e->tia, a);
    return 0;
}

static inline void orc_bus_write(orc_atari* e, uint16_t addr, uint8_t v) /* atari.rs:523-552 */
{
    uint16_t a = addr & 0x1FFF;
    if (e->scheme == FA_SCHEME_FE) orc_fe_note(e, a, v);
    if (a & 0x1000) {
        if (e->scheme == FA_SCHEME_DPC && (a & 0x1FC0) == 0x1040) orc_dpc_write(e, a, v);
        if (e->scheme != FA_SCHEME_FIXED) orc_check_bankswitch(e, addr);
        return;
    }
    if ((a & 0x80) && !(a & 0x200)) {
        e->pia.ram[a & 0x7F] = v;
        e->mem[(a | 0x80) & 0x1FF] = v;
        e->mem[((a | 0x80) & 0x1FF) ^ 0x100] = v;
        return;
    }
    if (a & 0x200) { orc_pia_write(&e->pia, a, v); return; }
    if (e->scheme == FA_SCHEME_3F && a < 0x40) {   /* 3F: the written value selects the 2K bank at $1000 */
        const int b = (int)(v % (e->rom_len / 2048));
        e->slice[0] = 2 * b;
        e->slice[1] = 2 * b + 1;
        orc_load_window(e, 0);
        orc_load_window(e, 1);
    }
    orc_tia_write(&e->tia, a, v);
}

/* Phantom accesses on the headless bus are issued unless a test switches
 * them off (orc_set_phantoms): with them off the oracle behaves like a core
 * that skips them, as the reference's CUDA kernels do, which lets a test
 * show that a cart depends on them. */
static int orc_phantoms = 1;

void orc_set_phantoms(int on) { orc_phantoms = on != 0; }

/* Cpu::step on the Atari bus. */
#define STEP_FN orc_step_bus
#define MEM_T orc_atari
#define MREAD(m, a) orc_bus_read((m), (uint16_t)(a))
#define MWRITE(m, a, v) orc_bus_write((m), (uint16_t)(a), (uint8_t)(v))
#define PHANTOM_READ(m, a) do { if (orc_phantoms) (void)MREAD(m, a); } while (0)
#define RMW_OLD_WRITE(m, a, v) do { if (orc_phantoms) MWRITE(m, a, v); } while (0)
#include "cpu_step.h"
#undef STEP_FN
#undef MEM_T
#undef MREAD
#undef MWRITE
#undef PHANTOM_READ
#undef RMW_OLD_WRITE

/* Cpu::step on FlatMemory (cpu.rs:69-90). */
typedef struct orc_flat { uint8_t* ram; } orc_flat;
#define STEP_FN orc_step_flat
#define MEM_T orc_flat
#define MREAD(m, a) ((m)->ram[(uint16_t)(a)])
#define MWRITE(m, a, v) ((m)->ram[(uint16_t)(a)] = (uint8_t)(v))
#define PHANTOM_READ(m, a) ((void)MREAD(m, a))
#define RMW_OLD_WRITE(m, a, v) MWRITE(m, a, v)
#include "cpu_step.h"
#undef PHANTOM_READ
#undef RMW_OLD_WRITE
#undef STEP_FN
#undef MEM_T
#undef MREAD
#undef MWRITE

static void orc_cpu_reset_bus(orc_atari* e)                        /* cpu.rs:125-134 */
{
    uint16_t lo = orc_bus_read(e, 0xFFFC);
    uint16_t hi = orc_bus_read(e, 0xFFFD);
    e->cpu.pc = (uint16_t)((hi << 8) | lo);
    e->cpu.sp = 0xFD;
    e->cpu.p = 0;
    e->cpu.a = e->cpu.x = e->cpu.y = 0;
}

orc_atari* orc_create(const uint8_t* rom, size_t rom_len)          /* atari.rs:410-430, 562-569 */
{
    const int scheme = orc_scheme_for(rom, rom_len);
    if (scheme < 0) return NULL;
    orc_atari* e = (orc_atari*)calloc(1, sizeof(orc_atari));
    if (!e) return NULL;
    e->rom = (uint8_t*)malloc(rom_len);
    if (!e->rom) { free(e); return NULL; }
    memcpy(e->rom, rom, rom_len);
    e->rom_len = rom_len;
    e->scheme = scheme;
    switch (e->scheme) {
    case FA_SCHEME_FIXED: e->bank = 0; break;
    case FA_SCHEME_F8: e->bank = 1; break;
    case FA_SCHEME_F6: e->bank = 3; break;
    case FA_SCHEME_E0: case FA_SCHEME_3F: case FA_SCHEME_DPC: case FA_SCHEME_FE:
        e->bank = 0;
        orc_power_on_slices(scheme, rom_len, e->slice);
        break;
    default: e->bank = 7; break;
    }
    if (scheme == FA_SCHEME_DPC) e->dpc.random = 1;
    orc_tia_default(&e->tia);
    orc_pia_default(&e->pia);
    e->cpu.sp = 0xFD;                                              /* Cpu::default, cpu.rs:107-119 */
    orc_load_bank(e, e->bank);
    orc_sync_ram_to_mem(e);
    orc_cpu_reset_bus(e);
    return e;
}

orc_atari* orc_clone(const orc_atari* e)
{
    orc_atari* c = (orc_atari*)malloc(sizeof(orc_atari));
    if (!c) return NULL;
    memcpy(c, e, sizeof(*c));
    c->rom = (uint8_t*)malloc(e->rom_len);
    if (!c->rom) { free(c); return NULL; }
    memcpy(c->rom, e->rom, e->rom_len);
    return c;
}

void orc_destroy(orc_atari* e)
{
    if (!e) return;
    free(e->rom);
    free(e);
}

void orc_set_action(orc_atari* e, unsigned action)                 /* atari.rs:34-81, 571-582 */
{
    /* (up, down, left, right, fire) per Action::decode, indexed by from_index */
    static const uint8_t dec[18][5] = {
        {0,0,0,0,0}, {0,0,0,0,1}, {1,0,0,0,0}, {0,0,0,1,0}, {0,0,1,0,0}, {0,1,0,0,0},
        {1,0,0,1,0}, {1,0,1,0,0}, {0,1,0,1,0}, {0,1,1,0,0}, {1,0,0,0,1}, {0,0,0,1,1},
        {0,0,1,0,1}, {0,1,0,0,1}, {1,0,0,1,1}, {1,0,1,0,1}, {0,1,0,1,1}, {0,1,1,0,1},
    };
    const uint8_t* d = dec[action < 18 ? action : 0];
    uint8_t swcha = 0xFF;
    if (d[0]) swcha &= (uint8_t)~0x10;
    if (d[1]) swcha &= (uint8_t)~0x20;
    if (d[2]) swcha &= (uint8_t)~0x40;
    if (d[3]) swcha &= (uint8_t)~0x80;
    e->pia.pa_in = swcha;
    e->tia.inpt4 = !d[4];
    e->tia.paddle0 = d[2] ? 200 : (d[3] ? 50 : 128);
}

static inline int orc_run_one_cycle(orc_atari* e, uint64_t* cycles) /* atari.rs:601-614 */
{
    if (e->tia.wsync) {
        uint16_t skipped = orc_tia_skip_to_scanline_end(&e->tia);
        orc_pia_tick_n(&e->pia, skipped);
        *cycles += skipped;
    } else {
        uint8_t c = orc_step_bus(&e->cpu, e);
        if (c == 0) { e->run_status |= FA_STATUS_ILLEGAL_OPCODE; return 0; }
        e->instructions++;
        *cycles += c;
        orc_tia_tick_n(&e->tia, c);
        orc_pia_tick_n(&e->pia, c);
    }
    return 1;
}

uint64_t orc_run_frame(orc_atari* e)                               /* atari.rs:584-598 */
{
    if (e->run_status & FA_STATUS_HALT_MASK) return 0;
    e->tia.frame_complete = 0;
    uint64_t cycles = 0;
    while (e->tia.vsync & 0x02) {
        if (!orc_run_one_cycle(e, &cycles)) return cycles;
        /* The reference has no bound here; a ROM that holds VSYNC forever
         * hangs it.  The oracle and the device stop such an instance. */
        if (cycles > FA_VSYNC_BUDGET) { e->run_status |= FA_STATUS_VSYNC_BUDGET; return cycles; }
    }
    while (!(e->tia.vsync & 0x02)) {
        if (!orc_run_one_cycle(e, &cycles)) return cycles;
        if (cycles > FA_FRAME_CYCLE_CAP) { e->run_status |= FA_STATUS_CYCLE_CAP; break; }
    }
    e->frame_no++;
    return cycles;
}

void orc_ram(const orc_atari* e, uint8_t* out128)                  /* atari.rs:617-619 */
{
    memcpy(out128, &e->mem[0x80], 128);
}

uint64_t orc_instructions(const orc_atari* e) { return e->instructions; }

void orc_get_state(const orc_atari* e, fa_state* s)                /* cuda_env.rs:44-93 */
{
    const orc_tia* t = &e->tia;
    const orc_pia* p = &e->pia;
    memset(s, 0, sizeof(*s));
    s->a = e->cpu.a; s->x = e->cpu.x; s->y = e->cpu.y; s->sp = e->cpu.sp;
    s->pc = e->cpu.pc; s->status = e->cpu.p;
    memcpy(s->ram, p->ram, 128);
    s->port_a_output = p->pa_out; s->port_a_ddr = p->pa_ddr; s->port_a_input = p->pa_in;
    s->port_b_output = p->pb_out; s->port_b_ddr = p->pb_ddr; s->port_b_input = p->pb_in;
    s->timer_value = p->timer_value; s->timer_prescaler = p->timer_prescaler;
    s->timer_prescaler_select = p->timer_select; s->timer_underflow = p->timer_underflow;
    s->tia_clock = t->clock; s->tia_scanline = t->scanline;
    s->tia_wsync = t->wsync; s->tia_frame_complete = t->frame_complete;
    s->tia_vsync = t->vsync; s->tia_vblank = t->vblank;
    s->cxm0p = t->cx[0]; s->cxm1p = t->cx[1]; s->cxp0fb = t->cx[2]; s->cxp1fb = t->cx[3];
    s->cxm0fb = t->cx[4]; s->cxm1fb = t->cx[5]; s->cxblpf = t->cx[6]; s->cxppmm = t->cx[7];
    s->inpt4 = t->inpt4; s->inpt5 = t->inpt5; s->paddle0 = t->paddle0; s->paddle1 = t->paddle1;
    s->paddle_counter = t->paddle_counter; s->paddle_dumped = t->paddle_dumped;
    s->pos_p0 = t->pos[0]; s->pos_p1 = t->pos[1]; s->pos_m0 = t->pos[2];
    s->pos_m1 = t->pos[3]; s->pos_bl = t->pos[4];
    s->hmp0 = t->hm[0]; s->hmp1 = t->hm[1]; s->hmm0 = t->hm[2]; s->hmm1 = t->hm[3]; s->hmbl = t->hm[4];
    s->grp0 = t->grp0; s->grp1 = t->grp1; s->grp0_old = t->grp0_old; s->grp1_old = t->grp1_old;
    s->enam0 = t->enam0; s->enam1 = t->enam1; s->enabl = t->enabl; s->enabl_old = t->enabl_old;
    s->vdelp0 = t->vdelp0; s->vdelp1 = t->vdelp1; s->vdelbl = t->vdelbl;
    s->resmp0 = t->resmp0; s->resmp1 = t->resmp1; s->nusiz0 = t->nusiz0; s->nusiz1 = t->nusiz1;
    s->colup0 = t->colup0; s->colup1 = t->colup1; s->colupf = t->colupf; s->colubk = t->colubk;
    s->ctrlpf = t->ctrlpf; s->refp0 = t->refp0; s->refp1 = t->refp1;
    s->pf0 = t->pf0; s->pf1 = t->pf1; s->pf2 = t->pf2;
    s->bank = (uint8_t)e->bank; s->scheme = (uint8_t)e->scheme;
    const unsigned m = orc_mapper_of(e->scheme, e->slice) | (e->scheme == FA_SCHEME_FE && e->fe_pend ? 0x100u : 0u);
    s->mapper[0] = (uint8_t)m; s->mapper[1] = (uint8_t)(m >> 8);
    s->cycles = e->cpu.cycles;
    s->frame_no = e->frame_no;
    s->run_status = e->run_status;
    memcpy(s->dpc_counter, e->dpc.counter, sizeof(s->dpc_counter));
    memcpy(s->dpc_top, e->dpc.top, 8);
    memcpy(s->dpc_bottom, e->dpc.bottom, 8);
    s->dpc_flags = e->dpc.flags; s->dpc_music = e->dpc.music; s->dpc_random = e->dpc.random;
    s->dpc_osc = e->dpc.osc;
}

void orc_set_state(orc_atari* e, const fa_state* s)
{
    orc_tia* t = &e->tia;
    orc_pia* p = &e->pia;
    e->cpu.a = s->a; e->cpu.x = s->x; e->cpu.y = s->y; e->cpu.sp = s->sp;
    e->cpu.pc = s->pc; e->cpu.p = s->status; e->cpu.cycles = s->cycles;
    memcpy(p->ram, s->ram, 128);
    p->pa_out = s->port_a_output; p->pa_ddr = s->port_a_ddr; p->pa_in = s->port_a_input;
    p->pb_out = s->port_b_output; p->pb_ddr = s->port_b_ddr; p->pb_in = s->port_b_input;
    p->timer_value = s->timer_value; p->timer_prescaler = s->timer_prescaler;
    p->timer_select = s->timer_prescaler_select; p->timer_underflow = s->timer_underflow;
    t->clock = s->tia_clock; t->scanline = s->tia_scanline;
    t->wsync = s->tia_wsync; t->frame_complete = s->tia_frame_complete;
    t->vsync = s->tia_vsync; t->vblank = s->tia_vblank;
    t->cx[0] = s->cxm0p; t->cx[1] = s->cxm1p; t->cx[2] = s->cxp0fb; t->cx[3] = s->cxp1fb;
    t->cx[4] = s->cxm0fb; t->cx[5] = s->cxm1fb; t->cx[6] = s->cxblpf; t->cx[7] = s->cxppmm;
    t->inpt4 = s->inpt4; t->inpt5 = s->inpt5; t->paddle0 = s->paddle0; t->paddle1 = s->paddle1;
    t->paddle_counter = s->paddle_counter; t->paddle_dumped = s->paddle_dumped;
    t->pos[0] = s->pos_p0; t->pos[1] = s->pos_p1; t->pos[2] = s->pos_m0;
    t->pos[3] = s->pos_m1; t->pos[4] = s->pos_bl;
    t->hm[0] = s->hmp0; t->hm[1] = s->hmp1; t->hm[2] = s->hmm0; t->hm[3] = s->hmm1; t->hm[4] = s->hmbl;
    t->grp0 = s->grp0; t->grp1 = s->grp1; t->grp0_old = s->grp0_old; t->grp1_old = s->grp1_old;
    t->enam0 = s->enam0; t->enam1 = s->enam1; t->enabl = s->enabl; t->enabl_old = s->enabl_old;
    t->vdelp0 = s->vdelp0; t->vdelp1 = s->vdelp1; t->vdelbl = s->vdelbl;
    t->resmp0 = s->resmp0; t->resmp1 = s->resmp1; t->nusiz0 = s->nusiz0; t->nusiz1 = s->nusiz1;
    t->colup0 = s->colup0; t->colup1 = s->colup1; t->colupf = s->colupf; t->colubk = s->colubk;
    t->ctrlpf = s->ctrlpf; t->refp0 = s->refp0; t->refp1 = s->refp1;
    t->pf0 = s->pf0; t->pf1 = s->pf1; t->pf2 = s->pf2;
    e->frame_no = s->frame_no;
    e->run_status = s->run_status;
    memset(&e->dpc, 0, sizeof(e->dpc));                /* other schemes: the DPC fields are not taken */
    if (e->scheme == FA_SCHEME_DPC) {
        memcpy(e->dpc.counter, s->dpc_counter, sizeof(e->dpc.counter));
        for (int k = 0; k < 8; k++) e->dpc.counter[k] &= 0x7FFu;
        memcpy(e->dpc.top, s->dpc_top, 8);
        memcpy(e->dpc.bottom, s->dpc_bottom, 8);
        e->dpc.flags = s->dpc_flags; e->dpc.music = s->dpc_music & 7u; e->dpc.random = s->dpc_random;
        e->dpc.osc = s->dpc_osc;
    }
    /* The bank index is clamped to the scheme's range when the flat array is
     * rebuilt; the scheme itself always follows the ROM. */
    int nb = s->bank;
    int maxb = e->scheme == FA_SCHEME_F8 ? 1 : e->scheme == FA_SCHEME_F6 ? 3 : e->scheme == FA_SCHEME_F4 ? 7 : 0;
    if (nb > maxb) nb = maxb;
    e->bank = nb;
    if (orc_sliced(e->scheme))
        orc_slices_of(e->scheme, e->rom_len, (unsigned)s->mapper[0] | ((unsigned)s->mapper[1] << 8), e->slice);
    e->fe_pend = e->scheme == FA_SCHEME_FE && (s->mapper[1] & 1);
    orc_load_bank(e, nb);
    orc_sync_ram_to_mem(e);
}

int orc_reset_state(const uint8_t* rom, size_t rom_len, fa_state* out) /* cuda_env.rs:134-139 */
{
    orc_atari* e = orc_create(rom, rom_len);
    if (!e) return -1;
    orc_run_frame(e);
    e->frame_no = 0;
    orc_get_state(e, out);
    orc_destroy(e);
    return 0;
}

/* ------------------------------------------------------- batch runner (CPU) */
typedef struct orc_job {
    const uint8_t* rom; size_t rom_len; size_t n; int k;
    fa_state* states; const uint8_t* actions; const fa_state* snapshot;
    uint32_t episode_frames; uint8_t* obs; uint8_t* trace;
    int tid, nthreads, pin, err;
    uint64_t instructions;
} orc_job;

static void* orc_worker(void* arg)
{
    orc_job* j = (orc_job*)arg;
    if (j->pin) {
        cpu_set_t set;
        CPU_ZERO(&set);
        CPU_SET(j->tid, &set);
        pthread_setaffinity_np(pthread_self(), sizeof(set), &set);
    }
    orc_atari* e = orc_create(j->rom, j->rom_len);
    if (!e) { j->err = 1; return NULL; }
    /* Contiguous instance range per thread: one emulator per core at a time,
     * as the reference CPU benchmark runs one HeadlessAtari per OS thread. */
    size_t per = (j->n + (size_t)j->nthreads - 1) / (size_t)j->nthreads;
    size_t lo = per * (size_t)j->tid, hi = lo + per;
    if (hi > j->n) hi = j->n;
    for (size_t i = lo; i < hi; i++) {
        orc_set_state(e, &j->states[i]);
        uint64_t before = e->instructions;
        for (int f = 0; f < j->k; f++) {
            if (j->episode_frames && e->frame_no >= j->episode_frames && j->snapshot)
                orc_set_state(e, j->snapshot);
            orc_set_action(e, j->actions[(size_t)f * j->n + i]);
            orc_run_frame(e);
            if (j->trace) orc_ram(e, &j->trace[((size_t)f * j->n + i) * 128]);
        }
        j->instructions += e->instructions - before;
        orc_get_state(e, &j->states[i]);
        if (j->obs) orc_ram(e, &j->obs[i * 128]);
    }
    orc_destroy(e);
    return NULL;
}

static uint64_t orc_run_batch_impl(const uint8_t* rom, size_t rom_len, size_t n, int k,
                                   fa_state* states, const uint8_t* actions,
                                   const fa_state* snapshot, uint32_t episode_frames,
                                   uint8_t* obs, uint8_t* trace, int nthreads, int pin)
{
    if (!rom || !states || (k > 0 && !actions) || k < 0 || orc_scheme_for(rom, rom_len) < 0) return (uint64_t)-1;
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > n && n > 0) nthreads = (int)n;
    orc_job* jobs = (orc_job*)calloc((size_t)nthreads, sizeof(orc_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return (uint64_t)-1; }
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = (orc_job){ rom, rom_len, n, k, states, actions, snapshot, episode_frames,
                             obs, trace, t, nthreads, pin, 0, 0 };
    }
    for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, orc_worker, &jobs[t]);
    orc_worker(&jobs[0]);
    uint64_t total = jobs[0].instructions;
    int err = jobs[0].err;
    for (int t = 1; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        total += jobs[t].instructions;
        err |= jobs[t].err;
    }
    free(jobs);
    free(th);
    return err ? (uint64_t)-1 : total;
}

uint64_t orc_run_batch(const uint8_t* rom, size_t rom_len, size_t n, int k,
                       fa_state* states, const uint8_t* actions,
                       const fa_state* snapshot, uint32_t episode_frames,
                       uint8_t* obs, int nthreads, int pin)
{
    return orc_run_batch_impl(rom, rom_len, n, k, states, actions, snapshot,
                              episode_frames, obs, NULL, nthreads, pin);
}

uint64_t orc_run_batch_trace(const uint8_t* rom, size_t rom_len, size_t n, int k,
                             fa_state* states, const uint8_t* actions,
                             const fa_state* snapshot, uint32_t episode_frames,
                             uint8_t* ram_trace, int nthreads)
{
    return orc_run_batch_impl(rom, rom_len, n, k, states, actions, snapshot,
                              episode_frames, NULL, ram_trace, nthreads, 0);
}

/* ------------------------------------------------- FlatMemory KAT runner */
int orc_flat_run_from(uint8_t* mem64k, int nsteps, uint8_t* cycles_out, orc_regs* r)
{
    orc_cpu c = { r->pc, r->sp, r->a, r->x, r->y, r->p, r->cycles };
    orc_flat m = { mem64k };
    int i;
    for (i = 0; i < nsteps; i++) {
        uint8_t cy = orc_step_flat(&c, &m);
        if (cycles_out) cycles_out[i] = cy;
        if (cy == 0) break;
    }
    r->pc = c.pc; r->sp = c.sp; r->a = c.a; r->x = c.x; r->y = c.y; r->p = c.p; r->cycles = c.cycles;
    return i;
}

int orc_flat_run(uint8_t* mem64k, int nsteps, uint8_t* cycles_out, orc_regs* r)
{
    /* Cpu::new + Cpu::reset (cpu.rs:107-134) */
    orc_regs s;
    memset(&s, 0, sizeof(s));
    s.pc = (uint16_t)(mem64k[0xFFFC] | (mem64k[0xFFFD] << 8));
    s.sp = 0xFD;
    int n = orc_flat_run_from(mem64k, nsteps, cycles_out, &s);
    *r = s;
    return n;
}

size_t orc_state_size(void) { return sizeof(fa_state); }

/* ======================================================== rendering console
 * The reference's rendering path, restated: the pixel-accurate Tia
 * (src/tia.rs), the per-cycle Bus (src/atari.rs:107-225), the Atari console
 * (src/atari.rs:227-306) and Pia::tick (src/pia.rs:80-103).  The 6502 issues
 * one bus access per cycle (cpu_step.h); every access ticks the TIA three
 * times and the PIA once, and a write lands on the third TIA clock of its
 * cycle (the Gopher2600 timing of Bus::write, src/atari.rs:206-222). */

#define R_FRAME_W 160
#define R_FRAME_H 192
#define R_EXT_TOP 23                 /* tia.rs:84-86 */
#define R_IDEAL_TOP 32
#define R_RESIZE_FRAMES 3
#define R_DELAYED_CAP 4              /* tia.rs:89 */

typedef struct { uint8_t remaining, reg, value; } orc_delayed;

typedef struct orc_rtia {            /* Tia, tia.rs:98-190 */
    uint16_t clock, scanline;
    uint8_t  wsync, hmove_pending;
    uint16_t visible_top, vblank_top, pending_top;
    uint8_t  pending_frames;
    orc_delayed delayed[R_DELAYED_CAP];
    uint8_t  delayed_len;
    uint8_t  frame_complete;
    uint8_t  vsync, vblank, colup0, colup1, colupf, colubk, ctrlpf, refp0, refp1, pf0, pf1, pf2;
    uint8_t  grp0, grp1, grp0_old, grp1_old, enam0, enam1, enabl, enabl_old;
    uint8_t  hmp0, hmp1, hmm0, hmm1, hmbl, nusiz0, nusiz1, vdelp0, vdelp1, vdelbl, resmp0, resmp1;
    uint16_t pos_p0, pos_p1, pos_m0, pos_m1, pos_bl;
    uint8_t  cxm0p, cxm1p, cxp0fb, cxp1fb, cxm0fb, cxm1fb, cxblpf, cxppmm;
    uint8_t  paddle0, paddle1;
    uint16_t paddle_counter;
    uint8_t  paddle_dumped;
    uint8_t  inpt4, inpt5, inpt4_latch, inpt5_latch, input_latch_enabled;
    uint8_t  fb[R_FRAME_W * R_FRAME_H];
} orc_rtia;

static void orc_rtia_default(orc_rtia* t)                          /* tia.rs:192-238 */
{
    memset(t, 0, sizeof(*t));
    t->visible_top = R_IDEAL_TOP;
    t->vblank_top = 262;
    t->pending_top = R_IDEAL_TOP;
    t->paddle0 = 128;
    t->paddle1 = 128;
    t->inpt4 = 1;
    t->inpt5 = 1;
    t->inpt4_latch = 0x80;
    t->inpt5_latch = 0x80;
}

static void orc_rtia_resize_commit(orc_rtia* t)                    /* tia.rs:247-268 */
{
    if (t->vblank_top > 262) return;
    uint16_t clamped = t->vblank_top < R_EXT_TOP ? R_EXT_TOP : t->vblank_top > R_IDEAL_TOP ? R_IDEAL_TOP : t->vblank_top;
    uint16_t candidate = clamped < t->visible_top ? clamped : t->visible_top;
    if (candidate != t->pending_top) {
        t->pending_top = candidate;
        t->pending_frames = R_RESIZE_FRAMES;
    } else if (t->pending_frames > 0) {
        t->pending_frames--;
        if (t->pending_frames == 0) t->visible_top = t->pending_top;
    }
    t->vblank_top = t->visible_top;
}

static int orc_rtia_pf_bit(const orc_rtia* t, uint8_t x)            /* tia.rs:406-420 */
{
    unsigned pf_x = x < 80 ? x / 4u : ((t->ctrlpf & 0x01) ? 19u - (unsigned)(x - 80) / 4u : (unsigned)(x - 80) / 4u);
    if (pf_x <= 3) return (t->pf0 & (0x10u << pf_x)) != 0;
    if (pf_x <= 11) return (t->pf1 & (0x80u >> (pf_x - 4))) != 0;
    if (pf_x <= 19) return (t->pf2 & (0x01u << (pf_x - 12))) != 0;
    return 0;
}

/* NUSIZ copy offsets (tia.rs:440-450, 480-488). */
static const uint16_t orc_copies[8][4] = {
    {1, 0, 0, 0}, {2, 0, 16, 0}, {2, 0, 32, 0}, {3, 0, 16, 32}, {2, 0, 64, 0}, {1, 0, 0, 0}, {3, 0, 32, 64}, {1, 0, 0, 0},
};

static int orc_rtia_player(const orc_rtia* t, int player, uint8_t x) /* tia.rs:423-465 */
{
    uint8_t grp = player ? (t->vdelp1 ? t->grp1_old : t->grp1) : (t->vdelp0 ? t->grp0_old : t->grp0);
    uint16_t pos = player ? t->pos_p1 : t->pos_p0;
    uint8_t refp = player ? t->refp1 : t->refp0;
    uint8_t nusiz = player ? t->nusiz1 : t->nusiz0;
    if (grp == 0) return 0;
    unsigned size_mode = nusiz & 7u;
    uint16_t pixel_width = size_mode == 5 ? 2 : size_mode == 7 ? 4 : 1;
    uint16_t pixel_span = (uint16_t)(8 * pixel_width);
    for (unsigned c = 0; c < orc_copies[size_mode][0]; c++) {
        uint16_t copy_pos = (uint16_t)((pos + orc_copies[size_mode][1 + c]) % 160);
        uint16_t offset = (uint16_t)((x + 160 - copy_pos) % 160);
        if (offset < pixel_span && offset < 80) {
            uint16_t bit = offset / pixel_width;
            int hit = refp ? (grp & (0x01u << bit)) != 0 : (grp & (0x80u >> bit)) != 0;
            if (hit) return 1;
        }
    }
    return 0;
}

static int orc_rtia_missile(const orc_rtia* t, int m, uint8_t x)    /* tia.rs:468-497 */
{
    uint8_t enabled = m ? t->enam1 : t->enam0;
    uint16_t pos = m ? t->pos_m1 : t->pos_m0;
    uint8_t nusiz = m ? t->nusiz1 : t->nusiz0;
    uint8_t resmp = m ? t->resmp1 : t->resmp0;
    if (!enabled || resmp) return 0;
    uint16_t width = (uint16_t)(1u << ((nusiz >> 4) & 3u));
    unsigned mode = nusiz & 7u;
    for (unsigned c = 0; c < orc_copies[mode][0]; c++) {
        uint16_t copy_pos = (uint16_t)((pos + orc_copies[mode][1 + c]) % 160);
        uint16_t offset = (uint16_t)((x + 160 - copy_pos) % 160);
        if (offset < width && offset < 80) return 1;
    }
    return 0;
}

static int orc_rtia_ball(const orc_rtia* t, uint8_t x)              /* tia.rs:500-507 */
{
    uint8_t enabled = t->vdelbl ? t->enabl_old : t->enabl;
    if (!enabled) return 0;
    uint16_t width = (uint16_t)(1u << ((t->ctrlpf >> 4) & 3u));
    uint16_t offset = (uint16_t)((x + 160 - t->pos_bl) % 160);
    return offset < width && offset < 80;
}

static void orc_rtia_tick(orc_rtia* t)                              /* tia.rs:271-372 */
{
    if (t->input_latch_enabled) {
        if (!t->inpt4) t->inpt4_latch = 0x00;
        if (!t->inpt5) t->inpt5_latch = 0x00;
    }
    if (!(t->vblank & 0x02) && t->scanline >= R_EXT_TOP && t->scanline < t->vblank_top) t->vblank_top = t->scanline;
    if (t->delayed_len > 0) {
        unsigned dst = 0;
        for (unsigned i = 0; i < t->delayed_len; i++) {
            orc_delayed e = t->delayed[i];
            e.remaining--;
            if (e.remaining == 0) {
                if (e.reg == 0x0D) t->pf0 = e.value;
                else if (e.reg == 0x0E) t->pf1 = e.value;
                else if (e.reg == 0x0F) t->pf2 = e.value;
            } else {
                t->delayed[dst++] = e;
            }
        }
        t->delayed_len = (uint8_t)dst;
    }
    uint16_t pixel_x = (uint16_t)(t->clock - 68);
    uint16_t vis_line = (uint16_t)(t->scanline - t->visible_top);
    if (t->clock >= 68 && pixel_x < R_FRAME_W && !(t->vblank & 0x02) && vis_line < R_FRAME_H) {
        uint8_t x = (uint8_t)pixel_x;
        int pf = orc_rtia_pf_bit(t, x), p0 = orc_rtia_player(t, 0, x), p1 = orc_rtia_player(t, 1, x);
        int m0 = orc_rtia_missile(t, 0, x), m1 = orc_rtia_missile(t, 1, x), bl = orc_rtia_ball(t, x);
        uint8_t pf_color = (t->ctrlpf & 0x02) ? (x < 80 ? t->colup0 : t->colup1) : t->colupf;    /* :382-389 */
        uint8_t color;
        if (t->ctrlpf & 0x04) color = (pf || bl) ? pf_color : (p0 || m0) ? t->colup0 : (p1 || m1) ? t->colup1 : t->colubk;
        else color = (p0 || m0) ? t->colup0 : (p1 || m1) ? t->colup1 : (pf || bl) ? pf_color : t->colubk;
        if (t->hmove_pending && pixel_x < 8) color = t->colubk;
        t->fb[vis_line * R_FRAME_W + pixel_x] = color;
        if (m0 && p1) t->cxm0p |= 0x80;
        if (m0 && p0) t->cxm0p |= 0x40;
        if (m1 && p0) t->cxm1p |= 0x80;
        if (m1 && p1) t->cxm1p |= 0x40;
        if (p0 && pf) t->cxp0fb |= 0x80;
        if (p0 && bl) t->cxp0fb |= 0x40;
        if (p1 && pf) t->cxp1fb |= 0x80;
        if (p1 && bl) t->cxp1fb |= 0x40;
        if (m0 && pf) t->cxm0fb |= 0x80;
        if (m0 && bl) t->cxm0fb |= 0x40;
        if (m1 && pf) t->cxm1fb |= 0x80;
        if (m1 && bl) t->cxm1fb |= 0x40;
        if (bl && pf) t->cxblpf |= 0x80;
        if (p0 && p1) t->cxppmm |= 0x80;
        if (m0 && m1) t->cxppmm |= 0x40;
    }
    t->clock++;
    if (t->clock >= 228) {
        t->clock = 0;
        t->scanline++;
        t->wsync = 0;
        t->hmove_pending = 0;
        if (t->scanline == t->visible_top) memset(t->fb, 0, sizeof(t->fb));
        if (!t->paddle_dumped && t->paddle_counter < 256) t->paddle_counter++;
        if (t->scanline >= 262) { t->scanline = 0; t->frame_complete = 1; }
    }
}

static uint16_t orc_rtia_resp(const orc_rtia* t)                    /* tia.rs:512-520: players */
{
    uint16_t delay = t->clock < 68 ? 3 : 4;
    uint16_t draw_clock = (uint16_t)((t->clock + delay + 156) % 228);
    return draw_clock >= 68 ? (uint16_t)(draw_clock - 68) : (uint16_t)(draw_clock + 160 - 68);
}

static uint16_t orc_rtia_resp_simple(const orc_rtia* t)             /* tia.rs:523-525: missiles, ball */
{
    int r = ((int)t->clock - 68 + 5) % 160;
    return (uint16_t)(r < 0 ? r + 160 : r);
}

static uint8_t orc_rtia_read(const orc_rtia* t, uint16_t addr)      /* tia.rs:533-566 */
{
    switch (addr & 0x0F) {
    case 0x0: return t->cxm0p;
    case 0x1: return t->cxm1p;
    case 0x2: return t->cxp0fb;
    case 0x3: return t->cxp1fb;
    case 0x4: return t->cxm0fb;
    case 0x5: return t->cxm1fb;
    case 0x6: return t->cxblpf;
    case 0x7: return t->cxppmm;
    case 0x8: return t->paddle_counter >= t->paddle0 ? 0x80 : 0x00;
    case 0x9: return t->paddle_counter >= t->paddle1 ? 0x80 : 0x00;
    case 0xA: case 0xB: return 0x80;
    case 0xC: return t->input_latch_enabled ? t->inpt4_latch : (t->inpt4 ? 0x80 : 0x00);
    case 0xD: return t->input_latch_enabled ? t->inpt5_latch : (t->inpt5 ? 0x80 : 0x00);
    default: return 0;
    }
}

static void orc_rtia_write(orc_rtia* t, uint16_t addr, uint8_t v)   /* tia.rs:570-674 */
{
    switch (addr & 0x3F) {
    case 0x00:
        if (!(t->vsync & 0x02) && (v & 0x02)) { orc_rtia_resize_commit(t); t->scanline = 0; t->frame_complete = 1; }
        t->vsync = v;
        break;
    case 0x01:
        if (v & 0x40) { t->input_latch_enabled = 1; t->inpt4_latch = 0x80; t->inpt5_latch = 0x80; }
        else t->input_latch_enabled = 0;
        if (v & 0x80) { t->paddle_counter = 0; t->paddle_dumped = 1; }
        else if (t->paddle_dumped) t->paddle_dumped = 0;
        t->vblank = v;
        break;
    case 0x02: t->wsync = 1; break;
    case 0x04: t->nusiz0 = v; break;
    case 0x05: t->nusiz1 = v; break;
    case 0x06: t->colup0 = v; break;
    case 0x07: t->colup1 = v; break;
    case 0x08: t->colupf = v; break;
    case 0x09: t->colubk = v; break;
    case 0x0A: t->ctrlpf = v; break;
    case 0x0B: t->refp0 = (v & 0x08) != 0; break;
    case 0x0C: t->refp1 = (v & 0x08) != 0; break;
    case 0x0D: case 0x0E: case 0x0F:
        if (t->delayed_len < R_DELAYED_CAP) {
            orc_delayed* e = &t->delayed[t->delayed_len++];
            e->remaining = 1;
            e->reg = (uint8_t)(addr & 0x3F);
            e->value = v;
        } else if ((addr & 0x3F) == 0x0D) t->pf0 = v;
        else if ((addr & 0x3F) == 0x0E) t->pf1 = v;
        else t->pf2 = v;
        break;
    case 0x10: t->pos_p0 = orc_rtia_resp(t); break;
    case 0x11: t->pos_p1 = orc_rtia_resp(t); break;
    case 0x12: t->pos_m0 = orc_rtia_resp_simple(t); break;
    case 0x13: t->pos_m1 = orc_rtia_resp_simple(t); break;
    case 0x14: t->pos_bl = orc_rtia_resp_simple(t); break;
    case 0x1B: t->grp0_old = t->grp0; t->grp0 = v; break;
    case 0x1C: t->grp1_old = t->grp1; t->grp1 = v; t->enabl_old = t->enabl; break;
    case 0x1D: t->enam0 = (v & 0x02) != 0; break;
    case 0x1E: t->enam1 = (v & 0x02) != 0; break;
    case 0x1F: t->enabl = (v & 0x02) != 0; break;
    case 0x20: t->hmp0 = v; break;
    case 0x21: t->hmp1 = v; break;
    case 0x22: t->hmm0 = v; break;
    case 0x23: t->hmm1 = v; break;
    case 0x24: t->hmbl = v; break;
    case 0x25: t->vdelp0 = v & 0x01; break;
    case 0x26: t->vdelp1 = v & 0x01; break;
    case 0x27: t->vdelbl = v & 0x01; break;
    case 0x28: t->resmp0 = (v & 0x02) != 0; break;
    case 0x29: t->resmp1 = (v & 0x02) != 0; break;
    case 0x2A:
        t->pos_p0 = orc_hmove(t->pos_p0, t->hmp0);
        t->pos_p1 = orc_hmove(t->pos_p1, t->hmp1);
        t->pos_m0 = orc_hmove(t->pos_m0, t->hmm0);
        t->pos_m1 = orc_hmove(t->pos_m1, t->hmm1);
        t->pos_bl = orc_hmove(t->pos_bl, t->hmbl);
        t->hmove_pending = 1;
        break;
    case 0x2B: t->hmp0 = t->hmp1 = t->hmm0 = t->hmm1 = t->hmbl = 0; break;
    case 0x2C: t->cxm0p = t->cxm1p = t->cxp0fb = t->cxp1fb = t->cxm0fb = t->cxm1fb = t->cxblpf = t->cxppmm = 0; break;
    default: break;                                                 /* RSYNC, audio */
    }
}

static void orc_pia_tick1(orc_pia* p)                              /* pia.rs:80-103 */
{
    if (p->timer_value == 0 && p->timer_underflow) { p->timer_value = 0xFF; return; }
    p->timer_prescaler = (uint16_t)(p->timer_prescaler - 1);
    if (p->timer_prescaler == 0) {
        p->timer_prescaler = p->timer_underflow ? 1 : p->timer_select;
        if (p->timer_value == 0) { p->timer_underflow = 1; p->timer_value = 0xFF; }
        else p->timer_value--;
    }
}

struct orc_ratari {
    orc_cpu  cpu;
    orc_rtia tia;
    orc_pia  pia;
    uint8_t* rom;
    size_t   rom_len;
    int      bank, scheme;
    int      slice[4];            /* E0 / 3F windows, as in orc_atari */
    uint32_t bus_ticks;
    uint32_t frame_no, run_status;
    uint64_t instructions;
};

static inline uint8_t orc_rrom_read(const orc_ratari* e, uint16_t addr) /* atari.rs:139-150 */
{
    if (e->scheme == FA_SCHEME_FIXED) return e->rom[(addr & 0x0FFF) % e->rom_len];
    if (orc_sliced(e->scheme)) return e->rom[(size_t)e->slice[(addr >> 10) & 3] * 1024 + (addr & 0x03FF)];
    size_t off = (size_t)e->bank * 4096 + (addr & 0x0FFF);
    return off < e->rom_len ? e->rom[off] : 0;
}

static inline void orc_rcheck_bankswitch(orc_ratari* e, uint16_t addr) /* atari.rs:153-180 */
{
    uint16_t a = addr & 0x1FFF;
    int first = e->scheme == FA_SCHEME_F8 ? 0x1FF8 : e->scheme == FA_SCHEME_F6 ? 0x1FF6 : e->scheme == FA_SCHEME_F4 ? 0x1FF4 : 0;
    int nb = e->scheme == FA_SCHEME_F8 ? 2 : e->scheme == FA_SCHEME_F6 ? 4 : e->scheme == FA_SCHEME_F4 ? 8 : 0;
    if (nb && a >= first && a < first + nb) e->bank = a - first;
    if (e->scheme == FA_SCHEME_E0 && a >= 0x1FE0 && a <= 0x1FF7) e->slice[(a - 0x1FE0) >> 3] = a & 7;
}

static inline void orc_rtick_components(orc_ratari* e)             /* atari.rs:273-279 */
{
    orc_rtia_tick(&e->tia);
    orc_rtia_tick(&e->tia);
    orc_rtia_tick(&e->tia);
    orc_pia_tick1(&e->pia);
}

static inline void orc_rtick_cycle(orc_ratari* e)                  /* atari.rs:186-192 */
{
    orc_rtick_components(e);
    e->bus_ticks++;
}

static uint8_t orc_rbus_read(orc_ratari* e, uint16_t addr)          /* atari.rs:195-205 */
{
    orc_rcheck_bankswitch(e, addr);
    uint16_t a = addr & 0x1FFF;
    uint8_t v;
    if ((a & 0x1080) == 0x0000) v = orc_rtia_read(&e->tia, a);
    else if ((a & 0x1280) == 0x0080 || (a & 0x1280) == 0x0280) v = orc_pia_read(&e->pia, a);
    else if (a & 0x1000) v = orc_rrom_read(e, a);
    else v = 0;
    orc_rtick_cycle(e);
    return v;
}

static void orc_rbus_write(orc_ratari* e, uint16_t addr, uint8_t v) /* atari.rs:207-222 */
{
    orc_rtia_tick(&e->tia);
    orc_rtia_tick(&e->tia);
    orc_rcheck_bankswitch(e, addr);
    uint16_t a = addr & 0x1FFF;
    if (e->scheme == FA_SCHEME_3F && a < 0x40) {   /* 3F bank select; the write also reaches the TIA */
        const int b = (int)(v % (e->rom_len / 2048));
        e->slice[0] = 2 * b;
        e->slice[1] = 2 * b + 1;
    }
    if ((a & 0x1080) == 0x0000) orc_rtia_write(&e->tia, a, v);
    else if ((a & 0x1280) == 0x0080 || (a & 0x1280) == 0x0280) orc_pia_write(&e->pia, a, v);
    orc_rtia_tick(&e->tia);
    orc_pia_tick1(&e->pia);
    e->bus_ticks++;
}

/* Cpu::step on the rendering bus. */
#define STEP_FN orc_step_rbus
#define MEM_T orc_ratari
#define MREAD(m, a) orc_rbus_read((m), (uint16_t)(a))
#define MWRITE(m, a, v) orc_rbus_write((m), (uint16_t)(a), (uint8_t)(v))
#define PHANTOM_READ(m, a) ((void)MREAD(m, a))
#define RMW_OLD_WRITE(m, a, v) MWRITE(m, a, v)
#include "cpu_step.h"
#undef PHANTOM_READ
#undef RMW_OLD_WRITE
#undef STEP_FN
#undef MEM_T
#undef MREAD
#undef MWRITE

orc_ratari* orc_rcreate(const uint8_t* rom, size_t rom_len)        /* atari.rs:120-136, 240-247 */
{
    const int scheme = orc_scheme_for(rom, rom_len);
    if (scheme < 0 || scheme == FA_SCHEME_DPC || scheme == FA_SCHEME_FE) return NULL;   /* headless only */
    orc_ratari* e = (orc_ratari*)calloc(1, sizeof(orc_ratari));
    if (!e) return NULL;
    e->rom = (uint8_t*)malloc(rom_len);
    if (!e->rom) { free(e); return NULL; }
    memcpy(e->rom, rom, rom_len);
    e->rom_len = rom_len;
    e->scheme = scheme;
    e->bank = e->scheme == FA_SCHEME_FIXED ? 0 : e->scheme == FA_SCHEME_F8 ? 1 : e->scheme == FA_SCHEME_F6 ? 3 : 7;
    if (orc_sliced(scheme)) { e->bank = 0; orc_power_on_slices(scheme, rom_len, e->slice); }
    orc_rtia_default(&e->tia);
    orc_pia_default(&e->pia);
    e->cpu.sp = 0xFD;                                              /* Cpu::default */
    uint16_t lo = orc_rbus_read(e, 0xFFFC);                        /* Cpu::reset, cpu.rs:125-134 */
    uint16_t hi = orc_rbus_read(e, 0xFFFD);
    e->cpu.pc = (uint16_t)((hi << 8) | lo);
    e->cpu.sp = 0xFD;
    e->cpu.p = 0;
    e->cpu.a = e->cpu.x = e->cpu.y = 0;
    return e;
}

orc_ratari* orc_rclone(const orc_ratari* e)
{
    orc_ratari* c = (orc_ratari*)malloc(sizeof(orc_ratari));
    if (!c) return NULL;
    memcpy(c, e, sizeof(*c));
    c->rom = (uint8_t*)malloc(e->rom_len);
    if (!c->rom) { free(c); return NULL; }
    memcpy(c->rom, e->rom, e->rom_len);
    return c;
}

void orc_rdestroy(orc_ratari* e)
{
    if (!e) return;
    free(e->rom);
    free(e);
}

void orc_rset_action(orc_ratari* e, unsigned action)              /* atari.rs:250-270 */
{
    static const uint8_t dec[18][5] = {
        {0,0,0,0,0}, {0,0,0,0,1}, {1,0,0,0,0}, {0,0,0,1,0}, {0,0,1,0,0}, {0,1,0,0,0},
        {1,0,0,1,0}, {1,0,1,0,0}, {0,1,0,1,0}, {0,1,1,0,0}, {1,0,0,0,1}, {0,0,0,1,1},
        {0,0,1,0,1}, {0,1,0,0,1}, {1,0,0,1,1}, {1,0,1,0,1}, {0,1,0,1,1}, {0,1,1,0,1},
    };
    const uint8_t* d = dec[action < 18 ? action : 0];
    uint8_t swcha = 0xFF;
    if (d[0]) swcha &= (uint8_t)~0x10;
    if (d[1]) swcha &= (uint8_t)~0x20;
    if (d[2]) swcha &= (uint8_t)~0x40;
    if (d[3]) swcha &= (uint8_t)~0x80;
    e->pia.pa_in = swcha;
    e->tia.inpt4 = !d[4];
    e->tia.paddle0 = d[2] ? 200 : (d[3] ? 50 : 128);
}

static inline int orc_rrun_one_cycle(orc_ratari* e, uint64_t* cycles) /* atari.rs:309-318 */
{
    if (e->tia.wsync) {
        orc_rtick_components(e);
        *cycles += 1;
    } else {
        uint8_t c = orc_step_rbus(&e->cpu, e);
        if (c == 0) { e->run_status |= FA_STATUS_ILLEGAL_OPCODE; return 0; }
        e->instructions++;
        *cycles += c;
    }
    return 1;
}

uint64_t orc_rrun_frame(orc_ratari* e)                             /* atari.rs:284-306 */
{
    if (e->run_status & FA_STATUS_HALT_MASK) return 0;
    e->tia.frame_complete = 0;
    uint64_t cycles = 0;
    while (e->tia.vsync & 0x02) {
        if (!orc_rrun_one_cycle(e, &cycles)) return cycles;
        if (cycles > FA_VSYNC_BUDGET) { e->run_status |= FA_STATUS_VSYNC_BUDGET; return cycles; }
    }
    while (!(e->tia.vsync & 0x02)) {
        if (!orc_rrun_one_cycle(e, &cycles)) return cycles;
        if (cycles > FA_FRAME_CYCLE_CAP) { e->run_status |= FA_STATUS_CYCLE_CAP; break; }
    }
    e->frame_no++;
    return cycles;
}

const uint8_t* orc_rframebuffer(const orc_ratari* e) { return e->tia.fb; }
void orc_rram(const orc_ratari* e, uint8_t* out128) { memcpy(out128, e->pia.ram, 128); }
size_t orc_rtia_size(void) { return sizeof(orc_rtia); }

/* Registers and frame bookkeeping of one rendering console. */
void orc_rregs(const orc_ratari* e, uint32_t* out8)
{
    out8[0] = e->cpu.a | (e->cpu.x << 8) | (e->cpu.y << 16) | ((uint32_t)e->cpu.sp << 24);
    out8[1] = e->cpu.pc | ((uint32_t)e->cpu.p << 16) | ((uint32_t)e->bank << 24);
    out8[2] = (uint32_t)e->cpu.cycles;
    out8[3] = (uint32_t)(e->cpu.cycles >> 32);
    out8[4] = e->tia.clock | ((uint32_t)e->tia.scanline << 16);
    out8[5] = e->frame_no;
    out8[6] = e->run_status;
    out8[7] = e->pia.timer_value | ((uint32_t)e->pia.timer_prescaler << 16);
}

/* E0 / 3F bank state, as fa_state::mapper (0 for the reference's schemes). */
unsigned orc_rmapper(const orc_ratari* e) { return orc_mapper_of(e->scheme, e->slice); }

/* The whole TIA record (orc_rtia, its framebuffer last) for full-state comparisons. */
void orc_rtia_copy(const orc_ratari* e, void* out) { memcpy(out, &e->tia, sizeof(e->tia)); }

/* k frames on each of n rendering consoles (actions [k][n]) with nthreads
 * threads, console i on thread i % nthreads.  Returns the instructions
 * executed, or (uint64_t)-1 on a bad argument. */
typedef struct orc_rjob {
    orc_ratari** cs;
    size_t n;
    int k, tid, nth;
    const uint8_t* actions;
    uint64_t instructions;
} orc_rjob;

static void* orc_rworker(void* arg)
{
    orc_rjob* j = (orc_rjob*)arg;
    for (size_t i = (size_t)j->tid; i < j->n; i += (size_t)j->nth) {
        orc_ratari* e = j->cs[i];
        uint64_t before = e->instructions;
        for (int f = 0; f < j->k; f++) {
            orc_rset_action(e, j->actions[(size_t)f * j->n + i]);
            orc_rrun_frame(e);
        }
        j->instructions += e->instructions - before;
    }
    return NULL;
}

uint64_t orc_rrun_batch(orc_ratari** cs, size_t n, int k, const uint8_t* actions, int nthreads)
{
    if (!cs || !actions || k < 0) return (uint64_t)-1;
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > n && n > 0) nthreads = (int)n;
    orc_rjob* jobs = (orc_rjob*)calloc((size_t)nthreads, sizeof(orc_rjob));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return (uint64_t)-1; }
    for (int t = 0; t < nthreads; t++) jobs[t] = (orc_rjob){ cs, n, k, t, nthreads, actions, 0 };
    for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, orc_rworker, &jobs[t]);
    orc_rworker(&jobs[0]);
    uint64_t total = jobs[0].instructions;
    for (int t = 1; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        total += jobs[t].instructions;
    }
    free(jobs);
    free(th);
    return total;
}

/* ------------------------------------------------------------ Atari::render */
/* Atari::render (src/atari.rs:356-369): R, G, B of ntsc_palette
 * (src/atari.rs:624-645: 128 entries indexed by (index >> 1) & 0x7F), then 255,
 * for each palette index of a framebuffer. */
void orc_rgba(const uint8_t* fb, size_t pixels, uint8_t* out)
{
    static const uint8_t pal[128][3] = {
        {0,0,0}, {0,0,0}, {68,68,0}, {68,68,0}, {112,40,0}, {112,40,0}, {132,24,0}, {132,24,0},
        {136,0,0}, {136,0,0}, {120,0,92}, {120,0,92}, {72,0,120}, {72,0,120}, {20,0,132}, {20,0,132},
        {0,0,136}, {0,0,136}, {0,0,120}, {0,0,120}, {0,0,96}, {0,0,96}, {0,20,44}, {0,20,44},
        {0,40,0}, {0,40,0}, {0,44,0}, {0,44,0}, {0,44,0}, {0,44,0}, {0,24,0}, {0,24,0},
        {40,40,40}, {40,40,40}, {100,100,16}, {100,100,16}, {144,72,16}, {144,72,16}, {168,56,0}, {168,56,0},
        {184,20,0}, {184,20,0}, {160,0,116}, {160,0,116}, {100,0,164}, {100,0,164}, {48,0,176}, {48,0,176},
        {0,0,184}, {0,0,184}, {0,24,168}, {0,24,168}, {0,44,128}, {0,44,128}, {0,60,76}, {0,60,76},
        {0,68,0}, {0,68,0}, {0,76,0}, {0,76,0}, {0,68,0}, {0,68,0}, {0,56,0}, {0,56,0},
        {84,84,84}, {84,84,84}, {132,132,36}, {132,132,36}, {176,100,36}, {176,100,36}, {200,80,16}, {200,80,16},
        {220,56,20}, {220,56,20}, {196,20,144}, {196,20,144}, {132,0,200}, {132,0,200}, {80,0,212}, {80,0,212},
        {24,0,220}, {24,0,220}, {0,48,212}, {0,48,212}, {0,76,164}, {0,76,164}, {0,92,108}, {0,92,108},
        {0,100,0}, {0,100,0}, {0,108,0}, {0,108,0}, {0,100,16}, {0,100,16}, {0,84,0}, {0,84,0},
        {120,120,120}, {120,120,120}, {168,168,56}, {168,168,56}, {204,136,56}, {204,136,56}, {232,112,36}, {232,112,36},
        {252,92,40}, {252,92,40}, {232,48,172}, {232,48,172}, {168,0,232}, {168,0,232}, {112,0,244}, {112,0,244},
        {56,0,252}, {56,0,252}, {12,76,248}, {12,76,248}, {0,108,196}, {0,108,196}, {0,128,140}, {0,128,140},
        {0,136,0}, {0,136,0}, {0,144,0}, {0,144,0}, {0,136,40}, {0,136,40}, {0,116,0}, {0,116,0},
    };
    for (size_t i = 0; i < pixels; i++) {
        const uint8_t* c = pal[(fb[i] >> 1) & 0x7F];
        out[4 * i] = c[0];
        out[4 * i + 1] = c[1];
        out[4 * i + 2] = c[2];
        out[4 * i + 3] = 255;
    }
}
