// fa_layout.h — structure-of-arrays layout of instance state in HBM.
//
// Each instance is one column of FA_ROWS 32-bit words; row w of instance i
// lives at state[w * stride + i], so a warp loading row w reads 128
// contiguous bytes.  Rows [0, FA_PRIV_WORDS) are the instance's "private
// bytes": its 128 bytes of PIA RAM followed by the TIA registers that only
// change on a register write.  The kernel keeps these in shared memory while
// it runs; the remaining rows are the hot fields it keeps in registers.
//
// Shared by the host packer (fa_state AoS <-> SoA) and the device code.
#pragma once
#include <stdint.h>

#include "../../include/fast_atari.h"

#define FA_PRIV_BYTES 176
#define FA_PRIV_WORDS (FA_PRIV_BYTES / 4)
// The kernel keeps only the RAM words in shared memory; the write-only TIA
// registers (rows FA_SMEM_WORDS..FA_PRIV_WORDS-1) stay in their HBM rows and
// are touched there by the rare TIA register writes and collision reads.
#define FA_SMEM_WORDS 32

// Private-byte offsets: RAM occupies [0, 128).
enum : uint32_t {
    PB_CX     = 128,   // 8 collision latches cxm0p..cxppmm
    PB_POS    = 136,   // 5 x u16: pos_p0 pos_p1 pos_m0 pos_m1 pos_bl
    PB_HM     = 146,   // 5 x u8: hmp0 hmp1 hmm0 hmm1 hmbl
    PB_GRP0   = 151, PB_GRP1 = 152, PB_GRP0_OLD = 153, PB_GRP1_OLD = 154,
    PB_ENAM0  = 155, PB_ENAM1 = 156, PB_ENABL = 157, PB_ENABL_OLD = 158,
    PB_VDELP0 = 159, PB_VDELP1 = 160, PB_VDELBL = 161,
    PB_RESMP0 = 162, PB_RESMP1 = 163,
    PB_NUSIZ0 = 164, PB_NUSIZ1 = 165,
    PB_COLUP0 = 166, PB_COLUP1 = 167, PB_COLUPF = 168, PB_COLUBK = 169,
    PB_CTRLPF = 170, PB_REFP0 = 171, PB_REFP1 = 172,
    PB_PF0    = 173, PB_PF1 = 174, PB_PF2 = 175,
};

// Hot rows (after the private words).
enum : uint32_t {
    R_AXYS   = FA_PRIV_WORDS + 0,   // a | x<<8 | y<<16 | sp<<24
    R_PC     = FA_PRIV_WORDS + 1,   // pc | p<<16 | bank<<24
    R_CYC_LO = FA_PRIV_WORDS + 2,
    R_CYC_HI = FA_PRIV_WORDS + 3,
    R_PIA0   = FA_PRIV_WORDS + 4,   // pa_out | pa_ddr<<8 | pa_in<<16 | pb_out<<24
    R_PIA1   = FA_PRIV_WORDS + 5,   // pb_ddr | pb_in<<8 | timer_underflow<<16 | paddle_dumped<<24
    R_TIMER  = FA_PRIV_WORDS + 6,   // timer_value | timer_prescaler<<16
    R_SELPC  = FA_PRIV_WORDS + 7,   // timer_prescaler_select | paddle_counter<<16
    R_TIA0   = FA_PRIV_WORDS + 8,   // clock | scanline<<16
    R_TIA1   = FA_PRIV_WORDS + 9,   // wsync | frame_complete<<8 | vsync<<16 | vblank<<24
    R_TIA2   = FA_PRIV_WORDS + 10,  // inpt4 | inpt5<<8 | paddle0<<16 | paddle1<<24
    R_FRAME  = FA_PRIV_WORDS + 11,  // frame_no
    R_STATUS = FA_PRIV_WORDS + 12,  // run_status
    // DPC registers (FA_SCHEME_DPC carts only; the device touches them only
    // on a DPC register access, in place in HBM).
    R_DPC_CNT = FA_PRIV_WORDS + 13, // 4 rows: counter 2r | counter 2r+1 << 16
    R_DPC_TOP = FA_PRIV_WORDS + 17, // 2 rows: top 4r..4r+3, one per byte
    R_DPC_BOT = FA_PRIV_WORDS + 19, // 2 rows: bottom 4r..4r+3
    R_DPC_MISC = FA_PRIV_WORDS + 21,// flags | music << 8 | random << 16
    R_DPC_OSC = FA_PRIV_WORDS + 22, // oscillator clock count at the last update
    FA_ROWS  = FA_PRIV_WORDS + 23,
};

// Bank-switch decode: a read or write of (addr & 0x1FFF) - hot_lo < nbanks
// selects that bank (src/atari.rs:460-492).  Fixed carts use hot_lo 0x2000,
// which no 13-bit address reaches.
static inline uint32_t fa_hot_lo(int scheme)
{
    return scheme == FA_SCHEME_F8 ? 0x1FF8u : scheme == FA_SCHEME_F6 ? 0x1FF6u
         : scheme == FA_SCHEME_F4 ? 0x1FF4u : 0x2000u;
}
static inline uint32_t fa_nbanks(int scheme)
{
    return scheme == FA_SCHEME_F8 ? 2u : scheme == FA_SCHEME_F6 ? 4u : scheme == FA_SCHEME_F4 ? 8u : 1u;
}
static inline int fa_detect_scheme(size_t len)        // BankScheme::detect, src/atari.rs:96-105
{
    return len <= 4096 ? FA_SCHEME_FIXED : len <= 8192 ? FA_SCHEME_F8
         : len <= 16384 ? FA_SCHEME_F6 : FA_SCHEME_F4;
}

#ifdef __CUDACC__
#define FA_HD __host__ __device__
#else
#define FA_HD
#endif

// Sliced carts (E0, 3F, DPC) map 1K slices of the ROM image into the four 1K
// windows of $1000-$1FFF; `slices` holds the slice of window k in byte k.
// Their hot_lo is FA_MAP_* << 8 (3F: | the number of 2K banks), below 0x1000,
// so no ROM address passes the 4K-bank hotspot decode or the 4K-bank fetch
// path.  The bank state a caller sees is 16 bits (fa_state::mapper): E0 =
// window 0 | window 1 << 4 | window 2 << 8; 3F = the 2K bank at $1000; DPC =
// the 4K program bank (slices 4b..4b+3).  A DPC image holds the 8K of
// program, then the 2K of display data at byte 8192.  FE = the 4K bank |
// 0x100 while the last bus access was to $01FE (bit 7 of `slices` on the
// device, which the slice decode ignores).
enum : uint32_t { FA_MAP_E0 = 1u, FA_MAP_3F = 2u, FA_MAP_DPC = 3u, FA_MAP_FE = 4u };

FA_HD static inline uint32_t fa_map_kind(uint32_t hot_lo) { return hot_lo < 0x1000u ? hot_lo >> 8 : 0u; }

// Kernel builds by the cores they hold (see run_unit): 4K-bank carts only,
// several kinds, E0 / 3F carts only, DPC carts only, FE carts only.
enum : int { FA_MAPS_4K = 0, FA_MAPS_BOTH = 1, FA_MAPS_SLICED = 2, FA_MAPS_DPC = 3, FA_MAPS_FE = 4 };

// E0 and 3F; the 4K-bank pair of DPC and FE (bank b: slices 4b..4b+3, FE's
// armed flag in bit 7); any scheme.  Each device core calls only its own.
FA_HD static inline uint32_t fa_slices_e0_3f(uint32_t hot_lo, uint32_t m)
{
    if (fa_map_kind(hot_lo) == FA_MAP_E0)
        return (m & 7u) | (((m >> 4) & 7u) << 8) | (((m >> 8) & 7u) << 16) | (7u << 24);
    if (fa_map_kind(hot_lo) == FA_MAP_3F) {
        const uint32_t n = hot_lo & 0xFFu, b = (m & 0xFFu) % n, l = n - 1u;
        return (2u * b) | ((2u * b + 1u) << 8) | ((2u * l) << 16) | ((2u * l + 1u) << 24);
    }
    return 0u;
}
FA_HD static inline uint32_t fa_slices_4k_bank(uint32_t m, bool fe)
{
    return ((m & 1u) * 0x04040404u + 0x03020100u) | (fe ? ((m >> 8) & 1u) << 7 : 0u);
}
FA_HD static inline uint32_t fa_slices_from_mapper(uint32_t hot_lo, uint32_t m)
{
    if (fa_map_kind(hot_lo) == FA_MAP_DPC || fa_map_kind(hot_lo) == FA_MAP_FE)
        return fa_slices_4k_bank(m, fa_map_kind(hot_lo) == FA_MAP_FE);
    return fa_slices_e0_3f(hot_lo, m);
}

FA_HD static inline uint32_t fa_mapper_e0_3f(uint32_t hot_lo, uint32_t slices)
{
    if (fa_map_kind(hot_lo) == FA_MAP_E0)
        return (slices & 7u) | (((slices >> 8) & 7u) << 4) | (((slices >> 16) & 7u) << 8);
    if (fa_map_kind(hot_lo) == FA_MAP_3F) return (slices & 0xFFu) >> 1;
    return 0u;
}
FA_HD static inline uint32_t fa_mapper_4k_bank(uint32_t slices, bool fe)
{
    return ((slices & 0x7Fu) >> 2) | (fe ? ((slices >> 7) & 1u) << 8 : 0u);
}
FA_HD static inline uint32_t fa_mapper_from_slices(uint32_t hot_lo, uint32_t slices)
{
    if (fa_map_kind(hot_lo) == FA_MAP_DPC || fa_map_kind(hot_lo) == FA_MAP_FE)
        return fa_mapper_4k_bank(slices, fa_map_kind(hot_lo) == FA_MAP_FE);
    return fa_mapper_e0_3f(hot_lo, slices);
}

// The bank state's 14 stored bits ride in R_TIA1's flag bytes, above the
// wsync and frame_complete bits: bits 1-7 of byte 0 and bits 1-7 of byte 1.
FA_HD static inline uint32_t fa_tia1_mapper(uint32_t w) { return ((w >> 1) & 0x7Fu) | (((w >> 9) & 0x7Fu) << 7); }
FA_HD static inline uint32_t fa_mapper_tia1(uint32_t m) { return ((m & 0x7Fu) << 1) | (((m >> 7) & 0x7Fu) << 9); }

// ---- rendering console (src/tia.rs, src/atari.rs:107-306)
// Its state is the headless layout's rows (the same R_* and PB_* meaning)
// followed by what only the pixel-accurate TIA has.  While a unit runs, the
// private bytes [0, FA_RPRIV_BYTES) sit in shared memory: the RAM, the
// graphics registers PB_*, and the RB_* extras, which are stored in rows
// FA_RROW_EXTRA.. of HBM.
enum : uint32_t {
    RB_DLEN    = 176,          // pending playfield writes (0..4)
    RB_DQ      = 177,          // 4 x (remaining, register, value)
    RB_PFRAMES = 189,          // resizer: pending_frames
    RB_PTOP    = 190,          // resizer: pending_top (u16, 2-byte aligned)
    FA_RPRIV_BYTES = 192,
    FA_RPRIV_WORDS = FA_RPRIV_BYTES / 4,
    FA_RSLAB_WORDS = FA_RPRIV_WORDS + 8,               // + the framebuffer sector buffer (shared memory only)
    FA_RROW_EXTRA = FA_ROWS,                           // rows holding RB_* words
    RR_VTOP  = FA_ROWS + (FA_RPRIV_WORDS - FA_PRIV_WORDS),   // visible_top | vblank_top << 16
    RR_FLAGS = RR_VTOP + 1,    // hmove_pending | input_latch_enabled << 1 | inpt4_latch << 2 | inpt5_latch << 3
    FA_RROWS = RR_FLAGS + 1,
};
#define FA_FB_W 160
#define FA_FB_H 192
#define FA_FB_BYTES (FA_FB_W * FA_FB_H)
