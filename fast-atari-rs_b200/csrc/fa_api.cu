// fa_api.cu — C ABI of the batched Atari core: the `BatchAtariGpu` handle.
//
// Mirrors src/cuda_env.rs:99-191 of the reference: a handle owns one ROM and
// n instances resident in HBM; reset/step/step_multi/download_states act on
// all of them.  Differences by design: state is structure-of-arrays, reset
// runs on the device from one post-reset snapshot, the action and
// observation buffers are preallocated (pinned on the host), and errors are
// status codes rather than panics.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

int fa_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

extern "C" const char* fa_last_error(void) { return g_err.c_str(); }
extern "C" const char* fa_version(void) { return "fast-atari-b200 0.1 (sm_100a)"; }

namespace {
std::atomic<uint64_t> g_wait_ns{2000000000ull};
}

uint64_t fa_wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }

extern "C" int fa_set_wait_limit_ns(uint64_t ns)
{
    if (ns > 10000000000ull) return fa_fail(FA_ERR_INVALID, "wait limit %llu ns is above 10 s", (unsigned long long)ns);
    g_wait_ns.store(ns, std::memory_order_relaxed);
    return FA_OK;
}

extern "C" uint64_t fa_wait_limit_ns_get(void) { return fa_wait_limit_ns(); }

extern "C" int fa_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

extern "C" int fa_set_device(int device)
{
    if (device < 0 || device >= fa_device_count()) return fa_fail(FA_ERR_NO_DEVICE, "no CUDA device %d", device);
    FA_CUDA(cudaSetDevice(device));
    return FA_OK;
}

// ------------------------------------------------------------------ packing
static inline uint32_t b4(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    return (a & 0xFFu) | ((b & 0xFFu) << 8) | ((c & 0xFFu) << 16) | ((d & 0xFFu) << 24);
}

// Private bytes of one instance (RAM then the write-only TIA registers).
static void priv_from_state(const fa_state& s, uint8_t* pb)
{
    memset(pb, 0, FA_PRIV_BYTES);
    memcpy(pb, s.ram, 128);
    const uint8_t cx[8] = { s.cxm0p, s.cxm1p, s.cxp0fb, s.cxp1fb, s.cxm0fb, s.cxm1fb, s.cxblpf, s.cxppmm };
    memcpy(pb + PB_CX, cx, 8);
    const uint16_t pos[5] = { s.pos_p0, s.pos_p1, s.pos_m0, s.pos_m1, s.pos_bl };
    memcpy(pb + PB_POS, pos, 10);
    const uint8_t hm[5] = { s.hmp0, s.hmp1, s.hmm0, s.hmm1, s.hmbl };
    memcpy(pb + PB_HM, hm, 5);
    pb[PB_GRP0] = s.grp0; pb[PB_GRP1] = s.grp1; pb[PB_GRP0_OLD] = s.grp0_old; pb[PB_GRP1_OLD] = s.grp1_old;
    pb[PB_ENAM0] = !!s.enam0; pb[PB_ENAM1] = !!s.enam1; pb[PB_ENABL] = !!s.enabl; pb[PB_ENABL_OLD] = !!s.enabl_old;
    pb[PB_VDELP0] = !!s.vdelp0; pb[PB_VDELP1] = !!s.vdelp1; pb[PB_VDELBL] = !!s.vdelbl;
    pb[PB_RESMP0] = !!s.resmp0; pb[PB_RESMP1] = !!s.resmp1;
    pb[PB_NUSIZ0] = s.nusiz0; pb[PB_NUSIZ1] = s.nusiz1;
    pb[PB_COLUP0] = s.colup0; pb[PB_COLUP1] = s.colup1; pb[PB_COLUPF] = s.colupf; pb[PB_COLUBK] = s.colubk;
    pb[PB_CTRLPF] = s.ctrlpf; pb[PB_REFP0] = !!s.refp0; pb[PB_REFP1] = !!s.refp1;
    pb[PB_PF0] = s.pf0; pb[PB_PF1] = s.pf1; pb[PB_PF2] = s.pf2;
}

void fa_pack_column(const fa_state& s, uint32_t* col, size_t stride)
{
    uint8_t pb[FA_PRIV_BYTES];
    priv_from_state(s, pb);
    for (uint32_t w = 0; w < FA_PRIV_WORDS; w++) {
        uint32_t v;
        memcpy(&v, pb + 4 * w, 4);
        col[w * stride] = v;
    }
    col[R_AXYS * stride] = b4(s.a, s.x, s.y, s.sp);
    col[R_PC * stride] = (uint32_t)s.pc | ((uint32_t)s.status << 16) | ((uint32_t)s.bank << 24);
    col[R_CYC_LO * stride] = (uint32_t)s.cycles;
    col[R_CYC_HI * stride] = (uint32_t)(s.cycles >> 32);
    col[R_PIA0 * stride] = b4(s.port_a_output, s.port_a_ddr, s.port_a_input, s.port_b_output);
    col[R_PIA1 * stride] = b4(s.port_b_ddr, s.port_b_input, !!s.timer_underflow, !!s.paddle_dumped);
    col[R_TIMER * stride] = (uint32_t)s.timer_value | ((uint32_t)s.timer_prescaler << 16);
    col[R_SELPC * stride] = (uint32_t)s.timer_prescaler_select | ((uint32_t)s.paddle_counter << 16);
    col[R_TIA0 * stride] = (uint32_t)s.tia_clock | ((uint32_t)s.tia_scanline << 16);
    col[R_TIA1 * stride] = b4(!!s.tia_wsync, !!s.tia_frame_complete, s.tia_vsync, s.tia_vblank) |
                           fa_mapper_tia1((uint32_t)s.mapper[0] | ((uint32_t)s.mapper[1] << 8));
    col[R_TIA2 * stride] = b4(!!s.inpt4, !!s.inpt5, s.paddle0, s.paddle1);
    col[R_FRAME * stride] = s.frame_no;
    col[R_STATUS * stride] = s.run_status;
    for (uint32_t r = 0; r < 4; r++)
        col[(R_DPC_CNT + r) * stride] = (uint32_t)(s.dpc_counter[2 * r] & 0x7FFu) |
                                        ((uint32_t)(s.dpc_counter[2 * r + 1] & 0x7FFu) << 16);
    for (uint32_t r = 0; r < 2; r++) {
        col[(R_DPC_TOP + r) * stride] = b4(s.dpc_top[4 * r], s.dpc_top[4 * r + 1], s.dpc_top[4 * r + 2], s.dpc_top[4 * r + 3]);
        col[(R_DPC_BOT + r) * stride] =
            b4(s.dpc_bottom[4 * r], s.dpc_bottom[4 * r + 1], s.dpc_bottom[4 * r + 2], s.dpc_bottom[4 * r + 3]);
    }
    col[R_DPC_MISC * stride] = (uint32_t)s.dpc_flags | ((uint32_t)(s.dpc_music & 7u) << 8) | ((uint32_t)s.dpc_random << 16);
    col[R_DPC_OSC * stride] = s.dpc_osc;
}

void fa_unpack_column(const uint32_t* col, size_t stride, int scheme, fa_state& s)
{
    memset(&s, 0, sizeof(s));
    uint8_t pb[FA_PRIV_BYTES];
    for (uint32_t w = 0; w < FA_PRIV_WORDS; w++) {
        uint32_t v = col[w * stride];
        memcpy(pb + 4 * w, &v, 4);
    }
    memcpy(s.ram, pb, 128);
    s.cxm0p = pb[PB_CX + 0]; s.cxm1p = pb[PB_CX + 1]; s.cxp0fb = pb[PB_CX + 2]; s.cxp1fb = pb[PB_CX + 3];
    s.cxm0fb = pb[PB_CX + 4]; s.cxm1fb = pb[PB_CX + 5]; s.cxblpf = pb[PB_CX + 6]; s.cxppmm = pb[PB_CX + 7];
    uint16_t pos[5];
    memcpy(pos, pb + PB_POS, 10);
    s.pos_p0 = pos[0]; s.pos_p1 = pos[1]; s.pos_m0 = pos[2]; s.pos_m1 = pos[3]; s.pos_bl = pos[4];
    s.hmp0 = pb[PB_HM + 0]; s.hmp1 = pb[PB_HM + 1]; s.hmm0 = pb[PB_HM + 2]; s.hmm1 = pb[PB_HM + 3];
    s.hmbl = pb[PB_HM + 4];
    s.grp0 = pb[PB_GRP0]; s.grp1 = pb[PB_GRP1]; s.grp0_old = pb[PB_GRP0_OLD]; s.grp1_old = pb[PB_GRP1_OLD];
    s.enam0 = pb[PB_ENAM0]; s.enam1 = pb[PB_ENAM1]; s.enabl = pb[PB_ENABL]; s.enabl_old = pb[PB_ENABL_OLD];
    s.vdelp0 = pb[PB_VDELP0]; s.vdelp1 = pb[PB_VDELP1]; s.vdelbl = pb[PB_VDELBL];
    s.resmp0 = pb[PB_RESMP0]; s.resmp1 = pb[PB_RESMP1];
    s.nusiz0 = pb[PB_NUSIZ0]; s.nusiz1 = pb[PB_NUSIZ1];
    s.colup0 = pb[PB_COLUP0]; s.colup1 = pb[PB_COLUP1]; s.colupf = pb[PB_COLUPF]; s.colubk = pb[PB_COLUBK];
    s.ctrlpf = pb[PB_CTRLPF]; s.refp0 = pb[PB_REFP0]; s.refp1 = pb[PB_REFP1];
    s.pf0 = pb[PB_PF0]; s.pf1 = pb[PB_PF1]; s.pf2 = pb[PB_PF2];
    uint32_t w;
    w = col[R_AXYS * stride]; s.a = w; s.x = w >> 8; s.y = w >> 16; s.sp = w >> 24;
    w = col[R_PC * stride]; s.pc = (uint16_t)w; s.status = (uint8_t)(w >> 16); s.bank = (uint8_t)(w >> 24);
    s.cycles = (uint64_t)col[R_CYC_LO * stride] | ((uint64_t)col[R_CYC_HI * stride] << 32);
    w = col[R_PIA0 * stride]; s.port_a_output = w; s.port_a_ddr = w >> 8; s.port_a_input = w >> 16; s.port_b_output = w >> 24;
    w = col[R_PIA1 * stride]; s.port_b_ddr = w; s.port_b_input = w >> 8; s.timer_underflow = w >> 16; s.paddle_dumped = w >> 24;
    w = col[R_TIMER * stride]; s.timer_value = (uint16_t)w; s.timer_prescaler = (uint16_t)(w >> 16);
    w = col[R_SELPC * stride]; s.timer_prescaler_select = (uint16_t)w; s.paddle_counter = (uint16_t)(w >> 16);
    w = col[R_TIA0 * stride]; s.tia_clock = (uint16_t)w; s.tia_scanline = (uint16_t)(w >> 16);
    w = col[R_TIA1 * stride]; s.tia_wsync = w & 1u; s.tia_frame_complete = (w >> 8) & 1u; s.tia_vsync = w >> 16; s.tia_vblank = w >> 24;
    const uint32_t m = fa_tia1_mapper(w);
    s.mapper[0] = (uint8_t)m;
    s.mapper[1] = (uint8_t)(m >> 8);
    w = col[R_TIA2 * stride]; s.inpt4 = w; s.inpt5 = w >> 8; s.paddle0 = w >> 16; s.paddle1 = w >> 24;
    s.frame_no = col[R_FRAME * stride];
    s.run_status = col[R_STATUS * stride];
    s.scheme = (uint8_t)scheme;
    for (uint32_t r = 0; r < 4; r++) {
        w = col[(R_DPC_CNT + r) * stride];
        s.dpc_counter[2 * r] = (uint16_t)(w & 0xFFFFu);
        s.dpc_counter[2 * r + 1] = (uint16_t)(w >> 16);
    }
    for (uint32_t r = 0; r < 2; r++)
        for (uint32_t b = 0; b < 4; b++) {
            s.dpc_top[4 * r + b] = (uint8_t)(col[(R_DPC_TOP + r) * stride] >> (8 * b));
            s.dpc_bottom[4 * r + b] = (uint8_t)(col[(R_DPC_BOT + r) * stride] >> (8 * b));
        }
    w = col[R_DPC_MISC * stride];
    s.dpc_flags = (uint8_t)w; s.dpc_music = (uint8_t)(w >> 8); s.dpc_random = (uint8_t)(w >> 16);
    s.dpc_osc = col[R_DPC_OSC * stride];
}

void fa_power_on_column(const uint8_t* img, uint32_t nbanks, int scheme, uint32_t hot_lo, uint32_t* col)
{
    // HeadlessBus::new (src/atari.rs:410-430): power-on bank is the last one;
    // Cpu::reset (src/cpu.rs:125-134) reads the vector at $FFFC/$FFFD.
    fa_state s;
    memset(&s, 0, sizeof(s));
    if (fa_map_kind(hot_lo)) {
        // Sliced carts: E0 windows 4, 5, 6, 7 (the image's last 4K, as the
        // reference powers on in its last bank); 3F bank 0; DPC program bank
        // 1 (the last), with its random number generator at 1; FE bank 1, not
        // armed.  The vector is in window 3 ($1C00-$1FFF), whose slice is
        // byte 3.
        const uint32_t kind = fa_map_kind(hot_lo);
        const uint32_t m = kind == FA_MAP_E0 ? (4u | 5u << 4 | 6u << 8) : (kind == FA_MAP_DPC || kind == FA_MAP_FE) ? 1u : 0u;
        if (kind == FA_MAP_DPC) s.dpc_random = 1;
        const uint32_t vec = (fa_slices_from_mapper(hot_lo, m) >> 24) * 1024u + 0x3FCu;
        s.mapper[0] = (uint8_t)m;
        s.mapper[1] = (uint8_t)(m >> 8);
        s.pc = (uint16_t)(img[vec] | (img[vec + 1] << 8));
    } else {
        const uint32_t bank = scheme == FA_SCHEME_FIXED ? 0u : nbanks - 1u;
        s.bank = (uint8_t)bank;
        s.pc = (uint16_t)(img[(bank << 12) | 0xFFC] | (img[(bank << 12) | 0xFFD] << 8));
    }
    s.sp = 0xFD;
    s.port_a_input = 0xFF;                   // Pia::default, src/pia.rs:46-62
    s.port_b_input = 0x3F;
    s.timer_prescaler = 1;
    s.timer_prescaler_select = 1;
    s.inpt4 = 1;                             // HeadlessTia::default, src/headless_tia.rs:90-118
    s.inpt5 = 1;
    fa_pack_column(s, col, 1);
}

// ------------------------------------------------------------------ ROM schemes
static int dpc_len(size_t len) { return len == 10240 || len == 10495; }

static int rom_len_ok(size_t len)          // lengths HeadlessBus::new accepts (src/atari.rs:410-449)
{
    if (len == 0) return 0;
    switch (fa_detect_scheme(len)) {
    case FA_SCHEME_FIXED: return 1;
    case FA_SCHEME_F8: return len >= 8192;
    case FA_SCHEME_F6: return len >= 16384;
    default: return len >= 32768;
    }
}

// The scheme for a ROM length with nothing registered: DPC for its two dump
// lengths (which the reference's size rule cannot construct), else the
// reference's size rule; -1 for a length neither can build.
static int auto_scheme(size_t len)
{
    if (dpc_len(len)) return FA_SCHEME_DPC;
    return rom_len_ok(len) ? fa_detect_scheme(len) : -1;
}

static int scheme_len_ok(int scheme, size_t len)
{
    switch (scheme) {
    case FA_SCHEME_E0: case FA_SCHEME_FE: return len == 8192;
    case FA_SCHEME_DPC: return dpc_len(len);
    case FA_SCHEME_3F: return len >= 2048 && len <= 32768 && len % 2048 == 0;
    case FA_SCHEME_FIXED: case FA_SCHEME_F8: case FA_SCHEME_F6: case FA_SCHEME_F4:
        return rom_len_ok(len) && fa_detect_scheme(len) == scheme;
    default: return 0;
    }
}

namespace {
std::mutex g_scheme_mu;
std::vector<std::pair<std::pair<uint64_t, size_t>, int>> g_schemes;   // (content hash, length) -> scheme

uint64_t rom_hash(const uint8_t* rom, size_t len)    // FNV-1a, 64-bit
{
    uint64_t h = 0xCBF29CE484222325ull;
    for (size_t i = 0; i < len; i++) h = (h ^ rom[i]) * 0x100000001B3ull;
    return h;
}

int registered_scheme(const uint8_t* rom, size_t len)
{
    const auto key = std::make_pair(rom_hash(rom, len), len);
    std::lock_guard<std::mutex> lk(g_scheme_mu);
    for (const auto& e : g_schemes)
        if (e.first == key) return e.second;
    return FA_SCHEME_AUTO;
}
}  // namespace

extern "C" int fa_rom_set_scheme(const uint8_t* rom, size_t rom_len, int scheme)
{
    if (!rom || rom_len == 0) return fa_fail(FA_ERR_INVALID, "need a ROM");
    if (scheme != FA_SCHEME_AUTO && !scheme_len_ok(scheme, rom_len))
        return fa_fail(FA_ERR_BAD_ROM, "scheme %d cannot hold a %zu-byte ROM", scheme, rom_len);
    const auto key = std::make_pair(rom_hash(rom, rom_len), rom_len);
    std::lock_guard<std::mutex> lk(g_scheme_mu);
    for (size_t i = 0; i < g_schemes.size(); i++)
        if (g_schemes[i].first == key) { g_schemes.erase(g_schemes.begin() + (ptrdiff_t)i); break; }
    if (scheme != FA_SCHEME_AUTO) g_schemes.emplace_back(key, scheme);
    return FA_OK;
}

extern "C" int fa_rom_scheme(const uint8_t* rom, size_t rom_len)
{
    if (!rom || rom_len == 0) return fa_fail(FA_ERR_BAD_ROM, "empty ROM");
    const int reg = registered_scheme(rom, rom_len);
    if (reg != FA_SCHEME_AUTO) return reg;
    const int s = auto_scheme(rom_len);
    if (s < 0) return fa_fail(FA_ERR_BAD_ROM, "ROM length %zu cannot be constructed (reference panics)", rom_len);
    return s;
}

extern "C" int fa_rom_guess_scheme(const uint8_t* rom, size_t rom_len)
{
    if (!rom || rom_len == 0) return fa_fail(FA_ERR_BAD_ROM, "empty ROM");
    // Absolute and absolute-indexed loads and stores (LDA/LDX/LDY/STA/STX/
    // STY/BIT/CMP) aimed at ROM-space hotspots, and zero-page stores to $3F.
    // Data bytes can look like either, so the counts are compared with the
    // accesses to the hotspots of the scheme the size rule gives.
    static const uint8_t abs_ops[] = { 0xAD, 0xAE, 0xAC, 0x8D, 0x8E, 0x8C, 0x2C, 0xCD,
                                       0xBD, 0xB9, 0xBE, 0xBC, 0x9D, 0x99 };
    const int by_size = auto_scheme(rom_len);
    if (by_size == FA_SCHEME_DPC) return by_size;
    const uint32_t hlo = by_size > 0 ? fa_hot_lo(by_size) : 0x2000u, hn = by_size > 0 ? fa_nbanks(by_size) : 0u;
    size_t e0 = 0, own = 0, st3f = 0, jsr_d = 0, jsr_f = 0;
    for (size_t i = 0; i + 2 < rom_len; i++) {
        const uint8_t op = rom[i];
        if ((op == 0x85 || op == 0x86 || op == 0x84) && rom[i + 1] == 0x3F) st3f++;
        if (op == 0x20) {                                   // JSR: FE carts call across banks by $Dxxx / $Fxxx
            jsr_d += (rom[i + 2] & 0xF0u) == 0xD0u;
            jsr_f += (rom[i + 2] & 0xF0u) == 0xF0u;
        }
        if (std::find(std::begin(abs_ops), std::end(abs_ops), op) == std::end(abs_ops)) continue;
        const uint32_t a = (uint32_t)rom[i + 1] | ((uint32_t)rom[i + 2] << 8);
        if (!(a & 0x1000u)) continue;
        const uint32_t a13 = a & 0x1FFFu;
        if (a13 >= 0x1FE0u && a13 <= 0x1FF7u) e0++;
        if (a13 - hlo < hn) own++;
    }
    // The reset vector (the image's last two words but two) must point into
    // the part of the address space that is fixed at power-on: window 3
    // ($1C00-$1FFF) for E0, the last 2K ($1800-$1FFF) for 3F.
    const uint32_t vec_hi = rom_len >= 4 ? rom[rom_len - 3] & 0x1Fu : 0u;
    if (rom_len == 8192 && e0 >= 3 && e0 > 8 * own && (vec_hi & 0x1Cu) == 0x1Cu) return FA_SCHEME_E0;
    if (st3f >= 3 && st3f > 8 * own && (vec_hi & 0x18u) == 0x18u && scheme_len_ok(FA_SCHEME_3F, rom_len))
        return FA_SCHEME_3F;
    // FE: no access to the F8 hotspots (an F8 cart cannot switch without
    // them), calls into both $Dxxx and $Fxxx, and a reset vector in one of
    // those two ranges.
    const uint32_t vec_top = rom_len >= 4 ? rom[rom_len - 3] & 0xF0u : 0u;
    if (rom_len == 8192 && own == 0 && jsr_d >= 6 && jsr_f >= 6 && (vec_top == 0xD0u || vec_top == 0xF0u))
        return FA_SCHEME_FE;
    if (by_size < 0)
        return fa_fail(FA_ERR_BAD_ROM, "ROM length %zu cannot be constructed (reference panics)", rom_len);
    return by_size;
}

// The shared-memory image of a ROM, in 4 KiB units: Fixed carts mirror into
// one 4K window (HeadlessBus::load_bank, src/atari.rs:433-449); 4K-bank carts
// use their first nbanks * 4 KiB; sliced carts (E0, 3F) the whole ROM,
// zero-padded to a 4K multiple; DPC carts their 10K, padded to 12K.  The
// scheme is the registered one for these bytes, else DPC for its lengths,
// else the reference's size rule.
int fa_make_bank_image(const uint8_t* rom, size_t len, std::vector<uint8_t>& img, int& scheme, uint32_t* nbanks,
                       uint32_t* hot_lo)
{
    if (!rom || len == 0) return fa_fail(FA_ERR_BAD_ROM, "empty ROM");
    scheme = registered_scheme(rom, len);
    if (scheme == FA_SCHEME_AUTO) {
        scheme = auto_scheme(len);
        if (scheme < 0) return fa_fail(FA_ERR_BAD_ROM, "ROM length %zu cannot be constructed (reference panics)", len);
    }
    uint32_t nb, hl;
    if (scheme == FA_SCHEME_DPC) {
        // 8K of program, then the 2K of display data; the 255 bytes some
        // dumps carry after them are not used.
        nb = 3;
        hl = FA_MAP_DPC << 8;
        img.assign((size_t)nb * 4096, 0);
        memcpy(img.data(), rom, 10240);
    } else if (scheme == FA_SCHEME_E0 || scheme == FA_SCHEME_3F || scheme == FA_SCHEME_FE) {
        nb = (uint32_t)((len + 4095) / 4096);
        hl = scheme == FA_SCHEME_E0   ? (FA_MAP_E0 << 8)
           : scheme == FA_SCHEME_FE   ? (FA_MAP_FE << 8)
                                      : ((FA_MAP_3F << 8) | (uint32_t)(len / 2048));
        img.assign((size_t)nb * 4096, 0);
        memcpy(img.data(), rom, len);
    } else {
        nb = fa_nbanks(scheme);
        hl = fa_hot_lo(scheme);
        img.resize((size_t)nb * 4096);
        if (scheme == FA_SCHEME_FIXED)
            for (size_t i = 0; i < 4096; i++) img[i] = rom[i % len];
        else
            memcpy(img.data(), rom, img.size());
    }
    if (nbanks) *nbanks = nb;
    if (hot_lo) *hot_lo = hl;
    return FA_OK;
}

// ------------------------------------------------------------------ handle
static void free_handle(fa_handle* h)
{
    if (!h) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_rom);
    cudaFree(h->d_state);
    cudaFree(h->d_snap);
    cudaFree(h->d_actions);
    cudaFree(h->d_obs);
    cudaFree(h->d_err);
    cudaFree(h->d_instr);
    cudaFreeHost(h->h_actions);
    cudaFreeHost(h->h_obs);
    if (h->stream) cudaStreamDestroy(h->stream);
    cudaSetDevice(prev);
    delete h;
}

#define CHECK_H(h)                                                                     \
    do {                                                                               \
        if (!(h)) return fa_fail(FA_ERR_INVALID, "null handle");                     \
        cudaError_t e_ = cudaSetDevice((h)->device);                                   \
        if (e_ != cudaSuccess) return fa_fail(FA_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_)); \
    } while (0)

extern "C" int fa_create(const uint8_t* rom, size_t rom_len, size_t n, fa_handle** out)
{
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    *out = nullptr;
    if (n == 0 || n > (size_t)0x7FFFFFFF) return fa_fail(FA_ERR_INVALID, "bad instance count %zu", n);
    if (fa_device_count() < 1) return fa_fail(FA_ERR_NO_DEVICE, "no CUDA device visible");
    fa_handle* h = new (std::nothrow) fa_handle();
    if (!h) return fa_fail(FA_ERR_CAPACITY, "out of host memory");
    int rc = fa_make_bank_image(rom, rom_len, h->image, h->scheme, &h->nbanks, &h->hot_lo);
    if (rc) { delete h; return rc; }
    h->n = n;
    h->stride = (uint32_t)((n + 31) & ~(size_t)31);
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
    // Default launch shape: the plain per-frame form, 128 threads per CTA.
    h->block = 128;
    h->sched = FA_SCHED_PC;
    cudaError_t e = cudaSuccess;
#define TRY(call) do { e = (call); if (e != cudaSuccess) { free_handle(h); \
        return fa_fail(FA_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e)); } } while (0)
    TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    TRY(cudaMalloc(&h->d_rom, h->image.size()));
    TRY(cudaMemcpy(h->d_rom, h->image.data(), h->image.size(), cudaMemcpyHostToDevice));
    const size_t state_words = (size_t)FA_ROWS * h->stride;
    TRY(cudaMalloc(&h->d_state, state_words * 4));
    TRY(cudaMemset(h->d_state, 0, state_words * 4));
    TRY(cudaMalloc(&h->d_snap, FA_ROWS * 4));
    TRY(cudaMalloc(&h->d_obs, n * 128));
    TRY(cudaMalloc(&h->d_err, 2 * sizeof(uint32_t)));
    TRY(cudaMemset(h->d_err, 0, 2 * sizeof(uint32_t)));
    TRY(cudaMalloc(&h->d_instr, 2 * sizeof(unsigned long long)));
    TRY(cudaMallocHost(&h->h_obs, n * 128));
    // The same pinned buffer as the kernels see it: host-buffer calls have
    // the kernel write observations there as its units finish, with no copy
    // after the launch.  Without a mapping they copy from d_obs instead.
    if (cudaHostGetDevicePointer((void**)&h->h_obs_dev, h->h_obs, 0) != cudaSuccess) {
        h->h_obs_dev = nullptr;
        (void)cudaGetLastError();
    }
    // Every instance starts zeroed and marked not-reset (stepping it is a no-op).
    {
        std::vector<uint32_t> st(h->stride, FA_STATUS_NOT_RESET);
        TRY(cudaMemcpy(h->d_state + (size_t)R_STATUS * h->stride, st.data(), h->stride * 4, cudaMemcpyHostToDevice));
    }
#undef TRY
    *out = h;
    return FA_OK;
}

extern "C" void fa_destroy(fa_handle* h) { free_handle(h); }

extern "C" size_t fa_num_envs(const fa_handle* h) { return h ? h->n : 0; }

extern "C" int fa_set_sorted(fa_handle* h, int sorted)
{
    if (!h) return fa_fail(FA_ERR_INVALID, "null handle");
    h->sched = sorted ? FA_SCHED_MATCH : FA_SCHED_LANE;
    return FA_OK;
}

static int ensure_actions(fa_handle* h, size_t bytes)
{
    if (bytes <= h->actions_cap) return FA_OK;
    cudaFree(h->d_actions);
    cudaFreeHost(h->h_actions);
    h->d_actions = nullptr;
    h->h_actions = nullptr;
    h->actions_cap = h->h_actions_cap = 0;
    FA_CUDA(cudaMalloc(&h->d_actions, bytes));
    FA_CUDA(cudaMallocHost(&h->h_actions, bytes));
    h->actions_cap = h->h_actions_cap = bytes;
    return FA_OK;
}

FaGroup fa_handle_group(fa_handle* h, const uint8_t* d_actions, uint32_t k, uint8_t* d_obs)
{
    FaGroup g;
    memset(&g, 0, sizeof(g));
    g.rom = h->d_rom;
    g.snapshot = h->have_snap ? h->d_snap : nullptr;
    g.state = h->d_state;
    g.actions = d_actions;
    g.obs = d_obs;
    g.stride = h->stride;
    g.n = (uint32_t)h->n;
    g.act_stride = (uint32_t)h->n;
    g.nbanks = h->nbanks;
    g.hot_lo = h->hot_lo;
    g.k = k;
    g.episode_frames = h->episode_frames;
    g.sched = (uint32_t)h->sched;
    g.unit_begin = 0;
    return g;
}

// Enqueue one launch over all instances of the handle.
static int enqueue_run(fa_handle* h, const FaGroup& g, cudaStream_t s)
{
    FaLaunch L;
    memset(&L, 0, sizeof(L));
    L.g[0] = g;
    L.ngroups = 1;
    L.nunits = (uint32_t)((g.n + h->block - 1) / h->block);
    L.rom_bytes_max = h->nbanks * 4096u;
    L.err = h->d_err;
    L.instr = h->d_instr;
    L.rounds = h->d_instr + 1;
    L.cta_warps = (uint32_t)h->cta_warps;
    if (h->persistent) {
        L.queue = h->d_err + 1;
        FA_CUDA(cudaMemsetAsync(L.queue, 0, sizeof(uint32_t), s));
    }
    FA_CUDA(fa_launch_run(L, h->block, h->persistent, h->sms, s));
    return FA_OK;
}

static int finish(fa_handle* h)
{
    FA_CUDA(cudaStreamSynchronize(h->stream));
    uint32_t err[2] = { 0, 0 };
    FA_CUDA(cudaMemcpy(err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    unsigned long long ctr[2];
    FA_CUDA(cudaMemcpy(ctr, h->d_instr, sizeof(ctr), cudaMemcpyDeviceToHost));
    h->last_instr = ctr[0];
    h->last_slots = ctr[1];
    if (err[0]) {
        cudaMemset(h->d_err, 0, sizeof(uint32_t));
        return fa_fail(FA_ERR_KERNEL, "device wait gave up (error word 0x%x)", err[0]);
    }
    return FA_OK;
}

extern "C" int fa_reset(fa_handle* h, uint8_t* obs_out)
{
    CHECK_H(h);
    // HeadlessAtari::new + one run_frame without set_action
    // (src/cuda_env.rs:134-139): one instance on the device, then broadcast.
    uint32_t col[FA_ROWS];
    fa_power_on_column(h->image.data(), h->nbanks, h->scheme, h->hot_lo, col);
    FA_CUDA(cudaMemcpyAsync(h->d_snap, col, sizeof(col), cudaMemcpyHostToDevice, h->stream));
    FaGroup g = fa_handle_group(h, nullptr, 1, nullptr);
    g.state = h->d_snap;
    g.stride = 1;
    g.n = 1;
    g.snapshot = nullptr;
    g.episode_frames = 0;
    g.sched = FA_SCHED_LANE;
    FA_CUDA(cudaMemsetAsync(h->d_instr, 0, 2 * sizeof(unsigned long long), h->stream));
    bool persistent = h->persistent;
    h->persistent = false;
    int rc = enqueue_run(h, g, h->stream);
    h->persistent = persistent;
    if (rc) return rc;
    FA_CUDA(cudaMemcpyAsync(col, h->d_snap, sizeof(col), cudaMemcpyDeviceToHost, h->stream));
    FA_CUDA(cudaStreamSynchronize(h->stream));
    col[R_FRAME] = 0;                      // episode counter restarts at reset
    FA_CUDA(cudaMemcpyAsync(h->d_snap, col, sizeof(col), cudaMemcpyHostToDevice, h->stream));
    FA_CUDA(fa_launch_broadcast(h->d_state, h->stride, (uint32_t)h->n, h->d_snap, h->stream));
    h->have_snap = true;
    rc = finish(h);
    if (rc) return rc;
    if (obs_out) {
        const uint8_t* ram = (const uint8_t*)col;
        for (size_t i = 0; i < h->n; i++) memcpy(obs_out + i * 128, ram, 128);
    }
    return FA_OK;
}

// Atari::new (src/atari.rs:240-247) as one rendering state column (FA_RROWS
// words): the headless power-on column with the rendering Tia's defaults
// (src/tia.rs:192-238), then the two bus reads of Cpu::reset
// (src/cpu.rs:125-134), which each tick three TIA clocks (in horizontal blank
// of scanline 0: nothing renders) and one PIA clock.
void fa_render_power_on_column(const uint8_t* image, uint32_t nbanks, int scheme, uint32_t hot_lo, uint32_t* col)
{
    memset(col, 0, FA_RROWS * sizeof(uint32_t));
    fa_power_on_column(image, nbanks, scheme, hot_lo, col);
    fa_state s;
    fa_unpack_column(col, 1, scheme, s);
    s.paddle0 = 128;
    s.paddle1 = 128;
    s.tia_clock = 6;
    // Pia::tick twice from its default (timer 0, prescaler 1, select 1).
    uint32_t tv = s.timer_value, ps = s.timer_prescaler, sel = s.timer_prescaler_select, uf = s.timer_underflow;
    for (int c = 0; c < 2; c++) {
        if (tv == 0 && uf) { tv = 0xFF; continue; }
        ps = (ps - 1u) & 0xFFFFu;
        if (ps == 0) {
            ps = uf ? 1u : sel;
            if (tv == 0) { uf = 1; tv = 0xFF; } else tv -= 1u;
        }
    }
    s.timer_value = (uint16_t)tv;
    s.timer_prescaler = (uint16_t)ps;
    s.timer_underflow = (uint8_t)uf;
    fa_pack_column(s, col, 1);
    // Rendering rows: pending_top 32 (RB_PTOP in the RB_* words), visible_top 32,
    // vblank_top 262, input latches 0x80.
    uint8_t rb[FA_RPRIV_BYTES - FA_PRIV_BYTES] = {};
    rb[RB_PTOP - FA_PRIV_BYTES] = 32;
    for (uint32_t w = 0; w < (FA_RPRIV_WORDS - FA_PRIV_WORDS); w++) memcpy(&col[FA_RROW_EXTRA + w], rb + 4 * w, 4);
    col[RR_VTOP] = 32u | (262u << 16);
    col[RR_FLAGS] = 4u | 8u;
}

// First-wave placement of a persistent launch (fa_pool_set_balance); host
// code, kept here so the host tests can run it.
void fa_plan_first_wave(const float* unit_cost, uint32_t nunits, uint32_t grid, uint32_t warps, uint32_t* table)
{
    const uint32_t slots = grid * warps, parts = grid * 4u, per_part = warps / 4u;
    std::fill(table, table + slots, 0xFFFFFFFFu);
    const uint32_t first = nunits < slots ? nunits : slots;
    // The first wave is units 0..first-1 (the device queue continues after
    // them), placed heaviest first, each on the least loaded sub-partition
    // that has a free slot: a (load, sub-partition) min-heap.
    std::vector<uint32_t> order(first);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return unit_cost[a] > unit_cost[b]; });
    std::vector<std::pair<double, uint32_t>> heap;
    heap.reserve(parts);
    for (uint32_t q = 0; q < parts; q++) heap.emplace_back(0.0, q);
    auto cmp = [](const std::pair<double, uint32_t>& a, const std::pair<double, uint32_t>& b) { return a > b; };
    std::make_heap(heap.begin(), heap.end(), cmp);
    std::vector<uint32_t> used(parts, 0);
    for (uint32_t u : order) {
        if (heap.empty()) break;
        std::pop_heap(heap.begin(), heap.end(), cmp);
        auto [load, q] = heap.back();
        heap.pop_back();
        const uint32_t cta = q / 4u, sub = q % 4u;
        const uint32_t warp = sub + 4u * used[q]++;                  // warp w issues from scheduler w % 4
        table[warp * grid + cta] = u;
        if (used[q] < per_part) {
            heap.emplace_back(load + unit_cost[u], q);
            std::push_heap(heap.begin(), heap.end(), cmp);
        }
    }
}

void fa_host_copy(void* dst, const void* src, size_t bytes)
{
    constexpr size_t kPerThread = 2u << 20;                           // below this one thread copies
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::min(std::min<size_t>(hw, 8), bytes / kPerThread);
    if (parts <= 1) {
        memcpy(dst, src, bytes);
        return;
    }
    const size_t per = (bytes + parts - 1) / parts;
    std::vector<std::thread> th;
    size_t covered = per;                                              // this thread copies [0, per)
    try {
        for (size_t off = per; off < bytes; off += per) {
            const size_t len = std::min(per, bytes - off);
            th.emplace_back([=] { memcpy((uint8_t*)dst + off, (const uint8_t*)src + off, len); });
            covered = off + len;
        }
    } catch (...) {                                                    // no thread: the rest here
    }
    memcpy(dst, src, per);
    if (covered < bytes) memcpy((uint8_t*)dst + covered, (const uint8_t*)src + covered, bytes - covered);
    for (auto& t : th) t.join();
}

static int step_host(fa_handle* h, const uint8_t* actions, int k, uint8_t* obs_out)
{
    CHECK_H(h);
    if (!actions || k < 1) return fa_fail(FA_ERR_INVALID, "actions null or k < 1");
    const size_t bytes = (size_t)k * h->n;
    int rc = ensure_actions(h, bytes);
    if (rc) return rc;
    memcpy(h->h_actions, actions, bytes);
    FA_CUDA(cudaMemcpyAsync(h->d_actions, h->h_actions, bytes, cudaMemcpyHostToDevice, h->stream));
    FA_CUDA(cudaMemsetAsync(h->d_instr, 0, 2 * sizeof(unsigned long long), h->stream));
    uint8_t* obs_dst = obs_out ? (h->h_obs_dev ? h->h_obs_dev : h->d_obs) : nullptr;
    rc = enqueue_run(h, fa_handle_group(h, h->d_actions, (uint32_t)k, obs_dst), h->stream);
    if (rc) return rc;
    if (obs_out && !h->h_obs_dev)
        FA_CUDA(cudaMemcpyAsync(h->h_obs, h->d_obs, h->n * 128, cudaMemcpyDeviceToHost, h->stream));
    rc = finish(h);
    if (rc) return rc;
    if (obs_out) fa_host_copy(obs_out, h->h_obs, h->n * 128);
    return FA_OK;
}

extern "C" int fa_step(fa_handle* h, const uint8_t* actions, uint8_t* obs_out)
{
    return step_host(h, actions, 1, obs_out);
}

extern "C" int fa_step_multi(fa_handle* h, const uint8_t* actions, int k, uint8_t* obs_out)
{
    return step_host(h, actions, k, obs_out);
}

extern "C" int fa_step_multi_async(fa_handle* h, const uint8_t* d_actions, int k, uint8_t* d_obs, void* stream)
{
    CHECK_H(h);
    if (!d_actions || k < 1) return fa_fail(FA_ERR_INVALID, "actions null or k < 1");
    if (((uintptr_t)d_obs & 15u) != 0) return fa_fail(FA_ERR_INVALID, "d_obs must be 16-byte aligned");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    return enqueue_run(h, fa_handle_group(h, d_actions, (uint32_t)k, d_obs), s);
}

extern "C" int fa_synchronize(fa_handle* h)
{
    CHECK_H(h);
    FA_CUDA(cudaDeviceSynchronize());
    return finish(h);
}

extern "C" int fa_get_states(fa_handle* h, fa_state* out)
{
    CHECK_H(h);
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    std::vector<uint32_t> buf((size_t)FA_ROWS * h->stride);
    FA_CUDA(cudaStreamSynchronize(h->stream));
    FA_CUDA(cudaMemcpy(buf.data(), h->d_state, buf.size() * 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < h->n; i++) fa_unpack_column(buf.data() + i, h->stride, h->scheme, out[i]);
    return FA_OK;
}

extern "C" int fa_set_states(fa_handle* h, const fa_state* in)
{
    CHECK_H(h);
    if (!in) return fa_fail(FA_ERR_INVALID, "in is null");
    std::vector<uint32_t> buf((size_t)FA_ROWS * h->stride, 0);
    for (size_t i = 0; i < h->n; i++) {
        if (in[i].timer_prescaler_select == 0)
            return fa_fail(FA_ERR_INVALID, "instance %zu: timer_prescaler_select 0 (reference divides by it)", i);
        fa_state s = in[i];
        if (s.bank >= h->nbanks) s.bank = (uint8_t)(h->nbanks - 1);
        if (fa_map_kind(h->hot_lo)) s.bank = 0;                 // sliced carts keep their banks in `mapper`
        // E0 slices to 3 bits, 3F banks modulo the bank count, 0 for the 4K-bank schemes.
        const uint32_t m = fa_mapper_from_slices(
            h->hot_lo, fa_slices_from_mapper(h->hot_lo, (uint32_t)s.mapper[0] | ((uint32_t)s.mapper[1] << 8)));
        s.mapper[0] = (uint8_t)m;
        s.mapper[1] = (uint8_t)(m >> 8);
        // The DPC registers end the struct; other schemes do not take them.
        if (fa_map_kind(h->hot_lo) != FA_MAP_DPC)
            memset(&s.dpc_counter, 0, sizeof(fa_state) - offsetof(fa_state, dpc_counter));
        fa_pack_column(s, buf.data() + i, h->stride);
    }
    FA_CUDA(cudaStreamSynchronize(h->stream));
    FA_CUDA(cudaMemcpy(h->d_state, buf.data(), buf.size() * 4, cudaMemcpyHostToDevice));
    return FA_OK;
}

extern "C" int fa_get_ram(fa_handle* h, size_t idx, uint8_t* out128)
{
    CHECK_H(h);
    if (!out128 || idx >= h->n) return fa_fail(FA_ERR_INVALID, "bad index %zu", idx);
    FA_CUDA(cudaStreamSynchronize(h->stream));
    uint32_t w[32];
    FA_CUDA(cudaMemcpy2D(w, 4, h->d_state + idx, (size_t)h->stride * 4, 4, 32, cudaMemcpyDeviceToHost));
    memcpy(out128, w, 128);
    return FA_OK;
}

extern "C" int fa_get_status(fa_handle* h, uint32_t* out)
{
    CHECK_H(h);
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    FA_CUDA(cudaStreamSynchronize(h->stream));
    FA_CUDA(cudaMemcpy(out, h->d_state + (size_t)R_STATUS * h->stride, h->n * 4, cudaMemcpyDeviceToHost));
    return FA_OK;
}

extern "C" int fa_set_episode_frames(fa_handle* h, uint32_t episode_frames)
{
    if (!h) return fa_fail(FA_ERR_INVALID, "null handle");
    h->episode_frames = episode_frames;
    return FA_OK;
}

extern "C" int fa_set_frame_numbers(fa_handle* h, const uint32_t* frame_no)
{
    CHECK_H(h);
    if (!frame_no) return fa_fail(FA_ERR_INVALID, "frame_no is null");
    FA_CUDA(cudaStreamSynchronize(h->stream));
    FA_CUDA(cudaMemcpy(h->d_state + (size_t)R_FRAME * h->stride, frame_no, h->n * 4, cudaMemcpyHostToDevice));
    return FA_OK;
}

extern "C" int fa_set_launch(fa_handle* h, int block, int sched, int persistent)
{
    if (!h) return fa_fail(FA_ERR_INVALID, "null handle");
    if (block != 64 && block != 128 && block != 256 && block != 512)
        return fa_fail(FA_ERR_INVALID, "block must be 64, 128, 256 or 512");
    if (sched < FA_SCHED_LANE || sched > FA_SCHED_MATCH) return fa_fail(FA_ERR_INVALID, "bad sched %d", sched);
    h->block = block;
    h->sched = sched;
    h->persistent = persistent != 0;
    return FA_OK;
}

extern "C" int fa_set_cta_warps(fa_handle* h, int warps)
{
    if (!h) return fa_fail(FA_ERR_INVALID, "null handle");
    if (warps != 0 && warps != 2 && warps != 4 && warps != 8 && warps != 16 && warps != 24 && warps != 28 &&
        warps != 32)
        return fa_fail(FA_ERR_INVALID, "warps per CTA must be 0 (auto), 2, 4, 8, 16, 24, 28 or 32");
    h->cta_warps = warps;
    return FA_OK;
}

extern "C" int fa_get_launch(const fa_handle* h, int* block, int* sched, int* persistent)
{
    if (!h) return fa_fail(FA_ERR_INVALID, "null handle");
    if (block) *block = h->block;
    if (sched) *sched = h->sched;
    if (persistent) *persistent = h->persistent ? 1 : 0;
    return FA_OK;
}

extern "C" unsigned long long fa_last_instructions(const fa_handle* h)
{
    return h ? h->last_instr : 0ull;
}

extern "C" unsigned long long fa_last_lane_slots(const fa_handle* h)
{
    return h ? h->last_slots : 0ull;
}

extern "C" int fa_get_snapshot(fa_handle* h, fa_state* out)
{
    CHECK_H(h);
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    if (!h->have_snap) return fa_fail(FA_ERR_INVALID, "no reset snapshot yet");
    uint32_t col[FA_ROWS];
    FA_CUDA(cudaStreamSynchronize(h->stream));
    FA_CUDA(cudaMemcpy(col, h->d_snap, sizeof(col), cudaMemcpyDeviceToHost));
    fa_unpack_column(col, 1, h->scheme, *out);
    return FA_OK;
}

extern "C" void* fa_device_state(fa_handle* h, uint32_t* stride_words)
{
    if (!h) return nullptr;
    if (stride_words) *stride_words = h->stride;
    return h->d_state;
}
