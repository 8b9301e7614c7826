// Test infrastructure: the device core run on the host.  fa_device.cuh's Emu
// and fa_run.cuh's Runner step one instance at a time (one lane, so the
// warp scheduler of run_lanes is not involved: it only orders the lanes),
// over the bank image, SoA state columns and packing of fa_api.cu.  run_one
// follows run_unit_as (fa_run.cuh) for one lane.
#include "shim.h"
#include "../../fast-atari-rs_b200/csrc/fa_api.cu"
#include "../../fast-atari-rs_b200/csrc/fa_run.cuh"
#include "../../fast-atari-rs_b200/csrc/fa_render.cuh"

template <bool SL, bool DPC = false, bool FE = false>
static void run_one(const FaGroup& G, uint32_t i, uint8_t* rom, unsigned long long* instr)
{
    uint32_t priv[FA_SMEM_WORDS];
    fa::Runner<1, SL, DPC, FE> r;
    r.f = 0; r.phase = 0; r.fcyc = 0; r.active = false;
    r.e.pv = (uint8_t*)priv;
    r.e.G = &G; r.e.i = i; r.e.rom = rom; r.e.hot_lo = G.hot_lo; r.e.nbanks = G.nbanks;
    r.e.instr = 0; r.e.cyc_acc = 0; r.e.pc = 0; r.e.bank = 0; r.e.slices = 0; r.e.scanline = 0;
    uint32_t* col = G.state + i;
    r.e.load_ram(col, G.stride);
    r.e.load_hot(col, G.stride);
    if (G.k > 0) r.active = r.begin_frame();
    while (r.active) r.iterate();
    r.e.fold_cycles();
    if (G.actions && r.f + 1u < G.k && (r.e.row(R_STATUS) & FA_STATUS_HALT_MASK))       // as run_unit_as
        r.e.apply_action(G.actions[(size_t)(G.k - 1u) * G.act_stride + r.e.i]);
    r.e.store_ram(col, G.stride);
    r.e.store_hot(col, G.stride);
    *instr += r.e.instr;
}

extern "C" long long hs_run(const uint8_t* rom, size_t len, fa_state* st, size_t n, const uint8_t* actions, int k)
{
    std::vector<uint8_t> img;
    int scheme = 0;
    uint32_t nbanks = 0, hot_lo = 0;
    if (fa_make_bank_image(rom, len, img, scheme, &nbanks, &hot_lo)) return -1;
    std::vector<uint8_t> simg(img.size() + 64, 0);
    memcpy(simg.data(), img.data(), img.size());
    std::vector<uint32_t> rows((size_t)FA_ROWS * n);
    for (size_t i = 0; i < n; i++) fa_pack_column(st[i], rows.data() + i, n);
    FaGroup G;
    memset(&G, 0, sizeof(G));
    G.rom = simg.data(); G.state = rows.data(); G.stride = (uint32_t)n; G.n = (uint32_t)n;
    G.actions = actions; G.act_stride = (uint32_t)n; G.nbanks = nbanks; G.hot_lo = hot_lo; G.k = (uint32_t)k;
    unsigned long long instr = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (fa_map_kind(hot_lo) == FA_MAP_DPC) run_one<true, true>(G, i, simg.data(), &instr);   // as run_unit
        else if (fa_map_kind(hot_lo) == FA_MAP_FE) run_one<true, false, true>(G, i, simg.data(), &instr);
        else if (fa_map_kind(hot_lo)) run_one<true>(G, i, simg.data(), &instr);
        else run_one<false>(G, i, simg.data(), &instr);
    }
    for (size_t i = 0; i < n; i++) fa_unpack_column(rows.data() + i, n, scheme, st[i]);
    return (long long)instr;
}

// The timer bookkeeping of the headless core: one console counts calls
// lazily (Emu::pia_count), the other runs every call exactly (Emu::pia_tick,
// Pia::tick_n).  After call c, settle[c] is 1: a settle (Emu::pia_settle),
// 2: a settle then an INTIM read (Emu::pia_intim: settles, clears the
// underflow flag), 3: an INTIM read alone.  Both then report (value,
// prescaler, select, underflow) as the state would be stored:
// out[8 * c + 0..3] lazy, out[8 * c + 4..7] exact.
extern "C" void hs_timer(const uint32_t* start, const uint32_t* ns, const uint8_t* settle, int m, uint32_t* out)
{
    fa::Emu<1> lz, ex;
    memset(&lz, 0, sizeof(lz));
    memset(&ex, 0, sizeof(ex));
    lz.tp = ex.tp = start[0] | (start[1] << 16);
    lz.su = ex.su = start[2] | (start[3] << 16);
    lz.tlim = lz.pia_span();
    for (int c = 0; c < m; c++) {
        lz.pia_count(ns[c]);
        ex.pia_tick(ns[c]);
        if (settle[c] == 1 || settle[c] == 2) lz.pia_settle();
        if (settle[c] >= 2) {
            lz.pia_intim();
            ex.su &= 0xFFFFu;
        }
        const uint2 t = lz.pia_now();
        uint32_t* o = out + 8 * (size_t)c;
        o[0] = t.x; o[1] = t.y; o[2] = lz.su & 0xFFFFu; o[3] = lz.su >> 16;
        o[4] = ex.tp & 0xFFFFu; o[5] = ex.tp >> 16; o[6] = ex.su & 0xFFFFu; o[7] = ex.su >> 16;
    }
}

// The persistent launch's first-wave placement (fa_pool_set_balance).
extern "C" void hs_plan(const float* cost, uint32_t nunits, uint32_t grid, uint32_t warps, uint32_t* table)
{
    fa_plan_first_wave(cost, nunits, grid, warps, table);
}

// The threaded copy of host-buffer calls' outputs into the caller's memory.
extern "C" void hs_host_copy(void* dst, const void* src, size_t bytes) { fa_host_copy(dst, src, bytes); }

// The rendering console (RRunner, fa_render.cuh, over the device console)
// on the host, one console at a time, the way fa_render_reset and
// fa_render_step_multi drive it: power-on column, one frame without an
// action (frame numbers then restart at 0), then `calls` calls of k frames
// with actions[call][frame][console].  Returns the framebuffers (n x 30,720),
// the states and the RAM after the last call; -1 for a bad ROM.
//
// render_one restates fa_render_run's start and end of a launch for one
// console (the kernel keeps those steps in its own body): private words and
// packed state in from the rows, the beam and framebuffer resumed, the TIA
// latches from the flags row, the first frame's set_action; at the end the
// visible framebuffer, the owed cycles, a halted console's last action, the
// rows written back and the RAM to obs.
template <bool SL>
static void render_one(FaGroup& G, uint32_t i, const uint8_t* rom, uint8_t* fb, uint8_t* obs)
{
    using namespace fa;
    uint32_t w[FA_RSLAB_WORDS * 32];
    memset(w, 0, sizeof(w));
    RRunner<SL> r;
    r.f = 0;
    r.phase = 0;
    r.fcyc = 0;
    r.active = false;
    Emu<32, true, SL>& e = r.e;
    e.pv = (uint8_t*)w;
    e.G = &G;
    e.i = i;
    e.rom = rom;
    e.hot_lo = G.hot_lo;
    e.nbanks = G.nbanks;
    e.instr = 0;
    e.cyc_acc = 0;
    e.pc = 0;
    e.bank = 0;
    e.slices = 0;
    e.scanline = 0;
    e.done = 0;
    e.lag = 0;
    e.sc = 0;
    e.zr = 0;
    e.vtop = 0;
    e.rx = 0;
    e.fbp = fb + (size_t)i * FA_FB_BYTES;
    uint32_t* col = G.state + i;
    const uint32_t S = G.stride;
    for (uint32_t q = 0; q < FA_PRIV_WORDS; q++) w[q * 32u] = col[(size_t)q * S];
    for (uint32_t q = FA_PRIV_WORDS; q < FA_RPRIV_WORDS; q++) w[q * 32u] = col[(size_t)(FA_RROW_EXTRA + (q - FA_PRIV_WORDS)) * S];
    e.load_hot(col, S);
    e.vtop = col[(size_t)RR_VTOP * S];
    e.rx = e.clock;
    e.fb_resume();
    const uint32_t fl = col[(size_t)RR_FLAGS * S];
    e.tw |= ((fl & 1u) ? TW_HMOVE : 0u) | ((fl & 2u) ? TW_LATCH : 0u) | ((fl & 4u) ? TW_L4 : 0u) | ((fl & 8u) ? TW_L5 : 0u);
    if (G.k > 0) r.active = r.begin_frame();
    while (r.active) r.iterate();
    e.fb_observe();
    e.fold_cycles();
    if (G.actions && r.f + 1u < G.k && (e.row(R_STATUS) & FA_STATUS_HALT_MASK))
        e.apply_action(G.actions[(size_t)(G.k - 1u) * G.act_stride + i]);
    for (uint32_t q = 0; q < FA_PRIV_WORDS; q++) col[(size_t)q * S] = w[q * 32u];
    for (uint32_t q = FA_PRIV_WORDS; q < FA_RPRIV_WORDS; q++) col[(size_t)(FA_RROW_EXTRA + (q - FA_PRIV_WORDS)) * S] = w[q * 32u];
    e.store_hot(col, S);
    col[(size_t)RR_VTOP * S] = e.vtop;
    col[(size_t)RR_FLAGS * S] = ((e.tw & TW_HMOVE) ? 1u : 0u) | ((e.tw & TW_LATCH) ? 2u : 0u) | ((e.tw & TW_L4) ? 4u : 0u) |
                                ((e.tw & TW_L5) ? 8u : 0u);
    if (obs)
        for (uint32_t q = 0; q < 32u; q++) memcpy(obs + (size_t)i * 128u + 4u * q, &w[q * 32u], 4);
}

extern "C" long long hs_render(const uint8_t* rom, size_t len, size_t n, const uint8_t* actions, int calls, int k,
                               uint8_t* fb, fa_state* st, uint8_t* ram)
{
    std::vector<uint8_t> img;
    int scheme = 0;
    uint32_t nbanks = 0, hot_lo = 0;
    if (fa_make_bank_image(rom, len, img, scheme, &nbanks, &hot_lo)) return -1;
    std::vector<uint8_t> simg(img.size() + 64, 0);
    memcpy(simg.data(), img.data(), img.size());
    std::vector<uint32_t> col(FA_RROWS);
    fa_render_power_on_column(img.data(), nbanks, scheme, hot_lo, col.data());
    std::vector<uint32_t> rows((size_t)FA_RROWS * n);
    for (uint32_t w = 0; w < FA_RROWS; w++)
        for (size_t i = 0; i < n; i++) rows[(size_t)w * n + i] = col[w];
    memset(fb, 0, n * (size_t)FA_FB_BYTES);
    FaGroup G;
    memset(&G, 0, sizeof(G));
    G.rom = simg.data(); G.state = rows.data(); G.stride = (uint32_t)n; G.n = (uint32_t)n;
    G.act_stride = (uint32_t)n; G.nbanks = nbanks; G.hot_lo = hot_lo;
    const bool sliced = fa_map_kind(hot_lo) != 0;
    long long instr = 0;
    for (int c = -1; c < calls; c++) {
        G.actions = c < 0 ? nullptr : actions + (size_t)c * k * n;
        G.k = c < 0 ? 1u : (uint32_t)k;
        for (uint32_t i = 0; i < n; i++) {
            if (sliced) render_one<true>(G, i, simg.data(), fb, ram);
            else render_one<false>(G, i, simg.data(), fb, ram);
        }
        if (c < 0)
            for (size_t i = 0; i < n; i++) rows[(size_t)R_FRAME * n + i] = 0;
    }
    for (size_t i = 0; i < n; i++) fa_unpack_column(rows.data() + i, n, scheme, st[i]);
    return instr;
}
