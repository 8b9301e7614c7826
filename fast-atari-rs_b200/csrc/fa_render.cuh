// fa_render.cuh — one rendering console per lane: the frame loop and the
// per-console start and end of a launch, shared by the rendering kernel
// (fa_render.cu) and the host tests that run the same code on the CPU.
#pragma once

#include "fa_run.cuh"

namespace fa {

// One rendering console per lane: HeadlessAtari's frame loop with the
// rendering console's per-cycle run_one_cycle (src/atari.rs:284-318).
template <bool SLICED>
struct RRunner {
    Emu<32, true, SLICED> e;
    uint32_t f, phase, fcyc;
    bool active;

    // set_action, then run_frame, which does nothing for a halted console
    // (src/atari.rs:250-270, 284-306): a halted console's inputs still take
    // the frame's action.
    __device__ __forceinline__ bool begin_frame()
    {
        const FaGroup* G = e.G;
        if (G->actions) e.apply_action(G->actions[(size_t)f * G->act_stride + e.i]);
        if (e.row(R_STATUS) & FA_STATUS_HALT_MASK) return false;
        e.tw &= ~TW_FCOMP;
        e.bank &= 7u;
        fcyc = 0;
        phase = e.vsync_on() ? 0u : 1u;
        return true;
    }
    // One run_one_cycle: a WSYNC cycle (tick_components) or an instruction,
    // then the frame-end checks of run_frame.
    __device__ __forceinline__ bool one()
    {
        uint32_t n;
        if (e.wsync()) e.settle();                                   // the wait starts where the beam is
        if (e.wsync()) {
            // The cycles of a WSYNC wait up to the end of the line, cut where
            // a per-cycle frame check would first fire: nothing else changes
            // from one cycle of the wait to the next.
            n = (228u - e.clock + 2u) / 3u;
            uint32_t lim;
            if (phase == 0u) lim = e.vsync_on() ? FA_VSYNC_BUDGET + 1u - fcyc : 1u;
            else lim = FA_FRAME_CYCLE_CAP + 1u - fcyc;
            n = n < lim ? n : lim;
            e.rcycles(n);
        } else {
            e.done = 0u - e.lag;
            n = e.step();
            if (n == 0) {
                // The reference's opcode fetch was a bus access (one cycle of
                // TIA and PIA) before it stopped (src/cpu.rs:1139-1141): the
                // TIA and PIA are owed up to the end of that cycle.
                e.lag = 1u - e.done;
                e.fold_cycles();
                e.set_status(FA_STATUS_ILLEGAL_OPCODE);
                active = false;
                return false;
            }
            e.lag = n - e.done;
            e.instr++;
            e.cyc_acc += n;
        }
        fcyc += n;
        if (phase == 0u) {
            if (fcyc > FA_VSYNC_BUDGET) {
                e.fold_cycles();
                e.set_status(FA_STATUS_VSYNC_BUDGET);
                active = false;
                return false;
            }
            if (!e.vsync_on()) phase = 1u;
        } else {
            const bool cap = fcyc > FA_FRAME_CYCLE_CAP;
            if (cap || e.vsync_on()) {
                if (cap) e.set_status(FA_STATUS_CYCLE_CAP);
                e.fb_observe();                                      // before the next frame's action moves the pins
                e.fold_cycles();
                e.row(R_FRAME) += 1u;
                f++;
                if (f >= e.G->k || !begin_frame()) { active = false; return false; }
                return false;
            }
        }
        return e.wsync();
    }
    __device__ __forceinline__ uint32_t key(uint32_t sched) const
    {
        const uint32_t fc = f < 0x7Fu ? f : 0x7Fu;
        const uint32_t mid = sched == FA_SCHED_LINE ? (e.scanline < 0x1FFu ? e.scanline : 0x1FFu) : (e.bank >> 3);
        return (fc << 25) | (mid << 16) | e.pc;
    }
    // A WSYNC wait is consumed without going back to the warp scheduler.
    __device__ __forceinline__ void iterate()
    {
#pragma unroll 1
        while (one() && active) {
        }
    }
};

// A console's start of a launch: its private bytes (RAM and the rendering
// registers) from the HBM rows into its slab words w (32-lane interleave),
// its packed state, the beam where the last call left it, its framebuffer
// sector, the TIA latches, then the first frame's set_action.
template <bool SLICED>
__device__ __forceinline__ void render_begin(RRunner<SLICED>& r, uint32_t* w, const FaGroup* G, uint32_t i, bool valid,
                                             const uint8_t* rom, uint8_t* fbp, uint32_t* col, uint32_t S)
{
    r.f = 0;
    r.phase = 0;
    r.fcyc = 0;
    r.active = false;
    Emu<32, true, SLICED>& e = r.e;
    e.pv = (uint8_t*)w;
    e.G = G;
    e.i = i;
    e.rom = rom;
    e.hot_lo = G->hot_lo;
    e.nbanks = G->nbanks;
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
    e.fbp = fbp;
    if (!valid) return;
#pragma unroll 4
    for (uint32_t k = 0; k < FA_PRIV_WORDS; k++) w[k * 32u] = col[(size_t)k * S];
    for (uint32_t k = FA_PRIV_WORDS; k < FA_RPRIV_WORDS; k++) w[k * 32u] = col[(size_t)(FA_RROW_EXTRA + (k - FA_PRIV_WORDS)) * S];
    e.load_hot(col, S);
    e.vtop = col[(size_t)RR_VTOP * S];
    e.rx = e.clock;
    e.fb_resume();
    const uint32_t fl = col[(size_t)RR_FLAGS * S];
    e.tw |= ((fl & 1u) ? TW_HMOVE : 0u) | ((fl & 2u) ? TW_LATCH : 0u) | ((fl & 4u) ? TW_L4 : 0u) | ((fl & 8u) ? TW_L5 : 0u);
    if (G->k > 0) r.active = r.begin_frame();
}

// A console's end of a launch: the framebuffer as it can be seen, the owed
// cycles, then everything back to its HBM rows, and its RAM to obs (128
// bytes, 16-byte aligned) when obs is not null.
template <bool SLICED>
__device__ __forceinline__ void render_end(RRunner<SLICED>& r, uint32_t* w, uint32_t* col, uint32_t S, uint8_t* obs)
{
    Emu<32, true, SLICED>& e = r.e;
    const FaGroup* G = e.G;
    e.fb_observe();
    e.fold_cycles();
    // A console that halted before the call's last frame took the later
    // frames' set_action too; the last one is what its inputs hold.
    if (G->actions && r.f + 1u < G->k && (e.row(R_STATUS) & FA_STATUS_HALT_MASK))
        e.apply_action(G->actions[(size_t)(G->k - 1u) * G->act_stride + e.i]);
#pragma unroll 4
    for (uint32_t k = 0; k < FA_PRIV_WORDS; k++) col[(size_t)k * S] = w[k * 32u];
    for (uint32_t k = FA_PRIV_WORDS; k < FA_RPRIV_WORDS; k++) col[(size_t)(FA_RROW_EXTRA + (k - FA_PRIV_WORDS)) * S] = w[k * 32u];
    e.store_hot(col, S);
    col[(size_t)RR_VTOP * S] = e.vtop;
    col[(size_t)RR_FLAGS * S] = ((e.tw & TW_HMOVE) ? 1u : 0u) | ((e.tw & TW_LATCH) ? 2u : 0u) |
                                ((e.tw & TW_L4) ? 4u : 0u) | ((e.tw & TW_L5) ? 8u : 0u);
    if (obs) {
        uint4* o = (uint4*)obs;
#pragma unroll
        for (uint32_t q = 0; q < 8u; q++)
            o[q] = make_uint4(w[(4u * q) * 32u], w[(4u * q + 1u) * 32u], w[(4u * q + 2u) * 32u], w[(4u * q + 3u) * 32u]);
    }
}

}  // namespace fa
