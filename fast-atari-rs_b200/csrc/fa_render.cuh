// fa_render.cuh — one rendering console per lane: the frame loop, shared by
// the rendering kernel (fa_render.cu) and the host tests that run the same
// code on the CPU.  The kernel's start and end of a launch (the console's
// rows in and out of HBM) stay in the kernel body: moved into helpers here,
// the same steps ran 8 % slower on the render cart.
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

}  // namespace fa
