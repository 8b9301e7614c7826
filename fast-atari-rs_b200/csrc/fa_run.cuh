// fa_run.cuh — device code shared by the library's kernels: bounded TMA bulk
// staging on an mbarrier, and the per-unit runner (frame loop, warp
// scheduling policies, one unit of instances from HBM rows to HBM rows).
// Included by fa_kernels.cu (pool/handle kernels) and fa_serve_kernel.cu
// (serving kernel, compiled with L1-bypassing global loads).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fa_device.cuh"
#include "fa_internal.h"

namespace fa {

// ------------------------------------------------------------------ TMA / mbarrier
// Default bound of every device wait (fa_set_wait_limit_ns changes the
// bound of the ROM staging wait of later launches).
constexpr uint64_t FA_WAIT_LIMIT_NS = 2000000000ull;   // 2 s

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Waits for phase `parity` of the barrier for at most limit_ns nanoseconds
// (a limit of 0 gives up without waiting).  Bounded in time, not in
// iterations: one try_wait may suspend for an implementation-defined interval.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns)
{
    const uint64_t t0 = globaltimer_ns();
    while (globaltimer_ns() - t0 < limit_ns)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// After a wait that gave up: the copies already issued still land in this
// CTA's shared memory, so the CTA waits for them (bounded by the default
// limit) before it reuses that memory or exits.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity)
{
    (void)mbar_wait_bounded(bar, parity, FA_WAIT_LIMIT_NS);
}

// Stage `bytes` (a multiple of 4 KiB) of ROM into shared memory.  Called by
// every thread of the CTA after a __syncthreads; returns false if the copy
// did not complete within limit_ns (the launch's wait bound).
static __device__ bool stage_rom(uint8_t* dst, const uint8_t* src, uint32_t bytes, uint64_t* bar, uint32_t& phase,
                                 uint64_t limit_ns)
{
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bar, bytes);
        for (uint32_t off = 0; off < bytes; off += 4096u) bulk_g2s(dst + off, src + off, 4096u, bar);
    }
    const bool ok = mbar_wait_bounded(bar, phase, limit_ns);
    if (!ok) mbar_drain(bar, phase);
    phase ^= 1u;
    return ok;
}

// ------------------------------------------------------------------ per-unit runner
template <int BLOCK, bool SLICED = false, bool DPC = false, bool FE = false>
struct Runner {
    Emu<BLOCK, false, SLICED, DPC, FE> e;
    uint32_t f, phase, fcyc;
    bool active;

    // Start frame f in the order of one frame of a batched step: the
    // periodic reset, set_action (src/atari.rs:571-582), then run_frame
    // (:584-586), which does nothing for a halted instance.  False if the
    // instance is halted: its inputs still take the frame's action.
    __device__ __forceinline__ bool begin_frame()
    {
        const FaGroup* G = e.G;
        if (G->episode_frames && G->snapshot && e.row(R_FRAME) >= G->episode_frames) {
            e.load_ram(G->snapshot, 1);
            // The DPC rows only for the DPC core: they stay 0 for every other
            // scheme, and a loop over them made the other cores' code longer
            // and slower.
            for (uint32_t w = FA_SMEM_WORDS; w < (DPC ? (uint32_t)FA_ROWS : (uint32_t)R_DPC_CNT); w++)
                e.row(w) = G->snapshot[w];
            e.load_hot(G->snapshot, 1);
        }
        if (G->actions) e.apply_action(G->actions[(size_t)f * G->act_stride + e.i]);
        if (e.row(R_STATUS) & FA_STATUS_HALT_MASK) return false;
        e.tw &= ~TW_FCOMP;
        fcyc = 0;
        e.bank &= 7u;
        phase = e.vsync_on() ? 0u : 1u;
        return true;
    }

    // One HeadlessAtari::run_one_cycle (src/atari.rs:601-614) plus the frame
    // loop checks of run_frame (src/atari.rs:584-598).  Returns true when the
    // lane should run again immediately (a WSYNC skip is pending).
    __device__ __forceinline__ bool one()
    {
        uint32_t n;
        if (e.wsync()) {
            n = e.tia_skip();
        } else {
            n = e.step();
            if (n == 0) { e.fold_cycles(); e.set_status(FA_STATUS_ILLEGAL_OPCODE); active = false; return false; }
            e.instr++;
            e.cyc_acc += n;
            e.tia_tick(n);
        }
        e.pia_count(n);
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
                e.fold_cycles();
                e.row(R_FRAME) += 1u;
                f++;
                if (f >= e.G->k || !begin_frame()) { active = false; return false; }
                return false;
            }
        }
        return e.wsync();
    }

    // Scheduling key, a measure of how far the lane has progressed: frame,
    // then the hotspot accesses of this frame (FA_SCHED_PC; the same code
    // address in two banks is two program points, and a lane that has
    // switched banks once more is ahead whatever its pc) or the scanline
    // (FA_SCHED_LINE), then pc.
    __device__ __forceinline__ uint32_t key(uint32_t sched) const
    {
        const uint32_t fc = f < 0x7Fu ? f : 0x7Fu;
        const uint32_t mid = sched == FA_SCHED_LINE ? (e.scanline < 0x1FFu ? e.scanline : 0x1FFu) : (e.bank >> 3);
        return (fc << 25) | (mid << 16) | e.pc;
    }

    // Up to three run_one_cycle calls per scheduler step (an instruction, a
    // WSYNC skip it starts, one more); on the mixed batch this measured 4 %
    // faster than two (19.4 against 18.6 M frames/s on one B200), with the
    // same results, since the policy only changes when lanes are polled.
    __device__ __forceinline__ void iterate()
    {
#pragma unroll 1
        for (int rep = 0; rep < 3; rep++)
            if (!one() || !active) break;
    }
};

// Runs every lane of the warp to the end of its frames.  The policy only
// decides which lanes execute in each round; all lanes share one call site of
// the emulator so its code is instantiated once.
// Instructions a converged group may run per scheduling round.
constexpr uint32_t FA_STEPS_PER_ROUND = 32;

template <class RUNNER>
__device__ __forceinline__ uint32_t run_lanes(RUNNER& r, uint32_t sched)
{
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const bool converge = sched == FA_SCHED_PC || sched == FA_SCHED_LINE;
    uint32_t rem = 0, grp = 0, rounds = 0;
    while (true) {
        const bool act = r.active;
        const uint32_t pcb = (r.e.bank << 16) | r.e.pc;
        bool go;
        uint32_t gm = FULL, lead = 0, wait_key = 0;
        if (sched == FA_SCHED_MATCH) {
            // __match_any_sync groups lanes by (bank, pc); each group runs its
            // instruction together, every group once per round.
            if (rem == 0) {
                rem = __ballot_sync(FULL, act);
                if (!rem) break;
                grp = __match_any_sync(FULL, act ? pcb : 0xFFFFFFFFu);
            }
            const uint32_t g = __shfl_sync(FULL, grp, __ffs(rem) - 1u);
            go = (g >> lane) & 1u;
            rem &= ~g;
        } else if (converge) {
            // Convergence scheduling: the lane furthest behind (key()) leads
            // and every lane at the leader's (bank and bank-switch count, pc)
            // runs with it.  Lanes that branched ahead wait
            // until the others reach the same pc, so the warp re-converges.
            if (!__any_sync(FULL, act)) break;
            const uint32_t key = act ? r.key(sched) : 0xFFFFFFFFu;
            const uint32_t mk = __reduce_min_sync(FULL, key);
            lead = __ffs(__ballot_sync(FULL, key == mk)) - 1u;
            // Every lane takes part in the full-mask shuffle, so it is not
            // folded into a short-circuit condition.
            const uint32_t lpcb = __shfl_sync(FULL, pcb, lead);
            go = act && pcb == lpcb;
            gm = __ballot_sync(FULL, go);
            // The smallest key among the lanes left waiting: the group keeps
            // running only while every member's key stays below it (so it
            // stops where a waiting lane could join); it may stop earlier than
            // needed, never later, so the order of execution is the one
            // one-instruction rounds would follow.
            wait_key = __reduce_min_sync(FULL, go ? 0xFFFFFFFFu : key);
        } else {
            if (!__any_sync(FULL, act)) break;
            go = act;
        }
        // One call site of the emulator for every policy.  A converged group
        // keeps running (up to FA_STEPS_PER_ROUND instructions) while its
        // lanes stay at one pc: one shuffle and one vote per instruction
        // instead of a full scheduling round.  With no lane waiting
        // (wait_key all ones, the common fully converged warp) the keys need
        // not be compared.
        uint32_t steps = 0;
        if (go) {
            while (true) {
                r.iterate();
                if (!converge || ++steps >= FA_STEPS_PER_ROUND) break;
                const uint32_t mp = (r.e.bank << 16) | r.e.pc;
                const uint32_t lp = __shfl_sync(gm, mp, lead);
                const bool cont = wait_key == 0xFFFFFFFFu ? (r.active && mp == lp)
                                                          : (r.active && mp == lp && r.key(sched) < wait_key);
                if (!__all_sync(gm, cont)) break;
            }
        }
        rounds += converge ? __shfl_sync(FULL, steps, lead) : 1u;
    }
    return rounds;
}

// Run one work unit: instances [first, first + count) of group G, one per
// thread; t is the thread's slot in a private-byte slab of BLOCK slots.
template <int BLOCK, bool SLICED, bool DPC = false, bool FE = false>
__device__ __forceinline__ void run_unit_as(const FaGroup& G, uint32_t first, uint32_t count, const uint8_t* rom_s,
                                            uint32_t* priv, uint32_t t, unsigned long long* instr_out,
                                            unsigned long long* rounds_out)
{
    Runner<BLOCK, SLICED, DPC, FE> r;
    r.f = 0;
    r.phase = 0;
    r.fcyc = 0;
    r.active = false;
    r.e.pv = (uint8_t*)(priv + t);
    r.e.G = &G;
    r.e.i = first + t;
    r.e.rom = rom_s;
    r.e.hot_lo = G.hot_lo;
    r.e.nbanks = G.nbanks;
    r.e.instr = 0;
    r.e.cyc_acc = 0;
    r.e.pc = 0;
    r.e.bank = 0;
    r.e.slices = 0;
    r.e.scanline = 0;
    const bool valid = t < count;
    uint32_t* col = G.state + r.e.i;
    if (valid) {
        r.e.load_ram(col, G.stride);
        r.e.load_hot(col, G.stride);
        if (G.k > 0) r.active = r.begin_frame();
    }
    const uint32_t rounds = run_lanes(r, G.sched);
    if (valid) {
        r.e.fold_cycles();
        // An instance that halted before the call's last frame still took
        // the later frames' set_action; the last one is what its inputs hold.
        if (G.actions && r.f + 1u < G.k && (r.e.row(R_STATUS) & FA_STATUS_HALT_MASK))
            r.e.apply_action(G.actions[(size_t)(G.k - 1u) * G.act_stride + r.e.i]);
        r.e.store_ram(col, G.stride);
        r.e.store_hot(col, G.stride);
        if (G.obs) {
            const uint32_t* w = priv + t;
            uint4* o = (uint4*)(G.obs + (size_t)r.e.i * 128u);
#pragma unroll
            for (uint32_t q = 0; q < 8u; q++)
                o[q] = make_uint4(w[(4u * q) * BLOCK], w[(4u * q + 1u) * BLOCK], w[(4u * q + 2u) * BLOCK],
                                  w[(4u * q + 3u) * BLOCK]);
        }
    }
    if (instr_out) {
        uint32_t n = valid ? r.e.instr : 0u;
        for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xFFFFFFFFu, n, d);
        if ((t & 31u) == 0 && n) atomicAdd(instr_out, (unsigned long long)n);
    }
    if (rounds_out && (t & 31u) == 0 && rounds) atomicAdd(rounds_out, 32ull * rounds);
}

// Kernels come in five builds, picked by the host from the carts of a
// launch: FA_MAPS_4K (only the reference's schemes) holds the 4K-bank core
// alone, FA_MAPS_SLICED (only E0 and 3F carts) the SLICED core alone,
// FA_MAPS_DPC (only DPC carts) the DPC core alone, FA_MAPS_FE (only FE
// carts) the FE core alone, and FA_MAPS_BOTH runs each unit on its cart's
// core (hot_lo below 0x1000: sliced; FA_MAP_DPC / FA_MAP_FE: those cores).  A build's register budget is the largest of the cores it
// holds, so the single-core builds keep their own.
template <int BLOCK, int MAPS>
__device__ __forceinline__ void run_unit(const FaGroup& G, uint32_t first, uint32_t count, const uint8_t* rom_s,
                                         uint32_t* priv, uint32_t t, unsigned long long* instr_out,
                                         unsigned long long* rounds_out)
{
    if constexpr (MAPS == FA_MAPS_4K) {
        run_unit_as<BLOCK, false>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
    } else if constexpr (MAPS == FA_MAPS_SLICED) {
        run_unit_as<BLOCK, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
    } else if constexpr (MAPS == FA_MAPS_DPC) {
        run_unit_as<BLOCK, true, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
    } else if constexpr (MAPS == FA_MAPS_FE) {
        run_unit_as<BLOCK, true, false, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
    } else {
        const uint32_t kind = fa_map_kind(G.hot_lo);
        if (kind == FA_MAP_DPC) run_unit_as<BLOCK, true, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
        else if (kind == FA_MAP_FE)
            run_unit_as<BLOCK, true, false, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
        else if (kind) run_unit_as<BLOCK, true>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
        else run_unit_as<BLOCK, false>(G, first, count, rom_s, priv, t, instr_out, rounds_out);
    }
}

}  // namespace fa
