// fa_serve_kernel.cu — the serving kernel (fa_serve) and its launcher.
//
// One warp per unit (up to 32 consecutive instances of one request, inside
// one state block of the server's arena), units packed densely into CTAs of
// WARPS warps in the order the host lists them (longest requests first), no
// queue and no persistence, so the CTAs of several launches in flight
// interleave on the SMs as the hardware block scheduler frees them: requests
// dispatched while others run start on whichever SM slots drain first.  Every
// unit of a launch belongs to one cart, whose ROM the CTA stages into shared
// memory with TMA bulk copies; the launch's shared memory is sized to that
// cart's ROM alone.
//
// Completion is per request, not per launch: the last warp of a request (a
// device counter per request) fences at system scope and raises the
// request's flag in host-mapped memory, after its observations — written
// straight into host-mapped memory — are visible.  The host then lets the
// session's next request run, possibly in another launch while this one is
// still running.  That next kernel must read the state rows this one wrote,
// so this file is compiled with global loads cached in L2 only
// (-Xptxas -dlcm=cg): L2 is the point of coherence, and no SM can serve a
// stale copy from its L1.
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>

#include "fa_run.cuh"

namespace fa {

constexpr uint32_t FA_REQ_FAILED = 0x80000000u;   // bit of a request's unit counter

template <int WARPS, int MAPS>
__global__ void __launch_bounds__(WARPS * 32, 32 / WARPS) fa_serve(const __grid_constant__ FaServeLaunch L)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ FaGroup sg[WARPS];
    __shared__ uint32_t s_count[WARPS], s_req[WARPS];

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t rom_bytes = L.nbanks * 4096u;
    uint32_t* priv = (uint32_t*)(smem + rom_bytes) + warp * (FA_SMEM_WORDS * 32u);
    const uint32_t u = blockIdx.x * WARPS + warp;
    const bool have = u < L.nunits;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    if (have && lane == 0) {
        const FaServeUnit U = L.unit[u];
        const FaServeReq R = L.req[U.req];
        FaGroup g;
        memset(&g, 0, sizeof(g));
        g.rom = L.rom;
        g.state = U.state;
        g.stride = FA_SERVE_BLOCK_COLS;
        g.nbanks = L.nbanks;
        g.hot_lo = L.hot_lo;
        g.sched = R.sched;
        g.act_stride = R.n;
        const uint32_t count = R.n - U.first < 32u ? R.n - U.first : 32u;
        g.n = count;
        if (L.per_frame) {
            g.actions = R.actions + (size_t)L.frame * R.n + U.first;
            g.k = L.frame < R.k ? 1u : 0u;
            g.obs = (L.frame + 1u == R.k && R.obs) ? R.obs + (size_t)U.first * 128u : nullptr;
        } else {
            g.actions = R.actions + U.first;
            g.k = R.k;
            g.obs = R.obs ? R.obs + (size_t)U.first * 128u : nullptr;
        }
        sg[warp] = g;
        s_count[warp] = count;
        s_req[warp] = U.req;
    }
    __syncthreads();
    uint32_t phase = 0;
    const bool staged = stage_rom(smem, L.rom, rom_bytes, &bar, phase, L.wait_ns);
    if (!have) return;
    if (staged) run_unit<32, MAPS>(sg[warp], 0, s_count[warp], smem, priv, lane, L.instr, L.rounds);
    else if (lane == 0) atomicOr(L.err, FA_DEVERR_TMA_TIMEOUT);
    if (L.done) {
        // Every lane's state and observation stores precede the warp barrier;
        // lane 0's fence after it is cumulative over them.
        __syncwarp();
        if (lane == 0) {
            const uint32_t r = s_req[warp];
            if (!staged) atomicOr(L.remaining + r, FA_REQ_FAILED);
            __threadfence_system();
            const uint32_t old = atomicSub(L.remaining + r, 1u);
            if ((old & ~FA_REQ_FAILED) == 1u) {
                __threadfence_system();
                *(volatile uint32_t*)(L.done + r) = (old & FA_REQ_FAILED) ? 2u : 1u;
            }
        }
    }
}

}  // namespace fa

namespace {
std::mutex g_serve_mu;
// (device, warps) pairs whose dynamic shared-memory limit was raised to the
// largest serving launch (32 KiB of ROM plus the RAM slab).
std::map<std::pair<int, int>, bool> g_serve_cfg;

template <int WARPS, int SL>
cudaError_t launch_serve(const FaServeLaunch& L, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_serve_mu);
        auto key = std::make_pair(dev, WARPS * 4 + SL);
        if (g_serve_cfg.find(key) == g_serve_cfg.end()) {
            e = cudaFuncSetAttribute(fa::fa_serve<WARPS, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     32768 + WARPS * FA_SMEM_WORDS * 32 * 4);
            if (e != cudaSuccess) return e;
            g_serve_cfg[key] = true;
        }
    }
    if (L.nunits == 0) return cudaSuccess;
    const size_t smem = (size_t)L.nbanks * 4096u + (size_t)WARPS * FA_SMEM_WORDS * 32u * 4u;
    FaServeLaunch Lw = L;
    Lw.wait_ns = fa_wait_limit_ns();
    fa::fa_serve<WARPS, SL><<<(L.nunits + WARPS - 1) / WARPS, WARPS * 32, smem, s>>>(Lw);
    return cudaGetLastError();
}
}  // namespace

cudaError_t fa_launch_serve(const FaServeLaunch& L, int block, cudaStream_t s)
{
    if (L.nbanks < 1 || L.nbanks > 8) return cudaErrorInvalidValue;
    const uint32_t kind = fa_map_kind(L.hot_lo);                       // one cart per launch
    switch (block) {
    case 128:
        return kind == FA_MAP_DPC ? launch_serve<4, FA_MAPS_DPC>(L, s)
             : kind == FA_MAP_FE  ? launch_serve<4, FA_MAPS_FE>(L, s)
             : kind               ? launch_serve<4, FA_MAPS_SLICED>(L, s) : launch_serve<4, FA_MAPS_4K>(L, s);
    case 256:
        return kind == FA_MAP_DPC ? launch_serve<8, FA_MAPS_DPC>(L, s)
             : kind == FA_MAP_FE  ? launch_serve<8, FA_MAPS_FE>(L, s)
             : kind               ? launch_serve<8, FA_MAPS_SLICED>(L, s) : launch_serve<8, FA_MAPS_4K>(L, s);
    case 512:
        return kind == FA_MAP_DPC ? launch_serve<16, FA_MAPS_DPC>(L, s)
             : kind == FA_MAP_FE  ? launch_serve<16, FA_MAPS_FE>(L, s)
             : kind               ? launch_serve<16, FA_MAPS_SLICED>(L, s) : launch_serve<16, FA_MAPS_4K>(L, s);
    default: return cudaErrorInvalidValue;
    }
}
