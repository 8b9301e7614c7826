// fa_kernels.cu — launches of the batched Atari core on sm_100a.
//
// One kernel, fa_run, serves both launch forms of the library:
//   * plain:      one CTA per work unit (grid = number of units);
//   * persistent: grid sized to the SMs, each CTA pops work units from a
//                 device counter until the queue is empty.
// A work unit is up to BLOCK consecutive instances of one group (one cart's
// instance set).  Groups of different carts, instance counts, frame counts
// and scheduling policies share one launch.  When a CTA's next unit belongs
// to a different cart than the ROM it holds, it re-stages the ROM into shared
// memory with TMA bulk copies (cp.async.bulk, no multicast) on an mbarrier.
//
// Every wait is bounded; on expiry the kernel records FA_DEVERR_* in the
// launch's error word and leaves the unit untouched.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fa_run.cuh"

namespace fa {

template <int BLOCK, int MAPS>
__global__ void __launch_bounds__(BLOCK) fa_run(const __grid_constant__ FaLaunch L)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_unit;

    uint8_t* rom_s = smem;
    uint32_t* priv = (uint32_t*)(smem + L.rom_bytes_max);
    uint32_t phase = 0;
    int staged = -1;

    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();

    for (uint32_t round = 0;; round++) {
        if (threadIdx.x == 0) {
            uint32_t u;
            if (L.queue) u = atomicAdd(L.queue, 1u);
            else u = round == 0 ? blockIdx.x : 0xFFFFFFFFu;
            s_unit = u;
        }
        __syncthreads();
        const uint32_t u = s_unit;
        if (u >= L.nunits) break;
        int g = 0;
        while (g + 1 < (int)L.ngroups && u >= L.g[g + 1].unit_begin) g++;
        const FaGroup& G = L.g[g];
        if (G.rom != (staged < 0 ? nullptr : L.g[staged].rom)) {
            if (!stage_rom(rom_s, G.rom, G.nbanks * 4096u, &bar, phase, L.wait_ns)) {
                if (threadIdx.x == 0) atomicOr(L.err, FA_DEVERR_TMA_TIMEOUT);
                break;
            }
            staged = g;
        }
        const uint32_t first = (u - G.unit_begin) * BLOCK;
        const uint32_t count = G.n - first < BLOCK ? G.n - first : BLOCK;
        run_unit<BLOCK, MAPS>(G, first, count, rom_s, priv, threadIdx.x, L.instr, L.rounds);
        __syncthreads();
    }
}

// Warp-granular form: every warp pops its own 32-instance work units, and
// every CTA holds all of the launch's ROM images at once (the "ROM library",
// staged once with TMA bulk copies), so units of any cart run in any warp
// and a CTA can be as large as shared memory allows.
template <int WARPS, int MAPS>
__global__ void __launch_bounds__(WARPS * 32) fa_run_warps(const __grid_constant__ FaLaunch L)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    const uint32_t FULL = 0xFFFFFFFFu;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t* priv = (uint32_t*)(smem + L.romlib_bytes) + warp * (FA_SMEM_WORDS * 32u);

    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar, L.romlib_bytes);
        for (uint32_t g = 0; g < L.ngroups; g++) {
            if (!L.g[g].rom_owner) continue;
            for (uint32_t off = 0; off < L.g[g].nbanks * 4096u; off += 4096u)
                bulk_g2s(smem + L.g[g].rom_off + off, L.g[g].rom + off, 4096u, &bar);
        }
    }
    if (!mbar_wait_bounded(&bar, 0, L.wait_ns)) {
        if (threadIdx.x == 0) atomicOr(L.err, FA_DEVERR_TMA_TIMEOUT);
        mbar_drain(&bar, 0);
        return;
    }
    for (uint32_t round = 0;; round++) {
        // First wave: unit warp*grid + cta, so consecutive (heaviest-first)
        // units land on different SMs; after that the device queue.
        uint32_t u = 0;
        if (lane == 0) {
            if (L.queue) {
                const uint32_t slot = warp * gridDim.x + blockIdx.x;
                u = round != 0 ? gridDim.x * WARPS + atomicAdd(L.queue, 1u) : L.first_wave ? L.first_wave[slot] : slot;
            }
            else u = round == 0 ? blockIdx.x * WARPS + warp : 0xFFFFFFFFu;
        }
        u = __shfl_sync(FULL, u, 0);
        if (u >= L.nunits) break;
        uint32_t g = 0;
        while (g + 1 < L.ngroups && u >= L.g[g + 1].unit_begin) g++;
        const FaGroup& G = L.g[g];
        const uint32_t first = (u - G.unit_begin) * 32u;
        const uint32_t count = G.n - first < 32u ? G.n - first : 32u;
        const uint64_t t0 = L.trace ? globaltimer_ns() : 0ull;
        run_unit<32, MAPS>(G, first, count, smem + G.rom_off, priv, lane, L.instr, L.rounds);
        if (L.trace && lane == 0 && u < L.trace_cap) {
            uint32_t smid;
            asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
            unsigned long long* rec = L.trace + 3ull * u;
            rec[0] = t0;
            rec[1] = globaltimer_ns();
            rec[2] = ((unsigned long long)smid << 32) | (warp << 16) | G.tag;
        }
    }
}

// Every instance column of `state` becomes a copy of `col` (FA_ROWS words).
__global__ void fa_broadcast(uint32_t* state, uint32_t stride, uint32_t n, const uint32_t* col)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (uint32_t w = 0; w < FA_ROWS; w++) state[(size_t)w * stride + i] = col[w];
}

}  // namespace fa

// ------------------------------------------------------------------ host launchers
#include <algorithm>
#include <map>
#include <numeric>
#include <mutex>
#include <vector>

namespace {
std::mutex g_cfg_mu;
std::map<std::pair<int, std::pair<int, size_t>>, int> g_per_sm;   // (device, block, smem) -> CTAs/SM

// The dynamic shared-memory limit is raised once per (device, BLOCK) to the
// largest any cart needs (32 KiB of ROM plus the private bytes), so launches
// of smaller carts never lower it under a larger one.
template <int BLOCK, int SL = 0>
int per_sm_for(size_t smem)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    auto key = std::make_pair(dev, std::make_pair(BLOCK * 4 + SL, smem));
    auto it = g_per_sm.find(key);
    if (it != g_per_sm.end()) return it->second;
    const auto max_key = std::make_pair(dev, std::make_pair(BLOCK * 4 + SL, (size_t)0));
    if (g_per_sm.find(max_key) == g_per_sm.end()) {
        const int max_smem = 32768 + FA_SMEM_WORDS * BLOCK * 4;
        if (cudaFuncSetAttribute(fa::fa_run<BLOCK, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem) !=
            cudaSuccess)
            return -1;
        g_per_sm[max_key] = 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fa::fa_run<BLOCK, SL>, BLOCK, smem) != cudaSuccess)
        return -1;
    g_per_sm[key] = per_sm;
    return per_sm;
}
}  // namespace

template <int BLOCK, int SL>
static cudaError_t launch_block(const FaLaunch& L, bool persistent, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)L.rom_bytes_max + (size_t)FA_SMEM_WORDS * BLOCK * 4u;
    const int per_sm = per_sm_for<BLOCK, SL>(smem);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (sms <= 0) return cudaSuccess;                                  // prepare only
    uint32_t grid = L.nunits;
    if (persistent) {
        uint32_t cap = (uint32_t)(per_sm * sms);
        grid = L.nunits < cap ? L.nunits : cap;
    }
    if (grid == 0) return cudaSuccess;
    fa::fa_run<BLOCK, SL><<<grid, BLOCK, smem, s>>>(L);
    return cudaGetLastError();
}

template <int BLOCK>
static cudaError_t launch_block_m(int maps, const FaLaunch& L, bool persistent, int sms, cudaStream_t s)
{
    return maps == FA_MAPS_4K   ? launch_block<BLOCK, FA_MAPS_4K>(L, persistent, sms, s)
         : maps == FA_MAPS_BOTH ? launch_block<BLOCK, FA_MAPS_BOTH>(L, persistent, sms, s)
         : maps == FA_MAPS_DPC  ? launch_block<BLOCK, FA_MAPS_DPC>(L, persistent, sms, s)
         : maps == FA_MAPS_FE   ? launch_block<BLOCK, FA_MAPS_FE>(L, persistent, sms, s)
                                : launch_block<BLOCK, FA_MAPS_SLICED>(L, persistent, sms, s);
}

namespace {
std::map<std::pair<int, std::pair<int, size_t>>, int> g_warps_per_sm;   // (device, warps, smem) -> CTAs/SM

template <int WARPS, int SL>
int warps_per_sm_for(size_t smem)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    auto key = std::make_pair(dev, std::make_pair(WARPS * 4 + SL, smem));
    auto it = g_warps_per_sm.find(key);
    if (it != g_warps_per_sm.end()) return it->second;
    const auto max_key = std::make_pair(dev, std::make_pair(WARPS * 4 + SL, (size_t)0));
    if (g_warps_per_sm.find(max_key) == g_warps_per_sm.end()) {
        if (cudaFuncSetAttribute(fa::fa_run_warps<WARPS, SL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 FA_SMEM_PER_CTA_MAX) != cudaSuccess)
            return -1;
        g_warps_per_sm[max_key] = 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fa::fa_run_warps<WARPS, SL>, WARPS * 32, smem) !=
        cudaSuccess)
        return -1;
    g_warps_per_sm[key] = per_sm;
    return per_sm;
}

template <int WARPS, int SL>
cudaError_t launch_warps(const FaLaunch& L, bool persistent, int sms, cudaStream_t s)
{
    const size_t smem = (size_t)L.romlib_bytes + (size_t)WARPS * FA_SMEM_WORDS * 32u * 4u;
    const int per_sm = warps_per_sm_for<WARPS, SL>(smem);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    if (sms <= 0) return cudaSuccess;                                  // prepare only
    uint32_t grid = (L.nunits + WARPS - 1) / WARPS;
    if (persistent) {
        // One CTA per resident slot on every SM (fewer only if there are fewer
        // units than slots), so no SM idles while units remain.
        const uint32_t cap = (uint32_t)(per_sm * sms);
        grid = L.nunits < cap ? L.nunits : cap;
    }
    if (grid == 0) return cudaSuccess;
    FaLaunch Lw = L;
    if (!persistent || per_sm != 1) Lw.first_wave = nullptr;            // a plan assumes one CTA per SM
    fa::fa_run_warps<WARPS, SL><<<grid, WARPS * 32, smem, s>>>(Lw);
    return cudaGetLastError();
}

template <int WARPS, int SL>
void warps_shape(const FaLaunch& L, bool persistent, int sms, uint32_t* grid, int* per_sm)
{
    const size_t smem = (size_t)L.romlib_bytes + (size_t)WARPS * FA_SMEM_WORDS * 32u * 4u;
    *per_sm = warps_per_sm_for<WARPS, SL>(smem);
    uint32_t g = (L.nunits + WARPS - 1) / WARPS;
    if (persistent) {
        const uint32_t cap = (uint32_t)(*per_sm * sms);
        g = L.nunits < cap ? L.nunits : cap;
    }
    *grid = g;
}

template <int SL>
cudaError_t launch_warps_n(int warps, const FaLaunch& L, bool persistent, int sms, cudaStream_t s)
{
    switch (warps) {
    case 2: return launch_warps<2, SL>(L, persistent, sms, s);
    case 4: return launch_warps<4, SL>(L, persistent, sms, s);
    case 8: return launch_warps<8, SL>(L, persistent, sms, s);
    case 16: return launch_warps<16, SL>(L, persistent, sms, s);
    case 24: return launch_warps<24, SL>(L, persistent, sms, s);
    case 28: return launch_warps<28, SL>(L, persistent, sms, s);
    case 32: return launch_warps<32, SL>(L, persistent, sms, s);
    default: return cudaErrorInvalidValue;
    }
}
}  // namespace

// Lay out the ROM library (one copy per distinct ROM buffer) and the work
// units; returns the library size, or 0 if it cannot fit beside one warp slab.
static uint32_t plan_romlib(FaLaunch& L)
{
    uint32_t bytes = 0;
    for (uint32_t g = 0; g < L.ngroups; g++) {
        L.g[g].rom_owner = 1;
        for (uint32_t h = 0; h < g; h++)
            if (L.g[h].rom == L.g[g].rom) { L.g[g].rom_off = L.g[h].rom_off; L.g[g].rom_owner = 0; break; }
        if (L.g[g].rom_owner) { L.g[g].rom_off = bytes; bytes += L.g[g].nbanks * 4096u; }
    }
    return bytes;
}

static void plan_units(FaLaunch& L, uint32_t unit)
{
    uint32_t units = 0;
    for (uint32_t g = 0; g < L.ngroups; g++) {
        L.g[g].unit_begin = units;
        units += (L.g[g].n + unit - 1) / unit;
    }
    L.nunits = units;
}

// The warp-granular layout of a launch: the ROM library, 32-instance work
// units and the warps per CTA.  False when the library leaves no room for
// block / 32 warp slabs (the launch is CTA-granular).
static bool warp_layout(FaLaunch& L, int block, bool persistent, int* warps)
{
    const uint32_t lib = plan_romlib(L);
    L.romlib_bytes = lib;
    const uint32_t slab = FA_SMEM_WORDS * 32u * 4u;
    const int fit = (int)((FA_SMEM_PER_CTA_MAX - (int)lib) / (int)slab);
    if (fit < block / 32) return false;
    int w = block / 32;
    if (persistent) {
        // As many warps per CTA as shared memory allows (one CTA per SM), or
        // fewer when a cap is set (the register budget per thread grows as
        // 65536 / (32 x warps)).  A launch of sliced carts alone defaults to
        // 24: at 32 warps its core is held to 64 registers and spills in the
        // interpreter loop (three E0/3F carts: 2.31 against 2.13 M frames/s).
        const int m = fa_maps_of(L.g, L.ngroups);
        const int cap = L.cta_warps ? (int)L.cta_warps : (m == FA_MAPS_4K || m == FA_MAPS_BOTH) ? 32 : 24;
        static const int sizes[] = { 32, 28, 24, 16, 8, 4, 2 };
        for (int x : sizes)
            if (x <= fit && x <= cap) { w = x; break; }
    }
    plan_units(L, 32u);
    *warps = w;
    return true;
}

cudaError_t fa_launch_run(const FaLaunch& L_in, int block, bool persistent, int sms, cudaStream_t s)
{
    FaLaunch L = L_in;
    L.wait_ns = fa_wait_limit_ns();
    const int maps = fa_maps_of(L.g, L.ngroups);                       // which cores the carts need
    int warps = 0;
    if (warp_layout(L, block, persistent, &warps)) {
        return maps == FA_MAPS_4K   ? launch_warps_n<FA_MAPS_4K>(warps, L, persistent, sms, s)
             : maps == FA_MAPS_BOTH ? launch_warps_n<FA_MAPS_BOTH>(warps, L, persistent, sms, s)
             : maps == FA_MAPS_DPC  ? launch_warps_n<FA_MAPS_DPC>(warps, L, persistent, sms, s)
             : maps == FA_MAPS_FE   ? launch_warps_n<FA_MAPS_FE>(warps, L, persistent, sms, s)
                                    : launch_warps_n<FA_MAPS_SLICED>(warps, L, persistent, sms, s);
    }
    // ROM library too large for shared memory: CTA-granular units that
    // re-stage one cart's ROM at a time.
    plan_units(L, (uint32_t)block);
    switch (block) {
    case 64: return launch_block_m<64>(maps, L, persistent, sms, s);
    case 128: return launch_block_m<128>(maps, L, persistent, sms, s);
    case 256: return launch_block_m<256>(maps, L, persistent, sms, s);
    case 512: return launch_block_m<512>(maps, L, persistent, sms, s);
    default: return cudaErrorInvalidValue;
    }
}

bool fa_launch_warp_shape(const FaLaunch& L_in, int block, bool persistent, int sms, uint32_t* grid, uint32_t* warps,
                          int* per_sm)
{
    FaLaunch L = L_in;
    const int maps = fa_maps_of(L.g, L.ngroups);
    int w = 0;
    if (!warp_layout(L, block, persistent, &w)) return false;
    *warps = (uint32_t)w;
#define FA_SHAPE(WW)                                                                                        \
    case WW:                                                                                                \
        if (maps == FA_MAPS_4K) warps_shape<WW, FA_MAPS_4K>(L, persistent, sms, grid, per_sm);              \
        else if (maps == FA_MAPS_BOTH) warps_shape<WW, FA_MAPS_BOTH>(L, persistent, sms, grid, per_sm);     \
        else if (maps == FA_MAPS_DPC) warps_shape<WW, FA_MAPS_DPC>(L, persistent, sms, grid, per_sm);       \
        else if (maps == FA_MAPS_FE) warps_shape<WW, FA_MAPS_FE>(L, persistent, sms, grid, per_sm);         \
        else warps_shape<WW, FA_MAPS_SLICED>(L, persistent, sms, grid, per_sm);                            \
        return true;
    switch (w) {
    FA_SHAPE(2) FA_SHAPE(4) FA_SHAPE(8) FA_SHAPE(16) FA_SHAPE(24) FA_SHAPE(28) FA_SHAPE(32)
    default: return false;
    }
#undef FA_SHAPE
}

cudaError_t fa_launch_prepare(const FaLaunch& L, int block, bool persistent)
{
    return fa_launch_run(L, block, persistent, 0, nullptr);
}

int fa_launch_occupancy(int block, uint32_t rom_bytes_max)
{
    const size_t base = (size_t)rom_bytes_max + (size_t)FA_SMEM_WORDS * block * 4u;
    switch (block) {
    case 64: return per_sm_for<64>(base);
    case 128: return per_sm_for<128>(base);
    case 256: return per_sm_for<256>(base);
    case 512: return per_sm_for<512>(base);
    default: return -1;
    }
}

cudaError_t fa_launch_broadcast(uint32_t* state, uint32_t stride, uint32_t n, const uint32_t* col, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    uint32_t grid = (n + 255u) / 256u;
    if (grid > 4096u) grid = 4096u;
    fa::fa_broadcast<<<grid, 256, 0, s>>>(state, stride, n, col);
    return cudaGetLastError();
}
