// fa_render.cu — the reference's rendering console on sm_100a.
//
// The rendering console (src/atari.rs:107-306 with the pixel-accurate Tia of
// src/tia.rs) differs from the headless one in time, not in instructions: its
// bus ticks the TIA three times and the PIA once on every CPU cycle, a write
// lands on the third TIA clock of its cycle, and every TIA clock inside the
// visible window renders a pixel of a 160 x 192 framebuffer of palette
// indices.  The 6502 here is the same core as the headless kernels
// (Emu<32, true, SLICED>): each of its bus accesses knows its cycle within the
// instruction, and before an access reaches a TIA or PIA register the TIA
// and PIA are ticked up to that cycle, so register writes land at the beam
// position the reference gives them.  Cycles of instructions that touch
// only ROM and RAM are owed and given at the next such access (or at the end
// of the frame), and pixels are drawn a span at a time, when something that
// affects them is about to change: the same framebuffer, fewer calls.
//
// One warp per unit of 32 consoles, WARPS units per CTA; the cart's ROM and
// one private-byte slab per warp (RAM + graphics registers, FA_RPRIV_BYTES
// per console, interleaved by lane) in shared memory; state rows in HBM
// (the headless layout plus the rendering rows); one framebuffer per console
// in HBM, persistent across launches (pixels the program does not redraw keep
// their value, as in the reference).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/fast_atari.h"
#include "fa_internal.h"
#include "fa_render.cuh"

struct FaRenderLaunch {
    const uint8_t* rom;
    uint32_t nbanks, hot_lo;
    uint32_t* state;             // FA_RROWS rows of `stride` words
    uint32_t stride, n;
    const uint8_t* actions;      // k * n frame-major, or null (no set_action: the reset frame)
    uint32_t k, sched;
    uint8_t* fb;                 // n * FA_FB_BYTES
    uint8_t* obs;                // n * 128, or null
    uint32_t* err;
    unsigned long long* instr;
    unsigned long long* rounds;
    uint64_t wait_ns;            // bound of the ROM staging wait (set by launch_render)
};

namespace fa {

// 128 registers: the pixel code and the bus run with almost no spills, and
// 16 warps are resident per SM (one 512-thread CTA at 16 warps, the default,
// or two 256-thread CTAs at 8).  Held to 80 registers for 24 resident warps,
// the spills cost more than the extra warps gain: 2.15 against 3.92 M
// frames/s on the render cart (113,664 consoles, one B200).  Uncapped,
// ptxas takes 148, which a 16-warp CTA cannot launch with.
template <int WARPS, bool SLICED>
__global__ void __maxnreg__(128) fa_render_run(const __grid_constant__ FaRenderLaunch L)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ FaGroup sg;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t rom_bytes = L.nbanks * 4096u;
    uint32_t* slab = (uint32_t*)(smem + rom_bytes) + warp * (FA_RSLAB_WORDS * 32u);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        FaGroup g;
        memset(&g, 0, sizeof(g));
        g.rom = L.rom;
        g.state = L.state;
        g.stride = L.stride;
        g.n = L.n;
        g.actions = L.actions;
        g.act_stride = L.n;
        g.nbanks = L.nbanks;
        g.hot_lo = L.hot_lo;
        g.k = L.k;
        g.sched = L.sched;
        g.obs = L.obs;
        sg = g;
    }
    __syncthreads();
    uint32_t phase = 0;
    if (!stage_rom(smem, L.rom, rom_bytes, &bar, phase, L.wait_ns)) {
        if (threadIdx.x == 0) atomicOr(L.err, FA_DEVERR_TMA_TIMEOUT);
        return;
    }
    const uint32_t first = (blockIdx.x * WARPS + warp) * 32u;
    if (first >= L.n) return;
    const uint32_t i = first + lane;
    const bool valid = i < L.n;

    RRunner<SLICED> r;
    r.f = 0;
    r.phase = 0;
    r.fcyc = 0;
    r.active = false;
    Emu<32, true, SLICED>& e = r.e;
    e.pv = (uint8_t*)(slab + lane);
    e.G = &sg;
    e.i = i;
    e.rom = smem;
    e.hot_lo = L.hot_lo;
    e.nbanks = L.nbanks;
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
    e.fbp = L.fb + (size_t)(valid ? i : 0u) * FA_FB_BYTES;
    uint32_t* col = L.state + i;
    const uint32_t S = L.stride;
    if (valid) {
        uint32_t* w = slab + lane;
#pragma unroll 4
        for (uint32_t k = 0; k < FA_PRIV_WORDS; k++) w[k * 32u] = col[(size_t)k * S];
        for (uint32_t k = FA_PRIV_WORDS; k < FA_RPRIV_WORDS; k++)
            w[k * 32u] = col[(size_t)(FA_RROW_EXTRA + (k - FA_PRIV_WORDS)) * S];
        e.load_hot(col, S);
        e.vtop = col[(size_t)RR_VTOP * S];
        e.rx = e.clock;
        e.fb_resume();
        const uint32_t fl = col[(size_t)RR_FLAGS * S];
        e.tw |= ((fl & 1u) ? TW_HMOVE : 0u) | ((fl & 2u) ? TW_LATCH : 0u) | ((fl & 4u) ? TW_L4 : 0u) |
                ((fl & 8u) ? TW_L5 : 0u);
        if (L.k > 0) r.active = r.begin_frame();
    }
    const uint32_t rounds = run_lanes(r, L.sched);
    if (valid) {
        e.fb_observe();
        e.fold_cycles();
        // A console that halted before the call's last frame took the later
        // frames' set_action too; the last one is what its inputs hold.
        if (L.actions && r.f + 1u < L.k && (e.row(R_STATUS) & FA_STATUS_HALT_MASK))
            e.apply_action(L.actions[(size_t)(L.k - 1u) * L.n + i]);
        uint32_t* w = slab + lane;
#pragma unroll 4
        for (uint32_t k = 0; k < FA_PRIV_WORDS; k++) col[(size_t)k * S] = w[k * 32u];
        for (uint32_t k = FA_PRIV_WORDS; k < FA_RPRIV_WORDS; k++)
            col[(size_t)(FA_RROW_EXTRA + (k - FA_PRIV_WORDS)) * S] = w[k * 32u];
        e.store_hot(col, S);
        col[(size_t)RR_VTOP * S] = e.vtop;
        col[(size_t)RR_FLAGS * S] = ((e.tw & TW_HMOVE) ? 1u : 0u) | ((e.tw & TW_LATCH) ? 2u : 0u) |
                                    ((e.tw & TW_L4) ? 4u : 0u) | ((e.tw & TW_L5) ? 8u : 0u);
        if (L.obs) {
            uint4* o = (uint4*)(L.obs + (size_t)i * 128u);
#pragma unroll
            for (uint32_t q = 0; q < 8u; q++)
                o[q] = make_uint4(w[(4u * q) * 32u], w[(4u * q + 1u) * 32u], w[(4u * q + 2u) * 32u],
                                  w[(4u * q + 3u) * 32u]);
        }
    }
    if (L.instr) {
        uint32_t c = valid ? e.instr : 0u;
        for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, d);
        if (lane == 0 && c) atomicAdd(L.instr, (unsigned long long)c);
    }
    if (L.rounds && lane == 0 && rounds) atomicAdd(L.rounds, 32ull * rounds);
}

}  // namespace fa

// ------------------------------------------------------------------ RGBA
// Atari::render (src/atari.rs:356-369): every palette index of a framebuffer
// becomes R, G, B, 255 through ntsc_palette (src/atari.rs:624-645), whose 128
// entries come in equal pairs indexed by (index >> 1) & 0x7F; so the colour
// depends on index >> 2 only, and the 64 distinct colours are kept here as
// packed little-endian RGBA words (R in the low byte, alpha 255).
#define FA_NTSC_RGBA \
    0xFF000000u, 0xFF004444u, 0xFF002870u, 0xFF001884u, 0xFF000088u, 0xFF5C0078u, 0xFF780048u, 0xFF840014u, \
    0xFF880000u, 0xFF780000u, 0xFF600000u, 0xFF2C1400u, 0xFF002800u, 0xFF002C00u, 0xFF002C00u, 0xFF001800u, \
    0xFF282828u, 0xFF106464u, 0xFF104890u, 0xFF0038A8u, 0xFF0014B8u, 0xFF7400A0u, 0xFFA40064u, 0xFFB00030u, \
    0xFFB80000u, 0xFFA81800u, 0xFF802C00u, 0xFF4C3C00u, 0xFF004400u, 0xFF004C00u, 0xFF004400u, 0xFF003800u, \
    0xFF545454u, 0xFF248484u, 0xFF2464B0u, 0xFF1050C8u, 0xFF1438DCu, 0xFF9014C4u, 0xFFC80084u, 0xFFD40050u, \
    0xFFDC0018u, 0xFFD43000u, 0xFFA44C00u, 0xFF6C5C00u, 0xFF006400u, 0xFF006C00u, 0xFF106400u, 0xFF005400u, \
    0xFF787878u, 0xFF38A8A8u, 0xFF3888CCu, 0xFF2470E8u, 0xFF285CFCu, 0xFFAC30E8u, 0xFFE800A8u, 0xFFF40070u, \
    0xFFFC0038u, 0xFFF84C0Cu, 0xFFC46C00u, 0xFF8C8000u, 0xFF008800u, 0xFF009000u, 0xFF288800u, 0xFF007400u
static const uint32_t kNtscRgba[64] = { FA_NTSC_RGBA };

namespace fa {

static __constant__ uint32_t c_ntsc_rgba[64] = { FA_NTSC_RGBA };

// Four pixels per thread: one 32-bit load of palette indices, one 16-byte
// store of RGBA, the 64 colours in shared memory (two lanes per bank at most).
__global__ void fa_fb_rgba(const uint32_t* __restrict__ fb4, uint4* __restrict__ rgba, size_t words)
{
    __shared__ uint32_t pal[64];
    if (threadIdx.x < 64) pal[threadIdx.x] = c_ntsc_rgba[threadIdx.x];
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t w = fb4[i];
        rgba[i] = make_uint4(pal[(w >> 2) & 63u], pal[(w >> 10) & 63u], pal[(w >> 18) & 63u], pal[(w >> 26) & 63u]);
    }
}

}  // namespace fa

// ------------------------------------------------------------------ host side
// One host thread's share of a device-to-host copy into pageable memory:
// two pinned chunks and a stream, so that the GPU fills one chunk while the
// thread copies the other into the caller's buffer.
struct FaStager {
    uint8_t* buf[2] = {nullptr, nullptr};
    cudaStream_t stream = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
};

struct fa_render {
    int device = 0;
    size_t n = 0;
    uint32_t stride = 0;
    int scheme = 0;
    uint32_t nbanks = 1, hot_lo = 0x2000;
    std::vector<uint8_t> image;
    uint8_t* d_rom = nullptr;
    uint32_t* d_state = nullptr;
    uint8_t* d_fb = nullptr;
    uint8_t* d_actions = nullptr;
    size_t actions_cap = 0;
    uint8_t* d_obs = nullptr;
    uint32_t* d_err = nullptr;
    unsigned long long* d_ctr = nullptr;
    cudaStream_t stream = nullptr;
    int warps = 16;
    int sched = FA_SCHED_PC;
    bool reset_done = false;
    unsigned long long last_instr = 0, last_slots = 0;
    std::vector<FaStager> stagers;   // made on the first large copy out
    uint8_t* d_rgba = nullptr;         // RGBA of a chunk of consoles for fa_render_get_rgba (made on first use)
};

namespace {
std::mutex g_rmu;
std::map<std::pair<int, int>, bool> g_rcfg;   // (device, warps) whose smem limit was raised

template <int WARPS, bool SLICED>
cudaError_t launch_render(const FaRenderLaunch& L, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const size_t smem = (size_t)L.nbanks * 4096u + (size_t)WARPS * FA_RSLAB_WORDS * 32u * 4u;
    {
        std::lock_guard<std::mutex> lk(g_rmu);
        auto key = std::make_pair(dev, WARPS * 2 + (SLICED ? 1 : 0));
        if (g_rcfg.find(key) == g_rcfg.end()) {
            e = cudaFuncSetAttribute(fa::fa_render_run<WARPS, SLICED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     32768 + WARPS * FA_RSLAB_WORDS * 32 * 4);
            if (e != cudaSuccess) return e;
            g_rcfg[key] = true;
        }
    }
    const uint32_t units = (L.n + 31u) / 32u;
    const uint32_t grid = (units + WARPS - 1u) / WARPS;
    if (grid == 0) return cudaSuccess;
    FaRenderLaunch Lw = L;
    Lw.wait_ns = fa_wait_limit_ns();
    fa::fa_render_run<WARPS, SLICED><<<grid, WARPS * 32, smem, s>>>(Lw);
    return cudaGetLastError();
}

cudaError_t launch_render_n(int warps, const FaRenderLaunch& L, cudaStream_t s)
{
    const bool sliced = fa_map_kind(L.hot_lo) != 0;                    // E0 / 3F carts
    switch (warps) {
    case 4: return sliced ? launch_render<4, true>(L, s) : launch_render<4, false>(L, s);
    case 8: return sliced ? launch_render<8, true>(L, s) : launch_render<8, false>(L, s);
    case 16: return sliced ? launch_render<16, true>(L, s) : launch_render<16, false>(L, s);
    default: return cudaErrorInvalidValue;
    }
}

void free_render(fa_render* r)
{
    if (!r) return;
    cudaSetDevice(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    cudaFree(r->d_rom);
    cudaFree(r->d_state);
    cudaFree(r->d_fb);
    cudaFree(r->d_actions);
    cudaFree(r->d_obs);
    cudaFree(r->d_err);
    cudaFree(r->d_ctr);
    cudaFree(r->d_rgba);
    for (FaStager& g : r->stagers) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        for (int b = 0; b < 2; b++) {
            if (g.buf[b]) cudaFreeHost(g.buf[b]);
            if (g.done[b]) cudaEventDestroy(g.done[b]);
        }
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
}

constexpr size_t kStageChunk = 8u << 20;   // bytes per pinned chunk
constexpr unsigned kStageThreads = 8;      // host threads of a staged copy (at most)

// bytes from device memory to pageable host memory, after the work already
// finished on the device.  A plain cudaMemcpy into pageable memory goes
// through the driver's own bounce buffer at a few GB/s; here up to
// kStageThreads host threads each move a contiguous share through their own
// two pinned chunks, so the PCIe transfer and the host-side copies overlap.
int copy_d2h(fa_render* r, uint8_t* dst, const uint8_t* src, size_t bytes)
{
    if (bytes < 2 * kStageChunk) {
        FA_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return FA_OK;
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned T = (unsigned)std::min<size_t>({(size_t)kStageThreads, (size_t)hw, bytes / kStageChunk});
    while (r->stagers.size() < T) {
        FaStager g;
        cudaError_t e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
        for (int b = 0; b < 2 && e == cudaSuccess; b++) {
            e = cudaHostAlloc((void**)&g.buf[b], kStageChunk, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.done[b], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {                    // keep only complete stagers
            for (int b = 0; b < 2; b++) {
                if (g.buf[b]) cudaFreeHost(g.buf[b]);
                if (g.done[b]) cudaEventDestroy(g.done[b]);
            }
            if (g.stream) cudaStreamDestroy(g.stream);
            return fa_fail(FA_ERR_CUDA, "pinned staging: %s", cudaGetErrorString(e));
        }
        r->stagers.push_back(g);
    }
    std::atomic<int> bad{0};
    std::vector<std::thread> th;
    th.reserve(T);
    for (unsigned t = 0; t < T; t++) {
        th.emplace_back([&, t] {
            if (cudaSetDevice(r->device) != cudaSuccess) { bad.store(1); return; }
            FaStager& g = r->stagers[t];
            const size_t lo = bytes * t / T, hi = bytes * (t + 1) / T;
            const size_t chunks = (hi - lo + kStageChunk - 1) / kStageChunk;
            auto issue = [&](size_t c) {
                const size_t off = lo + c * kStageChunk, len = std::min(kStageChunk, hi - off);
                if (cudaMemcpyAsync(g.buf[c & 1], src + off, len, cudaMemcpyDeviceToHost, g.stream) != cudaSuccess ||
                    cudaEventRecord(g.done[c & 1], g.stream) != cudaSuccess)
                    bad.store(1);
            };
            issue(0);
            for (size_t c = 0; c < chunks && !bad.load(); c++) {
                if (c + 1 < chunks) issue(c + 1);   // its chunk was emptied in the previous round
                if (cudaEventSynchronize(g.done[c & 1]) != cudaSuccess) { bad.store(1); break; }
                const size_t off = lo + c * kStageChunk;
                std::memcpy(dst + off, g.buf[c & 1], std::min(kStageChunk, hi - off));
            }
            cudaStreamSynchronize(g.stream);
        });
    }
    for (std::thread& x : th) x.join();
    if (bad.load()) return fa_fail(FA_ERR_CUDA, "staged device-to-host copy failed");
    return FA_OK;
}

// Atari::new (src/atari.rs:240-247) as one state column.
void render_power_on(const fa_render* r, std::vector<uint32_t>& col)
{
    col.assign(FA_RROWS, 0u);
    fa_render_power_on_column(r->image.data(), r->nbanks, r->scheme, r->hot_lo, col.data());
}

int enqueue(fa_render* r, const uint8_t* d_actions, int k, uint8_t* d_obs, cudaStream_t s)
{
    FaRenderLaunch L;
    memset(&L, 0, sizeof(L));
    L.rom = r->d_rom;
    L.nbanks = r->nbanks;
    L.hot_lo = r->hot_lo;
    L.state = r->d_state;
    L.stride = r->stride;
    L.n = (uint32_t)r->n;
    L.actions = d_actions;
    L.k = (uint32_t)k;
    L.sched = (uint32_t)r->sched;
    L.fb = r->d_fb;
    L.obs = d_obs;
    L.err = r->d_err;
    L.instr = r->d_ctr;
    L.rounds = r->d_ctr + 1;
    FA_CUDA(launch_render_n(r->warps, L, s));
    return FA_OK;
}

int finish(fa_render* r)
{
    FA_CUDA(cudaStreamSynchronize(r->stream));
    uint32_t err = 0;
    FA_CUDA(cudaMemcpy(&err, r->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    unsigned long long ctr[2];
    FA_CUDA(cudaMemcpy(ctr, r->d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost));
    r->last_instr = ctr[0];
    r->last_slots = ctr[1];
    if (err) {
        cudaMemset(r->d_err, 0, sizeof(uint32_t));
        return fa_fail(FA_ERR_KERNEL, "device wait gave up (error word 0x%x)", err);
    }
    return FA_OK;
}

int copy_out(fa_render* r, uint8_t* fb_out, uint8_t* ram_out)
{
    if (fb_out) {
        const int rc = copy_d2h(r, fb_out, r->d_fb, r->n * (size_t)FA_FB_BYTES);
        if (rc) return rc;
    }
    if (ram_out) return copy_d2h(r, ram_out, r->d_obs, r->n * 128u);
    return FA_OK;
}
}  // namespace

#define CHECK_R(r)                                                                      \
    do {                                                                                \
        if (!(r)) return fa_fail(FA_ERR_INVALID, "null render handle");                 \
        cudaError_t e_ = cudaSetDevice((r)->device);                                    \
        if (e_ != cudaSuccess) return fa_fail(FA_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_)); \
    } while (0)

extern "C" int fa_render_create(const uint8_t* rom, size_t rom_len, size_t n, fa_render** out)
{
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!rom || n == 0) return fa_fail(FA_ERR_INVALID, "need a ROM and n >= 1");
    if (n > (size_t)UINT32_MAX / 2) return fa_fail(FA_ERR_CAPACITY, "too many instances");
    if (fa_device_count() < 1) return fa_fail(FA_ERR_NO_DEVICE, "no CUDA device visible");
    fa_render* r = new (std::nothrow) fa_render();
    if (!r) return fa_fail(FA_ERR_CAPACITY, "out of host memory");
    int rc = fa_make_bank_image(rom, rom_len, r->image, r->scheme, &r->nbanks, &r->hot_lo);
    if (rc) { delete r; return rc; }
    if (r->scheme == FA_SCHEME_DPC || r->scheme == FA_SCHEME_FE) {
        delete r;
        return fa_fail(FA_ERR_BAD_ROM, "DPC and FE carts run on the headless console only");
    }
    cudaGetDevice(&r->device);
    r->n = n;
    r->stride = (uint32_t)((n + 31u) & ~(size_t)31u);
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&r->d_rom, r->image.size())) != cudaSuccess ||
        (e = cudaMemcpy(r->d_rom, r->image.data(), r->image.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&r->d_state, (size_t)FA_RROWS * r->stride * 4u)) != cudaSuccess ||
        (e = cudaMemset(r->d_state, 0, (size_t)FA_RROWS * r->stride * 4u)) != cudaSuccess ||
        (e = cudaMalloc(&r->d_fb, n * (size_t)FA_FB_BYTES)) != cudaSuccess ||
        (e = cudaMemset(r->d_fb, 0, n * (size_t)FA_FB_BYTES)) != cudaSuccess ||
        (e = cudaMalloc(&r->d_obs, n * 128u)) != cudaSuccess ||
        (e = cudaMalloc(&r->d_err, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMemset(r->d_err, 0, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMalloc(&r->d_ctr, 2 * sizeof(unsigned long long))) != cudaSuccess) {
        free_render(r);
        return fa_fail(FA_ERR_CUDA, "render allocation: %s", cudaGetErrorString(e));
    }
    // Until reset, every console is halted (as fa_create's NOT_RESET state).
    std::vector<uint32_t> st((size_t)r->stride, FA_STATUS_NOT_RESET);
    e = cudaMemcpy(r->d_state + (size_t)R_STATUS * r->stride, st.data(), st.size() * 4u, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { free_render(r); return fa_fail(FA_ERR_CUDA, "render init: %s", cudaGetErrorString(e)); }
    *out = r;
    return FA_OK;
}

extern "C" void fa_render_destroy(fa_render* r) { free_render(r); }

extern "C" int fa_render_set_launch(fa_render* r, int cta_warps, int sched)
{
    if (!r) return fa_fail(FA_ERR_INVALID, "null render handle");
    if (cta_warps != 4 && cta_warps != 8 && cta_warps != 16) return fa_fail(FA_ERR_INVALID, "cta_warps must be 4, 8 or 16");
    if (sched < FA_SCHED_LANE || sched > FA_SCHED_MATCH) return fa_fail(FA_ERR_INVALID, "bad sched %d", sched);
    r->warps = cta_warps;
    r->sched = sched;
    return FA_OK;
}

extern "C" int fa_render_reset(fa_render* r, uint8_t* fb_out, uint8_t* ram_out)
{
    CHECK_R(r);
    std::vector<uint32_t> col;
    render_power_on(r, col);
    std::vector<uint32_t> rows((size_t)FA_RROWS * r->stride);
    for (uint32_t w = 0; w < FA_RROWS; w++)
        for (size_t i = 0; i < r->n; i++) rows[(size_t)w * r->stride + i] = col[w];
    FA_CUDA(cudaMemcpyAsync(r->d_state, rows.data(), rows.size() * 4u, cudaMemcpyHostToDevice, r->stream));
    FA_CUDA(cudaMemsetAsync(r->d_fb, 0, r->n * (size_t)FA_FB_BYTES, r->stream));
    FA_CUDA(cudaMemsetAsync(r->d_ctr, 0, 2 * sizeof(unsigned long long), r->stream));
    // One frame without set_action, as the batched reset does.
    int rc = enqueue(r, nullptr, 1, r->d_obs, r->stream);
    if (rc) return rc;
    rc = finish(r);
    if (rc) return rc;
    // The reset frame is not counted: frame numbers restart at 0.
    FA_CUDA(cudaMemset(r->d_state + (size_t)R_FRAME * r->stride, 0, r->n * 4u));
    r->reset_done = true;
    return copy_out(r, fb_out, ram_out);
}

extern "C" int fa_render_step_multi_async(fa_render* r, const uint8_t* d_actions, int k, uint8_t* d_obs, void* stream)
{
    CHECK_R(r);
    if (!d_actions || k < 1) return fa_fail(FA_ERR_INVALID, "actions null or k < 1");
    if (((uintptr_t)d_obs & 15u) != 0) return fa_fail(FA_ERR_INVALID, "d_obs must be 16-byte aligned");
    return enqueue(r, d_actions, k, d_obs, stream ? (cudaStream_t)stream : r->stream);
}

extern "C" int fa_render_step_multi(fa_render* r, const uint8_t* actions, int k, uint8_t* fb_out, uint8_t* ram_out)
{
    CHECK_R(r);
    if (!actions || k < 1) return fa_fail(FA_ERR_INVALID, "actions null or k < 1");
    const size_t bytes = (size_t)k * r->n;
    if (bytes > r->actions_cap) {
        cudaFree(r->d_actions);
        r->d_actions = nullptr;
        r->actions_cap = 0;
        FA_CUDA(cudaMalloc(&r->d_actions, bytes));
        r->actions_cap = bytes;
    }
    FA_CUDA(cudaMemcpyAsync(r->d_actions, actions, bytes, cudaMemcpyHostToDevice, r->stream));
    FA_CUDA(cudaMemsetAsync(r->d_ctr, 0, 2 * sizeof(unsigned long long), r->stream));
    int rc = enqueue(r, r->d_actions, k, r->d_obs, r->stream);
    if (rc) return rc;
    rc = finish(r);
    if (rc) return rc;
    return copy_out(r, fb_out, ram_out);
}

extern "C" int fa_render_synchronize(fa_render* r)
{
    CHECK_R(r);
    return finish(r);
}

extern "C" size_t fa_render_num_envs(const fa_render* r) { return r ? r->n : 0; }

extern "C" uint8_t* fa_render_device_framebuffers(fa_render* r) { return r ? r->d_fb : nullptr; }

extern "C" int fa_render_get_framebuffers(fa_render* r, uint8_t* out)
{
    CHECK_R(r);
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    FA_CUDA(cudaStreamSynchronize(r->stream));
    return copy_d2h(r, out, r->d_fb, r->n * (size_t)FA_FB_BYTES);
}

namespace {
constexpr size_t kRgbaChunkConsoles = 2048;                        // 240 MiB of RGBA per device chunk

cudaError_t launch_rgba(const uint8_t* fb, uint8_t* rgba, size_t consoles, cudaStream_t s)
{
    const size_t words = consoles * (size_t)FA_FB_BYTES / 4u;
    if (words == 0) return cudaSuccess;
    size_t grid = (words + 255u) / 256u;
    if (grid > 148u * 16u) grid = 148u * 16u;
    fa::fa_fb_rgba<<<(unsigned)grid, 256, 0, s>>>((const uint32_t*)fb, (uint4*)rgba, words);
    return cudaGetLastError();
}
}  // namespace

extern "C" uint32_t fa_palette_rgba(uint8_t index) { return kNtscRgba[(index >> 2) & 63u]; }

extern "C" int fa_render_rgba_async(fa_render* r, size_t first, size_t count, uint8_t* d_rgba, void* stream)
{
    CHECK_R(r);
    if (first > r->n || count > r->n - first) return fa_fail(FA_ERR_INVALID, "consoles [%zu, %zu) out of range", first, first + count);
    if (!d_rgba || ((uintptr_t)d_rgba & 15u)) return fa_fail(FA_ERR_INVALID, "d_rgba null or not 16-byte aligned");
    FA_CUDA(launch_rgba(r->d_fb + first * (size_t)FA_FB_BYTES, d_rgba, count, stream ? (cudaStream_t)stream : r->stream));
    return FA_OK;
}

extern "C" int fa_render_get_rgba(fa_render* r, size_t first, size_t count, uint8_t* out)
{
    CHECK_R(r);
    if (first > r->n || count > r->n - first) return fa_fail(FA_ERR_INVALID, "consoles [%zu, %zu) out of range", first, first + count);
    if (!out) return fa_fail(FA_ERR_INVALID, "null output");
    const size_t per = (size_t)FA_FB_BYTES * 4u;
    if (!r->d_rgba) FA_CUDA(cudaMalloc(&r->d_rgba, std::min(r->n, kRgbaChunkConsoles) * per));
    for (size_t c0 = 0; c0 < count; c0 += kRgbaChunkConsoles) {
        const size_t m = std::min(kRgbaChunkConsoles, count - c0);
        FA_CUDA(launch_rgba(r->d_fb + (first + c0) * (size_t)FA_FB_BYTES, r->d_rgba, m, r->stream));
        FA_CUDA(cudaStreamSynchronize(r->stream));
        const int rc = copy_d2h(r, out + c0 * per, r->d_rgba, m * per);
        if (rc) return rc;
    }
    return FA_OK;
}

extern "C" int fa_render_get_states(fa_render* r, fa_state* out)
{
    CHECK_R(r);
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    FA_CUDA(cudaStreamSynchronize(r->stream));
    std::vector<uint32_t> rows((size_t)FA_RROWS * r->stride);
    FA_CUDA(cudaMemcpy(rows.data(), r->d_state, rows.size() * 4u, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < r->n; i++) fa_unpack_column(rows.data() + i, r->stride, r->scheme, out[i]);
    return FA_OK;
}

extern "C" unsigned long long fa_render_last_instructions(const fa_render* r) { return r ? r->last_instr : 0ull; }
