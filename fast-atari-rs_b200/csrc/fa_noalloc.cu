// fa_noalloc.cu — stepping entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: their HBM is owned by another
// allocator that reserved it up front (a training framework's caching
// allocator, a serving process with a fixed memory plan), or they step from a
// loop where cudaMalloc's implicit device synchronisation would stall work on
// other streams.  fa_step_static serves them: the caller passes the ROM image,
// the state rows, the actions and the observation buffer, and the only
// scratch the persistent kernel needs — one work-queue counter per call, the
// error word and two statistics counters — lives in the fixed array below,
// which is part of the library image on every GPU that loads it.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

// Words [0,8): error word, then two 64-bit counters at word 2 and word 4;
// words [8, 8 + FA_STATIC_MAX_CALLS): one queue counter per call.
static __device__ __align__(256) uint32_t g_static_scratch[8 + FA_STATIC_MAX_CALLS];

namespace {
std::mutex g_mu;
uint32_t* g_scratch_addr[64];   // device address of g_static_scratch, per device ordinal

// The array's device address on the current device.  In host code the name
// g_static_scratch is only a host-side stand-in, so the address is looked up
// once per device with that device current.
int scratch_on_current_device(uint32_t** out)
{
    int dev = 0;
    FA_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fa_fail(FA_ERR_NO_DEVICE, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return fa_fail(FA_ERR_CUDA, "cudaGetSymbolAddress(g_static_scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = (uint32_t*)p;
    }
    *out = g_scratch_addr[dev];
    return FA_OK;
}
}  // namespace

extern "C" int fa_step_static(const uint8_t* d_rom_image, int scheme, uint32_t* d_state, uint32_t stride,
                              uint32_t n, const uint8_t* d_actions, int k, int calls, uint8_t* d_obs,
                              int sched, void* stream)
{
    if (!d_rom_image || !d_state || !d_actions) return fa_fail(FA_ERR_INVALID, "null buffer");
    if (scheme < FA_SCHEME_FIXED || scheme > FA_SCHEME_F4) return fa_fail(FA_ERR_INVALID, "bad scheme %d", scheme);
    if (n == 0 || stride < n) return fa_fail(FA_ERR_INVALID, "need n >= 1 and stride >= n");
    if (k < 1) return fa_fail(FA_ERR_INVALID, "k < 1");
    if (calls < 1 || calls > FA_STATIC_MAX_CALLS)
        return fa_fail(FA_ERR_CAPACITY, "calls must be 1..%d (fixed scratch of the no-allocation entry point)",
                       FA_STATIC_MAX_CALLS);
    if (sched < FA_SCHED_LANE || sched > FA_SCHED_MATCH) return fa_fail(FA_ERR_INVALID, "bad sched %d", sched);
    if (((uintptr_t)d_rom_image & 15u) || ((uintptr_t)d_obs & 15u) || ((uintptr_t)d_state & 3u))
        return fa_fail(FA_ERR_INVALID, "ROM image and observations must be 16-byte aligned, state 4-byte");
    uint32_t* scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    int dev = 0, sms = 148;
    FA_CUDA(cudaGetDevice(&dev));
    FA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = (cudaStream_t)stream;

    // The array keeps the previous call's contents: clear what must start at zero.
    FA_CUDA(cudaMemsetAsync(scratch, 0, (8u + (uint32_t)calls) * sizeof(uint32_t), s));
    FaLaunch L;
    memset(&L, 0, sizeof(L));
    FaGroup& g = L.g[0];
    g.rom = d_rom_image;
    g.state = d_state;
    g.stride = stride;
    g.n = n;
    g.act_stride = n;
    g.nbanks = fa_nbanks(scheme);
    g.hot_lo = fa_hot_lo(scheme);
    g.k = (uint32_t)k;
    g.sched = (uint32_t)sched;
    g.obs = d_obs;
    L.ngroups = 1;
    L.nunits = (n + 127u) / 128u;
    L.rom_bytes_max = g.nbanks * 4096u;
    L.err = scratch;
    L.instr = (unsigned long long*)(scratch + 2);
    L.rounds = (unsigned long long*)(scratch + 4);
    for (int c = 0; c < calls; c++) {
        g.actions = d_actions + (size_t)c * (size_t)k * n;
        L.queue = scratch + 8 + c;
        FA_CUDA(fa_launch_run(L, 128, true, sms, s));
    }
    // The error word comes back on the caller's stream: only that stream is
    // waited for, not every blocking stream of the device.
    uint32_t err = 0;
    FA_CUDA(cudaMemcpyAsync(&err, scratch, sizeof(err), cudaMemcpyDeviceToHost, s));
    FA_CUDA(cudaStreamSynchronize(s));
    if (err) return fa_fail(FA_ERR_KERNEL, "device wait gave up (error word 0x%x)", err);
    return FA_OK;
}
