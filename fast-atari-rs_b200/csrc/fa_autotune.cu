// fa_autotune.cu — per-cart launch tuning.
//
// For one ROM and an instance count, measures (CUDA events on the handle's
// stream) frames/s over a staged sweep: the warp scheduling policy, then the
// launch shape (persistent CTAs of 8..32 warps, i.e. register caps of
// 256..64 registers per thread, or the plain form with 64..512-thread CTAs),
// then the frames per launch K.  Every configuration produces identical
// results; only the time differs.  The best record is what a pool or handle
// should use for the cart, and its cost per instance-frame is the pool's
// queue-ordering weight.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

namespace {

struct Tuner {
    fa_handle* h = nullptr;
    uint8_t* d_actions = nullptr;
    size_t n = 0;
    int kmax = 16;
    float target_ms = 30.0f;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<fa_tuning> table;

    ~Tuner()
    {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(d_actions);
        fa_destroy(h);
    }

    // Time one configuration; returns frames/s (0 on error).
    int measure(fa_tuning& t)
    {
        int rc = fa_set_launch(h, t.block, t.sched, t.persistent);
        if (!rc) rc = fa_set_cta_warps(h, t.cta_warps);
        if (rc) return rc;
        // One call to warm up and estimate, then enough calls for target_ms.
        FA_CUDA(cudaEventRecord(e0, h->stream));
        rc = fa_step_multi_async(h, d_actions, t.k, nullptr, h->stream);
        if (rc) return rc;
        FA_CUDA(cudaEventRecord(e1, h->stream));
        FA_CUDA(cudaEventSynchronize(e1));
        float ms1 = 0.0f;
        FA_CUDA(cudaEventElapsedTime(&ms1, e0, e1));
        int reps = (int)std::min(64.0f, std::max(1.0f, target_ms / std::max(ms1, 1e-3f)));
        FA_CUDA(cudaEventRecord(e0, h->stream));
        for (int r = 0; r < reps; r++) {
            rc = fa_step_multi_async(h, d_actions, t.k, nullptr, h->stream);
            if (rc) return rc;
        }
        FA_CUDA(cudaEventRecord(e1, h->stream));
        FA_CUDA(cudaEventSynchronize(e1));
        float ms = 0.0f;
        FA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const double frames = (double)n * t.k * reps;
        t.frames_per_s = (float)(frames / (ms * 1e-3));
        t.ns_per_instance_frame = (float)(ms * 1e6 / frames);
        table.push_back(t);
        return fa_synchronize(h);
    }
};

}  // namespace

extern "C" int fa_autotune(const uint8_t* rom, size_t rom_len, size_t n, fa_tuning* best, fa_tuning* table,
                           int table_cap, int* table_len)
{
    if (!best || n == 0) return fa_fail(FA_ERR_INVALID, "bad autotune arguments");
    Tuner T;
    T.n = n;
    int rc = fa_create(rom, rom_len, n, &T.h);
    if (rc) return rc;
    rc = fa_reset(T.h, nullptr);
    if (rc) return rc;
    FA_CUDA(cudaEventCreate(&T.e0));
    FA_CUDA(cudaEventCreate(&T.e1));
    // Actions uniform over the 18 joystick actions (a 32-bit LCG; the values
    // only need to exercise the cart's input-dependent paths).
    std::vector<uint8_t> acts((size_t)T.kmax * n);
    uint32_t s = 0x12345678u;
    for (auto& a : acts) { s = s * 1664525u + 1013904223u; a = (uint8_t)((s >> 16) % 18u); }
    FA_CUDA(cudaMalloc(&T.d_actions, acts.size()));
    FA_CUDA(cudaMemcpy(T.d_actions, acts.data(), acts.size(), cudaMemcpyHostToDevice));

    fa_tuning cur;
    memset(&cur, 0, sizeof(cur));
    cur.block = 128;
    cur.persistent = 1;
    cur.cta_warps = 0;
    cur.k = 4;
    // Stage 1: warp policy.
    int best_i = -1;
    for (int sched : { FA_SCHED_PC, FA_SCHED_LINE, FA_SCHED_LANE, FA_SCHED_MATCH }) {
        fa_tuning t = cur;
        t.sched = sched;
        if ((rc = T.measure(t))) return rc;
    }
    auto argmax = [&](size_t from) {
        size_t b = from;
        for (size_t i = from; i < T.table.size(); i++)
            if (T.table[i].frames_per_s > T.table[b].frames_per_s) b = i;
        return b;
    };
    cur = T.table[argmax(0)];
    // Stage 2: launch shape (persistent CTA size = register cap, or plain CTAs).
    size_t from = T.table.size();
    T.table.push_back(cur);
    for (int w : { 8, 16, 24 }) {
        fa_tuning t = cur;
        t.persistent = 1;
        t.cta_warps = w;
        if ((rc = T.measure(t))) return rc;
    }
    for (int b : { 64, 128, 256, 512 }) {
        fa_tuning t = cur;
        t.persistent = 0;
        t.block = b;
        t.cta_warps = 0;
        if ((rc = T.measure(t))) return rc;
    }
    cur = T.table[argmax(from)];
    // Stage 3: frames per launch.
    from = T.table.size();
    T.table.push_back(cur);
    for (int k : { 1, 2, 8, 16 }) {
        fa_tuning t = cur;
        t.k = k;
        if ((rc = T.measure(t))) return rc;
    }
    best_i = (int)argmax(from);
    *best = T.table[best_i];
    if (table_len) *table_len = (int)T.table.size();
    if (table)
        for (int i = 0; i < (int)T.table.size() && i < table_cap; i++) table[i] = T.table[i];
    return FA_OK;
}
