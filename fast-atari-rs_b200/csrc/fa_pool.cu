// fa_pool.cu — several carts' instance sets stepped by one launch.
//
// The batched form of the core: a pool holds one fa_handle per cart (each
// with its own ROM, SoA state and post-reset snapshot) and steps all of them
// with a single launch of fa_run whose work queue interleaves the carts'
// units, heaviest group first.  Repeated calls can be captured once into a
// CUDA graph (memset of the per-call queue counters + one launch per call)
// and replayed.  The plain form — one launch per frame per cart, as the
// reference's BatchAtariGpu::step does (src/cuda_env.rs:144-161) — is kept
// beside it on the same state for comparison.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

struct fa_pool {
    int device = 0;
    int sms = 148;
    std::vector<fa_handle*> groups;
    std::vector<float> weight;         // relative cost of one unit; heavier units are queued first
    int block = 128;
    bool persistent = true;
    int cta_warps = 0;
    cudaStream_t stream = nullptr;
    uint32_t* d_err = nullptr;         // device error word
    uint32_t* d_queue = nullptr;       // one work-queue counter per call
    uint32_t queue_cap = 0;
    unsigned long long* d_ctr = nullptr;   // [0] instructions, [1] lane slots
    unsigned long long last_instr = 0, last_slots = 0;
    unsigned long long* d_trace = nullptr;  // caller's per-unit trace buffer (fa_pool_set_trace), or null
    uint32_t trace_cap = 0;
    // First-wave placement of the persistent launch (fa_pool_set_balance):
    // one device table per (grid, warps, unit costs), written once and kept
    // until the pool is destroyed, so a launch queued on any stream, or held
    // by a graph, reads the table it was given.
    bool balance = false;
    std::vector<std::pair<std::vector<float>, uint32_t*>> plans;
};

struct fa_graph {
    fa_pool* pool = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int calls = 0, k = 0;
};

#define CHECK_P(p)                                                                      \
    do {                                                                                \
        if (!(p)) return fa_fail(FA_ERR_INVALID, "null pool");                          \
        cudaError_t e_ = cudaSetDevice((p)->device);                                    \
        if (e_ != cudaSuccess) return fa_fail(FA_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_)); \
    } while (0)

extern "C" int fa_pool_create(fa_pool** out)
{
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    *out = nullptr;
    if (fa_device_count() < 1) return fa_fail(FA_ERR_NO_DEVICE, "no CUDA device visible");
    fa_pool* p = new (std::nothrow) fa_pool();
    if (!p) return fa_fail(FA_ERR_CAPACITY, "out of host memory");
    cudaGetDevice(&p->device);
    cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device);
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&p->d_err, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMemset(p->d_err, 0, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMalloc(&p->d_ctr, 2 * sizeof(unsigned long long))) != cudaSuccess) {
        fa_pool_destroy(p);
        return fa_fail(FA_ERR_CUDA, "pool allocation: %s", cudaGetErrorString(e));
    }
    *out = p;
    return FA_OK;
}

extern "C" void fa_pool_destroy(fa_pool* p)
{
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (fa_handle* h : p->groups) fa_destroy(h);
    cudaFree(p->d_err);
    cudaFree(p->d_queue);
    cudaFree(p->d_ctr);
    for (auto& pl : p->plans) cudaFree(pl.second);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

extern "C" int fa_pool_add_cart(fa_pool* p, const uint8_t* rom, size_t rom_len, size_t n, int* group)
{
    CHECK_P(p);
    if ((int)p->groups.size() >= FA_MAX_GROUPS)
        return fa_fail(FA_ERR_CAPACITY, "a pool holds at most %d carts", FA_MAX_GROUPS);
    fa_handle* h = nullptr;
    int rc = fa_create(rom, rom_len, n, &h);
    if (rc) return rc;
    rc = fa_reset(h, nullptr);
    if (rc) { fa_destroy(h); return rc; }
    h->sched = FA_SCHED_PC;
    p->groups.push_back(h);
    p->weight.push_back(1.0f);
    if (group) *group = (int)p->groups.size() - 1;
    return FA_OK;
}

extern "C" int fa_pool_num_groups(const fa_pool* p) { return p ? (int)p->groups.size() : 0; }

extern "C" fa_handle* fa_pool_group(fa_pool* p, int group)
{
    if (!p || group < 0 || group >= (int)p->groups.size()) return nullptr;
    return p->groups[group];
}

extern "C" int fa_pool_set_group(fa_pool* p, int group, int sched, float weight)
{
    if (!p || group < 0 || group >= (int)p->groups.size()) return fa_fail(FA_ERR_INVALID, "bad group %d", group);
    if (sched < FA_SCHED_LANE || sched > FA_SCHED_MATCH) return fa_fail(FA_ERR_INVALID, "bad sched %d", sched);
    if (!(weight > 0.0f)) return fa_fail(FA_ERR_INVALID, "weight must be > 0");
    p->groups[group]->sched = sched;
    p->weight[group] = weight;
    return FA_OK;
}

extern "C" int fa_pool_set_launch(fa_pool* p, int block, int persistent)
{
    if (!p) return fa_fail(FA_ERR_INVALID, "null pool");
    if (block != 64 && block != 128 && block != 256 && block != 512)
        return fa_fail(FA_ERR_INVALID, "block must be 64, 128, 256 or 512");
    p->block = block;
    p->persistent = persistent != 0;
    return FA_OK;
}

extern "C" int fa_pool_set_cta_warps(fa_pool* p, int warps)
{
    if (!p) return fa_fail(FA_ERR_INVALID, "null pool");
    if (warps != 0 && warps != 2 && warps != 4 && warps != 8 && warps != 16 && warps != 24 && warps != 28 &&
        warps != 32)
        return fa_fail(FA_ERR_INVALID, "warps per CTA must be 0 (auto), 2, 4, 8, 16, 24, 28 or 32");
    p->cta_warps = warps;
    return FA_OK;
}

static int ensure_queues(fa_pool* p, uint32_t calls)
{
    if (calls <= p->queue_cap) return FA_OK;
    cudaFree(p->d_queue);
    p->d_queue = nullptr;
    p->queue_cap = 0;
    FA_CUDA(cudaMalloc(&p->d_queue, calls * sizeof(uint32_t)));
    p->queue_cap = calls;
    return FA_OK;
}

// Launch descriptor for one call: groups ordered heaviest first.
static int build_launch(fa_pool* p, const uint8_t* const* d_actions, uint32_t k, uint8_t* const* d_obs,
                        size_t call, FaLaunch& L)
{
    memset(&L, 0, sizeof(L));
    std::vector<int> order(p->groups.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return p->weight[a] > p->weight[b]; });
    uint32_t units = 0, rom_max = 0;
    for (int gi : order) {
        fa_handle* h = p->groups[gi];
        const uint8_t* acts = d_actions ? d_actions[gi] + call * (size_t)k * h->n : nullptr;
        FaGroup g = fa_handle_group(h, acts, k, d_obs ? d_obs[gi] : nullptr);
        g.tag = (uint32_t)gi;
        g.unit_begin = units;
        units += (uint32_t)((h->n + p->block - 1) / p->block);
        rom_max = std::max(rom_max, h->nbanks * 4096u);
        L.g[L.ngroups++] = g;
    }
    L.nunits = units;
    L.rom_bytes_max = rom_max;
    L.cta_warps = (uint32_t)p->cta_warps;
    L.err = p->d_err;
    L.instr = p->d_ctr;
    L.rounds = p->d_ctr + 1;
    L.trace = p->d_trace;
    L.trace_cap = p->trace_cap;
    return FA_OK;
}

// The first wave of a persistent warp-granular launch with one CTA per SM,
// placed by fa_plan_first_wave: a unit costs its cart's weight (relative cost
// of one instance-frame) times its instances times k.  A new table is
// computed and uploaded (synchronously, never inside a stream capture) the
// first time a shape and cost list appears; past kMaxPlans distinct ones the
// launch runs without a plan.
static int ensure_plan(fa_pool* p, FaLaunch& L, uint32_t k)
{
    constexpr size_t kMaxPlans = 16;
    L.first_wave = nullptr;
    if (!p->balance || !p->persistent) return FA_OK;
    uint32_t grid = 0, warps = 0;
    int per_sm = 0;
    if (!fa_launch_warp_shape(L, p->block, true, p->sms, &grid, &warps, &per_sm) || per_sm != 1 || warps % 4u != 0u)
        return FA_OK;
    std::vector<float> key;
    key.reserve(2 + L.nunits);
    key.push_back((float)grid);
    key.push_back((float)warps);
    for (uint32_t g = 0; g < L.ngroups; g++) {
        const uint32_t units = (L.g[g].n + 31u) / 32u;
        for (uint32_t u = 0; u < units; u++) {
            const uint32_t inst = std::min(32u, L.g[g].n - 32u * u);
            key.push_back(p->weight[L.g[g].tag] * (float)inst * (float)k);
        }
    }
    for (auto& pl : p->plans)
        if (pl.first == key) { L.first_wave = pl.second; return FA_OK; }
    if (p->plans.size() >= kMaxPlans) return FA_OK;
    std::vector<uint32_t> table((size_t)grid * warps);
    fa_plan_first_wave(key.data() + 2, (uint32_t)(key.size() - 2), grid, warps, table.data());
    uint32_t* d = nullptr;
    FA_CUDA(cudaMalloc(&d, table.size() * sizeof(uint32_t)));
    const cudaError_t e = cudaMemcpy(d, table.data(), table.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        FA_CUDA(e);
    }
    p->plans.emplace_back(std::move(key), d);
    L.first_wave = d;
    return FA_OK;
}

static int pool_enqueue(fa_pool* p, const uint8_t* const* d_actions, int k, uint8_t* const* d_obs,
                        cudaStream_t s)
{
    if (p->groups.empty()) return fa_fail(FA_ERR_INVALID, "pool has no carts");
    if (k < 1) return fa_fail(FA_ERR_INVALID, "k < 1");
    int rc = ensure_queues(p, 1);
    if (rc) return rc;
    FaLaunch L;
    build_launch(p, d_actions, (uint32_t)k, d_obs, 0, L);
    rc = ensure_plan(p, L, (uint32_t)k);
    if (rc) return rc;
    if (p->persistent) {
        L.queue = p->d_queue;
        FA_CUDA(cudaMemsetAsync(p->d_queue, 0, sizeof(uint32_t), s));
    }
    FA_CUDA(fa_launch_run(L, p->block, p->persistent, p->sms, s));
    return FA_OK;
}

// The plain form: every frame, one launch per cart, one CTA per unit.
static int pool_enqueue_plain(fa_pool* p, const uint8_t* const* d_actions, int k, uint8_t* const* d_obs,
                              cudaStream_t s)
{
    if (p->groups.empty()) return fa_fail(FA_ERR_INVALID, "pool has no carts");
    if (k < 1) return fa_fail(FA_ERR_INVALID, "k < 1");
    for (int f = 0; f < k; f++) {
        for (size_t gi = 0; gi < p->groups.size(); gi++) {
            fa_handle* h = p->groups[gi];
            FaLaunch L;
            memset(&L, 0, sizeof(L));
            const uint8_t* acts = d_actions ? d_actions[gi] + (size_t)f * h->n : nullptr;
            L.g[0] = fa_handle_group(h, acts, 1, (f == k - 1 && d_obs) ? d_obs[gi] : nullptr);
            L.ngroups = 1;
            L.nunits = (uint32_t)((h->n + p->block - 1) / p->block);
            L.rom_bytes_max = h->nbanks * 4096u;
            L.err = p->d_err;
            L.instr = p->d_ctr;
            L.rounds = p->d_ctr + 1;
            FA_CUDA(fa_launch_run(L, p->block, false, p->sms, s));
        }
    }
    return FA_OK;
}

static int pool_finish(fa_pool* p)
{
    FA_CUDA(cudaStreamSynchronize(p->stream));
    uint32_t err = 0;
    FA_CUDA(cudaMemcpy(&err, p->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    unsigned long long ctr[2];
    FA_CUDA(cudaMemcpy(ctr, p->d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost));
    p->last_instr = ctr[0];
    p->last_slots = ctr[1];
    if (err) {
        cudaMemset(p->d_err, 0, sizeof(uint32_t));
        return fa_fail(FA_ERR_KERNEL, "device wait gave up (error word 0x%x)", err);
    }
    return FA_OK;
}

// Host-buffer step of every cart: actions[g] holds k*n_g bytes frame-major,
// obs[g] (or NULL) receives n_g*128 bytes; plain != 0 uses the plain form.
static int pool_step_host(fa_pool* p, const uint8_t* const* actions, int k, uint8_t* const* obs, bool plain)
{
    CHECK_P(p);
    if (!actions) return fa_fail(FA_ERR_INVALID, "actions is null");
    const size_t G = p->groups.size();
    std::vector<const uint8_t*> d_act(G);
    std::vector<uint8_t*> d_obs(G);
    for (size_t gi = 0; gi < G; gi++) {
        fa_handle* h = p->groups[gi];
        if (!actions[gi]) return fa_fail(FA_ERR_INVALID, "actions[%zu] is null", gi);
        const size_t bytes = (size_t)k * h->n;
        if (bytes > h->actions_cap) {
            cudaFree(h->d_actions);
            cudaFreeHost(h->h_actions);
            h->d_actions = nullptr;
            h->h_actions = nullptr;
            h->actions_cap = h->h_actions_cap = 0;
            FA_CUDA(cudaMalloc(&h->d_actions, bytes));
            FA_CUDA(cudaMallocHost(&h->h_actions, bytes));
            h->actions_cap = h->h_actions_cap = bytes;
        }
        memcpy(h->h_actions, actions[gi], bytes);
        FA_CUDA(cudaMemcpyAsync(h->d_actions, h->h_actions, bytes, cudaMemcpyHostToDevice, p->stream));
        d_act[gi] = h->d_actions;
        // Observations go straight into the pinned buffer where it is mapped.
        d_obs[gi] = (obs && obs[gi]) ? (h->h_obs_dev ? h->h_obs_dev : h->d_obs) : nullptr;
    }
    FA_CUDA(cudaMemsetAsync(p->d_ctr, 0, 2 * sizeof(unsigned long long), p->stream));
    int rc = plain ? pool_enqueue_plain(p, d_act.data(), k, d_obs.data(), p->stream)
                   : pool_enqueue(p, d_act.data(), k, d_obs.data(), p->stream);
    if (rc) return rc;
    for (size_t gi = 0; gi < G; gi++)
        if (d_obs[gi] && !p->groups[gi]->h_obs_dev)
            FA_CUDA(cudaMemcpyAsync(p->groups[gi]->h_obs, d_obs[gi], p->groups[gi]->n * 128,
                                    cudaMemcpyDeviceToHost, p->stream));
    rc = pool_finish(p);
    if (rc) return rc;
    for (size_t gi = 0; gi < G; gi++)
        if (d_obs[gi]) fa_host_copy(obs[gi], p->groups[gi]->h_obs, p->groups[gi]->n * 128);
    return FA_OK;
}

extern "C" int fa_pool_step(fa_pool* p, const uint8_t* const* actions, int k, uint8_t* const* obs)
{
    return pool_step_host(p, actions, k, obs, false);
}

extern "C" int fa_pool_step_plain(fa_pool* p, const uint8_t* const* actions, int k, uint8_t* const* obs)
{
    return pool_step_host(p, actions, k, obs, true);
}

extern "C" int fa_pool_step_async(fa_pool* p, const uint8_t* const* d_actions, int k, uint8_t* const* d_obs,
                                  void* stream)
{
    CHECK_P(p);
    if (!d_actions) return fa_fail(FA_ERR_INVALID, "d_actions is null");
    return pool_enqueue(p, d_actions, k, d_obs, stream ? (cudaStream_t)stream : p->stream);
}

extern "C" int fa_pool_step_plain_async(fa_pool* p, const uint8_t* const* d_actions, int k,
                                        uint8_t* const* d_obs, void* stream)
{
    CHECK_P(p);
    if (!d_actions) return fa_fail(FA_ERR_INVALID, "d_actions is null");
    return pool_enqueue_plain(p, d_actions, k, d_obs, stream ? (cudaStream_t)stream : p->stream);
}

extern "C" int fa_pool_synchronize(fa_pool* p)
{
    CHECK_P(p);
    FA_CUDA(cudaDeviceSynchronize());
    return pool_finish(p);
}

extern "C" int fa_pool_set_balance(fa_pool* p, int on)
{
    if (!p) return fa_fail(FA_ERR_INVALID, "null pool");
    p->balance = on != 0;
    return FA_OK;
}

extern "C" int fa_pool_set_trace(fa_pool* p, unsigned long long* d_trace, uint32_t cap)
{
    if (!p) return fa_fail(FA_ERR_INVALID, "null pool");
    if (!d_trace != !cap) return fa_fail(FA_ERR_INVALID, "trace buffer and capacity go together");
    if ((uintptr_t)d_trace & 7u) return fa_fail(FA_ERR_INVALID, "trace buffer must be 8-byte aligned");
    p->d_trace = d_trace;
    p->trace_cap = cap;
    return FA_OK;
}

extern "C" int fa_pool_reset_counters(fa_pool* p)
{
    CHECK_P(p);
    FA_CUDA(cudaMemsetAsync(p->d_ctr, 0, 2 * sizeof(unsigned long long), p->stream));
    FA_CUDA(cudaStreamSynchronize(p->stream));
    return FA_OK;
}

extern "C" unsigned long long fa_pool_last_instructions(const fa_pool* p) { return p ? p->last_instr : 0ull; }
extern "C" unsigned long long fa_pool_last_lane_slots(const fa_pool* p) { return p ? p->last_slots : 0ull; }

extern "C" int fa_pool_graph_create(fa_pool* p, const uint8_t* const* d_actions, int k, int calls,
                                    uint8_t* const* d_obs, fa_graph** out)
{
    CHECK_P(p);
    if (!out || !d_actions || k < 1 || calls < 1) return fa_fail(FA_ERR_INVALID, "bad graph arguments");
    if (p->groups.empty()) return fa_fail(FA_ERR_INVALID, "pool has no carts");
    *out = nullptr;
    int rc = ensure_queues(p, (uint32_t)calls);
    if (rc) return rc;
    // Warm the launch configuration cache outside the capture.
    FaLaunch L;
    build_launch(p, d_actions, (uint32_t)k, d_obs, 0, L);
    FA_CUDA(fa_launch_prepare(L, p->block, p->persistent));
    rc = ensure_plan(p, L, (uint32_t)k);                                 // uploaded before the capture
    if (rc) return rc;
    const uint32_t* plan = L.first_wave;
    fa_graph* g = new (std::nothrow) fa_graph();
    if (!g) return fa_fail(FA_ERR_CAPACITY, "out of host memory");
    g->pool = p;
    g->calls = calls;
    g->k = k;
    cudaError_t e = cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { delete g; return fa_fail(FA_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e)); }
    cudaError_t le = cudaMemsetAsync(p->d_queue, 0, (size_t)calls * sizeof(uint32_t), p->stream);
    for (int c = 0; c < calls && le == cudaSuccess; c++) {
        build_launch(p, d_actions, (uint32_t)k, d_obs, (size_t)c, L);
        L.first_wave = plan;
        if (p->persistent) L.queue = p->d_queue + c;
        le = fa_launch_run(L, p->block, p->persistent, p->sms, p->stream);
    }
    e = cudaStreamEndCapture(p->stream, &g->graph);
    if (le != cudaSuccess || e != cudaSuccess) {
        if (g->graph) cudaGraphDestroy(g->graph);
        delete g;
        return fa_fail(FA_ERR_CUDA, "graph capture: %s", cudaGetErrorString(le != cudaSuccess ? le : e));
    }
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g->graph);
        delete g;
        return fa_fail(FA_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = g;
    return FA_OK;
}

extern "C" int fa_graph_launch(fa_graph* g, void* stream)
{
    if (!g) return fa_fail(FA_ERR_INVALID, "null graph");
    cudaSetDevice(g->pool->device);
    FA_CUDA(cudaGraphLaunch(g->exec, stream ? (cudaStream_t)stream : g->pool->stream));
    return FA_OK;
}

extern "C" void fa_graph_destroy(fa_graph* g)
{
    if (!g) return;
    cudaSetDevice(g->pool->device);
    cudaStreamSynchronize(g->pool->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

extern "C" void* fa_pool_stream(fa_pool* p) { return p ? (void*)p->stream : nullptr; }
