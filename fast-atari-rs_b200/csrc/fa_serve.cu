// fa_serve.cu — the serving engine: continuous batching of step requests.
//
// No reference counterpart: the reference's BatchAtariGpu (src/cuda_env.rs:
// 99-191) serves one caller, one ROM and one synchronous step at a time.  A
// server holds the carts' ROM images and every session's instance state in
// HBM; clients on any thread submit step requests (a session, a batch size n,
// a frame count k and k*n actions) and wait for their observations.
//
// Memory.  Instance state lives in blocks of FA_SERVE_BLOCK_COLS SoA columns
// (one block = FA_ROWS rows x 256 words = 68,608 bytes), carved from device
// slabs.  A session owns a list of blocks, so it grows by appending blocks,
// never by moving state.  New instances are admitted — their blocks allocated
// and set to the cart's post-reset snapshot — when a request names more
// instances than the session holds, against a budget of state bytes; when the
// budget is exhausted, admissions wait in FIFO order until closed sessions
// return their blocks (requests that need no new instances keep running).
//
// Scheduling.  One engine thread owns all CUDA work.  Whenever launch slots
// are free it takes the head request of every idle session (a session's
// requests run in submission order, one at a time), admits them in arrival
// order and dispatches them: one staging copy (request table, per-request
// unit counters, unit table, actions), the fresh-block initialisations, then
// one fa_serve launch per cart on that slot's per-cart streams.  Up to
// max_inflight such batches are on the GPU at once, and because fa_serve has
// no persistent CTAs, the CTAs of a batch dispatched while others run start on
// the SM slots that drain first: requests that arrive while others are on the
// GPU join the device's work without waiting for a batch boundary.
// Completion is per request: kernels write observations straight into the
// slot's host-mapped buffer and the last CTA of a request raises its flag
// there, so a request completes — and its session may run again — as soon as
// its own CTAs finish, not when its batch does.  The slot's buffers are
// reused once its event reports every launch finished.  The plain mode
// instead serves the FIFO as static batches, one batch on the GPU at a time,
// each frame a separate launch per cart, completing when the batch does —
// the reference's one-launch-per-frame kernel behind a queue.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr size_t kBlockWords = (size_t)FA_ROWS * FA_SERVE_BLOCK_COLS;
constexpr size_t kBlockBytes = kBlockWords * sizeof(uint32_t);
constexpr size_t kSlabBlocks = 256;            // blocks per device allocation (14.9 MB)
constexpr size_t kScratch = 64;                // per slot: error word, instruction / lane-slot counters
constexpr int kMaxSlots = 64;

inline double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}
inline size_t align16(size_t v) { return (v + 15u) & ~(size_t)15u; }
inline uint32_t blocks_for(uint32_t n) { return (n + FA_SERVE_BLOCK_COLS - 1u) / FA_SERVE_BLOCK_COLS; }

struct Request {
    uint64_t ticket = 0;
    int64_t sid = 0;
    uint32_t n = 0, k = 0;
    std::vector<uint8_t> actions;
    uint8_t* obs = nullptr;
    std::vector<uint32_t*> fresh;      // blocks admitted for this request (set to the snapshot first)
    Clock::time_point t_submit, t_dispatch, t_done;
    Clock::time_point t_ready;         // its session's earlier requests were done (>= t_submit)
    int status = FA_OK;
    bool done = false, waited_admission = false;
    uint32_t batch = 0;
};
using ReqP = std::shared_ptr<Request>;

struct Session {
    int cart = 0;
    uint32_t size = 0;                 // instances that exist: the largest n requested
    std::vector<uint32_t*> blocks;
    std::deque<ReqP> pending;          // not yet dispatched, in submission order
    bool busy = false;                 // a request of the session is on the GPU
    Clock::time_point t_free{};        // when its last request finished
    bool closing = false;
};

struct Cart {
    fa_handle* h = nullptr;            // device ROM image and post-reset snapshot
    uint32_t* d_block_img = nullptr;   // one state block whose every column is the snapshot
    uint32_t nbanks = 1, hot_lo = 0x2000;
    int scheme = 0;
};

struct Slot {
    cudaStream_t main = nullptr;
    std::vector<cudaStream_t> cs;      // one per cart
    std::vector<cudaEvent_t> ev_cart;
    cudaEvent_t ev_ready = nullptr, ev_done = nullptr;
    uint8_t* h_stage = nullptr;        // pinned: request table | unit counters | unit table | actions
    uint8_t* d_stage = nullptr;
    size_t stage_cap = 0;
    uint8_t* h_out = nullptr;          // pinned, mapped: completion flags | observations
    uint8_t* dh_out = nullptr;         // the same memory as the device addresses it
    size_t out_cap = 0;
    uint8_t* d_scratch = nullptr;      // device: error word, instruction / lane-slot counters
    uint8_t* h_scratch = nullptr;      // pinned copy of it
    std::vector<ReqP> reqs;
    std::vector<size_t> obs_off;
    std::vector<char> req_done;
    size_t flags_bytes = 0;
    size_t open_reqs = 0;              // requests of the slot not yet completed
    bool busy = false;
};

}  // namespace

struct fa_server {
    int device = 0;
    fa_server_config cfg{};
    std::vector<Cart> carts;
    std::vector<Slot> slots;
    // state arena
    std::vector<void*> slabs;
    std::vector<uint32_t*> free_blocks;
    size_t blocks_allocated = 0, blocks_used = 0, blocks_peak = 0, budget_blocks = 0;
    // sessions and requests
    std::unordered_map<int64_t, Session> sessions;
    int64_t next_sid = 1;
    uint64_t next_ticket = 1;
    std::unordered_map<uint64_t, ReqP> tickets;
    // engine
    std::mutex mu;
    std::condition_variable cv_engine, cv_done;
    std::thread engine;
    bool stop = false;
    int fatal = FA_OK;
    std::string fatal_msg;
    fa_server_stats st{};
};

namespace {

// Host-mapped pinned memory the kernels write observations and completion
// flags into directly (*d is its device address).
int grow_mapped(uint8_t** h, uint8_t** d, size_t* cap, size_t need)
{
    if (need <= *cap) return FA_OK;
    size_t c = std::max(need, *cap * 2);
    cudaFreeHost(*h);
    *h = nullptr;
    *d = nullptr;
    *cap = 0;
    FA_CUDA(cudaHostAlloc((void**)h, c, cudaHostAllocMapped | cudaHostAllocPortable));
    FA_CUDA(cudaHostGetDevicePointer((void**)d, *h, 0));
    *cap = c;
    return FA_OK;
}

int grow_pinned(uint8_t** h, uint8_t** d, size_t* cap, size_t need)
{
    if (need <= *cap) return FA_OK;
    size_t c = std::max(need, *cap * 2);
    cudaFreeHost(*h);
    cudaFree(*d);
    *h = nullptr;
    *d = nullptr;
    *cap = 0;
    FA_CUDA(cudaMallocHost(h, c));
    FA_CUDA(cudaMalloc(d, c));
    *cap = c;
    return FA_OK;
}

// One block from the arena, or null if the budget or the device is exhausted.
uint32_t* alloc_block(fa_server* s)
{
    if (s->blocks_used >= s->budget_blocks) return nullptr;
    if (s->free_blocks.empty()) {
        const size_t nb = std::min(kSlabBlocks, s->budget_blocks - s->blocks_allocated);
        if (nb == 0) return nullptr;
        void* p = nullptr;
        if (cudaMalloc(&p, nb * kBlockBytes) != cudaSuccess) return nullptr;
        s->slabs.push_back(p);
        s->blocks_allocated += nb;
        for (size_t i = nb; i-- > 0;) s->free_blocks.push_back((uint32_t*)((uint8_t*)p + i * kBlockBytes));
    }
    uint32_t* b = s->free_blocks.back();
    s->free_blocks.pop_back();
    s->blocks_used++;
    s->blocks_peak = std::max(s->blocks_peak, s->blocks_used);
    return b;
}

void release_session(fa_server* s, int64_t sid)
{
    auto it = s->sessions.find(sid);
    if (it == s->sessions.end()) return;
    for (uint32_t* b : it->second.blocks) s->free_blocks.push_back(b);
    s->blocks_used -= it->second.blocks.size();
    s->sessions.erase(it);
}

void finish_request(fa_server* s, const ReqP& r, int status)
{
    r->status = status;
    r->t_done = Clock::now();
    r->done = true;
    auto it = s->sessions.find(r->sid);
    if (it != s->sessions.end()) {
        it->second.busy = false;
        it->second.t_free = r->t_done;
        if (it->second.closing && it->second.pending.empty()) release_session(s, r->sid);
    }
    if (status == FA_OK) {
        s->st.requests_done++;
        s->st.instance_frames += (unsigned long long)r->n * r->k;
    } else {
        s->st.requests_failed++;
    }
}

// Complete request i of a slot: its observations (in the slot's mapped
// buffer) go to the caller, and its session may run its next request.
void complete_request(fa_server* s, Slot& sl, size_t i, int status)
{
    if (sl.req_done[i]) return;
    const ReqP& r = sl.reqs[i];
    if (status == FA_OK && r->obs)
        memcpy(r->obs, sl.h_out + sl.flags_bytes + sl.obs_off[i], (size_t)r->n * 128u);
    finish_request(s, r, status);
    sl.req_done[i] = 1;
    sl.open_reqs--;
}

// The slot's launches have all finished (status != FA_OK: they failed):
// requests not yet completed complete now, and the slot's buffers are free.
void release_slot(fa_server* s, Slot& sl, int status)
{
    uint32_t err = 0;
    unsigned long long ctr[2] = { 0, 0 };
    if (status == FA_OK) {
        memcpy(&err, sl.h_scratch, sizeof(err));
        memcpy(ctr, sl.h_scratch + 8, sizeof(ctr));
        if (err) status = FA_ERR_KERNEL;
    }
    s->st.guest_instructions += ctr[0];
    s->st.lane_slots += ctr[1];
    for (size_t i = 0; i < sl.reqs.size(); i++) complete_request(s, sl, i, status);
    sl.reqs.clear();
    sl.obs_off.clear();
    sl.req_done.clear();
    sl.busy = false;
}

void fail_server(fa_server* s, int code, const std::string& msg)
{
    if (s->fatal == FA_OK) {
        s->fatal = code;
        s->fatal_msg = msg;
    }
}

// Enqueue one batch on slot `si`.  The requests' fresh blocks are already
// allocated; they are set to the snapshot before the launches.
int launch_slot(fa_server* s, int si, std::vector<ReqP>& reqs)
{
    Slot& sl = s->slots[si];
    const bool plain = s->cfg.mode == FA_SERVE_PLAIN;
    const uint32_t B = (uint32_t)s->cfg.block;
    const size_t ncarts = s->carts.size();
    // Longest requests first: their CTAs start first, and in the plain form
    // the units still running at frame f are a prefix of each cart's table.
    std::stable_sort(reqs.begin(), reqs.end(), [](const ReqP& a, const ReqP& b) { return a->k > b->k; });

    std::vector<std::vector<FaServeUnit>> units(ncarts);
    std::vector<std::vector<uint32_t>> unit_k(ncarts);
    size_t act_bytes = 0, obs_bytes = 0;
    uint32_t kmax = 0;
    for (size_t ri = 0; ri < reqs.size(); ri++) {
        const Request& r = *reqs[ri];
        const Session& ss = s->sessions[r.sid];
        for (uint32_t first = 0; first < r.n; first += 32u) {
            const uint32_t j = first / FA_SERVE_BLOCK_COLS, c = first % FA_SERVE_BLOCK_COLS;
            units[ss.cart].push_back(FaServeUnit{ ss.blocks[j] + c, (uint32_t)ri, first });
            unit_k[ss.cart].push_back(r.k);
        }
        act_bytes += align16((size_t)r.k * r.n);
        obs_bytes += r.obs ? (size_t)r.n * 128u : 0u;
        kmax = std::max(kmax, r.k);
    }
    size_t nunits = 0;
    for (auto& u : units) nunits += u.size();
    const size_t m = reqs.size();
    const size_t req_off = 0;
    const size_t rem_off = align16(m * sizeof(FaServeReq));
    const size_t unit_off = align16(rem_off + m * sizeof(uint32_t));
    const size_t act_off = align16(unit_off + nunits * sizeof(FaServeUnit));
    const size_t stage_bytes = act_off + act_bytes;
    int rc = grow_pinned(&sl.h_stage, &sl.d_stage, &sl.stage_cap, stage_bytes);
    if (rc) return rc;
    sl.flags_bytes = (m * sizeof(uint32_t) + 127u) & ~(size_t)127u;
    rc = grow_mapped(&sl.h_out, &sl.dh_out, &sl.out_cap, sl.flags_bytes + obs_bytes);
    if (rc) return rc;
    memset(sl.h_out, 0, sl.flags_bytes);

    // Tables and actions into the pinned staging buffer.
    FaServeReq* rt = (FaServeReq*)(sl.h_stage + req_off);
    uint32_t* rem = (uint32_t*)(sl.h_stage + rem_off);
    size_t ao = act_off, oo = 0;
    sl.obs_off.assign(m, 0);
    for (size_t ri = 0; ri < m; ri++) {
        const Request& r = *reqs[ri];
        const size_t ab = (size_t)r.k * r.n;
        memcpy(sl.h_stage + ao, r.actions.data(), ab);
        rem[ri] = (r.n + 31u) / 32u;
        rt[ri].actions = sl.d_stage + ao;
        rt[ri].obs = r.obs ? sl.dh_out + sl.flags_bytes + oo : nullptr;
        rt[ri].n = r.n;
        rt[ri].k = r.k;
        rt[ri].sched = (uint32_t)s->cfg.sched;
        rt[ri].pad = 0;
        sl.obs_off[ri] = oo;
        ao += align16(ab);
        oo += r.obs ? (size_t)r.n * 128u : 0u;
    }
    std::vector<size_t> cart_unit0(ncarts, 0);
    {
        FaServeUnit* ut = (FaServeUnit*)(sl.h_stage + unit_off);
        size_t u0 = 0;
        for (size_t g = 0; g < ncarts; g++) {
            cart_unit0[g] = u0;
            if (!units[g].empty()) memcpy(ut + u0, units[g].data(), units[g].size() * sizeof(FaServeUnit));
            u0 += units[g].size();
        }
    }

    FA_CUDA(cudaMemsetAsync(sl.d_scratch, 0, kScratch, sl.main));
    FA_CUDA(cudaMemcpyAsync(sl.d_stage, sl.h_stage, stage_bytes, cudaMemcpyHostToDevice, sl.main));
    for (const ReqP& r : reqs) {
        const Cart& c = s->carts[s->sessions[r->sid].cart];
        for (uint32_t* b : r->fresh)
            FA_CUDA(cudaMemcpyAsync(b, c.d_block_img, kBlockBytes, cudaMemcpyDeviceToDevice, sl.main));
    }
    auto make_launch = [&](size_t g, uint32_t n_units, uint32_t per_frame, uint32_t frame) {
        FaServeLaunch L;
        memset(&L, 0, sizeof(L));
        const Cart& c = s->carts[g];
        L.rom = c.h->d_rom;
        L.nbanks = c.nbanks;
        L.hot_lo = c.hot_lo;
        L.req = (const FaServeReq*)(sl.d_stage + req_off);
        L.unit = (const FaServeUnit*)(sl.d_stage + unit_off) + cart_unit0[g];
        L.nunits = n_units;
        L.per_frame = per_frame;
        L.frame = frame;
        if (!plain) {
            L.remaining = (uint32_t*)(sl.d_stage + rem_off);
            L.done = (uint32_t*)sl.dh_out;
        }
        L.err = (uint32_t*)sl.d_scratch;
        L.instr = (unsigned long long*)(sl.d_scratch + 8);
        L.rounds = (unsigned long long*)(sl.d_scratch + 16);
        return L;
    };
    unsigned long long launches = 0;
    if (plain) {
        // One launch per frame per cart, in order on one stream.
        for (uint32_t f = 0; f < kmax; f++) {
            for (size_t g = 0; g < ncarts; g++) {
                uint32_t nu = 0;
                while (nu < unit_k[g].size() && unit_k[g][nu] > f) nu++;
                if (!nu) continue;
                FA_CUDA(fa_launch_serve(make_launch(g, nu, 1, f), (int)B, sl.main));
                launches++;
            }
        }
    } else {
        FA_CUDA(cudaEventRecord(sl.ev_ready, sl.main));
        for (size_t g = 0; g < ncarts; g++) {
            if (units[g].empty()) continue;
            FA_CUDA(cudaStreamWaitEvent(sl.cs[g], sl.ev_ready, 0));
            FA_CUDA(fa_launch_serve(make_launch(g, (uint32_t)units[g].size(), 0, 0), (int)B, sl.cs[g]));
            FA_CUDA(cudaEventRecord(sl.ev_cart[g], sl.cs[g]));
            FA_CUDA(cudaStreamWaitEvent(sl.main, sl.ev_cart[g], 0));
            launches++;
        }
    }
    FA_CUDA(cudaMemcpyAsync(sl.h_scratch, sl.d_scratch, kScratch, cudaMemcpyDeviceToHost, sl.main));
    FA_CUDA(cudaEventRecord(sl.ev_done, sl.main));

    const auto now = Clock::now();
    for (const ReqP& r : reqs) {
        r->t_dispatch = now;
        r->batch = (uint32_t)reqs.size();
        r->fresh.clear();
    }
    sl.reqs = reqs;
    sl.req_done.assign(m, 0);
    sl.open_reqs = m;
    sl.busy = true;
    s->st.dispatches++;
    s->st.launches += launches;
    s->st.dispatched_requests += reqs.size();
    return FA_OK;
}

// Take the head request of every idle session, admit in arrival order
// (FIFO: once one admission waits, every later one waits too) and dispatch
// over the free slots.
void dispatch_ready(fa_server* s)
{
    std::vector<int> free_slots;
    for (int i = 0; i < (int)s->slots.size(); i++)
        if (!s->slots[i].busy) free_slots.push_back(i);
    if (free_slots.empty()) return;
    std::vector<std::pair<uint64_t, int64_t>> heads;
    for (auto& kv : s->sessions)
        if (!kv.second.busy && !kv.second.pending.empty())
            heads.emplace_back(kv.second.pending.front()->ticket, kv.first);
    if (heads.empty()) return;
    std::sort(heads.begin(), heads.end());
    std::vector<ReqP> batch;
    bool blocked = false;
    for (auto& h : heads) {
        Session& ss = s->sessions[h.second];
        ReqP r = ss.pending.front();
        const uint32_t want = blocks_for(r->n);
        const uint32_t need = want > ss.blocks.size() ? want - (uint32_t)ss.blocks.size() : 0u;
        if (need) {
            if (blocked || s->blocks_used + need > s->budget_blocks) {
                if (!r->waited_admission) {
                    r->waited_admission = true;
                    s->st.admission_waits++;
                }
                blocked = true;
                continue;
            }
            for (uint32_t i = 0; i < need; i++) {
                uint32_t* b = alloc_block(s);
                if (!b) break;
                r->fresh.push_back(b);
            }
            if (r->fresh.size() != need) {
                // The device ran out of memory below the budget: the blocks
                // taken so far go back and the request fails.
                for (uint32_t* b : r->fresh) s->free_blocks.push_back(b);
                s->blocks_used -= r->fresh.size();
                r->fresh.clear();
                ss.pending.pop_front();
                finish_request(s, r, FA_ERR_CUDA);
                s->cv_done.notify_all();
                continue;
            }
            ss.blocks.insert(ss.blocks.end(), r->fresh.begin(), r->fresh.end());
        }
        ss.size = std::max(ss.size, r->n);
        ss.pending.pop_front();
        ss.busy = true;
        r->t_ready = std::max(r->t_submit, ss.t_free);
        batch.push_back(r);
    }
    if (batch.empty()) return;
    // Batched mode: spread a large batch over several free slots by frame
    // count, so that sessions whose requests are short come back sooner.
    size_t parts = 1;
    if (s->cfg.mode == FA_SERVE_BATCHED)
        parts = std::min<size_t>({ free_slots.size(), (batch.size() + 7) / 8, (size_t)4 });
    std::stable_sort(batch.begin(), batch.end(), [](const ReqP& a, const ReqP& b) { return a->k > b->k; });
    const size_t per = (batch.size() + parts - 1) / parts;
    for (size_t p = 0; p < parts; p++) {
        const size_t b0 = p * per, b1 = std::min(batch.size(), b0 + per);
        if (b0 >= b1) break;
        std::vector<ReqP> part(batch.begin() + b0, batch.begin() + b1);
        int rc = launch_slot(s, free_slots[p], part);
        if (rc) {
            fail_server(s, rc, fa_last_error());
            for (const ReqP& r : part) finish_request(s, r, rc);
            s->cv_done.notify_all();
        }
    }
}

// Completes requests whose flag is up and slots whose launches finished.
void poll_slots(fa_server* s)
{
    bool any_done = false;
    for (Slot& sl : s->slots) {
        if (!sl.busy) continue;
        if (s->cfg.mode == FA_SERVE_BATCHED && sl.open_reqs) {
            const volatile uint32_t* flags = (const volatile uint32_t*)sl.h_out;
            for (size_t i = 0; i < sl.reqs.size(); i++) {
                if (sl.req_done[i]) continue;
                const uint32_t f = flags[i];
                if (!f) continue;
                std::atomic_thread_fence(std::memory_order_acquire);   // flag before observations
                complete_request(s, sl, i, f == 1u ? FA_OK : FA_ERR_KERNEL);
                any_done = true;
            }
        }
        cudaError_t e = cudaEventQuery(sl.ev_done);
        if (e == cudaSuccess) {
            release_slot(s, sl, FA_OK);
            any_done = true;
        } else if (e != cudaErrorNotReady) {
            fail_server(s, FA_ERR_CUDA, cudaGetErrorString(e));
            release_slot(s, sl, FA_ERR_CUDA);
            any_done = true;
        }
    }
    if (any_done) s->cv_done.notify_all();
}

// Fail every request not yet dispatched (sessions may be released meanwhile,
// so the requests are collected before any is finished).
void fail_pending(fa_server* s, int code)
{
    std::vector<ReqP> rs;
    for (auto& kv : s->sessions) {
        for (const ReqP& r : kv.second.pending) rs.push_back(r);
        kv.second.pending.clear();
    }
    for (const ReqP& r : rs) finish_request(s, r, code);
    s->cv_done.notify_all();
}

void engine_main(fa_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        poll_slots(s);
        if (s->fatal == FA_OK) dispatch_ready(s);
        bool inflight = false;
        for (const Slot& sl : s->slots) inflight |= sl.busy;
        if (s->stop && !inflight) break;
        if (!inflight && s->fatal != FA_OK) fail_pending(s, s->fatal);   // nothing can run any more
        if (inflight) s->cv_engine.wait_for(lk, std::chrono::microseconds(20));
        else s->cv_engine.wait(lk);
    }
    // Stopping with nothing on the GPU: requests that could not be admitted fail.
    fail_pending(s, FA_ERR_CAPACITY);
}

void free_server(fa_server* s)
{
    cudaSetDevice(s->device);
    for (Slot& sl : s->slots) {
        if (sl.main) cudaStreamSynchronize(sl.main);
        for (cudaStream_t c : sl.cs) if (c) { cudaStreamSynchronize(c); cudaStreamDestroy(c); }
        for (cudaEvent_t e : sl.ev_cart) if (e) cudaEventDestroy(e);
        if (sl.ev_ready) cudaEventDestroy(sl.ev_ready);
        if (sl.ev_done) cudaEventDestroy(sl.ev_done);
        if (sl.main) cudaStreamDestroy(sl.main);
        cudaFreeHost(sl.h_stage);
        cudaFree(sl.d_stage);
        cudaFreeHost(sl.h_out);
        cudaFree(sl.d_scratch);
        cudaFreeHost(sl.h_scratch);
    }
    for (void* p : s->slabs) cudaFree(p);
    for (Cart& c : s->carts) {
        cudaFree(c.d_block_img);
        fa_destroy(c.h);
    }
    delete s;
}

}  // namespace

extern "C" int fa_server_create(const uint8_t* const* roms, const size_t* rom_lens, int ncarts,
                                const fa_server_config* cfg, fa_server** out)
{
    if (!out) return fa_fail(FA_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!roms || !rom_lens || ncarts < 1 || ncarts > FA_MAX_GROUPS)
        return fa_fail(FA_ERR_INVALID, "a server holds 1..%d carts", FA_MAX_GROUPS);
    if (fa_device_count() < 1) return fa_fail(FA_ERR_NO_DEVICE, "no CUDA device visible");
    fa_server_config c{};
    c.sched = FA_SCHED_PC;
    if (cfg) c = *cfg;
    if (c.mode != FA_SERVE_BATCHED && c.mode != FA_SERVE_PLAIN) return fa_fail(FA_ERR_INVALID, "bad mode %d", c.mode);
    if (c.state_budget_bytes == 0) c.state_budget_bytes = (size_t)64 << 30;
    if (c.block == 0) c.block = c.mode == FA_SERVE_PLAIN ? 128 : 512;
    if (c.block != 128 && c.block != 256 && c.block != 512)
        return fa_fail(FA_ERR_INVALID, "block must be 128, 256 or 512");
    if (c.max_inflight == 0) c.max_inflight = 32;
    if (c.mode == FA_SERVE_PLAIN) c.max_inflight = 1;
    if (c.max_inflight < 1 || c.max_inflight > kMaxSlots)
        return fa_fail(FA_ERR_INVALID, "max_inflight must be 1..%d", kMaxSlots);
    if (c.sched < FA_SCHED_LANE || c.sched > FA_SCHED_MATCH) return fa_fail(FA_ERR_INVALID, "bad sched %d", c.sched);
    if (c.state_budget_bytes / kBlockBytes == 0)
        return fa_fail(FA_ERR_INVALID, "state budget below one block (%zu bytes)", kBlockBytes);

    fa_server* s = new (std::nothrow) fa_server();
    if (!s) return fa_fail(FA_ERR_CAPACITY, "out of host memory");
    s->cfg = c;
    s->budget_blocks = c.state_budget_bytes / kBlockBytes;
    cudaGetDevice(&s->device);
    std::vector<uint32_t> img(kBlockWords);
    for (int g = 0; g < ncarts; g++) {
        Cart cart;
        int rc = fa_create(roms[g], rom_lens[g], 1, &cart.h);
        if (!rc) rc = fa_reset(cart.h, nullptr);
        if (rc) {
            fa_destroy(cart.h);
            free_server(s);
            return rc;
        }
        cart.nbanks = cart.h->nbanks;
        cart.hot_lo = cart.h->hot_lo;
        cart.scheme = cart.h->scheme;
        // The post-reset column (HeadlessAtari::new + one frame, computed on
        // the device by fa_reset), replicated into every column of a block.
        uint32_t snap[FA_ROWS];
        cudaError_t e = cudaMemcpy(snap, cart.h->d_snap, sizeof(snap), cudaMemcpyDeviceToHost);
        for (uint32_t w = 0; w < FA_ROWS; w++)
            for (uint32_t col = 0; col < FA_SERVE_BLOCK_COLS; col++) img[(size_t)w * FA_SERVE_BLOCK_COLS + col] = snap[w];
        if (e == cudaSuccess) e = cudaMalloc(&cart.d_block_img, kBlockBytes);
        if (e == cudaSuccess) e = cudaMemcpy(cart.d_block_img, img.data(), kBlockBytes, cudaMemcpyHostToDevice);
        s->carts.push_back(cart);
        if (e != cudaSuccess) {
            free_server(s);
            return fa_fail(FA_ERR_CUDA, "server cart setup: %s", cudaGetErrorString(e));
        }
    }
    s->slots.resize(c.max_inflight);
    for (Slot& sl : s->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.main, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_done, cudaEventDisableTiming);
        sl.cs.assign(ncarts, nullptr);
        sl.ev_cart.assign(ncarts, nullptr);
        for (int g = 0; g < ncarts && e == cudaSuccess; g++) {
            e = cudaStreamCreateWithFlags(&sl.cs[g], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev_cart[g], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            free_server(s);
            return fa_fail(FA_ERR_CUDA, "server streams: %s", cudaGetErrorString(e));
        }
        int rc = grow_pinned(&sl.h_stage, &sl.d_stage, &sl.stage_cap, (size_t)512 << 10);
        if (!rc) rc = grow_mapped(&sl.h_out, &sl.dh_out, &sl.out_cap, (size_t)4 << 20);
        if (!rc && (cudaMalloc(&sl.d_scratch, kScratch) != cudaSuccess ||
                    cudaMallocHost(&sl.h_scratch, kScratch) != cudaSuccess))
            rc = fa_fail(FA_ERR_CUDA, "server scratch allocation failed");
        if (rc) {
            free_server(s);
            return rc;
        }
    }
    s->st.state_budget_bytes = s->budget_blocks * kBlockBytes;
    s->engine = std::thread(engine_main, s);
    *out = s;
    return FA_OK;
}

extern "C" void fa_server_destroy(fa_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_engine.notify_all();
    if (s->engine.joinable()) s->engine.join();
    free_server(s);
}

extern "C" int fa_server_open(fa_server* s, int cart, int64_t* session)
{
    if (!s || !session) return fa_fail(FA_ERR_INVALID, "null argument");
    if (cart < 0 || cart >= (int)s->carts.size()) return fa_fail(FA_ERR_INVALID, "bad cart %d", cart);
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t sid = s->next_sid++;
    Session ss;
    ss.cart = cart;
    s->sessions.emplace(sid, std::move(ss));
    s->st.sessions_open++;
    *session = sid;
    return FA_OK;
}

extern "C" int fa_server_close(fa_server* s, int64_t session)
{
    if (!s) return fa_fail(FA_ERR_INVALID, "null server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->sessions.find(session);
        if (it == s->sessions.end() || it->second.closing)
            return fa_fail(FA_ERR_INVALID, "no open session %lld", (long long)session);
        it->second.closing = true;
        s->st.sessions_open--;
        if (!it->second.busy && it->second.pending.empty()) release_session(s, session);
    }
    s->cv_engine.notify_one();
    return FA_OK;
}

extern "C" int fa_server_submit(fa_server* s, int64_t session, const uint8_t* actions, uint32_t n, int k,
                                uint8_t* obs, uint64_t* ticket)
{
    const auto t0 = Clock::now();
    if (!s || !actions || !ticket) return fa_fail(FA_ERR_INVALID, "null argument");
    if (n < 1 || k < 1) return fa_fail(FA_ERR_INVALID, "need n >= 1 and k >= 1");
    auto r = std::make_shared<Request>();
    r->sid = session;
    r->n = n;
    r->k = (uint32_t)k;
    r->obs = obs;
    r->actions.assign(actions, actions + (size_t)k * n);
    r->t_submit = t0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->fatal != FA_OK) return fa_fail(s->fatal, "server failed: %s", s->fatal_msg.c_str());
        if (s->stop) return fa_fail(FA_ERR_INVALID, "server is stopping");
        auto it = s->sessions.find(session);
        if (it == s->sessions.end() || it->second.closing)
            return fa_fail(FA_ERR_INVALID, "no open session %lld", (long long)session);
        if (blocks_for(n) > s->budget_blocks)
            return fa_fail(FA_ERR_CAPACITY, "%u instances exceed the state budget (%zu bytes)", n,
                           s->budget_blocks * kBlockBytes);
        r->ticket = s->next_ticket++;
        it->second.pending.push_back(r);
        s->tickets.emplace(r->ticket, r);
        s->st.requests_submitted++;
        *ticket = r->ticket;
    }
    s->cv_engine.notify_one();
    return FA_OK;
}

extern "C" int fa_server_wait(fa_server* s, uint64_t ticket, int timeout_ms, fa_request_info* info)
{
    if (!s) return fa_fail(FA_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fa_fail(FA_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    ReqP r = it->second;
    auto done = [&] { return r->done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, done);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        return fa_fail(FA_ERR_TIMEOUT, "ticket %llu not done after %d ms", (unsigned long long)ticket, timeout_ms);
    }
    s->tickets.erase(ticket);
    if (info) {
        info->status = r->status;
        info->latency_ms = ms_between(r->t_submit, r->t_done);
        const bool sent = r->t_dispatch.time_since_epoch().count() != 0;
        info->queue_ms = sent ? ms_between(r->t_submit, r->t_dispatch) : 0.0;
        info->session_wait_ms = sent ? ms_between(r->t_submit, r->t_ready) : 0.0;
        info->service_ms = sent ? ms_between(r->t_dispatch, r->t_done) : 0.0;
        info->batch_requests = r->batch;
        info->waited_admission = r->waited_admission ? 1 : 0;
    }
    if (r->status != FA_OK) return fa_fail(r->status, "request %llu failed", (unsigned long long)ticket);
    return FA_OK;
}

extern "C" int fa_server_step(fa_server* s, int64_t session, const uint8_t* actions, uint32_t n, int k,
                              uint8_t* obs, fa_request_info* info)
{
    uint64_t t = 0;
    int rc = fa_server_submit(s, session, actions, n, k, obs, &t);
    if (rc) return rc;
    return fa_server_wait(s, t, -1, info);
}

extern "C" int fa_server_session_size(fa_server* s, int64_t session, uint32_t* size)
{
    if (!s || !size) return fa_fail(FA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->sessions.find(session);
    if (it == s->sessions.end()) return fa_fail(FA_ERR_INVALID, "no session %lld", (long long)session);
    *size = it->second.size;
    return FA_OK;
}

extern "C" int fa_server_get_states(fa_server* s, int64_t session, uint32_t first, uint32_t count, fa_state* out)
{
    if (!s || (!out && count)) return fa_fail(FA_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->sessions.find(session);
    if (it == s->sessions.end() || it->second.closing)
        return fa_fail(FA_ERR_INVALID, "no open session %lld", (long long)session);
    s->cv_done.wait(lk, [&] {
        auto j = s->sessions.find(session);
        return j == s->sessions.end() || (!j->second.busy && j->second.pending.empty()) || s->fatal != FA_OK;
    });
    it = s->sessions.find(session);
    if (it == s->sessions.end()) return fa_fail(FA_ERR_INVALID, "session %lld closed", (long long)session);
    if (s->fatal != FA_OK) return fa_fail(s->fatal, "server failed: %s", s->fatal_msg.c_str());
    const Session& ss = it->second;
    if ((uint64_t)first + count > ss.size)
        return fa_fail(FA_ERR_INVALID, "instances [%u, %u) beyond the session's %u", first, first + count, ss.size);
    FA_CUDA(cudaSetDevice(s->device));
    std::vector<uint32_t> host(kBlockWords);
    uint32_t cur = UINT32_MAX;
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t idx = first + i, j = idx / FA_SERVE_BLOCK_COLS;
        if (j != cur) {
            FA_CUDA(cudaMemcpy(host.data(), ss.blocks[j], kBlockBytes, cudaMemcpyDeviceToHost));
            cur = j;
        }
        fa_unpack_column(host.data() + idx % FA_SERVE_BLOCK_COLS, FA_SERVE_BLOCK_COLS, s->carts[ss.cart].scheme, out[i]);
    }
    return FA_OK;
}

extern "C" int fa_server_stats_get(fa_server* s, fa_server_stats* out)
{
    if (!s || !out) return fa_fail(FA_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->state_bytes_in_use = s->blocks_used * kBlockBytes;
    out->state_bytes_peak = s->blocks_peak * kBlockBytes;
    out->state_budget_bytes = s->budget_blocks * kBlockBytes;
    return FA_OK;
}

// ------------------------------------------------------------------ load generator
namespace {

inline uint64_t splitmix64(uint64_t& x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double unit01(uint64_t& x) { return (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0); }

struct TraceReq {
    double t;              // arrival, seconds from the start
    int client, cart;
    uint32_t n, k;
    std::vector<uint8_t> actions;
};

}  // namespace

extern "C" int fa_server_loadgen(fa_server* s, const fa_loadgen_config* cfg, fa_loadgen_result* out,
                                 fa_loadgen_record* records)
{
    if (!s || !cfg || !out) return fa_fail(FA_ERR_INVALID, "null argument");
    const int ncarts = (int)s->carts.size();
    const fa_loadgen_config& c = *cfg;
    if (c.clients < 1 || c.requests < 1 || c.k_min < 1 || c.k_max < c.k_min || c.batch_min < 1 ||
        c.batch_max < c.batch_min || c.batch_median < 1 || !(c.batch_sigma >= 0.0))
        return fa_fail(FA_ERR_INVALID, "bad load generator configuration");
    // The trace: a Poisson process (the superposition of the clients' own)
    // whose requests pick a client and a cart uniformly, a batch size
    // lognormal(median, sigma) clipped to [min, max] and k uniform in
    // [k_min, k_max]; actions are uniform over the 18 joystick actions.
    std::vector<TraceReq> tr(c.requests);
    uint64_t rng = c.seed * 0x2545F4914F6CDD1Dull + 1u;
    double t = 0.0, work = 0.0, insts = 0.0;
    for (int i = 0; i < c.requests; i++) {
        TraceReq& q = tr[i];
        t += -std::log(1.0 - unit01(rng));
        q.t = t;
        q.client = (int)(splitmix64(rng) % (uint64_t)c.clients);
        q.cart = (int)(splitmix64(rng) % (uint64_t)ncarts);
        const double u1 = unit01(rng), u2 = unit01(rng);
        const double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
        double b = std::exp(std::log((double)c.batch_median) + c.batch_sigma * z);
        b = std::min((double)c.batch_max, std::max((double)c.batch_min, std::round(b)));
        q.n = (uint32_t)b;
        q.k = (uint32_t)(c.k_min + (int)(splitmix64(rng) % (uint64_t)(c.k_max - c.k_min + 1)));
        q.actions.resize((size_t)q.n * q.k);
        uint64_t ar = c.seed ^ (0xA5A5A5A5ull + (uint64_t)i * 0x9E3779B97F4A7C15ull);
        for (auto& a : q.actions) a = (uint8_t)(splitmix64(ar) % FA_NUM_ACTIONS);
        work += (double)q.n * q.k;
        insts += q.n;
    }
    // Scale arrival times so the trace offers `offered_frames_per_s`
    // instance-frames per second; 0 submits everything at once (saturation).
    const double scale = c.offered_frames_per_s > 0.0 ? (work / c.requests) / c.offered_frames_per_s : 0.0;
    for (auto& q : tr) q.t *= scale;

    std::vector<int64_t> sid((size_t)c.clients * ncarts, 0);
    for (int cl = 0; cl < c.clients; cl++)
        for (int g = 0; g < ncarts; g++) {
            int rc = fa_server_open(s, g, &sid[(size_t)cl * ncarts + g]);
            if (rc) return rc;
        }
    std::vector<uint64_t> tickets(c.requests, 0);
    std::vector<double> t_sub(c.requests, 0.0);
    std::vector<std::unique_ptr<uint8_t[]>> obs(c.requests);
    std::vector<fa_request_info> info(c.requests);
    std::mutex mu;
    std::condition_variable cv;
    int submitted = 0, submit_err = FA_OK;
    Clock::time_point t_end;
    int errors = 0;
    std::thread collector([&] {
        for (int i = 0; i < c.requests; i++) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return submitted > i || submit_err != FA_OK; });
                if (submitted <= i) break;
            }
            int rc = fa_server_wait(s, tickets[i], -1, &info[i]);
            if (rc) errors++;
            obs[i].reset();
        }
        t_end = Clock::now();
    });
    const auto t0 = Clock::now();
    for (int i = 0; i < c.requests; i++) {
        const TraceReq& q = tr[i];
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(q.t));
        // Sleep most of the gap, spin the last 200 us for a precise arrival.
        while (true) {
            const auto now = Clock::now();
            if (now >= due) break;
            if (due - now > std::chrono::microseconds(300)) std::this_thread::sleep_for(due - now - std::chrono::microseconds(200));
        }
        obs[i].reset(new uint8_t[(size_t)q.n * 128u]);
        t_sub[i] = std::chrono::duration<double>(Clock::now() - t0).count();
        uint64_t tk = 0;
        int rc = fa_server_submit(s, sid[(size_t)q.client * ncarts + q.cart], q.actions.data(), q.n, (int)q.k,
                                  obs[i].get(), &tk);
        std::lock_guard<std::mutex> lk(mu);
        if (rc) { submit_err = rc; break; }
        tickets[i] = tk;
        submitted = i + 1;
        cv.notify_one();
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        cv.notify_one();
    }
    collector.join();
    for (int64_t id : sid) fa_server_close(s, id);
    if (submit_err != FA_OK) return fa_fail(submit_err, "load generator: submit failed");

    std::vector<double> lat(c.requests);
    double sum = 0.0, qsum = 0.0, bsum = 0.0;
    unsigned long long waited = 0;
    for (int i = 0; i < c.requests; i++) {
        lat[i] = info[i].latency_ms;
        if (records) {
            fa_loadgen_record& rec = records[i];
            rec.cart = (uint32_t)tr[i].cart;
            rec.n = tr[i].n;
            rec.k = tr[i].k;
            rec.batch_requests = info[i].batch_requests;
            rec.arrival_s = t_sub[i];
            rec.latency_ms = info[i].latency_ms;
            rec.session_wait_ms = info[i].session_wait_ms;
            rec.dispatch_ms = info[i].queue_ms - info[i].session_wait_ms;
            rec.service_ms = info[i].service_ms;
        }
        sum += info[i].latency_ms;
        qsum += info[i].queue_ms;
        bsum += info[i].batch_requests;
        waited += info[i].waited_admission;
    }
    // Steady-state completion rate: instance-frames of the requests that
    // complete between the 10th and the 60th percentile of completion times,
    // over that span (the run's start and its tail, where only the sessions
    // with the most work remain, are left out).
    std::vector<std::pair<double, double>> done_at(c.requests);
    for (int i = 0; i < c.requests; i++)
        done_at[i] = { t_sub[i] + info[i].latency_ms * 1e-3, (double)tr[i].n * tr[i].k };
    std::sort(done_at.begin(), done_at.end());
    const size_t i10 = (size_t)(0.10 * (c.requests - 1)), i60 = (size_t)(0.60 * (c.requests - 1));
    double steady_work = 0.0;
    for (size_t i = i10 + 1; i <= i60; i++) steady_work += done_at[i].second;
    const double steady_span = done_at[i60].first - done_at[i10].first;
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) { return lat[std::min((size_t)c.requests - 1, (size_t)std::llround(q * (c.requests - 1)))]; };
    memset(out, 0, sizeof(*out));
    out->requests = (unsigned long long)c.requests;
    out->instances = insts;
    out->instance_frames = work;
    out->elapsed_s = std::chrono::duration<double>(t_end - t0).count();
    out->frames_per_s = work / out->elapsed_s;
    out->steady_frames_per_s = steady_span > 0.0 ? steady_work / steady_span : out->frames_per_s;
    out->offered_frames_per_s = c.offered_frames_per_s;
    out->arrival_window_s = tr.back().t;
    out->p50_ms = pct(0.50);
    out->p90_ms = pct(0.90);
    out->p99_ms = pct(0.99);
    out->max_ms = lat.back();
    out->mean_ms = sum / c.requests;
    out->mean_queue_ms = qsum / c.requests;
    out->mean_batch_requests = bsum / c.requests;
    out->admission_waits = waited;
    out->errors = errors;
    return errors ? fa_fail(FA_ERR_KERNEL, "load generator: %d requests failed", errors) : FA_OK;
}
