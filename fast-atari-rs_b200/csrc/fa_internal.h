// fa_internal.h — host/device launch descriptors shared by the library files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "fa_layout.h"

#include <string>

// Device error word bits.
#define FA_DEVERR_TMA_TIMEOUT 0x1u

#define FA_MAX_GROUPS 16
// Calls one fa_step_static may chain (one queue counter each in its fixed scratch).
#define FA_STATIC_MAX_CALLS 1024
// Dynamic shared memory a CTA may use (227 KiB opt-in limit minus the static
// barrier word and headroom).
#define FA_SMEM_PER_CTA_MAX (227 * 1024 - 1024)

// One cart's instance set in a launch.
struct FaGroup {
    const uint8_t* rom;          // nbanks * 4 KiB bank image (16-byte aligned)
    const uint32_t* snapshot;    // FA_ROWS-word post-reset column, or null
    uint32_t* state;             // SoA rows: state[w * stride + i]
    const uint8_t* actions;      // actions[f * act_stride + i], or null (inputs unchanged)
    uint8_t* obs;                // n * 128 bytes (16-byte aligned), or null
    uint32_t stride, n, act_stride;
    uint32_t nbanks, hot_lo;
    uint32_t k;                  // frames to run per instance
    uint32_t episode_frames;     // 0 = no periodic reset
    uint32_t sched;              // FA_SCHED_*
    uint32_t unit_begin;         // first work unit of this group (set by fa_launch_run)
    uint32_t rom_off;            // offset of the ROM in the shared-memory library (set by fa_launch_run)
    uint32_t rom_owner;          // 1 if this group stages the ROM (set by fa_launch_run)
    uint32_t tag;                // the caller's number for the group (a pool's group index), in unit traces
};

// The kernel build a set of groups needs (FA_MAPS_*).
static inline int fa_maps_of(const FaGroup* g, uint32_t ngroups)
{
    bool sl = false, dpc = false, fe = false, std4k = false;
    for (uint32_t i = 0; i < ngroups; i++) {
        const uint32_t kind = fa_map_kind(g[i].hot_lo);
        (kind == FA_MAP_DPC ? dpc : kind == FA_MAP_FE ? fe : kind ? sl : std4k) = true;
    }
    if ((int)sl + (int)dpc + (int)fe + (int)std4k > 1) return FA_MAPS_BOTH;
    return dpc ? FA_MAPS_DPC : fe ? FA_MAPS_FE : sl ? FA_MAPS_SLICED : FA_MAPS_4K;
}

struct FaLaunch {
    FaGroup g[FA_MAX_GROUPS];
    uint32_t ngroups;
    uint32_t nunits;
    uint32_t rom_bytes_max;      // shared-memory ROM bytes reserved per CTA (CTA-granular form)
    uint32_t romlib_bytes;       // all ROMs of the launch (warp-granular form, set by fa_launch_run)
    uint32_t cta_warps;          // persistent form: warps per CTA cap (0 = as many as fit)
    uint32_t* queue;             // work-queue counter (persistent form) or null
    uint32_t* err;               // device error word
    unsigned long long* instr;   // guest-instruction counter, or null
    unsigned long long* rounds;  // scheduler rounds x 32 (lane slots offered), or null
    uint64_t wait_ns;            // bound of the ROM staging wait (set by fa_launch_run)
    unsigned long long* trace;   // per work unit: start ns, end ns, smid << 32 | warp << 16 | tag, or null
    uint32_t trace_cap;          // units the trace holds
    const uint32_t* first_wave;  // warp-granular persistent form: the unit of each warp's first round
                                 // (index warp * grid + cta; ~0 for none), or null for warp * grid + cta
};

// The launch shape fa_launch_run would use for L (warp-granular form only):
// grid CTAs of `warps` warps, `per_sm` CTAs resident per SM.  Returns false
// for the CTA-granular form.
bool fa_launch_warp_shape(const FaLaunch& L, int block, bool persistent, int sms, uint32_t* grid, uint32_t* warps,
                          int* per_sm);

// The first-wave plan of a persistent warp-granular launch with one CTA per
// SM: units [0, min(nunits, grid * warps)) placed on warp slots so that the
// summed cost per SM sub-partition (warp w of a CTA issues from scheduler
// w % 4) is as even as longest-processing-time-first makes it.  unit_cost is
// non-increasing; table gets grid * warps entries (index warp * grid + cta).
void fa_plan_first_wave(const float* unit_cost, uint32_t nunits, uint32_t grid, uint32_t warps, uint32_t* table);

// The bound in nanoseconds that launches give their ROM staging wait
// (fa_set_wait_limit_ns; 2 s by default).
uint64_t fa_wait_limit_ns();

// ------------------------------------------------------------------ serving form
// Instance state of the server lives in blocks of FA_SERVE_BLOCK_COLS columns
// (row w of column c of a block at block[w * FA_SERVE_BLOCK_COLS + c]); a
// session's instances are a list of such blocks, so it grows without moving.
#define FA_SERVE_BLOCK_COLS 256u

// One request of a serving launch (device table).
struct FaServeReq {
    const uint8_t* actions;      // k * n bytes, frame-major (actions[f * n + i])
    uint8_t* obs;                // n * 128 bytes, or null
    uint32_t n, k, sched, pad;
};

// One warp of a serving launch (device table): up to 32 consecutive
// instances of one request, all inside one state block.
struct FaServeUnit {
    uint32_t* state;             // first column of the unit (row stride FA_SERVE_BLOCK_COLS)
    uint32_t req;                // request index in the launch's table
    uint32_t first;              // index of the unit's first instance within the request
};

// A serving launch: every unit belongs to one cart (ROM staged per CTA).
// per_frame != 0 runs frame `frame` of every request only (the plain form:
// actions of that frame, observations only after the request's last frame).
// With `done` set, completion is signalled per request: remaining[r] counts
// the request's warp units still running; the
// last one sets done[r] (host-mapped) to 1, or 2 if a unit failed.
struct FaServeLaunch {
    const uint8_t* rom;
    uint32_t nbanks, hot_lo;
    const FaServeReq* req;
    const FaServeUnit* unit;
    uint32_t nunits;
    uint32_t per_frame, frame;
    uint32_t* remaining;         // device, one counter per request, or null
    uint32_t* done;              // host-mapped, one flag per request, or null
    uint32_t* err;
    unsigned long long* instr;
    unsigned long long* rounds;
    uint64_t wait_ns;            // bound of the ROM staging wait (set by fa_launch_serve)
};

// Launch fa_serve with CTAs of block / 32 warps (block 128, 256 or 512), one
// warp per unit.
cudaError_t fa_launch_serve(const FaServeLaunch& L, int block, cudaStream_t s);

// Launch fa_run.  For the persistent form the grid is the SM count times the
// CTAs per SM the occupancy calculator allows (cached per block and shared-
// memory size, so that the call is safe inside a stream capture).
cudaError_t fa_launch_run(const FaLaunch& L, int block, bool persistent, int sms, cudaStream_t s);
// Everything fa_launch_run does before launching (kernel choice, shared-memory
// attribute, occupancy), so that a later launch is safe inside a capture.
cudaError_t fa_launch_prepare(const FaLaunch& L, int block, bool persistent);
// CTAs of fa_run<block> resident per SM for this ROM size (-1 on error).
int fa_launch_occupancy(int block, uint32_t rom_bytes_max);
cudaError_t fa_launch_broadcast(uint32_t* state, uint32_t stride, uint32_t n, const uint32_t* col,
                                cudaStream_t s);

int fa_fail(int code, const char* fmt, ...);
// memcpy of a host-buffer call's outputs into the caller's memory, split over
// up to 8 threads when it is large (first-touch page faults included).
void fa_host_copy(void* dst, const void* src, size_t bytes);

#define FA_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fa_fail(FA_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

int fa_make_bank_image(const uint8_t* rom, size_t len, std::vector<uint8_t>& img, int& scheme,
                       uint32_t* nbanks = nullptr, uint32_t* hot_lo = nullptr);

// One ROM and its n instances resident in HBM (the C ABI's fa_handle).
struct fa_handle {
    int device = 0;
    int sms = 148;
    size_t n = 0;
    uint32_t stride = 0;
    int scheme = 0;
    uint32_t nbanks = 1, hot_lo = 0x2000;
    std::vector<uint8_t> image;        // host copy of the bank image
    uint8_t* d_rom = nullptr;
    uint32_t* d_state = nullptr;
    uint32_t* d_snap = nullptr;        // post-reset column (FA_ROWS words)
    bool have_snap = false;
    uint8_t* d_actions = nullptr;
    size_t actions_cap = 0;
    uint8_t* d_obs = nullptr;
    uint32_t* d_err = nullptr;         // [0] error word, [1] work-queue counter
    unsigned long long* d_instr = nullptr;
    uint8_t* h_actions = nullptr;      // pinned staging
    size_t h_actions_cap = 0;
    uint8_t* h_obs = nullptr;          // pinned, n*128
    uint8_t* h_obs_dev = nullptr;      // h_obs as the device addresses it (mapped), or null
    cudaStream_t stream = nullptr;
    int block = 128;
    int sched = FA_SCHED_PC;
    bool persistent = false;
    int cta_warps = 0;                 // persistent form: warps per CTA (0 = as many as fit)
    uint32_t episode_frames = 0;
    unsigned long long last_instr = 0;
    unsigned long long last_slots = 0;
};

// Enqueue one launch over every instance of the handle (fa_api.cu).
FaGroup fa_handle_group(fa_handle* h, const uint8_t* d_actions, uint32_t k, uint8_t* d_obs);

// Host packing between the fa_state AoS layout and one SoA column.
void fa_pack_column(const fa_state& s, uint32_t* col, size_t stride);
void fa_unpack_column(const uint32_t* col, size_t stride, int scheme, fa_state& s);
// Power-on state of HeadlessAtari::new (src/atari.rs:562-569) for a bank image.
void fa_power_on_column(const uint8_t* bank_image, uint32_t nbanks, int scheme, uint32_t hot_lo, uint32_t* col);
// The rendering console's power-on column: FA_RROWS words.
void fa_render_power_on_column(const uint8_t* image, uint32_t nbanks, int scheme, uint32_t hot_lo, uint32_t* col);
