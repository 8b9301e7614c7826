// fa_internal.h — host/device launch descriptors shared by the library files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fa_layout.h"

// Device error word bits.
#define FA_DEVERR_TMA_TIMEOUT 0x1u

#define FA_MAX_GROUPS 16

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
    uint32_t unit_begin;         // first work unit of this group
};

struct FaLaunch {
    FaGroup g[FA_MAX_GROUPS];
    uint32_t ngroups;
    uint32_t nunits;
    uint32_t rom_bytes_max;      // shared-memory ROM bytes reserved per CTA
    uint32_t* queue;             // work-queue counter (persistent form) or null
    uint32_t* err;               // device error word
    unsigned long long* instr;   // guest-instruction counter, or null
};

cudaError_t fa_launch_run(const FaLaunch& L, int block, bool persistent, int sms, cudaStream_t s);
int fa_launch_occupancy(int block, uint32_t rom_bytes_max);
cudaError_t fa_launch_broadcast(uint32_t* state, uint32_t stride, uint32_t n, const uint32_t* col,
                                cudaStream_t s);

// Host packing between the fa_state AoS layout and one SoA column.
void fa_pack_column(const fa_state& s, uint32_t* col, size_t stride);
void fa_unpack_column(const uint32_t* col, size_t stride, int scheme, fa_state& s);
// Power-on state of HeadlessAtari::new (src/atari.rs:562-569) for a bank image.
void fa_power_on_column(const uint8_t* bank_image, uint32_t nbanks, int scheme, uint32_t* col);
