// Test infrastructure: compiles the library's device core (fa_device.cuh,
// fa_run.cuh) with a host C++ compiler, so the CPU test suite can run the
// CUDA interpreter's own code against the oracle.  CUDA qualifiers vanish and
// the few intrinsics the core uses get host definitions.
#pragma once
#include <stdint.h>
#include <string.h>
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __noinline__
#define __constant__
#define __shared__
#define __grid_constant__
#define __launch_bounds__(x)
struct uint2 { uint32_t x, y; };
struct uint4 { uint32_t x, y, z, w; };
static inline uint2 make_uint2(uint32_t x, uint32_t y) { uint2 r{x, y}; return r; }
static inline uint4 make_uint4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) { uint4 r{x, y, z, w}; return r; }
static inline uint32_t __brev(uint32_t v) { uint32_t r = 0; for (int i = 0; i < 32; i++) if (v >> i & 1) r |= 1u << (31 - i); return r; }
static inline int __ffs(uint32_t v) { return v ? __builtin_ctz(v) + 1 : 0; }
static inline uint32_t __funnelshift_r(uint32_t lo, uint32_t hi, uint32_t sh) { sh &= 31; return sh ? (lo >> sh) | (hi << (32 - sh)) : lo; }
static inline uint32_t __byte_perm(uint32_t x, uint32_t y, uint32_t s) {
    uint8_t b[8]; memcpy(b, &x, 4); memcpy(b + 4, &y, 4); uint32_t r = 0;
    for (int i = 0; i < 4; i++) r |= (uint32_t)b[(s >> (4 * i)) & 7] << (8 * i); return r; }
// warp intrinsics and special registers: declared for parsing; the host
// runner drives one lane and never calls them
static inline uint32_t __cvta_generic_to_shared(const void* p) { return (uint32_t)(uintptr_t)p; }
uint32_t __shfl_sync(uint32_t, uint32_t, uint32_t);
uint32_t __shfl_xor_sync(uint32_t, uint32_t, uint32_t);
uint32_t __ballot_sync(uint32_t, bool);
bool __any_sync(uint32_t, bool);
bool __all_sync(uint32_t, bool);
uint32_t __match_any_sync(uint32_t, uint32_t);
uint32_t __reduce_min_sync(uint32_t, uint32_t);
unsigned long long atomicAdd(unsigned long long*, unsigned long long);
uint32_t atomicOr(uint32_t*, uint32_t);
struct { uint32_t x = 0; } static threadIdx;
