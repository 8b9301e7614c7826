// fa_env.cu — device side of the batched RL caller.
//
// BatchAtariGpuEnv (src/rl4burn_env.rs:269-380) turns the N x 128 RAM bytes
// into f32 observations b / 255 on the host (:320-322).  Here the conversion
// runs on the device into a caller buffer (e.g. a torch tensor), so a learner
// on the same GPU reads observations without a host round trip.  The
// division is the IEEE single-precision one, bit-identical to Rust's
// `b as f32 / 255.0`.
#include <cuda_runtime.h>

#include "../../include/fast_atari.h"
#include "fa_internal.h"

namespace {
__global__ void obs_to_unit_f32(const uint8_t* __restrict__ in, float* __restrict__ out, size_t count)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        out[i] = __fdiv_rn((float)in[i], 255.0f);
}
}  // namespace

extern "C" int fa_obs_to_unit_f32(const uint8_t* d_obs, float* d_out, size_t count, void* stream)
{
    if (!d_obs || !d_out) return fa_fail(FA_ERR_INVALID, "null buffer");
    if (count == 0) return FA_OK;
    size_t blocks = (count + 255) / 256;
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    obs_to_unit_f32<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_obs, d_out, count);
    FA_CUDA(cudaGetLastError());
    return FA_OK;
}
