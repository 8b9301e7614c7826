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

__global__ void obs_reward(const uint8_t* __restrict__ obs, size_t n, fa_reward_spec sp, int init,
                           int32_t* __restrict__ score, int32_t* __restrict__ lives, float* __restrict__ reward,
                           uint8_t* __restrict__ flags)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint8_t* ram = obs + i * 128u;
        int32_t s = 0;
        for (uint32_t b = 0; b < sp.score_bytes; b++) {
            const uint32_t v = ram[sp.score_addr[b] & 0x7Fu];
            s = sp.score_bcd ? s * 100 + (int32_t)((v >> 4) * 10u + (v & 0xFu)) : (int32_t)(((uint32_t)s << 8) | v);
        }
        const int32_t l = sp.lives_mask ? (int32_t)((ram[sp.lives_addr & 0x7Fu] & sp.lives_mask) >> sp.lives_shift) : 0;
        uint32_t f = 0;
        if (sp.terminal_mask && (ram[sp.terminal_addr & 0x7Fu] & sp.terminal_mask) == sp.terminal_value)
            f |= FA_EPISODE_TERMINAL;
        float r = 0.0f;
        if (!init) {
            r = (float)(s - score[i]);
            if (sp.lives_mask && l < lives[i]) f |= FA_EPISODE_LIFE_LOST;
        }
        score[i] = s;
        lives[i] = l;
        if (reward) reward[i] = r;
        if (flags) flags[i] = (uint8_t)f;
    }
}
}  // namespace

extern "C" int fa_obs_reward(const uint8_t* d_obs, size_t n, const fa_reward_spec* spec, int init, int32_t* d_score,
                             int32_t* d_lives, float* d_reward, uint8_t* d_flags, void* stream)
{
    if (!d_obs || !spec || !d_score || !d_lives) return fa_fail(FA_ERR_INVALID, "null buffer or spec");
    if (spec->score_bytes > 4) return fa_fail(FA_ERR_INVALID, "score_bytes %u > 4", (unsigned)spec->score_bytes);
    if (spec->lives_shift > 7) return fa_fail(FA_ERR_INVALID, "lives_shift %u > 7", (unsigned)spec->lives_shift);
    for (uint32_t b = 0; b < spec->score_bytes; b++)
        if (spec->score_addr[b] > 127) return fa_fail(FA_ERR_INVALID, "score byte %u outside RAM", b);
    if ((spec->lives_mask && spec->lives_addr > 127) || (spec->terminal_mask && spec->terminal_addr > 127))
        return fa_fail(FA_ERR_INVALID, "lives or terminal offset outside RAM");
    if (n == 0) return FA_OK;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    obs_reward<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(d_obs, n, *spec, init, d_score, d_lives, d_reward,
                                                                   d_flags);
    FA_CUDA(cudaGetLastError());
    return FA_OK;
}

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
