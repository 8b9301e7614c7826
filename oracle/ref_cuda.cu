// ref_cuda.cu — host launcher for the reference's own CUDA kernels
// (cuda/src/atari_kernel.cu of RPP1011/fast-atari-rs), compiled for sm_100a
// from the reference's sources where they lie by `make -C oracle ref`, into
// oracle/_ref/.  Test infrastructure only: it times the kernels the reference
// ships (the "kernel to beat") on the same carts and instance counts as this
// repository's kernels.  It is not an oracle: the reference kernels skip the
// Rust emulator's phantom bus accesses (cuda/src/cpu_6502.cuh), so their
// results are compared with the CPU oracle and reported, not trusted.
//
// Launch shape as the reference's host binding: grid ceil(n/128), block 128
// (src/cuda_env.rs:147-150); per-frame = one atari_frame_kernel launch per
// frame (BatchAtariGpu::step), multi = one atari_multi_frame_kernel launch of
// k frames (step_multi, src/cuda_env.rs:166-184); sorted selects the _sorted
// variants (set_sorted).  Only carts whose control flow cannot reach a byte
// that is not a legal opcode may be run: the reference kernels execute an
// illegal opcode as a 0-cycle NOP, so such a frame never ends.
#include <cuda_runtime.h>
#include <stdint.h>

#include "atari_kernel.cu"

extern "C" int ref_state_size(void) { return (int)sizeof(AtariState); }

// states: n * ref_state_size() bytes (in/out); actions: k * n bytes,
// frame-major; obs_out: n * 128 bytes (the last frame).  *ms_out receives the
// device time of the launches alone (CUDA events around them; states,
// actions and ROM already resident).  Returns 0 or a cudaError_t.
extern "C" int ref_run(const uint8_t* rom, uint32_t rom_len, void* states, int n, const uint8_t* actions, int k,
                       int multi, int sorted, uint8_t* obs_out, float* ms_out)
{
    if (n <= 0 || k <= 0 || rom_len == 0 || rom_len > MAX_ROM_SIZE) return (int)cudaErrorInvalidValue;
    const size_t sb = (size_t)n * sizeof(AtariState);
    AtariState* d_states = nullptr;
    uint8_t *d_actions = nullptr, *d_obs = nullptr, *d_rom = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&d_states, sb);
    if (e == cudaSuccess) e = cudaMalloc(&d_actions, (size_t)k * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_obs, (size_t)n * 128);
    if (e == cudaSuccess) e = cudaMalloc(&d_rom, rom_len);
    if (e == cudaSuccess) e = cudaMemcpy(d_states, states, sb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_actions, actions, (size_t)k * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_rom, rom, rom_len, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        const dim3 grid((unsigned)((n + BLOCK_SIZE - 1) / BLOCK_SIZE)), block(BLOCK_SIZE);
        cudaEventRecord(e0);
        if (multi) {
            if (sorted) atari_multi_frame_kernel_sorted<<<grid, block>>>(d_states, d_actions, d_obs, d_rom, rom_len, k, n);
            else atari_multi_frame_kernel<<<grid, block>>>(d_states, d_actions, d_obs, d_rom, rom_len, k, n);
        } else {
            for (int f = 0; f < k; f++) {
                if (sorted) atari_frame_kernel_sorted<<<grid, block>>>(d_states, d_actions + (size_t)f * n, d_obs, d_rom, rom_len, n);
                else atari_frame_kernel<<<grid, block>>>(d_states, d_actions + (size_t)f * n, d_obs, d_rom, rom_len, n);
            }
        }
        cudaEventRecord(e1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess && ms_out) e = cudaEventElapsedTime(ms_out, e0, e1);
    }
    if (e == cudaSuccess) e = cudaMemcpy(states, d_states, sb, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && obs_out) e = cudaMemcpy(obs_out, d_obs, (size_t)n * 128, cudaMemcpyDeviceToHost);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_states);
    cudaFree(d_actions);
    cudaFree(d_obs);
    cudaFree(d_rom);
    return (int)e;
}
