"""The no-allocation entry point, fa_step_static, against the existing one.

fa_step_static exists for callers that cannot call cudaMalloc (their device
memory is owned by another allocator, or their stepping loop must not trigger
cudaMalloc's implicit device synchronisation).  It runs the same persistent
kernel with its scratch in a fixed array inside the library.  Here a twin
handle is stepped through fa_step_multi_async (the existing entry point) and
the same instances through fa_step_static, on two calls in a row; RAM and the
full state must agree bit for bit.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal

pytestmark = pytest.mark.gpu


def bank_image(rom: bytes) -> np.ndarray:
    if len(rom) <= 4096:
        return np.frombuffer(bytes(rom[i % len(rom)] for i in range(4096)), np.uint8).copy()
    nb = 2 if len(rom) <= 8192 else 4 if len(rom) <= 16384 else 8
    return np.frombuffer(rom[:nb * 4096], np.uint8).copy()


def scheme_of(rom: bytes) -> int:
    return 0 if len(rom) <= 4096 else 1 if len(rom) <= 8192 else 2 if len(rom) <= 16384 else 3


@pytest.mark.parametrize("which", [1, 3])           # 8K F8 and 32K F4 carts
def test_static_entry_point_matches_existing(which):
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")
    import torch
    rom = carts.mixed_carts()[which].rom
    n, k = 777, 5
    L = fa.lib()
    acts = carts.actions(seed=90 + which, n=n, frames=2 * k)
    d_acts = torch.from_numpy(acts.reshape(-1).copy()).cuda()
    d_rom = torch.from_numpy(bank_image(rom)).cuda()
    d_obs = torch.zeros(n * 128, dtype=torch.uint8, device="cuda")
    d_obs_ref = torch.zeros(n * 128, dtype=torch.uint8, device="cuda")
    with fa.BatchAtariGpu(rom, n) as ref, fa.BatchAtariGpu(rom, n) as sub:
        ref.reset()
        sub.reset()
        stride = ctypes.c_uint32()
        d_state = L.fa_device_state(sub._h, ctypes.byref(stride))
        torch.cuda.synchronize()
        for call in range(2):
            off = call * k * n
            ref.step_multi_async(d_acts.data_ptr() + off, k, d_obs_ref.data_ptr())
            ref.synchronize()
            rc = L.fa_step_static(d_rom.data_ptr(), scheme_of(rom), d_state, stride.value, n,
                                  d_acts.data_ptr() + off, k, 1, d_obs.data_ptr(), fa.SCHED_PC, None)
            assert rc == 0, L.fa_last_error().decode()
            assert torch.equal(d_obs, d_obs_ref), f"observations differ on call {call + 1}"
            assert_states_equal(sub.download_states(), ref.download_states(), f"call {call + 1}")


def test_static_entry_point_rejects_oversize_calls():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")
    import torch
    L = fa.lib()
    rom = carts.mixed_carts()[0].rom
    d_rom = torch.from_numpy(bank_image(rom)).cuda()
    with fa.BatchAtariGpu(rom, 32) as h:
        h.reset()
        stride = ctypes.c_uint32()
        d_state = L.fa_device_state(h._h, ctypes.byref(stride))
        d_acts = torch.zeros(32, dtype=torch.uint8, device="cuda")
        rc = L.fa_step_static(d_rom.data_ptr(), 0, d_state, stride.value, 32, d_acts.data_ptr(), 1, 1025,
                              None, fa.SCHED_PC, None)
        assert rc == -6 and b"1..1024" in L.fa_last_error()
