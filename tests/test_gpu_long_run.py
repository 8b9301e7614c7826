"""Ten thousand frames, bit for bit: the four mappers of the mixed batch in one
pool, stepped 100 frames per batched call for 10,000 frames, against the oracle
after every call (RAM) and at the end (full state: registers, flags, cycle
counter, RAM, TIA/PIA fields, bank, frame counter, status).  The bar is 0
mismatches over 10^4 frames."""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal, oracle_states

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


def test_ten_thousand_frames_all_mappers():
    mixed = carts.mixed_carts()
    n, k, frames = 16, 100, 10_000
    states = [oracle_states(c.rom, n) for c in mixed]
    with fa.AtariPool() as pool:
        for c in mixed:
            pool.add_cart(c.rom, n)
        pool.set_launch(128, True)
        for call in range(frames // k):
            acts = [carts.actions(seed=500 + g, n=n, frames=k, frame0=call * k) for g in range(len(mixed))]
            obs = pool.step(acts, k)
            for g, c in enumerate(mixed):
                o_obs, _ = oracle.run_batch(c.rom, states[g], acts[g], k)
                assert np.array_equal(obs[g], o_obs), f"{c.spec.name}: RAM differs after frame {(call + 1) * k}"
        for g, c in enumerate(mixed):
            st = pool.group(g).download_states()
            assert_states_equal(st, states[g], f"{c.spec.name} after {frames} frames")
            assert (st["frame_no"] == frames).all()
            assert (st["run_status"] == 0).all()
