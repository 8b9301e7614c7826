"""GPU tests of the batched form (pools): one launch over several carts.

Each instance's result must be the same whether its cart runs alone (its own
handle, plain per-frame launches) or inside the mixed batch (persistent
multi-cart launch, or a CUDA graph of many calls), and must equal the oracle.
"""
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


@pytest.fixture(scope="module")
def mixed():
    return carts.mixed_carts()


COUNTS = (700, 300, 130, 33)     # ragged, several units per cart, one partial CTA each


def run_oracle(mixed, acts, k):
    outs, states = [], []
    for c, n, a in zip(mixed, COUNTS, acts):
        st = oracle_states(c.rom, n)
        o, _ = oracle.run_batch(c.rom, st, a, k)
        outs.append(o)
        states.append(st)
    return outs, states


@pytest.mark.parametrize("persistent,block", [(True, 128), (True, 256), (False, 128)])
def test_pool_step_matches_oracle(mixed, persistent, block):
    k = 6
    acts = [carts.actions(seed=31 + i, n=n, frames=k) for i, n in enumerate(COUNTS)]
    o_obs, o_st = run_oracle(mixed, acts, k)
    with fa.AtariPool() as pool:
        for c, n in zip(mixed, COUNTS):
            pool.add_cart(c.rom, n)
        pool.set_launch(block, persistent)
        for g, s in enumerate(["pc", "lane", "line", "match"]):
            pool.set_group(g, s, weight=1.0 + g)
        obs = pool.step(acts, k)
        for g in range(4):
            assert np.array_equal(obs[g], o_obs[g]), f"group {g}"
            assert_states_equal(pool.group(g).download_states(), o_st[g], f"group {g}")


def test_pool_plain_equals_batched(mixed):
    k = 5
    acts = [carts.actions(seed=41 + i, n=n, frames=k) for i, n in enumerate(COUNTS)]
    with fa.AtariPool() as a, fa.AtariPool() as b:
        for c, n in zip(mixed, COUNTS):
            a.add_cart(c.rom, n)
            b.add_cart(c.rom, n)
        oa = a.step(acts, k)
        ob = b.step_plain(acts, k)
        for g in range(4):
            assert np.array_equal(oa[g], ob[g])
            assert_states_equal(a.group(g).download_states(), b.group(g).download_states(), f"group {g}")


def test_alone_equals_in_the_mix(mixed):
    """A cart alone in its own handle and the same cart inside the batch."""
    k = 8
    acts = [carts.actions(seed=51 + i, n=n, frames=k) for i, n in enumerate(COUNTS)]
    with fa.AtariPool() as pool:
        for c, n in zip(mixed, COUNTS):
            pool.add_cart(c.rom, n)
        obs = pool.step(acts, k)
        for g, (c, n) in enumerate(zip(mixed, COUNTS)):
            with fa.BatchAtariGpu(c.rom, n) as h:
                h.reset()
                alone = h.step_multi(acts[g], k)
                assert np.array_equal(alone, obs[g])
                assert_states_equal(h.download_states(), pool.group(g).download_states(), f"group {g}")


def test_graph_replay_matches_oracle(mixed):
    import torch
    k, calls = 3, 7
    acts = [carts.actions(seed=61 + i, n=n, frames=k * calls) for i, n in enumerate(COUNTS)]
    o_obs, o_st = run_oracle(mixed, acts, k * calls)
    with fa.AtariPool() as pool:
        for c, n in zip(mixed, COUNTS):
            pool.add_cart(c.rom, n)
        d_act = [torch.from_numpy(a.reshape(-1).copy()).cuda() for a in acts]
        d_obs = [torch.zeros(n * 128, dtype=torch.uint8, device="cuda") for n in COUNTS]
        torch.cuda.synchronize()
        g = pool.graph([t.data_ptr() for t in d_act], k, calls, [t.data_ptr() for t in d_obs])
        g.launch()
        pool.synchronize()
        g.close()
        for gi in range(4):
            assert np.array_equal(d_obs[gi].cpu().numpy().reshape(-1, 128), o_obs[gi])
            assert_states_equal(pool.group(gi).download_states(), o_st[gi], f"group {gi}")


def test_pool_rejects_too_many_carts(mixed):
    with fa.AtariPool() as pool:
        for i in range(16):
            pool.add_cart(mixed[0].rom, 1)
        with pytest.raises(fa.FaError):
            pool.add_cart(mixed[0].rom, 1)
