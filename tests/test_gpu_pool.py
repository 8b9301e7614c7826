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


def test_unit_trace_records_every_unit():
    """fa_pool_set_trace: one record per 32-instance unit of a batched launch,
    each cart's units tagged with its group, end after start, on a real SM."""
    import torch
    mixed = carts.mixed_carts()
    counts = [300, 70]
    with fa.AtariPool() as pool:
        for c, n in zip(mixed[:2], counts):
            pool.add_cart(c.rom, n)
        nu = sum((n + 31) // 32 for n in counts)
        d = torch.zeros(nu * 3, dtype=torch.int64, device="cuda")
        pool.set_trace(d.data_ptr(), nu)
        pool.step([carts.actions(seed=1, n=n, frames=2) for n in counts], 2, obs=False)
        pool.set_trace()
        tr = d.cpu().numpy().view(np.uint64).reshape(nu, 3)
        pool.step([carts.actions(seed=2, n=n, frames=1) for n in counts], 1, obs=False)   # no longer traced
        assert np.array_equal(d.cpu().numpy().view(np.uint64).reshape(nu, 3), tr)
    assert (tr[:, 1] > tr[:, 0]).all() and (tr[:, 0] > 0).all()
    tags = (tr[:, 2] & np.uint64(0xFFFF)).astype(int)
    assert sorted(np.bincount(tags).tolist()) == sorted([(n + 31) // 32 for n in counts])
    assert ((tr[:, 2] >> np.uint64(32)) < 1024).all()


@pytest.mark.parametrize("graph", [False, True])
def test_first_wave_placement_runs_every_unit_once(mixed, graph):
    """fa_pool_set_balance: with 4 warps per CTA the persistent launch has
    4 x (SMs) first-wave slots; 596 units exceed them, so the planned first
    wave and the device queue after it share the units.  Every unit runs
    exactly once, and the states equal those of the launch without the plan
    and, on a sample of instances, the oracle."""
    import torch
    counts = [9000, 6000, 3000, 1000]
    k = 1
    acts = [carts.actions(seed=40 + i, n=n, frames=k) for i, n in enumerate(counts)]
    nu = sum((n + 31) // 32 for n in counts)
    states = {}
    for balance in (True, False):
        with fa.AtariPool() as pool:
            for c, n in zip(mixed, counts):
                pool.add_cart(c.rom, n)
            for g, w in enumerate([1.0, 2.5, 4.0, 7.0]):
                pool.set_group(g, "pc", w)
            pool.set_launch(128, True, 4)
            pool.set_balance(balance)
            d = torch.zeros(nu * 3, dtype=torch.int64, device="cuda")
            pool.set_trace(d.data_ptr(), nu)
            if graph:
                da = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in acts]
                gr = pool.graph([t.data_ptr() for t in da], k, 1)
                gr.launch()
                torch.cuda.synchronize()
                gr.close()
            else:
                pool.step(acts, k, obs=False)
            tr = d.cpu().numpy().view(np.uint64).reshape(nu, 3)
            assert (tr[:, 0] > 0).all() and (tr[:, 1] > tr[:, 0]).all(), f"balance={balance}: a unit did not run"
            tags = (tr[:, 2] & np.uint64(0xFFFF)).astype(int)
            assert np.bincount(tags).tolist() == [(n + 31) // 32 for n in counts]
            states[balance] = [pool.group(g).download_states() for g in range(len(counts))]
    assert nu > 4 * torch.cuda.get_device_properties(0).multi_processor_count
    rng = np.random.default_rng(3)
    for g, (c, n) in enumerate(zip(mixed, counts)):
        assert_states_equal(states[True][g], states[False][g], f"group {g}: balance on vs off")
        idx = np.sort(rng.choice(n, 64, replace=False))
        ref = oracle_states(c.rom, len(idx))
        oracle.run_batch(c.rom, ref, acts[g][:, idx], k)
        assert_states_equal(states[True][g][idx], ref, f"group {g}: oracle sample")


def test_host_step_fills_caller_arrays(mixed):
    """pool.step(out=...): the observations of a host-buffer call land in the
    caller's arrays, call after call, equal to the oracle's.  Host-buffer
    calls have the kernel write observations into mapped pinned memory and
    copy them out on several threads when they are large: one cart here has
    40,000 instances (5 MB of observations)."""
    counts = [40000, 300]
    k = 2
    carts_ = [mixed[0], mixed[1]]
    refs = [oracle_states(c.rom, n) for c, n in zip(carts_, counts)]
    outs = [np.full((n, 128), 0xAB, np.uint8) for n in counts]
    with fa.AtariPool() as pool:
        for c, n in zip(carts_, counts):
            pool.add_cart(c.rom, n)
        for call in range(2):
            acts = [carts.actions(seed=70 + 10 * call + i, n=n, frames=k) for i, n in enumerate(counts)]
            got = pool.step(acts, k, out=outs)
            assert all(g is o for g, o in zip(got, outs))
            for gi, (c, ref) in enumerate(zip(carts_, refs)):
                o, _ = oracle.run_batch(c.rom, ref, acts[gi], k)
                assert np.array_equal(outs[gi], o), f"call {call} group {gi}"
        with pytest.raises(ValueError):
            pool.step(acts, k, out=[outs[0]])
