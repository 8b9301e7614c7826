"""Failure paths on the GPU, each reached without faulting, trapping or
hanging the device.

* A cart that never raises VSYNC: every frame ends at the reference's
  100,000-cycle cap (src/atari.rs:592-595), with FA_STATUS_CYCLE_CAP set, as
  the oracle does.
* A cart that holds VSYNC: the reference waits for it to drop forever
  (src/atari.rs:588-590); this library halts the instance after 2,000,000
  cycles with FA_STATUS_VSYNC_BUDGET, as the oracle does; later frames run
  nothing, and only their set_action reaches its inputs.
* The device-side bound on the ROM staging wait set to 0 (give up at once),
  through the handle's warp-granular kernel, the CTA-granular kernel (a
  pool whose ROM library does not fit in shared memory), the rendering
  console and the server: the call returns FA_ERR_KERNEL, every instance's
  state is unchanged, and with the bound restored the same call runs and
  matches the oracle.
"""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal, oracle_states

pytestmark = pytest.mark.gpu

FA_ERR_KERNEL = -5
STATUS_VSYNC_BUDGET = 0x2
STATUS_CYCLE_CAP = 0x100
DEFAULT_WAIT_NS = 2_000_000_000


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


@pytest.fixture()
def zero_wait():
    """The staging wait bound at 0 for the test's body, restored after."""
    assert fa.wait_limit_ns() == DEFAULT_WAIT_NS
    yield lambda on: fa.set_wait_limit_ns(0 if on else DEFAULT_WAIT_NS)
    fa.set_wait_limit_ns(DEFAULT_WAIT_NS)


@pytest.mark.parametrize("sched", ["pc", "lane"])
def test_cycle_cap_cart_matches_oracle(sched):
    rom = carts.stall_cart("no_vsync").rom
    n, k = 70, 3
    acts = carts.actions(seed=5, n=n, frames=k)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, sched, True)
        g.reset()
        assert_states_equal(g.download_states(), ref, "reset")
        for f in range(k):
            obs = g.step(acts[f])
            o_obs, _ = oracle.run_batch(rom, ref, acts[f:f + 1], 1)
            assert np.array_equal(obs, o_obs)
            st = g.download_states()
            assert_states_equal(st, ref, f"frame {f}")
    assert (st["run_status"] & STATUS_CYCLE_CAP).all()
    assert (st["frame_no"] == k).all()                      # the cap ends the frame; the instance runs on


def test_vsync_held_cart_halts_with_budget_status():
    rom = carts.stall_cart("vsync_held").rom
    n = 40
    acts = carts.actions(seed=6, n=n, frames=3)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        assert (g.download_states()["run_status"] == 0).all()
        g.step(acts[0])
        oracle.run_batch(rom, ref, acts[0:1], 1)
        st = g.download_states()
        assert_states_equal(st, ref, "budget frame")
        assert (st["run_status"] & STATUS_VSYNC_BUDGET).all()
        assert (st["cycles"] > 1_000_000).all()
        # Halted: later frames run nothing; only set_action reaches the inputs.
        g.step_multi(acts[1:], 2)
        oracle.run_batch(rom, ref, acts[1:], 2)
        after = g.download_states()
        assert_states_equal(after, ref, "after halt")
        inputs = {"port_a_input", "inpt4", "paddle0"}
        for name in oracle.COMPARED_FIELDS:
            if name not in inputs:
                assert np.array_equal(after[name], st[name]), name
        assert (g.status() & STATUS_VSYNC_BUDGET).all()


def _expect_kernel_error(fn, text="error word 0x1"):
    with pytest.raises(fa.FaError) as ei:
        fn()
    assert ei.value.code == FA_ERR_KERNEL, ei.value
    assert text in str(ei.value)


@pytest.mark.parametrize("persistent", [True, False])
def test_zero_wait_bound_handle(zero_wait, persistent):
    rom = carts.mixed_carts()[1].rom
    n, k = 300, 2
    acts = carts.actions(seed=7, n=n, frames=k)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, "pc", persistent)
        g.reset()
        before = g.download_states()
        zero_wait(True)
        _expect_kernel_error(lambda: g.step_multi(acts, k))
        assert_states_equal(g.download_states(), before, "after the wait gave up")
        zero_wait(False)
        obs = g.step_multi(acts, k)
    ref = oracle_states(rom, n)
    o_obs, _ = oracle.run_batch(rom, ref, acts, k)
    assert np.array_equal(obs, o_obs)


def test_zero_wait_bound_cta_granular_pool(zero_wait):
    """Seven 32K carts: the ROM library (224 KiB) does not fit beside a warp's
    RAM slab, so the pool runs the CTA-granular kernel that stages one cart's
    ROM per unit."""
    rom = carts.mixed_carts()[3].rom
    counts = [50, 40, 33, 20, 64, 31, 45]
    k = 1
    acts = [carts.actions(seed=80 + i, n=n, frames=k) for i, n in enumerate(counts)]
    with fa.AtariPool() as pool:
        for n in counts:
            pool.add_cart(rom, n)
        before = [pool.group(i).download_states() for i in range(len(counts))]
        zero_wait(True)
        _expect_kernel_error(lambda: pool.step(acts, k))
        for i in range(len(counts)):
            assert_states_equal(pool.group(i).download_states(), before[i], f"group {i} after the wait gave up")
        zero_wait(False)
        obs = pool.step(acts, k)
    for i, n in enumerate(counts):
        ref = oracle_states(rom, n)
        o, _ = oracle.run_batch(rom, ref, acts[i], k)
        assert np.array_equal(obs[i], o), i


def test_zero_wait_bound_rendering_console(zero_wait):
    rom = carts.render_cart().rom
    n = 40
    acts = carts.actions(seed=9, n=n, frames=1)
    with fa.AtariRender(rom, n) as g:
        g.reset()
        before, fb_before = g.states(), g.framebuffers()
        zero_wait(True)
        _expect_kernel_error(lambda: g.step_multi(acts, 1))
        assert np.array_equal(g.states(), before)
        assert np.array_equal(g.framebuffers(), fb_before)
        zero_wait(False)
        g.step_multi(acts, 1)


def test_zero_wait_bound_server(zero_wait):
    rom = carts.mixed_carts()[0].rom
    n, k = 64, 2
    acts = carts.actions(seed=10, n=n, frames=k)
    with fa.AtariServer([rom]) as srv:
        sid = srv.open(0)
        zero_wait(True)
        _expect_kernel_error(lambda: srv.step(sid, acts, n, k), text="failed")
        zero_wait(False)
        obs, _ = srv.step(sid, acts, n, k)
        st = srv.states(sid)
    # The failed request admitted the instances (post-reset snapshot) and ran
    # nothing; the second request ran both frames from there.
    ref = oracle_states(rom, n)
    o, _ = oracle.run_batch(rom, ref, acts, k)
    assert np.array_equal(obs, o)
    assert_states_equal(st, ref, "server after a failed request")

