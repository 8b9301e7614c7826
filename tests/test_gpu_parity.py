"""GPU parity: the CUDA path against the CPU oracle, bit for bit.

Restates the reference's parity procedures (tests/test_cuda.rs:40-154,
tests/test_cuda_persistent.rs:12-109, tests/test_cuda_sorted.rs:20-85) on
seeded synthetic carts (Breakout.bin is not available), and widens them: the
full state is compared (registers, flags, cycle counter, RAM, TIA/PIA
registers, bank, frame counter, status), on all four mappers, under every
warp scheduling policy and launch shape.  Every call goes through the C ABI.
"""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa

pytestmark = pytest.mark.gpu

ACTION_SEQ = [0, 0, 2, 3, 4, 1, 0, 5, 0, 0, 1, 2, 3, 4, 5, 6, 7, 8]   # test_cuda.rs:92

_CARTS = {}


def cart(name):
    if name not in _CARTS:
        if name == "plain":
            c = carts.plain_cart()
        elif name == "divergence":
            c = carts.divergence_cart()
        elif name == "scale":
            c = carts.scale_cart()
        else:
            c = {m.spec.name: m for m in carts.mixed_carts()}[name]
        _CARTS[name] = c
    return _CARTS[name].rom


ALL_CARTS = ["plain", "divergence", "scale", "mixed_2k", "mixed_8k", "mixed_16k", "mixed_32k"]
COMPARED = oracle.COMPARED_FIELDS


def assert_states_equal(gpu, orc, what=""):
    assert gpu.shape == orc.shape
    for name in COMPARED:
        g, o = gpu[name], orc[name]
        if not np.array_equal(g, o):
            bad = np.nonzero((g != o).reshape(len(g), -1).any(axis=1))[0]
            i = int(bad[0])
            raise AssertionError(f"{what}: field {name} differs in {len(bad)} instances; "
                                 f"first i={i}: gpu={g[i]!r} oracle={o[i]!r}")


def oracle_states(rom, n):
    snap = oracle.reset_state(rom)
    return np.array([snap] * n, dtype=oracle.STATE_DTYPE)


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


# ---------------------------------------------------------------- reference procedures
@pytest.mark.parametrize("name", ALL_CARTS)
def test_reset_matches_oracle(name):
    rom = cart(name)
    with fa.BatchAtariGpu(rom, 37) as g:
        obs = g.reset()
        st = g.download_states()
    ref = oracle_states(rom, 37)
    assert_states_equal(st, ref, f"reset {name}")
    assert np.array_equal(obs, ref["ram"])


def test_parity_single_frame():                       # test_cuda.rs:40-73
    rom = cart("plain")
    n = 4
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        obs = g.step(np.zeros(n, np.uint8))
        st = g.download_states()
    ref = oracle_states(rom, n)
    o_obs, _ = oracle.run_batch(rom, ref, np.zeros(n, np.uint8), 1)
    assert np.array_equal(obs, o_obs)
    assert_states_equal(st, ref, "single frame")


@pytest.mark.parametrize("sorted_", [False, True])
def test_parity_500_frames(sorted_):                  # test_cuda.rs:76-116, test_cuda_sorted.rs:20-52
    rom = cart("plain")
    n, k = 10, 500
    acts = np.array([[ACTION_SEQ[f % len(ACTION_SEQ)]] * n for f in range(k)], np.uint8)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_sorted(sorted_)
        g.reset()
        for f in range(k):
            obs = g.step(acts[f])
            o_obs, _ = oracle.run_batch(rom, ref, acts[f], 1, nthreads=2)
            assert np.array_equal(obs, o_obs), f"RAM mismatch at frame {f + 1}"
            if f in (0, 49, 99, 249, 499):
                assert_states_equal(g.download_states(), ref, f"frame {f + 1}")


def test_parity_varied_actions():                     # test_cuda.rs:119-154
    rom = cart("plain")
    n, k = 18, 100
    acts = np.tile(np.arange(n, dtype=np.uint8), (k, 1))
    ref = oracle_states(rom, n)
    trace, _ = oracle.run_batch(rom, ref, acts, k, trace=True)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        for f in range(k):
            assert np.array_equal(g.step(acts[f]), trace[f]), f"frame {f + 1}"
        assert_states_equal(g.download_states(), ref, "varied actions")


@pytest.mark.parametrize("sorted_", [False, True])
@pytest.mark.parametrize("n,k,varied", [(10, 500, False), (18, 100, True)])
def test_multi_frame(n, k, varied, sorted_):          # test_cuda_persistent.rs:12-109, test_cuda_sorted.rs:55-85
    rom = cart("plain")
    if varied:
        acts = np.tile(np.arange(n, dtype=np.uint8), (k, 1))
    else:
        acts = np.array([[ACTION_SEQ[f % len(ACTION_SEQ)]] * n for f in range(k)], np.uint8)
    ref = oracle_states(rom, n)
    o_obs, _ = oracle.run_batch(rom, ref, acts, k)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_sorted(sorted_)
        g.reset()
        obs = g.step_multi(acts, k)
        st = g.download_states()
    assert np.array_equal(obs, o_obs)
    assert_states_equal(st, ref, f"K={k}")


# ---------------------------------------------------------------- widened coverage
@pytest.mark.parametrize("sched", ["lane", "pc", "line", "match"])
@pytest.mark.parametrize("name", ALL_CARTS)
def test_all_carts_all_policies(name, sched):
    """Every mapper x every warp policy: 200 instances (6 full warps and a
    ragged one, two CTAs), random actions, full state every 10 frames."""
    rom = cart(name)
    n, k, chunk = 200, 40, 10
    acts = carts.actions(seed=11, n=n, frames=k)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, sched, False)
        g.reset()
        for f0 in range(0, k, chunk):
            obs = g.step_multi(acts[f0:f0 + chunk], chunk)
            o_obs, _ = oracle.run_batch(rom, ref, acts[f0:f0 + chunk], chunk)
            assert np.array_equal(obs, o_obs), f"{name}/{sched} frames {f0}..{f0 + chunk}"
            assert_states_equal(g.download_states(), ref, f"{name}/{sched} after {f0 + chunk}")


@pytest.mark.parametrize("block,persistent", [(64, False), (256, False), (512, False), (128, True), (256, True)])
def test_launch_shapes(block, persistent):
    rom = cart("mixed_32k")
    n, k = 1000, 12
    acts = carts.actions(seed=5, n=n, frames=k)
    ref = oracle_states(rom, n)
    o_obs, _ = oracle.run_batch(rom, ref, acts, k)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(block, "pc", persistent)
        g.reset()
        obs = g.step_multi(acts, k)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, f"block {block} persistent {persistent}")


def test_per_frame_equals_multi_frame():
    rom = cart("divergence")
    n, k = 300, 16
    acts = carts.actions(seed=9, n=n, frames=k)
    with fa.BatchAtariGpu(rom, n) as a, fa.BatchAtariGpu(rom, n) as b:
        a.reset()
        b.reset()
        for f in range(k):
            oa = a.step(acts[f])
        ob = b.step_multi(acts, k)
        assert np.array_equal(oa, ob)
        assert_states_equal(a.download_states(), b.download_states(), "step vs step_multi")


def test_episode_reset_with_phase_offsets():
    rom = cart("scale")
    n, k, ep = 96, 30, 7
    acts = carts.actions(seed=4, n=n, frames=k)
    phase = (np.arange(n) * 5) % ep
    ref = oracle_states(rom, n)
    ref["frame_no"] = phase
    snap = oracle.reset_state(rom)
    o_obs, _ = oracle.run_batch(rom, ref, acts, k, snapshot=snap, episode_frames=ep)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        g.set_episode_frames(ep)
        g.set_frame_numbers(phase.astype(np.uint32))
        obs = g.step_multi(acts, k)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "episode reset")


def test_set_states_round_trip_and_continue():
    """Checkpoint: states taken from the oracle mid-run, uploaded, continued."""
    rom = cart("mixed_16k")
    n = 64
    ref = oracle_states(rom, n)
    oracle.run_batch(rom, ref, carts.actions(seed=1, n=n, frames=13), 13)
    with fa.BatchAtariGpu(rom, n) as g:
        g.upload_states(ref)
        assert_states_equal(g.download_states(), ref, "round trip")
        acts = carts.actions(seed=2, n=n, frames=9)
        obs = g.step_multi(acts, 9)
        o_obs, _ = oracle.run_batch(rom, ref, acts, 9)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "continued")


def test_illegal_opcode_halts_like_oracle():
    """A cart whose init jumps into an illegal opcode: the reference panics;
    both implementations latch ILLEGAL_OPCODE with the same state."""
    rom = bytearray([0xEA] * 4096)
    rom[0:6] = bytes([0xA9, 0x02, 0x85, 0x00, 0xE8, 0x02])   # LDA #2; STA VSYNC; INX; KIL
    rom[0xFFC:0xFFE] = bytes([0x00, 0xF0])
    rom = bytes(rom)
    n = 8
    ref = oracle_states(rom, n)
    oracle.run_batch(rom, ref, np.zeros(3 * n, np.uint8), 3)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        g.step_multi(np.zeros(3 * n, np.uint8), 3)
        st = g.download_states()
    assert (st["run_status"] & fa.FA_STATUS_ILLEGAL_OPCODE).all()
    assert_states_equal(st, ref, "illegal opcode")


def test_step_before_reset_is_noop():
    rom = cart("plain")
    with fa.BatchAtariGpu(rom, 5) as g:
        g.step(np.zeros(5, np.uint8))
        st = g.status()
    assert (st == fa.FA_STATUS_NOT_RESET).all()


def test_large_batch_identical_streams_and_spot_check():
    """Size-independent properties at a larger N: instances fed identical
    action streams end identical; a random sample matches the oracle."""
    rom = cart("divergence")
    n, k = 20000, 6
    rng = np.random.default_rng(3)
    base = carts.actions(seed=21, n=64, frames=k)
    acts = base[:, np.arange(n) % 64]
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(256, "pc", True)
        g.reset()
        obs = g.step_multi(acts, k)
        st = g.download_states()
    for j in range(64):
        same = st[j::64]
        assert (same["ram"] == same["ram"][0]).all() and (same["cycles"] == same["cycles"][0]).all()
    idx = rng.choice(n, 256, replace=False)
    ref = oracle_states(rom, 256)
    o_obs, _ = oracle.run_batch(rom, ref, acts[:, idx], k)
    assert np.array_equal(obs[idx], o_obs)
    assert_states_equal(st[idx], ref, "spot check")


def test_scale_config_spot_check():
    """The scale configuration at full size: 1,000,000 instances of the 32K F4
    cart, K=16 per call, reset to the post-init snapshot every 2,000 frames
    with per-instance phase offsets uniform in [0, 2000).  1,024 random
    instances, plus instances whose reset falls inside the call, match the
    oracle bit for bit; instances that share a phase and an action stream end
    identical."""
    rom = cart("scale")
    n, k, ep = 1_000_000, 16, 2000
    rng = np.random.default_rng(11)
    phase = rng.integers(0, ep, n, dtype=np.uint32)
    # 4,096 distinct action streams, repeated: instance i follows stream i % 4096.
    base = carts.actions(seed=77, n=4096, frames=k)
    acts = np.ascontiguousarray(base[:, np.arange(n) % 4096])
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, "pc", True)
        g.reset()
        g.set_episode_frames(ep)
        g.set_frame_numbers(phase)
        obs = g.step_multi(acts, k)
        st = g.download_states()
    resets = np.nonzero(phase > ep - k)[0]
    assert len(resets) > 1000
    idx = np.unique(np.concatenate([rng.choice(n, 1024, replace=False), resets[:256]]))
    ref = oracle_states(rom, len(idx))
    ref["frame_no"] = phase[idx]
    o_obs, _ = oracle.run_batch(rom, ref, acts[:, idx], k, snapshot=oracle.reset_state(rom), episode_frames=ep)
    assert np.array_equal(obs[idx], o_obs)
    assert_states_equal(st[idx], ref, "scale spot check")
    # Same stream and same phase: identical end state (a size-independent check over all n).
    key = (np.arange(n) % 4096).astype(np.int64) * ep + phase
    order = np.argsort(key, kind="stable")
    ks = key[order]
    first = np.r_[True, ks[1:] != ks[:-1]]
    head = order[np.maximum.accumulate(np.where(first, np.arange(n), 0))]
    assert (st["ram"][order] == st["ram"][head]).all()
    assert (st["cycles"][order] == st["cycles"][head]).all()


# ---------------------------------------------------------------- committed golden vectors
def _golden():
    import json
    from pathlib import Path
    return json.loads((Path(__file__).parent / "golden" / "oracle_vectors.json").read_text())


@pytest.mark.parametrize("name", ALL_CARTS)
def test_matches_committed_golden_vectors(name):
    """The CUDA path reproduces the frozen oracle vectors (tests/golden/) without
    running the oracle: RAM at checkpoint frames and the full final state."""
    import hashlib
    from make_golden import state_sha
    want = _golden()[name]
    rom = cart(name)
    assert hashlib.sha256(rom).hexdigest() == want["rom_sha256"]
    n, frames = want["n"], want["frames"]
    acts = carts.actions(seed=want["action_seed"], n=n, frames=frames)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        assert state_sha(g.download_states()[:1]) == want["reset_state_sha256"]
        done = 0
        for f_end in sorted(int(x) for x in want["ram_sha256_at"]):
            obs = g.step_multi(acts[done:f_end], f_end - done)
            done = f_end
            assert hashlib.sha256(obs.tobytes()).hexdigest() == want["ram_sha256_at"][str(f_end)], f_end
        st = g.download_states()
    assert state_sha(st) == want["final_state_sha256"]
