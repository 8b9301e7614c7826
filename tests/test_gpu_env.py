"""GPU tests of the batched RL caller (BatchAtariGpuEnv, src/rl4burn_env.rs:
269-380) and of the project autotuner."""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


def test_env_matches_oracle_with_frameskip_and_broadcast():
    import fast_atari_b200.env as fenv
    rom = carts.mixed_carts()[2].rom
    n = 40
    env = fenv.BatchAtariGpuEnv(rom, n).with_max_steps(3)
    obs = env.reset().cpu().numpy()
    snap = oracle.reset_state(rom)
    ref = np.array([snap] * n, dtype=oracle.STATE_DTYPE)
    assert np.array_equal(obs, (ref["ram"].reshape(-1).astype(np.float32) / np.float32(255.0)))
    for t, action in enumerate([1, 4, 17]):
        step = env.step(action)
        acts = np.full(4 * n, action, np.uint8)                      # broadcast x frameskip 4
        o_obs, _ = oracle.run_batch(rom, ref, acts, 4)
        want = o_obs.reshape(-1).astype(np.float32) / np.float32(255.0)
        assert np.array_equal(step.observation.cpu().numpy(), want), t
        assert step.reward == 0.0 and not step.terminated
        assert step.truncated == (t == 2)
    assert env.action_space() == ("Discrete", 18)
    env.close()


def test_obs_normalisation_is_exact():
    import torch
    src = torch.arange(256, dtype=torch.uint8, device="cuda").repeat(3)
    out = torch.empty(src.numel(), dtype=torch.float32, device="cuda")
    assert fa.lib().fa_obs_to_unit_f32(fa._vp(src.data_ptr()), fa._vp(out.data_ptr()), src.numel(), None) == 0
    torch.cuda.synchronize()
    want = np.tile(np.arange(256, dtype=np.float32) / np.float32(255.0), 3)
    assert np.array_equal(out.cpu().numpy(), want)


def test_autotune_returns_a_measured_best():
    best, table = fa.autotune(carts.divergence_cart().rom, 4096)
    assert best["frames_per_s"] > 0 and best["ns_per_instance_frame"] > 0
    assert len(table) >= 12
    # The last stage sweeps K at the launch shape chosen before it (the
    # carried-over record plus four other K): the best is its fastest entry.
    last = table[-5:]
    assert len({(t["sched"], t["persistent"], t["cta_warps"], t["block"]) for t in last}) == 1
    assert best == max(last, key=lambda t: t["frames_per_s"])
    assert best["sched"] in (0, 1, 2, 3) and best["k"] in (1, 2, 4, 8, 16)


def _decode(ram, spec_args):
    """The reward rule of fa_obs_reward restated in numpy (int32 arithmetic)."""
    score, bcd, lives, terminal = spec_args
    s = np.zeros(len(ram), np.int64)
    for a in score:
        v = ram[:, a].astype(np.int64)
        s = s * 100 + (v >> 4) * 10 + (v & 15) if bcd else (s << 8) | v
    s = s.astype(np.uint64).astype(np.uint32).view(np.int32)
    l = ((ram[:, lives[0]] & lives[1]) >> lives[2]).astype(np.int32) if lives else np.zeros(len(ram), np.int32)
    t = ((ram[:, terminal[0]] & terminal[1]) == terminal[2]) if terminal else np.zeros(len(ram), bool)
    return s, l, t


@pytest.mark.parametrize("spec_args", [((3, 4, 5), True, (7, 0x0C, 2), (9, 0x80, 0x80)),
                                       ((10, 11, 12, 13), False, (20, 0xFF, 0), None),
                                       ((), True, None, (30, 0x01, 0x00))])
def test_env_rewards_from_ram(spec_args):
    import fast_atari_b200.env as fenv
    score, bcd, lives, terminal = spec_args
    rom = carts.divergence_cart().rom
    n = 70
    spec = fa.RewardSpec.make(score, bcd, lives, terminal)
    env = fenv.BatchAtariGpuEnv(rom, n).with_reward(spec)
    env.reset()
    ref = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
    prev_s, prev_l, _ = _decode(ref["ram"], spec_args)
    saw_reward = False
    for t, action in enumerate([3, 12, 0, 7, 17, 5]):
        step = env.step(action)
        o_obs, _ = oracle.run_batch(rom, ref, np.full(4 * n, action, np.uint8), 4)
        s, l, term = _decode(o_obs, spec_args)
        want_r = (s - prev_s).astype(np.int32).astype(np.float32)
        assert np.array_equal(step.reward.cpu().numpy(), want_r), t
        assert np.array_equal(step.terminated.cpu().numpy(), term), t
        want_lost = (l < prev_l) if lives else np.zeros(n, bool)
        assert np.array_equal(step.life_lost.cpu().numpy(), want_lost), t
        saw_reward = saw_reward or bool((want_r != 0).any())
        prev_s, prev_l = s, l
    assert saw_reward or not score
    env.close()


def test_env_reward_table_from_file():
    """with_reward_table picks the divergence cart's entry of the shipped table
    by the ROM's SHA-256; rewards and flags equal those of the same spec given
    directly."""
    import fast_atari_b200.env as fenv
    from fa_pkg import ROOT
    rom = carts.divergence_cart().rom
    n = 48
    a = fenv.BatchAtariGpuEnv(rom, n).with_reward_table(ROOT / "fast-atari-rs_b200" / "reward_tables" / "synthetic_carts.json")
    b = fenv.BatchAtariGpuEnv(rom, n).with_reward(fa.RewardSpec.make((3, 4, 5), True, (7, 0x0C, 2), (9, 0x80, 0x80)))
    a.reset()
    b.reset()
    for action in (3, 12, 7, 17):
        sa, sb = a.step(action), b.step(action)
        assert np.array_equal(sa.reward.cpu().numpy(), sb.reward.cpu().numpy())
        assert np.array_equal(sa.terminated.cpu().numpy(), sb.terminated.cpu().numpy())
        assert np.array_equal(sa.life_lost.cpu().numpy(), sb.life_lost.cpu().numpy())
    a.close()
    b.close()
    with pytest.raises(KeyError):
        fenv.BatchAtariGpuEnv(carts.plain_cart().rom, 4).with_reward_table(
            ROOT / "fast-atari-rs_b200" / "reward_tables" / "synthetic_carts.json")
