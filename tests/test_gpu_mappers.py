"""GPU parity of the E0 and 3F bank-switching schemes (registered per ROM) and
of DPC carts (Pitfall II's scheme, picked by length).

The reference has none of these (it crashes on E0 and DPC carts), so the
oracle's restatement, pinned by the hand-checked programs of test_mappers.py,
is the checker here: full state (including the slice map and the DPC
registers) and RAM after every call, through the handle's persistent and
plain forms, every warp policy, a pool that mixes sliced and 4K-bank carts in
one launch, state upload, the server and the rendering console (which takes
E0 and 3F, and refuses DPC)."""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal, oracle_states
from test_gpu_render import check as render_check

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def sliced():
    out = {"e0": (carts.e0_cart(), "e0"), "3f16": (carts.f3_cart(16384), "3f"), "3f6": (carts.f3_cart(6144), "3f"),
           "fe": (carts.fe_cart(), "fe")}
    for c, sch in out.values():
        fa.set_rom_scheme(c.rom, sch)
        oracle.set_rom_scheme(c.rom, sch)
    yield {k: c for k, (c, _) in out.items()}
    for c, _ in out.values():
        fa.set_rom_scheme(c.rom, "auto")
        oracle.set_rom_scheme(c.rom, "auto")


@pytest.fixture(scope="module")
def dpc():
    return {"dpc": carts.dpc_cart(), "dpc_tail": carts.dpc_cart(dump_tail=True)}


@pytest.mark.parametrize("name", ["e0", "3f16", "3f6", "dpc", "dpc_tail", "fe"])
@pytest.mark.parametrize("sched", ["pc", "lane", "line", "match"])
def test_sliced_carts_match_oracle(sliced, dpc, name, sched):
    rom = (dpc[name] if name.startswith("dpc") else sliced[name]).rom
    n, k, chunk = 150, 12, 4
    acts = carts.actions(seed=21, n=n, frames=k)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, sched, False)
        obs = g.reset()
        assert np.array_equal(obs, ref["ram"])
        assert_states_equal(g.download_states(), ref, f"{name} reset")
        for f0 in range(0, k, chunk):
            obs = g.step_multi(acts[f0:f0 + chunk], chunk)
            o_obs, _ = oracle.run_batch(rom, ref, acts[f0:f0 + chunk], chunk)
            assert np.array_equal(obs, o_obs), f"{name}/{sched} frames {f0}..{f0 + chunk}"
            assert_states_equal(g.download_states(), ref, f"{name}/{sched} after {f0 + chunk}")
    maps = {int(m[0]) | int(m[1]) << 8 for m in ref["mapper"]}
    assert int(ref["scheme"][0]) in (4, 5, 6, 7)
    assert len(maps) >= 1
    if name.startswith("dpc"):                              # the cart reaches every DPC mechanism
        assert len(maps) == 2 and ref["dpc_music"].any() and (ref["dpc_music"] == 0).any()
        assert len({bytes(r) for r in ref["dpc_counter"]}) > n // 2


@pytest.mark.parametrize("block,persistent", [(256, False), (128, True)])
def test_sliced_launch_shapes_and_per_frame(sliced, block, persistent):
    rom = sliced["e0"].rom
    n, k = 500, 6
    acts = carts.actions(seed=22, n=n, frames=k)
    ref = oracle_states(rom, n)
    o_obs, _ = oracle.run_batch(rom, ref, acts, k)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(block, "pc", persistent)
        g.reset()
        for f in range(k):
            obs = g.step(acts[f])
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, f"block {block} persistent {persistent}")


def test_pool_mixes_sliced_and_4k_bank_carts(sliced, dpc):
    mixed = carts.mixed_carts()
    roms = [mixed[0].rom, sliced["e0"].rom, mixed[2].rom, sliced["3f16"].rom, sliced["3f6"].rom, mixed[3].rom,
            dpc["dpc"].rom, sliced["fe"].rom]
    counts = [300, 200, 90, 130, 64, 33, 77, 45]
    k = 5
    acts = [carts.actions(seed=50 + i, n=n, frames=k) for i, n in enumerate(counts)]
    with fa.AtariPool() as pool:
        for r, n in zip(roms, counts):
            pool.add_cart(r, n)
        obs = pool.step(acts, k)
        for g, (r, n) in enumerate(zip(roms, counts)):
            st = oracle_states(r, n)
            o, _ = oracle.run_batch(r, st, acts[g], k)
            assert np.array_equal(obs[g], o), f"group {g}"
            assert_states_equal(pool.group(g).download_states(), st, f"group {g}")


def test_sliced_state_upload_round_trip(sliced):
    rom = sliced["3f16"].rom
    n = 64
    ref = oracle_states(rom, n)
    oracle.run_batch(rom, ref, carts.actions(seed=3, n=n, frames=5), 5)
    ref["mapper"][:, 0] = np.arange(n) % 7                  # every lower bank, set by hand
    with fa.BatchAtariGpu(rom, n) as g:
        g.upload_states(ref)
        got = g.download_states()
        assert_states_equal(got, ref, "round trip")
        acts = carts.actions(seed=4, n=n, frames=3)
        obs = g.step_multi(acts, 3)
        # The oracle rebuilds its windows from the uploaded mapper field too.
        o_obs, _ = oracle.run_batch(rom, ref, acts, 3)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "continued")


def test_dpc_state_upload_round_trip(dpc):
    """DPC registers set by hand (counters, tops, bottoms, flags, music
    channels, random number, oscillator count) go up and come back unchanged,
    and running on from them matches the oracle started from the same
    states."""
    rom = dpc["dpc"].rom
    n = 96
    ref = oracle_states(rom, n)
    oracle.run_batch(rom, ref, carts.actions(seed=5, n=n, frames=3), 3)
    rng = np.random.default_rng(7)
    ref["dpc_counter"] = rng.integers(0, 2048, (n, 8))
    ref["dpc_top"] = rng.integers(0, 256, (n, 8))
    ref["dpc_bottom"] = rng.integers(0, 256, (n, 8))
    ref["dpc_flags"] = rng.integers(0, 256, n)
    ref["dpc_music"] = rng.integers(0, 8, n)
    ref["dpc_random"] = rng.integers(0, 256, n)
    ref["dpc_osc"] = rng.integers(0, 2**32, n, dtype=np.uint64)
    ref["mapper"][:, 0] = np.arange(n) % 2
    with fa.BatchAtariGpu(rom, n) as g:
        g.upload_states(ref)
        assert_states_equal(g.download_states(), ref, "round trip")
        acts = carts.actions(seed=6, n=n, frames=4)
        obs = g.step_multi(acts, 4)
        o_obs, _ = oracle.run_batch(rom, ref, acts, 4)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "continued")


def test_dpc_script_cart_matches_oracle():
    """The scripted DPC cart whose oracle run the step-by-step model of
    test_mappers.py predicts: every fetcher function, the 11-bit wrap, the
    random number generator around a reset and two music channels."""
    rom = carts.dpc_script_cart().rom
    n = 64
    ref = oracle_states(rom, n)
    acts = carts.actions(seed=8, n=n, frames=3)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        obs = g.step_multi(acts, 3)
        o_obs, _ = oracle.run_batch(rom, ref, acts, 3)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "dpc script")


def test_dpc_fields_not_taken_by_other_schemes():
    rom = carts.plain_cart().rom
    n = 40
    ref = oracle_states(rom, n)
    up = ref.copy()
    up["dpc_counter"] = 0x155
    up["dpc_bottom"] = 3
    up["dpc_flags"] = 0xFF
    up["dpc_osc"] = 99
    with fa.BatchAtariGpu(rom, n) as g:
        g.upload_states(up)
        got = g.download_states()
        assert_states_equal(got, ref, "DPC fields dropped")
        acts = carts.actions(seed=9, n=n, frames=2)
        g.step_multi(acts, 2)
        oracle.run_batch(rom, ref, acts, 2)
        assert_states_equal(g.download_states(), ref, "run on")


def test_fe_state_upload_round_trip(sliced):
    """FE bank state set by hand, armed (the last access was to $01FE) or
    not, goes up and comes back unchanged, and running on matches the oracle
    started from the same states: an armed console's first opcode fetch picks
    its bank."""
    rom = sliced["fe"].rom
    n = 64
    ref = oracle_states(rom, n)
    oracle.run_batch(rom, ref, carts.actions(seed=11, n=n, frames=2), 2)
    ref["mapper"][:, 0] = np.arange(n) % 2
    ref["mapper"][:, 1] = (np.arange(n) // 2) % 2
    with fa.BatchAtariGpu(rom, n) as g:
        g.upload_states(ref)
        assert_states_equal(g.download_states(), ref, "round trip")
        acts = carts.actions(seed=12, n=n, frames=3)
        obs = g.step_multi(acts, 3)
        o_obs, _ = oracle.run_batch(rom, ref, acts, 3)
        assert np.array_equal(obs, o_obs)
        assert_states_equal(g.download_states(), ref, "continued")


@pytest.mark.parametrize("name", ["dpc", "fe"])
def test_rendering_console_refuses_dpc_and_fe(sliced, dpc, name):
    rom = dpc["dpc"].rom if name == "dpc" else sliced["fe"].rom
    with pytest.raises(fa.FaError) as ei:
        fa.AtariRender(rom, 4)
    assert ei.value.code == fa.FA_ERR_BAD_ROM


@pytest.mark.parametrize("name", ["e0", "3f16"])
def test_sliced_rendering_console_matches_oracle(sliced, name):
    rom = sliced[name].rom
    n, k = 40, 3
    consoles = oracle.render_reset(rom, n)
    with fa.AtariRender(rom, n) as g:
        fb, ram = g.reset()
        render_check(fb, ram, g.states(), consoles, f"{name} reset")
        for c in range(2):
            acts = carts.actions(seed=70 + c, n=n, frames=k)
            fb, ram = g.step_multi(acts, k)
            oracle.render_steps(consoles, acts)
            st = g.states()
            render_check(fb, ram, st, consoles, f"{name} call {c}")
            for i, con in enumerate(consoles):
                assert int(st[i]["mapper"][0]) | int(st[i]["mapper"][1]) << 8 == con.mapper(), f"{name} mapper {i}"


def test_sliced_carts_in_the_server(sliced, dpc):
    roms = [sliced["e0"].rom, carts.mixed_carts()[1].rom, dpc["dpc"].rom, sliced["fe"].rom]
    sizes = {0: 70, 1: 40, 2: 33, 3: 50}
    reqs = [(0, 70, 3), (1, 40, 2), (2, 33, 4), (3, 50, 3), (0, 70, 2), (3, 50, 2)]
    with fa.AtariServer(roms) as srv:
        sids = {c: srv.open(c) for c in sizes}
        got = [srv.step(sids[c], carts.actions(seed=90 + i, n=n, frames=k), n, k)[0] for i, (c, n, k) in enumerate(reqs)]
        states = {c: srv.states(sids[c]) for c in sizes}
    ref = {c: oracle_states(roms[c], sizes[c]) for c in sizes}
    for i, (c, n, k) in enumerate(reqs):
        o, _ = oracle.run_batch(roms[c], ref[c], carts.actions(seed=90 + i, n=n, frames=k), k)
        assert np.array_equal(got[i], o), f"request {i}"
    for c in sizes:
        assert_states_equal(states[c], ref[c], f"cart {c}")


@pytest.mark.parametrize("name", ["e0_8k", "3f_16k", "3f_6k", "dpc_10k", "fe_8k"])
def test_sliced_carts_match_committed_golden_vectors(sliced, dpc, name):
    """The frozen oracle vectors of tests/golden/ (RAM at checkpoint frames and
    the full final state, mapper field included), without running the oracle."""
    import hashlib
    import json
    from pathlib import Path
    from make_golden import state_sha
    want = json.loads((Path(__file__).parent / "golden" / "oracle_vectors.json").read_text())[name]
    rom = {"e0_8k": sliced["e0"], "3f_16k": sliced["3f16"], "3f_6k": sliced["3f6"], "dpc_10k": dpc["dpc"],
           "fe_8k": sliced["fe"]}[name].rom
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
