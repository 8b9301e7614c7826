"""Phantom bus accesses and the reference's instruction KATs, on the GPU.

1. Phantom-access carts (carts.phantom_cart): 4K Fixed and F8/F6/F4 carts
   whose lines put the fix-up reads of indexed accesses, the next-pc and
   page-crossing reads of taken branches, RTS's read of the pulled address,
   and read-modify-write's first write on bank hotspots, an INTIM mirror
   just after a timer underflow, and GRP0/GRP1/ENABL under vertical delay
   (src/cpu.rs:415-1135, src/atari.rs:460-552, src/pia.rs:169-228,
   src/headless_tia.rs:225-298).  The full state is compared with the oracle
   after every frame, under every warp policy, in the 4K-bank build (a
   handle) and in the build that holds both cores (a pool that also holds an
   E0 cart).  test_phantom_carts_depend_on_phantom_accesses (CPU) shows the
   same carts give different states when the oracle skips those accesses.

2. The 29 known-answer tests of tests/cycle_counts.rs:38-366, with the
   values written in that file, relocated to the 2600 bus as kat_2600.py
   describes, plus decimal mode and the JMP (ind) page wrap.  Registers, pc
   and cycle counts are checked against the file's values, and the whole
   state against the oracle, under every warp policy and both builds.
"""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from kat_2600 import KATS, check_kat, kat_start_state
from test_gpu_parity import assert_states_equal, oracle_states

pytestmark = pytest.mark.gpu

POLICIES = ["lane", "pc", "line", "match"]


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


@pytest.fixture(scope="module")
def phantom():
    return {c.spec.name: c for c in carts.phantom_carts()}


@pytest.fixture(scope="module")
def e0():
    c = carts.e0_cart()
    fa.set_rom_scheme(c.rom, "e0")
    oracle.set_rom_scheme(c.rom, "e0")
    yield c
    fa.set_rom_scheme(c.rom, "auto")
    oracle.set_rom_scheme(c.rom, "auto")


PHANTOM_NAMES = [c.spec.name for c in carts.phantom_carts()]


# ---------------------------------------------------------------- phantom carts
@pytest.mark.parametrize("sched", POLICIES)
@pytest.mark.parametrize("name", PHANTOM_NAMES)
def test_phantom_cart_4k_bank_build(phantom, name, sched):
    rom = phantom[name].rom
    n, frames = 96, 8
    acts = carts.actions(seed=31, n=n, frames=frames)
    ref = oracle_states(rom, n)
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, sched, True)
        obs = g.reset()
        assert np.array_equal(obs, ref["ram"])
        for f in range(frames):
            obs = g.step(acts[f])
            o_obs, _ = oracle.run_batch(rom, ref, acts[f:f + 1], 1)
            assert np.array_equal(obs, o_obs), f"{name}/{sched} frame {f}: RAM"
            assert_states_equal(g.download_states(), ref, f"{name}/{sched} frame {f}")
    assert len(np.unique(ref["bank"])) >= (2 if "row" in name else 1)


@pytest.mark.parametrize("sched", POLICIES)
def test_phantom_carts_both_cores_build(phantom, e0, sched):
    """Every phantom cart beside an E0 cart in one pool launch (the kernel
    build that holds the 4K-bank and the sliced cores), one frame per call."""
    roms = [phantom[nm].rom for nm in PHANTOM_NAMES] + [e0.rom]
    counts = [40 + 7 * i for i in range(len(roms))]
    frames = 6
    acts = [carts.actions(seed=60 + i, n=n, frames=frames) for i, n in enumerate(counts)]
    refs = [oracle_states(r, n) for r, n in zip(roms, counts)]
    with fa.AtariPool() as pool:
        for r, n in zip(roms, counts):
            pool.add_cart(r, n)
        for gi in range(len(roms)):
            pool.set_group(gi, sched)
        for f in range(frames):
            obs = pool.step([a[f:f + 1] for a in acts], 1)
            for gi, (r, ref) in enumerate(zip(roms, refs)):
                o, _ = oracle.run_batch(r, ref, acts[gi][f:f + 1], 1)
                assert np.array_equal(obs[gi], o), f"group {gi} frame {f}"
                assert_states_equal(pool.group(gi).download_states(), ref, f"{sched} group {gi} frame {f}")


@pytest.mark.parametrize("sched", POLICIES)
def test_reference_kats_on_gpu_4k_bank_build(sched):
    n = 33
    for k in KATS:
        rom = k.image()
        start = np.repeat(kat_start_state(k, rom), n)
        ref = start.copy()
        oracle.run_batch(rom, ref, np.zeros((1, n), np.uint8), 1)
        check_kat(k, ref[0], "oracle")
        with fa.BatchAtariGpu(rom, n) as g:
            g.set_launch(128, sched, True)
            g.reset()
            g.upload_states(start)
            g.step(np.zeros(n, np.uint8), obs=False)
            st = g.download_states()
        assert_states_equal(st, ref, f"{k.name}/{sched}")
        for i in (0, n - 1):
            check_kat(k, st[i], f"gpu/{sched}")


@pytest.mark.parametrize("sched", POLICIES)
def test_reference_kats_on_gpu_both_cores_build(e0, sched):
    """The KAT carts in pools of 15 beside an E0 cart (the build holding both cores)."""
    n = 32
    for first in range(0, len(KATS), 15):
        chunk = KATS[first:first + 15]
        roms = [k.image() for k in chunk]
        starts = [np.repeat(kat_start_state(k, r), n) for k, r in zip(chunk, roms)]
        with fa.AtariPool() as pool:
            for r in roms:
                pool.add_cart(r, n)
            pool.add_cart(e0.rom, n)
            for gi in range(len(roms) + 1):
                pool.set_group(gi, sched)
            for gi, s in enumerate(starts):
                pool.group(gi).upload_states(s)
            pool.step([np.zeros(n, np.uint8)] * (len(roms) + 1), 1, obs=False)
            for gi, (k, r, s) in enumerate(zip(chunk, roms, starts)):
                ref = s.copy()
                oracle.run_batch(r, ref, np.zeros((1, n), np.uint8), 1)
                st = pool.group(gi).download_states()
                assert_states_equal(st, ref, f"{k.name}/{sched} (both cores)")
                check_kat(k, st[0], f"gpu both/{sched}")
