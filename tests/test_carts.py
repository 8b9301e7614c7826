"""Synthetic carts: determinism, structure, and the generator self-check
(every cart runs 10^4 frames in the oracle with no illegal opcode, no VSYNC
budget stop and no cycle cap)."""
import json
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np
import pytest

import oracle
from fa_pkg import carts

GOLDEN = json.loads((Path(__file__).parent / "golden" / "oracle_vectors.json").read_text())


def all_carts():
    return {"plain": carts.plain_cart(), "divergence": carts.divergence_cart(),
            "scale": carts.scale_cart(), **{c.spec.name: c for c in carts.mixed_carts()}}


def test_rom_bytes_are_reproducible():
    import hashlib
    for name, c in all_carts().items():
        assert hashlib.sha256(c.rom).hexdigest() == GOLDEN[name]["rom_sha256"], name


def test_rom_sizes_and_vectors():
    for name, c in all_carts().items():
        rom = c.rom
        assert len(rom) == c.spec.rom_size
        bank = min(len(rom), 4096)
        for b in range(max(1, len(rom) // 4096)):
            vec = rom[b * 4096 + bank - 4: b * 4096 + bank - 2]
            assert vec == bytes([0x00, 0xF0]), (name, b)


def test_only_legal_opcodes_reachable_statically():
    # every opcode byte the assembler emitted is legal (operands may be anything)
    assert len(carts.LEGAL_OPCODES) == 151


def test_actions_counter_based():
    a = carts.actions(seed=5, n=100, frames=20)
    b = carts.actions(seed=5, n=100, frames=10, frame0=10)
    assert a.shape == (20, 100) and a.dtype == np.uint8 and a.max() < 18
    assert np.array_equal(a[10:], b)
    assert len(np.unique(a)) == 18


def _run_long(args):
    c, frames = args
    st = np.array([oracle.reset_state(c.rom)] * 2, dtype=oracle.STATE_DTYPE)
    oracle.run_batch(c.rom, st, carts.actions(seed=77, n=2, frames=frames), frames, nthreads=2)
    return c.spec.name, st


def test_generator_self_check_10k_frames():
    cs = list(all_carts().values())
    with ThreadPoolExecutor(max_workers=len(cs)) as ex:
        for name, st in ex.map(_run_long, [(c, 10_000) for c in cs]):
            assert (st["run_status"] == 0).all(), (name, st["run_status"])
            assert (st["frame_no"] == 10_000).all(), name


def test_carts_exercise_the_mappers():
    """Bank switching happens.  Every banked cart has its trampoline (BIT of a
    hotspot) at the same address in every bank, followed by byte-identical
    skeleton code; the 32K F4 cart (12 switches per frame over 8 banks) ends
    consecutive frames in different banks."""
    for c in [carts.divergence_cart(), carts.scale_cart()] + carts.mixed_carts()[1:]:
        nb = c.spec.nbanks
        ge = c.labels["group_end"] - 0xF000
        hot = {2: 0xFFF8, 4: 0xFFF6, 8: 0xFFF4}[nb]
        banks = [c.rom[b * 4096:(b + 1) * 4096] for b in range(nb)]
        tail = c.labels["vis_done"] - 0xF000
        for bk in banks:
            code = bk[ge:tail]
            targets = [code[i + 1] | (code[i + 2] << 8) for i in range(len(code) - 2) if code[i] == 0x2C]
            assert any(hot <= t < hot + nb for t in targets), c.spec.name
        assert len({bk[tail:tail + 21] for bk in banks}) == 1, c.spec.name   # overscan skeleton
    c = carts.mixed_carts()[3]
    st = np.array([oracle.reset_state(c.rom)] * 4, dtype=oracle.STATE_DTYPE)
    seen = set()
    for f in range(4):
        oracle.run_batch(c.rom, st, carts.actions(seed=3, n=4, frames=1, frame0=f), 1)
        seen.update(int(b) for b in st["bank"])
    assert len(seen) >= 2, seen


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_matches_frozen_vectors(name):
    import sys
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    import make_golden
    got = make_golden.vectors(name)
    want = GOLDEN[name]
    for key in ("rom_sha256", "reset_state_sha256", "ram_sha256_at", "final_state_sha256", "instructions"):
        assert got[key] == want[key], (name, key)


# ---------------------------------------------------------------- phantom-access carts
def test_phantom_carts_run_2k_frames_without_a_halt():
    """The phantom-access carts (every bank the same code) never reach an
    illegal opcode, the VSYNC budget or the cycle cap."""
    cs = carts.phantom_carts()
    with ThreadPoolExecutor(max_workers=len(cs)) as ex:
        for name, st in ex.map(_run_long, [(c, 2_000) for c in cs]):
            assert (st["run_status"] == 0).all(), (name, st["run_status"])
            assert (st["frame_no"] == 2_000).all(), name


def test_phantom_carts_banks_identical_but_the_id_byte():
    for c in carts.phantom_carts():
        nb = c.spec.nbanks
        off = carts.PHANTOM_BANKID - 0xF000
        banks = [bytearray(c.rom[b * 4096:(b + 1) * 4096]) for b in range(nb)]
        assert [bk[off] for bk in banks] == [0x30 + 0x11 * b for b in range(nb)], c.spec.name
        for bk in banks:
            bk[off] = 0
        assert len({bytes(bk) for bk in banks}) == 1, c.spec.name


@pytest.mark.parametrize("c", carts.phantom_carts(), ids=lambda c: c.spec.name)
def test_phantom_carts_depend_on_phantom_accesses(c):
    """With the oracle's phantom reads and first RMW writes switched off (as
    a core that skips them would run), every instance ends in a different
    state: the carts detect a core that drops those accesses."""
    n, k = 32, 6
    acts = carts.actions(seed=11, n=n, frames=k)
    st_on = np.array([oracle.reset_state(c.rom)] * n, dtype=oracle.STATE_DTYPE)
    oracle.run_batch(c.rom, st_on, acts, k)
    with oracle.phantoms_off():
        st_off = np.array([oracle.reset_state(c.rom)] * n, dtype=oracle.STATE_DTYPE)
        oracle.run_batch(c.rom, st_off, acts, k)
    differs = np.zeros(n, bool)
    for f in oracle.COMPARED_FIELDS:
        differs |= (st_on[f] != st_off[f]).reshape(n, -1).any(axis=1)
    assert differs.all()
    assert not np.array_equal(st_on["grp0_old"], st_off["grp0_old"])      # RMW double write
    assert not np.array_equal(st_on["ram"], st_off["ram"])
    if c.spec.nbanks > 1:
        assert not np.array_equal(st_on["bank"], st_off["bank"]) or "rts" in c.spec.name
