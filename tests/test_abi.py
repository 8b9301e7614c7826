"""C ABI checks that need no GPU: the library loads, exports every symbol the
public header declares, and its state layout matches the header and the
oracle's restatement of the reference AtariStateGpu (src/cuda_env.rs:10-38)."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

from fa_pkg import ROOT, fa
import oracle

HEADER = ROOT / "include" / "fast_atari.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(fa.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (fa_[a-z0-9_]+)$", out, flags=re.M))
    missing = [s for s in declared_functions() if s not in exported]
    assert not missing, missing
    assert len(declared_functions()) >= 20


def test_binding_covers_header():
    assert set(declared_functions()) == set(fa._SIGS)


def test_library_loads_and_reports_version():
    L = fa.lib()
    assert b"sm_100a" in L.fa_version()


def test_state_dtype_matches_oracle_and_header():
    assert fa.STATE_DTYPE == oracle.STATE_DTYPE
    assert oracle.lib().orc_state_size() == 280
    off = {n: fa.STATE_DTYPE.fields[n][1] for n in fa.STATE_DTYPE.names}
    # offsets pinned by FA_STATIC_ASSERT in include/fast_atari.h
    assert (off["ram"], off["timer_value"], off["tia_clock"], off["paddle_counter"],
            off["pos_p0"], off["bank"], off["cycles"], off["run_status"]) == (8, 142, 152, 172, 176, 217, 224, 236)
    # the reference AtariStateGpu prefix ends at its _pad_end (221 bytes)
    assert off["_pad_end"] + 2 == 221


def test_no_device_fails_loudly():
    if fa.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(fa.FaError) as ei:
        fa.BatchAtariGpu(bytes(4096), 4)
    assert ei.value.code == -4


def test_bad_rom_lengths_rejected_before_device():
    # fa_create validates the ROM before touching the device only when one
    # exists; without one it reports no-device.  The oracle rejects the same
    # lengths the reference's HeadlessBus::new panics on.
    for n in (0, 5000, 9000, 20000):
        with pytest.raises(ValueError):
            oracle.Atari(bytes(n))
    for n in (1, 2048, 4096, 8192, 16384, 32768, 40000):
        oracle.Atari(bytes([0xEA] * n))


def test_server_without_device_fails_loudly():
    if fa.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(fa.FaError) as ei:
        fa.AtariServer([bytes(4096)])
    assert ei.value.code == -4


def test_reward_spec_rejected_before_any_device_work():
    # Invalid specs fail in host code, before a launch; the fake device
    # pointers are never dereferenced.
    L = fa.lib()
    fake = 4096
    for kw in ({"score": (1, 2, 3, 4, 5)}, {"score": (200,)}, {"lives": (130, 1, 0)}, {"lives": (1, 1, 9)},
               {"terminal": (128, 1, 1)}):
        sp = fa.RewardSpec()
        if "score" in kw:
            sc = kw["score"]
            for i, a in enumerate(sc[:4]):
                sp.score_addr[i] = a
            sp.score_bytes = len(sc)
        if "lives" in kw:
            sp.lives_addr, sp.lives_mask, sp.lives_shift = kw["lives"]
        if "terminal" in kw:
            sp.terminal_addr, sp.terminal_mask, sp.terminal_value = kw["terminal"]
        rc = L.fa_obs_reward(fa._vp(fake), 8, ctypes.byref(sp), 0, fa._vp(fake), fa._vp(fake), None, None, None)
        assert rc == -1, (kw, rc)                     # FA_ERR_INVALID


def test_wait_limit_setting_is_bounded():
    """fa_set_wait_limit_ns: host-side only (no device needed); 0..10 s."""
    assert fa.wait_limit_ns() == 2_000_000_000
    with pytest.raises(fa.FaError):
        fa.set_wait_limit_ns(10_000_000_001)
    assert fa.wait_limit_ns() == 2_000_000_000
    fa.set_wait_limit_ns(0)
    assert fa.wait_limit_ns() == 0
    fa.set_wait_limit_ns(2_000_000_000)


def test_palette_rgba_matches_the_oracle_for_every_index():
    """fa_palette_rgba (the device's packed 64-colour table) equals the oracle's
    restatement of ntsc_palette (src/atari.rs:624-645, 128 entries indexed by
    (index >> 1) & 0x7F) for all 256 palette indices; two entries by hand."""
    want = oracle.rgba(np.arange(256, dtype=np.uint8))
    got = np.array([fa.palette_rgba(i) for i in range(256)], np.uint8)
    assert np.array_equal(got, want)
    assert tuple(got[0x1E]) == (20, 0, 132, 255) and tuple(got[0xFC]) == (0, 116, 0, 255)
