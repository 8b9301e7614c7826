"""Random ROMs and random CPU states on the GPU against the oracle.

Every ROM size the reference accepts (2K/4K Fixed, 8K F8, 16K F6, 32K F4),
random bytes with the reset vector in each bank pointing at $F000, and
instances started from random A/X/Y/SP/P, a random pc in $F000-$FFFF and
random RAM.  Execution wanders through illegal opcodes (the instance halts
with FA_STATUS_ILLEGAL_OPCODE), stack pages in the TIA (SP below $80 pushes
into TIA registers, VSYNC and WSYNC included), bank hotspots hit by phantom
and real accesses, PIA timer writes, and frames that end at the 100,000-cycle
cap: the full state must match the oracle's after every call, and varied
actions keep reaching halted instances (set_action precedes run_frame, which
does nothing for them).
"""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa
from test_gpu_parity import assert_states_equal
from test_gpu_render import check as render_check

pytestmark = pytest.mark.gpu

SIZES = [2048, 4096, 8192, 16384, 32768]


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


def random_rom(rng, size):
    rom = bytearray(rng.integers(0, 256, size, dtype=np.uint8).tobytes())
    for b in range(max(1, size // 4096)):
        base = b * 4096 + min(size, 4096) - 4
        rom[base:base + 2] = bytes([0x00, 0xF0])
    return bytes(rom)


def random_states(rng, rom, n):
    st = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
    st["a"] = rng.integers(0, 256, n)
    st["x"] = rng.integers(0, 256, n)
    st["y"] = rng.integers(0, 256, n)
    st["sp"] = rng.integers(0, 256, n)
    st["status"] = rng.integers(0, 256, n) & 0xCF
    st["pc"] = 0xF000 + rng.integers(0, 0x1000, n)
    st["ram"] = rng.integers(0, 256, (n, 128))
    st["run_status"] = 0
    return st


@pytest.mark.parametrize("sched", ["pc", "lane", "match"])
@pytest.mark.parametrize("size", SIZES)
def test_random_roms_and_states(size, sched):
    rng = np.random.default_rng(size * 7 + len(sched))
    n, calls, k = 256, 2, 2
    for t in range(3):
        rom = random_rom(rng, size)
        start = random_states(rng, rom, n)
        ref = start.copy()
        with fa.BatchAtariGpu(rom, n) as g:
            g.set_launch(128, sched, True)
            g.reset()
            g.upload_states(start)
            for c in range(calls):
                acts = carts.actions(seed=100 * t + c, n=n, frames=k)
                obs = g.step_multi(acts, k)
                o, _ = oracle.run_batch(rom, ref, acts, k)
                assert np.array_equal(obs, o), f"{size}/{sched} rom {t} call {c}: RAM"
                assert_states_equal(g.download_states(), ref, f"{size}/{sched} rom {t} call {c}")


def test_halted_instances_take_later_actions():
    """A cart whose init runs into an illegal opcode, stepped with varied
    actions: the halted instances' input pins hold each call's last action,
    as the oracle's set_action-then-run_frame order leaves them."""
    rom = bytearray([0xEA] * 4096)
    rom[0:6] = bytes([0xA9, 0x02, 0x85, 0x00, 0xE8, 0x02])      # LDA #2; STA VSYNC; INX; illegal
    rom[0xFFC:0xFFE] = bytes([0x00, 0xF0])
    rom = bytes(rom)
    n = 40
    ref = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        for c in range(3):
            acts = carts.actions(seed=40 + c, n=n, frames=3)
            g.step_multi(acts, 3)
            oracle.run_batch(rom, ref, acts, 3)
            st = g.download_states()
            assert_states_equal(st, ref, f"call {c}")
    assert (st["run_status"] & fa.FA_STATUS_ILLEGAL_OPCODE).all()
    assert len(np.unique(st["port_a_input"])) > 1


def test_halted_consoles_take_later_actions_rendering():
    """The same for the rendering console: its TIA's INPT4 and paddle0 hold
    each call's last action (compared with every other field by check)."""
    rom = bytearray([0xEA] * 4096)
    rom[0:6] = bytes([0xA9, 0x02, 0x85, 0x00, 0xE8, 0x02])
    rom[0xFFC:0xFFE] = bytes([0x00, 0xF0])
    rom = bytes(rom)
    n = 33
    consoles = oracle.render_reset(rom, n)
    with fa.AtariRender(rom, n) as g:
        g.reset()
        for c in range(2):
            acts = carts.actions(seed=9 + c, n=n, frames=3)
            fb, ram = g.step_multi(acts, 3)
            oracle.render_steps(consoles, acts)
            st = g.states()
            render_check(fb, ram, st, consoles, f"halted consoles, call {c}")
    assert (st["run_status"] & fa.FA_STATUS_ILLEGAL_OPCODE).all()
    assert len(np.unique(st["paddle0"])) > 1
