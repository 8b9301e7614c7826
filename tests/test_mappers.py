"""Bank-switching schemes the reference lacks (E0, 3F), checked without a GPU.

The reference picks a scheme from the ROM length alone (BankScheme::detect,
src/atari.rs:96-105), so an 8K Parker Brothers E0 cart runs as F8 there and
crashes (montezuma_revenge and tutankham in bench_all_fast_atari.json).  The
library and the oracle take a scheme registered per ROM image instead.
These tests pin the oracle's E0 and 3F restatement on small hand-written
programs whose expected RAM is worked out from the ROM bytes, then check the
registry and the content guess through the C ABI (host code only)."""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa


def _program(origin, body, size, vectors_at=None):
    a = carts.Asm(origin)
    a.label("reset")
    for ins in body:
        a.ins(*ins)
    a.label("spin")
    a.ins("LDA", "imm", 0x02)
    a.ins("STA", "zp", carts.VSYNC)                 # ends the frame
    a.ins("JMP", "abs", "spin")
    img, labels, _ = a.assemble(size)
    return bytearray(img), labels


def _e0_rom():
    # Slice k holds the byte 0x10 + k at offset 0 and 0x20 + k at offset 0x3FF.
    rom = bytearray(8192)
    for k in range(8):
        rom[k * 1024] = 0x10 + k
        rom[k * 1024 + 0x3FF] = 0x20 + k
    body = [
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x80),      # power-on: window 0 = slice 4
        ("LDA", "abs", 0xFFE1), ("LDA", "abs", 0xF000), ("STA", "zp", 0x81),   # read hotspot: slice 1 -> window 0
        ("STA", "abs", 0xFFEB), ("LDA", "abs", 0xF400), ("STA", "zp", 0x82),   # write hotspot: slice 3 -> window 1
        ("LDX", "imm", 6), ("LDA", "absx", 0xFFF0),                             # abs,X at $FFF6: slice 6 -> window 2
        ("LDA", "abs", 0xFBFF), ("STA", "zp", 0x83),
        ("BIT", "abs", 0xFFE7), ("LDA", "abs", 0xF3FF), ("STA", "zp", 0x84),  # BIT: slice 7 -> window 0
        ("LDA", "abs", 0xFFF8), ("LDA", "abs", 0xF000), ("STA", "zp", 0x85),   # $FFF8 is not an E0 hotspot
    ]
    img, labels = _program(0xFC00, body, 1024)
    img[0x3FC:0x3FE] = bytes([0x00, 0xFC])
    rom[7 * 1024:8 * 1024] = img
    # slice 7's own offset-0 byte is the first opcode; keep the markers of slices 0-6
    return bytes(rom)


def test_oracle_e0_hotspots_map_slices():
    rom = _e0_rom()
    oracle.set_rom_scheme(rom, "e0")
    try:
        st = oracle.reset_state(rom)
    finally:
        oracle.set_rom_scheme(rom, "auto")
    ram = st["ram"]
    assert ram[0] == 0x14                                   # window 0 at power-on: slice 4
    assert ram[1] == 0x11                                   # $1FE1 read: slice 1
    assert ram[2] == 0x13                                   # $1FEB write: slice 3 in window 1
    assert ram[3] == 0x26                                   # $1FF6 via abs,X: slice 6 in window 2
    assert ram[4] == rom[7 * 1024 + 0x3FF]                  # slice 7 in window 0 reads slice 7's last byte
    assert ram[5] == rom[7 * 1024]                          # F8 hotspot address: no change
    m = int(st["mapper"][0]) | int(st["mapper"][1]) << 8
    assert m == 7 | 3 << 4 | 6 << 8
    assert int(st["bank"]) == 0 and int(st["scheme"]) == 4


def _3f_rom(n2k):
    rom = bytearray(2048 * n2k)
    for b in range(n2k):
        rom[b * 2048] = 0x40 + b
    body = [
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x80),       # power-on: bank 0
        ("LDA", "imm", n2k + 1), ("STA", "zp", 0x3F),      # bank (n+1) mod n = 1
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x81),
        ("LDX", "imm", 2 * n2k - 1), ("STX", "zp", 0x3F),  # (2n-1) mod n = n-1: the last bank below too
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x82),
        ("LDA", "imm", 0), ("STA", "zp", 0x09),            # COLUBK write: bank 0
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x83),
        ("LDA", "imm", 1), ("STA", "zp", 0x40),            # $40 is past the select range
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x84),
        ("LDA", "imm", 1), ("STA", "abs", 0x1FFF),          # ROM-space write: nothing
        ("LDA", "abs", 0xF000), ("STA", "zp", 0x85),
        ("LDA", "abs", 0xFFFD), ("STA", "zp", 0x86),       # the fixed last 2K
    ]
    img, labels = _program(0xF800, body, 2048)
    img[0x7FC:0x7FE] = bytes([0x00, 0xF8])
    rom[(n2k - 1) * 2048:] = img
    return bytes(rom)


@pytest.mark.parametrize("n2k", [3, 4, 16])
def test_oracle_3f_writes_select_banks(n2k):
    rom = _3f_rom(n2k)
    oracle.set_rom_scheme(rom, "3f")
    try:
        st = oracle.reset_state(rom)
    finally:
        oracle.set_rom_scheme(rom, "auto")
    ram = st["ram"]
    last = rom[(n2k - 1) * 2048]
    assert list(ram[:7]) == [0x40, 0x41, last, 0x40, 0x40, 0x40, 0xF8]
    assert int(st["mapper"][0]) == 2 % n2k and int(st["scheme"]) == 5   # the frame-ending STA VSYNC (A = 2) selects too


def test_oracle_rejects_lengths_a_scheme_cannot_hold():
    with pytest.raises(ValueError):
        oracle.set_rom_scheme(bytes(4096), "e0")
    with pytest.raises(ValueError):
        oracle.set_rom_scheme(bytes(3000), "3f")
    with pytest.raises(ValueError):
        oracle.set_rom_scheme(bytes(8192), "f6")


def test_oracle_sliced_carts_run_and_diverge():
    for c, sch in ((carts.e0_cart(), "e0"), (carts.f3_cart(16384), "3f"), (carts.f3_cart(6144), "3f")):
        oracle.set_rom_scheme(c.rom, sch)
        st = oracle.reset_state(c.rom)
        states = np.array([st] * 8, dtype=oracle.STATE_DTYPE)
        obs, instr = oracle.run_batch(c.rom, states, carts.actions(seed=2, n=8, frames=3), 3)
        assert (states["run_status"] == 0).all(), c.spec.name
        assert instr > 8 * 3 * 5000, c.spec.name
        assert len({o.tobytes() for o in obs}) == 8, c.spec.name          # the actions show in RAM
        # Under the size rule the same bytes run as a different machine.
        oracle.set_rom_scheme(c.rom, "auto")
        if len(c.rom) in (8192, 16384):
            st2 = oracle.reset_state(c.rom)
            assert int(st2["scheme"]) != int(st["scheme"])


def test_library_registry_and_guess():
    e0, f3 = carts.e0_cart(), carts.f3_cart(16384)
    assert fa.rom_scheme(e0.rom) == 1                        # F8 by size, as in the reference
    assert fa.guess_rom_scheme(e0.rom) == 4
    assert fa.guess_rom_scheme(f3.rom) == 5
    assert fa.guess_rom_scheme(carts.divergence_cart().rom) == 1
    for c in carts.mixed_carts():
        assert fa.guess_rom_scheme(c.rom) == fa.rom_scheme(c.rom)
    fa.set_rom_scheme(e0.rom, "e0")
    try:
        assert fa.rom_scheme(e0.rom) == 4
        assert fa.rom_scheme(e0.rom[:-1] + b"\x00" if e0.rom[-1] else e0.rom[:-1] + b"\x01") == 1
    finally:
        fa.set_rom_scheme(e0.rom, "auto")
    assert fa.rom_scheme(e0.rom) == 1
    with pytest.raises(fa.FaError) as ei:
        fa.set_rom_scheme(bytes(6000), "3f")
    assert ei.value.code == fa.FA_ERR_BAD_ROM
    fa.set_rom_scheme(bytes(6144), "3f")
    try:
        assert fa.rom_scheme(bytes(6144)) == 5
    finally:
        fa.set_rom_scheme(bytes(6144), "auto")
    with pytest.raises(fa.FaError):
        fa.rom_scheme(bytes(6144))                           # no size-rule scheme for 6K


def test_guess_rarely_fires_on_random_bytes():
    # Data regions look like code to a byte scan; the guess stays a hint.
    rng = np.random.default_rng(7)
    for size, by_size in ((4096, 0), (8192, 1), (16384, 2)):
        wrong = sum(fa.guess_rom_scheme(rng.integers(0, 256, size, dtype=np.uint8).tobytes()) != by_size
                    for _ in range(200))
        assert wrong <= 10, (size, wrong)


def test_guess_and_scheme_of_tiny_roms():
    for n in (1, 2, 3, 4):
        rom = bytes(range(1, n + 1))
        assert fa.guess_rom_scheme(rom) == 0                 # Fixed, mirrored: the size rule
        assert fa.rom_scheme(rom) == 0


def test_registry_is_safe_across_threads():
    import threading
    roms = [bytes([i]) * 8192 for i in range(16)]
    errors = []

    def worker(k):
        try:
            for rep in range(200):
                rom = roms[(k + rep) % len(roms)]
                fa.set_rom_scheme(rom, "e0" if rep % 2 else "auto")
                assert fa.rom_scheme(rom) in (1, 4)
        except Exception as e:                       # surfaced below
            errors.append(e)

    ts = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    for rom in roms:
        fa.set_rom_scheme(rom, "auto")
        assert fa.rom_scheme(rom) == 1
