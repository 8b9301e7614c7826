"""Bank-switching schemes the reference lacks (E0, 3F, DPC), checked without a GPU.

The reference picks a scheme from the ROM length alone (BankScheme::detect,
src/atari.rs:96-105), so an 8K Parker Brothers E0 cart runs as F8 there and
crashes (montezuma_revenge and tutankham in bench_all_fast_atari.json).  The
library and the oracle take a scheme registered per ROM image instead.
These tests pin the oracle's E0 and 3F restatement on small hand-written
programs whose expected RAM is worked out from the ROM bytes, then check the
registry and the content guess through the C ABI (host code only).  DPC
carts (Pitfall II, 10,240 or 10,495 bytes, which the reference's size rule
cannot construct: pitfall2 in bench_all_fast_atari.json) are picked by
length; the oracle's DPC is pinned against a second, step-by-step model of
the chip on a scripted cart."""
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


# ------------------------------------------------------------------ DPC
class DpcModel:
    """Pitfall II's DPC chip, restated a second time and step by step, as the
    check of the oracle's DPC: the music channels are clocked one oscillator
    clock at a time (the oracle and the device count many clocks in closed
    form), and the rules are written out again from their description:
    - reads of $1000-$103F: fetcher a & 7, function (a >> 3) & 7; music
      first brought up to the instruction's start cycle t (oscillator clock
      t * 60000 // 3579545), the random number generator stepped, a fetcher
      that is no music channel sets its flag at counter low byte == top, else
      clears it at == bottom; functions 0 (random number for fetchers 0-3,
      else the music amplitude 4/5/6 per sounding channel 5/6/7), 1 (display
      byte 2047 - counter), 2 (display byte AND flag), 7 (flag), else 0; then
      the counter (11 bits) counts down unless the fetcher is a music channel;
    - writes of $1040-$107F: music brought up to date; 0 top (flag cleared),
      1 bottom, 2 counter low, 3 counter high three bits (+ music mode from
      bit 4 for fetchers 5-7), 6 random number := 1;
    - a music clock counts the low byte down, the clock after 0 reloads top;
      after clocks were counted, a channel's flag is set while low > bottom."""

    def __init__(self, display):
        self.display = display
        self.counter = [0] * 8
        self.top = [0] * 8
        self.bottom = [0] * 8
        self.flag = [0] * 8
        self.music = [0] * 3
        self.random = 1
        self.osc = 0

    def update(self, t):
        now = (t * 60000 // 3579545) & 0xFFFFFFFF
        clocks = (now - self.osc) & 0xFFFFFFFF
        self.osc = now
        if not clocks:
            return
        for m in range(3):
            if not self.music[m]:
                continue
            f = 5 + m
            low = self.counter[f] & 0xFF
            for _ in range(clocks):
                low = self.top[f] if low == 0 else low - 1
            self.counter[f] = (self.counter[f] & 0x700) | low
            self.flag[f] = 1 if low > self.bottom[f] else 0

    def read(self, a, t):
        k, fn = a & 7, (a >> 3) & 7
        music = k >= 5 and self.music[k - 5]
        self.update(t)
        r = self.random
        feedback = 1 - (((r >> 7) ^ (r >> 5) ^ (r >> 4) ^ (r >> 3)) & 1)
        self.random = ((r << 1) | feedback) & 0xFF
        if not music:
            low = self.counter[k] & 0xFF
            if low == self.top[k]:
                self.flag[k] = 1
            elif low == self.bottom[k]:
                self.flag[k] = 0
        data = self.display[2047 - self.counter[k]]
        flag = 0xFF if self.flag[k] else 0
        if fn == 0:
            v = self.random if k < 4 else sum(4 + m for m in range(3) if self.music[m] and self.flag[5 + m])
        else:
            v = {1: data, 2: data & flag, 7: flag}.get(fn, 0)
        if not music:
            self.counter[k] = (self.counter[k] - 1) & 0x7FF
        return v

    def write(self, a, v, t):
        k, fn = a & 7, (a >> 3) & 7
        self.update(t)
        if fn == 0:
            self.top[k] = v
            self.flag[k] = 0
        elif fn == 1:
            self.bottom[k] = v
        elif fn == 2:
            self.counter[k] = (self.counter[k] & 0x700) | v
        elif fn == 3:
            self.counter[k] = ((v & 7) << 8) | (self.counter[k] & 0xFF)
            if k >= 5:
                self.music[k - 5] = (v >> 4) & 1
        elif fn == 6:
            self.random = 1


def test_oracle_dpc_matches_a_step_by_step_model():
    """dpc_script_cart runs carts.dpc_script() straight-line in its second
    frame; the model replays the same accesses at the same instruction start
    cycles (LDA # 2, STA abs 4, LDA abs 4, STA zp 3, NOP 2) and must predict
    every value read and every DPC register the oracle ends with."""
    c = carts.dpc_script_cart()
    st = np.array([oracle.reset_state(c.rom)], dtype=oracle.STATE_DTYPE)
    assert int(st["scheme"][0]) == 6 and int(st["mapper"][0][0]) == 1 and int(st["dpc_random"][0]) == 1
    t = int(st["cycles"][0]) + 2 + 3                       # the frame's LDA #0 / STA VSYNC
    oracle.run_batch(c.rom, st, np.zeros((1, 1), np.uint8), 1)
    m = DpcModel([carts.dpc_display_byte(i) for i in range(2048)])
    want = []
    for step in carts.dpc_script():
        if step[0] == "w":
            t += 2
            m.write(step[1], step[2], t)
            t += 4
        elif step[0] == "r":
            want.append(m.read(step[1], t))
            t += 4 + 3
        else:
            t += 2 * step[1]
    got = [int(x) for x in st["ram"][0][:len(want)]]
    assert got == want
    assert [int(x) for x in st["dpc_counter"][0]] == m.counter
    assert [int(x) for x in st["dpc_top"][0]] == m.top
    assert [int(x) for x in st["dpc_bottom"][0]] == m.bottom
    assert int(st["dpc_flags"][0]) == sum(f << k for k, f in enumerate(m.flag))
    assert int(st["dpc_music"][0]) == sum(b << i for i, b in enumerate(m.music))
    assert int(st["dpc_random"][0]) == m.random and int(st["dpc_osc"][0]) == m.osc
    # The script reached what it is for: a flag set and cleared, the 11-bit
    # wrap, a sounding amplitude of each channel alone and together.
    assert 0xFF in got and 0 in got and {4, 5, 9} <= set(got)


def test_oracle_dpc_schemes_by_length():
    c = carts.dpc_cart()
    assert int(oracle.reset_state(c.rom)["scheme"]) == 6
    assert int(oracle.reset_state(carts.dpc_cart(dump_tail=True).rom)["scheme"]) == 6
    assert fa.rom_scheme(c.rom) == 6 and fa.rom_scheme(carts.dpc_cart(dump_tail=True).rom) == 6
    assert fa.guess_rom_scheme(c.rom) == 6
    for n in (10239, 10241, 10494, 10496):
        with pytest.raises(fa.FaError):
            fa.rom_scheme(bytes(n))
    st = oracle.reset_state(carts.plain_cart().rom)                # other schemes keep the DPC fields at 0
    assert not st["dpc_counter"].any() and int(st["dpc_random"]) == 0 and int(st["dpc_osc"]) == 0


def test_oracle_ignores_dpc_fields_of_other_schemes():
    """A state of another scheme carrying nonzero DPC fields runs as if they
    were 0, and comes back with them 0 (fa_set_states does the same)."""
    rom = carts.plain_cart().rom
    a = np.array([oracle.reset_state(rom)] * 4, dtype=oracle.STATE_DTYPE)
    b = a.copy()
    b["dpc_counter"] = 0x3FF
    b["dpc_top"] = 7
    b["dpc_music"] = 7
    b["dpc_random"] = 9
    b["dpc_osc"] = 12345
    acts = carts.actions(seed=3, n=4, frames=3)
    oracle.run_batch(rom, a, acts, 3)
    oracle.run_batch(rom, b, acts, 3)
    assert a.tobytes() == b.tobytes()


# ------------------------------------------------------------------ FE
def test_oracle_fe_bank_follows_the_access_after_01fe():
    """An 8K FE image whose two banks hold the same code and differ only in a
    marker byte at $1E80 ($B0 in bank 0, $B1 in bank 1).  Each step's
    expected bank is worked out from the access order of the reference CPU
    (src/cpu.rs): power-on bank 1; JSR $FA00 / $DA00 with S = $FF (the low
    return byte is pushed to $01FE, the target's high byte selects: $FA has
    bit 5 set, bank 0; $DA clear, bank 1) and RTS with S = $FD (the high
    return byte $F1 selects bank 0); LDA $01FE then CLC (the opcode $18
    selects bank 1); PLA with S = $FE (its stack read arms, the pulled byte
    selects: $20 bank 0, $00 bank 1)."""
    a = carts.Asm(0xF000)
    a.org(0xF100)
    a.label("reset")
    a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x80)          # bank 1 (power-on)
    a.ins("JSR", "abs", 0xFA00); a.ins("STA", "zp", 0x81)          # sub ran in bank 0
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x82)          # back in bank 0
    a.ins("JSR", "abs", 0xDA00); a.ins("STA", "zp", 0x83)          # sub ran in bank 1
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x84)          # RTS: $F1 -> bank 0
    a.ins("LDA", "abs", 0x01FE); a.ins("CLC")                      # $18 -> bank 1
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x85)
    a.ins("LDA", "imm", 0x20); a.ins("STA", "zp", 0xFF)
    a.ins("LDX", "imm", 0xFE); a.ins("TXS"); a.ins("PLA")          # pulls $20 -> bank 0
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x86)
    a.ins("LDA", "imm", 0x00); a.ins("STA", "zp", 0xFF)
    a.ins("LDX", "imm", 0xFE); a.ins("TXS"); a.ins("PLA")          # pulls $00 -> bank 1
    a.ins("LDA", "abs", 0xFE80); a.ins("STA", "zp", 0x87)
    a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    a.label("spin")
    a.ins("LDA", "imm", 0x02); a.ins("STA", "zp", carts.VSYNC)
    a.ins("JMP", "abs", "spin")
    a.org(0xFA00)
    a.ins("LDA", "abs", 0xFE80); a.ins("RTS")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF1, 0x00, 0xF1]))
    img, _, _ = a.assemble(4096)
    banks = [bytearray(img), bytearray(img)]
    banks[0][0xE80], banks[1][0xE80] = 0xB0, 0xB1
    rom = bytes(banks[0] + banks[1])
    oracle.set_rom_scheme(rom, "fe")
    try:
        st = oracle.reset_state(rom)
        assert int(st["scheme"]) == 7
        assert [int(x) for x in st["ram"][0:8]] == [0xB1, 0xB0, 0xB0, 0xB1, 0xB0, 0xB1, 0xB0, 0xB1]
        with oracle.phantoms_off():                                 # PLA's stack read is a phantom access
            st = oracle.reset_state(rom)
        assert [int(x) for x in st["ram"][6:8]] != [0xB0, 0xB1]
    finally:
        oracle.set_rom_scheme(rom, "auto")


def test_fe_registry_lengths():
    c = carts.fe_cart()
    fa.set_rom_scheme(c.rom, "fe")
    try:
        assert fa.rom_scheme(c.rom) == 7
    finally:
        fa.set_rom_scheme(c.rom, "auto")
    with pytest.raises(fa.FaError):
        fa.set_rom_scheme(bytes(4096), "fe")


def test_guess_fe_from_cross_bank_calls():
    """Six JSRs into $Dxxx and six into $Fxxx, no F8 hotspot access and a
    reset vector at $F100: FE.  One LDA $FFF8 (an F8 bank switch) makes it the
    size rule's F8 again, and so do fewer calls."""
    def image(calls, hotspot):
        rom = bytearray(8192)
        at = 0x100
        for hi in (0xD1, 0xF1):
            for _ in range(calls):
                rom[at:at + 3] = bytes([0x20, 0x00, hi])
                at += 3
        if hotspot:
            rom[at:at + 3] = bytes([0xAD, 0xF8, 0xFF])
        for b in range(2):
            rom[b * 4096 + 0xFFC:b * 4096 + 0xFFE] = bytes([0x00, 0xF1])
        return bytes(rom)
    assert fa.guess_rom_scheme(image(6, False)) == 7
    assert fa.guess_rom_scheme(image(6, True)) == 1
    assert fa.guess_rom_scheme(image(5, False)) == 1
