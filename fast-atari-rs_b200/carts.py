"""Seeded synthetic Atari 2600 carts and action streams.

The reference measures on Breakout.bin (examples/bench_cuda.rs:6), which is not
available here; these carts stand in for it with the shapes of the benchmark
configurations: a frame skeleton of 3 VSYNC, 37 VBLANK, 192 visible and 30
overscan lines, visible lines running seeded basic blocks of legal 6502 ops
that read SWCHA/INPT4/INPT0/INTIM and mix them into RAM, Fixed 2K/4K, F8, F6
and F4 bank switching, WSYNC-terminated or DEX/BNE-timed lines, JSR/RTS and
balanced stack traffic.

Safety rules (so every cart runs forever without an illegal opcode):
  * only forward branches inside a block; every block ends by falling into
    its line terminator;
  * RAM writes go to $82-$EF ($80/$81 belong to the skeleton, $F0-$FF to the
    stack); TIA writes avoid VSYNC/VBLANK/WSYNC/RSYNC; indexed or indirect
    writes are preceded by the loads that pin their effective address;
  * on bank-switched carts no read can reach a hotspot except the skeleton's
    trampoline, and every bank carries the same skeleton at the same address,
    so execution continues in the new bank after a switch.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

MASK64 = (1 << 64) - 1

# ----------------------------------------------------------------- RNG
def splitmix64(x: int) -> int:
    """SplitMix64 finaliser (Steele, Lea, Flood 2014)."""
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


class Rng:
    """Counter-based SplitMix64 stream; identical on every host."""

    def __init__(self, seed: int):
        self.state = splitmix64(seed & MASK64)

    @classmethod
    def from_state(cls, state: int) -> "Rng":
        r = cls(0)
        r.state = state & MASK64
        return r

    def next(self) -> int:
        self.state = (self.state + 1) & MASK64
        return splitmix64(self.state)

    def below(self, n: int) -> int:
        return self.next() % n

    def range(self, lo: int, hi: int) -> int:      # inclusive
        return lo + self.below(hi - lo + 1)

    def chance(self, p: float) -> bool:
        return (self.next() >> 11) * (1.0 / (1 << 53)) < p

    def choice(self, seq):
        return seq[self.below(len(seq))]


def _splitmix64_np(x: np.ndarray) -> np.ndarray:
    x = x + np.uint64(0x9E3779B97F4A7C15)
    z = x
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def actions(seed: int, n: int, frames: int, frame0: int = 0, num_actions: int = 18) -> np.ndarray:
    """int8 actions uniform over 18, frame-major [frames, n]: SplitMix64 of
    (seed, frame, instance), so any sub-range can be regenerated exactly."""
    with np.errstate(over="ignore"):
        f = (np.arange(frame0, frame0 + frames, dtype=np.uint64)[:, None])
        i = np.arange(n, dtype=np.uint64)[None, :]
        key = (np.uint64(seed & MASK64) * np.uint64(0xD1B54A32D192ED03)
               ^ f * np.uint64(0x9E3779B97F4A7C15) ^ i * np.uint64(0xC2B2AE3D27D4EB4F))
        h = _splitmix64_np(key)
    return (h % np.uint64(num_actions)).astype(np.uint8)


# ------------------------------------------------------------ opcode table
# (mnemonic, mode) -> opcode, for the 151 legal opcodes.
_OPS: Dict[Tuple[str, str], int] = {}


def _reg(mn, **modes):
    for mode, op in modes.items():
        _OPS[(mn, mode)] = op


for _mn, _base in (("ORA", 0x00), ("AND", 0x20), ("EOR", 0x40), ("ADC", 0x60),
                   ("LDA", 0xA0), ("CMP", 0xC0), ("SBC", 0xE0)):
    _reg(_mn, indx=_base | 0x01, zp=_base | 0x05, imm=_base | 0x09, abs=_base | 0x0D,
         indy=_base | 0x11, zpx=_base | 0x15, absy=_base | 0x19, absx=_base | 0x1D)
_reg("STA", indx=0x81, zp=0x85, abs=0x8D, indy=0x91, zpx=0x95, absy=0x99, absx=0x9D)
for _mn, _base in (("ASL", 0x00), ("ROL", 0x20), ("LSR", 0x40), ("ROR", 0x60)):
    _reg(_mn, zp=_base | 0x06, acc=_base | 0x0A, abs=_base | 0x0E, zpx=_base | 0x16, absx=_base | 0x1E)
_reg("DEC", zp=0xC6, abs=0xCE, zpx=0xD6, absx=0xDE)
_reg("INC", zp=0xE6, abs=0xEE, zpx=0xF6, absx=0xFE)
_reg("STX", zp=0x86, abs=0x8E, zpy=0x96)
_reg("LDX", imm=0xA2, zp=0xA6, abs=0xAE, zpy=0xB6, absy=0xBE)
_reg("STY", zp=0x84, abs=0x8C, zpx=0x94)
_reg("LDY", imm=0xA0, zp=0xA4, abs=0xAC, zpx=0xB4, absx=0xBC)
_reg("CPX", imm=0xE0, zp=0xE4, abs=0xEC)
_reg("CPY", imm=0xC0, zp=0xC4, abs=0xCC)
_reg("BIT", zp=0x24, abs=0x2C)
_reg("JMP", abs=0x4C, ind=0x6C)
_reg("JSR", abs=0x20)
for _mn, _op in (("BPL", 0x10), ("BMI", 0x30), ("BVC", 0x50), ("BVS", 0x70),
                 ("BCC", 0x90), ("BCS", 0xB0), ("BNE", 0xD0), ("BEQ", 0xF0)):
    _reg(_mn, rel=_op)
for _mn, _op in (("BRK", 0x00), ("RTI", 0x40), ("RTS", 0x60), ("PHP", 0x08), ("PLP", 0x28),
                 ("PHA", 0x48), ("PLA", 0x68), ("CLC", 0x18), ("SEC", 0x38), ("CLI", 0x58),
                 ("SEI", 0x78), ("CLV", 0xB8), ("CLD", 0xD8), ("SED", 0xF8), ("DEY", 0x88),
                 ("TXA", 0x8A), ("TYA", 0x98), ("TXS", 0x9A), ("TAY", 0xA8), ("TAX", 0xAA),
                 ("TSX", 0xBA), ("INY", 0xC8), ("DEX", 0xCA), ("INX", 0xE8), ("NOP", 0xEA)):
    _reg(_mn, imp=_op)

assert len(_OPS) == 151 and len(set(_OPS.values())) == 151
OPCODES = dict(_OPS)
LEGAL_OPCODES = sorted(_OPS.values())
_SIZE = {"imp": 1, "acc": 1, "imm": 2, "zp": 2, "zpx": 2, "zpy": 2, "indx": 2, "indy": 2,
         "rel": 2, "abs": 3, "absx": 3, "absy": 3, "ind": 3}

READ_MN = {"LDA", "ADC", "AND", "CMP", "EOR", "ORA", "SBC", "LDX", "LDY", "CPX", "CPY", "BIT"}
WRITE_MN = {"STA", "STX", "STY"}
RMW_MN = {"ASL", "LSR", "ROL", "ROR", "INC", "DEC"}

# Hardware registers used by the skeleton and the blocks.
VSYNC, VBLANK, WSYNC = 0x00, 0x01, 0x02
INPT0, INPT4 = 0x08, 0x0C
SWCHA, SWACNT, SWCHB, INTIM, INSTAT = 0x280, 0x281, 0x282, 0x284, 0x285
TIM1T, TIM8T, TIM64T, T1024T = 0x294, 0x295, 0x296, 0x297
LINE_CTR, MIX = 0x80, 0x81
RAM_W_LO, RAM_W_HI = 0x82, 0xEF                 # writable by blocks
TIA_WRITABLE = [r for r in range(0x04, 0x2D)]    # not VSYNC/VBLANK/WSYNC/RSYNC
TIA_READ_REGS = list(range(0x00, 0x0E))


# ---------------------------------------------------------------- assembler
@dataclass
class Ins:
    mn: str
    mode: str
    arg: object = None          # int, label name, or ("fwd", unit index) for block branches

    def size(self) -> int:
        return _SIZE[self.mode]


class Asm:
    """Two-pass assembler for one 4K bank image at origin $F000."""

    def __init__(self, origin: int = 0xF000):
        self.origin = origin
        self.items: List[object] = []   # Ins | ("label", name) | ("org", addr) | ("bytes", b)

    def label(self, name: str):
        self.items.append(("label", name))

    def org(self, addr: int):
        self.items.append(("org", addr))

    def raw(self, b: bytes):
        self.items.append(("bytes", bytes(b)))

    def ins(self, mn, mode="imp", arg=None):
        assert (mn, mode) in _OPS, (mn, mode)
        self.items.append(Ins(mn, mode, arg))

    def assemble(self, size: int, labels_in: Optional[Dict[str, int]] = None):
        labels: Dict[str, int] = dict(labels_in or {})
        for _ in range(2):
            pc = self.origin
            for it in self.items:
                if isinstance(it, Ins):
                    pc += it.size()
                elif it[0] == "label":
                    labels[it[1]] = pc
                elif it[0] == "org":
                    assert it[1] >= pc, (hex(it[1]), hex(pc))
                    pc = it[1]
                else:
                    pc += len(it[1])
        img = bytearray(size)
        pc = self.origin
        end_limit = self.origin + size
        for it in self.items:
            if isinstance(it, Ins):
                op = _OPS[(it.mn, it.mode)]
                arg = it.arg
                if isinstance(arg, str):
                    arg = labels[arg]
                if it.mode == "rel":
                    off = arg - (pc + 2)
                    assert -128 <= off <= 127, (it, off)
                    enc = bytes([op, off & 0xFF])
                elif it.size() == 1:
                    enc = bytes([op])
                elif it.size() == 2:
                    assert 0 <= arg <= 0xFF, (it, arg)
                    enc = bytes([op, arg])
                else:
                    assert 0 <= arg <= 0xFFFF, (it, arg)
                    enc = bytes([op, arg & 0xFF, arg >> 8])
                assert pc + len(enc) <= end_limit, "bank overflow"
                img[(pc - self.origin) % size: (pc - self.origin) % size + len(enc)] = enc
                pc += len(enc)
            elif it[0] == "label":
                pass
            elif it[0] == "org":
                pc = it[1]
            else:
                b = it[1]
                img[(pc - self.origin) % size:(pc - self.origin) % size + len(b)] = b
                pc += len(b)
        return bytes(img), labels, pc


# --------------------------------------------------------------- cart spec
@dataclass
class CartSpec:
    """Parameters of one synthetic cart."""
    name: str
    rom_size: int                       # 2048, 4096, 8192, 16384, 32768
    seed: int
    wsync_density: float = 1.0          # fraction of visible lines ending in STA WSYNC
    ops_min: int = 8
    ops_max: int = 40
    lines_per_group: int = 16           # distinct line blocks per bank; group loop runs 192/this times
    subroutines: int = 0                # JSR targets per bank
    stack_pairs: bool = True            # PHA/PLA, PHP/PLP balanced groups
    bank_select: str = "cycle"          # "cycle": next bank each group; "data": bank from RAM bits

    @property
    def nbanks(self) -> int:
        return max(1, self.rom_size // 4096)


@dataclass
class Cart:
    spec: CartSpec
    rom: bytes
    labels: Dict[str, int] = field(default_factory=dict)
    scheme: str = ""            # a scheme to register for this ROM ("e0", "3f"); "" = the size rule


class _BlockGen:
    """Generates one visible-line block as a list of units (lists of Ins)."""

    def __init__(self, rng: Rng, spec: CartSpec, bank: int, subs: List[str]):
        self.r = rng
        self.spec = spec
        self.bank = bank
        self.banked = spec.nbanks > 1
        self.subs = subs
        pool = []
        for (mn, mode), op in _OPS.items():
            if mn in ("BRK", "RTI", "RTS", "JMP", "TXS"):
                continue
            if mn == "JSR" and not subs:
                continue
            if mn in ("PHA", "PLA", "PHP", "PLP") and not spec.stack_pairs:
                continue
            pool.append((mn, mode))
        self.pool = sorted(pool, key=lambda k: _OPS[k])

    # -- operand helpers
    def ram_w(self) -> int:
        return self.r.range(RAM_W_LO, RAM_W_HI)

    def ram_r(self) -> int:
        return self.r.range(0x80, 0xFF)

    def zp_read(self) -> int:
        return self.ram_r() if self.r.chance(0.8) else self.r.choice(TIA_READ_REGS) | (0x40 if self.r.chance(0.2) else 0)

    def tia_w(self) -> int:
        return self.r.choice(TIA_WRITABLE) | (0x40 if self.r.chance(0.2) else 0)

    def rom_addr(self, span: int = 0) -> int:
        hi = 0xFEFF - span if self.banked else 0xFFFF - span
        return self.r.range(0xF000, hi)

    def abs_read(self) -> int:
        k = self.r.below(6)
        if k <= 1:
            return self.rom_addr()
        if k == 2:
            return self.r.choice([0x0080, 0x0180]) + self.r.below(0x80)
        if k == 3:
            return self.r.choice([0x0480, 0x0880, 0x0C80]) + self.r.below(0x80)   # reads 0
        if k == 4:
            return self.r.choice([SWCHA, SWCHB, INTIM, INSTAT, SWACNT, 0x0283, 0x0380 | self.r.below(8)])
        return self.r.choice(TIA_READ_REGS) | self.r.choice([0x000, 0x040, 0x100, 0x240])

    def abs_write(self) -> int:
        k = self.r.below(5)
        if k <= 1:
            return self.r.choice([0x0000, 0x0100, 0x0400, 0x0500, 0x0900]) + self.ram_w()
        if k == 2:
            return self.tia_w() | self.r.choice([0x000, 0x100])
        if k == 3:
            return self.r.choice([TIM1T, TIM8T, TIM64T, T1024T, SWACNT, 0x0280, 0x0282, 0x0283])
        return self.rom_addr()          # writes to ROM space are ignored (non-hotspot)

    def abs_rmw(self) -> int:
        k = self.r.below(4)
        if k <= 1:
            return self.r.choice([0x0000, 0x0100]) + self.ram_w()
        if k == 2:
            return self.tia_w()
        return self.rom_addr()

    # -- units
    def unit(self) -> List[Ins]:
        mn, mode = self.r.choice(self.pool)
        r = self.r
        if mode in ("imp", "acc"):
            if mn in ("PHA", "PHP", "PLA", "PLP"):
                inner = [self.simple_unit() for _ in range(r.below(3))]
                push = "PHA" if mn in ("PHA", "PLA") else "PHP"
                pull = "PLA" if push == "PHA" else "PLP"
                return [Ins(push, "imp")] + [i for u in inner for i in u] + [Ins(pull, "imp")]
            return [Ins(mn, mode)]
        if mode == "rel":
            return [Ins(mn, "rel", ("fwd", r.range(1, 4)))]
        if mn == "JSR":
            return [Ins("JSR", "abs", r.choice(self.subs))]
        return self.memory_unit(mn, mode)

    def simple_unit(self) -> List[Ins]:
        while True:
            mn, mode = self.r.choice(self.pool)
            if mode in ("rel",) or mn in ("JSR", "PHA", "PHP", "PLA", "PLP"):
                continue
            if mode in ("imp", "acc"):
                return [Ins(mn, mode)]
            return self.memory_unit(mn, mode)

    def memory_unit(self, mn: str, mode: str) -> List[Ins]:
        r = self.r
        kind = "r" if mn in READ_MN else "w" if mn in WRITE_MN else "m"
        if mode == "imm":
            return [Ins(mn, "imm", r.below(256))]
        if mode == "zp":
            if kind == "r":
                return [Ins(mn, "zp", self.zp_read())]
            a = self.tia_w() if r.chance(0.15) else self.ram_w()
            return [Ins(mn, "zp", a)]
        if mode in ("zpx", "zpy"):
            idx = "X" if mode == "zpx" else "Y"
            if kind == "r":
                return [Ins(mn, mode, self.ram_r())]
            t, k = self.ram_w(), r.below(256)
            return [Ins("LD" + idx, "imm", k), Ins(mn, mode, (t - k) & 0xFF)]
        if mode == "abs":
            a = self.abs_read() if kind == "r" else self.abs_write() if kind == "w" else self.abs_rmw()
            return [Ins(mn, "abs", a)]
        if mode in ("absx", "absy"):
            idx = "X" if mode == "absx" else "Y"
            if mn == "LDX":
                idx = "Y"
            if kind == "r":
                base = r.choice([self.rom_addr(255), 0x0000 + r.below(0x100), 0x0280,
                                 0x0080 + r.below(0x80)])
                return [Ins(mn, mode, base)]
            t, k = self.r.choice([0x0000, 0x0100]) + self.ram_w(), r.below(0x60)
            return [Ins("LD" + idx, "imm", k), Ins(mn, mode, t - k)]
        if mode == "indx":
            if kind == "r" and not self.banked and r.chance(0.5):
                return [Ins(mn, "indx", r.below(256))]
            t = self.ptr_target(kind)
            p, k = self.r.range(RAM_W_LO, RAM_W_HI - 1), r.below(256)
            return [Ins("LDA", "imm", t & 0xFF), Ins("STA", "zp", p),
                    Ins("LDA", "imm", t >> 8), Ins("STA", "zp", p + 1),
                    Ins("LDX", "imm", k)] + ([Ins("TXA", "imp")] if mn == "STA" else []) + \
                   [Ins(mn, "indx", (p - k) & 0xFF)]
        if mode == "indy":
            if kind == "r" and not self.banked and r.chance(0.5):
                return [Ins(mn, "indy", self.ram_r())]
            t = self.ptr_target(kind)
            k = r.below(0x20)
            base = t - k
            p = self.r.range(RAM_W_LO, RAM_W_HI - 1)
            return [Ins("LDA", "imm", base & 0xFF), Ins("STA", "zp", p),
                    Ins("LDA", "imm", (base >> 8) & 0xFF), Ins("STA", "zp", p + 1),
                    Ins("LDY", "imm", k)] + ([Ins("TYA", "imp")] if mn == "STA" else []) + \
                   [Ins(mn, "indy", p)]
        raise AssertionError((mn, mode))

    def ptr_target(self, kind: str) -> int:
        if kind == "r":
            return self.r.choice([self.rom_addr(), 0x0080 + self.r.below(0x80), SWCHA, INTIM,
                                  0x0480 + self.r.below(0x80), INPT4])
        # a write target: RAM or one of its mirrors, never straddling a page
        return self.r.choice([0x0000, 0x0100, 0x0400, 0x0D00]) + self.r.range(RAM_W_LO + 0x20, RAM_W_HI)

    def mix_unit(self) -> List[Ins]:
        src = self.r.choice([("abs", SWCHA), ("zp", INPT4), ("zp", INPT0), ("abs", INTIM), ("abs", SWCHB)])
        op = self.r.choice(["EOR", "ADC", "ORA", "SBC", "AND"])
        return [Ins("LDA", src[0], src[1]), Ins(op, "zp", self.ram_r()), Ins("STA", "zp", self.ram_w())]

    def block(self) -> List[List[Ins]]:
        target = self.r.range(self.spec.ops_min, self.spec.ops_max)
        units: List[List[Ins]] = [self.mix_unit()]
        n = 3
        while n < target:
            u = self.unit()
            units.insert(self.r.below(len(units) + 1), u) if self.r.chance(0.2) else units.append(u)
            n += len(u)
        if self.r.chance(0.5):
            units.append([Ins("LDA", "zp", self.ram_r()), Ins(self.r.choice(["BMI", "BPL", "BEQ", "BNE"]),
                                                                 "rel", ("fwd", self.r.range(1, 3)))])
            units.append(self.simple_unit())
        return units


def _emit_block(asm: Asm, units: List[List[Ins]], tag: str):
    """Emit units; ("fwd", d) branch args become labels d units ahead (clamped
    to the block end), so every branch is forward and lands on a unit start."""
    nu = len(units)
    for ui, u in enumerate(units):
        asm.label(f"{tag}_u{ui}")
        for ins in u:
            if isinstance(ins.arg, tuple) and ins.arg[0] == "fwd":
                dest = min(ui + ins.arg[1], nu)
                asm.ins(ins.mn, "rel", f"{tag}_u{dest}")
            else:
                asm.ins(ins.mn, ins.mode, ins.arg)
    asm.label(f"{tag}_u{nu}")


def _wsync_lines(asm: Asm, n: int, tag: str):
    asm.ins("LDX", "imm", n)
    asm.label(tag)
    asm.ins("STA", "zp", WSYNC)
    asm.ins("DEX")
    asm.ins("BNE", "rel", tag)


def _hotspots(nbanks: int) -> List[int]:
    first = {2: 0xFFF8, 4: 0xFFF6, 8: 0xFFF4}[nbanks]
    return [first + b for b in range(nbanks)]


def build_cart(spec: CartSpec) -> Cart:
    """Assemble the cart.  All banks share the skeleton at identical
    addresses; the line blocks and subroutines differ per bank.  Each bank is
    generated twice from the same RNG state: once to measure its block
    region, then with the region padded to the largest one."""
    assert spec.rom_size in (2048, 4096, 8192, 16384, 32768)
    assert 192 % spec.lines_per_group == 0
    nb = spec.nbanks
    bank_size = min(spec.rom_size, 4096)
    groups = 192 // spec.lines_per_group
    rng = Rng(spec.seed * 0x10001 + spec.rom_size)
    # Per-line terminator choice is shared by all banks (same line structure).
    term = [rng.chance(spec.wsync_density) for _ in range(spec.lines_per_group)]
    for _attempt in range(16):
        starts = [rng.next() for _ in range(nb)]
        try:
            ends = []
            for b in range(nb):
                asm = _bank_asm(spec, b, nb, Rng.from_state(starts[b]), term, groups, None)
                ends.append(asm.assemble(bank_size)[1]["region_end"])
            region_end = max(ends)
            images, labels = [], {}
            for b in range(nb):
                asm = _bank_asm(spec, b, nb, Rng.from_state(starts[b]), term, groups, region_end)
                img, labels, _ = asm.assemble(bank_size)
                images.append(img)
        except AssertionError:
            continue
        rom = b"".join(images)
        assert len(rom) == spec.rom_size
        return Cart(spec, rom, labels)
    raise RuntimeError(f"cart {spec.name}: code does not fit in {bank_size} bytes")


def _bank_asm(spec: CartSpec, b: int, nb: int, rng: Rng, term, groups: int,
              region_end: Optional[int]) -> Asm:
    bank_size = min(spec.rom_size, 4096)
    asm = Asm(0xF000)
    # --- reset: SEI; CLD; clear RAM $80-$FF; SP=$FF
    asm.label("reset")
    asm.ins("SEI"); asm.ins("CLD")
    asm.ins("LDA", "imm", 0)
    asm.ins("LDX", "imm", 0x7F)
    asm.label("clr")
    asm.ins("STA", "zpx", 0x80)
    asm.ins("DEX")
    asm.ins("BPL", "rel", "clr")
    asm.ins("LDX", "imm", 0xFF)
    asm.ins("TXS")
    # --- frame: VSYNC (3 lines)
    asm.label("frame")
    asm.ins("LDA", "imm", 0x02)
    asm.ins("STA", "zp", VSYNC)
    asm.ins("STA", "zp", WSYNC); asm.ins("STA", "zp", WSYNC); asm.ins("STA", "zp", WSYNC)
    asm.ins("LDA", "imm", 0x00)
    asm.ins("STA", "zp", VSYNC)
    # --- VBLANK (37 lines): dump paddles, set the interval timer
    asm.ins("LDA", "imm", 0x82)
    asm.ins("STA", "zp", VBLANK)
    asm.ins("LDA", "imm", 43)
    asm.ins("STA", "abs", TIM64T)
    _wsync_lines(asm, 37, "vbl")
    asm.ins("LDA", "imm", 0x00)
    asm.ins("STA", "zp", VBLANK)
    # --- visible: groups x lines_per_group lines
    asm.ins("LDA", "imm", groups)
    asm.ins("STA", "zp", LINE_CTR)
    asm.label("vis_loop")
    gen = _BlockGen(rng, spec, b, [f"sub{i}" for i in range(spec.subroutines)])
    for j in range(spec.lines_per_group):
        _emit_block(asm, gen.block(), f"b{j}")
        if term[j]:
            asm.ins("STA", "zp", WSYNC)
        else:
            asm.ins("LDX", "imm", 1 + rng.below(8))
            asm.label(f"dly{j}")
            asm.ins("DEX")
            asm.ins("BNE", "rel", f"dly{j}")
    asm.ins("JMP", "abs", "group_end")
    asm.label("region_end")
    if region_end is not None:
        asm.org(region_end)
    # --- group end: trampoline (same address in every bank), loop
    asm.label("group_end")
    if nb > 1:
        hs = _hotspots(nb)
        if spec.bank_select == "data":
            # Always switches, along a path chosen by a RAM bit (the skeleton's
            # INTIM mix, which depends on each instance's timing); with more
            # than two banks the target bank depends on that bit too.
            asm.ins("LDA", "zp", MIX)
            asm.ins("LSR", "acc")
            asm.ins("BCC", "rel", "tr_b")
            asm.ins("BIT", "abs", hs[(b + 1) % nb])
            asm.ins("JMP", "abs", "tr_done")
            asm.label("tr_b")
            asm.ins("BIT", "abs", hs[(b + 2) % nb] if nb > 2 else hs[(b + 1) % nb])
            asm.label("tr_done")
        else:
            asm.ins("BIT", "abs", hs[(b + 1) % nb])
    asm.ins("DEC", "zp", LINE_CTR)
    asm.ins("BEQ", "rel", "vis_done")
    asm.ins("JMP", "abs", "vis_loop")
    asm.label("vis_done")
    # --- overscan (30 lines); mix INTIM into RAM
    asm.ins("LDA", "imm", 0x02)
    asm.ins("STA", "zp", VBLANK)
    _wsync_lines(asm, 30, "ovs")
    asm.ins("LDA", "abs", INTIM)
    asm.ins("EOR", "zp", MIX)
    asm.ins("STA", "zp", MIX)
    asm.ins("JMP", "abs", "frame")
    # --- subroutines (bank-specific)
    for i in range(spec.subroutines):
        asm.label(f"sub{i}")
        sg = _BlockGen(rng, CartSpec(spec.name, spec.rom_size, 0, ops_min=4, ops_max=12,
                                     stack_pairs=spec.stack_pairs), b, [])
        units = sg.block()
        _emit_block(asm, units, f"s{i}")
        asm.ins("RTS")
    # --- vectors
    asm.org(0xF000 + bank_size - 4)
    asm.raw(bytes([0x00, 0xF0, 0x00, 0xF0]))
    return asm


# ------------------------------------------------------- benchmark carts
def plain_cart(seed: int = 1) -> Cart:
    """4K Fixed, every visible line ends in STA WSYNC, 8-40 ops per block."""
    return build_cart(CartSpec("plain_4k_fixed", 4096, seed, wsync_density=1.0,
                               ops_min=8, ops_max=40))


def divergence_cart(seed: int = 2) -> Cart:
    """8K F8, no WSYNC in the visible kernel (DEX/BNE-timed lines), 20-60 ops,
    JSR/RTS, PHA/PLA, data-dependent bank switch every 16 lines."""
    return build_cart(CartSpec("divergence_8k_f8", 8192, seed, wsync_density=0.0,
                               ops_min=20, ops_max=60, subroutines=4, bank_select="data"))


def mixed_carts(seed: int = 3) -> List[Cart]:
    """2K Fixed / 8K F8 / 16K F6 / 32K F4 with WSYNC density 100/50/10/0%."""
    out = []
    for i, (size, dens) in enumerate(((2048, 1.0), (8192, 0.5), (16384, 0.1), (32768, 0.0))):
        out.append(build_cart(CartSpec(f"mixed_{size // 1024}k", size, seed + 17 * i,
                                       wsync_density=dens, ops_min=8, ops_max=40,
                                       subroutines=2 if size > 4096 else 0)))
    return out


MIXED_COUNTS = (100_000, 30_000, 5_000, 500)


def scale_cart(seed: int = 4) -> Cart:
    """32K F4, 0% WSYNC lines, bank switch every 8 lines."""
    return build_cart(CartSpec("scale_32k_f4", 32768, seed, wsync_density=0.0,
                               ops_min=8, ops_max=40, lines_per_group=8, subroutines=2))


# ------------------------------------------------------------- rendering cart
# Graphics registers the rendering cart writes (Tia::write, src/tia.rs:570-674).
_GFX_REGS = [0x04, 0x05, 0x06, 0x07, 0x08, 0x09, 0x0A, 0x0B, 0x0C, 0x0D, 0x0E, 0x0F,
             0x1B, 0x1C, 0x1D, 0x1E, 0x1F, 0x20, 0x21, 0x22, 0x23, 0x24, 0x25, 0x26, 0x27, 0x28, 0x29]
_POS_REGS = [0x10, 0x11, 0x12, 0x13, 0x14]       # RESP0 RESP1 RESM0 RESM1 RESBL
_CX_READS = [0x30, 0x31, 0x32, 0x33, 0x34, 0x35, 0x36, 0x37]


def render_cart(seed: int = 5) -> Cart:
    """A 4K Fixed cart for the rendering console (the pixel-accurate TIA):
    the frame skeleton (3 VSYNC, 37 VBLANK with the input-latch or paddle-dump
    bits, 192 visible, 30 overscan lines) with visible lines that write every
    graphics register from RAM-dependent values at varying cycles within the
    line -- colours, playfield (mid-line, through the delayed write), player,
    missile and ball graphics, NUSIZ copies and sizes, reflection, priority
    and score modes, vertical delay, mid-line RESPx/RESMx/RESBL, HMOVE and
    HMCLR, read-modify-write on TIA registers -- read the collision latches
    and the inputs back into RAM, and fold SWCHA into that RAM every line, so
    the picture depends on the actions.  Control flow is straight-line blocks
    and counted loops only."""
    rng = Rng(seed * 0x9E3779B1 + 4096)
    a = Asm()
    a.label("reset")
    for mn, mode, arg in (("SEI", "imp", None), ("CLD", "imp", None), ("LDX", "imm", 0xFF), ("TXS", "imp", None),
                          ("LDA", "imm", 0), ("LDX", "imm", 0x80)):
        a.ins(mn, mode, arg)
    a.label("clr")
    a.ins("STA", "zpx", 0)
    a.ins("INX")
    a.ins("BNE", "rel", "clr")
    a.label("frame")
    a.ins("LDA", "imm", 2)
    a.ins("STA", "zp", VSYNC)
    for _ in range(3):
        a.ins("STA", "zp", WSYNC)
    a.ins("LDA", "imm", 0)
    a.ins("STA", "zp", VSYNC)
    a.ins("LDA", "imm", 0x02 | (0x40 if rng.chance(0.5) else 0) | (0x80 if rng.chance(0.5) else 0))
    a.ins("STA", "zp", VBLANK)
    _wsync_lines(asm=a, n=36, tag="vbl")
    # per frame: inputs into RAM, a per-frame seed byte
    a.ins("LDA", "abs", SWCHA)
    a.ins("EOR", "zp", 0x81)
    a.ins("ADC", "imm", rng.below(256))
    a.ins("STA", "zp", 0x81)
    a.ins("LDA", "zp", INPT4)
    a.ins("STA", "zp", 0x82)
    a.ins("STA", "zp", WSYNC)
    a.ins("LDA", "imm", 0)
    a.ins("STA", "zp", VBLANK)
    a.ins("LDA", "imm", 192)
    a.ins("STA", "zp", 0x80)
    a.label("line")
    a.ins("STA", "zp", WSYNC)
    nblocks = 8
    # line dispatch: a RAM-counter-selected block (8 blocks of lines)
    a.ins("LDA", "zp", 0x80)
    a.ins("AND", "imm", 7)
    a.ins("TAX")
    for b in range(nblocks):
        a.ins("CPX", "imm", b)
        a.ins("BNE", "rel", f"nb{b}")
        a.ins("JMP", "abs", f"blk{b}")
        a.label(f"nb{b}")
    a.ins("JMP", "abs", "blk0")
    for b in range(nblocks):
        a.label(f"blk{b}")
        if rng.chance(0.3):
            a.ins("STA", "zp", 0x2A)                               # HMOVE right after WSYNC
        for _u in range(rng.range(6, 11)):
            k = rng.below(10)
            r1, r2 = rng.range(0x81, 0xBF), rng.range(0x83, 0xBF)
            if k <= 3:                                             # graphics register from RAM
                a.ins("LDA", "zp", r1)
                if rng.chance(0.5):
                    a.ins("EOR", "zp", 0x80)                       # the line counter
                a.ins("STA", "zp" if rng.chance(0.7) else "abs", rng.choice(_GFX_REGS))
            elif k == 4:                                           # position reset at this cycle
                if rng.chance(0.5):
                    a.ins("NOP")
                a.ins("STA", "zp", rng.choice(_POS_REGS))
            elif k == 5:                                           # collisions into RAM
                a.ins("LDA", "zp", rng.choice(_CX_READS))
                a.ins("ORA", "zp", r1)
                a.ins("STA", "zp", r2)
            elif k == 6:                                           # read-modify-write on a TIA register
                a.ins(rng.choice(["INC", "DEC", "ASL", "ROL"]), "zp", rng.choice([0x06, 0x07, 0x08, 0x09, 0x0E, 0x1B]))
            elif k == 7:                                           # motion registers
                a.ins("LDA", "imm", rng.below(256))
                a.ins("STA", "zp", rng.choice([0x20, 0x21, 0x22, 0x23, 0x24, 0x2B]))
            elif k == 8:                                           # RAM evolution from the inputs
                a.ins("LDA", "abs", SWCHA)
                a.ins("ADC", "zp", r1)
                a.ins("STA", "zp", r2)
            else:                                                  # timer and paddle reads into RAM
                if rng.chance(0.5):
                    a.ins("LDA", "abs", INTIM)
                else:
                    a.ins("LDA", "abs" if rng.chance(0.5) else "zp", INPT0)
                a.ins("EOR", "zp", r1)
                a.ins("STA", "zp", r2)
        a.ins("JMP", "abs", "lend")
    a.label("lend")
    a.ins("DEC", "zp", 0x80)
    a.ins("BEQ", "rel", "ovs")
    a.ins("JMP", "abs", "line")
    a.label("ovs")
    a.ins("LDA", "imm", 2)
    a.ins("STA", "zp", VBLANK)
    a.ins("STA", "zp", 0x2C)                                       # CXCLR
    _wsync_lines(asm=a, n=30, tag="ovl")
    a.ins("JMP", "abs", "frame")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF0, 0x00, 0xF0]))
    img, labels, _ = a.assemble(4096)
    return Cart(CartSpec("render_4k_fixed", 4096, seed, wsync_density=1.0), bytes(img), labels)


# ------------------------------------------------ sliced-bank carts (E0, 3F)
# Routines that run from a switchable window are position-independent:
# relative branches only, entered by JSR at the window's base, leaving by RTS.
# They write RAM ($82-$EF) and, where the scheme allows, TIA registers, and
# read ROM data through every window, so a wrong mapping changes RAM.

def _window_routine(rng: Rng, size: int, tia_writes: bool, data_lo: int, data_hi: int,
                    avoid=(0, 0), tail: bytes = b"") -> bytes:
    a = Asm(0xF000)
    nunits = rng.range(10, 24)

    def ram() -> int:
        return rng.range(RAM_W_LO, RAM_W_HI)

    def rom_data() -> int:
        while True:
            d = rng.range(data_lo, data_hi)
            if not (avoid[0] <= d <= avoid[1]):
                return d

    for u in range(nunits):
        k = rng.below(9)
        if k == 0:
            a.ins("LDA", "zp", ram()); a.ins("ADC", "imm", rng.below(256)); a.ins("STA", "zp", ram())
        elif k == 1:                                                # ROM data through any window
            a.ins("LDA", "zp", ram()); a.ins("EOR", "abs", rom_data()); a.ins("STA", "zp", ram())
        elif k == 2:                                                # indexed ROM data
            a.ins("LDX", "zp", ram()); a.ins("LDA", "absx", rom_data() & 0xFF00 | rng.below(0x80))
            a.ins("STA", "zp", ram())
        elif k == 3:
            a.ins(rng.choice(["INC", "DEC", "ASL", "ROR"]), "zp", ram())
        elif k == 4:                                                # counted loop
            a.ins("LDY", "imm", rng.range(1, 6)); a.label(f"l{u}"); a.ins("DEY"); a.ins("BNE", "rel", f"l{u}")
        elif k == 5:                                                # data-dependent skip
            a.ins("LDA", "zp", ram()); a.ins(rng.choice(["BMI", "BPL", "BEQ", "BNE"]), "rel", f"s{u}")
            a.ins("INC", "zp", ram()); a.label(f"s{u}")
        elif k == 6 and tia_writes:
            a.ins("LDA", "zp", ram()); a.ins("STA", "zp", rng.choice(TIA_WRITABLE))
        elif k == 7:                                                # timer and inputs
            a.ins("LDA", "abs", rng.choice([INTIM, SWCHA])); a.ins("EOR", "zp", ram()); a.ins("STA", "zp", ram())
        else:
            a.ins("LDA", "zp", ram()); a.ins("PHA"); a.ins("LDA", "zp", ram()); a.ins("STA", "zp", ram())
            a.ins("PLA"); a.ins("ADC", "zp", ram()); a.ins("STA", "zp", ram())
    a.ins("RTS")
    img = bytearray(a.assemble(size)[0])
    body_end = 0
    for i in range(len(img) - 1, -1, -1):
        if img[i]:
            body_end = i + 1
            break
    for i in range(body_end, size - len(tail)):                     # the rest is ROM data
        img[i] = rng.below(256)
    if tail:
        assert body_end <= size - len(tail)
        img[size - len(tail):] = tail
    return bytes(img)


def _frame_head(a: Asm, lines: int):
    a.label("frame")
    a.ins("LDA", "imm", 0x02); a.ins("STA", "zp", VSYNC)
    a.ins("STA", "zp", WSYNC); a.ins("STA", "zp", WSYNC); a.ins("STA", "zp", WSYNC)
    a.ins("LDA", "imm", 0x00); a.ins("STA", "zp", VSYNC)
    a.ins("LDA", "imm", 0x82); a.ins("STA", "zp", VBLANK)
    _wsync_lines(asm=a, n=36, tag="vbl")
    a.ins("LDA", "abs", SWCHA); a.ins("EOR", "zp", MIX); a.ins("STA", "zp", MIX)
    a.ins("LDA", "zp", INPT4); a.ins("ADC", "zp", MIX); a.ins("STA", "zp", MIX)
    a.ins("LDA", "imm", 0x00); a.ins("STA", "zp", VBLANK)
    a.ins("LDA", "imm", lines); a.ins("STA", "zp", LINE_CTR)


def _frame_tail(a: Asm):
    a.ins("DEC", "zp", LINE_CTR)
    a.ins("BEQ", "rel", "ovs")
    a.ins("JMP", "abs", "line")
    a.label("ovs")
    _wsync_lines(asm=a, n=30, tag="ovl")
    a.ins("JMP", "abs", "frame")


def _reset_code(a: Asm):
    a.label("reset")
    a.ins("SEI"); a.ins("CLD"); a.ins("LDA", "imm", 0); a.ins("LDX", "imm", 0x7F)
    a.label("clr")
    a.ins("STA", "zpx", 0x80); a.ins("DEX"); a.ins("BPL", "rel", "clr")
    a.ins("LDX", "imm", 0xFF); a.ins("TXS")


def e0_cart(seed: int = 6, lines: int = 64) -> Cart:
    """8K Parker Brothers E0 cart: 1K slices 0-6 hold position-independent
    routines (TIA writes included); slice 7 (window 3, fixed) holds the frame
    skeleton.  Every line picks the slices of windows 0-2 from RAM through
    the hotspots $1FE0-$1FF7 (an abs,X load, an abs,Y store and an abs,X load
    of the hotspot rows) and calls each window; every fourth line also runs
    an instruction that straddles windows 2 and 3 (LDA $0080 from $1BFE)."""
    rng = Rng(seed * 0x9E3779B1 + 0xE0)
    slices = [_window_routine(rng, 1024, True, 0xF000, 0xFFDF, avoid=(0xFFE0, 0xFFF7), tail=bytes([0xAD, 0x80]))
              for _ in range(7)]
    a = Asm(0xFC00)
    a.raw(bytes([0x00, 0x60]))                  # $1C00: high byte of the straddling LDA, then RTS
    _reset_code(a)
    _frame_head(a, lines)
    a.label("line")
    a.ins("STA", "zp", WSYNC)
    for w, (base, how) in enumerate(((0xFFE0, "ldx"), (0xFFE8, "sty"), (0xFFF0, "ldx"))):
        a.ins("LDA", "zp", MIX); a.ins("ADC", "zp", LINE_CTR)
        for _ in range(w):
            a.ins("LSR", "acc")
        a.ins("STA", "zp", MIX)
        a.ins("AND", "imm", 7)
        if how == "ldx":
            a.ins("TAX"); a.ins("LDA", "absx", "map7"); a.ins("TAX"); a.ins("LDA", "absx", base)
        else:
            a.ins("TAY"); a.ins("LDA", "absy", "map7"); a.ins("TAY"); a.ins("STA", "absy", base)
    for base in (0xF000, 0xF400, 0xF800):
        a.ins("JSR", "abs", base)
    a.ins("LDA", "zp", LINE_CTR); a.ins("AND", "imm", 3); a.ins("BNE", "rel", "nostr")
    a.ins("JSR", "abs", 0xFBFE)
    a.label("nostr")
    _frame_tail(a)
    a.label("map7")
    a.raw(bytes([0, 1, 2, 3, 4, 5, 6, rng.below(7)]))
    a.org(0xFFE0)
    a.raw(bytes(rng.below(256) for _ in range(0x18)))     # hotspot rows: data only
    a.org(0xFFFC)
    a.raw(bytes([0x02, 0xFC, 0x02, 0xFC]))
    img, labels, _ = a.assemble(1024)
    assert labels["reset"] == 0xFC02 and labels["map7"] < 0xFFE0
    rom = b"".join(slices) + img
    assert len(rom) == 8192
    return Cart(CartSpec("e0_8k", 8192, seed, wsync_density=1.0), rom, labels, scheme="e0")


def f3_cart(size: int = 16384, seed: int = 7, lines: int = 64) -> Cart:
    """Tigervision 3F cart of `size` bytes (a multiple of 2K): 2K banks
    0..n-2 hold position-independent routines (no TIA writes: any write to
    $00-$3F switches the bank under them); the last 2K (fixed at $1800)
    holds the frame skeleton.  Every line selects banks through STA/STX/STY
    $3F with values above n (the bank is the value mod n), writes a colour
    register (which selects bank COLUBK-value mod n), reads the lower window
    through that mapping, and calls the routines of three selected banks."""
    n = size // 2048
    assert size % 2048 == 0 and n >= 2
    rng = Rng(seed * 0x9E3779B1 + size)
    banks = [_window_routine(rng, 2048, False, 0xF000, 0xFFF0) for _ in range(n - 1)]
    sel = [b + n * rng.below(256 // n) for b in range(n - 1) for _ in range(2)]
    sel = (sel * 8)[:8]
    assert all(v % n != n - 1 and v < 256 for v in sel)
    a = Asm(0xF800)
    _reset_code(a)
    _frame_head(a, lines)
    a.label("line")
    a.ins("STA", "zp", WSYNC)
    for reg in ("A", "X", "Y"):
        a.ins("LDA", "zp", MIX); a.ins("ADC", "zp", LINE_CTR); a.ins("STA", "zp", MIX)
        a.ins("AND", "imm", 7); a.ins("TAX")
        if reg == "A":
            a.ins("LDA", "zp", MIX); a.ins("STA", "zp", 0x09)       # COLUBK: also a bank select
            a.ins("LDA", "abs", 0xF000 + rng.below(0x800)); a.ins("EOR", "zp", 0x83); a.ins("STA", "zp", 0x83)
            a.ins("LDA", "absx", "sel"); a.ins("STA", "zp", 0x3F)
        elif reg == "X":
            a.ins("LDA", "absx", "sel"); a.ins("TAX"); a.ins("STX", "zp", 0x3F)
        else:
            a.ins("LDY", "absx", "sel"); a.ins("STY", "zp", 0x3F)
        a.ins("JSR", "abs", 0xF000)
    _frame_tail(a)
    a.label("sel")
    a.raw(bytes(sel))
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF8, 0x00, 0xF8]))
    img, labels, _ = a.assemble(2048)
    assert labels["reset"] == 0xF800
    rom = b"".join(banks) + img
    assert len(rom) == size
    return Cart(CartSpec(f"3f_{size // 1024}k", size, seed, wsync_density=1.0), rom, labels, scheme="3f")


FE_BANKID = 0xFE80
FE_SUB = 0xFA00                                      # the subroutine, at $1A00 of both banks
FE_TABLE = 0xFB00                                    # 256 bytes of bank-specific data


def fe_cart(seed: int = 9, lines: int = 40) -> Cart:
    """Activision FE cart, 8K: two 4K banks with the same code at the same
    addresses (only the bank-id byte at $FE80 and a data table at $FB00
    differ), so a switch at any access keeps running.  Each visible line arms
    the cart through every kind of access to $01FE and lets the next access
    pick the bank:
      - JSR with S = $FF (the low return byte lands on $01FE; the target's
        high byte, $DA or $FA as a RAM bit chooses, selects bank 1 or 0), and
        RTS with S = $FD (pulls from $01FE; the high return byte selects);
      - JSR with S = $FE (its stack read at $01FE arms, the push of the high
        byte there selects and re-arms, the low byte's push selects), and the
        matching RTS with S = $FC (the high byte pulled from $01FE arms, the
        read at the return address selects);
      - PLA with S = $FE (its stack read arms, the pulled byte selects);
      - PHA and PLA at $01FE, LDA $01FE and LDA $01F0,X with X = $0E (the
        next opcode fetch selects), and INC $01FE on every 4th line (the
        read arms, the write of the original value selects by RAM data and
        re-arms, the final write does too).
    In the RTS with S = $FC and the PLA with S = $FE, a phantom access (the
    read of the return address, the stack read) decides the bank: the cart
    runs differently when they are left out.
    The subroutine mixes the bank-id byte and a bank-specific table byte into
    RAM."""
    rng = Rng(seed * 0x9E3779B1 + 0xFE)
    a = Asm(0xF000)
    a.org(0xF100)
    _reset_code(a)
    _frame_head(a, lines)
    a.label("line")
    a.ins("STA", "zp", WSYNC)
    a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    for i, (via, stack) in enumerate((("bit0", 0xFF), ("bit1", 0xFE))):
        a.ins("LDX", "imm", stack); a.ins("TXS")
        a.ins("LDA", "zp", MIX); a.ins("ADC", "zp", LINE_CTR); a.ins("STA", "zp", MIX)
        a.ins("AND", "imm", 1 if via == "bit0" else 2)
        a.ins("BEQ", "rel", f"f_{via}")
        a.ins("JSR", "abs", FE_SUB - 0x2000)                # $DA00: bank 1
        # The opcode after each JSR has bit 5 opposite to the JSR's high byte:
        # returning with S = $FC, the read of the return address ($DA / $FA)
        # selects the bank, not this fetch.
        a.ins("LDY", "imm", 0)                              # $A0
        a.ins("JMP", "abs", f"after_{via}")
        a.label(f"f_{via}")
        a.ins("JSR", "abs", FE_SUB)                         # $FA00: bank 0
        a.ins("CLC")                                        # $18
        a.label(f"after_{via}")
        a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x8A + i); a.ins("STA", "zp", 0x8A + i)
    # PLA with S = $FE: its stack read at $01FE arms, the pull of $01FF
    # (written from RAM just before) selects.
    a.ins("LDA", "zp", MIX); a.ins("EOR", "zp", 0x84); a.ins("STA", "zp", 0xFF)
    a.ins("LDX", "imm", 0xFE); a.ins("TXS"); a.ins("PLA")
    a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x8C); a.ins("STA", "zp", 0x8C)
    a.ins("LDX", "imm", 0xFE); a.ins("TXS")
    a.ins("LDA", "zp", MIX); a.ins("PHA")                   # writes $01FE
    a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x83); a.ins("STA", "zp", 0x83)
    a.ins("PLA")                                            # pulls $01FE
    a.ins("EOR", "abs", FE_BANKID); a.ins("STA", "zp", 0x86)
    a.ins("LDA", "abs", 0x01FE); a.ins("ADC", "zp", 0x87); a.ins("STA", "zp", 0x87)
    a.ins("LDX", "imm", 0x0E); a.ins("LDA", "absx", 0x01F0)
    a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x88); a.ins("STA", "zp", 0x88)
    a.ins("LDA", "zp", LINE_CTR); a.ins("AND", "imm", 3); a.ins("BNE", "rel", "noinc")
    a.ins("INC", "abs", 0x01FE)
    a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x89); a.ins("STA", "zp", 0x89)
    a.label("noinc")
    a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    _frame_tail(a)
    a.org(FE_SUB)
    a.ins("LDA", "abs", FE_BANKID); a.ins("ADC", "zp", 0x84); a.ins("STA", "zp", 0x84)
    a.ins("LDX", "zp", MIX); a.ins("LDA", "absx", FE_TABLE); a.ins("EOR", "zp", 0x85); a.ins("STA", "zp", 0x85)
    a.ins("RTS")
    a.org(FE_TABLE)
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF1, 0x00, 0xF1]))
    img, labels, _ = a.assemble(4096)
    assert labels["reset"] == 0xF100 and labels["noinc"] < FE_SUB
    banks = []
    for b in range(2):
        bank = bytearray(img)
        for i in range(256):
            bank[FE_TABLE - 0xF000 + i] = rng.below(256)
        bank[FE_BANKID - 0xF000] = 0xC0 + b
        banks.append(bytes(bank))
    rom = banks[0] + banks[1]
    return Cart(CartSpec("fe_8k", 8192, seed, wsync_density=1.0), rom, labels, scheme="fe")


DPC_BANKID = 0xFE80


def dpc_cart(seed: int = 8, lines: int = 48, dump_tail: bool = False) -> Cart:
    """Activision DPC cart (Pitfall II's scheme): two 4K program banks, then
    2K of display data; 10,240 bytes, or 10,495 with the 255-byte tail some
    dumps of the cart carry.  Both banks hold the same code at the same
    addresses (only the bank-id byte at $FE80 and the ROM data differ), so a
    switch anywhere keeps running.  Each frame loads all 8 fetchers' top,
    bottom and counter registers from RAM-mixed values, fetchers 5-7 turning
    into music channels by a RAM bit.  Each visible line reads a RAM-chosen
    fetcher's display data, masked data, flag and a no-value function, the
    random number and the music amplitude, mixes them into RAM, and switches
    the program bank through $1FF8/$1FF9 by a RAM bit.  Every 8th line resets
    the random number generator, rewrites fetcher 0's counter through a
    read-modify-write, and makes a page-crossing indexed read whose phantom
    read lands on a DPC read register ($1008)."""
    rng = Rng(seed * 0x9E3779B1 + 0xDC)
    tops = [rng.range(0x20, 0xF0) for _ in range(8)]
    his = [0x07] * 5 + [0x17] * 3                      # bit 4: music mode for fetchers 5-7

    def bank(b: int) -> bytes:
        a = Asm(0xF000)
        a.org(0xF100)
        _reset_code(a)
        _frame_head(a, lines)
        a.ins("LDX", "imm", 7)
        a.label("setup")
        a.ins("LDA", "zp", MIX); a.ins("ADC", "absx", "tops"); a.ins("STA", "absx", 0x1040)     # top
        a.ins("LSR", "acc"); a.ins("STA", "absx", 0x1048)                                       # bottom
        a.ins("EOR", "zp", 0x83); a.ins("STA", "absx", 0x1050)                                  # counter low
        a.ins("LDA", "zp", MIX); a.ins("AND", "absx", "his"); a.ins("STA", "absx", 0x1058)      # counter high
        a.ins("DEX"); a.ins("BPL", "rel", "setup")
        a.label("line")
        a.ins("STA", "zp", WSYNC)
        a.ins("LDA", "zp", MIX); a.ins("ADC", "zp", LINE_CTR); a.ins("AND", "imm", 7); a.ins("TAX")
        for base, op, acc in ((0x1008, "EOR", MIX), (0x1010, "ADC", 0x84), (0x1038, "EOR", 0x85),
                              (0x1018, "ADC", 0x86)):
            a.ins("LDA", "absx", base); a.ins(op, "zp", acc); a.ins("STA", "zp", acc)
        for addr, acc in ((0x1000, 0x87), (0x1004, 0x88), (0x1007, 0x88), (0x1002, 0x89)):
            a.ins("LDA", "abs", addr); a.ins("ADC", "zp", acc); a.ins("STA", "zp", acc)
        a.ins("LDA", "zp", MIX); a.ins("LSR", "acc"); a.ins("AND", "imm", 1); a.ins("TAX")
        a.ins("LDA", "absx", 0xFFF8)                                                            # bank 0 / 1
        a.ins("LDA", "abs", DPC_BANKID); a.ins("ADC", "zp", 0x8A); a.ins("STA", "zp", 0x8A)
        a.ins("LDA", "zp", LINE_CTR); a.ins("AND", "imm", 7); a.ins("BNE", "rel", "skip")
        a.ins("STA", "abs", 0x1070)                                                             # random reset
        a.ins("INC", "abs", 0x1050)                                                             # counter 0 low, twice
        a.ins("LDX", "imm", 0x10); a.ins("LDA", "absx", 0x10F8)                                 # phantom at $1008
        a.ins("ADC", "zp", 0x8B); a.ins("STA", "zp", 0x8B)
        a.label("skip")
        _frame_tail(a)
        a.label("tops")
        a.raw(bytes(tops))
        a.label("his")
        a.raw(bytes(his))
        a.org(DPC_BANKID)
        a.raw(bytes([0xB0 + b]))
        a.org(0xFFF8)
        a.raw(bytes([rng.below(256), rng.below(256)]))                                         # hotspot rows: data
        a.org(0xFFFC)
        a.raw(bytes([0x00, 0xF1, 0x00, 0xF1]))
        img, labels, end = a.assemble(4096)
        assert labels["reset"] == 0xF100 and labels["his"] + 8 <= DPC_BANKID
        img = bytearray(img)
        for i in list(range(0x000, 0x100)) + list(range(labels["his"] + 8 - 0xF000, DPC_BANKID - 0xF000)):
            img[i] = rng.below(256)                                                             # ROM data
        return bytes(img), labels

    (b0, labels), (b1, _) = bank(0), bank(1)
    display = bytes(rng.below(256) for _ in range(2048))
    rom = b0 + b1 + display + (bytes(rng.below(256) for _ in range(255)) if dump_tail else b"")
    assert len(rom) == (10495 if dump_tail else 10240)
    name = "dpc_10k_tail" if dump_tail else "dpc_10k"
    return Cart(CartSpec(name, len(rom), seed, wsync_density=1.0), rom, labels, scheme=None)


def dpc_display_byte(i: int) -> int:
    """Display data of dpc_script_cart: byte i of the 2K block."""
    return (i * 37 + 11) & 0xFF


def dpc_script() -> List[tuple]:
    """The DPC accesses dpc_script_cart makes, in order: ("w", addr, value),
    ("r", addr) (its value goes to the next RAM byte from $80 on) and
    ("nop", count).  It walks fetcher 0's counter through top and bottom,
    fetcher 3's across the 11-bit wrap, the random number generator before
    and after a reset, the no-value functions, and music channels sampled
    after gaps of 1 to 300 CPU cycles: one switched off again, one whose low
    byte starts above top with bottom above top, one with top 0."""
    s: List[tuple] = []
    s += [("w", 0x1040, 0x30), ("w", 0x1048, 0x2A), ("w", 0x1050, 0x32), ("w", 0x1058, 0x00)]
    s += [("r", 0x1000 + f * 8) for f in (1, 7, 2, 1, 7, 2, 1, 7, 1, 2, 7, 1, 2, 7, 1, 1)]
    s += [("w", 0x1053, 0x01), ("w", 0x105B, 0x00)]
    s += [("r", 0x100B), ("r", 0x103B), ("r", 0x100B), ("r", 0x1013)]
    s += [("r", 0x1000), ("r", 0x1001), ("r", 0x1003), ("r", 0x1000), ("w", 0x1070, 0x00), ("r", 0x1002), ("r", 0x1001)]
    s += [("r", 0x101A), ("r", 0x1022), ("r", 0x102A), ("r", 0x1032), ("r", 0x103A)]
    s += [("w", 0x1045, 0x04), ("w", 0x104D, 0x01), ("w", 0x1055, 0x03), ("w", 0x105D, 0x10),
          ("w", 0x1046, 0x02), ("w", 0x104E, 0x00), ("w", 0x1056, 0x00), ("w", 0x105E, 0x10)]
    for gap in (0, 20, 30, 31, 60, 1, 90, 150, 17, 45):
        s += [("nop", gap), ("r", 0x1004), ("r", 0x103D), ("r", 0x100E)]
    s += [("w", 0x105E, 0x00), ("r", 0x100E), ("r", 0x100E), ("r", 0x103E), ("r", 0x1007), ("r", 0x100D)]
    # Fetcher 7 as a music channel whose low byte starts above top, with
    # bottom above top; then fetcher 5's top set to 0.
    s += [("w", 0x1047, 0x03), ("w", 0x104F, 0x05), ("w", 0x1057, 0x0C), ("w", 0x105F, 0x10), ("w", 0x1045, 0x00)]
    for gap in (40, 7, 250, 300, 3):
        s += [("nop", gap), ("r", 0x1007), ("r", 0x103F), ("r", 0x100F), ("r", 0x103D)]
    return s


def dpc_script_cart() -> Cart:
    """A 10,240-byte DPC cart that runs dpc_script() once, straight-line, in
    its second frame.  The reset frame only raises VSYNC; the second clears
    it, runs the script (each read stored to $80, $81, ...), raises VSYNC
    again; later frames only toggle VSYNC.  Both banks are the same image."""
    a = Asm(0xF000)
    a.org(0xF100)
    a.label("reset")
    a.ins("SEI"); a.ins("CLD"); a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    a.ins("LDA", "imm", 0x02); a.ins("STA", "zp", VSYNC)
    a.ins("LDA", "imm", 0x00); a.ins("STA", "zp", VSYNC)
    slot = 0x80
    for step in dpc_script():
        if step[0] == "w":
            a.ins("LDA", "imm", step[2]); a.ins("STA", "abs", step[1])
        elif step[0] == "r":
            a.ins("LDA", "abs", step[1]); a.ins("STA", "zp", slot)
            slot += 1
        else:
            for _ in range(step[1]):
                a.ins("NOP")
    assert slot <= 0x100
    a.label("again")
    a.ins("LDA", "imm", 0x02); a.ins("STA", "zp", VSYNC)
    a.ins("LDA", "imm", 0x00); a.ins("STA", "zp", VSYNC)
    a.ins("JMP", "abs", "again")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF1, 0x00, 0xF1]))
    img, labels, _ = a.assemble(4096)
    rom = img + img + bytes(dpc_display_byte(i) for i in range(2048))
    assert len(rom) == 10240
    return Cart(CartSpec("dpc_script", len(rom), 0, wsync_density=0.0), rom, labels, scheme=None)


# ------------------------------------------------------- phantom-access carts
# The reference CPU makes a bus access on every cycle (src/cpu.rs:245-1146),
# including reads whose value it throws away: the fix-up read of an indexed
# access at the un-carried address, the read at the next pc of a taken
# branch, RTS's read of the address it pulled, and the write of the original
# value in a read-modify-write.  On the Atari bus such an access can switch
# banks (src/atari.rs:460-492), clear the timer's underflow flag through an
# INTIM mirror (src/pia.rs:187-190) or shift the TIA's GRP0/GRP1/ENABL
# shadow registers (src/headless_tia.rs:225-298).  These carts are built to
# make every one of those accesses matter.  They break the safety rules
# above on purpose, and stay hang-free a different way: every bank holds the
# same code at the same addresses (only a bank-id byte at $FE80 differs), so
# whatever bank a phantom access selects, the next fetch finds the same
# legal instruction.
PHANTOM_BANKID = 0xFE80


def phantom_cart(rom_size: int = 8192, variant: str = "rts", passes: int = 10) -> Cart:
    """A 4K Fixed, 8K F8, 16K F6 or 32K F4 cart whose visible lines each
    exercise phantom bus accesses, with the bank they select and the values
    they read mixed into RAM:

      * indexed accesses whose fix-up read lands on a hotspot while the real
        access lands in RAM: STA/LDA/ADC/SBC/CMP abs,X, LDA abs,Y,
        LDX abs,Y, LDY abs,X, LDA/STA (zp),Y from base $1FFF with an index
        that carries into $20xx (RAM $F4-$FB);
      * STA (zp),Y without a carry (the fix-up read is the hotspot itself);
      * fix-up reads on an INTIM mirror ($0384) just after the timer
        underflowed, with INSTAT read back (LDA abs,X, LDA (zp),Y, LDY
        abs,X, LDX abs,Y, STA abs,X), with an index that carries or not;
      * read-modify-writes on GRP0, GRP1 and ENABL with vertical delay on,
        on HMOVE, and on hotspots, directly and through a carrying abs,X;
      * taken branches whose page-crossing fix-up read is a hotspot
        ($FF00 -> $FExx);
      * variant "row": a branch at the hotspot row whose next-pc read is the
        first hotspot (and, not taken, a JMP fetched from the hotspots);
        variant "rts": a JSR whose last byte is the first hotspot, so RTS's
        read of the pulled address switches banks;
      * BRK/RTI, zero-page-indexed reads whose base read reaches RAM or TIA.

    Indices, carries and branch directions come from RAM mixed with the
    inputs, so instances of one cart diverge.  Frames keep the 3 VSYNC / 36
    VBLANK skeleton with `passes` passes over the lines."""
    assert rom_size in (4096, 8192, 16384, 32768) and variant in ("row", "rts")
    nb = rom_size // 4096
    hot = _hotspots(nb) if nb > 1 else [0xFFF8]
    mask = len(hot) - 1
    lo = [h & 0xFF for h in hot]
    t_cross = [v + 1 for v in lo]                  # $1FFF + this = $20xx: fix-up read at $1Fxx
    t_nocross = [v - 0xF0 for v in lo]             # $1FF0 + this = $1Fxx
    t_intim = [0x85, 0x05]                         # $03FF + this: fix-up at $0384 (INTIM) or $0304
    a = Asm(0xF000)
    _reset_code(a)
    for reg in (0x25, 0x26, 0x27):                 # VDELP0 VDELP1 VDELBL
        a.ins("LDA", "imm", 1); a.ins("STA", "zp", reg)
    for ptr, val in ((0xE0, 0x1FFF), (0xE2, 0x1FF0), (0xE4, 0x03FF)):
        a.ins("LDA", "imm", val & 0xFF); a.ins("STA", "zp", ptr)
        a.ins("LDA", "imm", val >> 8); a.ins("STA", "zp", ptr + 1)
    a.ins("LDA", "imm", 0x70); a.ins("STA", "zp", 0x20)          # HMP0
    a.ins("LDA", "imm", 0x90); a.ins("STA", "zp", 0x24)          # HMBL
    _frame_head(a, passes)
    a.label("line")

    def end_line():
        a.ins("LDA", "abs", PHANTOM_BANKID); a.ins("EOR", "zp", MIX)
        a.ins("ADC", "zp", LINE_CTR); a.ins("STA", "zp", MIX)
        a.ins("STA", "zp", WSYNC)

    def index(reg: str, table: str, shift: int, m: int = mask):
        """reg <- table[(MIX >> shift) & m], through the other index register."""
        a.ins("LDA", "zp", MIX)
        for _ in range(shift):
            a.ins("LSR", "acc")
        a.ins("AND", "imm", m)
        if reg == "X":
            a.ins("TAY"); a.ins("LDX", "absy", table)
        else:
            a.ins("TAX"); a.ins("LDY", "absx", table)

    # --- fix-up reads on hotspots, real accesses in RAM $F4-$FB
    index("X", "t_cross", 0); a.ins("LDA", "zp", MIX); a.ins("STA", "absx", 0x1FFF); end_line()
    index("X", "t_cross", 1); a.ins("LDA", "absx", 0x1FFF); a.ins("EOR", "zp", MIX); a.ins("STA", "zp", MIX)
    end_line()
    index("Y", "t_cross", 2); a.ins("LDA", "absy", 0x1FFF); a.ins("ADC", "zp", 0x82); a.ins("STA", "zp", 0x82)
    end_line()
    index("Y", "t_cross", 3); a.ins("LDX", "absy", 0x1FFF); a.ins("STX", "zp", 0x83); end_line()
    index("X", "t_cross", 4); a.ins("LDY", "absx", 0x1FFF); a.ins("STY", "zp", 0x84); end_line()
    index("X", "t_cross", 5); a.ins("SEC"); a.ins("SBC", "absx", 0x1FFF); a.ins("STA", "zp", 0x85)
    a.ins("CMP", "absx", 0x1FFF); a.ins("ROL", "zp", 0x85); end_line()
    index("Y", "t_cross", 1); a.ins("LDA", "indy", 0xE0); a.ins("EOR", "zp", MIX); a.ins("STA", "zp", MIX)
    index("Y", "t_cross", 3); a.ins("LDA", "zp", 0x86); a.ins("STA", "indy", 0xE0); end_line()
    index("Y", "t_nocross", 2); a.ins("LDA", "zp", 0x87); a.ins("STA", "indy", 0xE2); end_line()
    # --- fix-up reads on an INTIM mirror right after a timer underflow
    for k, (mn, mode) in enumerate((("LDA", "absx"), ("LDA", "indy"), ("LDY", "absx"), ("LDX", "absy"))):
        a.ins("LDA", "imm", 0); a.ins("STA", "abs", TIM1T)
        index("Y" if mode in ("indy", "absy") else "X", "t_intim", k, 1)
        if mode == "indy":
            a.ins(mn, "indy", 0xE4)
        else:
            a.ins(mn, mode, 0x03FF)
        a.ins("LDA", "abs", INSTAT); a.ins("EOR", "zp", MIX); a.ins("STA", "zp", MIX)
        if k % 2:
            end_line()
    a.ins("LDA", "imm", 0); a.ins("STA", "abs", TIM1T)
    a.ins("LDX", "imm", 4); a.ins("LDA", "zp", 0x88); a.ins("STA", "absx", 0x0380)   # always a fix-up read
    a.ins("LDA", "abs", INSTAT); a.ins("ADC", "zp", 0x88); a.ins("STA", "zp", 0x88); end_line()
    # --- read-modify-writes: GRP0/GRP1/ENABL under VDEL, HMOVE, hotspots
    a.ins("LDA", "zp", MIX); a.ins("STA", "zp", 0x1B)
    a.ins("INC", "zp", 0x1B); a.ins("ASL", "zp", 0x1C); a.ins("LDX", "imm", 0)
    a.ins("ROL", "zpx", 0x1B); a.ins("DEC", "zp", 0x1F); a.ins("LSR", "abs", 0x011C)
    a.ins("LDX", "imm", 1); a.ins("INC", "zpx", 0x1A); a.ins("INC", "zp", 0x2A); end_line()
    a.ins("INC", "abs", hot[-1])
    index("X", "t_cross", 2); a.ins("INC", "absx", 0x1FFF)
    index("X", "t_cross", 6); a.ins("ASL", "absx", 0x1FFF); end_line()
    # --- a taken branch whose page-crossing fix-up read is a hotspot
    a.ins("LDA", "zp", MIX); a.ins("LSR", "acc"); a.ins("JMP", "abs", 0xFF00)
    a.label("br_ret")
    end_line()
    # --- the hotspot row (variant) and BRK/RTI
    a.ins("LDA", "zp", MIX); a.ins("AND", "imm", 2)
    a.ins("JMP", "abs", hot[0] - 2)
    a.label("row_ret")
    a.ins("LDA", "zp", MIX); a.ins("BRK"); a.raw(b"\xEA")
    end_line()
    # --- zero-page-indexed reads: the base read reaches RAM or the TIA
    a.ins("LDX", "zp", MIX); a.ins("LDA", "zpx", 0x80); a.ins("STA", "zp", 0x8A)
    a.ins("LDX", "imm", 0x0C); a.ins("LDA", "indx", 0x00); a.ins("EOR", "zp", 0x8A); a.ins("STA", "zp", 0x8A)
    end_line()
    _frame_tail(a)
    # --- tables and the bank id
    a.org(0xFE00)
    a.label("t_cross"); a.raw(bytes((t_cross * 8)[:8]))
    a.label("t_nocross"); a.raw(bytes((t_nocross * 8)[:8]))
    a.label("t_intim"); a.raw(bytes(t_intim))
    a.org(PHANTOM_BANKID)
    a.raw(b"\x00")
    # branch targets at $FExx (xx a hotspot's low byte): the fix-up read of
    # a taken branch from page $FF lands on $FFxx
    sites = [(0xFF00, "BCS", lo[0])]
    if lo[-1] - lo[0] >= 3:
        sites.append((0xFF10, "BCC", lo[-1]))
    for _, _, t in sorted(sites, key=lambda s: s[2]):
        a.org(0xFE00 | t)
        a.ins("JMP", "abs", "br_ret")
    for site, mn, t in sites:
        a.org(site)
        a.ins(mn, "rel", 0xFE00 | t)
        if site == 0xFF00 and len(sites) > 1:
            a.ins("JMP", "abs", 0xFF10)                             # not taken: try the other site
        else:
            a.ins("JMP", "abs", "br_ret")
    a.org(0xFF40)
    a.label("sub")
    a.ins("INC", "zp", 0x89); a.ins("RTS")
    a.org(0xFF60)
    a.label("brk")
    a.ins("PHA"); a.ins("LDA", "zp", 0x89); a.ins("ADC", "imm", 3); a.ins("STA", "zp", 0x89); a.ins("PLA")
    a.ins("RTI")
    a.org(0xFF80)
    a.label("row_far")
    a.ins("JMP", "abs", "row_ret")
    a.org(hot[0] - 2)
    if variant == "row":
        a.ins("BNE", "rel", "row_far")          # taken: next-pc read at hot[0]
        a.ins("JMP", "abs", "row_ret")          # not taken: fetched from the hotspots
    else:
        a.ins("JSR", "abs", "sub")              # its last byte is hot[0]; RTS reads it
        a.ins("JMP", "abs", "row_ret")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF0]))
    img, labels, _ = a.assemble(4096)
    img = bytearray(img)
    img[0xFFE:0x1000] = bytes([labels["brk"] & 0xFF, labels["brk"] >> 8])
    banks = []
    for b in range(nb):
        bank = bytearray(img)
        bank[PHANTOM_BANKID - 0xF000] = 0x30 + 0x11 * b
        banks.append(bytes(bank))
    name = f"phantom_{rom_size // 1024}k_{variant}"
    return Cart(CartSpec(name, rom_size, 0, wsync_density=1.0), b"".join(banks), labels)


def phantom_carts() -> List[Cart]:
    """Every phantom-access cart: 4K Fixed, and F8, F6 and F4 in both variants."""
    out = [phantom_cart(4096, "rts")]
    for size in (8192, 16384, 32768):
        out += [phantom_cart(size, "row"), phantom_cart(size, "rts")]
    return out


# ------------------------------------------------------------- failure carts
def stall_cart(kind: str) -> Cart:
    """A 4K Fixed cart for the frame loop's limits (src/atari.rs:584-598):

      * "no_vsync": never writes VSYNC, so every frame runs to the
        reference's 100,000-cycle cap (FA_STATUS_CYCLE_CAP, informational);
      * "vsync_held": raises VSYNC once and never lowers it, so the frame
        after the reset frame waits for VSYNC to drop forever (the reference
        loops; this library halts the instance with FA_STATUS_VSYNC_BUDGET
        after 2,000,000 cycles).

    Both loops read the inputs and the timer into RAM and end lines with
    STA WSYNC, so the state keeps changing while they run."""
    assert kind in ("no_vsync", "vsync_held")
    a = Asm(0xF000)
    _reset_code(a)
    a.ins("LDA", "imm", 43); a.ins("STA", "abs", TIM64T)
    if kind == "vsync_held":
        a.ins("LDA", "imm", 2); a.ins("STA", "zp", VSYNC)
    a.label("loop")
    a.ins("LDA", "abs", SWCHA); a.ins("EOR", "zp", MIX); a.ins("ADC", "abs", INTIM); a.ins("STA", "zp", MIX)
    a.ins("INC", "zp", LINE_CTR)
    a.ins("BNE", "rel", "skip")
    a.ins("LDA", "imm", 43); a.ins("STA", "abs", TIM64T)
    a.label("skip")
    a.ins("LDA", "zp", LINE_CTR); a.ins("AND", "imm", 0x7F); a.ins("TAX")
    a.ins("LDA", "zp", MIX); a.ins("STA", "zpx", 0x80)                 # RAM $80-$FF
    a.ins("STA", "zp", WSYNC)
    a.ins("JMP", "abs", "loop")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF0, 0x00, 0xF0]))
    img, labels, _ = a.assemble(4096)
    return Cart(CartSpec(f"stall_{kind}", 4096, 0, wsync_density=1.0), img, labels)


# ------------------------------------------------------- instruction-cost carts
MICRO_KINDS = {
    "nop": [("NOP", "imp", None)],
    "lda_imm": [("LDA", "imm", 0x12)],
    "lda_zp": [("LDA", "zp", 0x85)],
    "sta_zp": [("STA", "zp", 0x86)],
    "adc_zp": [("ADC", "zp", 0x87)],
    "inc_zp": [("INC", "zp", 0x88)],
    "lda_absx": [("LDA", "absx", 0x0090)],
    "lda_rom": [("LDA", "abs", 0xF800)],
    "lda_indy": [("LDA", "indy", 0x90)],
    "sta_tia": [("STA", "zp", 0x09)],
    "lda_intim": [("LDA", "abs", 0x284)],
    "tax_inx": [("TAX", "imp", None), ("INX", "imp", None)],
}


def micro_cart(kind: str, reps: int = 24) -> Cart:
    """A 4K Fixed cart whose 192 visible lines each run `reps` copies of one
    instruction kind (MICRO_KINDS) and STA WSYNC, inside the frame skeleton
    (3 VSYNC, 37 VBLANK, 192 visible, 30 overscan lines).  Run converged
    (identical instances and actions), it gives the cost of one guest
    instruction of that kind."""
    a = Asm()
    a.label("reset"); a.ins("SEI"); a.ins("CLD"); a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    a.ins("LDA", "imm", 0); a.ins("LDX", "imm", 0x80)
    a.label("clr"); a.ins("STA", "zpx", 0); a.ins("INX"); a.ins("BNE", "rel", "clr")
    a.label("frame")
    a.ins("LDA", "imm", 2); a.ins("STA", "zp", VSYNC)
    for _ in range(3):
        a.ins("STA", "zp", WSYNC)
    a.ins("LDA", "imm", 0); a.ins("STA", "zp", VSYNC)
    _wsync_lines(a, 37, "vb")
    a.ins("LDA", "imm", 192); a.ins("STA", "zp", LINE_CTR)
    a.ins("LDX", "imm", 0); a.ins("LDY", "imm", 0)
    a.label("line")
    for _ in range(reps):
        for mn, mode, arg in MICRO_KINDS[kind]:
            a.ins(mn, mode, arg)
    a.ins("STA", "zp", WSYNC); a.ins("DEC", "zp", LINE_CTR); a.ins("BEQ", "rel", "ov"); a.ins("JMP", "abs", "line")
    a.label("ov")
    _wsync_lines(a, 30, "os")
    a.ins("JMP", "abs", "frame")
    a.org(0xFFFC)
    a.raw(bytes([0x00, 0xF0, 0x00, 0xF0]))
    img, labels, _ = a.assemble(4096)
    return Cart(CartSpec(f"micro_{kind}", 4096, 0, wsync_density=1.0), img, labels)
