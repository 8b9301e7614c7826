"""The reference's instruction KATs (tests/cycle_counts.rs:38-366) as 4K
Fixed carts for the 2600 bus, with the terminator that lets a frame-stepping
core report one instruction sequence's registers, pc and cycles.

The reference runs its KATs on a flat 64K memory from $8000; on the 2600 bus
$8000 is the TIA, so each byte sequence runs from $F100 of a 4K Fixed cart
(the reference's $80xx becomes $F1xx), zero-page fixtures move up by $80
into the PIA RAM ($20 -> $A0, $42 -> $C2; $00-$7F are TIA registers), and
absolute operands ($9000, $90FF) stay as they are (ROM on the 2600 bus).
Cycle counts do not depend on the address.  The start state is the
reference's post-reset register file (A=X=Y=0, SP=$FD, P=0, cycles 0) at the
sequence's first byte, with VSYNC off; one frame runs the sequence and then
a terminator that ends the frame without disturbing what is checked:
  brk   - a BRK where the checked instructions leave the pc: it pushes pc+2
          and P|B|U, and its handler stores A in $80 and writes VSYNC
          (7 + 8 cycles);
  plain - STA $80, LDA #2, STA VSYNC (8 cycles), where the KAT's own BRK
          owns the interrupt vector.
"""
import numpy as np

import oracle

E = 0xF100                   # the reference's $8000
HANDLER = 0xFE00             # BRK terminator's handler
T_PLAIN = bytes([0x85, 0x80, 0xA9, 0x02, 0x85, 0x00])      # STA $80; LDA #2; STA VSYNC


class Kat:
    def __init__(self, name, code, stop, expect, ram=None, rom=None, entry=E, term="brk", vector=None, line=0):
        self.name, self.code, self.stop, self.expect = name, bytes(code), stop, expect
        self.ram, self.rom, self.entry, self.term, self.vector = ram or {}, rom or {}, entry, term, vector
        self.line = line

    def image(self) -> bytes:
        img = bytearray(4096)
        for i, b in enumerate(self.code):
            img[(self.entry + i) & 0xFFF] = b
        for a, b in self.rom.items():
            img[a & 0xFFF] = b
        if self.term == "brk":
            img[self.stop & 0xFFF] = 0x00
            img[HANDLER & 0xFFF:(HANDLER & 0xFFF) + len(T_PLAIN)] = T_PLAIN
            vec = HANDLER
        else:
            img[self.stop & 0xFFF:(self.stop & 0xFFF) + len(T_PLAIN)] = T_PLAIN
            vec = self.vector
        img[0xFFC:0x1000] = bytes([self.entry & 0xFF, self.entry >> 8, vec & 0xFF, vec >> 8])
        return bytes(img)


# (name, bytes at $F100, where the checked instructions leave the pc, checks)
# with the line of tests/cycle_counts.rs that holds the values.
KATS = [
    Kat("nop", [0xEA], E + 1, {"cycles": 2}, line=39),
    Kat("tax", [0xAA], E + 1, {"cycles": 2}, line=45),
    Kat("inx", [0xE8], E + 1, {"cycles": 2}, line=51),
    Kat("asl_accumulator", [0x0A], E + 1, {"cycles": 2}, line=57),
    Kat("lda_immediate", [0xA9, 0x42], E + 2, {"cycles": 2, "a": 0x42}, line=65),
    Kat("adc_immediate", [0x69, 0x10], E + 2, {"cycles": 2}, line=72),
    Kat("lda_zero_page", [0xA5, 0xC2], E + 2, {"cycles": 3, "a": 0xBE}, ram={0xC2: 0xBE}, line=80),
    Kat("inc_zero_page", [0xE6, 0x50], E + 2, {"cycles": 5}, line=94),
    Kat("lda_zero_page_x", [0xB5, 0x10], E + 2, {"cycles": 4}, line=102),
    Kat("lda_absolute", [0xAD, 0x00, 0x90], E + 3, {"cycles": 4}, line=110),
    Kat("jmp_absolute", [0x4C, 0x00, 0x90], 0x9000, {"cycles": 3, "pc": 0x9000}, line=116),
    Kat("jsr", [0x20, 0x10, 0xF1], E + 0x10, {"cycles": 6, "pc": E + 0x10}, line=129),
    Kat("jsr_rts", [0x20, 0x10, 0xF1], E + 3, {"cycles": 6 + 6, "pc": E + 3}, rom={E + 0x10: 0x60}, line=129),
    Kat("inc_absolute", [0xEE, 0x00, 0x90], E + 3, {"cycles": 6}, line=150),
    Kat("lda_absolute_x_no_cross", [0xA2, 0x01, 0xBD, 0x00, 0x90], E + 5, {"cycles": 2 + 4}, line=158),
    Kat("lda_absolute_x_page_cross", [0xA2, 0xFF, 0xBD, 0xFF, 0x90], E + 5, {"cycles": 2 + 5}, line=168),
    Kat("lda_absolute_y_no_cross", [0xA0, 0x01, 0xB9, 0x00, 0x90], E + 5, {"cycles": 2 + 4}, line=178),
    Kat("lda_absolute_y_page_cross", [0xA0, 0xFF, 0xB9, 0xFF, 0x90], E + 5, {"cycles": 2 + 5}, line=187),
    Kat("sta_absolute_x_always_5", [0xA2, 0xFF, 0x9D, 0xFF, 0x90], E + 5, {"cycles": 2 + 5}, line=196),
    Kat("ldy_immediate_prefix", [0xA0, 0x01], E + 2, {"cycles": 2, "y": 1}, line=217),
    Kat("lda_indirect_y_no_cross", [0xA0, 0x01, 0xB1, 0xA0], E + 4, {"cycles": 2 + 5},
        ram={0xA0: 0x00, 0xA1: 0x90}, line=205),
    Kat("lda_indirect_y_page_cross", [0xA0, 0x01, 0xB1, 0xA0], E + 4, {"cycles": 2 + 6},
        ram={0xA0: 0xFF, 0xA1: 0x90}, line=223),
    Kat("lda_indirect_x", [0xA2, 0x01, 0xA1, 0xA0], E + 4, {"cycles": 2 + 6},
        ram={0xA1: 0x00, 0xA2: 0x90}, line=243),
    Kat("branch_not_taken", [0x18, 0xB0, 0x10], E + 3, {"cycles": 2 + 2}, line=262),
    Kat("branch_taken_no_cross", [0x38, 0xB0, 0x02], E + 5, {"cycles": 2 + 3, "pc": E + 5}, line=270),
    Kat("branch_page_cross_sec", [0x38], 0xF1FE, {"cycles": 2, "pc": 0xF1FE}, entry=0xF1FD, line=280),
    Kat("branch_taken_page_cross", [0x38, 0xB0, 0xFB], 0xF1FB, {"cycles": 2 + 4, "pc": 0xF1FB},
        entry=0xF1FD, line=280),
    Kat("pha_pla", [0xA9, 0x42, 0x48, 0xA9, 0x00, 0x68], E + 6, {"cycles": 2 + 3 + 2 + 4, "a": 0x42}, line=313),
    Kat("php_plp", [0x08, 0x28], E + 2, {"cycles": 3 + 4}, line=321),
    Kat("asl_absolute", [0x0E, 0x00, 0x90], E + 3, {"cycles": 6}, line=329),
    Kat("asl_absolute_x", [0xA2, 0xFF, 0x1E, 0xFF, 0x90], E + 5, {"cycles": 2 + 7}, line=337),
    Kat("brk", [0x00], 0x9000, {"cycles": 7, "pc": 0x9000}, term="plain", vector=0x9000, line=346),
    Kat("brk_rti", [0x00], E + 2, {"cycles": 7 + 6, "pc": E + 2}, rom={0x9000: 0x40}, term="plain",
        vector=0x9000, line=346),
    # beyond the file: decimal mode and the JMP (ind) page wrap (src/cpu.rs:153-200, 961-978)
    Kat("decimal_adc_sbc", [0xF8, 0x18, 0xA9, 0x45, 0x69, 0x38, 0x38, 0xE9, 0x19], E + 9,
        {"cycles": 2 * 6, "a": 0x64, "p_c": 1}),
    Kat("jmp_indirect_page_wrap", [0x6C, 0xFF, 0xF3], 0xF234, {"cycles": 5, "pc": 0xF234},
        rom={0xF3FF: 0x34, 0xF300: 0xF2, 0xF400: 0x99}),
]


def kat_start_state(k: Kat, rom: bytes) -> np.ndarray:
    s = np.array([oracle.reset_state(rom)], dtype=oracle.STATE_DTYPE)
    s["a"], s["x"], s["y"], s["sp"], s["status"] = 0, 0, 0, 0xFD, 0     # Cpu::new + reset (cpu.rs:125-134)
    s["pc"] = k.entry
    s["cycles"], s["frame_no"], s["run_status"] = 0, 0, 0
    s["tia_vsync"], s["tia_wsync"] = 0, 0
    s["ram"] = 0
    for a, v in k.ram.items():
        s["ram"][0, a & 0x7F] = v
    return s


def kat_recover(k: Kat, st) -> dict:
    """The checked instructions' registers, pc and cycles from the state the
    terminator left."""
    ram = st["ram"]
    if k.term == "brk":
        sp = int(st["sp"])
        pc = (int(ram[(sp + 3) & 0x7F]) << 8 | int(ram[(sp + 2) & 0x7F])) - 2
        return {"a": int(ram[0]), "x": int(st["x"]), "y": int(st["y"]), "sp": (sp + 3) & 0xFF,
                "p_c": int(ram[(sp + 1) & 0x7F]) & 1, "pc": pc & 0xFFFF, "cycles": int(st["cycles"]) - 15}
    return {"a": int(ram[0]), "x": int(st["x"]), "y": int(st["y"]), "sp": int(st["sp"]),
            "pc": (int(st["pc"]) - 6) & 0xFFFF, "cycles": int(st["cycles"]) - 8}


def check_kat(k: Kat, st, what):
    got = kat_recover(k, st)
    for key, want in k.expect.items():
        assert got[key] == want, f"{what} {k.name} (cycle_counts.rs:{k.line}): {key} = {got[key]:#x}, want {want:#x}"
