"""Known-answer tests of the oracle CPU core.

Restates the reference's instruction-level golden values, tests/cycle_counts.rs
(29 tests, lines 38-366), on FlatMemory with the reset vector at $8000.  These
pin the oracle's 6502 to the reference at instruction level.
"""
import numpy as np
import pytest

import oracle


def mem_with(code=b"", at=0x8000, extra=None, vec=0x8000):
    m = np.zeros(65536, np.uint8)
    m[at:at + len(code)] = np.frombuffer(bytes(code), np.uint8)
    m[0xFFFC] = vec & 0xFF
    m[0xFFFD] = vec >> 8
    for a, v in (extra or {}).items():
        m[a] = v
    return m


def run_one(code):                      # cycle_counts.rs:4-17
    regs, cyc, n = oracle.flat_run(mem_with(code), 1)
    assert n == 1
    return regs, int(cyc[0])


def run_n(code, n):                     # cycle_counts.rs:20-34
    m = mem_with(code)
    regs, cyc, ran = oracle.flat_run(m, n)
    assert ran == n
    return regs, m, int(cyc.sum())


def test_reset_vector():                # cycle_counts.rs:13
    regs, _, _ = oracle.flat_run(mem_with(b"\xEA"), 0)
    assert regs.pc == 0x8000 and regs.sp == 0xFD and regs.p == 0


def test_nop_cycles():
    assert run_one([0xEA])[1] == 2


def test_tax_cycles():
    assert run_one([0xAA])[1] == 2


def test_inx_cycles():
    assert run_one([0xE8])[1] == 2


def test_asl_accumulator_cycles():
    assert run_one([0x0A])[1] == 2


def test_lda_immediate_cycles():
    regs, c = run_one([0xA9, 0x42])
    assert c == 2 and regs.a == 0x42


def test_adc_immediate_cycles():
    assert run_one([0x69, 0x10])[1] == 2


def test_lda_zero_page_cycles():
    m = mem_with([0xA5, 0x42], extra={0x42: 0xBE})
    regs, cyc, _ = oracle.flat_run(m, 1)
    assert cyc[0] == 3 and regs.a == 0xBE


def test_inc_zero_page_cycles():
    assert run_n([0xE6, 0x50], 1)[2] == 5


def test_lda_zero_page_x_cycles():
    assert run_one([0xB5, 0x10])[1] == 4


def test_lda_absolute_cycles():
    assert run_one([0xAD, 0x00, 0x90])[1] == 4


def test_jmp_absolute_cycles():
    regs, c = run_one([0x4C, 0x00, 0x90])
    assert c == 3 and regs.pc == 0x9000


def test_jsr_rts_cycles():
    m = mem_with([0x20, 0x10, 0x80], extra={0x8010: 0x60})
    regs, cyc, _ = oracle.flat_run(m, 1)
    assert cyc[0] == 6 and regs.pc == 0x8010
    regs, cyc, _ = oracle.flat_run(m, 1, regs)
    assert cyc[0] == 6 and regs.pc == 0x8003


def test_inc_absolute_cycles():
    assert run_n([0xEE, 0x00, 0x90], 1)[2] == 6


def test_lda_absolute_x_no_cross_cycles():
    assert run_n([0xA2, 0x01, 0xBD, 0x00, 0x90], 2)[2] == 2 + 4


def test_lda_absolute_x_page_cross_cycles():
    assert run_n([0xA2, 0xFF, 0xBD, 0xFF, 0x90], 2)[2] == 2 + 5


def test_lda_absolute_y_no_cross_cycles():
    assert run_n([0xA0, 0x01, 0xB9, 0x00, 0x90], 2)[2] == 2 + 4


def test_lda_absolute_y_page_cross_cycles():
    assert run_n([0xA0, 0xFF, 0xB9, 0xFF, 0x90], 2)[2] == 2 + 5


def test_sta_absolute_x_always_5_cycles():
    assert run_n([0xA2, 0xFF, 0x9D, 0xFF, 0x90], 2)[2] == 2 + 5


def test_lda_indirect_y_no_cross_cycles():
    m = mem_with([0xA0, 0x01, 0xB1, 0x20], extra={0x20: 0x00, 0x21: 0x90})
    _, cyc, _ = oracle.flat_run(m, 2)
    assert list(cyc) == [2, 5]


def test_lda_indirect_y_page_cross_cycles():
    m = mem_with([0xA0, 0x01, 0xB1, 0x20], extra={0x20: 0xFF, 0x21: 0x90})
    _, cyc, _ = oracle.flat_run(m, 2)
    assert list(cyc) == [2, 6]


def test_lda_indirect_x_cycles():
    m = mem_with([0xA2, 0x01, 0xA1, 0x20], extra={0x21: 0x00, 0x22: 0x90})
    _, cyc, _ = oracle.flat_run(m, 2)
    assert cyc[1] == 6


def test_branch_not_taken_cycles():
    assert run_n([0x18, 0xB0, 0x10], 2)[2] == 2 + 2


def test_branch_taken_no_cross_cycles():
    regs, _, c = run_n([0x38, 0xB0, 0x02], 2)
    assert c == 2 + 3 and regs.pc == 0x8005


def test_branch_taken_page_cross_cycles():
    m = mem_with(extra={0x80FD: 0x38, 0x80FE: 0xB0, 0x80FF: 0xFB}, vec=0x80FD)
    regs, cyc, _ = oracle.flat_run(m, 1)
    assert cyc[0] == 2 and regs.pc == 0x80FE
    regs, cyc, _ = oracle.flat_run(m, 1, regs)
    assert cyc[0] == 4 and regs.pc == 0x80FB


def test_pha_pla_cycles():
    regs, _, c = run_n([0xA9, 0x42, 0x48, 0xA9, 0x00, 0x68], 4)
    assert c == 2 + 3 + 2 + 4 and regs.a == 0x42


def test_php_plp_cycles():
    assert run_n([0x08, 0x28], 2)[2] == 3 + 4


def test_asl_absolute_cycles():
    assert run_n([0x0E, 0x00, 0x90], 1)[2] == 6


def test_asl_absolute_x_cycles():
    assert run_n([0xA2, 0xFF, 0x1E, 0xFF, 0x90], 2)[2] == 2 + 7


def test_brk_cycles():
    m = mem_with([0x00], extra={0xFFFE: 0x00, 0xFFFF: 0x90, 0x9000: 0x40})
    regs, cyc, _ = oracle.flat_run(m, 1)
    assert cyc[0] == 7 and regs.pc == 0x9000
    regs, cyc, _ = oracle.flat_run(m, 1, regs)
    assert cyc[0] == 6 and regs.pc == 0x8002


# ---- beyond the reference KATs: properties the reference code implies ----

def test_illegal_opcode_stops():
    """Illegal opcodes panic in the reference (src/cpu.rs:1139); the oracle
    reports 0 cycles and stops with pc past the opcode."""
    regs, cyc, n = oracle.flat_run(mem_with([0xEA, 0x02]), 3)
    assert n == 1 and cyc[1] == 0 and regs.pc == 0x8002


def test_legal_opcode_count():
    """151 legal opcodes (src/cpu.rs:253-1141)."""
    legal = 0
    for op in range(256):
        m = mem_with([op, 0x00, 0x90])
        _, cyc, n = oracle.flat_run(m, 1)
        legal += int(n == 1)
    assert legal == 151


def test_decimal_adc_sbc():
    """BCD: SED; CLC; LDA #$45; ADC #$38 -> $83; SEC; SBC #$19 -> $64."""
    regs, _, _ = run_n([0xF8, 0x18, 0xA9, 0x45, 0x69, 0x38], 4)
    assert regs.a == 0x83
    regs, _, _ = run_n([0xF8, 0x18, 0xA9, 0x45, 0x69, 0x38, 0x38, 0xE9, 0x19], 6)
    assert regs.a == 0x64 and regs.p & 1


def test_jmp_indirect_page_bug():
    m = mem_with([0x6C, 0xFF, 0x30], extra={0x30FF: 0x34, 0x3000: 0x12, 0x3100: 0x99})
    regs, cyc, _ = oracle.flat_run(m, 1)
    assert cyc[0] == 5 and regs.pc == 0x1234


# ---- the same KATs on the 2600 bus (the form the GPU tests run them in) ----

@pytest.mark.parametrize("name", [k.name for k in __import__("kat_2600").KATS])
def test_reference_kats_relocated_to_the_2600_bus(name):
    """Each KAT as a 4K Fixed cart from $F100, run for one frame by the
    oracle's Atari console, gives the values of tests/cycle_counts.rs once
    the terminator's share is taken off (kat_2600.py)."""
    import kat_2600
    k = next(k for k in kat_2600.KATS if k.name == name)
    rom = k.image()
    st = kat_2600.kat_start_state(k, rom)
    oracle.run_batch(rom, st, np.zeros((1, 1), np.uint8), 1)
    assert st["run_status"][0] == 0
    kat_2600.check_kat(k, st[0], "oracle")
