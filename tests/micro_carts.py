"""Instruction-cost micro-carts: one instruction kind per visible line.

    python tests/micro_carts.py [kind ...]

Not collected by pytest (it times).  Each 4K Fixed cart has the frame skeleton
(3 VSYNC, 37 VBLANK, 192 visible, 30 overscan lines) and visible lines of 24
copies of one instruction kind (NOP, LDA #imm, LDA zp, STA zp, ADC zp, INC zp,
LDA abs,X, LDA from ROM, LDA (zp),Y, STA to a TIA register, LDA INTIM, TAX+INX).
151,552 identical instances with all actions 0 run converged (K=2, three
calls, CUDA events on the launching stream); the oracle gives the exact guest
instructions per frame.  The result is the cost of one guest instruction of
that kind in warp-issue slots at 100 % issue (148 SMs x 4 schedulers x clock /
(guest instr/s / 32)), which separates the fixed per-instruction work (fetch,
decode, ticks, scheduling) from the work each kind adds.
"""
import json
import sys
from pathlib import Path
ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests")); sys.path.insert(0, str(ROOT / "oracle"))
import numpy as np
from fa_pkg import carts, fa
from fast_atari_b200.carts import Asm
import oracle

def micro(kind, reps=24):
    a = Asm()
    a.label("reset"); a.ins("SEI"); a.ins("CLD"); a.ins("LDX", "imm", 0xFF); a.ins("TXS")
    a.ins("LDA", "imm", 0); a.ins("LDX", "imm", 0x80)
    a.label("clr"); a.ins("STA", "zpx", 0); a.ins("INX"); a.ins("BNE", "rel", "clr")
    a.label("frame")
    a.ins("LDA", "imm", 2); a.ins("STA", "zp", 0x00)
    for _ in range(3): a.ins("STA", "zp", 0x02)
    a.ins("LDA", "imm", 0); a.ins("STA", "zp", 0x00)
    a.ins("LDX", "imm", 37); a.label("vb"); a.ins("STA", "zp", 0x02); a.ins("DEX"); a.ins("BNE", "rel", "vb")
    a.ins("LDA", "imm", 192); a.ins("STA", "zp", 0x80)
    a.ins("LDX", "imm", 0); a.ins("LDY", "imm", 0)
    a.label("line")
    body = {
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
    }[kind]
    for _ in range(reps):
        for mn, mode, arg in body:
            a.ins(mn, mode, arg)
    a.ins("STA", "zp", 0x02); a.ins("DEC", "zp", 0x80); a.ins("BEQ", "rel", "ov"); a.ins("JMP", "abs", "line")
    a.label("ov")
    a.ins("LDX", "imm", 30); a.label("os"); a.ins("STA", "zp", 0x02); a.ins("DEX"); a.ins("BNE", "rel", "os")
    a.ins("JMP", "abs", "frame")
    a.org(0xFFFC); a.raw(bytes([0x00, 0xF0, 0x00, 0xF0]))
    out = a.assemble(4096)
    img = out[0]
    return bytes(img)

KINDS = ["nop", "lda_imm", "lda_zp", "sta_zp", "adc_zp", "inc_zp", "lda_absx", "lda_rom", "lda_indy",
         "sta_tia", "lda_intim", "tax_inx"]


def main(kinds):
    import torch
    n, k, calls = 151552, 2, 3
    s = torch.cuda.Stream()
    acts = torch.zeros(k * n, dtype=torch.uint8, device="cuda")
    for kind in kinds:
        rom = micro(kind)
        at = oracle.Atari(rom)
        at.run_frame()
        i0 = at.instructions()
        at.run_frame()
        ipf = at.instructions() - i0
        with fa.BatchAtariGpu(rom, n) as g:
            g.set_launch(128, "pc", True)
            g.reset()
            g.step_multi_async(acts.data_ptr(), k, 0, s.cuda_stream)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(calls):
                g.step_multi_async(acts.data_ptr(), k, 0, s.cuda_stream)
            e1.record(s)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        gis = ipf * n * k * calls / (ms / 1e3)
        res = {"instr_per_frame": ipf, "guest_instr_per_s": gis,
               "issue_slots_per_guest_instr_at_100pct": 148 * 4 * 1.965e9 / (gis / 32)}
        print(kind, json.dumps({k2: round(v, 1) for k2, v in res.items()}), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or KINDS)
