"""Generate tests/golden/oracle_vectors.json: self-generated regression vectors.

The reference's frame-level tests need Breakout.bin, which is unavailable, so
frame-level parity is anchored on these frozen oracle outputs for the seeded
synthetic carts (the oracle itself is pinned at instruction level by the
reference's tests/cycle_counts.rs KATs).  Run from the repository root:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
from fa_pkg import carts  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "plain": (carts.plain_cart, 16, 120, 101),
    "divergence": (carts.divergence_cart, 16, 60, 102),
    "scale": (carts.scale_cart, 16, 60, 103),
    "mixed_2k": (lambda: carts.mixed_carts()[0], 16, 60, 104),
    "mixed_8k": (lambda: carts.mixed_carts()[1], 16, 60, 105),
    "mixed_16k": (lambda: carts.mixed_carts()[2], 16, 60, 106),
    "mixed_32k": (lambda: carts.mixed_carts()[3], 16, 60, 107),
    # Schemes the reference lacks, registered per ROM for the run (cart.scheme).
    "e0_8k": (carts.e0_cart, 16, 30, 108),
    "3f_16k": (lambda: carts.f3_cart(16384), 16, 30, 109),
    "3f_6k": (lambda: carts.f3_cart(6144), 16, 30, 110),
    # DPC, picked by its length.
    "dpc_10k": (carts.dpc_cart, 16, 30, 111),
    # FE, registered per ROM.
    "fe_8k": (carts.fe_cart, 16, 30, 112),
}
CHECKPOINTS = (1, 10, 30)


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


# fa_state's bytes before the DPC registers.  A state whose DPC registers are
# all zero (every scheme but DPC) hashes as those bytes, which keeps the
# vectors frozen before the registers were added valid; any other hashes whole.
PRE_DPC_BYTES = 240


def state_sha(st) -> str:
    b = np.ascontiguousarray(st).view(np.uint8).reshape(len(st), -1)
    return sha(b[:, :PRE_DPC_BYTES].tobytes() if not b[:, PRE_DPC_BYTES:].any() else b.tobytes())


def vectors(name):
    make, n, frames, seed = CASES[name]
    cart = make()
    rom = cart.rom
    if cart.scheme:
        oracle.set_rom_scheme(rom, cart.scheme)
    try:
        acts = carts.actions(seed=seed, n=n, frames=frames)
        st = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
        trace, instr = oracle.run_batch(rom, st, acts, frames, trace=True)
        reset_sha = state_sha(np.array([oracle.reset_state(rom)], dtype=oracle.STATE_DTYPE))
    finally:
        if cart.scheme:
            oracle.set_rom_scheme(rom, "auto")
    return {
        "rom_sha256": sha(rom), "n": n, "frames": frames, "action_seed": seed,
        "reset_state_sha256": reset_sha,
        "ram_sha256_at": {str(f): sha(trace[f - 1].tobytes()) for f in CHECKPOINTS + (frames,)},
        "final_state_sha256": state_sha(st),
        "instructions": instr,
        "final_pc": [int(x) for x in st["pc"]],
        "final_cycles": [int(x) for x in st["cycles"]],
    }


if __name__ == "__main__":
    out = {name: vectors(name) for name in CASES}
    (HERE / "oracle_vectors.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "oracle_vectors.json")
