"""Tune every cart of a benchmark workload and write the tuning records.

    python fast-atari-rs_b200/tune.py [--workload mixed] [--out tuning.json]

Each record is fa_autotune's best configuration for that cart at its
workload instance count (warp policy, launch shape / register cap, frames per
launch) plus its measured cost per instance-frame, which bench.py and pools
use as the queue-ordering weight (heaviest units first).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent


def _pkg():
    if "fast_atari_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            "fast_atari_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["fast_atari_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["fast_atari_b200"]


def tune_workload(carts_with_counts, cap: int = 150_000, keep: int = 6):
    """Per cart: fa_autotune's best record, its cost per instance-frame as
    the queue weight, and the `keep` fastest measured configurations (the
    sweep's table of alternatives).  In a pool every cart shares one launch,
    so only the policy and the weight apply there; the launch shape and K
    apply when the cart runs on a handle of its own (fa_set_launch,
    fa_set_cta_warps, step_multi's k)."""
    fa = _pkg()
    names = {v: k for k, v in fa.SCHED_NAMES.items()}
    out = {}
    for cart, n in carts_with_counts:
        best, table = fa.autotune(cart.rom, min(n, cap))
        best["sched_name"] = names[best["sched"]]
        best["weight"] = best["ns_per_instance_frame"]
        best["instances"] = min(n, cap)
        best["measurements"] = len(table)
        alts = sorted(table, key=lambda t: -t["frames_per_s"])[:keep]
        best["alternatives"] = [{"sched": names[t["sched"]], "persistent": t["persistent"], "cta_warps": t["cta_warps"],
                                 "block": t["block"], "k": t["k"], "frames_per_s": round(t["frames_per_s"])}
                                for t in alts]
        best["applied_in_pool"] = ["sched", "weight"]
        out[cart.spec.name] = best
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixed", choices=["mixed", "divergence", "plain", "scale"])
    ap.add_argument("--out", default="tuning.json")
    args = ap.parse_args()
    _pkg()
    from fast_atari_b200 import carts
    spec = {"mixed": lambda: list(zip(carts.mixed_carts(), carts.MIXED_COUNTS)),
            "divergence": lambda: [(carts.divergence_cart(), 50_000)],
            "plain": lambda: [(carts.plain_cart(), 1000)],
            "scale": lambda: [(carts.scale_cart(), 1_000_000)]}[args.workload]()
    rec = tune_workload(spec)
    Path(args.out).write_text(json.dumps(rec, indent=1) + "\n")
    for name, r in rec.items():
        print(f"{name}: sched={r['sched_name']} persistent={r['persistent']} cta_warps={r['cta_warps']} "
              f"block={r['block']} k={r['k']} {r['frames_per_s']:.0f} frames/s")


if __name__ == "__main__":
    main()
