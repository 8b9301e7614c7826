"""The reference's own CUDA kernels vs this repository's, on one B200.

    python tests/ref_cuda_compare.py [--instances 50000] [--frames 16]

Not collected by pytest (it times; it asserts nothing about speed).  The
reference kernels (cuda/src/atari_kernel.cu of RPP1011/fast-atari-rs, built
for sm_100a by `make -C oracle ref` into oracle/_ref/) and this library run
the same seeded Fixed-mapper carts — the plain 4K cart of the CPU-runnable
configuration and the 2K cart of the mixed batch — from the same post-reset
states with the same actions; each side is timed with CUDA events around its
launches only (state resident on the device).  Both sides' RAM is compared
with the CPU oracle: this library must match it bit for bit; the reference
kernels skip the Rust emulator's phantom bus accesses and may not.  Only
Fixed-mapper carts are run: on them control flow cannot reach a byte that is
not a legal opcode, which the reference kernels would execute as a 0-cycle
NOP and never finish the frame.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))
from fa_pkg import carts, fa  # noqa: E402
import oracle  # noqa: E402

REF_LIB = ROOT / "oracle" / "_ref" / "libref_cuda.so"


def ref_lib():
    if not REF_LIB.exists():
        raise SystemExit(f"{REF_LIB} missing: run `make -C oracle ref` where the reference is mounted")
    L = ctypes.CDLL(str(REF_LIB))
    L.ref_state_size.restype = ctypes.c_int
    L.ref_run.restype = ctypes.c_int
    L.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
    return L


def ref_states(rom: bytes, n: int, size: int) -> np.ndarray:
    """n copies of the post-reset state in the reference's AtariState layout:
    the first 221 bytes of fa_state are that layout (include/fast_atari.h)."""
    snap = np.array([oracle.reset_state(rom)], dtype=oracle.STATE_DTYPE).view(np.uint8)[:221]
    one = np.zeros(size, np.uint8)
    one[:221] = snap
    return np.tile(one, n)


def time_ref(L, rom, n, acts, k, multi, sorted_):
    st = ref_states(rom, n, L.ref_state_size())
    r = np.frombuffer(rom, np.uint8).copy()
    obs = np.empty((n, 128), np.uint8)
    a = np.ascontiguousarray(acts, dtype=np.uint8).reshape(-1)
    ms = ctypes.c_float()
    rc = L.ref_run(r.ctypes.data, len(r), st.ctypes.data, n, a.ctypes.data, k, multi, sorted_, obs.ctypes.data,
                   ctypes.byref(ms))
    if rc:
        raise RuntimeError(f"ref_run failed: cudaError {rc}")
    return ms.value, obs


def time_ours(rom, n, acts, k, multi):
    import torch
    d_acts = torch.from_numpy(np.ascontiguousarray(acts).reshape(-1)).cuda()
    s = torch.cuda.Stream()
    d_obs = torch.empty(n * 128, dtype=torch.uint8, device="cuda")
    with fa.BatchAtariGpu(rom, n) as g:
        g.set_launch(128, "pc", bool(multi))
        g.reset()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        if multi:
            g.step_multi_async(d_acts.data_ptr(), k, d_obs.data_ptr(), s.cuda_stream)
        else:
            for f in range(k):
                g.step_multi_async(d_acts.data_ptr() + f * n, 1, d_obs.data_ptr(), s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), d_obs.cpu().numpy().reshape(n, 128)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, nargs="*", default=[1000, 50000])
    ap.add_argument("--frames", type=int, default=16)
    ap.add_argument("--check", type=int, default=256, help="instances compared with the oracle")
    args = ap.parse_args()
    L = ref_lib()
    out = {"ref_state_bytes": L.ref_state_size(), "rows": []}
    mixed2k = carts.mixed_carts()[0]
    for name, rom in (("plain_4k_fixed", carts.plain_cart().rom), ("mixed_2k_fixed", mixed2k.rom)):
        for n in args.instances:
            k = args.frames
            acts = carts.actions(seed=9, n=n, frames=k)
            m = min(n, args.check)
            ref_st = np.array([oracle.reset_state(rom)] * m, dtype=oracle.STATE_DTYPE)
            o_obs, _ = oracle.run_batch(rom, ref_st, np.ascontiguousarray(acts[:, :m]), k)
            # warm-up of both sides (module load, first-launch costs)
            time_ref(L, rom, min(n, 1024), acts[:, :min(n, 1024)], 1, 0, 0)
            time_ours(rom, min(n, 1024), acts[:, :min(n, 1024)], 1, 0)
            for form, multi in (("per_frame", 0), ("step_multi", 1)):
                row = {"cart": name, "instances": n, "frames": k, "form": form}
                for sorted_ in (0, 1):
                    ms, obs = time_ref(L, rom, n, acts, k, multi, sorted_)
                    tag = "ref_sorted" if sorted_ else "ref"
                    row[f"{tag}_frames_per_s"] = n * k / (ms / 1e3)
                    row[f"{tag}_matches_oracle"] = bool(np.array_equal(obs[:m], o_obs))
                ms, obs = time_ours(rom, n, acts, k, multi)
                row["ours_frames_per_s"] = n * k / (ms / 1e3)
                row["ours_matches_oracle"] = bool(np.array_equal(obs[:m], o_obs))
                row["speedup_vs_ref"] = row["ours_frames_per_s"] / max(row["ref_frames_per_s"], row["ref_sorted_frames_per_s"])
                out["rows"].append(row)
                print(json.dumps({k2: (round(v, 1) if isinstance(v, float) else v) for k2, v in row.items()}), flush=True)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
