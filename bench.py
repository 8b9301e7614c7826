"""Benchmark of the batched Atari 2600 core on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload mixed|divergence|plain|scale|serve|render|mappers|dpc|fe|micro]

Default workload (the batched configuration the headline metric is quoted
on): four seeded synthetic carts — 2K Fixed, 8K F8, 16K F6, 32K F4 with
WSYNC density 100/50/10/0% — at 100,000 / 30,000 / 5,000 / 500 instances,
K=4 frames per call, int8 actions uniform over 18 precomputed per frame.
One step = one batched call (K frames of every instance), launched as one
persistent kernel over all four carts.  Beside it the same trace runs through
the plain form (one launch per frame per cart) for the batched-vs-plain
ratio, and once more as one CUDA graph of all timed calls.

`value` is device time (CUDA events on the launching stream, L2 flushed
before every timed call); `e2e` is the same metric through the public C ABI
with host buffers: every call copies the actions from host memory and
returns the observations into the caller's host arrays (reused across calls)
inside the timed region.  Under torchrun every rank runs its own replica of the
workload on its GPU (instances are independent: weak scaling, no exchange).

Serving (`--workload serve`, and a short summary in the default line): 64
simulated actor clients send step requests by Poisson arrival to the
continuous-batching server; each request picks one of the four carts
uniformly, a batch size lognormal (median 256, sigma 1) clipped to
16..16,384 and K uniform in 1..8.  The peak is the sustained completion rate
of a saturation run (every request queued at once, first arrival to last
completion); at 20/40/70/100% of it each level reports achieved / offered
(the completion rate in the middle 80% of the arrival window) and the growth of the
median latency from the first to the last third of the arrivals (kept up:
at least 0.95 and under 1.5), p50/p99 step latency and its parts (waiting for
the same session's earlier requests, dispatch, service), per (cart, K) at
70%, beside the idle-GPU floor of one request per (cart, K); the plain
per-frame server runs the same trace.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "fast-atari-rs_b200"

METRIC = "frames/s bit-exact: batched/served vs plain kernel, 1 B200; p99 step latency"
UNIT = "frames/s"

# SASS thread-instructions per emulated 6502 instruction when all 32 lanes of
# a warp run identical instances (fully converged), from the ncu capture in
# profiles/fa_run_warps_converged_plain.md.  Used to express guest-instruction
# throughput in warp-issue slots for the roofline.
I_CONV = 165.5
# DRAM bytes moved per instance-frame by fa_run on this workload, from the ncu
# capture in profiles/fa_run_warps_mixed_batch_full.md (29.6 MB per 4-frame
# call of 135,500 instances).
DRAM_BYTES_PER_INSTANCE_FRAME = 54.6
# The rendering kernel (fa_render_run) per rendered console-frame, from
# the ncu capture in profiles/fa_render_run_render_cart.md: SASS
# thread-instructions and DRAM bytes (framebuffer writes included).
RENDER_THREAD_INST_PER_FRAME = 2.936e6   # smsp__thread_inst_executed / console-frames
RENDER_DRAM_BYTES_PER_FRAME = 61_600     # (dram read + write) / console-frames


def load_pkg():
    if "fast_atari_b200" in sys.modules:
        return sys.modules["fast_atari_b200"]
    spec = importlib.util.spec_from_file_location(
        "fast_atari_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["fast_atari_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------ workloads
def workload(name: str, carts):
    """(description, [(cart, n)], k, episode_frames)."""
    if name == "mixed":
        cs = carts.mixed_carts()
        return ("mixed 4-cart batch: 2K Fixed/8K F8/16K F6/32K F4, WSYNC 100/50/10/0%, "
                "100000/30000/5000/500 instances, K=4 frames per call",
                list(zip(cs, carts.MIXED_COUNTS)), 4, 0)
    if name == "divergence":
        return ("divergence-heavy 8K F8 cart, 50000 instances, per-frame step (K=1)",
                [(carts.divergence_cart(), 50_000)], 1, 0)
    if name == "plain":
        return ("plain 4K Fixed cart, 1000 instances, per-frame step (K=1)",
                [(carts.plain_cart(), 1000)], 1, 0)
    if name == "converged":
        # Calibration: identical instances and actions, so every warp runs
        # fully converged (the instruction cost per guest instruction).
        return ("converged calibration: plain 4K Fixed cart, 151552 identical instances, "
                "all actions 0, K=2", [(carts.plain_cart(), 151_552)], 2, 0)
    if name == "serve":
        # The serving trace's cart mix (uniform over the four carts per
        # request; mean batch 422 instances, mean K 4.5) for the CPU baseline.
        cs = carts.mixed_carts()
        return (SERVE_DESC, [(c, 422) for c in cs], 4, 0)
    if name == "scale":
        return ("scale: 1000000 instances of the 32K F4 cart, K=16, reset every 2000 frames",
                [(carts.scale_cart(), 1_000_000)], 16, 2000)
    if name == "mappers":
        # Schemes the reference lacks, registered per ROM (fa_rom_set_scheme).
        return ("sliced-bank carts: 8K E0 / 16K 3F / 6K 3F, 40000/40000/20000 instances, K=4 frames per call",
                [(carts.e0_cart(), 40_000), (carts.f3_cart(16384), 40_000), (carts.f3_cart(6144), 20_000)], 4, 0)
    if name == "dpc":
        # Pitfall II's scheme, picked by ROM length (10,240 and 10,495 bytes).
        return ("DPC carts (fetchers, random numbers, music channels): 10240- and 10495-byte images, "
                "40000/40000 instances, K=4 frames per call",
                [(carts.dpc_cart(), 40_000), (carts.dpc_cart(dump_tail=True), 40_000)], 4, 0)
    if name == "fe":
        # Activision FE, registered per ROM (fa_rom_set_scheme).
        return ("FE cart (bank chosen by the access after one to $01FE): 8K, 80000 instances, K=4 frames per call",
                [(carts.fe_cart(), 80_000)], 4, 0)
    raise SystemExit(f"unknown workload {name}")


SERVE_DESC = ("serving: 64 Poisson actor clients, carts 2K Fixed/8K F8/16K F6/32K F4 uniform per request, "
              "batch lognormal(median 256, sigma 1) clipped 16..16384, K uniform 1..8, "
              "states resident in HBM, 64 GiB state budget")


def _pcts(v):
    v = np.sort(np.asarray(v, dtype=np.float64))
    if v.size == 0:
        return {"p50": None, "p99": None}
    q = lambda f: float(v[min(v.size - 1, int(round(f * (v.size - 1))))])
    return {"p50": round(q(0.5), 3), "p99": round(q(0.99), 3)}


def serve_breakdown(rec, by_shape=False):
    """p50/p99 of the latency and of its parts (waiting for the same
    session's earlier requests, dispatch, service), and per (cart, K)."""
    out = {part: _pcts(rec[part]) for part in ("latency_ms", "session_wait_ms", "dispatch_ms", "service_ms")}
    if by_shape:
        shapes = {}
        for c in np.unique(rec["cart"]):
            for k in np.unique(rec["k"]):
                sel = rec[(rec["cart"] == c) & (rec["k"] == k)]
                if sel.size:
                    shapes[f"cart{int(c)}/K{int(k)}"] = {"requests": int(sel.size),
                                                         "latency_ms": _pcts(sel["latency_ms"]),
                                                         "service_ms": _pcts(sel["service_ms"])}
        out["by_cart_k"] = shapes
    return out


def serve_floor(fa, roms, n=256, reps=3):
    """The idle-GPU floor: one request at a time on an otherwise idle
    server, per (cart, K), n = the trace's median batch; the fastest of
    `reps` (latency and service ms)."""
    floor = {}
    with fa.AtariServer(roms) as srv:
        for c in range(len(roms)):
            sid = srv.open(c)
            srv.step(sid, np.zeros(n, np.uint8), n, 1)                 # admission, first launch
            for k in range(1, 9):
                best = None
                for r in range(reps):
                    _, info = srv.step(sid, np.zeros(n * k, np.uint8), n, k)
                    if best is None or info["latency_ms"] < best["latency_ms"]:
                        best = info
                floor[f"cart{c}/K{k}"] = {"latency_ms": round(best["latency_ms"], 3),
                                          "service_ms": round(best["service_ms"], 3)}
            srv.close_session(sid)
    return floor


def serve_measure(fa, carts, sat_requests, level_requests, plain_requests, levels=(0.2, 0.4, 0.7, 1.0)):
    """Batched server: its sustained peak (the whole saturation run: every
    request queued at once, first arrival to last completion), then Poisson
    load at fractions of that peak with achieved / offered and the latency
    breakdown; the idle-GPU floor per (cart, K); the plain server's peak on
    the same trace."""
    roms = [c.rom for c in carts.mixed_carts()]
    out = {"clients": 64, "levels": []}
    with fa.AtariServer(roms) as srv:
        srv.loadgen(requests=400, offered_frames_per_s=0.0, seed=99)              # warm-up
        st0 = srv.stats()
        sat, sat_rec = srv.loadgen(requests=sat_requests, offered_frames_per_s=0.0, seed=1)
        st1 = srv.stats()
        peak = sat["frames_per_s"]
        out["saturation"] = sat
        out["saturation_breakdown"] = serve_breakdown(sat_rec)
        out["guest_instructions_per_s"] = (st1["guest_instructions"] - st0["guest_instructions"]) / sat["elapsed_s"]
        out["lane_efficiency"] = ((st1["guest_instructions"] - st0["guest_instructions"]) /
                                  max(1, st1["lane_slots"] - st0["lane_slots"]))
        out["launches"] = st1["launches"] - st0["launches"]
        for frac in levels:
            r, rec = srv.loadgen(requests=level_requests, offered_frames_per_s=frac * peak, seed=2)
            # Achieved rate: the instance-frames of the requests that complete
            # inside the middle 80% of the arrival window, over that span (the
            # start and the drain after the last arrival left out).  A server
            # that keeps up also shows no growth of latency over the run.
            order = np.argsort(rec["arrival_s"])
            third = max(1, len(order) // 3)
            growth = (np.median(rec["latency_ms"][order[-third:]]) /
                      max(1e-9, np.median(rec["latency_ms"][order[:third]])))
            w = r["arrival_window_s"]
            done_at = rec["arrival_s"] + rec["latency_ms"] * 1e-3
            mid = (done_at >= 0.1 * w) & (done_at <= 0.9 * w)
            frames_mid = float((rec["n"][mid].astype(np.float64) * rec["k"][mid]).sum())
            achieved = (frames_mid / max(1e-9, 0.8 * w)) / r["offered_frames_per_s"]
            out["levels"].append({"load": frac, "offered_frames_per_s": r["offered_frames_per_s"],
                                  "frames_per_s": r["frames_per_s"], "achieved_over_offered": achieved,
                                  "latency_growth": float(growth),
                                  "drain_ms": (r["elapsed_s"] - r["arrival_window_s"]) * 1e3,
                                  "kept_up": bool(achieved >= 0.95 and growth < 1.5),
                                  "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "max_ms": r["max_ms"],
                                  "mean_queue_ms": r["mean_queue_ms"], "mean_batch_requests": r["mean_batch_requests"],
                                  "requests": r["requests"],
                                  "breakdown": serve_breakdown(rec, by_shape=(frac == 0.7))})
    out["floor"] = serve_floor(fa, roms)
    with fa.AtariServer(roms, mode="plain") as srv:
        srv.loadgen(requests=200, offered_frames_per_s=0.0, seed=99)
        psat, _ = srv.loadgen(requests=plain_requests, offered_frames_per_s=0.0, seed=1)
    out["plain_saturation"] = psat
    out["peak_frames_per_s"] = peak
    out["plain_peak_frames_per_s"] = psat["frames_per_s"]
    return out


def serve_summary(sv):
    lv = {l["load"]: l for l in sv["levels"]}
    at70 = lv.get(0.7, sv["levels"][-1])
    return {"workload": SERVE_DESC,
            "peak": "sustained completion rate of the saturation run (every request queued at once, "
                    "first arrival to last completion)",
            "peak_frames_per_s": sv["peak_frames_per_s"],
            "plain_peak_frames_per_s": sv["plain_peak_frames_per_s"],
            "served_vs_plain": sv["peak_frames_per_s"] / sv["plain_peak_frames_per_s"],
            "p50_ms_at_70pct": at70["p50_ms"], "p99_ms_at_70pct": at70["p99_ms"],
            "achieved_over_offered_at_70pct": at70["achieved_over_offered"],
            "kept_up_at_70pct": at70["kept_up"],
            "floor_ms": sv["floor"],
            "levels": [{k: round(v, 3) if isinstance(v, float) else v for k, v in l.items()} for l in sv["levels"]]}


def divergence_policies(fa, carts, n=50_000, frames=32, k_multi=16):
    """The divergence cart under every warp policy (opcode grouping on/off),
    per-frame launches (K=1, one launch per frame) vs step_multi (K=16 per
    persistent launch): frames/s by CUDA events on the launching stream, and
    the SIMT lane efficiency of each policy."""
    import torch
    rom = carts.divergence_cart().rom
    dev = torch.device("cuda", torch.cuda.current_device())
    acts = torch.from_numpy(np.ascontiguousarray(carts.actions(seed=5, n=n, frames=frames)).reshape(-1)).to(dev)
    stream = torch.cuda.Stream()          # a real stream: the library launches on it, the events see it
    out = {}
    for sched in ("lane", "match", "pc", "line"):
        for form, persistent, k in (("per_frame", False, 1), ("step_multi", True, k_multi)):
            with fa.BatchAtariGpu(rom, n) as g:
                g.set_launch(128, sched, persistent)
                g.reset()
                g.step_multi_async(acts.data_ptr(), k, 0, stream.cuda_stream)      # warm-up
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for c in range(frames // k):
                    g.step_multi_async(acts.data_ptr() + c * k * n, k, 0, stream.cuda_stream)
                e1.record(stream)
                torch.cuda.synchronize()
                fps = n * (frames // k) * k / (e0.elapsed_time(e1) / 1e3)
                g.step_multi(carts.actions(seed=6, n=n, frames=k), k, obs=False)
                eff = g.last_instructions() / max(1, g.last_lane_slots())
            out[f"{sched}/{form}"] = {"frames_per_s": fps, "lane_efficiency": eff}
    return out


# ------------------------------------------------------------------ the reference's own kernel
REF_CUDA_LIB = ROOT / "oracle" / "_ref" / "libref_cuda.so"


def ref_kernel_compare(fa, carts, n=50_000, frames=16):
    """The kernel the reference ships (atari_frame_kernel and
    atari_multi_frame_kernel of cuda/src/atari_kernel.cu, built for sm_100a
    from the reference's sources into oracle/_ref/ by `make -C oracle ref`,
    launched as its host binding does: grid ceil(n/128), block 128) against
    this library on the plain 4K Fixed cart, the one cart on which the two
    agree with the oracle.  Both start from this library's post-reset states
    (the first 221 bytes of fa_state are the reference's AtariState) with the
    same actions; each side is timed by CUDA events around its launches only.
    Per-frame form (one launch per frame, BatchAtariGpu::step) and
    step_multi form (all frames in one launch).  None where the reference's
    kernels were not built."""
    import ctypes
    if not REF_CUDA_LIB.exists():
        return None
    import torch
    L = ctypes.CDLL(str(REF_CUDA_LIB))
    L.ref_state_size.restype = ctypes.c_int
    L.ref_run.restype = ctypes.c_int
    L.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
    rom = carts.plain_cart().rom
    acts = np.ascontiguousarray(carts.actions(seed=9, n=n, frames=frames))
    size = L.ref_state_size()
    with fa.BatchAtariGpu(rom, n) as g:
        g.reset()
        snap = g.download_states().view(np.uint8).reshape(n, -1)[:, :221]
    ref_st = np.zeros((n, size), np.uint8)
    ref_st[:, :221] = snap
    r = np.frombuffer(rom, np.uint8).copy()

    def ref_ms(multi, nn, a):
        st = ref_st[:nn].copy()                                      # ref_run writes the states back
        obs = np.empty((nn, 128), np.uint8)
        ms = ctypes.c_float()
        rc = L.ref_run(r.ctypes.data, len(r), st.ctypes.data, nn, np.ascontiguousarray(a).ctypes.data,
                       a.shape[0], multi, 0, obs.ctypes.data, ctypes.byref(ms))
        if rc:
            raise RuntimeError(f"reference kernel launch failed: cudaError {rc}")
        return ms.value, obs

    d_acts = torch.from_numpy(acts.reshape(-1)).cuda()
    stream = torch.cuda.Stream()
    d_obs = torch.empty(n * 128, dtype=torch.uint8, device="cuda")

    def ours_ms(multi):
        with fa.BatchAtariGpu(rom, n) as g:
            g.set_launch(128, "pc", bool(multi))
            g.reset()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if multi:
                g.step_multi_async(d_acts.data_ptr(), frames, d_obs.data_ptr(), stream.cuda_stream)
            else:
                for f in range(frames):
                    g.step_multi_async(d_acts.data_ptr() + f * n, 1, d_obs.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), d_obs.cpu().numpy().reshape(n, 128)

    ref_ms(0, min(n, 1024), acts[:1, :min(n, 1024)])                   # module load, first launch
    out = {"cart": "plain_4k_fixed", "instances": n, "frames": frames,
           "reference": "cuda/src/atari_kernel.cu built for sm_100a (the kernels the reference ships)"}
    for form, multi in (("per_frame", 0), ("step_multi", 1)):
        ms_ref, obs_ref = ref_ms(multi, n, acts)
        ms_our, obs_our = ours_ms(multi)
        out[form] = {"reference_frames_per_s": n * frames / (ms_ref / 1e3),
                     "ours_frames_per_s": n * frames / (ms_our / 1e3),
                     "speedup": ms_ref / ms_our,
                     "instances_with_different_ram": int((obs_ref != obs_our).any(axis=1).sum())}
    return out


def run_micro_arm(args, fa, carts, rank, world, local_rank):
    """Instruction-cost micro-carts (carts.micro_cart): one instruction kind
    per visible line, 151,552 identical instances with all actions 0 (fully
    converged), K=2, three calls timed with CUDA events on the launching
    stream.  The cost of one guest instruction of each kind is given in
    warp-issue slots at 100 % issue: 148 SMs x 4 schedulers x the sampled
    clock / (guest instructions/s / 32).  The guest instruction count is the
    kernel's own."""
    import torch
    fa.set_device(local_rank)
    torch.cuda.set_device(local_rank)
    n, k, calls = 151_552, 2, 3
    s = torch.cuda.Stream()
    acts = torch.zeros(k * n, dtype=torch.uint8, device="cuda")
    kinds = {}
    with ClockSampler(local_rank) as clk:
        for kind in carts.MICRO_KINDS:
            with fa.BatchAtariGpu(carts.micro_cart(kind).rom, n) as g:
                g.set_launch(args.block, "pc", True)
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
                g.step_multi_async(acts.data_ptr(), k, 0, s.cuda_stream)
                g.synchronize()
                instr = g.last_instructions()
            kinds[kind] = {"frames_per_s": n * k * calls / (ms / 1e3), "guest_instr_per_frame": instr / (n * k),
                           "guest_instr_per_s": instr * calls / (ms / 1e3)}
    clocks = clk.summary()
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    for v in kinds.values():
        v["issue_slots_per_guest_instr_at_100pct"] = 148 * 4 * f_sm / (v["guest_instr_per_s"] / 32.0)
    nop = kinds["nop"]
    line = {"metric": METRIC, "value": nop["frames_per_s"], "unit": UNIT, "n_gpus": world, "steps": calls,
            "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"instruction-cost micro-carts, {n} identical instances, K={k}; value = the NOP cart",
                       "l2": "state (34 MB) resident; not flushed", "parallelism": "single GPU"},
            "clocks": clocks, "gpu_launches": calls * len(kinds),
            "micro": {kk: {k2: round(v2, 2) for k2, v2 in v.items()} for kk, v in kinds.items()}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def unit_trace_summary(tr, names, bins=20):
    """Per-unit records of one batched call (fa_pool_set_trace): per cart the
    latest start and the median and last finish (ms from the call's first
    start), and the warps still running and SMs busy at `bins` points."""
    tr = tr[tr[:, 1] > 0]
    if tr.size == 0:
        return None
    t0 = tr[:, 0].min()
    start = (tr[:, 0] - t0).astype(np.float64) / 1e6
    end = (tr[:, 1] - t0).astype(np.float64) / 1e6
    tag = (tr[:, 2] & np.uint64(0xFFFF)).astype(int)
    sm = (tr[:, 2] >> np.uint64(32)).astype(int)
    out = {"call_ms": round(float(end.max()), 3), "carts": {}}
    for g, name in enumerate(names):
        m = tag == g
        if m.any():
            out["carts"][name] = {"units": int(m.sum()), "start_max_ms": round(float(start[m].max()), 3),
                                  "end_p50_ms": round(float(np.median(end[m])), 3),
                                  "end_max_ms": round(float(end[m].max()), 3)}
    pts = np.linspace(0.0, float(end.max()), bins + 1)[:-1]
    out["warps_running"] = [int(((start <= t) & (end > t)).sum()) for t in pts]
    out["sms_busy"] = [int(np.unique(sm[(start <= t) & (end > t)]).size) for t in pts]
    return out


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3] not in ("", "[N/A]"))}


# ------------------------------------------------------------------ ranks
def dist_backend() -> str:
    """NCCL between GPUs; gloo where no GPU is visible (the CPU tests of the
    multi-rank path)."""
    import torch
    return "nccl" if torch.cuda.is_available() else "gloo"


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest of every rank's x (times: the job ends with its slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank: int, group: int) -> int:
    """Action seed of cart group `group` on rank `rank`: every rank steps its own
    replica of the workload (instances are independent; no exchange)."""
    return 1000 * rank + 17 * group + 1


# ------------------------------------------------------------------ CPU reference
def cpu_reference(carts, spec, k, seconds_target=15.0):
    """The oracle (a C restatement of the reference's HeadlessAtari) on the
    host cores.  Each cart is timed on its own, with every host thread busy
    (4 instances per thread, k-frame calls, an equal share of the time), and
    the workload's rate combines the per-cart rates with the workload's true
    instance counts: total instance-frames / sum over carts of (that cart's
    instance-frames / its rate).  Returns (frames/s, threads, sample text,
    per-cart frames/s)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    for c, _ in spec:
        if c.scheme:
            oracle.set_rom_scheme(c.rom, c.scheme)
    m = 4 * cores
    share = seconds_target / len(spec)
    rates, parts = {}, []
    for c, _ in spec:
        st = np.array([oracle.reset_state(c.rom)] * m, dtype=oracle.STATE_DTYPE)
        frames, call = 0, 0
        t0 = time.perf_counter()
        while True:
            acts = carts.actions(seed=7, n=m, frames=k, frame0=call * k)
            oracle.run_batch(c.rom, st, acts, k, nthreads=cores, pin=False)
            frames += m * k
            call += 1
            if time.perf_counter() - t0 >= share:
                break
        dt = time.perf_counter() - t0
        rates[c.spec.name] = frames / dt
        parts.append(f"{c.spec.name}: {frames} instance-frames in {dt:.1f} s")
    total = sum(n for _, n in spec)
    value = total / sum(n / rates[c.spec.name] for c, n in spec)
    weights = ", ".join(f"{n} x {c.spec.name}" for c, n in spec)
    sample = (f"each cart alone on {cores} threads ({m} instances, K={k} calls): " + "; ".join(parts) +
              f"; combined with the workload's instance counts [{weights}]")
    return value, cores, sample, rates


def run_reference_arm(args, carts, rank, world):
    if rank != 0:
        return
    if args.workload == "render":
        per_step_s = args.ref_step_seconds or max(0.2, min(10.0, 120.0 / max(1, args.steps + args.warmup)))
        vals = []
        for i in range(args.warmup + args.steps):
            fps, cores, sample = render_cpu_baseline(carts, per_step_s)
            if i >= args.warmup:
                vals.append(fps)
        value = statistics.mean(vals)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
                          "config": {"workload": RENDER_DESC, "parallelism": "one console per host thread"},
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                                           "sample": sample + "; C restatement of the reference's rendering Atari + Tia"},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    desc, spec, k, _ = workload(args.workload, carts)
    # Each step is one bounded CPU sample; warmup steps are run untimed.
    # Each step is a bounded sample sized so the whole run takes about two minutes.
    per_step_s = args.ref_step_seconds or max(0.2, min(10.0, 120.0 / max(1, args.steps + args.warmup)))
    vals, per_cart = [], {}
    for i in range(args.warmup + args.steps):
        fps, cores, sample, rates = cpu_reference(carts, spec, k, seconds_target=per_step_s)
        if i >= args.warmup:
            vals.append(fps)
            for name, r in rates.items():
                per_cart.setdefault(name, []).append(r)
    value = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": desc, "parallelism": "one emulator per host thread"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; C restatement of the reference HeadlessAtari",
                             "per_cart_frames_per_s": {n2: statistics.mean(v) for n2, v in per_cart.items()}},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def run_gpu_arm(args, fa, carts, rank, world, local_rank):
    import torch
    desc, spec, k, episode = workload(args.workload, carts)
    fa.set_device(local_rank)
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    for c, _ in spec:
        if c.scheme:
            fa.set_rom_scheme(c.rom, c.scheme)
    pool = fa.AtariPool()
    groups = []
    for c, n in spec:
        g = pool.add_cart(c.rom, n)
        groups.append(g)
    if episode:
        # Periodic reset to the post-init snapshot with per-instance phase
        # offsets uniform in [0, episode).
        rng = np.random.default_rng(1234 + rank)
        for g, (c, n) in zip(groups, spec):
            view = pool.group(g)
            view.set_episode_frames(episode)
            view.set_frame_numbers(rng.integers(0, episode, n, dtype=np.uint32))
    tuning = args.tuning
    if not tuning and not args.no_autotune and args.workload != "converged":
        # The project autotuner, per cart at up to 8,192 instances: it times
        # every warp policy, launch shape and K; the batched launch takes each
        # cart's policy and its measured cost per instance-frame (the queue
        # order, heaviest units first).  K stays the workload's.
        sys.path.insert(0, str(PKG_DIR))
        import tune
        tuning = tune.tune_workload([(c, n) for c, n in spec], cap=8192)
    args.tuning_used = tuning
    for g, (c, n) in zip(groups, spec):
        t = tuning.get(c.spec.name, {})
        pool.set_group(g, t.get("sched", "pc"), float(t.get("weight", 1.0 + c.spec.rom_size / 32768.0)))
    pool.set_launch(args.block, True)

    calls = args.warmup + args.steps
    # Device-resident actions for every call: per cart [calls, k, n] uint8.
    d_act = []
    for gi, (c, n) in enumerate(spec):
        t = torch.empty(calls * k * n, dtype=torch.uint8, device=dev)
        chunk = max(1, (64 << 20) // max(1, k * n))
        if args.workload == "converged":
            t.zero_()
            d_act.append(t)
            continue
        for c0 in range(0, calls, chunk):
            c1 = min(calls, c0 + chunk)
            a = carts.actions(seed=replica_seed(rank, gi), n=n, frames=(c1 - c0) * k, frame0=c0 * k)
            t[c0 * k * n:c1 * k * n].copy_(torch.from_numpy(a.reshape(-1)))
        d_act.append(t)
    d_obs = [torch.empty(n * 128, dtype=torch.uint8, device=dev) for _, n in spec]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)       # > 126 MB L2
    stream = torch.cuda.ExternalStream(pool.stream(), device=dev)
    sptr = pool.stream()
    torch.cuda.synchronize()

    def acts_at(call):
        return [d_act[gi].data_ptr() + call * k * n for gi, (_, n) in enumerate(spec)]

    obs_ptrs = [o.data_ptr() for o in d_obs]

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def timed_calls(step_fn, first_call, ncalls):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ncalls)]
        with torch.cuda.stream(stream):
            for i in range(ncalls):
                flush.zero_()
                evs[i][0].record(stream)
                step_fn(acts_at(first_call + i), k, obs_ptrs, sptr)
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    # ---- warmup (batched and plain forms)
    for i in range(args.warmup):
        pool.step_async(acts_at(i), k, obs_ptrs, sptr)
    pool.synchronize()
    # ---- timed: batched persistent form
    barrier()
    pool.reset_counters()
    with ClockSampler(local_rank) as clk:
        ms = timed_calls(pool.step_async, args.warmup, args.steps)
    pool.synchronize()
    instr = pool.last_instructions()
    slots = pool.last_lane_slots()
    clocks = clk.summary()
    total_ms = sum(ms)
    total_ms = max_over_ranks(total_ms, world, dev)
    n_total = sum(n for _, n in spec)
    frames = n_total * k * args.steps * world
    value = frames / (total_ms / 1e3)

    # ---- one more batched call with per-unit records: when each cart's
    # warps finish, and how many warps run as the call drains
    unit_trace = None
    if world == 1:
        nu = sum((n + 31) // 32 for _, n in spec)
        d_tr = torch.zeros(nu * 3, dtype=torch.int64, device=dev)
        pool.set_trace(d_tr.data_ptr(), nu)
        pool.step_async(acts_at(args.warmup), k, obs_ptrs, sptr)
        pool.synchronize()
        pool.set_trace()
        unit_trace = unit_trace_summary(d_tr.cpu().numpy().view(np.uint64).reshape(nu, 3),
                                        [c.spec.name for c, _ in spec])

    # ---- the plain kernel on the same trace (one launch per frame per cart)
    plain_value = None
    if not args.no_plain:
        plain_steps = max(3, min(args.steps, 20))
        pool.step_plain_async(acts_at(0), k, obs_ptrs, sptr)
        pool.synchronize()
        barrier()
        ms_plain = timed_calls(pool.step_plain_async, args.warmup, min(plain_steps, args.steps))
        plain_value = n_total * k * len(ms_plain) / (sum(ms_plain) / 1e3)

    # ---- the whole timed trace as one CUDA graph (no flushes between calls)
    graph_value = None
    if not args.no_graph:
        graph = pool.graph([d.data_ptr() + args.warmup * k * n for d, (_, n) in zip(d_act, spec)], k,
                           args.steps, obs_ptrs)
        graph.launch()
        pool.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        torch.cuda.synchronize()
        e0.record(stream)
        graph.launch(sptr)
        e1.record(stream)
        torch.cuda.synchronize()
        graph_value = n_total * k * args.steps / (e0.elapsed_time(e1) / 1e3)
        graph.close()

    # ---- end to end through the public API with host buffers
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 30))
    host_acts = [[np.ascontiguousarray(d_act[gi][(args.warmup + i) * k * n:(args.warmup + i + 1) * k * n].cpu().numpy())
                  for gi, (_, n) in enumerate(spec)] for i in range(e2e_steps)]
    e2e_value = None
    if e2e_steps:
        host_obs = [np.empty((n, 128), np.uint8) for _, n in spec]      # the caller's buffers, reused
        pool.step(host_acts[0], k, out=host_obs)
        barrier()
        t0 = time.perf_counter()
        for i in range(e2e_steps):
            pool.step(host_acts[i], k, out=host_obs)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
        e2e_value = n_total * k * e2e_steps * world / e2e_s
    h2d = n_total * k
    d2h = n_total * 128

    # ---- roofline: guest instructions in warp-issue slots vs SM issue peak
    guest_per_s = instr / (total_ms / 1e3)
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    peak = 148 * 4 * f_sm                        # warp-instructions per second
    achieved = guest_per_s * I_CONV / 32.0
    traffic = None
    if DRAM_BYTES_PER_INSTANCE_FRAME is not None:
        traffic = DRAM_BYTES_PER_INSTANCE_FRAME * n_total * k

    lat = sorted(ms)
    p = lambda q: lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": desc, "instances": n_total, "frames_per_call": k,
                   "launch": f"one persistent kernel per call, block {args.block}",
                   "l2": "flushed (256 MB write) before every timed call",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "tuning": {name: {k2: (round(v, 3) if isinstance(v, float) else v) for k2, v in t.items()
                          if k2 in ("sched_name", "weight", "k", "persistent", "cta_warps", "block", "frames_per_s",
                                    "instances", "alternatives", "applied_in_pool")}
                   for name, t in (args.tuning_used or {}).items()} or None,
        "gpu_launches": args.steps,
        "roofline": {"bound": "issue", "achieved": achieved / 1e12, "peak": peak / 1e12,
                     "unit": "T warp-inst/s", "frac": achieved / peak, "traffic": traffic,
                     "note": f"guest 6502 instr/s x {I_CONV} SASS thread-instr per guest instr (converged) / 32"},
        "plain_kernel": {"value": plain_value, "unit": UNIT,
                         "form": "one launch per frame per cart"} if plain_value else None,
        "batched_vs_plain": value / plain_value if plain_value else None,
        "graph": {"value": graph_value, "unit": UNIT, "calls": args.steps} if graph_value else None,
        "step_latency_ms": {"p50": p(0.5), "p99": p(0.99), "max": lat[-1]},
        "guest_instructions_per_s": guest_per_s,
        "guest_instructions_per_step": instr / args.steps,
        "lane_efficiency": instr / slots if slots else None,
        "unit_trace": unit_trace,
    }
    if world == 1 and args.workload == "divergence":
        line["policies"] = divergence_policies(fa, carts)
    if world == 1 and args.workload == "mixed" and not args.no_serve:
        line["serving"] = serve_summary(serve_measure(fa, carts, 8000, 3000, 2000, levels=(0.7,)))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fps, cores, sample, rates = cpu_reference(carts, spec, k, seconds_target=args.cpu_seconds)
        line["cpu_baseline"] = {"value": fps, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": sample + "; C restatement of the reference HeadlessAtari",
                                "per_cart_frames_per_s": rates}
    if rank == 0 and world == 1 and args.workload == "mixed" and not args.no_ref_kernel:
        line["ref_kernel"] = ref_kernel_compare(fa, carts)
    if rank == 0:
        print(json.dumps(line), flush=True)
    pool.close()


RENDER_DESC = ("rendering console (pixel-accurate TIA, 160x192 palette-index framebuffer per console): "
               "render_4k_fixed cart, 75776 consoles (one wave: 148 SMs x 16 warps x 32), K=4 frames per call")
RENDER_N, RENDER_K = 75_776, 4


def render_cpu_baseline(carts, seconds_target):
    """The rendering oracle (C restatement of the reference's Atari + Tia) on
    every host thread: a bounded sample of consoles, frames/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    rom = carts.render_cart().rom
    m = 4 * cores
    consoles = oracle.render_reset(rom, m)
    frames, call = 0, 0
    t0 = time.perf_counter()
    while True:
        oracle.render_steps(consoles, carts.actions(seed=11, n=m, frames=RENDER_K, frame0=call * RENDER_K),
                            nthreads=cores, outputs=False)
        frames += m * RENDER_K
        call += 1
        if time.perf_counter() - t0 >= seconds_target:
            break
    dt = time.perf_counter() - t0
    return frames / dt, cores, f"{call} calls of K={RENDER_K} frames over {m} consoles ({frames} frames, {dt:.1f} s)"


def run_render_arm(args, fa, carts, rank, world, local_rank):
    """The rendering console: frames/s with framebuffers (its own JSON line)."""
    import torch
    fa.set_device(local_rank)
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, k = args.render_instances, RENDER_K
    steps = max(1, min(args.steps, 20))
    calls = args.warmup + steps
    rom = carts.render_cart().rom
    g = fa.AtariRender(rom, n, cta_warps=args.render_cta_warps)
    g.reset()
    acts = torch.empty(calls * k * n, dtype=torch.uint8, device=dev)
    for c in range(calls):
        a = carts.actions(seed=replica_seed(rank, 0), n=n, frames=k, frame0=c * k)
        acts[c * k * n:(c + 1) * k * n].copy_(torch.from_numpy(a.reshape(-1)))
    d_obs = torch.empty(n * 128, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    for c in range(args.warmup):
        g.step_multi_async(acts.data_ptr() + c * k * n, k, d_obs.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for i in range(steps):
                flush.zero_()
                evs[i][0].record(stream)
                g.step_multi_async(acts.data_ptr() + (args.warmup + i) * k * n, k, d_obs.data_ptr(), stream.cuda_stream)
                evs[i][1].record(stream)
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(ms), world, dev)
    value = n * k * steps * world / (total_ms / 1e3)
    g.synchronize()
    # End to end through the C ABI: host actions in, every framebuffer and the RAM out.
    host_acts = [acts[(args.warmup + i) * k * n:(args.warmup + i + 1) * k * n].cpu().numpy() for i in range(min(steps, 3))]
    host_out = (np.empty((n, 192, 160), np.uint8), np.empty((n, 128), np.uint8))    # the caller's, reused
    g.step_multi(host_acts[0], k, out=host_out)
    t0 = time.perf_counter()
    for a in host_acts:
        g.step_multi(a, k, out=host_out)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e = n * k * len(host_acts) * world / e2e_s
    g.step_multi(host_acts[0], k, fb=False)
    instr_per_frame = g.last_instructions() / (n * k)
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    peak = 148 * 4 * f_sm
    achieved = value * RENDER_THREAD_INST_PER_FRAME / 32.0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": total_ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic",
        "config": {"workload": RENDER_DESC.replace("75776 consoles (one wave: 148 SMs x 16 warps x 32)", f"{n} consoles"),
                   "instances": n, "frames_per_call": k,
                   "framebuffer_bytes_per_frame": 160 * 192,
                   "l2": "flushed (256 MB write) before every timed call",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clocks,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": n * k, "d2h_bytes_per_step": n * (160 * 192 + 128)},
        "gpu_launches": steps,
        "roofline": {"bound": "issue", "achieved": achieved / 1e12, "peak": peak / 1e12,
                     "unit": "T warp-inst/s", "frac": achieved / peak,
                     "traffic": RENDER_DRAM_BYTES_PER_FRAME * n * k,
                     "note": f"frames/s x {RENDER_THREAD_INST_PER_FRAME:.4g} SASS thread-instr per rendered frame (ncu) / 32"},
        "guest_instructions_per_frame": instr_per_frame,
        "step_latency_ms": {"p50": sorted(ms)[len(ms) // 2], "max": max(ms)},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fps, cores, sample = render_cpu_baseline(carts, min(args.cpu_seconds, 15.0))
        line["cpu_baseline"] = {"value": fps, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": sample + "; C restatement of the reference's rendering Atari + Tia"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()


def run_serve_arm(args, fa, carts, rank, world, local_rank):
    """The serving workload: its own JSON line (replicas under torchrun)."""
    fa.set_device(local_rank)
    n_sat = args.serve_requests
    with ClockSampler(local_rank) as clk:
        sv = serve_measure(fa, carts, n_sat, max(1000, n_sat // 6), max(1000, n_sat // 4))
    clocks = clk.summary()
    sat = sv["saturation"]
    value = sv["peak_frames_per_s"]
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([value], device=torch.device("cuda", local_rank), dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        value = float(t.item()) * world        # replicas: the slowest rank's rate on every GPU
    f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
    peak_issue = 148 * 4 * f_sm
    achieved = sv["guest_instructions_per_s"] * I_CONV / 32.0
    mean_req_frames = sat["instance_frames"] / sat["requests"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": int(sat["requests"]),
        "warmup": 400, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": SERVE_DESC, "step": "one step request (n instances x K frames)",
                   "requests": int(sat["requests"]), "mean_instance_frames_per_request": mean_req_frames,
                   "l2": "inputs resident in HBM between requests; not flushed",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "clocks": clocks,
        "e2e": {"value": sat["frames_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": mean_req_frames, "d2h_bytes_per_step": 128.0 * sat["instances"] / sat["requests"],
                "note": "whole saturation run (first arrival to last completion), actions from and observations to host memory"},
        "gpu_launches": sv["launches"],
        "roofline": {"bound": "issue", "achieved": achieved / 1e12, "peak": peak_issue / 1e12,
                     "unit": "T warp-inst/s", "frac": achieved / peak_issue, "traffic": None,
                     "note": f"guest 6502 instr/s x {I_CONV} SASS thread-instr per guest instr (converged) / 32"},
        "plain_kernel": {"value": sv["plain_peak_frames_per_s"], "unit": UNIT,
                         "form": "FIFO of static batches, one launch per frame per cart"},
        "batched_vs_plain": value / world / sv["plain_peak_frames_per_s"] if world == 1 else None,
        "serving": serve_summary(sv),
        "lane_efficiency": sv["lane_efficiency"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed",
                    choices=["mixed", "divergence", "plain", "scale", "converged", "serve", "render", "mappers",
                             "dpc", "fe", "micro"])
    ap.add_argument("--serve-requests", type=int, default=20000, help="saturation requests of the serve workload")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving summary of the default line")
    ap.add_argument("--render-instances", type=int, default=RENDER_N, help="consoles of the render workload")
    ap.add_argument("--render-cta-warps", type=int, default=16, choices=[4, 8, 16],
                    help="warps per CTA of the render kernel (128 registers: 16 warps/SM either way)")
    ap.add_argument("--block", type=int, default=128)
    ap.add_argument("--tuning", default=None, help="JSON file of per-cart tuning records (skips the autotuner)")
    ap.add_argument("--no-autotune", action="store_true", help="default policy and weights instead of the autotuner")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-buffer leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-kernel", action="store_true",
                    help="skip the timing of the reference's own CUDA kernel (oracle/_ref) in the default line")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-step-seconds", type=float, default=0.0,
                    help="CPU sample per step of the reference arm (0: sized so the run takes about 2 minutes)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    args.tuning = json.load(open(args.tuning)) if args.tuning else {}

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    fa = load_pkg()
    from fast_atari_b200 import carts

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local_rank)
        dist.init_process_group(dist_backend(), timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference":
            run_reference_arm(args, carts, rank, world)
        elif args.workload == "serve":
            run_serve_arm(args, fa, carts, rank, world, local_rank)
        elif args.workload == "render":
            run_render_arm(args, fa, carts, rank, world, local_rank)
        elif args.workload == "micro":
            run_micro_arm(args, fa, carts, rank, world, local_rank)
        else:
            run_gpu_arm(args, fa, carts, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
