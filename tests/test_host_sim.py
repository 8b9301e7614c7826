"""The CUDA interpreter's own device code, compiled for the host, against the
oracle (CPU only).

tests/hostsim/ compiles fa_device.cuh (the 6502, bus, mappers, headless TIA
and PIA) and fa_run.cuh (the frame loop of run_frame / run_one_cycle) with
g++, one instance per lane of a host loop.  The full state after every call
must equal the oracle's on every cart family (the mixed batch, divergence,
scale, phantom-access, stall, E0 and 3F carts), on the reference's KATs
relocated to the 2600 bus, and on random ROMs started from random CPU
states.  The warp scheduling of the GPU only orders the lanes, so this
checks the interpreter's arithmetic and bus order without a GPU; the -m gpu
tests check the same on the device.
"""
import ctypes
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import kat_2600
import oracle
from fa_pkg import ROOT, carts

HERE = Path(__file__).resolve().parent / "hostsim"


@pytest.fixture(scope="module")
def sim():
    out = Path(tempfile.mkdtemp(prefix="fa_hostsim_")) / "libhostsim.so"
    cxx = os.environ.get("CXX", "g++")
    subprocess.run([cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-I", str(HERE), "-I", str(ROOT / "include"),
                    str(HERE / "host_run.cpp"), "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    L.hs_run.restype = ctypes.c_longlong
    L.hs_run.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p,
                         ctypes.c_int]
    L.fa_rom_set_scheme.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    L.hs_render.restype = ctypes.c_longlong
    L.hs_render.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.hs_host_copy.restype = None
    L.hs_host_copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    L.hs_plan.restype = None
    L.hs_plan.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    L.hs_timer.restype = None
    L.hs_timer.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return L


def run_both(L, rom, start, acts, k):
    ref, got = start.copy(), start.copy()
    oracle.run_batch(rom, ref, acts, k)
    r = np.frombuffer(rom, np.uint8).copy()
    a = np.ascontiguousarray(acts, dtype=np.uint8)
    assert L.hs_run(r.ctypes.data, len(r), got.ctypes.data, len(got), a.ctypes.data, k) >= 0
    return got, ref


def assert_same(got, ref, what):
    for f in oracle.COMPARED_FIELDS:
        if not np.array_equal(got[f], ref[f]):
            i = int(np.nonzero((got[f] != ref[f]).reshape(len(got), -1).any(axis=1))[0][0])
            raise AssertionError(f"{what}: {f} differs, first instance {i}: device code {got[f][i]} oracle {ref[f][i]}")


def cart_list():
    out = carts.mixed_carts() + [carts.plain_cart(), carts.divergence_cart(), carts.scale_cart()]
    out += carts.phantom_carts() + [carts.stall_cart("no_vsync"), carts.stall_cart("vsync_held")]
    return out


@pytest.mark.parametrize("c", cart_list(), ids=lambda c: c.spec.name)
def test_device_core_matches_oracle_on_carts(sim, c):
    n, k = 48, 5
    start = np.array([oracle.reset_state(c.rom)] * n, dtype=oracle.STATE_DTYPE)
    got, ref = run_both(sim, c.rom, start, carts.actions(seed=1, n=n, frames=k), k)
    assert_same(got, ref, c.spec.name)


@pytest.mark.parametrize("name", ["e0", "3f16", "3f6", "dpc", "dpc_tail", "dpc_script", "fe"])
def test_device_core_matches_oracle_on_sliced_carts(sim, name):
    """E0, 3F and FE registered per ROM; DPC picked by its lengths (10,240
    and 10,495 bytes) on both sides."""
    c, code = {"e0": (carts.e0_cart(), 4), "3f16": (carts.f3_cart(16384), 5), "3f6": (carts.f3_cart(6144), 5),
               "dpc": (carts.dpc_cart(), -1), "dpc_tail": (carts.dpc_cart(dump_tail=True), -1),
               "dpc_script": (carts.dpc_script_cart(), -1), "fe": (carts.fe_cart(), 7)}[name]
    r = np.frombuffer(c.rom, np.uint8).copy()
    sim.fa_rom_set_scheme(r.ctypes.data, len(r), code)
    oracle.set_rom_scheme(c.rom, code)
    try:
        n, k = 40, 12 if code < 0 else 4
        start = np.array([oracle.reset_state(c.rom)] * n, dtype=oracle.STATE_DTYPE)
        got, ref = run_both(sim, c.rom, start, carts.actions(seed=2, n=n, frames=k), k)
        assert_same(got, ref, name)
    finally:
        sim.fa_rom_set_scheme(r.ctypes.data, len(r), -1)
        oracle.set_rom_scheme(c.rom, "auto")


def test_device_core_runs_the_reference_kats(sim):
    for k in kat_2600.KATS:
        rom = k.image()
        start = np.repeat(kat_2600.kat_start_state(k, rom), 2)
        got, ref = run_both(sim, rom, start, np.zeros((1, 2), np.uint8), 1)
        assert_same(got, ref, k.name)
        kat_2600.check_kat(k, got[0], "device code")


@pytest.mark.parametrize("size", [2048, 4096, 8192, 16384, 32768])
def test_device_core_on_random_roms_and_states(sim, size):
    rng = np.random.default_rng(size)
    for t in range(6):
        rom = bytearray(rng.integers(0, 256, size, dtype=np.uint8).tobytes())
        for b in range(max(1, size // 4096)):
            base = b * 4096 + min(size, 4096) - 4
            rom[base:base + 2] = bytes([0x00, 0xF0])
        rom = bytes(rom)
        n = 64
        st = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
        st["a"], st["x"], st["y"] = rng.integers(0, 256, n), rng.integers(0, 256, n), rng.integers(0, 256, n)
        st["sp"], st["status"] = rng.integers(0, 256, n), rng.integers(0, 256, n) & 0xCF
        st["pc"] = 0xF000 + rng.integers(0, 0x1000, n)
        st["ram"] = rng.integers(0, 256, (n, 128))
        st["run_status"] = 0
        got, ref = run_both(sim, rom, st, carts.actions(seed=t, n=n, frames=3), 3)
        assert_same(got, ref, f"random {size}-byte ROM {t}")


@pytest.mark.parametrize("scheme,code", [("fe", 7), ("dpc", 6)])
def test_extra_cores_on_random_roms_and_states(sim, scheme, code):
    """The FE and DPC cores on random images from random CPU states and RAM,
    some started armed (FE) or with random DPC registers: random stack
    pointers ($F8-$FF and, wrapping, $00-$07) put JSR, RTS, RTI, PHA, PLA,
    BRK and indexed or indirect accesses on $01FE, and every phantom access
    the reference CPU makes
    (zero-page bases, stack reads, old-value writes, fix-ups) must reach the
    FE decode in the oracle's order; random reads and writes hit the DPC
    registers in every function."""
    rng = np.random.default_rng(code)
    size = 8192 if scheme == "fe" else 10240
    for t in range(8):
        rom = bytearray(rng.integers(0, 256, size, dtype=np.uint8).tobytes())
        for b in range(2):
            rom[b * 4096 + 4092:b * 4096 + 4094] = bytes([0x00, 0xF0])
        rom = bytes(rom)
        r = np.frombuffer(rom, np.uint8).copy()
        if scheme == "fe":
            sim.fa_rom_set_scheme(r.ctypes.data, len(r), code)
            oracle.set_rom_scheme(rom, code)
        try:
            n = 96
            st = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
            st["a"], st["x"], st["y"] = rng.integers(0, 256, n), rng.integers(0, 256, n), rng.integers(0, 256, n)
            # Stacks at $01F8-$01FF put $01FE in reach; at $0100-$0107 they
            # wrap and push into the TIA's mirror.
            st["sp"] = (rng.integers(0xF8, 0x108, n) & 0xFF)
            st["status"] = rng.integers(0, 256, n) & 0xCF
            st["pc"] = 0xF000 + rng.integers(0, 0x1000, n)
            st["ram"] = rng.integers(0, 256, (n, 128))
            st["mapper"][:, 0] = rng.integers(0, 2, n)
            st["mapper"][:, 1] = rng.integers(0, 2, n) if scheme == "fe" else 0
            if scheme == "dpc":
                st["dpc_counter"] = rng.integers(0, 2048, (n, 8))
                st["dpc_top"] = rng.integers(0, 256, (n, 8))
                st["dpc_bottom"] = rng.integers(0, 256, (n, 8))
                st["dpc_flags"] = rng.integers(0, 256, n)
                st["dpc_music"] = rng.integers(0, 8, n)
                st["dpc_random"] = rng.integers(0, 256, n)
            st["run_status"] = 0
            got, ref = run_both(sim, rom, st, carts.actions(seed=t, n=n, frames=3), 3)
            assert_same(got, ref, f"random {scheme} image {t}")
        finally:
            if scheme == "fe":
                sim.fa_rom_set_scheme(r.ctypes.data, len(r), -1)
                oracle.set_rom_scheme(rom, "auto")


def test_device_core_every_opcode_first(sim):
    """Instance i starts on a byte equal to i, with random registers and RAM:
    every one of the 256 opcodes (the 151 and the illegal ones) executes
    first at least once."""
    rng = np.random.default_rng(99)
    for size in (4096, 32768):
        rom = bytearray(rng.integers(0, 256, size, dtype=np.uint8).tobytes())
        for b in range(size // 4096):
            rom[b * 4096 + 0xFFC:b * 4096 + 0xFFE] = bytes([0x00, 0xF0])
            rom[b * 4096 + 0x800:b * 4096 + 0x900] = bytes(range(256))     # opcode i at $F800 + i
        rom = bytes(rom)
        n = 256
        st = np.array([oracle.reset_state(rom)] * n, dtype=oracle.STATE_DTYPE)
        st["a"], st["x"], st["y"] = rng.integers(0, 256, n), rng.integers(0, 256, n), rng.integers(0, 256, n)
        st["sp"], st["status"] = rng.integers(0, 256, n), rng.integers(0, 256, n) & 0xCF
        st["pc"] = 0xF800 + np.arange(n)
        st["ram"] = rng.integers(0, 256, (n, 128))
        st["run_status"] = 0
        got, ref = run_both(sim, rom, st, carts.actions(seed=5, n=n, frames=2), 2)
        assert_same(got, ref, f"every opcode first, {size}-byte ROM")
        assert (ref["run_status"] & 1).sum() >= 105          # the illegal opcodes halt at once


def _timer_run(L, start, ns, settle):
    ns = np.ascontiguousarray(ns, dtype=np.uint32)
    settle = np.ascontiguousarray(settle, dtype=np.uint8)
    st = np.ascontiguousarray(start, dtype=np.uint32)
    out = np.zeros((len(ns), 8), np.uint32)
    L.hs_timer(st.ctypes.data, ns.ctypes.data, settle.ctypes.data, len(ns), out.ctypes.data)
    return out[:, :4], out[:, 4:]


def test_lazy_timer_counting_equals_per_call_ticks(sim):
    """The headless core counts instruction cycles off the timer lazily and
    settles them on INTIM reads, PIA writes and state stores; after every
    call, and after INTIM reads that clear the underflow flag, its state as
    stored must equal
    Pia::tick_n run on every call
    (src/pia.rs:107-166), across underflows, the post-underflow wrap, every
    interval, prescalers of 0 and above the interval, and calls of 0 to 80
    cycles (instructions and WSYNC skips) and a few of up to 700."""
    rng = np.random.default_rng(2600)
    starts = [(tv, ps, sel, uf) for sel in (1, 8, 64, 1024) for tv in (0, 1, 2, 3, 200, 255)
              for ps in (0, 1, 2, sel, sel + 3) for uf in (0, 1)]
    starts += [(int(rng.integers(0, 256)), int(rng.integers(0, 1100)), int(rng.choice([1, 8, 64, 1024])),
                int(rng.integers(0, 2))) for _ in range(1500)]
    starts += [(5, 3, 3, 0), (300, 2, 8, 0)]                      # states only an upload makes
    for start in starts:
        m = 3000 if start[2] >= 64 else 1200
        ns = np.where(rng.random(m) < 0.05, rng.integers(0, 81, m), rng.integers(1, 8, m))
        ns = np.where(rng.random(m) < 0.003, rng.integers(81, 700, m), ns)
        settle = np.where(rng.random(m) < 0.03, rng.integers(1, 4, m), 0)
        lazy, exact = _timer_run(sim, start, ns, settle)
        bad = np.nonzero((lazy != exact).any(axis=1))[0]
        assert len(bad) == 0, (f"start {start}: call {bad[0]} (n={ns[bad[0]]}) lazy {lazy[bad[0]]} "
                               f"exact {exact[bad[0]]}")
        if start[2] == 1 and start[0] >= 1:
            assert exact[:, 3].any()                               # the run went through underflows


@pytest.mark.parametrize("grid,warps,nunits", [(148, 32, 4236), (10, 8, 100), (5, 4, 7), (148, 28, 4144), (20, 32, 300)])
def test_first_wave_plan(sim, grid, warps, nunits):
    """fa_plan_first_wave (fa_pool_set_balance): slot warp * grid + cta gets
    units 0 .. min(units, slots) - 1 exactly once (the device queue hands out
    the rest), every unit on a warp of its (SM, scheduler) sub-partition
    (warp % 4), at most warps / 4 per sub-partition, placed longest first on
    the least-loaded one."""
    rng = np.random.default_rng(grid * warps + nunits)
    cost = np.concatenate([rng.choice([1.0, 1.1, 1.8, 17.0], nunits, p=[0.7, 0.2, 0.07, 0.03])]).astype(np.float32)
    table = np.zeros(grid * warps, np.uint32)
    sim.hs_plan(cost.ctypes.data, nunits, grid, warps, table.ctypes.data)
    slots = grid * warps
    first = min(nunits, slots)
    used = table[table != 0xFFFFFFFF]
    assert sorted(used.tolist()) == list(range(first))
    parts = grid * 4
    load = np.zeros(parts)
    count = np.zeros(parts, int)
    for slot, u in enumerate(table):
        if u == 0xFFFFFFFF:
            continue
        warp, cta = divmod(slot, grid)
        q = cta * 4 + warp % 4
        load[q] += cost[u]
        count[q] += 1
    assert count.max() <= warps // 4
    if nunits <= slots and count.max() < warps // 4:
        # capacity never bound: longest-first keeps every load within one unit of the lightest
        assert load.max() - load.min() <= cost.max() + 1e-4
    elif (grid, warps, nunits) == (20, 32, 300):
        raise AssertionError("the unconstrained case must exercise the balance check")
    heaviest = np.argsort(-cost[:first], kind="stable")[:min(parts, first)]
    qs = {}
    for slot, u in enumerate(table):
        if u != 0xFFFFFFFF:
            warp, cta = divmod(slot, grid)
            qs[int(u)] = cta * 4 + warp % 4
    assert len({qs[int(u)] for u in heaviest}) == len(heaviest)


@pytest.mark.parametrize("nbytes", [0, 1, 4097, (2 << 20) - 1, 2 << 20, (5 << 20) + 3, (17 << 20) + 12345])
def test_host_copy(sim, nbytes):
    """fa_host_copy, the copy of a host-buffer call's outputs into the
    caller's memory: one thread below 2 MB, up to 8 above, every byte in
    place, nothing written past the end."""
    rng = np.random.default_rng(nbytes)
    src = rng.integers(0, 256, nbytes, dtype=np.uint8)
    dst = np.full(nbytes + 64, 0x5A, np.uint8)
    sim.hs_host_copy(dst.ctypes.data, src.ctypes.data, nbytes)
    assert np.array_equal(dst[:nbytes], src)
    assert (dst[nbytes:] == 0x5A).all()


@pytest.mark.parametrize("name", ["render", "divergence", "mixed_32k", "e0", "3f16"])
def test_rendering_console_device_code_matches_oracle(sim, name):
    """The rendering console's device code (fa_render.cuh's frame loop over
    fa_device.cuh with RENDER) compiled for the host, driven as
    fa_render_reset and fa_render_step_multi drive it (the kernel's start and
    end of a launch restated in host_run.cpp), against the rendering oracle (the
    reference's Atari + Tia restated): framebuffers, RAM, registers, cycles,
    beam, timer and every TIA register after two calls of 3 frames."""
    from fa_pkg import fa
    from test_gpu_render import check
    c, code = {"render": (carts.render_cart(), None), "divergence": (carts.divergence_cart(), None),
               "mixed_32k": (carts.mixed_carts()[3], None), "e0": (carts.e0_cart(), 4),
               "3f16": (carts.f3_cart(16384), 5)}[name]
    rom = c.rom
    r = np.frombuffer(rom, np.uint8).copy()
    if code is not None:
        sim.fa_rom_set_scheme(r.ctypes.data, len(r), code)
        oracle.set_rom_scheme(rom, code)
    try:
        n, calls, k = 6, 2, 3
        acts = np.stack([carts.actions(seed=70 + i, n=n, frames=k) for i in range(calls)])
        fb = np.zeros((n, 192, 160), np.uint8)
        ram = np.zeros((n, 128), np.uint8)
        st = np.zeros(n, fa.STATE_DTYPE)
        a = np.ascontiguousarray(acts, dtype=np.uint8)
        assert sim.hs_render(r.ctypes.data, len(r), n, a.ctypes.data, calls, k, fb.ctypes.data, st.ctypes.data,
                             ram.ctypes.data) >= 0
        consoles = oracle.render_reset(rom, n)
        for i in range(calls):
            oracle.render_steps(consoles, acts[i])
        check(fb, ram, st, consoles, f"{name} on the host")
    finally:
        if code is not None:
            sim.fa_rom_set_scheme(r.ctypes.data, len(r), -1)
            oracle.set_rom_scheme(rom, "auto")
