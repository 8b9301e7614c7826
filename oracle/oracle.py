"""ctypes binding of the CPU oracle (oracle/fa_oracle.c).

TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the benchmark's
CPU-baseline leg use this module as the checker / timed CPU reference.  The
product path (the CUDA library) never imports it.

The oracle restates the reference's CPU emulator (RPP1011/fast-atari-rs
src/cpu.rs, src/atari.rs:9-105 and :384-620, src/headless_tia.rs, src/pia.rs).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libfa_oracle.so"

STATE_BYTES = 280

# fa_state (include/fast_atari.h), restated for the checker.
_fields = [
    ("a", "u1"), ("x", "u1"), ("y", "u1"), ("sp", "u1"),
    ("pc", "<u2"), ("status", "u1"), ("_pad0", "u1"),
    ("ram", "u1", (128,)),
    ("port_a_output", "u1"), ("port_a_ddr", "u1"), ("port_a_input", "u1"),
    ("port_b_output", "u1"), ("port_b_ddr", "u1"), ("port_b_input", "u1"),
    ("timer_value", "<u2"), ("timer_prescaler", "<u2"), ("timer_prescaler_select", "<u2"),
    ("timer_underflow", "u1"), ("_pad1", "u1"), ("_pad2", "u1"), ("_pad3", "u1"),
    ("tia_clock", "<u2"), ("tia_scanline", "<u2"),
    ("tia_wsync", "u1"), ("tia_frame_complete", "u1"), ("tia_vsync", "u1"), ("tia_vblank", "u1"),
    ("cxm0p", "u1"), ("cxm1p", "u1"), ("cxp0fb", "u1"), ("cxp1fb", "u1"),
    ("cxm0fb", "u1"), ("cxm1fb", "u1"), ("cxblpf", "u1"), ("cxppmm", "u1"),
    ("inpt4", "u1"), ("inpt5", "u1"), ("paddle0", "u1"), ("paddle1", "u1"),
    ("paddle_counter", "<u2"), ("paddle_dumped", "u1"), ("_pad4", "u1"),
    ("pos_p0", "<u2"), ("pos_p1", "<u2"), ("pos_m0", "<u2"), ("pos_m1", "<u2"), ("pos_bl", "<u2"),
    ("hmp0", "u1"), ("hmp1", "u1"), ("hmm0", "u1"), ("hmm1", "u1"), ("hmbl", "u1"), ("_pad5", "u1"),
    ("grp0", "u1"), ("grp1", "u1"), ("grp0_old", "u1"), ("grp1_old", "u1"),
    ("enam0", "u1"), ("enam1", "u1"), ("enabl", "u1"), ("enabl_old", "u1"),
    ("vdelp0", "u1"), ("vdelp1", "u1"), ("vdelbl", "u1"),
    ("resmp0", "u1"), ("resmp1", "u1"), ("nusiz0", "u1"), ("nusiz1", "u1"),
    ("colup0", "u1"), ("colup1", "u1"), ("colupf", "u1"), ("colubk", "u1"),
    ("ctrlpf", "u1"), ("refp0", "u1"), ("refp1", "u1"),
    ("pf0", "u1"), ("pf1", "u1"), ("pf2", "u1"),
    ("bank", "u1"), ("scheme", "u1"), ("_pad_end", "u1", (2,)),
    ("mapper", "u1", (2,)), ("_pad_ext", "u1"),
    ("cycles", "<u8"), ("frame_no", "<u4"), ("run_status", "<u4"),
    ("dpc_counter", "<u2", (8,)), ("dpc_top", "u1", (8,)), ("dpc_bottom", "u1", (8,)),
    ("dpc_flags", "u1"), ("dpc_music", "u1"), ("dpc_random", "u1"), ("_pad_dpc", "u1"),
    ("dpc_osc", "<u4"),
]
STATE_DTYPE = np.dtype(_fields, align=False)
assert STATE_DTYPE.itemsize == STATE_BYTES, STATE_DTYPE.itemsize

PAD_FIELDS = ("_pad0", "_pad1", "_pad2", "_pad3", "_pad4", "_pad5", "_pad_end", "_pad_ext", "_pad_dpc")
COMPARED_FIELDS = tuple(n for n in STATE_DTYPE.names if n not in PAD_FIELDS)


class OrcRegs(ctypes.Structure):
    _fields_ = [("pc", ctypes.c_uint16), ("sp", ctypes.c_uint8), ("a", ctypes.c_uint8),
                ("x", ctypes.c_uint8), ("y", ctypes.c_uint8), ("p", ctypes.c_uint8),
                ("_pad", ctypes.c_uint8), ("cycles", ctypes.c_uint64)]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, u8p, sz = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t
        L.orc_create.restype = vp
        L.orc_create.argtypes = [u8p, sz]
        L.orc_clone.restype = vp
        L.orc_clone.argtypes = [vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_action.argtypes = [vp, ctypes.c_uint]
        L.orc_run_frame.restype = ctypes.c_uint64
        L.orc_run_frame.argtypes = [vp]
        L.orc_ram.argtypes = [vp, u8p]
        L.orc_instructions.restype = ctypes.c_uint64
        L.orc_instructions.argtypes = [vp]
        L.orc_get_state.argtypes = [vp, vp]
        L.orc_set_state.argtypes = [vp, vp]
        L.orc_reset_state.restype = ctypes.c_int
        L.orc_reset_state.argtypes = [u8p, sz, vp]
        L.orc_run_batch.restype = ctypes.c_uint64
        L.orc_run_batch.argtypes = [u8p, sz, sz, ctypes.c_int, vp, u8p, vp, ctypes.c_uint32,
                                    u8p, ctypes.c_int, ctypes.c_int]
        L.orc_run_batch_trace.restype = ctypes.c_uint64
        L.orc_run_batch_trace.argtypes = [u8p, sz, sz, ctypes.c_int, vp, u8p, vp, ctypes.c_uint32,
                                          u8p, ctypes.c_int]
        L.orc_flat_run.restype = ctypes.c_int
        L.orc_flat_run.argtypes = [u8p, ctypes.c_int, u8p, ctypes.POINTER(OrcRegs)]
        L.orc_flat_run_from.restype = ctypes.c_int
        L.orc_flat_run_from.argtypes = [u8p, ctypes.c_int, u8p, ctypes.POINTER(OrcRegs)]
        L.orc_state_size.restype = ctypes.c_size_t
        L.orc_rcreate.restype = vp
        L.orc_rcreate.argtypes = [u8p, sz]
        L.orc_rclone.restype = vp
        L.orc_rclone.argtypes = [vp]
        L.orc_rdestroy.argtypes = [vp]
        L.orc_rset_action.argtypes = [vp, ctypes.c_uint]
        L.orc_rrun_frame.restype = ctypes.c_uint64
        L.orc_rrun_frame.argtypes = [vp]
        L.orc_rframebuffer.restype = vp
        L.orc_rframebuffer.argtypes = [vp]
        L.orc_rram.argtypes = [vp, u8p]
        L.orc_rregs.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32)]
        L.orc_rmapper.restype = ctypes.c_uint
        L.orc_rmapper.argtypes = [vp]
        L.orc_rom_set_scheme.restype = ctypes.c_int
        L.orc_rom_set_scheme.argtypes = [u8p, sz, ctypes.c_int]
        L.orc_rtia_size.restype = sz
        L.orc_rtia_copy.argtypes = [vp, vp]
        L.orc_rrun_batch.restype = ctypes.c_uint64
        L.orc_rrun_batch.argtypes = [ctypes.POINTER(vp), sz, ctypes.c_int, u8p, ctypes.c_int]
        L.orc_set_phantoms.argtypes = [ctypes.c_int]
        L.orc_rgba.argtypes = [u8p, sz, u8p]
        _lib = L
    return _lib


def _u8(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _bytes_arr(b) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(bytes(b), dtype=np.uint8))


class Atari:
    """One HeadlessAtari (src/atari.rs:556-620)."""

    def __init__(self, rom: bytes, _ptr=None):
        L = lib()
        if _ptr is None:
            r = _bytes_arr(rom)
            _ptr = L.orc_create(_u8(r), len(r))
            if not _ptr:
                raise ValueError(f"ROM length {len(rom)} cannot be constructed")
        self._p = _ptr

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_destroy(self._p)
            self._p = None

    def clone(self) -> "Atari":
        return Atari(b"", _ptr=lib().orc_clone(self._p))

    def set_action(self, action: int) -> None:
        lib().orc_set_action(self._p, int(action))

    def run_frame(self) -> int:
        return int(lib().orc_run_frame(self._p))

    def ram(self) -> np.ndarray:
        out = np.zeros(128, np.uint8)
        lib().orc_ram(self._p, _u8(out))
        return out

    def instructions(self) -> int:
        return int(lib().orc_instructions(self._p))

    def state(self) -> np.ndarray:
        s = np.zeros(1, STATE_DTYPE)
        lib().orc_get_state(self._p, s.ctypes.data)
        return s[0]

    def set_state(self, s) -> None:
        a = np.ascontiguousarray(np.array(s, dtype=STATE_DTYPE).reshape(1))
        lib().orc_set_state(self._p, a.ctypes.data)


# orc_rtia (oracle/fa_oracle.c), the rendering Tia's record, C layout.
RTIA_DTYPE = np.dtype([
    ("clock", "<u2"), ("scanline", "<u2"), ("wsync", "u1"), ("hmove_pending", "u1"),
    ("visible_top", "<u2"), ("vblank_top", "<u2"), ("pending_top", "<u2"), ("pending_frames", "u1"),
    ("delayed", "u1", (12,)), ("delayed_len", "u1"), ("frame_complete", "u1"),
    ("vsync", "u1"), ("vblank", "u1"), ("colup0", "u1"), ("colup1", "u1"), ("colupf", "u1"), ("colubk", "u1"),
    ("ctrlpf", "u1"), ("refp0", "u1"), ("refp1", "u1"), ("pf0", "u1"), ("pf1", "u1"), ("pf2", "u1"),
    ("grp0", "u1"), ("grp1", "u1"), ("grp0_old", "u1"), ("grp1_old", "u1"),
    ("enam0", "u1"), ("enam1", "u1"), ("enabl", "u1"), ("enabl_old", "u1"),
    ("hmp0", "u1"), ("hmp1", "u1"), ("hmm0", "u1"), ("hmm1", "u1"), ("hmbl", "u1"),
    ("nusiz0", "u1"), ("nusiz1", "u1"), ("vdelp0", "u1"), ("vdelp1", "u1"), ("vdelbl", "u1"),
    ("resmp0", "u1"), ("resmp1", "u1"),
    ("pos_p0", "<u2"), ("pos_p1", "<u2"), ("pos_m0", "<u2"), ("pos_m1", "<u2"), ("pos_bl", "<u2"),
    ("cxm0p", "u1"), ("cxm1p", "u1"), ("cxp0fb", "u1"), ("cxp1fb", "u1"),
    ("cxm0fb", "u1"), ("cxm1fb", "u1"), ("cxblpf", "u1"), ("cxppmm", "u1"),
    ("paddle0", "u1"), ("paddle1", "u1"), ("paddle_counter", "<u2"), ("paddle_dumped", "u1"),
    ("inpt4", "u1"), ("inpt5", "u1"), ("inpt4_latch", "u1"), ("inpt5_latch", "u1"), ("input_latch_enabled", "u1"),
    ("fb", "u1", (192, 160)),
], align=True)


class RenderAtari:
    """One rendering console, Atari (src/atari.rs:227-306) with the pixel-
    accurate Tia (src/tia.rs): a 160 x 192 framebuffer of palette indices."""

    FRAME_W, FRAME_H = 160, 192

    def __init__(self, rom: bytes, _ptr=None):
        L = lib()
        if _ptr is None:
            r = _bytes_arr(rom)
            _ptr = L.orc_rcreate(_u8(r), len(r))
            if not _ptr:
                raise ValueError(f"ROM length {len(rom)} cannot be constructed")
        self._p = _ptr

    def __del__(self):
        if getattr(self, "_p", None):
            lib().orc_rdestroy(self._p)
            self._p = None

    def clone(self) -> "RenderAtari":
        return RenderAtari(b"", _ptr=lib().orc_rclone(self._p))

    def set_action(self, action: int) -> None:
        lib().orc_rset_action(self._p, int(action))

    def run_frame(self) -> int:
        return int(lib().orc_rrun_frame(self._p))

    def framebuffer(self) -> np.ndarray:
        ptr = lib().orc_rframebuffer(self._p)
        buf = (ctypes.c_uint8 * (self.FRAME_W * self.FRAME_H)).from_address(ptr)
        return np.frombuffer(buf, np.uint8).reshape(self.FRAME_H, self.FRAME_W).copy()

    def ram(self) -> np.ndarray:
        out = np.zeros(128, np.uint8)
        lib().orc_rram(self._p, _u8(out))
        return out

    def regs(self) -> np.ndarray:
        """[axys, pc|p<<16|bank<<24, cycles lo, cycles hi, clock|scanline<<16, frame_no, run_status, timer]"""
        out = np.zeros(8, np.uint32)
        lib().orc_rregs(self._p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return out

    def mapper(self) -> int:
        """E0 / 3F bank state, as fa_state.mapper (little-endian 16 bits)."""
        return int(lib().orc_rmapper(self._p))

    def tia_record(self) -> np.ndarray:
        out = np.zeros(1, RTIA_DTYPE)
        assert RTIA_DTYPE.itemsize == lib().orc_rtia_size()
        lib().orc_rtia_copy(self._p, out.ctypes.data)
        return out[0]


def render_reset(rom: bytes, n: int):
    """n rendering consoles after new + one frame (the batched reset)."""
    first = RenderAtari(rom)
    first.run_frame()
    return [first] + [first.clone() for _ in range(n - 1)]


def render_steps(consoles, actions: np.ndarray, nthreads: int | None = None, outputs: bool = True):
    """Run k frames (actions [k, n]) on every console, on all host threads;
    returns the last frame's framebuffers [n, 192, 160] and RAM [n, 128]
    (None with outputs=False)."""
    k, n = actions.shape
    ptrs = (ctypes.c_void_p * n)(*[c._p for c in consoles])
    a = np.ascontiguousarray(actions, dtype=np.uint8)
    instr = lib().orc_rrun_batch(ptrs, n, k, _u8(a), nthreads or os.cpu_count() or 1)
    if instr == 2**64 - 1:
        raise RuntimeError("oracle render batch failed")
    if not outputs:
        return None
    return (np.stack([c.framebuffer() for c in consoles]), np.stack([c.ram() for c in consoles]))


SCHEMES = {"fixed": 0, "f8": 1, "f6": 2, "f4": 3, "e0": 4, "3f": 5, "dpc": 6, "fe": 7, "auto": -1}


def set_rom_scheme(rom: bytes, scheme) -> None:
    """The oracle's fa_rom_set_scheme: these bytes run under `scheme` in every
    later Atari / RenderAtari / reset_state / run_batch ("auto" forgets it)."""
    r = _bytes_arr(rom)
    code = SCHEMES[scheme.lower()] if isinstance(scheme, str) else int(scheme)
    if lib().orc_rom_set_scheme(_u8(r), len(r), code) != 0:
        raise ValueError(f"scheme {scheme!r} cannot hold a {len(r)}-byte ROM")


def rgba(fb: np.ndarray) -> np.ndarray:
    """Atari::render of framebuffers (any shape of palette indices): the same
    shape plus a last axis of R, G, B, A."""
    f = np.ascontiguousarray(fb, dtype=np.uint8)
    out = np.empty(f.shape + (4,), np.uint8)
    lib().orc_rgba(_u8(f.reshape(-1)), f.size, _u8(out.reshape(-1)))
    return out


class phantoms_off:
    """Context manager: inside it the oracle skips the headless bus's phantom
    reads and read-modify-write's first write (a deliberately wrong oracle,
    for tests that show a cart depends on those accesses)."""

    def __enter__(self):
        lib().orc_set_phantoms(0)
        return self

    def __exit__(self, *exc):
        lib().orc_set_phantoms(1)


def reset_state(rom: bytes) -> np.ndarray:
    """State after BatchAtariGpu::reset for one instance (new + one frame)."""
    r = _bytes_arr(rom)
    s = np.zeros(1, STATE_DTYPE)
    if lib().orc_reset_state(_u8(r), len(r), s.ctypes.data) != 0:
        raise ValueError("bad ROM")
    return s[0]


def run_batch(rom: bytes, states: np.ndarray, actions: np.ndarray, k: int,
              snapshot: np.ndarray | None = None, episode_frames: int = 0,
              nthreads: int | None = None, pin: bool = False,
              trace: bool = False):
    """Run len(states) instances for k frames; states are updated in place.

    actions: uint8 array of k*n, frame-major.  Returns (obs[n,128], instructions)
    or, with trace=True, (ram_trace[k,n,128], instructions).
    """
    L = lib()
    n = len(states)
    assert states.dtype == STATE_DTYPE and states.flags.c_contiguous
    acts = np.ascontiguousarray(actions, dtype=np.uint8).reshape(-1)
    assert acts.size == k * n, (acts.size, k, n)
    r = _bytes_arr(rom)
    snap_p = None
    if snapshot is not None:
        snap = np.ascontiguousarray(np.array(snapshot, dtype=STATE_DTYPE).reshape(1))
        snap_p = snap.ctypes.data
    nt = nthreads or os.cpu_count() or 1
    if trace:
        out = np.zeros((k, n, 128), np.uint8)
        instr = L.orc_run_batch_trace(_u8(r), len(r), n, k, states.ctypes.data, _u8(acts), snap_p,
                                      episode_frames, _u8(out), nt)
    else:
        out = np.zeros((n, 128), np.uint8)
        instr = L.orc_run_batch(_u8(r), len(r), n, k, states.ctypes.data, _u8(acts), snap_p,
                                episode_frames, _u8(out), nt, 1 if pin else 0)
    if instr == 2**64 - 1:
        raise RuntimeError("oracle batch run failed")
    return out, int(instr)


def flat_run(mem: np.ndarray, nsteps: int, regs: OrcRegs | None = None):
    """Run nsteps on a 64 KiB FlatMemory image (in place).

    Without regs: Cpu::new + reset from $FFFC.  Returns (regs, cycles[], steps_run).
    """
    assert mem.dtype == np.uint8 and mem.size == 65536 and mem.flags.c_contiguous
    cyc = np.zeros(max(nsteps, 1), np.uint8)
    if regs is None:
        regs = OrcRegs()
        n = lib().orc_flat_run(_u8(mem), nsteps, _u8(cyc), ctypes.byref(regs))
    else:
        n = lib().orc_flat_run_from(_u8(mem), nsteps, _u8(cyc), ctypes.byref(regs))
    return regs, cyc[:nsteps], n
