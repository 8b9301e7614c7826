"""B200 batched Atari 2600 emulator core — Python binding of the C ABI.

`BatchAtariGpu` mirrors the reference's Rust API (RPP1011/fast-atari-rs
src/cuda_env.rs:99-191): construct from ROM bytes and an instance count, then
reset / step / step_multi / set_sorted / download_states / num_envs.  All
emulation runs in the sm_100a library (lib/libfast_atari.so, built by
build.py); this module only marshals buffers.  There is no CPU fallback: if
the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Optional

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libfast_atari.so"

FA_OK = 0
FA_STATUS_ILLEGAL_OPCODE = 0x1
FA_STATUS_VSYNC_BUDGET = 0x2
FA_STATUS_NOT_RESET = 0x4
FA_STATUS_HALT_MASK = 0x7
FA_STATUS_CYCLE_CAP = 0x100

SCHED_LANE, SCHED_PC, SCHED_LINE, SCHED_MATCH = 0, 1, 2, 3
SCHED_NAMES = {"lane": SCHED_LANE, "pc": SCHED_PC, "line": SCHED_LINE, "match": SCHED_MATCH}

# fa_state, include/fast_atari.h (the reference AtariStateGpu prefix + extension).
STATE_DTYPE = np.dtype([
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
])
assert STATE_DTYPE.itemsize == 280

# Symbols declared in include/fast_atari.h, with ctypes signatures.
_vp, _u8p, _sz, _i, _u32 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t, ctypes.c_int, ctypes.c_uint32
_SIGS = {
    "fa_last_error": (ctypes.c_char_p, []),
    "fa_version": (ctypes.c_char_p, []),
    "fa_device_count": (_i, []),
    "fa_set_device": (_i, [_i]),
    "fa_set_wait_limit_ns": (_i, [ctypes.c_uint64]),
    "fa_wait_limit_ns_get": (ctypes.c_uint64, []),
    "fa_create": (_i, [_u8p, _sz, _sz, ctypes.POINTER(_vp)]),
    "fa_destroy": (None, [_vp]),
    "fa_num_envs": (_sz, [_vp]),
    "fa_set_sorted": (_i, [_vp, _i]),
    "fa_reset": (_i, [_vp, _u8p]),
    "fa_step": (_i, [_vp, _u8p, _u8p]),
    "fa_step_multi": (_i, [_vp, _u8p, _i, _u8p]),
    "fa_step_multi_async": (_i, [_vp, _vp, _i, _vp, _vp]),
    "fa_synchronize": (_i, [_vp]),
    "fa_get_states": (_i, [_vp, _vp]),
    "fa_set_states": (_i, [_vp, _vp]),
    "fa_get_ram": (_i, [_vp, _sz, _u8p]),
    "fa_get_status": (_i, [_vp, ctypes.POINTER(_u32)]),
    "fa_set_episode_frames": (_i, [_vp, _u32]),
    "fa_set_frame_numbers": (_i, [_vp, ctypes.POINTER(_u32)]),
    "fa_set_launch": (_i, [_vp, _i, _i, _i]),
    "fa_get_launch": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)]),
    "fa_last_instructions": (ctypes.c_ulonglong, [_vp]),
    "fa_last_lane_slots": (ctypes.c_ulonglong, [_vp]),
    "fa_get_snapshot": (_i, [_vp, _vp]),
    "fa_device_state": (_vp, [_vp, ctypes.POINTER(_u32)]),
    "fa_pool_create": (_i, [ctypes.POINTER(_vp)]),
    "fa_pool_destroy": (None, [_vp]),
    "fa_pool_add_cart": (_i, [_vp, _u8p, _sz, _sz, ctypes.POINTER(_i)]),
    "fa_pool_num_groups": (_i, [_vp]),
    "fa_pool_group": (_vp, [_vp, _i]),
    "fa_pool_set_group": (_i, [_vp, _i, _i, ctypes.c_float]),
    "fa_pool_set_launch": (_i, [_vp, _i, _i]),
    "fa_pool_step": (_i, [_vp, _vp, _i, _vp]),
    "fa_pool_step_plain": (_i, [_vp, _vp, _i, _vp]),
    "fa_pool_step_async": (_i, [_vp, _vp, _i, _vp, _vp]),
    "fa_pool_step_plain_async": (_i, [_vp, _vp, _i, _vp, _vp]),
    "fa_pool_synchronize": (_i, [_vp]),
    "fa_pool_set_balance": (_i, [_vp, _i]),
    "fa_pool_set_trace": (_i, [_vp, _vp, ctypes.c_uint32]),
    "fa_pool_reset_counters": (_i, [_vp]),
    "fa_pool_last_instructions": (ctypes.c_ulonglong, [_vp]),
    "fa_pool_last_lane_slots": (ctypes.c_ulonglong, [_vp]),
    "fa_pool_stream": (_vp, [_vp]),
    "fa_pool_graph_create": (_i, [_vp, _vp, _i, _i, _vp, ctypes.POINTER(_vp)]),
    "fa_graph_launch": (_i, [_vp, _vp]),
    "fa_graph_destroy": (None, [_vp]),
    "fa_step_static": (_i, [_vp, _i, _vp, _u32, _u32, _vp, _i, _i, _vp, _i, _vp]),
    "fa_set_cta_warps": (_i, [_vp, _i]),
    "fa_pool_set_cta_warps": (_i, [_vp, _i]),
    "fa_autotune": (_i, [_u8p, _sz, _sz, _vp, _vp, _i, ctypes.POINTER(_i)]),
    "fa_obs_to_unit_f32": (_i, [_vp, _vp, _sz, _vp]),
    "fa_obs_reward": (_i, [_vp, _sz, _vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "fa_server_create": (_i, [_vp, _vp, _i, _vp, ctypes.POINTER(_vp)]),
    "fa_server_destroy": (None, [_vp]),
    "fa_server_open": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int64)]),
    "fa_server_close": (_i, [_vp, ctypes.c_int64]),
    "fa_server_submit": (_i, [_vp, ctypes.c_int64, _vp, _u32, _i, _vp, ctypes.POINTER(ctypes.c_uint64)]),
    "fa_server_wait": (_i, [_vp, ctypes.c_uint64, _i, _vp]),
    "fa_server_step": (_i, [_vp, ctypes.c_int64, _vp, _u32, _i, _vp, _vp]),
    "fa_server_session_size": (_i, [_vp, ctypes.c_int64, ctypes.POINTER(_u32)]),
    "fa_server_get_states": (_i, [_vp, ctypes.c_int64, _u32, _u32, _vp]),
    "fa_server_stats_get": (_i, [_vp, _vp]),
    "fa_server_loadgen": (_i, [_vp, _vp, _vp, _vp]),
    "fa_rom_set_scheme": (_i, [_u8p, _sz, _i]),
    "fa_rom_scheme": (_i, [_u8p, _sz]),
    "fa_rom_guess_scheme": (_i, [_u8p, _sz]),
    "fa_render_create": (_i, [_u8p, _sz, _sz, ctypes.POINTER(_vp)]),
    "fa_render_destroy": (None, [_vp]),
    "fa_render_num_envs": (_sz, [_vp]),
    "fa_render_set_launch": (_i, [_vp, _i, _i]),
    "fa_render_reset": (_i, [_vp, _vp, _vp]),
    "fa_render_step_multi": (_i, [_vp, _u8p, _i, _vp, _vp]),
    "fa_render_step_multi_async": (_i, [_vp, _vp, _i, _vp, _vp]),
    "fa_render_synchronize": (_i, [_vp]),
    "fa_render_device_framebuffers": (_vp, [_vp]),
    "fa_render_get_framebuffers": (_i, [_vp, _vp]),
    "fa_render_get_states": (_i, [_vp, _vp]),
    "fa_render_last_instructions": (ctypes.c_ulonglong, [_vp]),
    "fa_render_rgba_async": (_i, [_vp, _sz, _sz, _vp, _vp]),
    "fa_render_get_rgba": (_i, [_vp, _sz, _sz, _vp]),
    "fa_palette_rgba": (ctypes.c_uint32, [ctypes.c_uint8]),
}

FA_ERR_BAD_ROM = -2
FA_ERR_CAPACITY = -6
FA_ERR_TIMEOUT = -7
SERVE_BATCHED, SERVE_PLAIN = 0, 1


class FaTuning(ctypes.Structure):
    """fa_tuning (include/fast_atari.h)."""
    _fields_ = [("block", ctypes.c_int), ("persistent", ctypes.c_int), ("cta_warps", ctypes.c_int),
                ("sched", ctypes.c_int), ("k", ctypes.c_int), ("frames_per_s", ctypes.c_float),
                ("ns_per_instance_frame", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}

_lib: Optional[ctypes.CDLL] = None


class FaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fast_atari error {code}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run build.py (no CPU fallback exists)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != FA_OK:
        raise FaError(rc, lib().fa_last_error().decode())


def _u8(a: np.ndarray):
    return a.ctypes.data_as(_u8p)


def device_count() -> int:
    return int(lib().fa_device_count())


def set_device(device: int) -> None:
    _check(lib().fa_set_device(int(device)))


def palette_rgba(index: int) -> tuple:
    """ntsc_palette of one palette index as (R, G, B, A)."""
    v = int(lib().fa_palette_rgba(int(index) & 0xFF))
    return (v & 0xFF, (v >> 8) & 0xFF, (v >> 16) & 0xFF, v >> 24)


def set_wait_limit_ns(ns: int) -> None:
    """Bound of the device-side ROM staging wait for later launches (0 gives
    up at once; the call then returns FA_ERR_KERNEL with states untouched)."""
    _check(lib().fa_set_wait_limit_ns(int(ns)))


def wait_limit_ns() -> int:
    return int(lib().fa_wait_limit_ns_get())


SCHEME_NAMES = {"fixed": 0, "f8": 1, "f6": 2, "f4": 3, "e0": 4, "3f": 5, "dpc": 6, "fe": 7, "auto": -1}


def _scheme_code(scheme) -> int:
    return SCHEME_NAMES[scheme.lower()] if isinstance(scheme, str) else int(scheme)


def set_rom_scheme(rom: bytes, scheme) -> None:
    """Every later handle, pool, server or rendering console given these ROM
    bytes uses `scheme` ("e0", "3f", ... or "auto" to forget it) instead of
    the reference's size rule (fa_rom_set_scheme)."""
    r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
    _check(lib().fa_rom_set_scheme(_u8(r), len(r), _scheme_code(scheme)))


def rom_scheme(rom: bytes) -> int:
    """The scheme the library will use for these bytes (fa_rom_scheme)."""
    r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
    rc = int(lib().fa_rom_scheme(_u8(r), len(r)))
    _check(min(rc, 0))
    return rc


def guess_rom_scheme(rom: bytes) -> int:
    """A scheme guessed from the ROM's code (fa_rom_guess_scheme); not applied."""
    r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
    rc = int(lib().fa_rom_guess_scheme(_u8(r), len(r)))
    _check(min(rc, 0))
    return rc


class RewardSpec(ctypes.Structure):
    """fa_reward_spec: where a game keeps its score, lives and end flag in RAM
    (offsets 0..127).  Score bytes most significant first, BCD or binary."""
    _fields_ = [("score_addr", ctypes.c_uint8 * 4), ("score_bytes", ctypes.c_uint8), ("score_bcd", ctypes.c_uint8),
                ("lives_addr", ctypes.c_uint8), ("lives_mask", ctypes.c_uint8), ("lives_shift", ctypes.c_uint8),
                ("terminal_addr", ctypes.c_uint8), ("terminal_mask", ctypes.c_uint8),
                ("terminal_value", ctypes.c_uint8)]

    @classmethod
    def make(cls, score=(), bcd=True, lives=None, terminal=None) -> "RewardSpec":
        """score: RAM offsets (most significant first); lives: (offset, mask,
        shift); terminal: (offset, mask, value)."""
        sp = cls()
        for i, a in enumerate(score):
            sp.score_addr[i] = a
        sp.score_bytes = len(score)
        sp.score_bcd = 1 if bcd else 0
        if lives:
            sp.lives_addr, sp.lives_mask, sp.lives_shift = lives
        if terminal:
            sp.terminal_addr, sp.terminal_mask, sp.terminal_value = terminal
        return sp


EPISODE_TERMINAL, EPISODE_LIFE_LOST = 0x1, 0x2


def obs_reward(d_obs: int, n: int, spec: RewardSpec, init: bool, d_score: int, d_lives: int,
               d_reward: int = 0, d_flags: int = 0, stream: int = 0) -> None:
    """fa_obs_reward on device pointers (torch tensors' data_ptr())."""
    _check(lib().fa_obs_reward(_vp(d_obs), int(n), ctypes.byref(spec), 1 if init else 0, _vp(d_score), _vp(d_lives),
                               _vp(d_reward or None), _vp(d_flags or None), _vp(stream or None)))


class BatchAtariGpu:
    """n emulated consoles of one ROM, resident on the current CUDA device."""

    def __init__(self, rom: bytes, n: int, _handle=None):
        L = lib()
        self._owned = _handle is None
        if _handle is None:
            r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
            h = _vp()
            _check(L.fa_create(_u8(r), len(r), int(n), ctypes.byref(h)))
            _handle = h
        self._h = _handle
        self.n = int(n)
        self.rom = bytes(rom)

    def close(self) -> None:
        if getattr(self, "_h", None):
            if self._owned:
                lib().fa_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- the reference method set
    def num_envs(self) -> int:
        return int(lib().fa_num_envs(self._h))

    def set_sorted(self, sorted_: bool) -> None:
        _check(lib().fa_set_sorted(self._h, 1 if sorted_ else 0))

    def reset(self) -> np.ndarray:
        obs = np.zeros((self.n, 128), np.uint8)
        _check(lib().fa_reset(self._h, _u8(obs)))
        return obs

    def step(self, actions, obs: bool = True) -> Optional[np.ndarray]:
        a = np.ascontiguousarray(actions, dtype=np.uint8).reshape(-1)
        if a.size != self.n:
            raise ValueError(f"expected {self.n} actions, got {a.size}")
        out = np.empty((self.n, 128), np.uint8) if obs else None
        _check(lib().fa_step(self._h, _u8(a), _u8(out) if obs else None))
        return out

    def step_multi(self, actions, k: int, obs: bool = True) -> Optional[np.ndarray]:
        a = np.ascontiguousarray(actions, dtype=np.uint8).reshape(-1)
        if a.size != k * self.n:
            raise ValueError(f"expected {k}*{self.n} actions, got {a.size}")
        out = np.empty((self.n, 128), np.uint8) if obs else None
        _check(lib().fa_step_multi(self._h, _u8(a), int(k), _u8(out) if obs else None))
        return out

    def download_states(self) -> np.ndarray:
        s = np.zeros(self.n, STATE_DTYPE)
        _check(lib().fa_get_states(self._h, s.ctypes.data))
        return s

    # ---- extensions
    def upload_states(self, states: np.ndarray) -> None:
        s = np.ascontiguousarray(states, dtype=STATE_DTYPE)
        assert s.size == self.n
        _check(lib().fa_set_states(self._h, s.ctypes.data))

    def ram(self, idx: int) -> np.ndarray:
        out = np.zeros(128, np.uint8)
        _check(lib().fa_get_ram(self._h, int(idx), _u8(out)))
        return out

    def status(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        _check(lib().fa_get_status(self._h, out.ctypes.data_as(ctypes.POINTER(_u32))))
        return out

    def snapshot(self) -> np.ndarray:
        s = np.zeros(1, STATE_DTYPE)
        _check(lib().fa_get_snapshot(self._h, s.ctypes.data))
        return s[0]

    def set_episode_frames(self, frames: int) -> None:
        _check(lib().fa_set_episode_frames(self._h, int(frames)))

    def set_frame_numbers(self, frame_no) -> None:
        f = np.ascontiguousarray(frame_no, dtype=np.uint32)
        assert f.size == self.n
        _check(lib().fa_set_frame_numbers(self._h, f.ctypes.data_as(ctypes.POINTER(_u32))))

    def set_launch(self, block: int = 128, sched="lane", persistent: bool = False, cta_warps: int = 0) -> None:
        s = SCHED_NAMES[sched] if isinstance(sched, str) else int(sched)
        _check(lib().fa_set_launch(self._h, int(block), s, 1 if persistent else 0))
        _check(lib().fa_set_cta_warps(self._h, int(cta_warps)))

    def get_launch(self):
        b, s, p = _i(), _i(), _i()
        _check(lib().fa_get_launch(self._h, ctypes.byref(b), ctypes.byref(s), ctypes.byref(p)))
        return b.value, s.value, bool(p.value)

    def last_instructions(self) -> int:
        return int(lib().fa_last_instructions(self._h))

    def last_lane_slots(self) -> int:
        return int(lib().fa_last_lane_slots(self._h))

    def step_multi_async(self, d_actions: int, k: int, d_obs: int = 0, stream: int = 0) -> None:
        """Enqueue k frames from device actions (e.g. torch tensor data_ptr())."""
        _check(lib().fa_step_multi_async(self._h, _vp(d_actions), int(k), _vp(d_obs or None),
                                          _vp(stream or None)))

    def synchronize(self) -> None:
        _check(lib().fa_synchronize(self._h))


def _ptrs(seq):
    arr = (_vp * len(seq))()
    for i, v in enumerate(seq):
        arr[i] = v or None
    return arr


class AtariPool:
    """Several carts' instance sets stepped together (the batched form)."""

    def __init__(self):
        h = _vp()
        _check(lib().fa_pool_create(ctypes.byref(h)))
        self._p = h
        self.groups = []          # (rom, n)

    def close(self) -> None:
        if getattr(self, "_p", None):
            lib().fa_pool_destroy(self._p)
            self._p = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_cart(self, rom: bytes, n: int) -> int:
        r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
        g = _i()
        _check(lib().fa_pool_add_cart(self._p, _u8(r), len(r), int(n), ctypes.byref(g)))
        self.groups.append((bytes(rom), int(n)))
        return g.value

    def group(self, g: int) -> BatchAtariGpu:
        """Non-owning view of group g's handle (states, status, episodes)."""
        rom, n = self.groups[g]
        return BatchAtariGpu(rom, n, _handle=_vp(lib().fa_pool_group(self._p, g)))

    def set_group(self, g: int, sched="pc", weight: float = 1.0) -> None:
        s = SCHED_NAMES[sched] if isinstance(sched, str) else int(sched)
        _check(lib().fa_pool_set_group(self._p, g, s, float(weight)))

    def set_launch(self, block: int = 128, persistent: bool = True, cta_warps: int = 0) -> None:
        _check(lib().fa_pool_set_launch(self._p, int(block), 1 if persistent else 0))
        _check(lib().fa_pool_set_cta_warps(self._p, int(cta_warps)))

    def _host_step(self, fn, actions, k, obs, out=None):
        acts = [np.ascontiguousarray(a, dtype=np.uint8).reshape(-1) for a in actions]
        for a, (_, n) in zip(acts, self.groups):
            if a.size != k * n:
                raise ValueError("actions size mismatch")
        if out is not None:
            if len(out) != len(self.groups):
                raise ValueError("one output array per cart")
            for o, (_, n) in zip(out, self.groups):
                if not (isinstance(o, np.ndarray) and o.dtype == np.uint8 and o.size == n * 128
                        and o.flags.c_contiguous and o.flags.writeable):
                    raise ValueError("each output must be a writable C-contiguous uint8 array of n*128 bytes")
            outs, obs = list(out), True
        else:
            outs = [np.empty((n, 128), np.uint8) for _, n in self.groups] if obs else None
        _check(fn(self._p, _ptrs([a.ctypes.data for a in acts]), int(k),
                  _ptrs([o.ctypes.data for o in outs]) if obs else None))
        return outs

    def step(self, actions, k: int, obs: bool = True, out=None):
        """One batched call from host buffers; returns each cart's RAM after
        the last frame.  `out`: the caller's (n, 128) uint8 arrays to fill,
        one per cart, instead of new ones."""
        return self._host_step(lib().fa_pool_step, actions, k, obs, out)

    def step_plain(self, actions, k: int, obs: bool = True, out=None):
        return self._host_step(lib().fa_pool_step_plain, actions, k, obs, out)

    def step_async(self, d_actions, k: int, d_obs=None, stream: int = 0) -> None:
        _check(lib().fa_pool_step_async(self._p, _ptrs(d_actions), int(k),
                                         _ptrs(d_obs) if d_obs else None, _vp(stream or None)))

    def step_plain_async(self, d_actions, k: int, d_obs=None, stream: int = 0) -> None:
        _check(lib().fa_pool_step_plain_async(self._p, _ptrs(d_actions), int(k),
                                               _ptrs(d_obs) if d_obs else None, _vp(stream or None)))

    def synchronize(self) -> None:
        _check(lib().fa_pool_synchronize(self._p))

    def reset_counters(self) -> None:
        _check(lib().fa_pool_reset_counters(self._p))

    def set_balance(self, on: bool = True) -> None:
        """Spread the persistent launch's first wave over the warp schedulers
        by cart weight (off by default)."""
        _check(lib().fa_pool_set_balance(self._p, 1 if on else 0))

    def set_trace(self, d_trace: int = 0, cap: int = 0) -> None:
        """Per-unit records of later batched launches into a device buffer of
        cap x 3 uint64 (start ns, end ns, smid << 32 | warp << 16 | group);
        set_trace() stops them."""
        _check(lib().fa_pool_set_trace(self._p, _vp(d_trace or None), int(cap)))

    def last_instructions(self) -> int:
        return int(lib().fa_pool_last_instructions(self._p))

    def last_lane_slots(self) -> int:
        return int(lib().fa_pool_last_lane_slots(self._p))

    def stream(self) -> int:
        return int(lib().fa_pool_stream(self._p) or 0)

    def graph(self, d_actions, k: int, calls: int, d_obs=None) -> "PoolGraph":
        g = _vp()
        _check(lib().fa_pool_graph_create(self._p, _ptrs(d_actions), int(k), int(calls),
                                           _ptrs(d_obs) if d_obs else None, ctypes.byref(g)))
        return PoolGraph(g, self)


class PoolGraph:
    def __init__(self, g, pool: AtariPool):
        self._g = g
        self.pool = pool

    def launch(self, stream: int = 0) -> None:
        _check(lib().fa_graph_launch(self._g, _vp(stream or None)))

    def close(self) -> None:
        if getattr(self, "_g", None):
            lib().fa_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        self.close()


def autotune(rom: bytes, n: int):
    """Run the project tuner for one cart; returns (best, table) as dicts."""
    r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
    best = FaTuning()
    table = (FaTuning * 64)()
    count = _i()
    _check(lib().fa_autotune(_u8(r), len(r), int(n), ctypes.byref(best), table, 64, ctypes.byref(count)))
    return best.as_dict(), [table[i].as_dict() for i in range(min(count.value, 64))]


# ------------------------------------------------------------------ serving
class ServerConfig(ctypes.Structure):
    """fa_server_config (include/fast_atari.h)."""
    _fields_ = [("state_budget_bytes", ctypes.c_size_t), ("mode", ctypes.c_int), ("block", ctypes.c_int),
                ("max_inflight", ctypes.c_int), ("sched", ctypes.c_int)]


class RequestInfo(ctypes.Structure):
    """fa_request_info (include/fast_atari.h)."""
    _fields_ = [("status", ctypes.c_int), ("waited_admission", ctypes.c_int), ("batch_requests", ctypes.c_uint),
                ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("session_wait_ms", ctypes.c_double), ("service_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class ServerStats(ctypes.Structure):
    """fa_server_stats (include/fast_atari.h)."""
    _fields_ = [(n, ctypes.c_ulonglong) for n in (
        "requests_submitted", "requests_done", "requests_failed", "instance_frames", "dispatches",
        "dispatched_requests", "launches", "admission_waits", "guest_instructions", "lane_slots")] + \
        [("sessions_open", ctypes.c_longlong), ("state_bytes_in_use", ctypes.c_size_t),
         ("state_bytes_peak", ctypes.c_size_t), ("state_budget_bytes", ctypes.c_size_t)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class LoadgenConfig(ctypes.Structure):
    """fa_loadgen_config (include/fast_atari.h)."""
    _fields_ = [("clients", ctypes.c_int), ("requests", ctypes.c_int), ("offered_frames_per_s", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("batch_median", ctypes.c_uint32), ("batch_min", ctypes.c_uint32),
                ("batch_max", ctypes.c_uint32), ("batch_sigma", ctypes.c_double), ("k_min", ctypes.c_int),
                ("k_max", ctypes.c_int)]


class LoadgenResult(ctypes.Structure):
    """fa_loadgen_result (include/fast_atari.h)."""
    _fields_ = [("requests", ctypes.c_ulonglong), ("admission_waits", ctypes.c_ulonglong)] + \
        [(n, ctypes.c_double) for n in (
            "instances", "instance_frames", "elapsed_s", "frames_per_s", "steady_frames_per_s", "offered_frames_per_s", "arrival_window_s",
            "p50_ms", "p90_ms", "p99_ms", "max_ms", "mean_ms", "mean_queue_ms", "mean_batch_requests")] + \
        [("errors", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# fa_loadgen_record (include/fast_atari.h).
LOADGEN_RECORD = np.dtype([("cart", "<u4"), ("n", "<u4"), ("k", "<u4"), ("batch_requests", "<u4"),
                           ("arrival_s", "<f8"), ("latency_ms", "<f8"), ("session_wait_ms", "<f8"),
                           ("dispatch_ms", "<f8"), ("service_ms", "<f8")])


class AtariServer:
    """Continuous-batching server over several carts (fa_server_*).

    Sessions are instance sets of one cart resident in HBM; `submit` queues a
    step of instances [0, n) of a session for k frames and returns a ticket,
    `wait` returns that request's observations (n x 128 RAM bytes) and timing.
    Thread-safe: ctypes releases the GIL, so clients on several Python threads
    overlap.
    """

    def __init__(self, roms, mode: str = "batched", state_budget_bytes: int = 0, block: int = 0,
                 max_inflight: int = 0, sched="pc"):
        self.roms = [np.frombuffer(bytes(r), dtype=np.uint8).copy() for r in roms]
        cfg = ServerConfig(int(state_budget_bytes), SERVE_PLAIN if mode == "plain" else SERVE_BATCHED,
                           int(block), int(max_inflight), SCHED_NAMES[sched] if isinstance(sched, str) else int(sched))
        ptrs = (_vp * len(self.roms))(*[r.ctypes.data for r in self.roms])
        lens = (ctypes.c_size_t * len(self.roms))(*[len(r) for r in self.roms])
        h = _vp()
        _check(lib().fa_server_create(ptrs, lens, len(self.roms), ctypes.byref(cfg), ctypes.byref(h)))
        self._s = h
        self._held = {}           # ticket -> (actions, obs) kept alive until waited

    def close(self) -> None:
        if getattr(self, "_s", None):
            lib().fa_server_destroy(self._s)
            self._s = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def open(self, cart: int) -> int:
        sid = ctypes.c_int64()
        _check(lib().fa_server_open(self._s, int(cart), ctypes.byref(sid)))
        return sid.value

    def close_session(self, session: int) -> None:
        _check(lib().fa_server_close(self._s, int(session)))

    def submit(self, session: int, actions, n: int, k: int, obs: bool = True) -> int:
        a = np.ascontiguousarray(actions, dtype=np.uint8).reshape(-1)
        if a.size != n * k:
            raise ValueError("actions must hold k * n bytes")
        out = np.empty((n, 128), np.uint8) if obs else None
        t = ctypes.c_uint64()
        _check(lib().fa_server_submit(self._s, int(session), a.ctypes.data, int(n), int(k),
                                      out.ctypes.data if obs else None, ctypes.byref(t)))
        self._held[t.value] = (a, out)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(observations or None, info dict); raises FaError on failure."""
        info = RequestInfo()
        rc = lib().fa_server_wait(self._s, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(info))
        if rc == FA_ERR_TIMEOUT:
            raise FaError(rc, lib().fa_last_error().decode())
        _, out = self._held.pop(ticket, (None, None))
        _check(rc)
        return out, info.as_dict()

    def step(self, session: int, actions, n: int, k: int):
        return self.wait(self.submit(session, actions, n, k))

    def session_size(self, session: int) -> int:
        v = _u32()
        _check(lib().fa_server_session_size(self._s, int(session), ctypes.byref(v)))
        return v.value

    def states(self, session: int, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        if count is None:
            count = self.session_size(session) - first
        out = np.zeros(count, dtype=STATE_DTYPE)
        _check(lib().fa_server_get_states(self._s, int(session), int(first), int(count), out.ctypes.data))
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().fa_server_stats_get(self._s, ctypes.byref(st)))
        return st.as_dict()

    def loadgen(self, requests: int, offered_frames_per_s: float, clients: int = 64, seed: int = 1,
                batch_median: int = 256, batch_min: int = 16, batch_max: int = 16384, batch_sigma: float = 1.0,
                k_min: int = 1, k_max: int = 8):
        """Run the simulated actor clients; returns (result dict, per-request
        records: a LOADGEN_RECORD structured array in arrival order)."""
        cfg = LoadgenConfig(int(clients), int(requests), float(offered_frames_per_s), int(seed), int(batch_median),
                            int(batch_min), int(batch_max), float(batch_sigma), int(k_min), int(k_max))
        res = LoadgenResult()
        rec = np.zeros(int(requests), LOADGEN_RECORD)
        _check(lib().fa_server_loadgen(self._s, ctypes.byref(cfg), ctypes.byref(res), rec.ctypes.data))
        return res.as_dict(), rec


# ------------------------------------------------------------------ rendering
FB_H, FB_W = 192, 160


class AtariRender:
    """The rendering console (src/atari.rs:107-306, src/tia.rs) for n consoles
    of one ROM: each frame also renders a 160 x 192 framebuffer of NTSC
    palette indices (Atari::framebuffer), kept on the device."""

    def __init__(self, rom: bytes, n: int, cta_warps: int = 16, sched="pc"):
        r = np.frombuffer(bytes(rom), dtype=np.uint8).copy()
        h = _vp()
        _check(lib().fa_render_create(_u8(r), len(r), int(n), ctypes.byref(h)))
        self._r = h
        self.n = int(n)
        _check(lib().fa_render_set_launch(h, int(cta_warps), SCHED_NAMES[sched] if isinstance(sched, str) else int(sched)))

    def close(self) -> None:
        if getattr(self, "_r", None):
            lib().fa_render_destroy(self._r)
            self._r = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def reset(self):
        """(framebuffers [n, 192, 160], RAM [n, 128]) after new + one frame."""
        fb = np.empty((self.n, FB_H, FB_W), np.uint8)
        ram = np.empty((self.n, 128), np.uint8)
        _check(lib().fa_render_reset(self._r, fb.ctypes.data, ram.ctypes.data))
        return fb, ram

    def step_multi(self, actions, k: int, fb: bool = True, out=None):
        """k frames; returns (framebuffers (n, 192, 160) or None, RAM (n, 128)).
        `out`: the caller's (framebuffers, RAM) uint8 arrays to fill instead of
        new ones (framebuffers may be None when fb is False)."""
        a = np.ascontiguousarray(actions, dtype=np.uint8).reshape(-1)
        if a.size != k * self.n:
            raise ValueError(f"expected {k}*{self.n} actions, got {a.size}")
        if out is not None:
            fbo, ram = out
            fbo = fbo if fb else None
            wanted = [(ram, self.n * 128)] + ([(fbo, self.n * FB_H * FB_W)] if fb else [])
            for arr, size in wanted:
                if not (isinstance(arr, np.ndarray) and arr.dtype == np.uint8 and arr.size == size
                        and arr.flags.c_contiguous and arr.flags.writeable):
                    raise ValueError("outputs must be writable C-contiguous uint8 arrays of the right size")
        else:
            fbo = np.empty((self.n, FB_H, FB_W), np.uint8) if fb else None
            ram = np.empty((self.n, 128), np.uint8)
        _check(lib().fa_render_step_multi(self._r, _u8(a), int(k), fbo.ctypes.data if fb else None, ram.ctypes.data))
        return fbo, ram

    def step_multi_async(self, d_actions: int, k: int, d_obs: int = 0, stream: int = 0) -> None:
        _check(lib().fa_render_step_multi_async(self._r, _vp(d_actions), int(k), _vp(d_obs or None), _vp(stream or None)))

    def synchronize(self) -> None:
        _check(lib().fa_render_synchronize(self._r))

    def rgba(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        """Atari::render of consoles [first, first + count): (count, 192, 160, 4)
        uint8 RGBA, converted on the device."""
        if count is None:
            count = self.n - first
        out = np.empty((count, FB_H, FB_W, 4), np.uint8)
        _check(lib().fa_render_get_rgba(self._r, int(first), int(count), out.ctypes.data))
        return out

    def rgba_async(self, first: int, count: int, d_rgba: int, stream: int = 0) -> None:
        _check(lib().fa_render_rgba_async(self._r, int(first), int(count), _vp(d_rgba), _vp(stream or None)))

    def framebuffers(self) -> np.ndarray:
        out = np.empty((self.n, FB_H, FB_W), np.uint8)
        _check(lib().fa_render_get_framebuffers(self._r, out.ctypes.data))
        return out

    def device_framebuffers(self) -> int:
        return int(lib().fa_render_device_framebuffers(self._r) or 0)

    def states(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=STATE_DTYPE)
        _check(lib().fa_render_get_states(self._r, out.ctypes.data))
        return out

    def last_instructions(self) -> int:
        return int(lib().fa_render_last_instructions(self._r))
