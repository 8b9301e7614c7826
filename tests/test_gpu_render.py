"""GPU parity of the rendering console (src/atari.rs:107-306, src/tia.rs).

Every console's framebuffer (160 x 192 palette indices), RAM, CPU registers,
cycle counter and TIA registers after each call equal the CPU oracle's
restatement of the rendering console, bit for bit: on the rendering cart
(every graphics register, mid-line writes, HMOVE, collisions, input latches),
on the divergence cart (F8 bank switching, no WSYNC) and on the 32K F4 cart.
The rendering oracle is unpinned: the reference's own rendering checks need
Breakout.bin or the Gopher2600 tool, and neither is available."""
import numpy as np
import pytest

import oracle
from fa_pkg import carts, fa

pytestmark = pytest.mark.gpu

TIA_FIELDS = ["colup0", "colup1", "colupf", "colubk", "ctrlpf", "refp0", "refp1", "pf0", "pf1", "pf2",
              "grp0", "grp1", "grp0_old", "grp1_old", "enam0", "enam1", "enabl", "enabl_old",
              "hmp0", "hmp1", "hmm0", "hmm1", "hmbl", "nusiz0", "nusiz1", "vdelp0", "vdelp1", "vdelbl",
              "resmp0", "resmp1", "pos_p0", "pos_p1", "pos_m0", "pos_m1", "pos_bl",
              "cxm0p", "cxm1p", "cxp0fb", "cxp1fb", "cxm0fb", "cxm1fb", "cxblpf", "cxppmm",
              "paddle0", "paddle1", "paddle_counter", "paddle_dumped", "inpt4", "inpt5"]


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    if fa.device_count() < 1:
        pytest.skip("no CUDA device")


def check(gpu_fb, gpu_ram, gpu_st, consoles, what):
    for i, c in enumerate(consoles):
        t = c.tia_record()
        assert np.array_equal(gpu_fb[i], t["fb"]), f"{what}: framebuffer of console {i}, " \
            f"{int((gpu_fb[i] != t['fb']).sum())} pixels differ, first at {np.argwhere(gpu_fb[i] != t['fb'])[0].tolist()}"
        assert np.array_equal(gpu_ram[i], c.ram()), f"{what}: RAM of console {i}"
        r = c.regs()
        s = gpu_st[i]
        got = [int(s["a"]) | int(s["x"]) << 8 | int(s["y"]) << 16 | int(s["sp"]) << 24,
               int(s["pc"]) | int(s["status"]) << 16 | int(s["bank"]) << 24,
               int(s["cycles"]) & 0xFFFFFFFF, int(s["cycles"]) >> 32,
               int(s["tia_clock"]) | int(s["tia_scanline"]) << 16, int(s["frame_no"]), int(s["run_status"]),
               int(s["timer_value"]) | int(s["timer_prescaler"]) << 16]
        want = [int(v) for v in r]
        want[5] -= 1                       # the library's frame counter restarts after the reset frame
        assert got == want, f"{what}: registers of console {i}: gpu {got} oracle {want}"
        for f in TIA_FIELDS:
            assert int(s[f]) == int(t[f]), f"{what}: {f} of console {i}: gpu {int(s[f])} oracle {int(t[f])}"
        assert int(s["tia_vsync"]) == int(t["vsync"]) and int(s["tia_vblank"]) == int(t["vblank"]), what


@pytest.mark.parametrize("name", ["render", "divergence", "mixed_32k"])
def test_render_matches_oracle(name):
    rom = {"render": carts.render_cart, "divergence": carts.divergence_cart,
           "mixed_32k": lambda: carts.mixed_carts()[3]}[name]().rom
    n, calls, k = 40, 3, 4
    consoles = oracle.render_reset(rom, n)
    with fa.AtariRender(rom, n) as g:
        fb, ram = g.reset()
        check(fb, ram, g.states(), consoles, f"{name} reset")
        for c in range(calls):
            acts = carts.actions(seed=60 + c, n=n, frames=k)
            fb, ram = g.step_multi(acts, k)
            oracle.render_steps(consoles, acts)
            check(fb, ram, g.states(), consoles, f"{name} call {c}")


@pytest.mark.parametrize("warps,sched", [(4, "lane"), (16, "line")])
def test_render_launch_shapes_and_policies(warps, sched):
    rom = carts.render_cart().rom
    n, k = 70, 5                                    # a partial warp
    acts = carts.actions(seed=71, n=n, frames=k)
    consoles = oracle.render_reset(rom, n)
    oracle.render_steps(consoles, acts)
    with fa.AtariRender(rom, n, cta_warps=warps, sched=sched) as g:
        g.reset()
        fb, ram = g.step_multi(acts, k)
        check(fb, ram, g.states(), consoles, f"{warps} warps, {sched}")


def test_render_frames_are_pictures_and_depend_on_actions():
    rom = carts.render_cart().rom
    n, k = 64, 6
    with fa.AtariRender(rom, n) as g:
        g.reset()
        fb, _ = g.step_multi(carts.actions(seed=5, n=n, frames=k), k)
    assert (fb != 0).sum(axis=(1, 2)).min() > 1000                 # every console drew something
    assert len(np.unique(fb)) > 8                                    # several colours
    assert len({fb[i].tobytes() for i in range(n)}) >= 4             # the actions show in the pictures


def test_render_large_batch_copy_out():
    # 1,500 framebuffers (46 MB) leave the device through the pipelined copy
    # (several host threads with pinned chunks, uneven shares, a short last
    # chunk); every byte must land where the oracle puts it.
    rom = carts.render_cart().rom
    n, k = 1500, 2
    acts = carts.actions(seed=91, n=n, frames=k)
    consoles = oracle.render_reset(rom, n)
    oracle.render_steps(consoles, acts)
    with fa.AtariRender(rom, n) as g:
        g.reset()
        fb, ram = g.step_multi(acts, k)
        assert np.array_equal(g.framebuffers(), fb)
        check(fb, ram, g.states(), consoles, "1500 consoles")


def test_rgba_output_matches_oracle_render():
    """Atari::render on the device: fa_render_get_rgba (host buffer, converted
    a chunk at a time on the GPU) and fa_render_rgba_async (device buffer)
    equal the oracle's RGBA of its own framebuffers."""
    import torch
    rom = carts.render_cart().rom
    n = 37
    consoles = oracle.render_reset(rom, n)
    with fa.AtariRender(rom, n) as g:
        g.reset()
        acts = carts.actions(seed=12, n=n, frames=2)
        g.step_multi(acts, 2)
        oracle.render_steps(consoles, acts)
        want = oracle.rgba(np.stack([c.tia_record()["fb"] for c in consoles]))
        got = g.rgba()
        assert got.shape == (n, 192, 160, 4)
        assert np.array_equal(got, want.reshape(got.shape))
        part = g.rgba(5, 9)
        assert np.array_equal(part, got[5:14])
        d = torch.empty(9 * 192 * 160 * 4, dtype=torch.uint8, device="cuda")
        g.rgba_async(5, 9, d.data_ptr())
        g.synchronize()
        assert np.array_equal(d.cpu().numpy().reshape(part.shape), part)
        with pytest.raises(fa.FaError):
            g.rgba(30, 8)


def test_render_fills_caller_arrays():
    """AtariRender.step_multi(out=...): framebuffers and RAM land in the
    caller's arrays, call after call, equal to the oracle's."""
    rom = carts.render_cart().rom
    n, k = 24, 2
    consoles = oracle.render_reset(rom, n)
    fb_out = np.full((n, 192, 160), 0xAB, np.uint8)
    ram_out = np.full((n, 128), 0xCD, np.uint8)
    with fa.AtariRender(rom, n) as g:
        g.reset()
        for c in range(2):
            acts = carts.actions(seed=90 + c, n=n, frames=k)
            fb, ram = g.step_multi(acts, k, out=(fb_out, ram_out))
            assert fb is fb_out and ram is ram_out
            oracle.render_steps(consoles, acts)
            check(fb_out, ram_out, g.states(), consoles, f"caller arrays, call {c}")
        with pytest.raises(ValueError):
            g.step_multi(acts, k, out=(fb_out[:1], ram_out))
