"""bench.py's workload table, without a GPU: every name the command line takes
for the batched core resolves to carts, instance counts and K, and the carts
of the scheme workloads resolve to their schemes through the library's own
registry (DPC by length, FE and E0/3F as registered for the run)."""
import sys

import pytest

from fa_pkg import ROOT, carts, fa

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402

BATCHED = ["mixed", "divergence", "plain", "converged", "scale", "mappers", "dpc", "fe"]


@pytest.mark.parametrize("name", BATCHED)
def test_workload_resolves(name):
    desc, spec, k, episode = bench.workload(name, carts)
    assert desc and k >= 1 and episode >= 0
    assert spec and all(n >= 1 and len(c.rom) > 0 for c, n in spec)


@pytest.mark.parametrize("name,schemes", [("dpc", {6}), ("fe", {7}), ("mappers", {4, 5})])
def test_scheme_workloads_reach_their_schemes(name, schemes):
    _, spec, _, _ = bench.workload(name, carts)
    got = set()
    for c, _ in spec:
        if c.scheme:
            fa.set_rom_scheme(c.rom, c.scheme)
        try:
            got.add(fa.rom_scheme(c.rom))
        finally:
            if c.scheme:
                fa.set_rom_scheme(c.rom, "auto")
    assert got == schemes


def test_unknown_workload_is_refused():
    with pytest.raises(SystemExit):
        bench.workload("no-such-workload", carts)
