"""Shared pytest setup: the `gpu` marker and import paths.

`-m "not gpu"` runs the oracle checks, host logic and ABI checks on CPU;
`-m gpu` runs the CUDA parity tests through the C ABI on a B200.
"""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "oracle", ROOT / "tests", ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
