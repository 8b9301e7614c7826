"""Import helper: the package directory is named `fast-atari-rs_b200`, which
is not a Python identifier, so it is loaded under the name `fast_atari_b200`."""
import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "fast-atari-rs_b200"


def load():
    if "fast_atari_b200" in sys.modules:
        return sys.modules["fast_atari_b200"]
    spec = importlib.util.spec_from_file_location(
        "fast_atari_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["fast_atari_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


fa = load()
import fast_atari_b200.carts as carts  # noqa: E402
