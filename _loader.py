"""Import helper for the package directory `midnight-zk_b200/`.

Its name is not a Python identifier, so it is loaded from its path under the
module name `mzk_b200`.
"""
import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "midnight-zk_b200"


def load():
    if "mzk_b200" in sys.modules:
        return sys.modules["mzk_b200"]
    spec = importlib.util.spec_from_file_location(
        "mzk_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mzk_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
