"""The C-ABI library loads and exports every entry point declared in include/*.h."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(gfnff_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_api():
    names = declared_functions()
    for required in ["gfnff_create", "gfnff_setup", "gfnff_energy_and_gradient", "gfnff_destroy",
                     "gfnff_last_error", "gfnff_charges", "gfnff_get_topology"]:
        assert required in names


def test_library_exports_every_declared_symbol(built_library):
    lib = ctypes.CDLL(str(built_library))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_declared_symbols():
    from curcuma_b200 import _lib
    assert set(_lib.EXPORTED) <= set(declared_functions())
