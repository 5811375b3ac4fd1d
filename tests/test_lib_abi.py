"""CPU checks of the C ABI: the library loads and exports every declared symbol."""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "dogpup_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgp_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    import ctypes
    from dogpup_b200 import _lib
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_the_header():
    from dogpup_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.DECLARED)


def test_reference_named_dropins_are_exported():
    import subprocess
    from dogpup_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", str(_lib.LIB_PATH)], capture_output=True,
                         text=True).stdout
    for name in ("smv_call(", "FSAImv_call(", "FSAIP_call("):
        assert name in out, name


def test_status_strings_and_defaults_without_a_gpu():
    from dogpup_b200 import _lib
    assert _lib.lib.dgp_status_string(5).decode() == "not converged"
    o = _lib.default_opts()
    assert o.tol == 1e-12 and o.maxit == 1000 and o.fsai_cap == 30   # dMesh.m:1243, :1363
