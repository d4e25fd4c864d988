"""The C-ABI library loads without a GPU and exports every entry point the header declares."""
import ctypes
import glob
import os
import re

from philip_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(ph_\w+)\s*\(", text, flags=re.M))
    return names


def test_header_declares_the_abi():
    names = declared_symbols()
    assert {"ph_ctx_create", "ph_residual", "ph_rk_step", "ph_apply_inverse_mass", "ph_integrals",
            "ph_residual_noalloc"} <= names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) == declared_symbols()


def test_errors_without_a_device_are_reported_not_raised():
    L = _lib.load()
    assert L.ph_ctx_create(None, None, None, None) == 1
    assert b"null argument" in L.ph_last_error()
