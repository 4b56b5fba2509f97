"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU calls)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(apollo_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("apollo_dg_create", "apollo_dg_set_mesh", "apollo_dg_rhs", "apollo_dg_step", "apollo_dg_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from apollo_b200.dg import LIB_PATH
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_declares_every_symbol():
    from apollo_b200 import dg
    lib = dg.load_library()
    for n in declared_symbols():
        fn = getattr(lib, n)
        assert fn.argtypes is not None, n


def test_create_rejects_bad_config_without_gpu():
    """Argument checks happen before any CUDA call."""
    from apollo_b200 import dg
    lib = dg.load_library()
    h = ctypes.c_void_p()
    cfg = dg._Config(9, 0.5, 0, None)
    assert lib.apollo_dg_create(ctypes.byref(cfg), ctypes.byref(h)) == 1  # APOLLO_ERR_CONFIG
    cfg = dg._Config(3, -1.0, 0, None)
    assert lib.apollo_dg_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert lib.apollo_dg_create(None, ctypes.byref(h)) == 8  # APOLLO_ERR_ARG
