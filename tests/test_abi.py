"""The C-ABI library loads and exports every symbol the public header declares.

No compute call is made here (these tests run without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rumd_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^B2MD_API\s+[\w\s\*]+?\b(b2md_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_symbols():
    names = declared()
    assert len(names) >= 30
    assert "b2md_run" in names and "b2md_calc_f" in names


def test_library_exports_every_declared_symbol():
    from rumd_b200 import build, capi
    build.build_lib()
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from rumd_b200 import capi
    assert sorted(capi.EXPORTS) == declared()


def test_error_reporting_without_gpu():
    """Argument validation happens before any device work."""
    from rumd_b200 import capi
    lib = capi.lib()
    h = ctypes.c_void_p()
    # RUMD's shapes (pb 16..192, tp up to 64) are mapped, not refused; only
    # shapes outside pb 1..1024, tp 1..64 are rejected
    rc = lib.b2md_engine_create(0, 0, 1, 0, 0, 4, ctypes.byref(h))
    assert rc == capi.B2MD_ERR_ARG
    assert b"pb" in lib.b2md_last_error()
    rc = lib.b2md_engine_create(0, 0, 1, 0, 64, 65, ctypes.byref(h))
    assert rc == capi.B2MD_ERR_ARG
    assert lib.b2md_version().startswith(b"rumd_b200")
    # a null engine is rejected before any device work
    assert lib.b2md_engine_set_variant(None, capi.VARIANT_BUILD_LANES, 4) == capi.B2MD_ERR_ARG
    v = ctypes.c_int()
    assert lib.b2md_engine_get_variant(None, capi.VARIANT_BUILD_LANES, ctypes.byref(v)) == capi.B2MD_ERR_ARG
