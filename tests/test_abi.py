"""The C-ABI library loads and exports every entry point include/unidock_b200.h declares."""
import ctypes

from unidock_tools import engine


def test_library_exports_all_declared_symbols():
    L = engine.lib()
    names = engine.exported_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert L.ud_version() >= 100


def test_errors_are_codes_not_exceptions():
    L = engine.lib()
    h = ctypes.c_void_p()
    bad = b"ATOM  garbage\n"
    rc = L.ud_ligand_parse(bad, len(bad), ctypes.byref(h))
    assert rc == 2
    assert L.ud_last_error()
    rc = L.ud_batch_create(None, None, 0, None, ctypes.byref(h))
    assert rc == 1
