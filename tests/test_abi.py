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


def test_batch_device_bytes_estimate():
    """ud_batch_device_bytes (host-only) counts what a batch allocates: it
    grows with the ligands and the chains, AD4 adds charges and pair
    coefficients, and one rigid ligand at exhaustiveness 1 is the sum of its
    buffers (each with a quarter of headroom)."""
    from unidock_tools import synth
    ligs = [engine.Ligand(synth.make_ligand(12 + 6 * k, k, seed=300 + k).to_pdbqt()) for k in range(6)]
    b = [engine.batch_device_bytes(ligs[:n], exhaustiveness=64) for n in range(1, 7)]
    assert all(x < y for x, y in zip(b, b[1:]))
    assert engine.batch_device_bytes(ligs, exhaustiveness=128) > engine.batch_device_bytes(ligs, exhaustiveness=64)
    assert engine.batch_device_bytes(ligs, sf=engine.SF_AD4) > engine.batch_device_bytes(ligs, sf=engine.SF_VINA)
    one = engine.Ligand(synth.make_ligand(2, 0, seed=5).to_pdbqt())   # 2 atoms, 1 node, no pairs
    h = lambda n, size: max(n + n // 4, 1) * size
    expect = (h(1, 48) + h(2, 16) + h(1, 40) + h(0, 4) + h(2, 4) + h(1, 4)          # topology, order
              + h(7, 4) + h(1, 24) + h(1, 4)                                         # chain results, queue
              + h(9 * 3 * 2, 4) + h(1, 4) + 2 * h(9, 4) + h(9 * 7, 4) + h(36, 4))    # modes
    assert engine.batch_device_bytes([one], exhaustiveness=1, num_modes=9) == expect
    with __import__("pytest").raises(engine.UdError):
        engine.batch_device_bytes(ligs, sf=7)


def _header_struct_fields(name):
    """Field names, in order, of `typedef struct { ... } name;` in include/unidock_b200.h."""
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parent.parent / "include" / "unidock_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct \{([^}]*)\}\s*" + name + r"\s*;", text).group(1)
    return [re.match(r"\s*[\w\s]+?\b(\w+)\s*$", decl).group(1) for decl in body.split(";") if decl.strip()]


def test_python_structs_match_the_header():
    """The ctypes mirrors of the ABI's parameter structs list the header's
    fields in the header's order (a field added on one side only would shift
    every field after it)."""
    assert [f for f, _ in engine.SearchParams._fields_] == _header_struct_fields("ud_search_params")
    assert [f for f, _ in engine.TuneResult._fields_] == _header_struct_fields("ud_tune_result")
