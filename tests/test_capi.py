"""C ABI: the library loads and exports every function include/*.h declares
(no compute calls here -- those need a GPU)."""
import ctypes
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", text):
            name = m.group(1)
            if name not in {"if", "while", "for", "return", "sizeof"}:
                names.add(name)
    return sorted(names)


def test_header_declares_reference_surface():
    names = declared_functions()
    for required in ["csr2tile_row_major", "csr2tile_col_major", "tilespgemm", "tile2csr", "matrix_destroy",
                     "apply_bipermutation_csr", "restore_bipermutation_csr", "build_original_reorder_plan",
                     "build_external_reorder_plan"]:
        assert required in names


def test_library_exports_every_declared_symbol(tsg):
    lib = tsg.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_library_is_sm100a_build(tsg):
    data = tsg.LIB_PATH.read_bytes()
    assert b"sm_100a" in data or b"sm_100" in data


def test_cli_binary_prints_usage_without_gpu():
    import subprocess
    out = subprocess.run([str(ROOT / "rw-spgemm_b200" / "bin" / "test"), "-d", "0"], capture_output=True, text=True,
                         timeout=60)
    assert out.returncode == 0 and "Run the code by './test -d 0 -aat 0 matrixA.mtx" in out.stdout


def test_overlap_wrapper_grows_buffers_and_retries(tsg, monkeypatch):
    """spgemm_csr_host_overlap: a first call whose buffers are too small gets
    TSG_ERR_OVERFLOW with nnz(C); the wrapper grows the buffers (keeping them
    pageable) and calls again (host logic only, through a stand-in library)."""
    calls = []

    class FakeLib:
        def tsg_spgemm_csr_host_into(self, ctx, m, k, n, nnzA, arp, aci, av, nnzB, brp, bci, bv, crp, cci, cv, cap,
                                     p_nnz, p_info):
            calls.append(cap)
            p_nnz._obj.value = 5
            if cap < 5:
                return tsg.TSG_ERR_OVERFLOW
            (ctypes.c_int * (m + 1)).from_address(crp)[:] = [0, 2, 3, 5]
            (ctypes.c_int * 5).from_address(cci)[:] = [0, 2, 1, 0, 2]
            (ctypes.c_double * 5).from_address(cv)[:] = [1.0, 2.0, 3.0, 4.0, 5.0]
            return 0

    monkeypatch.setattr(tsg, "lib", lambda: FakeLib())

    class Ctx:
        handle = None

    mat = (3, 3, np.array([0, 1, 2, 3], np.int32), np.array([0, 1, 2], np.int32), np.ones(3))
    out = tsg.HostResultBuffers(3, 2, pinned=False)
    (m, n, rp, ci, v), info = tsg.spgemm_csr_host_overlap(Ctx(), mat, None, out)
    assert calls == [2, 5] and out.cap == 5 and out.pinned is False
    assert list(rp) == [0, 2, 3, 5] and list(ci) == [0, 2, 1, 0, 2] and list(v) == [1.0, 2.0, 3.0, 4.0, 5.0]


def test_bench_byte_accounting_matches_the_documented_figures():
    """The roofline's byte counts: compulsory bytes (tiled A and B read, tiled
    C written) and the numeric step's algorithmic bytes, from the tile and
    nonzero counts of the stencil 64^3 product (the bench line's 528,497,108
    and 505,262,028) and of the 5-point Laplacian 256^2 product (18.99 MB)."""
    import importlib.util
    from types import SimpleNamespace as NS
    spec = importlib.util.spec_from_file_location("bench_for_bytes", ROOT / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)

    def tiled(tilem, tilen, T, nnz):
        return NS(s=NS(tilem=tilem, tilen=tilen), numtile=T, nnz=nnz)

    A = tiled(16384, 16384, 361_000, 6_859_000)
    assert b.compulsory_bytes(A, A, 1_380_344, 30_959_144) == 528_497_108
    assert b.step3_algorithmic_bytes(A, A, 1_380_344, 30_959_144) == 505_262_028
    L = tiled(4096, 4096, 19_936, 326_656)
    assert b.compulsory_bytes(L, L, 50_532, 846_852) == 18_991_280
