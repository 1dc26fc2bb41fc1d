"""C ABI: the library loads and exports every function include/*.h declares
(no compute calls here -- those need a GPU)."""
import ctypes
import re
from pathlib import Path

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
