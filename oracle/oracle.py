"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/libtsg_oracle.so (the plain-C restatement) and, when present,
oracle/_ref/libtsgref.so (the reference's own CPU code compiled from its
sources).  Used by tests/, the smoke check and bench.py's CPU-baseline leg as
the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libtsg_oracle.so"
REF_SO = HERE / "_ref" / "libtsgref.so"

_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_ubyte)
_u16p = ctypes.POINTER(ctypes.c_ushort)


class OMatrix(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_int), ("n", ctypes.c_int), ("nnz", ctypes.c_int), ("isSymmetric", ctypes.c_int),
        ("value", _dp), ("columnindex", _ip), ("rowpointer", _ip),
        ("tilem", ctypes.c_int), ("tilen", ctypes.c_int),
        ("tile_ptr", _ip), ("tile_columnidx", _ip), ("tile_rowidx", _ip),
        ("tile_nnz", _ip), ("numtile", ctypes.c_int),
        ("tile_csr_Value", _dp), ("tile_csr_Col", _u8p), ("tile_csr_Ptr", _u8p),
        ("mask", _u16p), ("csc_tile_ptr", _ip), ("csc_tile_rowidx", _ip),
    ]


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]
_o = None
_r = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def olib():
    global _o
    if _o is None:
        if not ORACLE_SO.exists():
            build()
        _o = ctypes.CDLL(str(ORACLE_SO))
        vp = ctypes.c_void_p
        _o.tsgo_count_products.restype = ctypes.c_longlong
        _o.tsgo_count_products.argtypes = [ctypes.c_int, vp, vp]
        _o.tsgo_gustavson_symbolic.restype = ctypes.c_longlong
        _o.tsgo_gustavson_symbolic.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int]
        _o.tsgo_gustavson_row_nnz.restype = ctypes.c_longlong
        _o.tsgo_gustavson_row_nnz.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int]
        _o.tsgo_gustavson_numeric.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                              ctypes.c_int]
        _o.tsgo_order_degree.argtypes = [ctypes.c_int, vp, vp]
        _o.tsgo_order_random.argtypes = [ctypes.c_int, ctypes.c_ulonglong, vp]
        _o.tsgo_order_rcm.argtypes = [ctypes.c_int, vp, vp, vp]
        _o.tsgo_order_gray.argtypes = [ctypes.c_int, ctypes.c_int, vp, vp, vp]
        _o.tsgo_apply_bipermutation.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    return _o


def ref_available() -> bool:
    return REF_SO.exists()


def rlib():
    global _r
    if _r is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (reference tree absent when oracle/Makefile ran)")
        _r = ctypes.CDLL(str(REF_SO))
        vp = ctypes.c_void_p
        _r.ref_spgemm_spa_rowptr.restype = ctypes.c_int
        _r.ref_spgemm_spa_rowptr.argtypes = [ctypes.c_int] * 3 + [vp, vp] + [ctypes.c_int] * 3 + [vp, vp, vp]
        _r.ref_spgemm_spa_cols.argtypes = [ctypes.c_int] * 3 + [vp, vp] + [ctypes.c_int] * 3 + [vp, vp, vp, vp]
        _r.ref_omp_max_threads.restype = ctypes.c_int
    return _r


def _arr(ptr, count, dtype, free=False):
    if count <= 0 or not ptr:
        out = np.zeros(0, dtype=dtype)
    else:
        addr = ctypes.cast(ptr, ctypes.c_void_p).value
        buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(addr)
        out = np.frombuffer(buf, dtype=dtype).copy()
    if free and ptr:
        _libc.free(ctypes.cast(ptr, ctypes.c_void_p))
    return out


class _CSRHold:
    def __init__(self, mat):
        m, n, rp, ci, v = mat
        self.rp = np.ascontiguousarray(rp, dtype=np.int32)
        self.ci = np.ascontiguousarray(ci, dtype=np.int32)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        self.om = OMatrix()
        self.om.m, self.om.n, self.om.nnz = int(m), int(n), int(self.ci.size)
        self.om.rowpointer = self.rp.ctypes.data_as(_ip)
        self.om.columnindex = self.ci.ctypes.data_as(_ip)
        self.om.value = self.v.ctypes.data_as(_dp)


def _tiles(om: OMatrix, colmajor=False, free=True, rowidx=True):
    T, nnz = om.numtile, om.nnz
    d = dict(m=om.m, n=om.n, nnz=nnz, tilem=om.tilem, tilen=om.tilen, numtile=T)
    d["tile_ptr"] = _arr(om.tile_ptr, om.tilem + 1, np.int32, free)
    d["tile_columnidx"] = _arr(om.tile_columnidx, T, np.int32, free)
    d["tile_rowidx"] = _arr(om.tile_rowidx, T, np.int32, free) if rowidx else None
    d["tile_nnz"] = _arr(om.tile_nnz, T + 1, np.int32, free)
    d["tile_csr_Ptr"] = _arr(om.tile_csr_Ptr, 16 * T, np.uint8, free)
    d["tile_csr_Col"] = _arr(om.tile_csr_Col, nnz, np.uint8, free)
    d["tile_csr_Value"] = _arr(om.tile_csr_Value, nnz, np.float64, free)
    d["mask"] = _arr(om.mask, 16 * T, np.uint16, free) if om.mask else None
    if colmajor:
        d["csc_tile_ptr"] = _arr(om.csc_tile_ptr, om.tilen + 1, np.int32, free)
        d["csc_tile_rowidx"] = _arr(om.csc_tile_rowidx, T, np.int32, free)
    return d


def _om_from_tiles(d):
    hold = {k: np.ascontiguousarray(v) for k, v in d.items() if isinstance(v, np.ndarray)}
    om = OMatrix()
    for k in ("m", "n", "nnz", "tilem", "tilen", "numtile"):
        setattr(om, k, int(d[k]))
    types = dict(tile_ptr=_ip, tile_columnidx=_ip, tile_rowidx=_ip, tile_nnz=_ip, tile_csr_Ptr=_u8p,
                 tile_csr_Col=_u8p, tile_csr_Value=_dp, mask=_u16p, csc_tile_ptr=_ip, csc_tile_rowidx=_ip)
    for k, t in types.items():
        if k in hold:
            setattr(om, k, hold[k].ctypes.data_as(t))
    return om, hold


# --- oracle restatement -----------------------------------------------------
def csr2tile_row_major(mat):
    h = _CSRHold(mat)
    olib().tsgo_csr2tile_row_major(ctypes.byref(h.om))
    return _tiles(h.om)


def csr2tile_col_major(mat):
    h = _CSRHold(mat)
    olib().tsgo_csr2tile_col_major(ctypes.byref(h.om))
    return _tiles(h.om, colmajor=True)


def spgemm_tiled(tA, tB):
    omA, hA = _om_from_tiles(tA)
    omB, hB = _om_from_tiles(tB)
    omC = OMatrix()
    olib().tsgo_spgemm_tiled(ctypes.byref(omA), ctypes.byref(omB), ctypes.byref(omC))
    return _tiles(omC)


def tile2csr(tiles):
    om, hold = _om_from_tiles(tiles)
    olib().tsgo_tile2csr(ctypes.byref(om))
    rp = _arr(om.rowpointer, om.m + 1, np.int32, True)
    ci = _arr(om.columnindex, om.nnz, np.int32, True)
    v = _arr(om.value, om.nnz, np.float64, True)
    return rp, ci, v


def count_products(matA, matB):
    _, _, _, ciA, _ = matA
    _, _, rpB, _, _ = matB
    ciA = np.ascontiguousarray(ciA, dtype=np.int32)
    rpB = np.ascontiguousarray(rpB, dtype=np.int32)
    return olib().tsgo_count_products(int(ciA.size), ciA.ctypes.data, rpB.ctypes.data)


def gustavson(matA, matB, nthreads=1):
    """Element-level CSR SpGEMM: (m, n, rowptr, col, val)."""
    mA, nA, rpA, ciA, vA = [np.ascontiguousarray(x) if isinstance(x, np.ndarray) else x for x in matA]
    mB, nB, rpB, ciB, vB = [np.ascontiguousarray(x) if isinstance(x, np.ndarray) else x for x in matB]
    rpC = np.zeros(mA + 1, dtype=np.int32)
    nnz = olib().tsgo_gustavson_symbolic(mA, nB, rpA.ctypes.data, ciA.ctypes.data, rpB.ctypes.data,
                                         ciB.ctypes.data, rpC.ctypes.data, nthreads)
    if nnz < 0:
        raise OverflowError("nnz(C) exceeds int32")
    ciC = np.zeros(max(nnz, 1), dtype=np.int32)
    vC = np.zeros(max(nnz, 1), dtype=np.float64)
    olib().tsgo_gustavson_numeric(mA, nB, rpA.ctypes.data, ciA.ctypes.data, vA.ctypes.data, rpB.ctypes.data,
                                  ciB.ctypes.data, vB.ctypes.data, rpC.ctypes.data, ciC.ctypes.data,
                                  vC.ctypes.data, nthreads)
    return mA, nB, rpC, ciC[:nnz], vC[:nnz]


def gustavson_row_nnz(matA, matB, nthreads=1):
    """nnz of every row of C = A*B (int32 per row) and the 64-bit total."""
    mA, nA, rpA, ciA, _ = matA
    mB, nB, rpB, ciB, _ = matB
    rpA, ciA, rpB, ciB = (np.ascontiguousarray(x, dtype=np.int32) for x in (rpA, ciA, rpB, ciB))
    counts = np.zeros(max(mA, 1), dtype=np.int32)
    total = olib().tsgo_gustavson_row_nnz(mA, nB, rpA.ctypes.data, ciA.ctypes.data, rpB.ctypes.data,
                                          ciB.ctypes.data, counts.ctypes.data, nthreads)
    return counts[:mA], int(total)


def order(kind, mat, seed=1):
    m, n, rp, ci, _ = mat
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    out = np.zeros(m, dtype=np.int32)
    L = olib()
    if kind == "original":
        return np.arange(m, dtype=np.int32)
    if kind == "degree":
        L.tsgo_order_degree(m, rp.ctypes.data, out.ctypes.data)
    elif kind == "random":
        L.tsgo_order_random(m, ctypes.c_ulonglong(seed), out.ctypes.data)
    elif kind == "rcm":
        L.tsgo_order_rcm(m, rp.ctypes.data, ci.ctypes.data, out.ctypes.data)
    elif kind == "gray":
        L.tsgo_order_gray(m, n, rp.ctypes.data, ci.ctypes.data, out.ctypes.data)
    else:
        raise ValueError(kind)
    return out


def apply_bipermutation(mat, row_old, col_new):
    m, n, rp, ci, v = mat
    rp = np.ascontiguousarray(rp, dtype=np.int32)
    ci = np.ascontiguousarray(ci, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    row_old = np.ascontiguousarray(row_old, dtype=np.int32)
    col_new = np.ascontiguousarray(col_new, dtype=np.int32)
    orp = np.zeros(m + 1, dtype=np.int32)
    oci = np.zeros(max(ci.size, 1), dtype=np.int32)
    ov = np.zeros(max(ci.size, 1), dtype=np.float64)
    olib().tsgo_apply_bipermutation(m, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, row_old.ctypes.data,
                                    col_new.ctypes.data, orp.ctypes.data, oci.ctypes.data, ov.ctypes.data)
    return m, n, orp, oci[:ci.size], ov[:ci.size]


# --- the reference's own CPU code (compiled from its sources) ----------------
def ref_csr2tile_row_major(mat):
    h = _CSRHold(mat)
    rlib().ref_csr2tile_row_major(ctypes.byref(h.om))
    return _tiles(h.om)


def ref_csr2tile_col_major(mat):
    h = _CSRHold(mat)
    rlib().ref_csr2tile_col_major(ctypes.byref(h.om))
    return _tiles(h.om, colmajor=True)


def ref_spgemm_cpu(tA, tB):
    """Reference spgemm_cpu (src/spgemm-cpu.h:369); C has tile_ptr, tile_columnidx,
    tile_nnz, tile_csr_Ptr/Col/Value, numtile, nnz (no mask, no rowidx)."""
    omA, hA = _om_from_tiles(tA)
    omB, hB = _om_from_tiles(tB)
    omC = OMatrix()
    omC.m, omC.n, omC.tilem, omC.tilen = tA["m"], tB["n"], tA["tilem"], tB["tilen"]
    rlib().ref_spgemm_cpu(ctypes.byref(omA), ctypes.byref(omB), ctypes.byref(omC))
    omC.tilem = tA["tilem"]
    omC.tilen = tB["tilen"]
    omC.m, omC.n = tA["m"], tB["n"]
    return _tiles(omC, rowidx=False)


def ref_tile2csr(tiles):
    om, hold = _om_from_tiles(tiles)
    rlib().ref_tile2csr(ctypes.byref(om))
    rp = _arr(om.rowpointer, om.m + 1, np.int32, True)
    ci = _arr(om.columnindex, om.nnz, np.int32, True)
    v = _arr(om.value, om.nnz, np.float64, True)
    return rp, ci, v


def ref_spgemm_spa(matA, matB):
    """Reference spgemm_spa (src/spgemm_serialref_spa_new.h:7): rowptr, cols."""
    mA, nA, rpA, ciA, _ = matA
    mB, nB, rpB, ciB, _ = matB
    rpA = np.ascontiguousarray(rpA, dtype=np.int32)
    ciA = np.ascontiguousarray(ciA, dtype=np.int32)
    rpB = np.ascontiguousarray(rpB, dtype=np.int32)
    ciB = np.ascontiguousarray(ciB, dtype=np.int32)
    rpC = np.zeros(mA + 2, dtype=np.int32)
    R = rlib()
    nnz = R.ref_spgemm_spa_rowptr(mA, nA, int(ciA.size), rpA.ctypes.data, ciA.ctypes.data, mB, nB, int(ciB.size),
                                  rpB.ctypes.data, ciB.ctypes.data, rpC.ctypes.data)
    ciC = np.zeros(max(nnz, 1), dtype=np.int32)
    R.ref_spgemm_spa_cols(mA, nA, int(ciA.size), rpA.ctypes.data, ciA.ctypes.data, mB, nB, int(ciB.size),
                          rpB.ctypes.data, ciB.ctypes.data, rpC.ctypes.data, ciC.ctypes.data)
    return rpC[:mA + 1], ciC[:nnz]


def intersection_bitmaps(tilesA, tilesB):
    """The driver's intersection bitmaps, src/main.cu:430-465: len =
    ceil(tilen_A / 32) words per A tile row (bit 31 - j % 32 of word j / 32
    for each tile column j) and per B tile column (the same for each of its
    tile rows)."""
    n = (int(tilesA["tilen"]) + 31) // 32

    def build(rows, ptr, idx):
        out = np.zeros((rows, max(n, 1)), dtype=np.uint32)
        for i in range(rows):
            for j in np.asarray(idx[ptr[i]:ptr[i + 1]], dtype=np.int64):
                out[i, j // 32] |= np.uint32(1 << (31 - (j % 32)))
        return out

    return (build(int(tilesA["tilem"]), tilesA["tile_ptr"], tilesA["tile_columnidx"]),
            build(int(tilesB["tilen"]), tilesB["csc_tile_ptr"], tilesB["csc_tile_rowidx"]))


# --- reorder-plan estimators -------------------------------------------------
REF_REORDER_SO = HERE / "_ref" / "libtsgref_reorder.so"
PLAN_SAMPLE_ROWS = 24  # GTSP_PROXY_SAMPLE_ROWS, src/reorder.h:23
_rr = None


class OAxis(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("old_id", _ip), ("new_id", _ip)]


class OReorderInfo(ctypes.Structure):
    """ReorderInfo, src/reorder.h:33-63."""
    _fields_ = [("enabled", ctypes.c_int), ("n", ctypes.c_int), ("row_perm", OAxis), ("inner_perm", OAxis),
                ("col_perm", OAxis)] + \
               [(f, ctypes.c_longlong) for f in ("input_tiles_A_before", "input_tiles_A_after", "input_tiles_B_before",
                                                 "input_tiles_B_after", "estimated_c_tiles_before",
                                                 "estimated_c_tiles_after")] + \
               [(f, ctypes.c_double) for f in ("reorder_time_ms", "signature_time_ms", "tile_profile_time_ms",
                                               "affinity_time_ms", "sort_time_ms", "local_refine_time_ms",
                                               "proxy_time_ms", "permute_time_ms", "risk_input_tile_ratio",
                                               "risk_c_tile_ratio")] + \
               [(f, ctypes.c_int) for f in ("local_refine_window", "proxy_sample_rows", "guard_degraded_to_identity",
                                            "structural_conservative", "shared_symmetric_csr")] + \
               [("mode", ctypes.c_char * 64), ("risk_reason", ctypes.c_char * 128)]


ESTIMATE_FIELDS = ("input_tiles_A_before", "input_tiles_A_after", "input_tiles_B_before", "input_tiles_B_after",
                   "estimated_c_tiles_before", "estimated_c_tiles_after", "risk_input_tile_ratio",
                   "risk_c_tile_ratio")


def ref_reorder_available() -> bool:
    return REF_REORDER_SO.exists()


def rrlib():
    global _rr
    if _rr is None:
        _rr = ctypes.CDLL(str(REF_REORDER_SO))
        vp = ctypes.c_void_p
        for f in ("ref_est_input_tiles",):
            getattr(_rr, f).restype = ctypes.c_longlong
            getattr(_rr, f).argtypes = [vp, vp, vp]
        _rr.ref_est_c_tiles.restype = ctypes.c_longlong
        _rr.ref_est_c_tiles.argtypes = [vp, vp, vp, vp]
        _rr.ref_est_c_tiles_ab.restype = ctypes.c_longlong
        _rr.ref_est_c_tiles_ab.argtypes = [vp, vp, vp, vp, vp]
        _rr.ref_fill_reorder_estimates.argtypes = [ctypes.c_int, vp, vp, vp]
        _rr.ref_build_original_reorder_plan.argtypes = [ctypes.c_int, vp, vp, vp]
        _rr.ref_reorder_info_init.argtypes = [vp]
        _rr.ref_reorder_info_destroy.argtypes = [vp]
        _rr.ref_build_reorder_plan.argtypes = [ctypes.c_int, vp, vp, vp]
    return _rr


class _AxisHold:
    """AxisPermutation of a new -> old permutation (None: identity -> NULL)."""

    def __init__(self, old):
        self.ax = None
        if old is not None:
            self.old = np.ascontiguousarray(old, dtype=np.int32)
            self.new = np.empty_like(self.old)
            self.new[self.old] = np.arange(self.old.size, dtype=np.int32)
            self.ax = OAxis(int(self.old.size), self.old.ctypes.data_as(_ip), self.new.ctypes.data_as(_ip))

    def ref(self):
        return ctypes.byref(self.ax) if self.ax is not None else None


def ref_reorder_estimates(kind, matA, matB, row_old, inner_old, col_old):
    """The reference's fill_reorder_estimates (src/external_reorder.h:143-171)
    for the plan's three axis permutations (new -> old); kind "AA"/"AAT"/"AB"."""
    R = rrlib()
    hA = _CSRHold(matA)
    hB = _CSRHold(matB) if matB is not None else hA
    info = OReorderInfo()
    R.ref_reorder_info_init(ctypes.byref(info))
    axes = [_AxisHold(p) for p in (row_old, inner_old, col_old)]
    info.row_perm, info.inner_perm, info.col_perm = (a.ax for a in axes)
    R.ref_fill_reorder_estimates({"AA": 0, "AAT": 1, "AB": 2}[kind], ctypes.byref(hA.om), ctypes.byref(hB.om),
                                 ctypes.byref(info))
    return {f: getattr(info, f) for f in ESTIMATE_FIELDS}


def _samples(tiles):
    sc = min(tiles, PLAN_SAMPLE_ROWS)
    stride = (tiles + sc - 1) // sc if sc > 0 else 1
    return [s * stride for s in range(sc) if s * stride < tiles]


def _scaled(total, tiles, samples):
    return int(float(total) * float(tiles) / float(samples)) if samples else 0


def _tile_row_cols(mat, tile_row, row_old, col_new):
    """Tile columns (new ids) of the new tile row's rows, src/reorder.h:837-858."""
    m, _, rp, ci, _ = mat
    cols = []
    for new_row in range(tile_row * 16, min(tile_row * 16 + 16, m)):
        old = int(row_old[new_row]) if row_old is not None else new_row
        c = np.asarray(ci[rp[old]:rp[old + 1]], dtype=np.int64)
        cols.append((col_new[c] if col_new is not None else c) // 16)
    return np.unique(np.concatenate(cols)) if cols else np.zeros(0, np.int64)


def _inv(old):
    if old is None:
        return None
    new = np.empty(len(old), dtype=np.int64)
    new[np.asarray(old)] = np.arange(len(old))
    return new


def est_input_tiles(mat, row_old=None, col_old=None):
    """estimate_input_tile_count_biperm, src/reorder.h:785-829: distinct tile
    columns of 24 evenly strided tile rows, scaled to all tile rows."""
    tilem = (mat[0] + 15) // 16
    col_new = _inv(col_old)
    smp = _samples(tilem)
    total = sum(int(_tile_row_cols(mat, t, row_old, col_new).size) for t in smp)
    return _scaled(total, tilem, len(smp))


def est_c_tiles(matA, matB, row_old=None, inner_old=None, col_old=None, ab=True):
    """estimate_symbolic_c_tile_count(_ab), src/reorder.h:890-975: for 24
    strided tile rows of A, the distinct tile columns of the B tile rows its
    tile columns name, scaled.  ab=False is the one-matrix form (B = A, every
    axis counted in A's tile rows)."""
    rows = (matA[0] + 15) // 16
    inner = (matA[1] + 15) // 16 if ab else rows
    inner_new, col_new = _inv(inner_old), _inv(col_old)
    smp = _samples(rows)
    total = 0
    for t in smp:
        marked = set()
        for it in _tile_row_cols(matA, t, row_old, inner_new):
            if 0 <= it < inner:
                marked.update(_tile_row_cols(matB, int(it), inner_old, col_new).tolist())
        total += len(marked)
    return _scaled(total, rows, len(smp))


def reorder_estimates(kind, matA, matB, row_old, inner_old, col_old):
    """The plan's estimate fields by the restatement above (the layout of
    src/external_reorder.h:143-171)."""
    if kind == "AA":
        a0 = est_input_tiles(matA)
        a1 = est_input_tiles(matA, row_old, inner_old)
        b0, b1 = a0, a1
        c0 = est_c_tiles(matA, matA, ab=False)
        c1 = est_c_tiles(matA, matA, row_old, inner_old, col_old, ab=False)
    else:
        a0, a1 = est_input_tiles(matA), est_input_tiles(matA, row_old, inner_old)
        b0, b1 = est_input_tiles(matB), est_input_tiles(matB, inner_old, col_old)
        c0 = est_c_tiles(matA, matB)
        c1 = est_c_tiles(matA, matB, row_old, inner_old, col_old)
    ratio = lambda after, before: 1.0 if before <= 0 else after / before  # noqa: E731
    return dict(input_tiles_A_before=a0, input_tiles_A_after=a1, input_tiles_B_before=b0, input_tiles_B_after=b1,
                estimated_c_tiles_before=c0, estimated_c_tiles_after=c1,
                risk_input_tile_ratio=max(ratio(a1, a0), ratio(b1, b0)), risk_c_tile_ratio=ratio(c1, c0))


PLAN_FIELDS = ("enabled", "n", "input_tiles_A_before", "input_tiles_A_after", "input_tiles_B_before",
               "input_tiles_B_after", "estimated_c_tiles_before", "estimated_c_tiles_after", "risk_input_tile_ratio",
               "risk_c_tile_ratio", "local_refine_window", "proxy_sample_rows", "guard_degraded_to_identity",
               "structural_conservative", "shared_symmetric_csr")


def ref_build_reorder_plan(kind, matA, matB=None, symmetric=False):
    """The reference's tile-aware planner build_reorder_plan
    (src/reorder.h:2407-2428) compiled from its sources: (status, plan dict
    with the three new -> old permutations, PLAN_FIELDS, mode, risk_reason).
    Symmetric A*A plans run on the host; the others need a GPU."""
    R = rrlib()
    hA = _CSRHold(matA)
    hB = _CSRHold(matB) if matB is not None else hA
    hA.om.isSymmetric = hB.om.isSymmetric = 1 if symmetric else 0
    info = OReorderInfo()
    R.ref_reorder_info_init(ctypes.byref(info))
    st = R.ref_build_reorder_plan({"AA": 0, "AAT": 1, "AB": 2}[kind], ctypes.byref(hA.om), ctypes.byref(hB.om),
                                  ctypes.byref(info))
    out = {f: getattr(info, f) for f in PLAN_FIELDS}
    out["mode"] = info.mode.decode()
    out["risk_reason"] = info.risk_reason.decode()
    for ax in ("row_perm", "inner_perm", "col_perm"):
        p = getattr(info, ax)
        out[ax] = np.ctypeslib.as_array(p.old_id, shape=(p.n,)).copy() if p.n > 0 and p.old_id else \
            np.zeros(0, np.int32)
    R.ref_reorder_info_destroy(ctypes.byref(info))
    return st, out
