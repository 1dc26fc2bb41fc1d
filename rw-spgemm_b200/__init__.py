"""B200 (sm_100a) tiled SpGEMM -- Python host side over the C ABI.

The compute path is libtilespgemm_b200.so (hand-written CUDA for sm_100a,
built in-tree by ``make -C rw-spgemm_b200``); this module only binds it with
ctypes.  Nothing here computes: if the library is missing, every call raises.

Two surfaces mirror the C ABI (include/tilespgemm_b200.h):

* the reference's drop-in functions on host arrays -- ``csr2tile_row_major``,
  ``csr2tile_col_major``, ``tilespgemm``, ``tile2csr`` (same names, same
  argument meaning, same outputs as for-the-juan/RW-SpGEMM's src/csr2tile.h,
  src/tilespgemm-cuda.h and src/tile2csr.h);
* the device-resident handle API -- ``Context``, ``csr_to_tiled``,
  ``spgemm``, ``tiled_to_csr``, ``spgemm_csr_host``.

The package directory is named ``rw-spgemm_b200``; load it with
``importlib`` (see ``load_package`` in tests/conftest.py or bench.py).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libtilespgemm_b200.so"

TSG_TILED_PACKED_COL = 1
TSG_TILED_CSC_VIEW = 2

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_c_u8_p = ctypes.POINTER(ctypes.c_ubyte)
_c_u16_p = ctypes.POINTER(ctypes.c_ushort)
_c_u32_p = ctypes.POINTER(ctypes.c_uint)


class SMatrix(ctypes.Structure):
    """Reference matrix container (src/common.h:113-135), host pointers."""
    _fields_ = [
        ("m", ctypes.c_int), ("n", ctypes.c_int), ("nnz", ctypes.c_int), ("isSymmetric", ctypes.c_int),
        ("value", _c_dbl_p), ("columnindex", _c_int_p), ("rowpointer", _c_int_p),
        ("tilem", ctypes.c_int), ("tilen", ctypes.c_int),
        ("tile_ptr", _c_int_p), ("tile_columnidx", _c_int_p), ("tile_rowidx", _c_int_p),
        ("tile_nnz", _c_int_p), ("numtile", ctypes.c_int),
        ("tile_csr_Value", _c_dbl_p), ("tile_csr_Col", _c_u8_p), ("tile_csr_Ptr", _c_u8_p),
        ("mask", _c_u16_p), ("csc_tile_ptr", _c_int_p), ("csc_tile_rowidx", _c_int_p),
    ]


class TsgTiled(ctypes.Structure):
    """Device-resident tiled matrix (tsg_tiled), device pointers."""
    _fields_ = [
        ("m", ctypes.c_int), ("n", ctypes.c_int), ("nnz", ctypes.c_int),
        ("tilem", ctypes.c_int), ("tilen", ctypes.c_int), ("numtile", ctypes.c_int),
        ("col_packed", ctypes.c_int),
        ("tile_ptr", ctypes.c_void_p), ("tile_columnidx", ctypes.c_void_p), ("tile_rowidx", ctypes.c_void_p),
        ("tile_nnz", ctypes.c_void_p), ("tile_csr_Ptr", ctypes.c_void_p), ("tile_csr_Col", ctypes.c_void_p),
        ("tile_csr_Value", ctypes.c_void_p), ("mask", ctypes.c_void_p),
        ("csc_tile_ptr", ctypes.c_void_p), ("csc_tile_rowidx", ctypes.c_void_p), ("csc_tile_pos", ctypes.c_void_p),
        ("mask_t", ctypes.c_void_p),
        ("row_ptr", ctypes.c_void_p), ("row_col", ctypes.c_void_p), ("row_val", ctypes.c_void_p),
        ("_alloc", ctypes.c_void_p),
    ]


STEP3_KERNELS = {0: "none", 1: "k_step3", 2: "k_step3_elems", 3: "k_step3_rows", 4: "k_step3_spa<flat>",
                 5: "k_step3_spa", 6: "k_step3_stg + k_step3_rest"}


class TsgInfo(ctypes.Structure):
    _fields_ = [
        ("numtile_C", ctypes.c_longlong), ("nnz_C", ctypes.c_longlong), ("nnzCub", ctypes.c_longlong),
        ("tile_pairs", ctypes.c_longlong),
        ("ms_step1", ctypes.c_double), ("ms_step2", ctypes.c_double), ("ms_step3", ctypes.c_double),
        ("ms_total", ctypes.c_double), ("bins", ctypes.c_int * 4), ("step3_kernel", ctypes.c_int),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "bins"}
        d["bins"] = list(self.bins)
        d["step3_name"] = STEP3_KERNELS.get(self.step3_kernel, "?")
        return d


class TsgError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"tilespgemm_b200 status {status}: {message}")
        self.status = status


_lib = None
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def lib():
    """The loaded C library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C rw-spgemm_b200` "
                               "(the CUDA library is required; there is no fallback)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L):
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.tsg_status_string.restype = ctypes.c_char_p
    L.tsg_last_error.restype = ctypes.c_char_p
    L.tsg_context_create.argtypes = [ip, ctypes.POINTER(vp)]
    L.tsg_context_destroy.argtypes = [vp]
    L.tsg_context_set_stream.argtypes = [vp, vp]
    L.tsg_context_set_timing.argtypes = [vp, ip]
    L.tsg_context_launches.argtypes = [vp]
    L.tsg_context_allocations.argtypes = [vp]
    L.tsg_tiled_device_bytes.argtypes = [ctypes.c_void_p]
    L.tsg_tiled_device_bytes.restype = ctypes.c_longlong
    L.tsg_context_pool_used.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.tsg_context_allocations.restype = ctypes.c_longlong
    L.tsg_context_synchronize.argtypes = [vp]
    L.tsg_context_query.argtypes = [vp]
    L.tsg_context_set_fusion.argtypes = [vp, ip]
    L.tsg_context_set_schedule.argtypes = [vp, ip, ip, ip]
    L.tsg_context_set_dense_threshold.argtypes = [vp, ip]
    L.tsg_context_launches.restype = ctypes.c_longlong
    L.tsg_csr_to_tiled.argtypes = [vp, ip, ip, ip, vp, vp, vp, ip, ctypes.POINTER(TsgTiled)]
    L.tsg_tiled_free.argtypes = [vp, ctypes.POINTER(TsgTiled)]
    L.tsg_spgemm.argtypes = [vp, ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled),
                             ctypes.POINTER(TsgInfo)]
    L.tsg_tiled_to_csr.argtypes = [vp, ctypes.POINTER(TsgTiled), vp, vp, vp]
    L.tsg_tiled_download.argtypes = [vp, ctypes.POINTER(TsgTiled), ip, ctypes.POINTER(SMatrix)]
    L.tsg_tiled_upload_rowmajor.argtypes = [vp, ctypes.POINTER(SMatrix), ctypes.POINTER(TsgTiled)]
    L.tsg_tiled_upload_colmajor.argtypes = [vp, ctypes.POINTER(SMatrix), ctypes.POINTER(TsgTiled)]
    L.tsg_count_products.argtypes = [vp, ip, vp, vp, ctypes.POINTER(ctypes.c_longlong)]
    L.tsg_spgemm_csr_host.argtypes = [vp, ip, ip, ip,
                                      ip, vp, vp, vp, ip, vp, vp, vp,
                                      ctypes.POINTER(ip), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                      ctypes.POINTER(vp), ctypes.POINTER(TsgInfo)]
    L.tsg_spgemm_csr_host_ex.argtypes = list(L.tsg_spgemm_csr_host.argtypes) + [ip]
    L.tsg_host_free.argtypes = [vp]
    L.tsg_host_free.restype = None
    for name in ("csr2tile_row_major", "csr2tile_col_major", "tile2csr", "matrix_destroy"):
        getattr(L, name).argtypes = [ctypes.POINTER(SMatrix)]
        getattr(L, name).restype = None
    L.tilespgemm.argtypes = [ctypes.POINTER(SMatrix)] * 3 + [
        vp, vp, ip, ctypes.c_double, ctypes.c_double, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong),
        _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_char_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
    L.tilespgemm.restype = None


def check(status):
    if status != 0:
        L = lib()
        raise TsgError(status, f"{L.tsg_status_string(status).decode()}: {L.tsg_last_error().decode()}")


# ---------------------------------------------------------------------------
# host array helpers
# ---------------------------------------------------------------------------
def _np_from(ptr, count, dtype, free=False):
    if count == 0 or not ptr:
        out = np.zeros(0, dtype=dtype)
    else:
        addr = ctypes.cast(ptr, ctypes.c_void_p).value
        buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(addr)
        out = np.frombuffer(buf, dtype=dtype).copy()
    if free and ptr:
        _libc.free(ctypes.cast(ptr, ctypes.c_void_p))
    return out


TILE_FIELDS = ("tile_ptr", "tile_columnidx", "tile_rowidx", "tile_nnz", "tile_csr_Ptr", "tile_csr_Col",
               "tile_csr_Value", "mask", "csc_tile_ptr", "csc_tile_rowidx")


def smatrix_tiles_to_numpy(sm: SMatrix, free=True, colmajor=False) -> dict:
    T, nnz = sm.numtile, sm.nnz
    d = dict(m=sm.m, n=sm.n, nnz=nnz, tilem=sm.tilem, tilen=sm.tilen, numtile=T)
    d["tile_ptr"] = _np_from(sm.tile_ptr, sm.tilem + 1, np.int32, free)
    d["tile_columnidx"] = _np_from(sm.tile_columnidx, T, np.int32, free)
    d["tile_rowidx"] = _np_from(sm.tile_rowidx, T, np.int32, free)
    d["tile_nnz"] = _np_from(sm.tile_nnz, T + 1, np.int32, free)
    d["tile_csr_Ptr"] = _np_from(sm.tile_csr_Ptr, 16 * T, np.uint8, free)
    d["tile_csr_Col"] = _np_from(sm.tile_csr_Col, nnz, np.uint8, free)
    d["tile_csr_Value"] = _np_from(sm.tile_csr_Value, nnz, np.float64, free)
    d["mask"] = _np_from(sm.mask, 16 * T, np.uint16, free)
    if colmajor:
        d["csc_tile_ptr"] = _np_from(sm.csc_tile_ptr, sm.tilen + 1, np.int32, free)
        d["csc_tile_rowidx"] = _np_from(sm.csc_tile_rowidx, T, np.int32, free)
    for f in TILE_FIELDS:
        setattr(sm, f, None)
    return d


class HostCSR:
    """Keeps numpy CSR arrays alive behind an SMatrix."""

    def __init__(self, mat):
        m, n, rp, ci, v = mat
        self.rp = np.ascontiguousarray(rp, dtype=np.int32)
        self.ci = np.ascontiguousarray(ci, dtype=np.int32)
        self.v = np.ascontiguousarray(v, dtype=np.float64)
        self.sm = SMatrix()
        self.sm.m, self.sm.n, self.sm.nnz = int(m), int(n), int(self.ci.size)
        self.sm.rowpointer = self.rp.ctypes.data_as(_c_int_p)
        self.sm.columnindex = self.ci.ctypes.data_as(_c_int_p)
        self.sm.value = self.v.ctypes.data_as(_c_dbl_p)


def smatrix_from_tiles(d: dict):
    """SMatrix over numpy tile arrays (kept alive by the returned holder)."""
    hold = {k: np.ascontiguousarray(v) for k, v in d.items() if isinstance(v, np.ndarray)}
    sm = SMatrix()
    for k in ("m", "n", "nnz", "tilem", "tilen", "numtile"):
        setattr(sm, k, int(d[k]))
    types = dict(tile_ptr=_c_int_p, tile_columnidx=_c_int_p, tile_rowidx=_c_int_p, tile_nnz=_c_int_p,
                 tile_csr_Ptr=_c_u8_p, tile_csr_Col=_c_u8_p, tile_csr_Value=_c_dbl_p, mask=_c_u16_p,
                 csc_tile_ptr=_c_int_p, csc_tile_rowidx=_c_int_p)
    for k, t in types.items():
        if k in hold:
            setattr(sm, k, hold[k].ctypes.data_as(t))
    return sm, hold


# ---------------------------------------------------------------------------
# drop-in functions on host arrays
# ---------------------------------------------------------------------------
def csr2tile_row_major(mat) -> dict:
    """src/csr2tile.h:196 on the GPU; returns the tile arrays as numpy."""
    h = HostCSR(mat)
    lib().csr2tile_row_major(ctypes.byref(h.sm))
    return smatrix_tiles_to_numpy(h.sm)


def csr2tile_col_major(mat) -> dict:
    """src/csr2tile.h:261 on the GPU; returns the tile arrays as numpy."""
    h = HostCSR(mat)
    lib().csr2tile_col_major(ctypes.byref(h.sm))
    return smatrix_tiles_to_numpy(h.sm, colmajor=True)


def tile2csr(tiles: dict):
    """src/tile2csr.h:71 on the GPU; returns (rowptr, colidx, val)."""
    sm, hold = smatrix_from_tiles(tiles)
    lib().tile2csr(ctypes.byref(sm))
    rp = _np_from(sm.rowpointer, sm.m + 1, np.int32, True)
    ci = _np_from(sm.columnindex, sm.nnz, np.int32, True)
    v = _np_from(sm.value, sm.nnz, np.float64, True)
    return rp, ci, v


def tile_intersection_bitmaps(tilesA: dict, tilesB: dict):
    """The reference driver's intersection bitmaps (src/main.cu:430-465) on
    the GPU: (bitmask_A [tilem x len], bitmask_B [tilen_B x len]) uint32."""
    smA, holdA = smatrix_from_tiles(tilesA)
    smB, holdB = smatrix_from_tiles(tilesB)
    pa, pb, ln = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_int(0)
    L = lib()
    L.tile_intersection_bitmaps.argtypes = [ctypes.POINTER(SMatrix), ctypes.POINTER(SMatrix), ctypes.POINTER(ctypes.c_void_p),
                                            ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int)]
    check(L.tile_intersection_bitmaps(ctypes.byref(smA), ctypes.byref(smB), ctypes.byref(pa), ctypes.byref(pb),
                                      ctypes.byref(ln)))
    n = ln.value
    bmA = _np_from(ctypes.cast(pa, _c_u32_p), int(tilesA["tilem"]) * n, np.uint32, True).reshape(-1, max(n, 1))
    bmB = _np_from(ctypes.cast(pb, _c_u32_p), int(tilesB["tilen"]) * n, np.uint32, True).reshape(-1, max(n, 1))
    return bmA, bmB


def tilespgemm(tilesA: dict, tilesB: dict, nnzCub: int = 0) -> tuple[dict, dict]:
    """src/tilespgemm-cuda.h:2610 on host tiles (A row-major, B column-major).
    Returns (C tiles, timings)."""
    smA, holdA = smatrix_from_tiles(tilesA)
    smB, holdB = smatrix_from_tiles(tilesB)
    smC = SMatrix()
    nnzC = ctypes.c_ulonglong(0)
    dbl = [ctypes.c_double(0.0) for _ in range(7)]
    lib().tilespgemm(ctypes.byref(smA), ctypes.byref(smB), ctypes.byref(smC), None, None, 0, 0.0, 0.0,
                     ctypes.c_ulonglong(nnzCub), ctypes.byref(nnzC), *[ctypes.byref(x) for x in dbl[:3]],
                     b"", *[ctypes.byref(x) for x in dbl[3:]])
    C = smatrix_tiles_to_numpy(smC)
    t = dict(nnzC=nnzC.value, compression_rate=dbl[0].value, time_ms=dbl[1].value, gflops=dbl[2].value,
             step1_ms=dbl[3].value, step2_ms=dbl[4].value, step3_ms=dbl[5].value, malloc_ms=dbl[6].value)
    return C, t


# ---------------------------------------------------------------------------
# handle API (device-resident)
# ---------------------------------------------------------------------------
CUDA_STREAM_LEGACY = 0x1
SCHEDULE_IDS = {"tiles": 0, "rows": 1, "elems": 2, "spa": 3}


class Context:
    """tsg_context on one device.  Work goes to ``stream`` (a cudaStream_t as
    int) when given, else to torch's current stream on that device when torch
    is importable, so library calls are ordered with the caller's torch work;
    ``own_stream=True`` keeps the context's private stream."""

    def __init__(self, device: int = 0, stream=None, timing: bool = False, own_stream: bool = False):
        self.handle = ctypes.c_void_p()
        check(lib().tsg_context_create(device, ctypes.byref(self.handle)))
        if stream is None and not own_stream:
            try:
                import torch
                stream = torch.cuda.current_stream(device).cuda_stream
            except Exception:
                stream = None
        if stream is not None:
            # torch reports its legacy default stream as 0, which the C API
            # reads as "own stream": name it explicitly (cudaStreamLegacy)
            self.set_stream(stream if int(stream) != 0 else CUDA_STREAM_LEGACY)
        if timing:
            self.set_timing(True)

    def set_stream(self, stream_ptr: int):
        check(lib().tsg_context_set_stream(self.handle, ctypes.c_void_p(int(stream_ptr))))

    def set_timing(self, on: bool):
        check(lib().tsg_context_set_timing(self.handle, 1 if on else 0))

    def set_schedule(self, schedule: str = "spa", seg_tiles: int = 8, acc_cap: int = 512, dense: int = 0):
        """'tiles' (half-warp per C tile, intersection) or 'rows' (half-warp per
        run of seg_tiles C tiles of one tile row, acc_cap FP64 slots); 'spa'
        takes `dense`, the C values per tile from which a product runs the
        tile kernel (0: the default 64)."""
        check(lib().tsg_context_set_schedule(self.handle, SCHEDULE_IDS[schedule], seg_tiles,
                                             acc_cap))
        check(lib().tsg_context_set_dense_threshold(self.handle, int(dense)))

    def set_fusion(self, on: bool):
        check(lib().tsg_context_set_fusion(self.handle, 1 if on else 0))

    def synchronize(self):
        check(lib().tsg_context_synchronize(self.handle))

    def launches(self) -> int:
        return int(lib().tsg_context_launches(self.handle))

    def allocations(self) -> int:
        """Device allocations the library made on this context so far."""
        return int(lib().tsg_context_allocations(self.handle))

    def pool_used(self) -> int:
        """Bytes in use in the device's default memory pool (the library's
        allocations)."""
        out = ctypes.c_ulonglong(0)
        check(lib().tsg_context_pool_used(self.handle, ctypes.byref(out)))
        return int(out.value)

    def close(self):
        if self.handle:
            lib().tsg_context_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tiled:
    """Owner of a device tsg_tiled."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.s = TsgTiled()

    @property
    def numtile(self):
        return self.s.numtile

    @property
    def nnz(self):
        return self.s.nnz

    @property
    def device_bytes(self) -> int:
        """Device bytes the library holds for this matrix (every array as
        allocated; 0 for a borrowed view)."""
        return int(lib().tsg_tiled_device_bytes(ctypes.byref(self.s)))

    def download(self, colmajor: bool = False) -> dict:
        sm = SMatrix()
        check(lib().tsg_tiled_download(self.ctx.handle, ctypes.byref(self.s), 1 if colmajor else 0,
                                       ctypes.byref(sm)))
        return smatrix_tiles_to_numpy(sm, colmajor=colmajor)

    def free(self):
        if self.ctx is not None and self.ctx.handle:
            lib().tsg_tiled_free(self.ctx.handle, ctypes.byref(self.s))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def csr_to_tiled(ctx: Context, m: int, n: int, rowptr, colidx, val, flags: int) -> Tiled:
    """GPU CSR -> tiles from device tensors (torch int32/int32/float64)."""
    t = Tiled(ctx)
    check(lib().tsg_csr_to_tiled(ctx.handle, int(m), int(n), int(colidx.numel()), ctypes.c_void_p(rowptr.data_ptr()),
                                 ctypes.c_void_p(colidx.data_ptr()), ctypes.c_void_p(val.data_ptr()), int(flags),
                                 ctypes.byref(t.s)))
    return t


def upload_rowmajor(ctx: Context, tiles: dict) -> Tiled:
    sm, hold = smatrix_from_tiles(tiles)
    t = Tiled(ctx)
    check(lib().tsg_tiled_upload_rowmajor(ctx.handle, ctypes.byref(sm), ctypes.byref(t.s)))
    t._hold = hold
    return t


def upload_colmajor(ctx: Context, tiles: dict) -> Tiled:
    sm, hold = smatrix_from_tiles(tiles)
    t = Tiled(ctx)
    check(lib().tsg_tiled_upload_colmajor(ctx.handle, ctypes.byref(sm), ctypes.byref(t.s)))
    t._hold = hold
    return t


def spgemm(ctx: Context, A: Tiled, B: Tiled) -> tuple[Tiled, dict]:
    C = Tiled(ctx)
    info = TsgInfo()
    check(lib().tsg_spgemm(ctx.handle, ctypes.byref(A.s), ctypes.byref(B.s), ctypes.byref(C.s), ctypes.byref(info)))
    return C, info.as_dict()


def tiled_to_csr(ctx: Context, C: Tiled):
    """Device CSR (torch tensors) of a tiled matrix."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    rp = torch.empty(C.s.m + 1, dtype=torch.int32, device=dev)
    ci = torch.empty(max(C.s.nnz, 1), dtype=torch.int32, device=dev)
    v = torch.empty(max(C.s.nnz, 1), dtype=torch.float64, device=dev)
    check(lib().tsg_tiled_to_csr(ctx.handle, ctypes.byref(C.s), ctypes.c_void_p(rp.data_ptr()),
                                 ctypes.c_void_p(ci.data_ptr()), ctypes.c_void_p(v.data_ptr())))
    ctx.synchronize()
    return rp, ci[:C.s.nnz], v[:C.s.nnz]


def count_products(ctx: Context, a_colidx, b_rowptr) -> int:
    out = ctypes.c_longlong(0)
    check(lib().tsg_count_products(ctx.handle, int(a_colidx.numel()), ctypes.c_void_p(a_colidx.data_ptr()),
                                   ctypes.c_void_p(b_rowptr.data_ptr()), ctypes.byref(out)))
    return out.value


class _PinnedHostArray:
    """Owner of a page-locked result array; freed with tsg_host_free."""

    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            lib().tsg_host_free(self.ptr)
        except Exception:
            pass


def _wrap_pinned(ptr, count, dtype):
    owner = _PinnedHostArray(ptr)
    if count == 0:
        return np.zeros(0, dtype=dtype)
    buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr.value)
    arr = np.frombuffer(buf, dtype=dtype)
    arr_owner = arr.view()  # keep the owner alive as long as the array
    buf._owner = owner
    return arr_owner


def spgemm_csr_host(ctx: Context, matA, matB=None, pinned: bool = True):
    """End to end through the C ABI with host buffers: CSR A * CSR B -> CSR C
    (numpy).  matB=None computes A*A.  pinned=True returns page-locked result
    arrays without a copy."""
    hA = HostCSR(matA)
    hB = hA if matB is None else HostCSR(matB)
    nnzC = ctypes.c_int(0)
    prp, pci, pv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    info = TsgInfo()
    m, k = hA.sm.m, hA.sm.n
    n = hB.sm.n
    check(lib().tsg_spgemm_csr_host_ex(
        ctx.handle, m, k, n,
        hA.sm.nnz, hA.rp.ctypes.data, hA.ci.ctypes.data, hA.v.ctypes.data,
        hB.sm.nnz, hB.rp.ctypes.data, hB.ci.ctypes.data, hB.v.ctypes.data,
        ctypes.byref(nnzC), ctypes.byref(prp), ctypes.byref(pci), ctypes.byref(pv), ctypes.byref(info),
        1 if pinned else 0))
    if pinned:
        rp = _wrap_pinned(prp, m + 1, np.int32)
        ci = _wrap_pinned(pci, nnzC.value, np.int32)
        v = _wrap_pinned(pv, nnzC.value, np.float64)
    else:
        rp = _np_from(prp, m + 1, np.int32, True)
        ci = _np_from(pci, nnzC.value, np.int32, True)
        v = _np_from(pv, nnzC.value, np.float64, True)
    return (m, n, rp, ci, v), info.as_dict()


# ---------------------------------------------------------------------------
# orderings and bipermutations
# ---------------------------------------------------------------------------
ORDER_KINDS = {"original": 0, "rcm": 1, "degree": 2, "gray": 3, "random": 4}


class AxisPermutation(ctypes.Structure):
    """src/reorder.h:26-31: new -> old (old_id) and old -> new (new_id)."""
    _fields_ = [("n", ctypes.c_int), ("old_id", _c_int_p), ("new_id", _c_int_p)]


class ReorderInfo(ctypes.Structure):
    """src/reorder.h:33-64 (field order kept)."""
    _fields_ = [
        ("enabled", ctypes.c_int), ("n", ctypes.c_int),
        ("row_perm", AxisPermutation), ("inner_perm", AxisPermutation), ("col_perm", AxisPermutation),
        ("input_tiles_A_before", ctypes.c_longlong), ("input_tiles_A_after", ctypes.c_longlong),
        ("input_tiles_B_before", ctypes.c_longlong), ("input_tiles_B_after", ctypes.c_longlong),
        ("estimated_c_tiles_before", ctypes.c_longlong), ("estimated_c_tiles_after", ctypes.c_longlong),
        ("reorder_time_ms", ctypes.c_double), ("signature_time_ms", ctypes.c_double),
        ("tile_profile_time_ms", ctypes.c_double), ("affinity_time_ms", ctypes.c_double),
        ("sort_time_ms", ctypes.c_double), ("local_refine_time_ms", ctypes.c_double),
        ("proxy_time_ms", ctypes.c_double), ("permute_time_ms", ctypes.c_double),
        ("risk_input_tile_ratio", ctypes.c_double), ("risk_c_tile_ratio", ctypes.c_double),
        ("local_refine_window", ctypes.c_int), ("proxy_sample_rows", ctypes.c_int),
        ("guard_degraded_to_identity", ctypes.c_int), ("structural_conservative", ctypes.c_int),
        ("shared_symmetric_csr", ctypes.c_int), ("mode", ctypes.c_char * 64), ("risk_reason", ctypes.c_char * 128),
    ]


class ReorderProblem(ctypes.Structure):
    """src/reorder.h:72-77."""
    _fields_ = [("kind", ctypes.c_int), ("matrixA", ctypes.POINTER(SMatrix)), ("matrixB", ctypes.POINTER(SMatrix))]


def _declare_reorder(L):
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.tsg_order.argtypes = [vp, ip, ip, ip, ip, vp, vp, ctypes.c_ulonglong, vp]
    L.tsg_order_from_name.argtypes = [ctypes.c_char_p]
    L.tsg_permute_csr.argtypes = [vp, ip, ip, ip, vp, vp, vp, vp, vp, vp, vp, vp]
    L.reorder_info_init.argtypes = [ctypes.POINTER(ReorderInfo)]
    L.reorder_info_init.restype = None
    L.reorder_info_destroy.argtypes = [ctypes.POINTER(ReorderInfo)]
    L.reorder_info_destroy.restype = None
    L.build_original_reorder_plan.argtypes = [ip, ctypes.POINTER(SMatrix), ctypes.POINTER(SMatrix),
                                              ctypes.POINTER(ReorderInfo)]
    L.build_external_reorder_plan.argtypes = [ip, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                              ctypes.POINTER(SMatrix), ctypes.POINTER(SMatrix),
                                              ctypes.POINTER(ReorderInfo), ctypes.POINTER(ctypes.c_double)]
    L.build_reorder_plan.argtypes = [ctypes.POINTER(ReorderProblem), ctypes.POINTER(ReorderInfo)]
    L.apply_bipermutation_csr.argtypes = [ctypes.POINTER(SMatrix), ctypes.POINTER(AxisPermutation),
                                          ctypes.POINTER(AxisPermutation), ctypes.POINTER(SMatrix)]
    L.restore_bipermutation_csr.argtypes = [ctypes.POINTER(SMatrix), ctypes.POINTER(AxisPermutation),
                                            ctypes.POINTER(AxisPermutation)]


_declare_base = _declare


def _declare(L):  # noqa: F811
    _declare_base(L)
    _declare_reorder(L)


def order(ctx: Context, kind: str, m: int, n: int, rowptr, colidx, seed: int = 1):
    """GPU ordering (new -> old, torch int32 tensor on the current device)."""
    import torch
    out = torch.empty(max(m, 1), dtype=torch.int32, device=rowptr.device)
    check(lib().tsg_order(ctx.handle, ORDER_KINDS[kind], int(m), int(n), int(colidx.numel()),
                          ctypes.c_void_p(rowptr.data_ptr()), ctypes.c_void_p(colidx.data_ptr()),
                          ctypes.c_ulonglong(seed), ctypes.c_void_p(out.data_ptr())))
    ctx.synchronize()
    return out[:m]


def permute_csr(ctx: Context, m: int, n: int, rowptr, colidx, val, row_old, col_new):
    """Device bipermutation P_r A P_c^T (torch tensors in and out)."""
    import torch
    nnz = int(colidx.numel())
    orp = torch.empty(m + 1, dtype=torch.int32, device=rowptr.device)
    oci = torch.empty(max(nnz, 1), dtype=torch.int32, device=rowptr.device)
    ov = torch.empty(max(nnz, 1), dtype=torch.float64, device=rowptr.device)
    check(lib().tsg_permute_csr(ctx.handle, int(m), int(n), nnz, *[ctypes.c_void_p(t.data_ptr()) for t in
                                (rowptr, colidx, val, row_old, col_new, orp, oci, ov)]))
    ctx.synchronize()
    return orp, oci[:nnz], ov[:nnz]


class _Axis:
    def __init__(self, old_id):
        self.old = np.ascontiguousarray(old_id, dtype=np.int32)
        self.new = np.empty_like(self.old)
        self.new[self.old] = np.arange(self.old.size, dtype=np.int32)
        self.s = AxisPermutation(int(self.old.size), self.old.ctypes.data_as(_c_int_p), self.new.ctypes.data_as(_c_int_p))


PLAN_ESTIMATES = ("input_tiles_A_before", "input_tiles_A_after", "input_tiles_B_before", "input_tiles_B_after",
                  "estimated_c_tiles_before", "estimated_c_tiles_after", "risk_input_tile_ratio", "risk_c_tile_ratio")


def reorder_estimates(kind: str, matA, matB, row_old, inner_old, col_old) -> dict:
    """tsg_reorder_estimates: a plan's sampled tile-count estimates for three
    new -> old permutations (host computation, no device work)."""
    hA = HostCSR(matA)
    hB = HostCSR(matB) if matB is not None else hA
    axes = [_Axis(p) for p in (row_old, inner_old, col_old)]
    info = ReorderInfo()
    info.row_perm, info.inner_perm, info.col_perm = (a.s for a in axes)
    L = lib()
    L.tsg_reorder_estimates.argtypes = [ctypes.c_int, ctypes.POINTER(SMatrix), ctypes.POINTER(SMatrix),
                                        ctypes.POINTER(ReorderInfo)]
    check(L.tsg_reorder_estimates(REORDER_PROBLEM[kind], ctypes.byref(hA.sm), ctypes.byref(hB.sm), ctypes.byref(info)))
    return {f: getattr(info, f) for f in PLAN_ESTIMATES}


def _csr_from_smatrix(sm: SMatrix, free=True):
    rp = _np_from(sm.rowpointer, sm.m + 1, np.int32, free)
    ci = _np_from(sm.columnindex, sm.nnz, np.int32, free)
    v = _np_from(sm.value, sm.nnz, np.float64, free)
    return sm.m, sm.n, rp, ci, v


def apply_bipermutation_csr(mat, row_old, col_old):
    """src/reorder.h:2429 on the GPU; permutations given new -> old."""
    h = HostCSR(mat)
    r, c = _Axis(row_old), _Axis(col_old)
    out = SMatrix()
    st = lib().apply_bipermutation_csr(ctypes.byref(h.sm), ctypes.byref(r.s), ctypes.byref(c.s), ctypes.byref(out))
    if st != 0:
        raise TsgError(st, "apply_bipermutation_csr failed")
    return _csr_from_smatrix(out)


def restore_bipermutation_csr(mat, row_old, col_old):
    """src/reorder.h:2506 on the GPU (the inverse of apply)."""
    m, n, rp, ci, v = mat
    sm = SMatrix()
    sm.m, sm.n, sm.nnz = int(m), int(n), int(len(ci))
    # the function frees and replaces the CSR arrays: hand it malloc'd copies
    for field, arr, ctype in (("rowpointer", rp, ctypes.c_int), ("columnindex", ci, ctypes.c_int),
                              ("value", v, ctypes.c_double)):
        a = np.ascontiguousarray(arr)
        nbytes = max(a.nbytes, 1)
        _libc.malloc.restype = ctypes.c_void_p
        _libc.malloc.argtypes = [ctypes.c_size_t]
        p = _libc.malloc(nbytes)
        ctypes.memmove(p, a.ctypes.data, a.nbytes)
        setattr(sm, field, ctypes.cast(p, ctypes.POINTER(ctype)))
    r, c = _Axis(row_old), _Axis(col_old)
    st = lib().restore_bipermutation_csr(ctypes.byref(sm), ctypes.byref(r.s), ctypes.byref(c.s))
    if st != 0:
        raise TsgError(st, "restore_bipermutation_csr failed")
    return _csr_from_smatrix(sm)


REORDER_PROBLEM = {"AA": 0, "AAT": 1, "AB": 2}


def build_reorder_plan(kind: str, algorithm: str, matA, matB=None, symmetric: bool = False) -> dict:
    """build_original_reorder_plan / build_external_reorder_plan
    (src/external_reorder.h:173-321) with the ordering computed on the GPU;
    algorithm "tasa": the tile-aware planner build_reorder_plan
    (src/reorder.h:2407), whose A*A plan depends on `symmetric` (the
    matrices' isSymmetric flag, as a symmetric Matrix Market file sets it)."""
    L = lib()
    hA = HostCSR(matA)
    hB = HostCSR(matB) if matB is not None else None
    for h in (hA, hB):
        if h is not None:
            h.sm.isSymmetric = 1 if symmetric else 0
    info = ReorderInfo()
    L.reorder_info_init(ctypes.byref(info))
    ms = ctypes.c_double(0.0)
    pB = ctypes.byref(hB.sm) if hB else None
    if algorithm == "tasa":
        prob = ReorderProblem(REORDER_PROBLEM[kind], ctypes.pointer(hA.sm),
                              ctypes.pointer(hB.sm) if hB else ctypes.pointer(hA.sm))
        st = L.build_reorder_plan(ctypes.byref(prob), ctypes.byref(info))
    elif algorithm == "original":
        st = L.build_original_reorder_plan(REORDER_PROBLEM[kind], ctypes.byref(hA.sm), pB, ctypes.byref(info))
    else:
        st = L.build_external_reorder_plan(REORDER_PROBLEM[kind], algorithm.encode(), b"", b"", ctypes.byref(hA.sm),
                                           pB, ctypes.byref(info), ctypes.byref(ms))
    if st != 0:
        L.reorder_info_destroy(ctypes.byref(info))
        raise TsgError(st, f"reorder plan '{algorithm}' failed")
    d = {f: getattr(info, f) for f, _ in ReorderInfo._fields_ if not f.endswith("_perm")}
    d["mode"] = info.mode.decode()
    d["risk_reason"] = info.risk_reason.decode()
    for ax in ("row_perm", "inner_perm", "col_perm"):
        p = getattr(info, ax)
        d[ax] = _np_from(p.old_id, p.n, np.int32, False)
    d["ordergen_ms"] = ms.value
    L.reorder_info_destroy(ctypes.byref(info))
    return d


# ---------------------------------------------------------------------------
# batched products (one persistent, graph-captured launch for many products)
# ---------------------------------------------------------------------------
class BatchParams(ctypes.Structure):
    _fields_ = [("schedule", ctypes.c_int), ("seg_tiles", ctypes.c_int), ("acc_cap", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("dense_threshold", ctypes.c_int)]


def _declare_batch(L):
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.tsg_batch_create.argtypes = [vp, ip, ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled),
                                   ctypes.POINTER(BatchParams), ctypes.POINTER(vp)]
    L.tsg_batch_create_bounded.argtypes = [vp, ip, ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled),
                                           ctypes.POINTER(BatchParams), ctypes.POINTER(ctypes.c_longlong),
                                           ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(vp)]
    L.tsg_batch_run.argtypes = [vp]
    L.tsg_batch_sync.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.tsg_batch_product.argtypes = [vp, ip, ctypes.POINTER(TsgTiled)]
    L.tsg_batch_info.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_size_t),
                                 ctypes.POINTER(ctypes.c_longlong)]
    L.tsg_batch_destroy.argtypes = [vp]
    L.tsg_batch_phase_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.tsg_batch_set_wait_limit.argtypes = [vp, ctypes.c_double]
    L.tsg_product_bounds.argtypes = [vp, ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled),
                                     ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]
    L.tsg_product_bounds_many.argtypes = [vp, ip, ctypes.POINTER(TsgTiled), ctypes.POINTER(TsgTiled),
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.POINTER(ctypes.c_longlong)]


_declare_prev = _declare


def _declare(L):  # noqa: F811
    _declare_prev(L)
    _declare_batch(L)


def product_bounds(ctx: Context, A: Tiled, B: Tiled):
    """(scalar products, matched tile pairs) of A*B from the tile structure."""
    pr, tp = ctypes.c_longlong(0), ctypes.c_longlong(0)
    check(lib().tsg_product_bounds(ctx.handle, ctypes.byref(A.s), ctypes.byref(B.s), ctypes.byref(pr),
                                   ctypes.byref(tp)))
    return pr.value, tp.value


def product_bounds_many(ctx: Context, pairs, c_tiles: bool = False):
    """product_bounds of every (A, B) in pairs with one synchronisation:
    a list of (products, tile pairs), or of (products, tile pairs, C tiles)
    with c_tiles (step 1's exact count)."""
    n = len(pairs)
    if n == 0:
        return []
    As = (TsgTiled * n)(*[a.s for a, _ in pairs])
    Bs = (TsgTiled * n)(*[b.s for _, b in pairs])
    pr, tp, ct = (ctypes.c_longlong * n)(), (ctypes.c_longlong * n)(), (ctypes.c_longlong * n)()
    check(lib().tsg_product_bounds_many(ctx.handle, n, As, Bs, pr, tp, ct if c_tiles else None))
    if c_tiles:
        return [(pr[i], tp[i], ct[i]) for i in range(n)]
    return [(pr[i], tp[i]) for i in range(n)]


class Batch:
    """tsg_batch over device-resident (A, B) operand pairs."""

    def __init__(self, ctx: Context, pairs, schedule: str = "spa", seg_tiles: int = 8, acc_cap: int = 512,
                 graph: bool = True, dense: int = 0, bounds=None):
        """dense: the 'spa' schedule's C values per tile from which a product
        runs the tile kernel (0: the default 64).  bounds: per pair its
        (scalar products, C tiles) from product_bounds_many(c_tiles=True);
        given, the batch is planned without waiting for the device."""
        self.ctx = ctx
        self.pairs = list(pairs)  # keep operands alive
        n = len(self.pairs)
        arrA = (TsgTiled * n)(*[a.s for a, _ in self.pairs])
        arrB = (TsgTiled * n)(*[b.s for _, b in self.pairs])
        prm = BatchParams(SCHEDULE_IDS[schedule], seg_tiles, acc_cap, 1 if graph else 0, int(dense))
        self.handle = ctypes.c_void_p()
        if bounds is None:
            check(lib().tsg_batch_create(ctx.handle, n, arrA, arrB, ctypes.byref(prm), ctypes.byref(self.handle)))
        else:
            if len(bounds) != n:
                raise ValueError("one (products, C tiles) bound per pair")
            pr = (ctypes.c_longlong * n)(*[int(b[0]) for b in bounds])
            ct = (ctypes.c_longlong * n)(*[int(b[1]) for b in bounds])
            check(lib().tsg_batch_create_bounded(ctx.handle, n, arrA, arrB, ctypes.byref(prm), pr, ct,
                                                 ctypes.byref(self.handle)))
        self.count = n
        self.params = dict(schedule=schedule, seg_tiles=seg_tiles, acc_cap=acc_cap, dense=dense)

    def run(self):
        check(lib().tsg_batch_run(self.handle))

    def phase_ms(self):
        """Per-phase GPU time (ms) of the last finished run (see
        tsg_batch_phase_ms)."""
        out = (ctypes.c_double * 7)()
        check(lib().tsg_batch_phase_ms(self.handle, out))
        names = ["step1_counts", "row_scans", "item_prefix", "step1_emit_step2", "step2_rest", "tile_scans", "step3"]
        return {k: round(v, 4) for k, v in zip(names, out)}

    def set_wait_limit(self, seconds: float):
        """Grid-barrier wait bound in seconds (tsg_batch_set_wait_limit)."""
        check(lib().tsg_batch_set_wait_limit(self.handle, float(seconds)))

    def sync(self):
        t, z = ctypes.c_longlong(0), ctypes.c_longlong(0)
        check(lib().tsg_batch_sync(self.handle, ctypes.byref(t), ctypes.byref(z)))
        return t.value, z.value

    def product(self, p: int) -> Tiled:
        """Borrowed view of product p's C (valid until the next run / close)."""
        v = Tiled(self.ctx)
        check(lib().tsg_batch_product(self.handle, int(p), ctypes.byref(v.s)))
        return v

    def info(self) -> dict:
        g, gr = ctypes.c_int(0), ctypes.c_int(0)
        ab, ln = ctypes.c_size_t(0), ctypes.c_longlong(0)
        check(lib().tsg_batch_info(self.handle, ctypes.byref(g), ctypes.byref(gr), ctypes.byref(ab), ctypes.byref(ln)))
        return dict(graph=bool(g.value), grid=gr.value, arena_bytes=ab.value, launches=ln.value)

    def close(self):
        if self.handle:
            lib().tsg_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _declare_host_io(L):
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.tsg_csr_host_to_tiled.argtypes = [vp, ip, ip, ip, vp, vp, vp, ip, ctypes.POINTER(TsgTiled)]
    L.tsg_tiled_to_csr_host.argtypes = [vp, ctypes.POINTER(TsgTiled), ip, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                        ctypes.POINTER(vp)]


_declare_prev2 = _declare


def _declare(L):  # noqa: F811
    _declare_prev2(L)
    _declare_host_io(L)


def csr_host_to_tiled(ctx: Context, mat, flags: int) -> Tiled:
    """Host CSR (numpy) -> device tiles in one C call."""
    h = HostCSR(mat)
    t = Tiled(ctx)
    check(lib().tsg_csr_host_to_tiled(ctx.handle, h.sm.m, h.sm.n, h.sm.nnz, h.rp.ctypes.data, h.ci.ctypes.data,
                                      h.v.ctypes.data, int(flags), ctypes.byref(t.s)))
    return t


def tiled_to_csr_host(ctx: Context, C: Tiled, pinned: bool = True):
    """Device tiles -> host CSR (numpy; page-locked without a copy when pinned)."""
    prp, pci, pv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    check(lib().tsg_tiled_to_csr_host(ctx.handle, ctypes.byref(C.s), 1 if pinned else 0, ctypes.byref(prp),
                                      ctypes.byref(pci), ctypes.byref(pv)))
    m, n, nnz = C.s.m, C.s.n, C.s.nnz
    if pinned:
        return m, n, _wrap_pinned(prp, m + 1, np.int32), _wrap_pinned(pci, nnz, np.int32), _wrap_pinned(pv, nnz, np.float64)
    return (m, n, _np_from(prp, m + 1, np.int32, True), _np_from(pci, nnz, np.int32, True),
            _np_from(pv, nnz, np.float64, True))


def _declare_result(L):
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.tsg_spgemm_csr_host_start.argtypes = [vp, ip, ip, ip, ip, vp, vp, vp, ip, vp, vp, vp, ctypes.POINTER(vp),
                                            ctypes.POINTER(ip), ctypes.POINTER(TsgInfo)]
    L.tsg_result_copy.argtypes = [vp, vp, vp, vp]
    L.tsg_result_free.argtypes = [vp]
    L.tsg_spgemm_csr_host_into.argtypes = [vp, ip, ip, ip, ip, vp, vp, vp, ip, vp, vp, vp, vp, vp, vp,
                                           ctypes.c_longlong, ctypes.POINTER(ip), ctypes.POINTER(TsgInfo)]


_declare_prev3 = _declare


def _declare(L):  # noqa: F811
    _declare_prev3(L)
    _declare_result(L)


class HostResultBuffers:
    """Reusable (page-locked when torch is available) output buffers for the
    two-phase end-to-end call."""

    def __init__(self, m: int, nnz_cap: int, pinned: bool = True):
        self.resize(m, nnz_cap, pinned)

    def resize(self, m, nnz_cap, pinned=None):
        """Reallocates for m rows and nnz_cap entries; page-locked or not as
        before unless pinned says otherwise."""
        pinned = getattr(self, "pinned", True) if pinned is None else pinned
        self.m, self.cap, self.pinned = m, nnz_cap, pinned
        if pinned:
            import torch
            self._t = [torch.empty(m + 1, dtype=torch.int32).pin_memory(),
                       torch.empty(max(nnz_cap, 1), dtype=torch.int32).pin_memory(),
                       torch.empty(max(nnz_cap, 1), dtype=torch.float64).pin_memory()]
            self.rp, self.ci, self.v = (t.numpy() for t in self._t)
        else:
            self.rp = np.empty(m + 1, np.int32)
            self.ci = np.empty(max(nnz_cap, 1), np.int32)
            self.v = np.empty(max(nnz_cap, 1), np.float64)


TSG_ERR_OVERFLOW = -5


def spgemm_csr_host_overlap(ctx: Context, matA, matB, out: HostResultBuffers):
    """End to end in one C call (tsg_spgemm_csr_host_into): the result is
    written into out while it is computed, C's CSR copied to the host chunk
    by chunk during the numeric step.  out is grown (and the product run
    again) when C has more nonzeros than it holds.  Returns (m, n, rowptr,
    colidx, val) views into out, and the info dict."""
    hA = HostCSR(matA)
    hB = hA if matB is None else HostCSR(matB)
    m, k, n = hA.sm.m, hA.sm.n, hB.sm.n
    for _ in range(2):
        if out.m != m:
            out.resize(m, out.cap)
        nnzC = ctypes.c_int(0)
        info = TsgInfo()
        st = lib().tsg_spgemm_csr_host_into(
            ctx.handle, m, k, n, hA.sm.nnz, hA.rp.ctypes.data, hA.ci.ctypes.data, hA.v.ctypes.data,
            hB.sm.nnz, hB.rp.ctypes.data, hB.ci.ctypes.data, hB.v.ctypes.data,
            out.rp.ctypes.data, out.ci.ctypes.data, out.v.ctypes.data, out.cap, ctypes.byref(nnzC),
            ctypes.byref(info))
        if st == TSG_ERR_OVERFLOW and nnzC.value > out.cap:
            out.resize(m, nnzC.value)
            continue
        check(st)
        nz = nnzC.value
        return (m, n, out.rp, out.ci[:nz], out.v[:nz]), info.as_dict()
    raise TsgError(TSG_ERR_OVERFLOW, "result buffers could not be sized")


def spgemm_csr_host_into(ctx: Context, matA, matB, out: HostResultBuffers):
    """End to end with host buffers through the two-phase C call; the result
    lands in out (grown if too small).  Returns (m, n, rowptr, colidx, val)
    views into out, and the info dict."""
    hA = HostCSR(matA)
    hB = hA if matB is None else HostCSR(matB)
    res = ctypes.c_void_p()
    nnzC = ctypes.c_int(0)
    info = TsgInfo()
    m, k, n = hA.sm.m, hA.sm.n, hB.sm.n
    check(lib().tsg_spgemm_csr_host_start(
        ctx.handle, m, k, n, hA.sm.nnz, hA.rp.ctypes.data, hA.ci.ctypes.data, hA.v.ctypes.data,
        hB.sm.nnz, hB.rp.ctypes.data, hB.ci.ctypes.data, hB.v.ctypes.data,
        ctypes.byref(res), ctypes.byref(nnzC), ctypes.byref(info)))
    try:
        if out.m != m or out.cap < nnzC.value:
            out.resize(m, nnzC.value)
        check(lib().tsg_result_copy(res, out.rp.ctypes.data, out.ci.ctypes.data, out.v.ctypes.data))
    finally:
        lib().tsg_result_free(res)
    nz = nnzC.value
    return (m, n, out.rp, out.ci[:nz], out.v[:nz]), info.as_dict()
