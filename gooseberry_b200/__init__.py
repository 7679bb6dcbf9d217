"""gooseberry_b200 -- B200 (sm_100a) implementation of gooseberry's sparse hot
path: CSR SpMV (reference ``src/blas.c:552-606``) and the conjugate-gradient
solver built on it (``src/cgd.c:40-129``).

Everything here is a thin ctypes layer over ``libgooseberry_b200.so``, whose
C ABI is declared in ``include/gooseberry.h`` (the reference's drop-in entry
points, host pointers) and ``include/gooseberry_b200.h`` (device-resident
matrices, SpMV, BLAS-1 and CG solvers).  There is no CPU fallback: if the
library is missing every call raises.

Host-pointer API (mirrors the reference's public functions)::

    spmult(rowptr, rowind, rowval, B, ...)   # gooseberry_spmult
    scale(v, s), add_scalar(v, s)            # gooseberry_scale / _add_scalar
    cgd(rowptr, rowind, rowval, b, error, niter)   # cgd

Device API (torch CUDA tensors as device memory)::

    A = CsrMatrix.from_host(csr)            # or CsrMatrix.from_device(...)
    A.spmv(x, y)                             # y = A x
    CgSolver(A).solve(b, x, tol=1e-8, relative=True, niter=5000)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "GooseberryError", "lib", "spmult", "scale", "add_scalar", "cgd", "pagerank",
    "read_csr", "read_grid", "write_csr", "write_grid", "cuthillmckee", "permute_sparse",
    "permute_dense", "permute_vector",
    "CsrMatrix", "CgSolver", "CgResult", "dot", "spdot", "add", "sub", "SUCCESS",
    "SCHED_AUTO", "SCHED_THREAD", "SCHED_GROUP4", "SCHED_GROUP8", "SCHED_WARP",
    "SCHED_MERGE", "SCHED_ROW", "SCHED_WTILE", "SCHED_WMERGE", "SCHED_SEG", "CG_F64",
    "CG_MIXED",
    "CG_PLAIN_ENTRIES", "plan_tiles",
    "Server", "ServerResult",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgooseberry_b200.so")

SUCCESS = 1
ERROR_NAMES = {
    1: "SUCCESS", 2: "UNIMPLEMENTED", 3: "INVALIDINPUT", 4: "READ", 5: "WRITE",
    6: "FILENOTFOUND", 7: "PERMISSIONDENIED", 8: "UNKNOWN",
}
VALUES_F64, VALUES_F32, DEVICE_POINTERS = 0x1, 0x2, 0x4
(SCHED_AUTO, SCHED_THREAD, SCHED_GROUP4, SCHED_GROUP8, SCHED_WARP, SCHED_MERGE, SCHED_ROW,
 SCHED_WTILE, SCHED_WMERGE, SCHED_SEG) = range(10)
SCHED_NAMES = {0: "auto", 1: "thread", 2: "group4", 3: "group8", 4: "warp", 5: "merge",
               6: "row", 7: "wtile", 8: "wmerge", 9: "seg"}
CG_F64, CG_MIXED = 0, 1
CG_PERSISTENT = 0x100
CG_PLAIN_ENTRIES = 0x200
CG_STATUS = {0: "converged", 1: "maxiter", 2: "breakdown", 3: "nonfinite", 4: "cancelled",
             5: "timeout"}


class GooseberryError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class CsrInfo(C.Structure):
    _fields_ = [("nrows", C.c_uint32), ("ncols", C.c_uint32), ("nnz", C.c_uint32),
                ("ntiles", C.c_uint32), ("nlong", C.c_uint32), ("max_row", C.c_uint32),
                ("mean_row", C.c_double), ("row_p50", C.c_uint32), ("row_p90", C.c_uint32),
                ("row_p99", C.c_uint32), ("schedule", C.c_int), ("schedule_f32", C.c_int),
                ("tile_items", C.c_uint32)]


class _CgResult(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("refinements", C.c_size_t),
                ("rnorm", C.c_double), ("bnorm", C.c_double), ("status", C.c_int),
                ("kernel_launches", C.c_size_t)]


_LIB = None

_vp, _u32, _sz, _d, _f, _i = C.c_void_p, C.c_uint32, C.c_size_t, C.c_double, C.c_float, C.c_int

# name -> (restype, argtypes); every symbol the headers declare
SIGNATURES = {
    "gb_last_error": (C.c_char_p, []),
    "gooseberry_scale": (_i, [_u32, _vp, _f]),
    "gooseberry_scale_f64": (_i, [_u32, _vp, _d]),
    "gooseberry_add_scalar": (_i, [_u32, _vp, _f]),
    "gooseberry_add_scalar_f64": (_i, [_u32, _vp, _d]),
    "gooseberry_spmult": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _u32]),
    "gooseberry_spmult_f64": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _vp, _vp, _vp, _u32]),
    "gooseberry_cgd": (_i, [_u32, _vp, _vp, _vp, _vp, _vp, _f, _sz, _vp, _vp, _vp, _sz]),
    "gooseberry_cgd_f64": (_i, [_u32, _vp, _vp, _vp, _vp, _vp, _d, _sz, _vp, _vp, _vp, _sz]),
    "gooseberry_pagerank": (_i, [_u32, _vp, _vp, _vp, _f, _f, _sz, _vp, _vp, _vp]),
    "gooseberry_pagerank_f64": (_i, [_u32, _vp, _vp, _vp, _d, _d, _sz, _vp, _vp, _vp]),
    "gooseberry_read_sparse_matrix": (_i, [_i, C.c_char_p, _vp, _vp, _vp, _vp, _vp]),
    "gooseberry_read_sparse_matrix_f64": (_i, [_i, C.c_char_p, _vp, _vp, _vp, _vp, _vp]),
    "gooseberry_read_dense_matrix": (_i, [_i, C.c_char_p, _vp, _vp, _vp]),
    "gooseberry_read_dense_matrix_f64": (_i, [_i, C.c_char_p, _vp, _vp, _vp]),
    "gooseberry_write_dense_matrix": (_i, [_i, C.c_char_p, _u32, _u32, _vp]),
    "gooseberry_write_dense_matrix_f64": (_i, [_i, C.c_char_p, _u32, _u32, _vp]),
    "gooseberry_write_sparse_matrix": (_i, [_i, C.c_char_p, _u32, _u32, _vp, _vp, _vp]),
    "gooseberry_write_sparse_matrix_f64": (_i, [_i, C.c_char_p, _u32, _u32, _vp, _vp, _vp]),
    "gooseberry_permute_cuthillmckee": (_i, [_u32, _u32, _vp, _vp, _vp, _vp, _u32, _vp]),
    "gooseberry_permute_sparse": (_i, [_u32, _u32, _vp, _vp, _vp, _vp, _vp]),
    "gooseberry_permute_sparse_f64": (_i, [_u32, _u32, _vp, _vp, _vp, _vp, _vp]),
    "gooseberry_permute_dense": (_i, [_u32, _u32, _vp, _vp, _vp]),
    "gooseberry_permute_dense_f64": (_i, [_u32, _u32, _vp, _vp, _vp]),
    "gooseberry_permute_dense_rev": (_i, [_u32, _u32, _vp, _vp, _vp]),
    "gooseberry_permute_dense_rev_f64": (_i, [_u32, _u32, _vp, _vp, _vp]),
    "gb_csr_cuthillmckee": (_i, [_vp, _vp, _u32, _vp, _vp]),
    "gb_csr_permute": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "gb_permute_vector_f64": (_i, [_sz, _vp, _vp, _i, _vp, _vp]),
    "gb_csr_create": (_i, [_u32, _u32, _u32, _vp, _vp, _vp, _vp, C.c_uint, _vp, _vp]),
    "gb_csr_read": (_i, [C.c_char_p, C.c_uint, _vp, _vp]),
    "gb_csr_destroy": (_i, [_vp]),
    "gb_csr_get_info": (_i, [_vp, _vp]),
    "gb_csr_set_schedule": (_i, [_vp, C.c_uint, _i, _u32]),
    "gb_csr_autotune": (_i, [_vp, C.c_uint, _vp]),
    "gb_plan_tiles_host": (_i, [_u32, _vp, _u32, _u32, _vp, _sz, _vp, _vp, _vp]),
    "gb_spmv_f64": (_i, [_vp, _vp, _vp, _vp]),
    "gb_spmv_f32": (_i, [_vp, _vp, _vp, _vp]),
    "gb_spmm_f64": (_i, [_vp, _u32, _vp, _vp, _vp]),
    "gb_dot_f64": (_i, [_sz, _vp, _vp, _vp, _vp]),
    "gb_dot_f32": (_i, [_sz, _vp, _vp, _vp, _vp]),
    "gb_spdot_f64": (_i, [_sz, _vp, _vp, _vp, _sz, _vp, _vp]),
    "gb_spdot_f32": (_i, [_sz, _vp, _vp, _vp, _sz, _vp, _vp]),
    "gb_dot_f64_noalloc": (_i, [_sz, _vp, _vp, _vp, _vp]),
    "gb_scale_f64": (_i, [_sz, _vp, _d, _vp]),
    "gb_add_scalar_f64": (_i, [_sz, _vp, _d, _vp]),
    "gb_add_f64": (_i, [_sz, _vp, _vp, _vp, _vp]),
    "gb_sub_f64": (_i, [_sz, _vp, _vp, _vp, _vp]),
    "gb_scale_f32": (_i, [_sz, _vp, _f, _vp]),
    "gb_add_scalar_f32": (_i, [_sz, _vp, _f, _vp]),
    "gb_cg_create": (_i, [_vp, _i, _vp]),
    "gb_cg_destroy": (_i, [_vp]),
    "gb_cg_solve": (_i, [_vp, _vp, _vp, _d, _i, _sz, _vp, _sz, _vp, _vp]),
    "gb_cg_profile": (_i, [_vp, _vp, _sz, _vp, _sz, _vp, _vp]),
    "gb_cg_entry_bytes": (_i, [_vp, _vp]),
    "gb_cg_row_bytes": (_i, [_vp, _vp]),
    "gb_cg_cancel": (_i, [_vp]),
    "gb_cg_set_barrier_fault": (_i, [_vp, C.c_int, C.c_uint]),
    "gb_server_cancel": (_i, [_vp, C.c_uint64]),
    "gb_server_stats": (_i, [_vp, _vp]),
    "gb_server_tuned_tile_rows": (_i, [C.c_int, C.c_uint32, C.c_uint32, _vp]),
    "gb_server_create": (_i, [_vp, _vp]),
    "gb_server_destroy": (_i, [_vp]),
    "gb_server_submit": (_i, [_vp, C.c_uint64, _u32, _vp, _vp, _vp, _vp, _vp, _d, _sz]),
    "gb_server_step": (_i, [_vp, _vp, _vp]),
    "gb_server_poll": (_i, [_vp, _vp, _sz, _vp]),
    "gb_server_clock": (_d, [_vp]),
}


def lib():
    """The loaded C library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m gooseberry_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def last_error() -> str:
    return (lib().gb_last_error() or b"").decode(errors="replace")


def _check(rc: int, where: str) -> None:
    if rc != SUCCESS:
        raise GooseberryError(rc, where, last_error())


def _ptr(a) -> int | None:
    """Data pointer of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


# ---- host-pointer API (the reference's entry points) ----------------------------

def _real(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"values must be float32 or float64, got {dt}")


def spmult(rowptr, rowind, rowval, B, ncols: int | None = None, bncols: int = 1,
           blocks=None, out=None):
    """C = A B through ``gooseberry_spmult`` (reference ``include/gooseberry.h:174-184``).

    ``B`` is column-major (``B[j*ncols + l]``), the result row-major
    (``C[i*bncols + j]``).  float64 values use ``gooseberry_spmult_f64``,
    float32 the float ABI.  With ``blocks`` only those row ranges are written
    (``out`` keeps its other rows)."""
    rowval = np.ascontiguousarray(rowval)
    real = _real(rowval.dtype)
    dt = rowval.dtype
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    B = np.ascontiguousarray(B, dtype=dt).reshape(-1)
    n = len(rowptr) - 1
    ncols = n if ncols is None else int(ncols)
    if out is None:
        out = np.zeros(n * bncols, dtype=dt)
    assert out.dtype == dt and out.flags.c_contiguous and out.size >= n * bncols
    bl = None if blocks is None else np.ascontiguousarray(blocks, dtype=np.uint32)
    nb = 0 if bl is None else len(bl) - 1
    fn = lib().gooseberry_spmult_f64 if real == "f64" else lib().gooseberry_spmult
    _check(fn(n, ncols, bncols, _ptr(rowptr), _ptr(rowind), _ptr(rowval), _ptr(B),
              _ptr(out), _ptr(bl), nb), "gooseberry_spmult")
    return out


def scale(v: np.ndarray, s: float) -> np.ndarray:
    """v *= s in place through ``gooseberry_scale`` (``include/gooseberry.h:134-137``)."""
    real = _real(v.dtype)
    assert v.flags.c_contiguous
    fn = lib().gooseberry_scale_f64 if real == "f64" else lib().gooseberry_scale
    _check(fn(v.size, _ptr(v), s), "gooseberry_scale")
    return v


def add_scalar(v: np.ndarray, s: float) -> np.ndarray:
    """v += s in place through ``gooseberry_add_scalar`` (``include/gooseberry.h:150-153``)."""
    real = _real(v.dtype)
    assert v.flags.c_contiguous
    fn = lib().gooseberry_add_scalar_f64 if real == "f64" else lib().gooseberry_add_scalar
    _check(fn(v.size, _ptr(v), s), "gooseberry_add_scalar")
    return v


def cgd(rowptr, rowind, rowval, b, error: float, niter: int, history: bool = False,
        out=None):
    """Conjugate gradient with the reference's contract (``src/cgd.c:40-129``):
    x0 = 0, stop when ||r||_2 <= error (absolute) or after niter iterations.

    ``out``: optional contiguous host array (n entries of the value type) that
    receives x -- e.g. pinned memory, which the final device-to-host copy
    reaches without staging.  Returns ``(x, iterations, rnorm)`` (plus the
    ||r|| history if asked)."""
    rowval = np.ascontiguousarray(rowval)
    real = _real(rowval.dtype)
    dt = rowval.dtype
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=dt)
    n = len(b)
    if out is None:
        x = np.zeros(n, dtype=dt)
    else:
        if out.dtype != dt or out.shape != (n,) or not out.flags["C_CONTIGUOUS"] \
                or not out.flags["WRITEABLE"]:
            raise ValueError(f"out must be a writable contiguous {dt} array of {n} entries")
        x = out
    it = C.c_size_t(0)
    rn = C.c_double(0)
    hist = np.zeros(max(int(niter), 1), dtype=np.float64) if history else None
    fn = lib().gooseberry_cgd_f64 if real == "f64" else lib().gooseberry_cgd
    _check(fn(n, _ptr(rowptr), _ptr(rowind), _ptr(rowval), _ptr(b), _ptr(x), error,
              int(niter), C.addressof(it), C.addressof(rn), _ptr(hist),
              0 if hist is None else len(hist)), "gooseberry_cgd")
    if history:
        return x, int(it.value), rn.value, hist[: it.value]
    return x, int(it.value), rn.value


def pagerank(rowptr, rowind, rowval, damping: float = 0.85, minerror: float = 0.0,
             niter: int = 0):
    """PageRank with the reference's contract (``src/gooseberry_bin.c:2610-2741``,
    see ``gooseberry_pagerank``).  Returns ``(rank, iterations, error)``."""
    rowval = np.ascontiguousarray(rowval)
    real = _real(rowval.dtype)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    n = len(rowptr) - 1
    rank = np.zeros(n, dtype=rowval.dtype)
    it = C.c_size_t(0)
    err = C.c_double(0)
    fn = lib().gooseberry_pagerank_f64 if real == "f64" else lib().gooseberry_pagerank
    _check(fn(n, _ptr(rowptr), _ptr(rowind), _ptr(rowval), damping, minerror, int(niter),
              _ptr(rank), C.addressof(it), C.addressof(err)), "gooseberry_pagerank")
    return rank, int(it.value), err.value


FORMAT_GRID, FORMAT_CSR = 1, 2  # gooseberry_format_t
_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]
_libc.free.restype = None


class _MallocBuffer:
    """A malloc'ed C array seen as a numpy array without a copy; freed when the
    last array that uses it goes away."""

    def __init__(self, addr: int, n: int, dtype):
        self._addr = addr
        self.__array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str,
                                    "data": (addr, False), "version": 3}

    def __del__(self):
        _libc.free(C.c_void_p(self._addr))


def _take(ptr, ctype, n, dtype):
    """n elements of a malloc'ed C array as a numpy array that owns it."""
    if n and ptr.value:
        return np.asarray(_MallocBuffer(ptr.value, n, dtype))
    _libc.free(ptr)
    return np.zeros(0, dtype=dtype)


def read_csr(path, f64: bool = True):
    """Read a CSR text file (``gooseberry_read_sparse_matrix``, the reference's
    format, src/io.c:369-498).  Returns ``(rowptr, rowind, rowval, ncols)``."""
    nr, nc = C.c_uint32(0), C.c_uint32(0)
    rp, ri, rv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    fn = lib().gooseberry_read_sparse_matrix_f64 if f64 else lib().gooseberry_read_sparse_matrix
    _check(fn(FORMAT_CSR, str(path).encode(), C.addressof(nr), C.addressof(nc),
              C.addressof(rp), C.addressof(ri), C.addressof(rv)), "gooseberry_read_sparse_matrix")
    n = nr.value
    rowptr = _take(rp, C.c_uint32, n + 1, np.uint32)
    nnz = int(rowptr[-1])
    rowind = _take(ri, C.c_uint32, nnz, np.uint32)
    rowval = _take(rv, C.c_double if f64 else C.c_float, nnz,
                   np.float64 if f64 else np.float32)
    return rowptr, rowind, rowval, nc.value


def read_grid(path, f64: bool = True):
    """Read a grid (dense) text file (src/io.c:145-239).  Returns a 2-D array."""
    nr, nc = C.c_uint32(0), C.c_uint32(0)
    rv = C.c_void_p()
    fn = lib().gooseberry_read_dense_matrix_f64 if f64 else lib().gooseberry_read_dense_matrix
    _check(fn(FORMAT_GRID, str(path).encode(), C.addressof(nr), C.addressof(nc),
              C.addressof(rv)), "gooseberry_read_dense_matrix")
    vals = _take(rv, C.c_double if f64 else C.c_float, nr.value * nc.value,
                 np.float64 if f64 else np.float32)
    return vals.reshape(nr.value, nc.value)


def write_grid(path, values):
    """Write a 2-D array as a grid text file (src/io.c:1195-1229)."""
    v = np.ascontiguousarray(values)
    if v.ndim == 1:
        v = v.reshape(-1, 1)
    f64 = _real(v.dtype) == "f64"
    fn = lib().gooseberry_write_dense_matrix_f64 if f64 else lib().gooseberry_write_dense_matrix
    _check(fn(FORMAT_GRID, str(path).encode(), v.shape[0], v.shape[1], _ptr(v)),
           "gooseberry_write_dense_matrix")


def write_csr(path, rowptr, rowind, rowval, ncols: int = 0):
    """Write a CSR text file (src/io.c:1233-1275)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval)
    f64 = _real(rowval.dtype) == "f64"
    fn = (lib().gooseberry_write_sparse_matrix_f64 if f64
          else lib().gooseberry_write_sparse_matrix)
    _check(fn(FORMAT_CSR, str(path).encode(), len(rowptr) - 1, ncols, _ptr(rowptr),
              _ptr(rowind), _ptr(rowval)), "gooseberry_write_sparse_matrix")


def cuthillmckee(rowptr, rowind, nrows: int, ncols: int | None = None, blocks=None):
    """Cuthill-McKee order of a host CSR (``gooseberry_permute_cuthillmckee``,
    reference src/permute.c:288-337), computed on the GPU: ``perm[new] = old``.
    ``blocks`` (nblocks+1 row boundaries) orders each diagonal block alone."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    ncols = nrows if ncols is None else int(ncols)
    perm = np.zeros(max(nrows, 1), dtype=np.uint32)
    b = None if blocks is None else np.ascontiguousarray(blocks, dtype=np.uint32)
    nb = 0 if b is None else len(b) - 1
    _check(lib().gooseberry_permute_cuthillmckee(nrows, ncols, _ptr(rowptr), _ptr(rowind), None,
                                                 _ptr(b), nb, _ptr(perm)),
           "gooseberry_permute_cuthillmckee")
    return perm[:nrows]


def permute_sparse(rowptr, rowind, rowval, ncols: int, rowperm=None, colperm=None):
    """Permuted copy of a host CSR (``gooseberry_permute_sparse[_f64]``, reference
    src/permute.c:120-205): new row i is row ``rowperm[i]``, column
    ``colperm[j]`` becomes j.  Returns ``(rowptr, rowind, rowval)``."""
    rowptr = np.array(rowptr, dtype=np.uint32)
    rowind = np.array(rowind, dtype=np.uint32)
    real = _real(np.asarray(rowval).dtype)
    rowval = np.array(rowval, dtype=np.float64 if real == "f64" else np.float32)
    rp = None if rowperm is None else np.ascontiguousarray(rowperm, dtype=np.uint32)
    cp = None if colperm is None else np.ascontiguousarray(colperm, dtype=np.uint32)
    fn = lib().gooseberry_permute_sparse_f64 if real == "f64" else lib().gooseberry_permute_sparse
    _check(fn(len(rowptr) - 1, ncols, _ptr(rowptr), _ptr(rowind), _ptr(rowval), _ptr(rp),
              _ptr(cp)), "gooseberry_permute_sparse")
    return rowptr, rowind, rowval


def permute_dense(vals, nrows: int, ncols: int, rowperm=None, colperm=None,
                  reverse: bool = False):
    """Permuted copy of a row-major host matrix (``gooseberry_permute_dense``
    / ``_rev``, reference src/permute.c:208-283): forward ``out[i][j] =
    in[rowperm[i]][colperm[j]]``, reverse ``out[rowperm[i]][colperm[j]] =
    in[i][j]``."""
    real = _real(np.asarray(vals).dtype)
    a = np.array(vals, dtype=np.float64 if real == "f64" else np.float32).reshape(-1)
    rp = None if rowperm is None else np.ascontiguousarray(rowperm, dtype=np.uint32)
    cp = None if colperm is None else np.ascontiguousarray(colperm, dtype=np.uint32)
    name = "gooseberry_permute_dense" + ("_rev" if reverse else "") + (
        "_f64" if real == "f64" else "")
    _check(getattr(lib(), name)(nrows, ncols, _ptr(a), _ptr(rp), _ptr(cp)), name)
    return a


def permute_vector(x, perm, reverse: bool = False, stream=None):
    """``y[i] = x[perm[i]]`` (or ``y[perm[i]] = x[i]`` with ``reverse``) for
    float64 CUDA tensors; ``perm`` a uint32/int32 CUDA tensor."""
    torch = _torch()
    y = torch.empty_like(x)
    _check(lib().gb_permute_vector_f64(x.numel(), x.data_ptr(), perm.data_ptr(), int(reverse),
                                       y.data_ptr(), _stream_ptr(stream)),
           "gb_permute_vector_f64")
    return y


def plan_tiles(rowptr, tile_items: int = 2048):
    """Run the SpMV tile planner on a host rowptr (no GPU).  Returns
    ``(tiles[ntiles, 4], nlong, info)``; see ``gb_plan_tiles_host``."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    n = len(rowptr) - 1
    nt, nl = C.c_uint32(0), C.c_uint32(0)
    info = CsrInfo()
    _check(lib().gb_plan_tiles_host(n, _ptr(rowptr), int(rowptr[-1]), tile_items, None, 0,
                                    C.addressof(nt), C.addressof(nl), C.addressof(info)),
           "gb_plan_tiles_host")
    tiles = np.zeros((max(nt.value, 1), 4), dtype=np.uint32)
    _check(lib().gb_plan_tiles_host(n, _ptr(rowptr), int(rowptr[-1]), tile_items,
                                    _ptr(tiles), nt.value, None, None, None),
           "gb_plan_tiles_host")
    return tiles[: nt.value], nl.value, info


# ---- device API ----------------------------------------------------------------------

def _torch():
    import torch
    return torch


def dot(a, b, stream=None) -> float:
    """sum a*b of two CUDA tensors (float64 accumulation, fixed order)."""
    torch = _torch()
    out = torch.empty(1, dtype=torch.float64, device=a.device)
    fn = lib().gb_dot_f64 if a.dtype == torch.float64 else lib().gb_dot_f32
    _check(fn(a.numel(), a.data_ptr(), b.data_ptr(), out.data_ptr(), _stream_ptr(stream)),
           "gb_dot")
    return float(out.item())


def add(a, b, out=None, stream=None):
    """out = a + b for float64 CUDA tensors (``gb_add_f64``, the reference's
    blas_add, ``src/blas.c:275-290``); ``out`` may be ``a`` or ``b``."""
    return _axpby(a, b, out, "gb_add_f64", stream)


def sub(a, b, out=None, stream=None):
    """out = a - b for float64 CUDA tensors (``gb_sub_f64``, the reference's
    blas_sub, ``src/blas.c:321-336``); ``out`` may be ``a`` or ``b``."""
    return _axpby(a, b, out, "gb_sub_f64", stream)


def _axpby(a, b, out, name, stream):
    torch = _torch()
    if out is None:
        out = torch.empty_like(a)
    assert a.dtype == b.dtype == out.dtype == torch.float64
    assert a.is_contiguous() and b.is_contiguous() and out.is_contiguous()
    assert a.numel() == b.numel() == out.numel()
    _check(getattr(lib(), name)(a.numel(), a.data_ptr(), b.data_ptr(), out.data_ptr(),
                                _stream_ptr(stream)), name)
    return out


def spdot(ind, val, x, stream=None) -> float:
    """sum val[k] * x[ind[k]] for CUDA tensors (ind uint32/int32, val and x of
    one float type; float64 accumulation, fixed order)."""
    torch = _torch()
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    fn = lib().gb_spdot_f64 if x.dtype == torch.float64 else lib().gb_spdot_f32
    _check(fn(ind.numel(), ind.data_ptr(), val.data_ptr(), x.data_ptr(), x.numel(),
              out.data_ptr(), _stream_ptr(stream)), "gb_spdot")
    return float(out.item())


class CsrMatrix:
    """A device-resident CSR matrix (``gb_csr_t``)."""

    def __init__(self, handle: int, nrows: int, ncols: int, nnz: int, keep=()):
        self._h = C.c_void_p(handle)
        self.nrows, self.ncols, self.nnz = nrows, ncols, nnz
        self._keep = keep  # borrowed device tensors must outlive the handle

    @classmethod
    def read(cls, path, f64: bool = True, f32: bool = False, stream=None) -> "CsrMatrix":
        """Read a CSR text file straight into a device matrix (``gb_csr_read``)."""
        h = C.c_void_p()
        flags = (VALUES_F64 if f64 else 0) | (VALUES_F32 if f32 else 0)
        _check(lib().gb_csr_read(str(path).encode(), flags, _stream_ptr(stream),
                                 C.addressof(h)), "gb_csr_read")
        info = CsrInfo()
        _check(lib().gb_csr_get_info(h, C.addressof(info)), "gb_csr_get_info")
        m = cls(h.value, info.nrows, info.ncols, info.nnz)
        return m

    @classmethod
    def from_host(cls, csr=None, *, rowptr=None, rowind=None, rowval=None, ncols=None,
                  f64: bool = True, f32: bool = False, stream=None) -> "CsrMatrix":
        """Upload a host CSR (numpy arrays or a ``workloads.Csr``)."""
        if csr is not None:
            rowptr, rowind, rowval, ncols = csr.rowptr, csr.rowind, csr.rowval, csr.ncols
        rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
        rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
        v64 = np.ascontiguousarray(rowval, dtype=np.float64)
        n = len(rowptr) - 1
        ncols = n if ncols is None else int(ncols)
        flags = (VALUES_F64 if f64 else 0) | (VALUES_F32 if f32 else 0)
        h = C.c_void_p()
        _check(lib().gb_csr_create(n, ncols, int(rowptr[-1]), _ptr(rowptr), _ptr(rowind),
                                   _ptr(v64), None, flags,
                                   _stream_ptr(stream) if stream is not None else None,
                                   C.addressof(h)), "gb_csr_create")
        return cls(h.value, n, ncols, int(rowptr[-1]))

    @classmethod
    def from_device(cls, rowptr, rowind, val64=None, val32=None, ncols=None,
                    stream=None) -> "CsrMatrix":
        """Borrow CSR arrays that are already CUDA tensors (uint32/int32 indices)."""
        n = rowptr.numel() - 1
        ncols = n if ncols is None else int(ncols)
        flags = DEVICE_POINTERS | (VALUES_F64 if val64 is not None else 0) | (
            VALUES_F32 if val32 is not None else 0)
        h = C.c_void_p()
        _check(lib().gb_csr_create(n, ncols, rowind.numel(), rowptr.data_ptr(),
                                   rowind.data_ptr(), _ptr(val64), _ptr(val32), flags,
                                   _stream_ptr(stream), C.addressof(h)), "gb_csr_create")
        return cls(h.value, n, ncols, rowind.numel(), keep=(rowptr, rowind, val64, val32))

    def close(self):
        if self._h and self._h.value:
            lib().gb_csr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        return self._h.value

    def info(self) -> CsrInfo:
        i = CsrInfo()
        _check(lib().gb_csr_get_info(self._h, C.addressof(i)), "gb_csr_get_info")
        return i

    def set_schedule(self, schedule: int, tile_items: int = 0, f32: bool = False):
        _check(lib().gb_csr_set_schedule(self._h, VALUES_F32 if f32 else VALUES_F64,
                                         schedule, tile_items), "gb_csr_set_schedule")

    def autotune(self, f32: bool = False, stream=None):
        _check(lib().gb_csr_autotune(self._h, VALUES_F32 if f32 else VALUES_F64,
                                     _stream_ptr(stream)), "gb_csr_autotune")

    def spmv(self, x, y=None, stream=None):
        """y = A x for CUDA tensors (float64 or float32)."""
        torch = _torch()
        if y is None:
            y = torch.empty(self.nrows, dtype=x.dtype, device=x.device)
        assert x.is_contiguous() and y.is_contiguous() and x.dtype == y.dtype
        fn = lib().gb_spmv_f64 if x.dtype == torch.float64 else lib().gb_spmv_f32
        _check(fn(self._h, x.data_ptr(), y.data_ptr(), _stream_ptr(stream)), "gb_spmv")
        return y

    def cuthillmckee(self, blocks=None, stream=None):
        """Cuthill-McKee order on the device (``gb_csr_cuthillmckee``): an int32
        CUDA tensor ``perm`` with ``perm[new] = old``."""
        torch = _torch()
        perm = torch.empty(max(self.nrows, 1), dtype=torch.int32, device="cuda")
        b = None if blocks is None else np.ascontiguousarray(blocks, dtype=np.uint32)
        nb = 0 if b is None else len(b) - 1
        _check(lib().gb_csr_cuthillmckee(self._h, _ptr(b), nb, perm.data_ptr(),
                                         _stream_ptr(stream)), "gb_csr_cuthillmckee")
        return perm[: self.nrows]

    def permute(self, rowperm=None, colperm=None, stream=None) -> "CsrMatrix":
        """A new matrix with rows ``rowperm`` and columns renamed by ``colperm``
        (int32/uint32 CUDA tensors or None; ``gb_csr_permute``)."""
        h = C.c_void_p()
        _check(lib().gb_csr_permute(self._h, _ptr(rowperm), _ptr(colperm), _stream_ptr(stream),
                                    C.addressof(h)), "gb_csr_permute")
        return CsrMatrix(h.value, self.nrows, self.ncols, self.nnz)

    def spmm(self, B, bncols: int, out=None, stream=None):
        torch = _torch()
        if out is None:
            out = torch.empty(self.nrows * bncols, dtype=torch.float64, device=B.device)
        _check(lib().gb_spmm_f64(self._h, bncols, B.data_ptr(), out.data_ptr(),
                                 _stream_ptr(stream)), "gb_spmm_f64")
        return out


@dataclass
class CgResult:
    iterations: int
    refinements: int
    rnorm: float
    bnorm: float
    status: str
    kernel_launches: int


class CgSolver:
    """CG workspace bound to one matrix (``gb_cg_t``)."""

    def __init__(self, A: CsrMatrix, mode: int = CG_F64, persistent: bool = False,
                 plain_entries: bool = False):
        self.A = A
        h = C.c_void_p()
        flags = mode | (CG_PERSISTENT if persistent else 0) | (
            CG_PLAIN_ENTRIES if plain_entries else 0)
        _check(lib().gb_cg_create(A._h, flags, C.addressof(h)), "gb_cg_create")
        self._h = h

    def close(self):
        if self._h and self._h.value:
            lib().gb_cg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, b, x=None, tol: float = 1e-8, relative: bool = True, niter: int = 0,
              history: bool = False, stream=None):
        torch = _torch()
        if x is None:
            x = torch.empty_like(b)
        res = _CgResult()
        hist = np.zeros(max(int(niter), 1), dtype=np.float64) if history else None
        _check(lib().gb_cg_solve(self._h, b.data_ptr(), x.data_ptr(), tol, int(relative),
                                 int(niter), _ptr(hist), 0 if hist is None else len(hist),
                                 C.addressof(res), _stream_ptr(stream)), "gb_cg_solve")
        out = CgResult(res.iterations, res.refinements, res.rnorm, res.bnorm,
                       CG_STATUS.get(res.status, str(res.status)), res.kernel_launches)
        if history:
            return x, out, hist[: res.iterations]
        return x, out

    def cancel(self):
        """Stop the solve running on another thread (``gb_cg_cancel``); with
        no solve running, the next solve stops at its first check."""
        _check(lib().gb_cg_cancel(self._h), "gb_cg_cancel")

    def set_barrier_fault(self, drop_cta: int = -1, limit_ms: int = 0):
        """Failure-path hook of a persistent solver (``gb_cg_set_barrier_fault``):
        CTA ``drop_cta`` skips the first grid barrier of the following solves,
        which then give up after ``limit_ms`` (0: the 2 s default) and raise
        (status "timeout"); ``drop_cta < 0`` turns it off."""
        _check(lib().gb_cg_set_barrier_fault(self._h, int(drop_cta), int(limit_ms)),
               "gb_cg_set_barrier_fault")

    def entry_bytes(self) -> int:
        """Bytes per matrix entry the solver's SpMV streams (12 = plain CSR)."""
        v = C.c_size_t(0)
        _check(lib().gb_cg_entry_bytes(self._h, C.addressof(v)), "gb_cg_entry_bytes")
        return int(v.value)

    def row_bytes(self) -> int:
        """Bytes per row the solver's SpMV streams besides the entries (4 =
        rowptr; 5 with a column-pattern byte)."""
        v = C.c_size_t(0)
        _check(lib().gb_cg_row_bytes(self._h, C.addressof(v)), "gb_cg_row_bytes")
        return int(v.value)

    def profile(self, b, iterations: int = 20, stream=None):
        """Mean device time (ms) of each kernel of one iteration, timed launch
        by launch with CUDA events over the first `iterations` iterations."""
        ms = np.zeros(4, dtype=np.float64)
        nk = C.c_size_t(0)
        _check(lib().gb_cg_profile(self._h, b.data_ptr(), int(iterations), _ptr(ms), 4,
                                   C.addressof(nk), _stream_ptr(stream)), "gb_cg_profile")
        return ms[: nk.value].tolist()


# ---- batched solve server ------------------------------------------------------------

class _ServerConfig(C.Structure):
    _fields_ = [("pool_bytes", C.c_size_t), ("max_slots", C.c_uint32), ("mode", C.c_int),
                ("iters_per_step", C.c_uint32), ("tile_rows", C.c_uint32)]


class _ServerStats(C.Structure):
    _fields_ = [("steps", C.c_size_t), ("gpu_ms", C.c_double), ("wait_ms", C.c_double),
                ("host_ms", C.c_double), ("submit_ms", C.c_double), ("tunings", C.c_size_t)]


class _ServerResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("iterations", C.c_size_t), ("refinements", C.c_size_t),
                ("rnorm", C.c_double), ("bnorm", C.c_double), ("status", C.c_int),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


@dataclass
class ServerResult:
    id: int
    iterations: int
    refinements: int
    rnorm: float
    bnorm: float
    status: str
    t_submit: float
    t_admit: float
    t_done: float
    x: np.ndarray


def server_tuned_tile_rows(mode: int, n: int, max_row_nnz: int) -> int:
    """The serving tile autotuner's cached tile size for requests of this
    class (``gb_server_tuned_tile_rows``); 0 when not tuned yet."""
    v = C.c_uint32(0)
    _check(lib().gb_server_tuned_tile_rows(int(mode), int(n), int(max_row_nnz),
                                           C.addressof(v)), "gb_server_tuned_tile_rows")
    return int(v.value)


class Server:
    """Continuous-batching CG server (``gb_server_t``): submit host CSR
    systems, call ``step()`` repeatedly, collect results with ``poll()``."""

    def __init__(self, pool_bytes: int = 16 << 30, max_slots: int = 128,
                 mode: int = CG_MIXED, iters_per_step: int = 16, tile_rows: int = 0):
        cfg = _ServerConfig(pool_bytes, max_slots, mode, iters_per_step, tile_rows)
        h = C.c_void_p()
        _check(lib().gb_server_create(C.addressof(cfg), C.addressof(h)), "gb_server_create")
        self._h = h
        self._out = {}  # id -> x buffer kept alive until reported

    def close(self):
        if self._h and self._h.value:
            lib().gb_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, rid: int, csr, b, tol: float = 1e-10, niter: int = 0, x_out=None):
        rowptr = np.ascontiguousarray(csr.rowptr, dtype=np.uint32)
        rowind = np.ascontiguousarray(csr.rowind, dtype=np.uint32)
        rowval = np.ascontiguousarray(csr.rowval, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(len(b)) if x_out is None else x_out
        _check(lib().gb_server_submit(self._h, int(rid), len(b), _ptr(rowptr), _ptr(rowind),
                                      _ptr(rowval), _ptr(b), _ptr(x), float(tol), int(niter)),
               "gb_server_submit")
        self._out[int(rid)] = x

    def step(self):
        a, q = C.c_size_t(0), C.c_size_t(0)
        _check(lib().gb_server_step(self._h, C.addressof(a), C.addressof(q)), "gb_server_step")
        return a.value, q.value

    def poll(self, max_results: int = 4096):
        buf = (_ServerResult * max_results)()
        cnt = C.c_size_t(0)
        _check(lib().gb_server_poll(self._h, C.addressof(buf), max_results, C.addressof(cnt)),
               "gb_server_poll")
        out = []
        for i in range(cnt.value):
            r = buf[i]
            out.append(ServerResult(r.id, r.iterations, r.refinements, r.rnorm, r.bnorm,
                                    CG_STATUS.get(r.status, str(r.status)), r.t_submit,
                                    r.t_admit, r.t_done, self._out.pop(int(r.id))))
        return out

    def cancel(self, rid: int):
        """Cancel a queued or resident request (``gb_server_cancel``); it is
        reported by ``poll`` with status "cancelled" (x_out untouched)."""
        _check(lib().gb_server_cancel(self._h, int(rid)), "gb_server_cancel")

    def clock(self) -> float:
        return float(lib().gb_server_clock(self._h))

    def stats(self) -> dict:
        """Where the server's time went (``gb_server_stats``): graph replays and
        their device ms, host ms waiting for them and doing the rest of each
        step, host ms in submit, tile autotuner runs."""
        st = _ServerStats()
        _check(lib().gb_server_stats(self._h, C.addressof(st)), "gb_server_stats")
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def drain(self, timeout_s: float = 600.0):
        """Step until every submitted request is reported."""
        import time
        res = []
        t0 = time.time()
        while self._out and time.time() - t0 < timeout_s:
            self.step()
            res += self.poll()
        return res
