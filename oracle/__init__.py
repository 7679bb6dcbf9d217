"""CPU oracle for the SpMV / CG hot path -- TEST INFRASTRUCTURE ONLY.

Two checkers, both loaded with ctypes:

* ``liboracle.so`` -- our C restatement (``oracle/gb_oracle.c``) of
  ``src/blas.c:82-91`` (per-row sequential SpMV), ``src/blas.c:413-430``
  (dot) and ``src/cgd.c:81-119`` (CG update order).
* ``_ref/libgbref_{f64,f32}.so`` -- the reference's OWN ``src/blas.c``,
  ``src/cgd.c`` and ``src/matrix.c`` compiled unmodified against a
  project-written domlib shim (``oracle/Makefile``), reached through
  ``oracle/ref_driver.c``.  Present only where it was built (it needs the
  reference sources at build time; the built files travel with the repo).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package.  The product (``gooseberry_b200``)
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def build(ref_root: str | None = None, quiet: bool = True) -> None:
    """Compile the restatement, and the reference build when its sources exist.

    ``ref_root`` is the reference checkout; None takes the environment
    variable GOOSEBERRY_REFERENCE, else the default of oracle/Makefile.  The
    reference build is skipped when that directory has no ``src/``."""
    targets = ["oracle"]
    cmd = ["make", "-C", _HERE]
    if ref_root is None:
        ref_root = os.environ.get("GOOSEBERRY_REFERENCE") or _makefile_reference()
    if ref_root and os.path.isdir(os.path.join(ref_root, "src")):
        targets.append("ref")
        cmd.append(f"REF={ref_root}")
    subprocess.run(cmd + targets, check=True, capture_output=quiet)


def _makefile_reference() -> str | None:
    """The reference checkout oracle/Makefile defaults to."""
    r = subprocess.run(["make", "-s", "-C", _HERE, "--no-print-directory", "print-ref"],
                       capture_output=True, text=True)
    return r.stdout.strip() or None if r.returncode == 0 else None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build(quiet=True)
        lib = C.CDLL(path)
        for real, p in (("f64", _f64p), ("f32", _f32p)):
            ctype = C.c_double if real == "f64" else C.c_float
            f = getattr(lib, f"oracle_spmm_{real}")
            f.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p, _u32p, p, p, p,
                          C.c_void_p, C.c_uint32, C.c_int]
            f.restype = None
            f = getattr(lib, f"oracle_dot_{real}")
            f.argtypes = [C.c_size_t, p, p]
            f.restype = ctype
            f = getattr(lib, f"oracle_spdot_{real}")
            f.argtypes = [C.c_size_t, _u32p, p, p]
            f.restype = ctype
            for nm in ("scale", "add_scalar"):
                f = getattr(lib, f"oracle_{nm}_{real}")
                f.argtypes = [C.c_size_t, p, ctype]
                f.restype = None
            if real == "f64":
                f = lib.oracle_pagerank_f64
                f.argtypes = [C.c_uint32, _u32p, _u32p, p, C.c_double, C.c_double,
                              C.c_size_t, p, C.POINTER(C.c_double)]
                f.restype = C.c_size_t
            if real == "f64":
                lib.oracle_cuthillmckee.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p,
                                                    C.c_void_p, C.c_uint32, _u32p]
                lib.oracle_cuthillmckee.restype = C.c_int
                lib.oracle_permute_sparse_f64.argtypes = [C.c_uint32, C.c_uint32, _u32p,
                                                          _u32p, p, C.c_void_p, C.c_void_p,
                                                          _u32p, _u32p, p]
                lib.oracle_permute_sparse_f64.restype = None
                lib.oracle_permute_dense_f64.argtypes = [C.c_uint32, C.c_uint32, p, p,
                                                         C.c_void_p, C.c_void_p, C.c_int]
                lib.oracle_permute_dense_f64.restype = None
            f = getattr(lib, f"oracle_cgd_{real}")
            f.argtypes = [C.c_uint32, _u32p, _u32p, p, p, p, ctype, C.c_size_t,
                          C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.c_int]
            f.restype = C.c_size_t
        _LIB = lib
    return _LIB


def ref_available(real: str = "f64") -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", f"libgbref_{real}.so"))


def _ref(real: str = "f64"):
    if real not in _REF:
        path = os.path.join(_HERE, "_ref", f"libgbref_{real}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path}")
        lib = C.CDLL(path)
        p = _f64p if real == "f64" else _f32p
        lib.gbref_real_size.restype = C.c_int
        lib.gbref_set_threads.argtypes = [C.c_int]
        lib.gbref_set_threads.restype = None
        lib.gbref_spmult.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p, _u32p,
                                     p, p, p, C.c_void_p, C.c_uint32]
        lib.gbref_spmult.restype = C.c_int
        lib.gbref_dot.argtypes = [C.c_uint32, p, p]
        lib.gbref_dot.restype = C.c_double
        for nm in ("gbref_add", "gbref_sub"):
            getattr(lib, nm).argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
            getattr(lib, nm).restype = C.c_int
        lib.gbref_spdot.argtypes = [C.c_uint32, _u32p, p, p]
        lib.gbref_spdot.restype = C.c_double
        lib.gbref_pagerank.argtypes = [C.c_uint32, _u32p, _u32p, p, C.c_double, C.c_double,
                                       C.c_size_t, p, C.POINTER(C.c_double)]
        lib.gbref_pagerank.restype = C.c_size_t
        vp = C.c_void_p
        lib.gbref_read_sparse.argtypes = [C.c_int, C.c_char_p, vp, vp, vp, vp, vp]
        lib.gbref_read_sparse.restype = C.c_int
        lib.gbref_read_dense.argtypes = [C.c_int, C.c_char_p, vp, vp, vp]
        lib.gbref_read_dense.restype = C.c_int
        lib.gbref_write_sparse.argtypes = [C.c_int, C.c_char_p, C.c_uint32, C.c_uint32,
                                           _u32p, _u32p, p]
        lib.gbref_write_sparse.restype = C.c_int
        lib.gbref_write_dense.argtypes = [C.c_int, C.c_char_p, C.c_uint32, C.c_uint32, p]
        lib.gbref_write_dense.restype = C.c_int
        lib.gbref_free.argtypes = [vp]
        lib.gbref_free.restype = None
        lib.gbref_cuthillmckee.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, vp,
                                           C.c_uint32, _u32p]
        lib.gbref_cuthillmckee.restype = C.c_int
        lib.gbref_permute_sparse.argtypes = [C.c_uint32, C.c_uint32, _u32p, _u32p, p, vp, vp]
        lib.gbref_permute_sparse.restype = C.c_int
        lib.gbref_permute_dense.argtypes = [C.c_uint32, C.c_uint32, p, vp, vp, C.c_int]
        lib.gbref_permute_dense.restype = C.c_int
        lib.gbref_cgd.argtypes = [C.c_uint32, _u32p, _u32p, p, p, p, C.c_double,
                                  C.c_size_t, C.POINTER(C.c_size_t),
                                  C.POINTER(C.c_double), C.c_void_p, C.c_size_t]
        lib.gbref_cgd.restype = C.c_int
        want = 8 if real == "f64" else 4
        if lib.gbref_real_size() != want:
            raise RuntimeError(f"{path}: real_t has {lib.gbref_real_size()} bytes")
        _REF[real] = lib
    return _REF[real]


def ref_set_threads(n: int) -> None:
    """OpenMP threads used by the reference build (both widths)."""
    for real in ("f64", "f32"):
        if ref_available(real):
            _ref(real).gbref_set_threads(int(n))


def _dt(real):
    return np.float64 if real == "f64" else np.float32


def _blocks_arg(blocks):
    if blocks is None:
        return None, 0, None
    b = np.ascontiguousarray(blocks, dtype=np.uint32)
    return b.ctypes.data_as(C.c_void_p), len(b) - 1, b


def spmm(rowptr, rowind, rowval, B, ncols=None, bncols=1, blocks=None, out=None,
         threads=1, real="f64"):
    """C = A*B via the restatement (src/blas.c:82-91).  B is column-major."""
    dt = _dt(real)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=dt)
    B = np.ascontiguousarray(B, dtype=dt).reshape(-1)
    n = len(rowptr) - 1
    ncols = n if ncols is None else ncols
    C_ = np.zeros(n * bncols, dtype=dt) if out is None else out
    bp, nb, keep = _blocks_arg(blocks)
    getattr(_lib(), f"oracle_spmm_{real}")(n, ncols, bncols, rowptr, rowind, rowval, B,
                                           C_, bp, nb, int(threads))
    del keep
    return C_


def spmv(rowptr, rowind, rowval, x, threads=1, real="f64"):
    return spmm(rowptr, rowind, rowval, x, ncols=len(x), threads=threads, real=real)


def dot(a, b, real="f64"):
    dt = _dt(real)
    a = np.ascontiguousarray(a, dtype=dt)
    b = np.ascontiguousarray(b, dtype=dt)
    return float(getattr(_lib(), f"oracle_dot_{real}")(len(a), a, b))


def spdot(ind, val, x, real="f64"):
    """Restated blas_spdot (src/blas.c:433-451): sum val[k]*x[ind[k]], k ascending."""
    dt = _dt(real)
    ind = np.ascontiguousarray(ind, dtype=np.uint32)
    val = np.ascontiguousarray(val, dtype=dt)
    x = np.ascontiguousarray(x, dtype=dt)
    return float(getattr(_lib(), f"oracle_spdot_{real}")(len(ind), ind, val, x))


def scale(v, s, real="f64"):
    v = np.array(v, dtype=_dt(real), copy=True)
    getattr(_lib(), f"oracle_scale_{real}")(len(v), v, s)
    return v


def add_scalar(v, s, real="f64"):
    v = np.array(v, dtype=_dt(real), copy=True)
    getattr(_lib(), f"oracle_add_scalar_{real}")(len(v), v, s)
    return v


def cgd(rowptr, rowind, rowval, b, error, niter, threads=1, real="f64", history=False):
    """Restated cgd (src/cgd.c:40-129).  Returns (x, iterations, last_norm[, hist])."""
    dt = _dt(real)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=dt)
    b = np.ascontiguousarray(b, dtype=dt)
    n = len(b)
    x = np.zeros(n, dtype=dt)
    last = C.c_double(0)
    hist = np.zeros(niter if niter else 0, dtype=np.float64)
    hp = hist.ctypes.data_as(C.c_void_p) if history and niter else None
    it = getattr(_lib(), f"oracle_cgd_{real}")(n, rowptr, rowind, rowval, b, x, error,
                                               niter, hp, len(hist), C.byref(last),
                                               int(threads))
    if history:
        return x, int(it), last.value, hist[:it]
    return x, int(it), last.value


def ref_spmm(rowptr, rowind, rowval, B, ncols=None, bncols=1, blocks=None, out=None,
             real="f64"):
    """C = A*B through the reference's own blas_spmult (src/blas.c:552-606)."""
    dt = _dt(real)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=dt)
    B = np.ascontiguousarray(B, dtype=dt).reshape(-1)
    n = len(rowptr) - 1
    ncols = n if ncols is None else ncols
    C_ = np.zeros(n * bncols, dtype=dt) if out is None else out
    bp, nb, keep = _blocks_arg(blocks)
    rc = _ref(real).gbref_spmult(n, ncols, bncols, rowptr, rowind, rowval, B, C_, bp, nb)
    del keep
    if rc != 1:
        raise RuntimeError(f"blas_spmult returned {rc}")
    return C_


def ref_axpby(a, b, c, subtract=False, real="f64"):
    """c = a + b (blas_add, src/blas.c:275-290) or c = a - b (blas_sub,
    src/blas.c:321-336) through the reference build, in place on numpy arrays
    of the build's real type; c may be the same array as a or b."""
    dt = _dt(real)
    for v in (a, b, c):
        assert v.dtype == dt and v.flags.c_contiguous and len(v) == len(c)
    fn = _ref(real).gbref_sub if subtract else _ref(real).gbref_add
    rc = fn(len(c), a.ctypes.data, b.ctypes.data, c.ctypes.data)
    if rc != 1:
        raise RuntimeError(f"blas_{'sub' if subtract else 'add'} returned {rc}")
    return c


def ref_dot(a, b, real="f64"):
    dt = _dt(real)
    a = np.ascontiguousarray(a, dtype=dt)
    b = np.ascontiguousarray(b, dtype=dt)
    return float(_ref(real).gbref_dot(len(a), a, b))


def pagerank(rowptr, rowind, rowval, damping=0.85, minerror=0.0, niter=0):
    """Restated pagerank command (src/gooseberry_bin.c:2610-2741), FP64.
    Returns (result, iterations, error)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=np.float64)
    n = len(rowptr) - 1
    out = np.zeros(n)
    err = C.c_double(0)
    it = _lib().oracle_pagerank_f64(n, rowptr, rowind, rowval, damping, minerror, niter, out,
                                    C.byref(err))
    return out, int(it), err.value


def ref_pagerank(rowptr, rowind, rowval, damping=0.85, minerror=0.0, niter=0, real="f64"):
    """The pagerank loop around the reference's own blas_spmult / blas_scale /
    blas_add_scalar.  Returns (result, iterations, error)."""
    dt = _dt(real)
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=dt)
    n = len(rowptr) - 1
    out = np.zeros(n, dtype=dt)
    err = C.c_double(0)
    it = _ref(real).gbref_pagerank(n, rowptr, rowind, rowval, damping, minerror, niter, out,
                                   C.byref(err))
    return out, int(it), err.value


FORMAT_GRID, FORMAT_CSR = 1, 2  # gooseberry_format_t (include/gooseberry.h:97-106)


def ref_read_csr(path, real="f64"):
    """The reference's CSR reader (src/io.c:369-498).  Returns
    (rc, nrows, ncols, rowptr, rowind, rowval) -- arrays copied out."""
    L = _ref(real)
    nr, nc = C.c_uint32(0), C.c_uint32(0)
    rp, ri, rv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = L.gbref_read_sparse(FORMAT_CSR, str(path).encode(), C.addressof(nr), C.addressof(nc),
                             C.addressof(rp), C.addressof(ri), C.addressof(rv))
    if rc != 1:
        return rc, 0, 0, None, None, None
    n = nr.value
    nnz = C.cast(rp, C.POINTER(C.c_uint32))[n] if rp.value else 0
    rowptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_uint32)), (n + 1,)).copy()
    rowind = (np.ctypeslib.as_array(C.cast(ri, C.POINTER(C.c_uint32)), (nnz,)).copy()
              if nnz else np.zeros(0, np.uint32))
    ct = C.c_double if real == "f64" else C.c_float
    rowval = (np.ctypeslib.as_array(C.cast(rv, C.POINTER(ct)), (nnz,)).copy()
              if nnz else np.zeros(0, _dt(real)))
    for q in (rp, ri, rv):
        L.gbref_free(q)
    return rc, n, nc.value, rowptr, rowind, rowval


def ref_read_grid(path, real="f64"):
    """The reference's grid reader (src/io.c:145-239): (rc, nrows, ncols, values)."""
    L = _ref(real)
    nr, nc = C.c_uint32(0), C.c_uint32(0)
    rv = C.c_void_p()
    rc = L.gbref_read_dense(FORMAT_GRID, str(path).encode(), C.addressof(nr), C.addressof(nc),
                            C.addressof(rv))
    if rc != 1:
        return rc, 0, 0, None
    m = nr.value * nc.value
    ct = C.c_double if real == "f64" else C.c_float
    vals = (np.ctypeslib.as_array(C.cast(rv, C.POINTER(ct)), (m,)).copy()
            if m else np.zeros(0, _dt(real)))
    L.gbref_free(rv)
    return rc, nr.value, nc.value, vals


def ref_write_grid(path, vals, nrows, ncols, real="f64"):
    """The reference's grid writer (src/io.c:1195-1229)."""
    v = np.ascontiguousarray(vals, dtype=_dt(real))
    return _ref(real).gbref_write_dense(FORMAT_GRID, str(path).encode(), nrows, ncols, v)


def ref_write_csr(path, rowptr, rowind, rowval, ncols, real="f64"):
    """The reference's CSR writer (src/io.c:1233-1275)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=_dt(real))
    return _ref(real).gbref_write_sparse(FORMAT_CSR, str(path).encode(), len(rowptr) - 1,
                                         ncols, rowptr, rowind, rowval)


def ref_spdot(ind, val, x, real="f64"):
    """The reference's own blas_spdot (src/blas.c:433-451)."""
    dt = _dt(real)
    ind = np.ascontiguousarray(ind, dtype=np.uint32)
    val = np.ascontiguousarray(val, dtype=dt)
    x = np.ascontiguousarray(x, dtype=dt)
    return float(_ref(real).gbref_spdot(len(ind), ind, val, x))


def ref_cgd(rowptr, rowind, rowval, b, error, niter, real="f64", history=False):
    """The reference's own cgd (src/cgd.c:40-129); iterations parsed from its ITER lines."""
    dt = _dt(real)
    rowptr = np.array(rowptr, dtype=np.uint32)
    rowind = np.array(rowind, dtype=np.uint32)
    rowval = np.array(rowval, dtype=dt)
    b = np.array(b, dtype=dt)
    n = len(b)
    x = np.zeros(n, dtype=dt)
    it = C.c_size_t(0)
    last = C.c_double(0)
    hist = np.zeros(niter if niter else 0, dtype=np.float64)
    hp = hist.ctypes.data_as(C.c_void_p) if history and niter else None
    rc = _ref(real).gbref_cgd(n, rowptr, rowind, rowval, b, x, float(error), niter,
                              C.byref(it), C.byref(last), hp, len(hist))
    if rc != 1:
        raise RuntimeError(f"cgd returned {rc}")
    if history:
        return x, int(it.value), last.value, hist[: it.value]
    return x, int(it.value), last.value


def _perm_arg(perm):
    if perm is None:
        return None, None
    a = np.ascontiguousarray(perm, dtype=np.uint32)
    return a.ctypes.data_as(C.c_void_p), a


def cuthillmckee(rowptr, rowind, nrows, ncols=None, blocks=None):
    """Restated Cuthill-McKee order (src/permute.c:45-104,288-337); equal
    degrees smaller id first.  Returns perm (perm[new] = old), or None when the
    matrix is not square (the reference's INVALIDINPUT)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    ncols = nrows if ncols is None else ncols
    perm = np.zeros(max(nrows, 1), dtype=np.uint32)
    bp, nb, keep = _blocks_arg(blocks)
    rc = _lib().oracle_cuthillmckee(nrows, ncols, rowptr, rowind, bp, nb, perm)
    del keep
    return None if rc != 0 else perm[:nrows]


def ref_cuthillmckee(rowptr, rowind, nrows, ncols=None, blocks=None, real="f64"):
    """The reference's own permute_cuthillmckee (src/permute.c:288-337), with
    the oracle shim's priority queue.  Returns (rc, perm)."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    ncols = nrows if ncols is None else ncols
    perm = np.zeros(max(nrows, 1), dtype=np.uint32)
    bp, nb, keep = _blocks_arg(blocks)
    rc = _ref(real).gbref_cuthillmckee(nrows, ncols, rowptr, rowind, bp, nb, perm)
    del keep
    return rc, perm[:nrows]


def permute_sparse(rowptr, rowind, rowval, ncols, rowperm=None, colperm=None):
    """Restated permute_sparse (src/permute.c:120-205), FP64, out of place:
    returns (rowptr, rowind, rowval) of the permuted matrix."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    rowind = np.ascontiguousarray(rowind, dtype=np.uint32)
    rowval = np.ascontiguousarray(rowval, dtype=np.float64)
    n = len(rowptr) - 1
    nnz = int(rowptr[-1])
    prp = np.zeros(n + 1, dtype=np.uint32)
    pri = np.zeros(max(nnz, 1), dtype=np.uint32)
    prv = np.zeros(max(nnz, 1), dtype=np.float64)
    rp, rk = _perm_arg(rowperm)
    cp, ck = _perm_arg(colperm)
    _lib().oracle_permute_sparse_f64(n, ncols, rowptr, rowind, rowval, rp, cp, prp, pri, prv)
    del rk, ck
    return prp, pri[:nnz], prv[:nnz]


def ref_permute_sparse(rowptr, rowind, rowval, ncols, rowperm=None, colperm=None, real="f64"):
    """The reference's own permute_sparse (src/permute.c:120-205), applied to
    copies: returns (rc, rowptr, rowind, rowval)."""
    rowptr = np.array(rowptr, dtype=np.uint32)
    rowind = np.array(rowind, dtype=np.uint32)
    rowval = np.array(rowval, dtype=_dt(real))
    if len(rowind) == 0:
        rowind = np.zeros(1, np.uint32)
        rowval = np.zeros(1, _dt(real))
    rp, rk = _perm_arg(rowperm)
    cp, ck = _perm_arg(colperm)
    rc = _ref(real).gbref_permute_sparse(len(rowptr) - 1, ncols, rowptr, rowind, rowval, rp, cp)
    del rk, ck
    nnz = int(rowptr[-1])
    return rc, rowptr, rowind[:nnz], rowval[:nnz]


def permute_dense(vals, nrows, ncols, rowperm=None, colperm=None, reverse=False):
    """Restated permute_dense / permute_dense_rev (src/permute.c:208-283), FP64,
    row-major, out of place."""
    a = np.ascontiguousarray(vals, dtype=np.float64)
    out = np.zeros_like(a) if reverse else np.empty_like(a)
    rp, rk = _perm_arg(rowperm)
    cp, ck = _perm_arg(colperm)
    _lib().oracle_permute_dense_f64(nrows, ncols, a, out, rp, cp, int(reverse))
    del rk, ck
    return out


def ref_permute_dense(vals, nrows, ncols, rowperm=None, colperm=None, reverse=False,
                      real="f64"):
    """The reference's own permute_dense / permute_dense_rev on a copy."""
    a = np.array(vals, dtype=_dt(real))
    rp, rk = _perm_arg(rowperm)
    cp, ck = _perm_arg(colperm)
    rc = _ref(real).gbref_permute_dense(nrows, ncols, a, rp, cp, int(reverse))
    del rk, ck
    return rc, a

