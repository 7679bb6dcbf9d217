"""The CPU oracle: the restatement (oracle/gb_oracle.c) against the reference's
own outputs (golden fixtures generated by tests/golden/make_golden.py from
oracle/_ref), and against the reference build itself where it is present."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import oracle
from gooseberry_b200 import workloads as W


def test_known_answer_tridiagonal():
    # tridiag(-1, 2, -1) * [1..5] = [0, 0, 0, 0, 6]
    rp = np.array([0, 2, 5, 8, 11, 13], np.uint32)
    ri = np.array([0, 1, 0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4], np.uint32)
    rv = np.array([2, -1, -1, 2, -1, -1, 2, -1, -1, 2, -1, -1, 2], float)
    x = np.arange(1, 6, dtype=float)
    y = oracle.spmv(rp, ri, rv, x)
    assert y.tolist() == [0, 0, 0, 0, 6]
    xs, it, _ = oracle.cgd(rp, ri, rv, y, 1e-12, 100)
    assert it == 5
    np.testing.assert_allclose(xs, x, rtol=0, atol=1e-12)


def test_spmv_restatement_bitwise_equals_reference(spmv_golden):
    for name, c in spmv_golden.items():
        if "rowptr" not in c:
            continue
        y64 = oracle.spmv(c["rowptr"], c["rowind"], c["rowval"], c["x"])
        assert np.array_equal(y64, c["y64"]), name
        y32 = oracle.spmv(c["rowptr"], c["rowind"], c["rowval"].astype(np.float32),
                          c["x"].astype(np.float32), real="f32")
        assert np.array_equal(y32, c["y32"]), name
        # the row split over threads never changes a row's sum
        y64t = oracle.spmv(c["rowptr"], c["rowind"], c["rowval"], c["x"], threads=4)
        assert np.array_equal(y64t, c["y64"]), name


def test_spmm_and_blocks_restatement(spmv_golden):
    u = spmv_golden["uniform300"]
    C = oracle.spmm(u["rowptr"], u["rowind"], u["rowval"], spmv_golden["spmm3"]["B"],
                    bncols=3)
    assert np.array_equal(C, spmv_golden["spmm3"]["C"])
    bl = spmv_golden["blocks"]
    out = bl["init"].copy()
    oracle.spmm(u["rowptr"], u["rowind"], u["rowval"], u["x"],
                blocks=bl["blocks_partial"], out=out)
    assert np.array_equal(out, bl["C"])
    # rows outside the blocks keep their previous contents
    assert np.all(out[120:] == 7.0)


def test_cg_restatement_bitwise_equals_reference(cg_golden):
    for name, c in cg_golden.items():
        x, it, _ = oracle.cgd(c["rowptr"], c["rowind"], c["rowval"], c["b"],
                              float(c["error"]), int(c["niter"]))
        assert it == int(c["iterations"]), name
        assert np.array_equal(x, c["x"]), name


def test_full_uniform_spmv_checksum(full_golden):
    g = full_golden["spmv_uniform_100k"]
    A = W.uniform_rows(g["n"], g["k"], seed=g["seed"])
    x = W.dense_x(g["n"], g["seed"])
    y = oracle.spmv(A.rowptr, A.rowind, A.rowval, x, threads=4)
    assert hashlib.sha256(y.tobytes()).hexdigest() == g["y_sha256"]


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_reference_build_matches_restatement_random():
    A = W.powerlaw_rows(3000, 40000, seed=99, cap=3000)
    x = W.dense_x(3000, 99)
    assert np.array_equal(oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, x),
                          oracle.spmv(A.rowptr, A.rowind, A.rowval, x))
    b = W.rhs(400, 98)
    L = W.laplacian_2d(20)
    oracle.ref_set_threads(1)
    xr, itr, _ = oracle.ref_cgd(L.rowptr, L.rowind, L.rowval, b, 1e-9, 500)
    xo, ito, _ = oracle.cgd(L.rowptr, L.rowind, L.rowval, b, 1e-9, 500)
    assert itr == ito and np.array_equal(xr, xo)


def test_dot_scale_add_scalar():
    a = W.dense_x(1001, 5)
    b = W.rhs(1001, 6)
    assert oracle.dot(a, b) == float(np.sum(a * b)) or abs(oracle.dot(a, b) - a @ b) < 1e-12
    s = oracle.scale(a, 3.0)
    assert np.array_equal(s, a * 3.0)
    t = oracle.add_scalar(a, -0.5)
    assert np.array_equal(t, a - 0.5)


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_reference_add_sub_known_answers():
    """blas_add / blas_sub through the reference build equal the IEEE sums
    and differences elementwise, also written in place over either input."""
    a = W.dense_x(5003, 11)
    b = W.rhs(5003, 12)
    assert np.array_equal(oracle.ref_axpby(a, b, np.empty_like(a)), a + b)
    assert np.array_equal(oracle.ref_axpby(a, b, np.empty_like(a), subtract=True), a - b)
    c = b.copy()
    assert np.array_equal(oracle.ref_axpby(a, c, c, subtract=True), a - b)
    c = a.copy()
    assert np.array_equal(oracle.ref_axpby(c, b, c), a + b)


def test_spdot_restatement():
    A = W.powerlaw_rows(2000, 30000, seed=7, cap=2000)
    x = W.dense_x(2000, 7)
    s = oracle.spdot(A.rowind, A.rowval, x)
    acc = 0.0
    for k in range(A.nnz):  # the loop of src/blas.c:445-448, k ascending
        acc += A.rowval[k] * x[A.rowind[k]]
    assert s == acc
    assert oracle.spdot(A.rowind[:0], A.rowval[:0], x) == 0.0


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_spdot_matches_reference_build():
    A = W.powerlaw_rows(2000, 30000, seed=8, cap=2000)
    x = W.dense_x(2000, 8)
    oracle.ref_set_threads(1)  # one OpenMP thread: k ascending
    assert oracle.ref_spdot(A.rowind, A.rowval, x) == oracle.spdot(A.rowind, A.rowval, x)
    x32 = x.astype(np.float32)
    v32 = A.rowval.astype(np.float32)
    assert (oracle.ref_spdot(A.rowind, v32, x32, real="f32")
            == oracle.spdot(A.rowind, v32, x32, real="f32"))


def _pr_graph(n, nnz, seed, nsinks=0):
    A = W.powerlaw_rows(n, nnz, seed=seed, cap=n)
    rv = np.abs(A.rowval) + 0.1
    if not nsinks:
        return A.rowptr, A.rowind, rv
    rp = A.rowptr.astype(np.int64)
    keep = np.ones(A.nnz, bool)
    L = np.diff(rp)
    for k in range(nsinks):
        keep[rp[k]:rp[k + 1]] = False
        L[k] = 0
    return (np.concatenate([[0], np.cumsum(L)]).astype(np.uint32), A.rowind[keep], rv[keep])


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_pagerank_restatement_matches_reference_loop():
    """The restated pagerank command equals the same loop around the
    reference's own blas_spmult / blas_scale / blas_add_scalar, bit for bit:
    converging (no sinks) and at an iteration limit (with sinks, whose mass the
    reference adds whole to every entry)."""
    oracle.ref_set_threads(1)
    rp, ri, rv = _pr_graph(3000, 30000, 5)
    a = oracle.pagerank(rp, ri, rv, 0.85, 1e-10, 0)
    b = oracle.ref_pagerank(rp, ri, rv, 0.85, 1e-10, 0)
    assert a[1] == b[1] and a[1] % 10 == 1 and a[2] == b[2] and np.array_equal(a[0], b[0])
    assert abs(a[0].sum() - 1.0) < 1e-9
    rp, ri, rv = _pr_graph(3000, 30000, 6, nsinks=7)
    a = oracle.pagerank(rp, ri, rv, 0.9, 0.0, 13)
    b = oracle.ref_pagerank(rp, ri, rv, 0.9, 0.0, 13)
    assert a[1] == b[1] == 13 and a[2] == b[2] and np.array_equal(a[0], b[0])


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_spmm_blocks_fuzz_matches_reference_build():
    """Random matrices with empty rows, 1-4 right-hand columns and random
    block lists (increasing, decreasing = empty, overlapping, not covering
    every row): the restatement and the reference's blas_spmult write the same
    rows with the same bits and leave the others alone (src/blas.c:576-595),
    both value widths."""
    rng = np.random.default_rng(31)
    for case in range(60):
        n = int(rng.integers(1, 300))
        ncols = int(rng.integers(1, 300))
        lengths = rng.integers(0, 12, n) * (rng.random(n) < 0.8)
        rp = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint32)
        nnz = int(rp[-1])
        ri = rng.integers(0, ncols, nnz).astype(np.uint32)
        rv = rng.uniform(-1, 1, nnz)
        k = int(rng.integers(1, 5))
        B = rng.uniform(-1, 1, ncols * k)
        blocks = None
        if rng.random() < 0.75:
            blocks = rng.integers(0, n + 1, int(rng.integers(1, 7)))
            if rng.random() < 0.5:
                blocks = np.sort(blocks)
        for real in ("f64", "f32"):
            dt = np.float64 if real == "f64" else np.float32
            init = np.full(n * k, 7.0, dt)
            a = oracle.spmm(rp, ri, rv.astype(dt), B.astype(dt), ncols=ncols, bncols=k,
                            blocks=blocks, out=init.copy(), real=real)
            b = oracle.ref_spmm(rp, ri, rv.astype(dt), B.astype(dt), ncols=ncols, bncols=k,
                                blocks=blocks, out=init.copy(), real=real)
            assert a.tobytes() == b.tobytes(), (case, real, blocks)


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_cgd_fuzz_matches_reference_build():
    """Random symmetric diagonally dominant systems (random sparsity, sizes
    1-400, tolerances from loose to unreachable, iteration limits that stop
    early): the restatement's iterations, last norm and x equal the reference
    cgd's bit for bit, both value widths (one OpenMP thread, so the
    reference's dot products add in index order)."""
    rng = np.random.default_rng(5)
    oracle.ref_set_threads(1)
    for case in range(40):
        n = int(rng.integers(1, 400))
        m = int(rng.integers(0, 4 * n + 1))
        r = rng.integers(0, n, m)
        c = rng.integers(0, n, m)
        w = rng.uniform(-1, 1, m)
        A = np.zeros((n, n))
        np.add.at(A, (r, c), w)
        A = A + A.T
        A[np.arange(n), np.arange(n)] = np.abs(A).sum(axis=1) + rng.uniform(0.1, 2, n)
        rows, cols = np.nonzero(A)
        rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.uint32)
        ri, rv = cols.astype(np.uint32), A[rows, cols]
        b = rng.uniform(-1, 1, n)
        err = float(10.0 ** rng.uniform(-14, -1)) * float(np.linalg.norm(b))
        niter = int(rng.choice([3, 10, 1000]))
        for real in ("f64", "f32"):
            dt = np.float64 if real == "f64" else np.float32
            xo, ito, _ = oracle.cgd(rp, ri, rv.astype(dt), b.astype(dt), err, niter, real=real)
            xr, itr, _ = oracle.ref_cgd(rp, ri, rv.astype(dt), b.astype(dt), err, niter,
                                         real=real)
            ctx = (case, real, n, niter, err)
            assert ito == itr, ctx
            assert xo.tobytes() == xr.tobytes(), ctx
