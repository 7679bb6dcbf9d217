"""Seeded generators: shapes, exact sizes, reproducibility, SPD structure."""
from __future__ import annotations

import numpy as np

from gooseberry_b200 import workloads as W


def _rows_sorted_distinct(A):
    r = A.rowind.astype(np.int64)
    L = A.row_lengths()
    starts = np.zeros(len(r), bool)
    starts[A.rowptr[:-1][L > 0].astype(np.int64)] = True
    d = np.diff(r)
    return bool(np.all(d[~starts[1:]] > 0)) and (len(r) == 0 or r.max() < A.ncols)


def test_counter_rng_is_position_independent():
    a = W.rand_u64(7, 3, 0, 1000)
    b = W.rand_u64(7, 3, 500, 500)
    assert np.array_equal(a[500:], b)
    assert not np.array_equal(W.rand_u64(7, 3, 0, 10), W.rand_u64(8, 3, 0, 10))
    u = W.rand_unit(1, 1, 100000)
    assert 0.0 <= u.min() and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01


def test_uniform_rows_shape():
    A = W.uniform_rows(2000, 10, seed=3)
    assert A.nnz == 20000 and np.all(A.row_lengths() == 10)
    assert _rows_sorted_distinct(A)
    assert -1.0 <= A.rowval.min() and A.rowval.max() <= 1.0
    B = W.uniform_rows(2000, 10, seed=3)
    assert np.array_equal(A.rowind, B.rowind) and np.array_equal(A.rowval, B.rowval)


def test_powerlaw_exact_nnz_and_cap():
    A = W.powerlaw_rows(20000, 320000, seed=5, cap=20000)
    L = A.row_lengths()
    assert A.nnz == 320000 and L.min() >= 1 and L.max() <= 20000
    assert _rows_sorted_distinct(A)
    # heavy tail: the longest row is far above the mean
    assert L.max() > 20 * L.mean()


def test_laplacian_2d_structure():
    A = W.laplacian_2d(32)
    assert A.nrows == 1024 and A.nnz == 5 * 1024 - 4 * 32
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0
    assert np.all(S.diagonal() == 4.0)
    full = W.laplacian_2d(1024)
    assert full.nnz == 5_238_784


def test_diffusion_spd():
    A = W.diffusion_3d(10, seed=2)
    S = A.to_scipy()
    assert A.nnz == 7 * 1000 - 6 * 100
    assert abs(S - S.T).max() == 0
    ev = np.linalg.eigvalsh(S.toarray())
    assert ev.min() > 0
    off = np.abs(S).sum(1).A1 - S.diagonal()
    assert np.all(S.diagonal() >= off * (1 - 1e-12))


def test_serving_sides_range():
    s = W.serving_sides(10000, seed=9)
    assert s.min() >= 32 and s.max() <= 512
    t = W.poisson_arrivals(1000, 100.0, seed=9)
    assert np.all(np.diff(t) > 0) and 5 < t[-1] < 20
