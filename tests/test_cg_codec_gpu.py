"""The FP64 CG's compressed matrix entries (16-bit column distances, 8-bit
value codes, exact float values, and on pattern matrices a pattern byte with
the row's values or codes in a row of 6 or 8; GB_CG_PLAIN_ENTRIES turns them
off) change only the bytes streamed: every solve is bit-identical to the solve
over the plain CSR arrays, on matrices that take each encoding."""
from __future__ import annotations

import numpy as np
import pytest

import gooseberry_b200 as gb
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _csr(n, rows, cols, vals):
    o = np.lexsort((cols, rows))
    rows, cols, vals = rows[o], cols[o], vals[o]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    return W.Csr(n, n, np.cumsum(rp).astype(np.uint32), cols.astype(np.uint32), vals)


def graph_laplacian(n, deg, seed, weights=False):
    """I + L of a random graph: SPD, columns spread over the whole range."""
    rng = np.random.default_rng(seed)
    a = rng.integers(0, n, n * deg)
    b = rng.integers(0, n, n * deg)
    keep = a != b
    e = np.unique(np.stack([np.minimum(a[keep], b[keep]), np.maximum(a[keep], b[keep])], 1),
                  axis=0)
    w = rng.uniform(0.5, 2.0, len(e)) if weights else np.ones(len(e))
    d = np.ones(n)
    np.add.at(d, e[:, 0], w)
    np.add.at(d, e[:, 1], w)
    rows = np.concatenate([e[:, 0], e[:, 1], np.arange(n)])
    cols = np.concatenate([e[:, 1], e[:, 0], np.arange(n)])
    vals = np.concatenate([-w, -w, d])
    return _csr(n, rows, cols, vals)


def float_exact(A):
    return W.Csr(A.nrows, A.ncols, A.rowptr, A.rowind,
                 A.rowval.astype(np.float32).astype(np.float64))


def banded(n, offsets, seed):
    """A symmetric diagonally dominant matrix with the given diagonals: its
    rows have only a few distinct column patterns until the band is wider than
    256 patterns allow, then 16-bit distances take over."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for d in offsets:
        i = np.arange(max(0, -d), min(n, n - d))
        rows.append(i)
        cols.append(i + d)
        vals.append(-rng.uniform(0.1, 1.0, len(i)))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    keep = r < c
    r, c, v = r[keep], c[keep], v[keep]
    d = np.ones(n)
    np.add.at(d, r, -v)
    np.add.at(d, c, -v)
    return _csr(n, np.concatenate([r, c, np.arange(n)]), np.concatenate([c, r, np.arange(n)]),
                np.concatenate([v, v, d + 1.0]))


def many_patterns(n, seed):
    """Rows of up to 7 entries whose column offsets are drawn per row: far
    more than 256 distinct patterns, all within 16-bit distance."""
    rng = np.random.default_rng(seed)
    rows, cols = [np.arange(n)], [np.arange(n)]
    for k in range(3):
        off = rng.integers(1, 3000, n)
        j = np.arange(n) + off
        ok = j < n
        rows += [np.arange(n)[ok], j[ok]]
        cols += [j[ok], np.arange(n)[ok]]
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    e = np.unique(np.stack([r, c], 1), axis=0)
    r, c = e[:, 0], e[:, 1]
    v = np.where(r == c, 0.0, -rng.uniform(0.1, 1.0, len(r)))
    v = np.where(r < c, v, 0.0)
    # symmetric values: take the upper triangle's
    up = {(a, b): w for a, b, w in zip(r, c, v) if a < b}
    v = np.array([up[(a, b)] if a < b else (up[(b, a)] if a > b else 0.0)
                  for a, b in zip(r, c)])
    d = np.zeros(n)
    np.add.at(d, r, -v)
    v = np.where(r == c, d[r] + 1.0, v)
    return _csr(n, r, c, v)


CASES = {
    # name: (matrix builder, expected bytes per entry, per row)
    # row patterns: a pattern byte and a row of value codes (8), doubles (6 when
    # no row has more than 5 entries, else 8) or floats (8) per row
    "laplace64": (lambda: W.laplacian_2d(64), 0, 9),
    "diffusion2d": (lambda: W.diffusion_2d(48, seed=5), 0, 49),
    "diffusion2d_f32": (lambda: float_exact(W.diffusion_2d(48, seed=6)), 0, 33),
    "diffusion3d": (lambda: W.diffusion_3d(24, seed=11), 0, 65),
    "diffusion3d_f32": (lambda: float_exact(W.diffusion_3d(24, seed=13)), 0, 33),
    "band": (lambda: banded(5000, [-200, -3, -1, 0, 1, 3, 200], 8), 0, 65),
    # too many patterns: 16-bit columns and doubles (or exact floats) per entry
    "many_patterns": (lambda: many_patterns(20000, 10), 10, 4),
    "many_patterns_f32": (lambda: float_exact(many_patterns(20000, 14)), 6, 4),
    "graph": (lambda: graph_laplacian(40000, 4, 7), 5, 4),      # 32-bit columns, codes
    "graph_weighted": (lambda: graph_laplacian(40000, 4, 8, weights=True), 12, 4),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_compressed_entries_are_bit_identical(name):
    import torch
    build, want_bytes, want_row = CASES[name]
    A = build()
    M = gb.CsrMatrix.from_host(A)
    M.set_schedule(gb.SCHED_ROW)
    S = gb.CgSolver(M)
    P = gb.CgSolver(M, plain_entries=True)
    assert (S.entry_bytes(), S.row_bytes()) == (want_bytes, want_row)
    assert (P.entry_bytes(), P.row_bytes()) == (12, 4)
    b = torch.from_numpy(W.rhs(A.nrows, 9)).cuda()
    for tol, niter in ((1e-10, 0), (1e-30, 25)):
        x1, r1 = S.solve(b, tol=tol, niter=niter)
        x2, r2 = P.solve(b, tol=tol, niter=niter)
        assert r1.iterations == r2.iterations and r1.status == r2.status
        assert torch.equal(x1, x2), name
        assert r1.rnorm == r2.rnorm
    S.close()
    P.close()
    M.close()


@pytest.mark.parametrize("name,want", [("diffusion3d", (0, 33)), ("diffusion2d", (0, 33)),
                                       ("band", (0, 33)), ("many_patterns", (6, 4))])
def test_mixed_solver_compressed_columns_are_bit_identical(name, want):
    """The mixed solver's FP32 SpMV over row patterns (stencils and bands: a
    byte per row naming one of at most 256 lists of column offsets, with the
    values in rows of 8: 33 stored bytes per row, none per nonzero) or, past
    that, 16-bit column distances gives the same iterates, refinements and
    solution as over the plain columns."""
    import torch
    A = {"diffusion3d": lambda: W.diffusion_3d(24, seed=11),
         "diffusion2d": lambda: W.diffusion_2d(70, seed=12),
         "band": lambda: banded(5000, [-200, -3, -1, 0, 1, 3, 200], 8),
         "many_patterns": lambda: many_patterns(20000, 10)}[name]()
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    M.set_schedule(gb.SCHED_ROW)
    M.set_schedule(gb.SCHED_ROW, f32=True)
    S = gb.CgSolver(M, gb.CG_MIXED)
    P = gb.CgSolver(M, gb.CG_MIXED, plain_entries=True)
    assert (S.entry_bytes(), S.row_bytes()) == want and P.entry_bytes() == 8
    b = torch.from_numpy(W.rhs(A.nrows, 12)).cuda()
    x1, r1 = S.solve(b, tol=1e-10)
    x2, r2 = P.solve(b, tol=1e-10)
    assert r1.status == r2.status == "converged"
    assert (r1.iterations, r1.refinements) == (r2.iterations, r2.refinements)
    assert torch.equal(x1, x2)
    S.close()
    P.close()
    M.close()
