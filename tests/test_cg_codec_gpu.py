"""The FP64 CG's compressed matrix entries (16-bit column distances, 8-bit
value codes, exact float values; GB_CG_PLAIN_ENTRIES turns them off) change
only the bytes streamed: every solve is bit-identical to the solve over the
plain CSR arrays, on matrices that take each encoding."""
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


CASES = {
    # name: (matrix builder, expected bytes per entry)
    "laplace64": (lambda: W.laplacian_2d(64), 3),           # 16-bit columns, value codes
    "diffusion2d": (lambda: W.diffusion_2d(48, seed=5), 10),  # 16-bit columns, doubles
    "diffusion2d_f32": (lambda: float_exact(W.diffusion_2d(48, seed=6)), 6),
    "graph": (lambda: graph_laplacian(40000, 4, 7), 5),         # 32-bit columns, codes
    "graph_weighted": (lambda: graph_laplacian(40000, 4, 8, weights=True), 12),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_compressed_entries_are_bit_identical(name):
    import torch
    build, want_bytes = CASES[name]
    A = build()
    M = gb.CsrMatrix.from_host(A)
    M.set_schedule(gb.SCHED_ROW)
    S = gb.CgSolver(M)
    P = gb.CgSolver(M, plain_entries=True)
    assert S.entry_bytes() == want_bytes
    assert P.entry_bytes() == 12
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


def test_mixed_solver_16bit_columns_are_bit_identical():
    """The mixed solver's FP32 SpMV over 16-bit column distances gives the
    same iterates, refinements and solution as over the plain columns."""
    import torch
    A = W.diffusion_3d(24, seed=11)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    M.set_schedule(gb.SCHED_ROW)
    M.set_schedule(gb.SCHED_ROW, f32=True)
    S = gb.CgSolver(M, gb.CG_MIXED)
    P = gb.CgSolver(M, gb.CG_MIXED, plain_entries=True)
    assert S.entry_bytes() == 6 and P.entry_bytes() == 8
    b = torch.from_numpy(W.rhs(A.nrows, 12)).cuda()
    x1, r1 = S.solve(b, tol=1e-10)
    x2, r2 = P.solve(b, tol=1e-10)
    assert r1.status == r2.status == "converged"
    assert (r1.iterations, r1.refinements) == (r2.iterations, r2.refinements)
    assert torch.equal(x1, x2)
    S.close()
    P.close()
    M.close()
