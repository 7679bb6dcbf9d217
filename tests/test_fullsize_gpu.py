"""Parity at the benchmark's full sizes, against results of the reference's
own build (oracle/_ref) recorded in tests/golden/full_sizes.json by
tests/golden/make_golden.py:

* the power-law SpMV: n = 8,000,000 rows, 128,000,000 nonzeros (Zipf 2.1 row
  lengths capped at 200,000), every row, both value widths.  The schedules
  that sum in the reference's order (src/blas.c:82-91) must give the
  reference's y bit for bit (SHA-256 of all 8M entries); every other schedule,
  and the one the autotuner picks, must stay within the per-row
  condition-scaled bound of that y;
* CG on the 160^3 variable-coefficient 3D operator (n = 4,096,000): the
  FP64 solve against the reference cgd's iteration count and solution, and
  the mixed solve's true FP64 residual and its error against the reference
  solution (src/cgd.c:40-129)."""
from __future__ import annotations

import hashlib
import os

import numpy as np
import pytest

import gooseberry_b200 as gb
from gooseberry_b200 import workloads as W
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 64 * 2.0 ** -24


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def powerlaw(full_golden):
    g = full_golden["spmv_powerlaw_8m"]
    A = W.powerlaw_rows(g["n"], g["nnz"], seed=g["seed"], cap=g["cap"])
    assert _sha(A.rowptr) == g["rowptr_sha256"], "generator drifted from the golden input"
    x = W.dense_x(A.ncols, g["seed"])
    import scipy.sparse as sp
    S = sp.csr_matrix((np.abs(A.rowval), A.rowind.astype(np.int64), A.rowptr.astype(np.int64)),
                      shape=(A.nrows, A.ncols))
    scale64 = S @ np.abs(x)
    return A, x, scale64


def _worst(y, y_ref, scale):
    return float(np.max(np.abs(y.astype(np.float64) - y_ref.astype(np.float64)) /
                        np.maximum(scale, 1e-300)))


def test_powerlaw_8m_every_row_matches_reference(torch, full_golden, powerlaw):
    g = full_golden["spmv_powerlaw_8m"]
    A, x, scale = powerlaw
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    xd = torch.from_numpy(x).cuda()
    x32 = x.astype(np.float32)
    xd32 = torch.from_numpy(x32).cuda()
    # reference-order schedules: the reference's bits on all 8M rows
    M.set_schedule(gb.SCHED_ROW)
    y_ref = M.spmv(xd).cpu().numpy()
    assert _sha(y_ref) == g["y_sha256"]
    M.set_schedule(gb.SCHED_ROW, f32=True)
    y32_ref = M.spmv(xd32).cpu().numpy()
    assert _sha(y32_ref) == g["y32_sha256"]
    # reordered sums (and, on every tile schedule, rows longer than a tile
    # summed in chunks): within the condition-scaled bound of the reference's y
    scale32 = scale  # |A||x| in FP64; the FP32 bound is relative to it
    for s, t in ((gb.SCHED_SEG, 2048), (gb.SCHED_MERGE, 2048), (gb.SCHED_GROUP4, 512),
                 (gb.SCHED_WMERGE, 128), (gb.SCHED_WTILE, 256)):
        M.set_schedule(s, tile_items=t)
        y = M.spmv(xd).cpu().numpy()
        assert _worst(y, y_ref, scale) <= TOL64, gb.SCHED_NAMES[s]
        assert np.array_equal(y, M.spmv(xd).cpu().numpy()), gb.SCHED_NAMES[s]
        M.set_schedule(s, tile_items=t, f32=True)
        y32 = M.spmv(xd32).cpu().numpy()
        assert _worst(y32, y32_ref, scale32) <= TOL32, gb.SCHED_NAMES[s]
    # the autotuned schedules
    M.autotune()
    M.autotune(f32=True)
    y = M.spmv(xd).cpu().numpy()
    assert _worst(y, y_ref, scale) <= TOL64, gb.SCHED_NAMES[M.info().schedule]
    y32 = M.spmv(xd32).cpu().numpy()
    assert _worst(y32, y32_ref, scale32) <= TOL32, gb.SCHED_NAMES[M.info().schedule_f32]
    # FP32 accumulation against the FP64 reference: the error the bench states
    err32 = _worst(y32, y_ref, scale)
    assert err32 <= TOL32, err32


@pytest.fixture(scope="module")
def diffusion160(full_golden):
    g = full_golden["cg_diffusion_160"]
    A = W.diffusion_3d(g["side"], seed=g["seed"])
    b = W.rhs(A.nrows, g["b_seed"])
    xs = np.load(os.path.join(GOLDEN, "cg_diffusion_160_xsample.npz"))
    return g, A, b, int(xs["step"]), xs["x"]


def test_diffusion_160_fp64_cg_matches_reference(torch, diffusion160):
    """FP64 CG to rel-res 1e-10 on the ill-conditioned 160^3 operator
    (coefficients over four decades).  Here the reference's own iteration
    count depends on its OpenMP thread count (its dot products reduce in
    thread order): 2937, 2932, 2933 and 2930 iterations on 1, 2, 4 and 8
    threads.  The GPU count must lie within that spread (7) of the
    reference's range, and the solution must agree with the reference's to
    the accuracy the stopping rule leaves."""
    g, A, b, step, x_ref = diffusion160
    M = gb.CsrMatrix.from_host(A)
    S = gb.CgSolver(M)
    x, r = S.solve(torch.from_numpy(b).cuda(), tol=g["rtol"], niter=g["niter"])
    assert r.status == "converged", r
    lo, hi = g["reference_iterations_range"]
    spread = hi - lo
    assert lo - spread <= r.iterations <= hi + spread, (r.iterations, lo, hi)
    xh = x.cpu().numpy()
    res = np.linalg.norm(b - A.to_scipy() @ xh) / np.linalg.norm(b)
    assert res <= 1.5 * g["rtol"], res
    err = np.linalg.norm(xh[::step] - x_ref) / np.linalg.norm(x_ref)
    assert err <= g["solution_tolerance"], err
    S.close()


def test_diffusion_160_mixed_cg_reaches_fp64_accuracy(torch, diffusion160):
    """Mixed precision (FP32 values and Krylov vectors, FP64 residual,
    refinement and dots) to true rel-res 1e-10, with its error against the
    reference's FP64 solution on the same bound as the FP64 GPU solve."""
    g, A, b, step, x_ref = diffusion160
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    S = gb.CgSolver(M, mode=gb.CG_MIXED)
    x, r = S.solve(torch.from_numpy(b).cuda(), tol=g["rtol"], niter=g["niter"])
    assert r.status == "converged" and r.refinements > 0, r
    xh = x.cpu().numpy()
    res = np.linalg.norm(b - A.to_scipy() @ xh) / np.linalg.norm(b)
    assert res <= g["rtol"] * (1 + 1e-6), res
    err = np.linalg.norm(xh[::step] - x_ref) / np.linalg.norm(x_ref)
    assert err <= g["solution_tolerance"], err
    S.close()
