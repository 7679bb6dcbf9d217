"""Mixed-precision CG (FP32 values and Krylov vectors, FP64 dots and FP64
residual refinement): converges to the requested relative residual measured
in FP64 on the host, in about the iterations plain FP64 CG needs, and agrees
with the FP64 solution to the accuracy both reached."""
from __future__ import annotations

import numpy as np
import pytest

import gooseberry_b200 as gb
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _rel_res(A, x, b):
    return float(np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b))


@pytest.mark.parametrize("name,make,rtol", [
    ("diffusion3d_24", lambda: W.diffusion_3d(24, seed=31), 1e-10),
    ("diffusion2d_96", lambda: W.diffusion_2d(96, seed=32), 1e-10),
    ("laplace2d_128", lambda: W.laplacian_2d(128), 1e-10),
])
def test_mixed_reaches_fp64_accuracy(torch, name, make, rtol):
    A = make()
    b = W.rhs(A.nrows, 33)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    bd = torch.from_numpy(b).cuda()
    x64, r64 = gb.CgSolver(M).solve(bd, tol=rtol, relative=True, niter=20000)
    xm, rm = gb.CgSolver(M, mode=gb.CG_MIXED).solve(bd, tol=rtol, relative=True, niter=20000)
    assert r64.status == "converged" and rm.status == "converged", (r64, rm)
    xm_h = xm.cpu().numpy()
    # the solver's own true residual and the host FP64 residual agree
    assert _rel_res(A, xm_h, b) <= 1.05 * rtol, (name, _rel_res(A, xm_h, b))
    assert rm.rnorm == pytest.approx(_rel_res(A, xm_h, b) * np.linalg.norm(b), rel=1e-3)
    assert rm.refinements >= 1
    # inner FP32 iterations stay close to the FP64 count
    assert rm.iterations <= 1.25 * r64.iterations + 10, (rm.iterations, r64.iterations)
    x64_h = x64.cpu().numpy()
    assert np.linalg.norm(xm_h - x64_h) <= 1e-6 * np.linalg.norm(x64_h) + 1e-12


def test_mixed_iteration_limit_folds_the_correction(torch):
    A = W.diffusion_3d(16, seed=41)
    b = W.rhs(A.nrows, 41)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    xm, rm, hist = gb.CgSolver(M, mode=gb.CG_MIXED).solve(
        torch.from_numpy(b).cuda(), tol=1e-14, relative=True, niter=25, history=True)
    assert rm.status == "maxiter" and rm.iterations == 25 and len(hist) == 25
    # the reported norm is the true residual of the returned x
    true = np.linalg.norm(b - A.to_scipy() @ xm.cpu().numpy())
    assert rm.rnorm == pytest.approx(true, rel=1e-6)


def test_mixed_is_deterministic(torch):
    A = W.diffusion_2d(64, seed=51)
    b = torch.from_numpy(W.rhs(A.nrows, 51)).cuda()
    S = gb.CgSolver(gb.CsrMatrix.from_host(A, f64=True, f32=True), mode=gb.CG_MIXED)
    x1, r1 = S.solve(b, tol=1e-10)
    x2, r2 = S.solve(b, tol=1e-10)
    assert r1.iterations == r2.iterations and torch.equal(x1, x2)


def test_mixed_needs_both_value_widths():
    A = W.laplacian_2d(8)
    with pytest.raises(gb.GooseberryError):
        gb.CgSolver(gb.CsrMatrix.from_host(A, f64=True, f32=False), mode=gb.CG_MIXED)


@pytest.mark.parametrize("mode", [gb.CG_F64, gb.CG_MIXED])
def test_profile_times_each_kernel_and_leaves_the_solver_ready(torch, mode):
    """gb_cg_profile runs the first iterations launch by launch (the mixed
    solver's FP64 step every time) and reports one mean time per kernel; a
    solve afterwards equals a solve on a fresh solver bit for bit."""
    A = W.diffusion_3d(20, seed=33)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    b = torch.from_numpy(W.rhs(A.nrows, 34)).cuda()
    S = gb.CgSolver(M, mode)
    ms = S.profile(b, iterations=7)
    assert len(ms) == (2 if mode == gb.CG_F64 else 3)
    assert all(t > 0 for t in ms)
    x1, r1 = S.solve(b, tol=1e-10)
    F = gb.CgSolver(M, mode)
    x2, r2 = F.solve(b, tol=1e-10)
    assert r1.status == r2.status == "converged" and r1.iterations == r2.iterations
    assert torch.equal(x1, x2)
    S.close()
    F.close()
    M.close()
