"""CG parity on the GPU: same stopping rule and iteration count as the
reference's cgd (within +-2 iterations) and a true residual at the requested
level, on the golden cases and on the full 1024x1024 Laplacian."""
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


def _true_res(c, x):
    import scipy.sparse as sp
    n = len(c["b"])
    A = sp.csr_matrix((c["rowval"], c["rowind"].astype(np.int64),
                       c["rowptr"].astype(np.int64)), shape=(n, n))
    return float(np.linalg.norm(c["b"] - A @ x))


def test_dropin_cgd_matches_reference_iterations(cg_golden):
    for name, c in cg_golden.items():
        err, niter = float(c["error"]), int(c["niter"])
        x, it, rn, hist = gb.cgd(c["rowptr"], c["rowind"], c["rowval"], c["b"], err, niter,
                                 history=True)
        ref_it = int(c["iterations"])
        assert abs(it - ref_it) <= 2, (name, it, ref_it)
        assert len(hist) == it and hist[-1] == pytest.approx(rn)
        if name == "maxiter":
            assert it == niter
        else:
            assert rn <= err and hist[-2] > err
            assert _true_res(c, x) <= 1.5 * err, name
        # the solution agrees with the reference's to the accuracy CG reached
        xr = c["x"]
        assert np.linalg.norm(x - xr) <= 1e-4 * np.linalg.norm(xr) + 1e-12, name


def test_dropin_cgd_into_pinned_out(torch, cg_golden):
    """cgd(out=) writes x into the caller's (here pinned) array: the same bits as
    the default path, and the same array object comes back."""
    c = cg_golden["laplace64"]
    err, niter = float(c["error"]), int(c["niter"])
    x0, it0, rn0 = gb.cgd(c["rowptr"], c["rowind"], c["rowval"], c["b"], err, niter)
    out = torch.empty(len(c["b"]), dtype=torch.float64, pin_memory=True).numpy()
    out[:] = np.nan
    x1, it1, rn1 = gb.cgd(c["rowptr"], c["rowind"], c["rowval"], c["b"], err, niter, out=out)
    assert x1 is out and it1 == it0 and rn1 == rn0
    assert np.array_equal(x1, x0)


def test_device_solver_relative_tolerance(torch, cg_golden):
    c = cg_golden["laplace64"]
    A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"], rowval=c["rowval"])
    S = gb.CgSolver(A)
    b = torch.from_numpy(c["b"]).cuda()
    bn = float(np.linalg.norm(c["b"]))
    x1, r1 = S.solve(b, tol=float(c["error"]) / bn, relative=True, niter=5000)
    x2, r2 = S.solve(b, tol=float(c["error"]), relative=False, niter=5000)
    assert r1.status == "converged" and r1.iterations == r2.iterations
    assert torch.equal(x1, x2)  # bitwise reproducible
    assert abs(r1.iterations - int(c["iterations"])) <= 2
    assert r1.bnorm == pytest.approx(bn, rel=1e-14)


def test_zero_rhs_and_breakdown(torch):
    L = W.laplacian_2d(8)
    A = gb.CsrMatrix.from_host(L)
    S = gb.CgSolver(A)
    x, r = S.solve(torch.zeros(64, dtype=torch.float64, device="cuda"), niter=10)
    assert r.status == "converged" and r.iterations == 0
    assert torch.count_nonzero(x).item() == 0
    neg = W.Csr(L.nrows, L.ncols, L.rowptr, L.rowind, -L.rowval)  # negative definite
    S2 = gb.CgSolver(gb.CsrMatrix.from_host(neg))
    _, r2 = S2.solve(torch.ones(64, dtype=torch.float64, device="cuda"), niter=10)
    assert r2.status == "breakdown"


def test_full_laplacian_1024_matches_reference(torch, full_golden):
    g = full_golden["cg_laplace_1024"]
    L = W.laplacian_2d(g["side"])
    b = W.rhs(L.nrows, g["seed"])
    A = gb.CsrMatrix.from_host(L)
    S = gb.CgSolver(A)
    x, r = S.solve(torch.from_numpy(b).cuda(), tol=g["rtol"], relative=True, niter=g["niter"])
    assert r.status == "converged"
    assert abs(r.iterations - g["iterations"]) <= 2, (r.iterations, g["iterations"])
    xs = x.cpu().numpy()
    res = np.linalg.norm(b - L.to_scipy() @ xs) / np.linalg.norm(b)
    assert res <= 1.5 * g["rtol"]


def test_persistent_and_graph_paths_agree(torch, cg_golden):
    """The one-launch cooperative solve and the graph-replayed two-kernel
    solve run the same algorithm: same iteration count (+-2 of the
    reference), both converged, solutions equal to CG accuracy."""
    for name in ("laplace64", "diffusion3d12"):
        c = cg_golden[name]
        b = torch.from_numpy(c["b"]).cuda()
        out = {}
        for pers in (False, True):
            for sched in (gb.SCHED_ROW, gb.SCHED_THREAD, gb.SCHED_MERGE, gb.SCHED_WTILE):
                A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"],
                                           rowval=c["rowval"])
                A.set_schedule(sched, tile_items=256)
                S = gb.CgSolver(A, persistent=pers)
                x, r = S.solve(b, tol=float(c["error"]), relative=False, niter=int(c["niter"]))
                assert r.status == "converged", (name, pers, sched, r)
                assert abs(r.iterations - int(c["iterations"])) <= 2, (name, pers, sched, r)
                if pers:
                    assert r.kernel_launches == 1
                out[(pers, sched)] = x.cpu().numpy()
        ref = c["x"]
        for k, x in out.items():
            assert np.linalg.norm(x - ref) <= 1e-4 * np.linalg.norm(ref), (name, k)



def test_float_abi_cgd_matches_float_reference(cg_golden):
    """The float drop-in (gooseberry_cgd, the reference's default real_t build)
    solves in double on the device and rounds x to float.  Against the FP64
    oracle on the same float-rounded matrix, right-hand side and threshold:
    iterations +-2, x to CG accuracy.  Against the reference's own float build
    (iterations parsed from its ITER lines): iterations +-2, x to 1e-4."""
    import oracle
    c = cg_golden["laplace64"]
    v32 = c["rowval"].astype(np.float32)
    b32 = c["b"].astype(np.float32)
    err = float(np.float32(c["error"]))
    niter = int(c["niter"])
    x, it, rn = gb.cgd(c["rowptr"], c["rowind"], v32, b32, err, niter)
    assert x.dtype == np.float32
    assert rn <= err
    xo, ito, _ = oracle.cgd(c["rowptr"], c["rowind"], v32.astype(np.float64),
                            b32.astype(np.float64), err, niter)
    assert abs(it - ito) <= 2, (it, ito)
    assert np.linalg.norm(x - xo) <= 1e-4 * np.linalg.norm(xo)
    if oracle.ref_available("f32"):
        oracle.ref_set_threads(1)
        xr, itr, _ = oracle.ref_cgd(c["rowptr"], c["rowind"], v32, b32, err, niter,
                                    real="f32")
        assert abs(it - itr) <= 2, (it, itr)
        assert np.linalg.norm(x - xr) <= 1e-4 * np.linalg.norm(xr)


@pytest.mark.parametrize("mode,persistent", [(gb.CG_F64, True), (gb.CG_F64, False),
                                             (gb.CG_MIXED, False)])
def test_cancel_before_and_during_a_solve(torch, mode, persistent):
    """gb_cg_cancel stops a solve at its next check with status "cancelled".
    A request made before the solve stops it at once (the persistent solve at
    its first grid barrier, which every CTA then leaves, before x moves); a
    request from another thread stops a solve that could not converge long
    before its iteration limit.  The solver works normally afterwards."""
    import threading
    import time
    L = W.laplacian_2d(512)
    A = gb.CsrMatrix.from_host(L, f64=True, f32=(mode == gb.CG_MIXED))
    b = torch.from_numpy(W.rhs(L.nrows, 5)).cuda()
    S = gb.CgSolver(A, mode=mode, persistent=persistent)
    # cancelled before it starts
    S.cancel()
    x, r = S.solve(b, tol=1e-12, niter=200_000)
    assert r.status == "cancelled", r
    assert r.iterations <= (0 if persistent else 128), r
    if persistent:
        assert torch.count_nonzero(x).item() == 0  # stopped before x moved
    # cancelled while running: an unreachable tolerance, a long iteration limit
    t = threading.Timer(0.3, S.cancel)
    t0 = time.time()
    t.start()
    x, r = S.solve(b, tol=1e-300, relative=False, niter=2_000_000)
    dt = time.time() - t0
    t.join()
    assert r.status == "cancelled", r
    assert 0 < r.iterations < 2_000_000 and dt < 30.0, (r, dt)
    assert np.isfinite(r.rnorm)
    # the request was consumed: the next solve runs to convergence
    x, r = S.solve(b, tol=1e-8, niter=20_000)
    assert r.status == "converged", r
    res = np.linalg.norm(b.cpu().numpy() - L.to_scipy() @ x.cpu().numpy())
    assert res <= 2e-8 * np.linalg.norm(b.cpu().numpy())
    S.close()


@pytest.mark.parametrize("drop", ["first", "last"])
def test_persistent_barrier_times_out_and_reports_it(torch, drop):
    """The persistent solve's grid barriers wait with a limit.  With one CTA
    held back from the first barrier (the failure-path hook; no CTA waits
    without a limit), the others give up after the limit, leave, and the
    solve reports "timeout" with a NaN residual -- and the context stays
    usable: the same solver, with the hook off, then converges normally."""
    import time
    L = W.laplacian_2d(256)
    A = gb.CsrMatrix.from_host(L)
    b = torch.from_numpy(W.rhs(L.nrows, 9)).cuda()
    S = gb.CgSolver(A, persistent=True)
    with pytest.raises(gb.GooseberryError):
        S.set_barrier_fault(10 ** 6, 100)  # not a CTA of this solve
    S.set_barrier_fault(0 if drop == "first" else lib_grid(S) - 1, 100)
    t0 = time.time()
    with pytest.raises(gb.GooseberryError) as e:
        S.solve(b, tol=1e-8, niter=5000)
    dt = time.time() - t0
    assert e.value.code == 8 and "timed out" in str(e.value), e.value
    assert 0.1 <= dt < 30.0, dt
    # the limit is per barrier: a longer one takes longer to give up
    S.set_barrier_fault(0 if drop == "first" else lib_grid(S) - 1, 600)
    t0 = time.time()
    with pytest.raises(gb.GooseberryError):
        S.solve(b, tol=1e-8, niter=5000)
    assert time.time() - t0 >= 0.6
    S.set_barrier_fault(-1)
    x, r = S.solve(b, tol=1e-8, niter=5000)
    assert r.status == "converged", r
    res = np.linalg.norm(b.cpu().numpy() - L.to_scipy() @ x.cpu().numpy())
    assert res <= 2e-8 * np.linalg.norm(b.cpu().numpy())
    S.close()


def lib_grid(S):
    """CTAs of a persistent solver's cooperative launch (found by asking the
    hook for CTA indices until it refuses one)."""
    lo, hi = 0, 1 << 20
    while hi - lo > 1:
        mid = (lo + hi) // 2
        try:
            S.set_barrier_fault(mid, 100)
            lo = mid
        except gb.GooseberryError:
            hi = mid
    S.set_barrier_fault(-1)
    return lo + 1
