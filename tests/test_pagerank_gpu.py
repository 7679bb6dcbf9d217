"""PageRank on the device SpMV (gooseberry_pagerank, the reference's pagerank
command, src/gooseberry_bin.c:2610-2741) against the oracle restatement: same
iteration count, rank within 1e-12 relative (the SpMV and the reductions may
associate sums differently from the sequential reference)."""
from __future__ import annotations

import numpy as np
import pytest

import gooseberry_b200 as gb
import oracle
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _graph(n, nnz, seed, nsinks=0):
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


def _close(a, b, rel=1e-12):
    return float(np.max(np.abs(a - b))) <= rel * float(np.max(np.abs(b)))


@pytest.mark.parametrize("n,nnz", [(3000, 30000), (200_000, 3_200_000)])
def test_pagerank_converges_like_oracle(n, nnz):
    rp, ri, rv = _graph(n, nnz, 11)
    r, it, err = gb.pagerank(rp, ri, rv, 0.85, 1e-10, 0)
    r0, it0, err0 = oracle.pagerank(rp, ri, rv, 0.85, 1e-10, 0)
    assert it == it0 and err <= 1e-10
    assert err == pytest.approx(err0, rel=1e-6)
    assert _close(r, r0)
    assert abs(r.sum() - 1.0) < 1e-9


def test_pagerank_iteration_limit_with_sinks():
    """At the limit the result is the second-to-last iterate, and the sink mass
    is added whole to every entry -- both as the reference does."""
    rp, ri, rv = _graph(5000, 60000, 12, nsinks=9)
    for niter in (1, 10, 17):
        r, it, err = gb.pagerank(rp, ri, rv, 0.9, 0.0, niter)
        r0, it0, err0 = oracle.pagerank(rp, ri, rv, 0.9, 0.0, niter)
        assert it == it0 == niter
        assert _close(r, r0) and err == pytest.approx(err0, rel=1e-9)


def test_pagerank_float_abi():
    rp, ri, rv = _graph(3000, 30000, 13)
    r32, it, _ = gb.pagerank(rp, ri, rv.astype(np.float32), 0.85, 1e-6, 0)
    r0, it0, _ = oracle.pagerank(rp, ri, rv.astype(np.float32).astype(np.float64), 0.85,
                                 1e-6, 0)
    assert r32.dtype == np.float32 and it == it0
    assert np.allclose(r32, r0, rtol=1e-6, atol=0)


def test_pagerank_rejects_bad_input():
    rp, ri, rv = _graph(100, 500, 14)
    bad = ri.copy()
    bad[3] = 100
    with pytest.raises(gb.GooseberryError):
        gb.pagerank(rp, bad, rv, 0.85, 1e-8, 10)
