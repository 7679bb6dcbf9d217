"""Cuthill-McKee ordering and sparse permutation on the device
(gooseberry_permute_cuthillmckee / gb_csr_cuthillmckee, src/permute.c:288-337;
gooseberry_permute_sparse / gb_csr_permute, src/permute.c:120-205) against the
golden orders made by the reference's own permute.c and against the oracle
restatement.  An order is a permutation: equality is exact."""
from __future__ import annotations

import numpy as np
import pytest

import gooseberry_b200 as gb
import oracle
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _blocks(c):
    return c["blocks"] if "blocks" in c else None


def test_drop_in_order_matches_golden(rcm_golden):
    for name, c in rcm_golden.items():
        if name.startswith("perm_"):
            continue
        n = len(c["rowptr"]) - 1
        perm = gb.cuthillmckee(c["rowptr"], c["rowind"], n, blocks=_blocks(c))
        assert np.array_equal(perm, c["perm"]), name


def test_device_order_matches_golden(rcm_golden):
    import torch
    for name, c in rcm_golden.items():
        if name.startswith("perm_"):
            continue
        A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"],
                                   rowval=np.ones(len(c["rowind"])))
        perm = A.cuthillmckee(blocks=_blocks(c))
        torch.cuda.synchronize()
        assert np.array_equal(perm.cpu().numpy().astype(np.uint32), c["perm"]), name
        A.close()


def _star(n, extra_seed):
    """Vertex 0 joined to every other vertex, plus a sparse random part: the
    first levels have one vertex but more entries than one CTA expands."""
    rng = np.random.default_rng(extra_seed)
    rows = [np.zeros(n - 1, np.int64), np.arange(1, n)]
    cols = [np.arange(1, n), np.zeros(n - 1, np.int64)]
    r = rng.integers(1, n, 3 * n)
    c = rng.integers(1, n, 3 * n)
    rows += [r, c]
    cols += [c, r]
    R = np.concatenate(rows)
    Cc = np.concatenate(cols)
    o = np.lexsort((Cc, R))
    R, Cc = R[o], Cc[o]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, R + 1, 1)
    return np.cumsum(rp).astype(np.uint32), Cc.astype(np.uint32)


@pytest.mark.parametrize("case", ["uniform200k", "powerlaw300k", "laplace300", "star100k",
                                  "uniform_blocks", "isolated50k"])
def test_large_orders_match_oracle(case):
    """Sizes that take the device-wide level path (wide levels, a hub row) as
    well as the single-CTA one (a long thin mesh BFS, many components)."""
    blocks = None
    if case == "uniform200k":
        A = W.uniform_rows(200_000, 10, seed=41)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
    elif case == "powerlaw300k":
        A = W.powerlaw_rows(300_000, 4_800_000, seed=42, cap=200_000)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
    elif case == "laplace300":
        A = W.laplacian_2d(300)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
    elif case == "star100k":
        n = 100_000
        rp, ri = _star(n, 43)
    elif case == "uniform_blocks":
        A = W.uniform_rows(120_000, 8, seed=44)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
        blocks = np.array([0, 10_000, 10_000, 70_000, 119_999, 120_000], np.uint32)
    else:
        n = 50_000
        keep = (np.arange(n) % 50) == 0  # every 50th row links to its successor
        lens = 1 + keep.astype(np.int64)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
        ri = np.empty(int(rp[-1]), np.uint32)
        ri[rp[:-1]] = np.arange(n)
        ri[rp[:-1][keep] + 1] = (np.arange(n)[keep] + 1) % n
    want = oracle.cuthillmckee(rp, ri, n, blocks=blocks)
    got = gb.cuthillmckee(rp, ri, n, blocks=blocks)
    assert np.array_equal(got, want)


def test_drop_in_permute_sparse_matches_golden(rcm_golden):
    for name, c in rcm_golden.items():
        n = len(c["rowptr"]) - 1
        if name.startswith("perm_"):
            rp = c["rowperm"] if len(c["rowperm"]) else None
            cp = c["colperm"] if len(c["colperm"]) else None
        else:
            rp = cp = c["perm"]
        for dt in (np.float64, np.float32):
            vals = np.arange(len(c["rowind"])).astype(dt)
            prp, pri, prv = gb.permute_sparse(c["rowptr"], c["rowind"], vals, n, rp, cp)
            assert np.array_equal(prp, c["p_rowptr"]), name
            assert np.array_equal(pri, c["p_rowind"]), name
            assert np.array_equal(prv.astype(np.uint32), c["p_source"]), (name, dt)


def test_device_permute_then_spmv_is_the_permuted_product():
    """P A P^T (P x) = P (A x), bit for bit: rows keep their entry order and the
    row-per-thread schedule sums them in that order."""
    import torch
    A = W.powerlaw_rows(200_000, 3_200_000, seed=45, cap=50_000)
    x = W.dense_x(A.nrows, 45)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    perm = M.cuthillmckee()
    P = M.permute(perm, perm)
    assert (P.nrows, P.ncols, P.nnz) == (M.nrows, M.ncols, M.nnz)
    M.set_schedule(gb.SCHED_ROW)
    P.set_schedule(gb.SCHED_ROW)
    xd = torch.from_numpy(x).cuda()
    y = M.spmv(xd)
    px = gb.permute_vector(xd, perm)
    py = P.spmv(px)
    assert torch.equal(py, gb.permute_vector(y, perm))
    assert torch.equal(gb.permute_vector(py, perm, reverse=True), y)
    # the f32 copy was permuted too
    P.set_schedule(gb.SCHED_ROW, f32=True)
    M.set_schedule(gb.SCHED_ROW, f32=True)
    y32 = M.spmv(xd.float())
    assert torch.equal(P.spmv(px.float()), gb.permute_vector(y32.double(), perm).float())
    P.close()
    M.close()


def test_invalid_inputs_are_rejected():
    import torch
    A = W.uniform_rows(1000, 5, seed=46)
    with pytest.raises(gb.GooseberryError) as e:
        gb.cuthillmckee(A.rowptr, A.rowind, 1000, 1001)
    assert e.value.code == 3
    with pytest.raises(gb.GooseberryError):
        gb.cuthillmckee(A.rowptr, A.rowind, 1000, blocks=[0, 500, 999])
    bad = np.arange(1000, dtype=np.uint32)
    bad[5] = 6  # not a permutation
    with pytest.raises(gb.GooseberryError) as e:
        gb.permute_sparse(A.rowptr, A.rowind, A.rowval, 1000, bad, None)
    assert e.value.code == 3
    M = gb.CsrMatrix.from_host(A)
    with pytest.raises(gb.GooseberryError):
        M.permute(torch.from_numpy(bad.astype(np.int32)).cuda(), None)
    M.close()
    # empty block list: nothing ordered, as in the reference
    perm = gb.cuthillmckee(A.rowptr, A.rowind, 1000, blocks=[0])
    assert perm.shape == (1000,)


@pytest.mark.parametrize("case", ["one", "no_entries", "two_components", "anti_diagonal",
                                  "empty_blocks", "outside_columns"])
def test_edge_cases_match_oracle(case):
    """Degenerate graphs: one vertex, rows without entries (every vertex its own
    component, taken in id order), two components, an anti-diagonal (vertex i
    joined to n-1-i), empty row
    blocks, columns outside the matrix (ignored, as the reference's range
    test ignores them)."""
    blocks = None
    if case == "one":
        rp, ri, n = np.array([0, 1], np.uint32), np.array([0], np.uint32), 1
    elif case == "no_entries":
        n = 50
        rp, ri = np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32)
    elif case == "two_components":
        n = 6  # 0-1-2 and 3-4-5 paths, listed backwards
        rows = [[1], [0, 2], [1], [4], [3, 5], [4]]
        rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
        ri = np.array([c for r in rows for c in r], np.uint32)
    elif case == "anti_diagonal":
        n = 40
        rp, ri = np.arange(n + 1, dtype=np.uint32), np.arange(n, dtype=np.uint32)[::-1].copy()
    elif case == "empty_blocks":
        A = W.uniform_rows(2000, 6, seed=47)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
        blocks = np.array([0, 0, 700, 700, 700, 2000, 2000], np.uint32)
    else:
        A = W.uniform_rows(3000, 6, seed=48)
        rp, ri, n = A.rowptr, A.rowind, A.nrows
        blocks = np.array([0, 1000, 3000], np.uint32)  # columns past a block are outside it
    want = oracle.cuthillmckee(rp, ri, n, blocks=blocks)
    got = gb.cuthillmckee(rp, ri, n, blocks=blocks)
    assert np.array_equal(got, want)
    assert np.array_equal(np.sort(got), np.arange(n))


def test_drop_in_permute_dense_matches_oracle():
    """gooseberry_permute_dense[_rev] (src/permute.c:208-283) on a row-major
    matrix and on a vector (one column), both widths, both directions."""
    rng = np.random.default_rng(49)
    for nr, nc in ((1000, 1), (257, 33)):
        a = rng.random(nr * nc)
        rp = rng.permutation(nr).astype(np.uint32)
        cp = rng.permutation(nc).astype(np.uint32)
        for r, c in ((rp, cp), (rp, None), (None, cp)):
            for rev in (False, True):
                want = oracle.permute_dense(a, nr, nc, r, c, rev)
                assert np.array_equal(gb.permute_dense(a, nr, nc, r, c, rev), want)
                got32 = gb.permute_dense(a.astype(np.float32), nr, nc, r, c, rev)
                assert np.array_equal(got32, want.astype(np.float32))
