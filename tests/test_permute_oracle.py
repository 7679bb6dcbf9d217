"""The Cuthill-McKee and sparse-permutation restatements (oracle/gb_oracle.c)
against the reference's own src/permute.c: the committed golden orders, and
random graphs through the reference build where it exists.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from gooseberry_b200 import workloads as W


def bandwidth(rowptr, rowind):
    rows = np.repeat(np.arange(len(rowptr) - 1), np.diff(rowptr.astype(np.int64)))
    return int(np.max(np.abs(rows - rowind.astype(np.int64)))) if len(rowind) else 0


def test_restatement_matches_golden_orders(rcm_golden):
    for name, c in rcm_golden.items():
        if name.startswith("perm_"):
            continue
        n = len(c["rowptr"]) - 1
        perm = oracle.cuthillmckee(c["rowptr"], c["rowind"], n, blocks=c.get("blocks"))
        assert np.array_equal(perm, c["perm"]), name
        assert np.array_equal(np.sort(perm), np.arange(n)), name


def test_permute_sparse_restatement_matches_golden(rcm_golden):
    for name, c in rcm_golden.items():
        n = len(c["rowptr"]) - 1
        vals = np.arange(len(c["rowind"]), dtype=np.float64)
        if name.startswith("perm_"):
            rp = c["rowperm"] if len(c["rowperm"]) else None
            cp = c["colperm"] if len(c["colperm"]) else None
        else:
            rp = cp = c["perm"]
        prp, pri, prv = oracle.permute_sparse(c["rowptr"], c["rowind"], vals, n, rp, cp)
        assert np.array_equal(prp, c["p_rowptr"]), name
        assert np.array_equal(pri, c["p_rowind"]), name
        assert np.array_equal(prv.astype(np.uint32), c["p_source"]), name


def test_reordering_restores_a_scrambled_band(rcm_golden):
    c = rcm_golden["band2000"]
    assert bandwidth(c["rowptr"], c["rowind"]) > 1000
    assert bandwidth(c["p_rowptr"], c["p_rowind"]) <= 2 * 4 * 2


def _random_graph(n, seed, maxlen=12, dup=False, outside=False):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, maxlen, n)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    hi = n + 50 if outside else n  # columns >= n lie outside every block
    ri = rng.integers(0, hi, int(rp[-1])).astype(np.uint32)
    if dup and len(ri) > 10:
        ri[1::5] = ri[0::5][: len(ri[1::5])]  # repeated columns within rows
    return rp, ri


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_matches_reference_random(seed):
    n = 3000
    for kw in ({}, {"dup": True}, {"outside": True}):
        rp, ri = _random_graph(n, seed, **kw)
        for blocks in (None, [0, n], [0, 700, 700, 2000, n], [0, 1, 2, n]):
            b = None if blocks is None else np.array(blocks, np.uint32)
            rc, ref = oracle.ref_cuthillmckee(rp, ri, n, blocks=b)
            assert rc == 1
            assert np.array_equal(oracle.cuthillmckee(rp, ri, n, blocks=b), ref), (kw, blocks)


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_non_square_is_invalid_input():
    rp, ri = _random_graph(100, 5)
    assert oracle.cuthillmckee(rp, ri, 100, 101) is None
    rc, _ = oracle.ref_cuthillmckee(rp, ri, 100, 101)
    assert rc == 3  # GOOSEBERRY_ERROR_INVALIDINPUT


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_permute_sparse_matches_reference_random():
    A = W.powerlaw_rows(5000, 60000, seed=7, cap=5000)
    rng = np.random.default_rng(8)
    rp_ = rng.permutation(5000).astype(np.uint32)
    cp_ = rng.permutation(5000).astype(np.uint32)
    for a, b in ((rp_, cp_), (rp_, None), (None, cp_)):
        o = oracle.permute_sparse(A.rowptr, A.rowind, A.rowval, 5000, a, b)
        rc, *r = oracle.ref_permute_sparse(A.rowptr, A.rowind, A.rowval, 5000, a, b)
        assert rc == 1
        assert all(np.array_equal(x, y) for x, y in zip(o, r))


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_degenerate_graphs_match_reference():
    cases = [
        (np.array([0, 1], np.uint32), np.array([0], np.uint32), 1, None),
        (np.zeros(51, np.uint32), np.zeros(0, np.uint32), 50, None),
        (np.arange(41, dtype=np.uint32), np.arange(40, dtype=np.uint32)[::-1].copy(), 40, None),
        (np.zeros(11, np.uint32), np.zeros(0, np.uint32), 10, np.array([0, 0, 5, 5, 10], np.uint32)),
    ]
    for rp, ri, n, blocks in cases:
        rc, ref = oracle.ref_cuthillmckee(rp, ri if len(ri) else np.zeros(1, np.uint32), n,
                                          blocks=blocks)
        assert rc == 1
        assert np.array_equal(oracle.cuthillmckee(rp, ri, n, blocks=blocks), ref)


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")
def test_permute_dense_restatement_matches_reference():
    rng = np.random.default_rng(9)
    nr, nc = 31, 7
    a = rng.random(nr * nc)
    rp = rng.permutation(nr).astype(np.uint32)
    cp = rng.permutation(nc).astype(np.uint32)
    for r, c in ((rp, cp), (rp, None), (None, cp)):
        for rev in (False, True):
            rc, ref = oracle.ref_permute_dense(a, nr, nc, r, c, rev)
            assert rc == 1
            assert np.array_equal(oracle.permute_dense(a, nr, nc, r, c, rev), ref)
    # the reverse undoes the forward permutation
    f = oracle.permute_dense(a, nr, nc, rp, cp)
    assert np.array_equal(oracle.permute_dense(f, nr, nc, rp, cp, reverse=True), a)
