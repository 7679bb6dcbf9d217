"""The C-ABI library without a GPU: it loads, exports every entry point the
headers declare, and its host-side planner behaves."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

import gooseberry_b200 as gb
from gooseberry_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("gooseberry.h", "gooseberry_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"GOOSEBERRY_API\s+[\w\s\*]+?\b(\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = gb.lib()
    decl = declared_symbols()
    assert len(decl) >= 25
    missing = [n for n in decl if not hasattr(L, n)]
    assert not missing, missing
    # and the Python layer binds exactly what the headers declare
    assert decl == set(gb.SIGNATURES), decl ^ set(gb.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", gb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert decl <= exported


def test_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(gb, "_LIB", None)
    monkeypatch.setattr(gb, "LIB_PATH", "/nonexistent/libgooseberry_b200.so")
    with pytest.raises(ImportError):
        gb.lib()


def _check_plan(rowptr, tiles, nlong, T):
    n = len(rowptr) - 1
    covered = np.zeros(n, np.int64)
    long_rows = []
    for rb, rc, nb, nc in tiles.astype(np.int64):
        if rc == 0:
            long_rows.append(nb)
            continue
        assert rowptr[rb] == nb and rowptr[rb + rc] - nb == nc
        assert nc + rc <= T
        covered[rb:rb + rc] += 1
    lengths = np.diff(rowptr.astype(np.int64))
    is_long = lengths + 1 > T
    assert np.all(covered[~is_long] == 1) and np.all(covered[is_long] == 0)
    assert nlong == int(is_long.sum())
    # chunks of a long row cover it exactly, in order
    chunks = tiles[tiles[:, 1] == 0].astype(np.int64)
    assert chunks[:, 3].sum() == lengths[is_long].sum()


def test_planner_uniform_and_powerlaw():
    for A in (W.uniform_rows(5000, 10, seed=1), W.powerlaw_rows(20000, 320000, seed=2,
                                                                  cap=20000)):
        for T in (256, 2048):
            tiles, nlong, info = gb.plan_tiles(A.rowptr, T)
            _check_plan(A.rowptr, tiles, nlong, T)
            L = A.row_lengths()
            assert info.max_row == L.max()
            assert info.row_p50 == int(np.quantile(L, 0.5, method="inverted_cdf"))


def test_planner_empty_rows_and_empty_matrix():
    rp = np.array([0, 0, 0, 3, 3, 3, 10], np.uint32)
    tiles, nlong, _ = gb.plan_tiles(rp, 64)
    _check_plan(rp, tiles, nlong, 64)
    tiles, nlong, info = gb.plan_tiles(np.zeros(1, np.uint32), 64)
    assert len(tiles) == 0 and nlong == 0


def test_planner_rejects_bad_rowptr():
    with pytest.raises(gb.GooseberryError) as e:
        gb.plan_tiles(np.array([0, 5, 3, 8], np.uint32), 64)
    assert e.value.code == 3 and "decreases" in str(e.value)


def test_reordering_entry_points_reject_bad_input_before_any_device_work():
    """Shape and argument errors of the Cuthill-McKee and permutation drop-ins
    (src/permute.c:120-205,288-337) come back as GOOSEBERRY_ERROR_INVALIDINPUT
    from host-side checks, with no GPU needed."""
    rowptr = np.array([0, 2, 3, 5], np.uint32)
    rowind = np.array([0, 1, 1, 0, 2], np.uint32)
    vals = np.ones(5)
    with pytest.raises(gb.GooseberryError) as e:
        gb.cuthillmckee(rowptr, rowind, 3, 4)  # not square, as the reference
    assert e.value.code == 3 and "symmetric" in str(e.value)
    with pytest.raises(gb.GooseberryError) as e:
        gb.cuthillmckee(rowptr, rowind, 3, blocks=[0, 2])  # blocks miss row 2
    assert e.value.code == 3
    with pytest.raises(gb.GooseberryError) as e:
        gb.cuthillmckee(np.array([0, 2, 1, 5], np.uint32), rowind, 3)
    assert e.value.code == 3
    with pytest.raises(gb.GooseberryError) as e:
        gb.permute_sparse(np.array([0, 3, 2, 5], np.uint32), rowind, vals, 3,
                          np.array([2, 1, 0], np.uint32))
    assert e.value.code == 3
    with pytest.raises(gb.GooseberryError) as e:  # a column past ncols with colperm
        gb.permute_sparse(rowptr, np.array([0, 1, 1, 0, 7], np.uint32), vals, 3, None,
                          np.array([2, 1, 0], np.uint32))
    assert e.value.code == 3
    with pytest.raises(gb.GooseberryError) as e:  # not a permutation
        gb.permute_dense(np.ones(6), 3, 2, np.array([0, 0, 1], np.uint32))
    assert e.value.code == 3
    assert np.array_equal(gb.permute_dense(np.arange(6.0), 3, 2), np.arange(6.0))
    # no permutation: nothing to do, arrays come back unchanged
    rp, ri, rv = gb.permute_sparse(rowptr, rowind, vals, 3)
    assert np.array_equal(rp, rowptr) and np.array_equal(ri, rowind)


def _plan_model(rp, T):
    """The planner's greedy rule, restated: tiles of whole rows while rows +
    nonzeros fit in T; a row with more than T - 1 nonzeros becomes a long row
    cut into chunks of 4T nonzeros.  Tiles are {first row | long-row id, row
    count (0 for a chunk), first nonzero, nonzero count}."""
    rp = rp.astype(np.int64)
    n, chunk = len(rp) - 1, 4 * T
    tiles, nlong, r = [], 0, 0
    while r < n:
        b, L = rp[r], rp[r + 1] - rp[r]
        if L + 1 > T:
            for q in range((L + chunk - 1) // chunk):
                tiles.append((nlong, 0, b + q * chunk, min(chunk, L - q * chunk)))
            nlong += 1
            r += 1
            continue
        r0, items = r, 0
        while r < n:
            l = rp[r + 1] - rp[r]
            if l + 1 > T or items + l + 1 > T:
                break
            items += l + 1
            r += 1
        tiles.append((r0, r - r0, b, rp[r] - b))
    return np.array(tiles, np.int64).reshape(-1, 4), nlong


def _quantile_model(lengths, q):
    """Row-length quantile as the planner reports it: exact below 1024, the
    top of the row's power-of-two bucket above."""
    want = int(np.ceil(q * len(lengths)))
    if want == 0:
        return 0
    v = int(np.sort(lengths)[want - 1])
    return v if v < 1024 else (1 << int(v).bit_length()) - 1


def test_planner_fuzz_matches_greedy_rule():
    """Random row-length mixes (empty rows, short rows, rows just under and
    over a tile, rows of several chunks, lengths past 1024) and tile sizes:
    the planner's tiles, long-row count and row-length summary equal the
    restated rule exactly."""
    rng = np.random.default_rng(12)
    for case in range(80):
        T = int(rng.choice([64, 100, 256, 1000, 2048, 4096]))
        n = int(rng.integers(0, 3000))
        kind = rng.random(n)
        L = np.where(kind < 0.2, 0,
            np.where(kind < 0.8, rng.integers(1, 40, n),
            np.where(kind < 0.9, rng.integers(T - 3, T + 3, n),
                     rng.integers(1, 9 * T, n)))).astype(np.int64)
        rp = np.concatenate([[0], np.cumsum(L)]).astype(np.uint32)
        tiles, nlong, info = gb.plan_tiles(rp, T)
        mt, mlong = _plan_model(rp, T)
        assert nlong == mlong and np.array_equal(tiles.astype(np.int64), mt), (case, T, n)
        if n:
            assert info.max_row == L.max(), case
            for q, got in ((0.5, info.row_p50), (0.9, info.row_p90), (0.99, info.row_p99)):
                assert got == _quantile_model(L, q), (case, q)


def test_planner_parallel_path_matches_greedy_rule():
    """Matrices large enough for the planner to split the rows over host
    threads (each plans its segment from the segment's start, then one pass
    follows the true chain of tiles): the plan equals the sequential rule when
    the segments' chains never meet the true one (uniform rows), meet it at
    long rows, or meet it anywhere."""
    rng = np.random.default_rng(44)
    n = 140_000
    mixes = {
        "uniform": np.full(n, 9),
        "long_rows": np.where(rng.random(n) < 0.002, 5000, rng.integers(1, 30, n)),
        "mixed": np.where(rng.random(n) < 0.2, 0, rng.integers(1, 60, n)),
    }
    for name, L in mixes.items():
        rp = np.concatenate([[0], np.cumsum(L)]).astype(np.uint32)
        for T in (256, 2048):
            tiles, nlong, info = gb.plan_tiles(rp, T)
            mt, mlong = _plan_model(rp, T)
            assert nlong == mlong and np.array_equal(tiles.astype(np.int64), mt), (name, T)
            assert info.max_row == L.max() and info.row_p50 == _quantile_model(L, 0.5), name
    A = W.laplacian_2d(300)  # 90k rows
    tiles, nlong, _ = gb.plan_tiles(A.rowptr, 2048)
    mt, mlong = _plan_model(A.rowptr, 2048)
    assert nlong == mlong and np.array_equal(tiles.astype(np.int64), mt)


def test_planner_many_segments_match_greedy_rule():
    """More than 32 x 32768 rows of mixed lengths: the planner cuts the rows
    into as many segments as the host has threads (up to 32), so the stitch
    along the true chain of tiles crosses every segment boundary."""
    if (os.cpu_count() or 1) < 2:
        pytest.skip("the host has one thread: the planner takes its sequential path")
    rng = np.random.default_rng(45)
    n = 32 * 32768 + 5000
    L = np.where(rng.random(n) < 0.1, 0,
        np.where(rng.random(n) < 0.001, rng.integers(2000, 9000, n),
                 rng.integers(1, 40, n))).astype(np.int64)
    rp = np.concatenate([[0], np.cumsum(L)]).astype(np.uint32)
    tiles, nlong, info = gb.plan_tiles(rp, 2048)
    mt, mlong = _plan_model(rp, 2048)
    assert nlong == mlong and np.array_equal(tiles.astype(np.int64), mt)
    assert info.max_row == L.max()


def test_cgd_out_is_checked_before_any_call():
    """A wrong `out` array is refused on the host, before the library runs."""
    L = W.laplacian_2d(8)
    b = W.rhs(L.nrows, 1)
    for bad in (np.zeros(L.nrows, dtype=np.float32), np.zeros(L.nrows + 1),
                np.zeros((L.nrows, 2))[:, 0]):
        with pytest.raises(ValueError):
            gb.cgd(L.rowptr, L.rowind, L.rowval, b, 1e-8, 100, out=bad)


def test_cgd_rejects_an_empty_system_on_the_host():
    """CG on a 0 x 0 system is refused as an input error before any device
    work, both value widths (the reference's first step would form
    alpha = 0 / 0, src/cgd.c:90)."""
    for dt in (np.float64, np.float32):
        with pytest.raises(gb.GooseberryError) as e:
            gb.cgd(np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0, dt),
                   np.zeros(0, dt), 1e-8, 10)
        assert e.value.code == 3 and "non-empty" in str(e.value)
