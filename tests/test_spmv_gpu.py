"""SpMV parity on the GPU against the reference (golden fixtures) and the
oracle restatement.  FP64 bar: |y - y_ref| <= 1e-13 * sum_k |a_ik x_k| per row
(the 1e-13 relative-per-row target, scaled by the row's condition so rows that
cancel to ~0 are judged fairly).  FP32 (float values, float accumulation as in
the reference's float build): the same form at 64 * 2^-24."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import gooseberry_b200 as gb
import oracle
from gooseberry_b200 import workloads as W
from conftest import cond_scaled_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 64 * 2.0 ** -24
SCHEDS = [gb.SCHED_THREAD, gb.SCHED_GROUP4, gb.SCHED_GROUP8, gb.SCHED_WARP, gb.SCHED_MERGE,
          gb.SCHED_ROW, gb.SCHED_WTILE, gb.SCHED_WMERGE, gb.SCHED_SEG]


def _tile_for(sched, tile):
    """Per-warp schedules take small tiles (WTILE <= 512, WMERGE <= 128)."""
    if sched == gb.SCHED_WTILE:
        return max(64, tile // 8)
    if sched == gb.SCHED_WMERGE:
        return min(128, max(64, tile // 8))
    return tile


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_golden_cases_all_schedules_f64(torch, spmv_golden):
    for name, c in spmv_golden.items():
        if "rowptr" not in c:
            continue
        A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"], rowval=c["rowval"],
                                   f64=True, f32=True)
        x = _dev(torch, c["x"])
        for tile in (256, 2048):
            for s in SCHEDS:
                A.set_schedule(s, tile_items=_tile_for(s, tile))
                y = A.spmv(x).cpu().numpy()
                err = cond_scaled_err(y, c["y64"], c["rowptr"], c["rowind"], c["rowval"], c["x"])
                assert err <= TOL64, (name, s, tile, err)
                # deterministic: a second run is bitwise identical
                assert np.array_equal(y, A.spmv(x).cpu().numpy()), (name, s, tile)
        A.close()


@pytest.mark.parametrize("sched,tile", [(gb.SCHED_ROW, 2048), (gb.SCHED_WTILE, 128),
                                        (gb.SCHED_WTILE, 256), (gb.SCHED_WTILE, 512)])
def test_reference_order_schedules_are_bit_identical(torch, spmv_golden, sched, tile):
    """The row and per-warp-tile schedules sum each row in the reference's
    order without fused multiply-adds, so their y equals blas_spmult's bit for
    bit (f64 and f32 builds); rows too long for a tile are chunked instead and
    checked to the usual bound."""
    for name, c in spmv_golden.items():
        if "rowptr" not in c:
            continue
        A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"], rowval=c["rowval"],
                                   f64=True, f32=True)
        A.set_schedule(sched, tile_items=tile)
        A.set_schedule(sched, f32=True)
        y = A.spmv(_dev(torch, c["x"])).cpu().numpy()
        y32 = A.spmv(_dev(torch, c["x"].astype(np.float32))).cpu().numpy()
        if sched == gb.SCHED_WTILE and A.info().nlong > 0:
            assert cond_scaled_err(y, c["y64"], c["rowptr"], c["rowind"], c["rowval"],
                                   c["x"]) <= TOL64, name
            continue
        assert np.array_equal(y, c["y64"]), name
        assert np.array_equal(y32, c["y32"]), name


def test_golden_cases_f32(torch, spmv_golden):
    for name, c in spmv_golden.items():
        if "rowptr" not in c:
            continue
        A = gb.CsrMatrix.from_host(rowptr=c["rowptr"], rowind=c["rowind"], rowval=c["rowval"],
                                   f64=False, f32=True)
        x = _dev(torch, c["x"].astype(np.float32))
        for s in SCHEDS:
            A.set_schedule(s, f32=True)
            y = A.spmv(x).cpu().numpy()
            err = cond_scaled_err(y, c["y32"], c["rowptr"], c["rowind"],
                                  c["rowval"].astype(np.float32), c["x"].astype(np.float32))
            assert err <= TOL32, (name, s, err)


def test_dropin_spmult_f64_and_f32(spmv_golden):
    for name, c in spmv_golden.items():
        if "rowptr" not in c:
            continue
        y = gb.spmult(c["rowptr"], c["rowind"], c["rowval"], c["x"])
        assert cond_scaled_err(y, c["y64"], c["rowptr"], c["rowind"], c["rowval"],
                               c["x"]) <= TOL64, name
        y32 = gb.spmult(c["rowptr"], c["rowind"], c["rowval"].astype(np.float32),
                        c["x"].astype(np.float32))
        assert y32.dtype == np.float32
        assert cond_scaled_err(y32, c["y32"], c["rowptr"], c["rowind"],
                               c["rowval"].astype(np.float32),
                               c["x"].astype(np.float32)) <= TOL32, name


def test_dropin_spmm_and_blocks(spmv_golden):
    u = spmv_golden["uniform300"]
    C = gb.spmult(u["rowptr"], u["rowind"], u["rowval"], spmv_golden["spmm3"]["B"], bncols=3)
    # the fused multi-column kernel sums in the reference's order: bitwise
    assert np.array_equal(C, spmv_golden["spmm3"]["C"])
    bl = spmv_golden["blocks"]
    out = bl["init"].copy()
    gb.spmult(u["rowptr"], u["rowind"], u["rowval"], u["x"], blocks=bl["blocks_partial"],
              out=out)
    np.testing.assert_allclose(out, bl["C"], rtol=1e-13, atol=1e-13)
    assert np.all(out[120:] == 7.0)
    # nblocks == 0 computes nothing (the reference's cgd -R case)
    out2 = bl["init"].copy()
    gb.spmult(u["rowptr"], u["rowind"], u["rowval"], u["x"], blocks=np.zeros(1, np.uint32),
              out=out2)
    assert np.all(out2 == 7.0)


def test_full_uniform_100k(torch, full_golden):
    g = full_golden["spmv_uniform_100k"]
    A = W.uniform_rows(g["n"], g["k"], seed=g["seed"])
    x = W.dense_x(g["n"], g["seed"])
    y_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval, x, threads=8)
    assert hashlib.sha256(y_ref.tobytes()).hexdigest() == g["y_sha256"]
    M = gb.CsrMatrix.from_host(A)
    xd = _dev(torch, x)
    for s in SCHEDS:
        M.set_schedule(s)
        y = M.spmv(xd).cpu().numpy()
        assert cond_scaled_err(y, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64, s
    M.autotune()
    y = M.spmv(xd).cpu().numpy()
    assert cond_scaled_err(y, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64
    y2 = gb.spmult(A.rowptr, A.rowind, A.rowval, x)
    assert cond_scaled_err(y2, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64


def test_powerlaw_long_rows(torch):
    # rows up to 200k nonzeros: many chunked long rows
    A = W.powerlaw_rows(400_000, 6_400_000, seed=31, cap=200_000)
    x = W.dense_x(A.ncols, 31)
    y_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval, x, threads=8)
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    assert M.info().nlong > 0
    xd = _dev(torch, x)
    for s, t in ((gb.SCHED_MERGE, 2048), (gb.SCHED_GROUP8, 2048), (gb.SCHED_THREAD, 2048),
                 (gb.SCHED_WTILE, 256), (gb.SCHED_WMERGE, 128), (gb.SCHED_WMERGE, 64),
                 (gb.SCHED_SEG, 2048)):
        M.set_schedule(s, tile_items=t)
        y = M.spmv(xd).cpu().numpy()
        assert cond_scaled_err(y, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64, s
        assert np.array_equal(y, M.spmv(xd).cpu().numpy())
    y32_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval.astype(np.float32),
                          x.astype(np.float32), threads=8, real="f32")
    for s in (gb.SCHED_MERGE, gb.SCHED_SEG):
        M.set_schedule(s, f32=True)
        y32 = M.spmv(_dev(torch, x.astype(np.float32))).cpu().numpy()
        assert cond_scaled_err(y32, y32_ref, A.rowptr, A.rowind, A.rowval.astype(np.float32),
                               x.astype(np.float32)) <= TOL32, s


def _lens_csr(lens, ncols, seed):
    """A CSR matrix with the given row lengths, uniform columns and values."""
    rng = np.random.default_rng(seed)
    lens = np.asarray(lens, dtype=np.int64)
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    nnz = int(rowptr[-1])
    rowind = rng.integers(0, ncols, nnz).astype(np.uint32)
    rowval = rng.uniform(-1, 1, nnz)
    return rowptr, rowind, rowval


@pytest.mark.parametrize("case", ["empty_runs", "one_huge_row", "huge_rows_between_empties",
                                  "trailing_empties", "leading_empties", "ragged_pareto",
                                  "tiny"])
def test_segmented_schedule_edge_cases(torch, case):
    """The SEG schedule cuts nonzeros into per-warp ranges wherever the
    merge-path split lands: rows that cross ranges (and runs of empty rows at
    range starts, or after the last nonzero) must come out once and right,
    and bitwise the same on every run (the cross-range sums go in warp order)."""
    rng = np.random.default_rng(7)
    lens = {
        "empty_runs": [0] * 3000 + [5] * 20_000 + [0] * 7000 + [3] * 9000 + [0] * 100,
        "one_huge_row": [300_000],
        "huge_rows_between_empties": [0, 150_000, 0, 0, 70_001, 1, 0, 90_003, 0],
        "trailing_empties": [7] * 50_000 + [0] * 40_000,
        "leading_empties": [0] * 40_000 + [9] * 50_000,
        "ragged_pareto": list((rng.pareto(1.1, 200_000) * 3).astype(int)),
        "tiny": [1, 0, 2],
    }[case]
    ncols = 50_000
    rp, ri, rv = _lens_csr(lens, ncols, seed=len(lens))
    x = W.dense_x(ncols, 3)
    y_ref = oracle.spmv(rp, ri, rv, x, threads=8)
    M = gb.CsrMatrix.from_host(rowptr=rp, rowind=ri, rowval=rv, ncols=ncols, f64=True, f32=True)
    M.set_schedule(gb.SCHED_SEG)
    M.set_schedule(gb.SCHED_SEG, f32=True)
    xd = _dev(torch, x)
    y = M.spmv(xd).cpu().numpy()
    assert cond_scaled_err(y, y_ref, rp, ri, rv, x) <= TOL64
    for _ in range(3):
        assert np.array_equal(y, M.spmv(xd).cpu().numpy())
    y32_ref = oracle.spmv(rp, ri, rv.astype(np.float32), x.astype(np.float32), threads=8,
                          real="f32")
    y32 = M.spmv(_dev(torch, x.astype(np.float32))).cpu().numpy()
    assert cond_scaled_err(y32, y32_ref, rp, ri, rv.astype(np.float32),
                           x.astype(np.float32)) <= TOL32


def test_segmented_plan_survives_tile_rebuilds(torch):
    """SEG's plan is built when SEG is first chosen and kept when another
    schedule rebuilds the tile plan at a new tile size: switching back to SEG
    gives the same bits, and the tile schedule in between is right too."""
    A = W.powerlaw_rows(60_000, 900_000, seed=12, cap=40_000)
    x = W.dense_x(A.ncols, 12)
    y_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval, x, threads=8)
    M = gb.CsrMatrix.from_host(A)
    xd = _dev(torch, x)
    M.set_schedule(gb.SCHED_SEG)
    y1 = M.spmv(xd).cpu().numpy()
    assert cond_scaled_err(y1, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64
    for tile in (512, 4096):
        M.set_schedule(gb.SCHED_MERGE, tile_items=tile)
        y2 = M.spmv(xd).cpu().numpy()
        assert cond_scaled_err(y2, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64
        M.set_schedule(gb.SCHED_SEG)
        assert np.array_equal(M.spmv(xd).cpu().numpy(), y1)
    M.autotune()  # the tuner's SEG candidate reuses the kept plan
    y3 = M.spmv(xd).cpu().numpy()
    assert cond_scaled_err(y3, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64


def test_segmented_schedule_needs_aligned_arrays(torch):
    """Borrowed device arrays that do not start on a 16-byte boundary cannot
    take the SEG schedule's 16-byte loads: choosing it is refused."""
    A = W.uniform_rows(3000, 7, seed=41)
    rp = _dev(torch, A.rowptr.view(np.int32))
    ri = _dev(torch, np.concatenate([np.zeros(1, np.uint32), A.rowind]).view(np.int32))[1:]
    v = _dev(torch, A.rowval)
    M = gb.CsrMatrix.from_device(rp, ri, val64=v)
    with pytest.raises(gb.GooseberryError) as e:
        M.set_schedule(gb.SCHED_SEG)
    assert e.value.code == 3 and "16-byte" in str(e.value)
    M.set_schedule(gb.SCHED_MERGE)
    x = W.dense_x(3000, 41)
    y = M.spmv(_dev(torch, x)).cpu().numpy()
    y_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval, x)
    assert cond_scaled_err(y, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64


def test_device_pointer_matrix(torch):
    A = W.uniform_rows(3000, 7, seed=41)
    x = W.dense_x(3000, 41)
    rp = _dev(torch, A.rowptr.view(np.int32))
    ri = _dev(torch, A.rowind.view(np.int32))
    v = _dev(torch, A.rowval)
    M = gb.CsrMatrix.from_device(rp, ri, val64=v)
    y = M.spmv(_dev(torch, x)).cpu().numpy()
    y_ref = oracle.spmv(A.rowptr, A.rowind, A.rowval, x)
    assert cond_scaled_err(y, y_ref, A.rowptr, A.rowind, A.rowval, x) <= TOL64


def test_empty_and_degenerate(torch):
    # all rows empty: y = 0
    rp = np.zeros(101, np.uint32)
    M = gb.CsrMatrix.from_host(rowptr=rp, rowind=np.zeros(0, np.uint32),
                               rowval=np.zeros(0), ncols=100)
    for s in (gb.SCHED_AUTO, gb.SCHED_SEG):
        M.set_schedule(s)
        y = M.spmv(torch.ones(100, dtype=torch.float64, device="cuda"))
        assert torch.count_nonzero(y).item() == 0
    # zero rows: nothing to do
    y = gb.spmult(np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0), np.zeros(4),
                  ncols=4)
    assert y.size == 0


def test_invalid_input_is_rejected_before_any_kernel():
    rp = np.array([0, 2, 3], np.uint32)
    ri = np.array([0, 5, 1], np.uint32)  # column 5 of a 2-column matrix
    with pytest.raises(gb.GooseberryError) as e:
        gb.spmult(rp, ri, np.ones(3), np.ones(2), ncols=2)
    assert e.value.code == 3 and "out of range" in str(e.value)
    with pytest.raises(gb.GooseberryError):
        gb.spmult(np.array([0, 2, 1], np.uint32), ri, np.ones(3), np.ones(2), ncols=2)


def test_blas1_device(torch):
    a = _dev(torch, W.dense_x(100_003, 1))
    b = _dev(torch, W.rhs(100_003, 2))
    ref = float(np.dot(a.cpu().numpy(), b.cpu().numpy()))
    assert abs(gb.dot(a, b) - ref) <= 1e-12 * float(torch.sum(torch.abs(a * b)))
    assert gb.dot(a, b) == gb.dot(a, b)
    v = np.arange(10, dtype=np.float64)
    gb.scale(v, 2.5)
    assert np.array_equal(v, np.arange(10) * 2.5)
    gb.add_scalar(v, 1.0)
    assert np.array_equal(v, np.arange(10) * 2.5 + 1.0)
    w = np.arange(10, dtype=np.float32)
    gb.scale(w, 0.5)
    assert np.array_equal(w, np.arange(10, dtype=np.float32) * np.float32(0.5))


@pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build missing")
def test_add_sub_match_reference_bitwise(torch):
    """gb_add_f64 / gb_sub_f64 against the reference's own blas_add / blas_sub
    (src/blas.c:275-290,321-336) on the same vectors, bit for bit, including
    the aliased forms cgd uses (c = b at src/cgd.c:105, and c = a)."""
    n = 1_000_003
    a = W.dense_x(n, 61)
    b = W.rhs(n, 62) * 1e3
    for subtract in (False, True):
        fn = gb.sub if subtract else gb.add
        ref = oracle.ref_axpby(a, b, np.empty(n), subtract=subtract)
        got = fn(_dev(torch, a), _dev(torch, b)).cpu().numpy()
        assert np.array_equal(got, ref), subtract
        # c aliases b, then a
        bb = b.copy()
        oracle.ref_axpby(a, bb, bb, subtract=subtract)
        bd = _dev(torch, b)
        fn(_dev(torch, a), bd, out=bd)
        assert np.array_equal(bd.cpu().numpy(), bb), ("c = b", subtract)
        aa = a.copy()
        oracle.ref_axpby(aa, b, aa, subtract=subtract)
        ad = _dev(torch, a)
        fn(ad, _dev(torch, b), out=ad)
        assert np.array_equal(ad.cpu().numpy(), aa), ("c = a", subtract)
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    assert gb.add(e, e).numel() == 0


def test_spdot_matches_oracle(torch):
    """gb_spdot (blas_spdot, src/blas.c:433-451) on a power-law matrix's own
    indices/values: FP64 within the condition-scaled bound of the sequential
    oracle sum; FP32 inputs are multiplied and summed in double, so they are
    checked against the FP64 oracle of the same float values."""
    A = W.powerlaw_rows(300_000, 4_800_000, seed=41, cap=50_000)
    x = W.dense_x(A.ncols, 41)
    ind = _dev(torch, A.rowind.astype(np.int32))
    ref = oracle.spdot(A.rowind, A.rowval, x)
    scale = float(np.sum(np.abs(A.rowval * x[A.rowind])))
    got = gb.spdot(ind, _dev(torch, A.rowval), _dev(torch, x))
    assert abs(got - ref) <= 1e-13 * scale
    assert got == gb.spdot(ind, _dev(torch, A.rowval), _dev(torch, x))  # fixed order
    v32, x32 = A.rowval.astype(np.float32), x.astype(np.float32)
    ref32 = oracle.spdot(A.rowind, v32.astype(np.float64), x32.astype(np.float64))
    got32 = gb.spdot(ind, _dev(torch, v32), _dev(torch, x32))
    assert abs(got32 - ref32) <= 1e-13 * scale
    assert gb.spdot(ind[:0], _dev(torch, A.rowval[:0]), _dev(torch, x)) == 0.0


@pytest.mark.parametrize("k", [2, 3, 5, 8, 13])
def test_fused_spmm_bitwise(torch, k):
    """gb_spmm_f64 reads A once for all k columns; every output is summed
    k ascending with unfused multiply and add, so C equals the reference
    order bit for bit (stencil, uniform and short power-law rows).  Rows too
    long for the fused kernel take the per-column SpMV, within the SpMV bound."""
    mats = [W.diffusion_2d(90, seed=3), W.uniform_rows(20_000, 10, seed=4),
            W.powerlaw_rows(30_000, 240_000, seed=5, cap=200)]
    for A in mats:
        B = np.random.default_rng(k).uniform(-1, 1, A.ncols * k)
        ref = oracle.spmm(A.rowptr, A.rowind, A.rowval, B, ncols=A.ncols, bncols=k)
        M = gb.CsrMatrix.from_host(A)
        C = M.spmm(_dev(torch, B), k).cpu().numpy()
        assert np.array_equal(C, ref), (A.nrows, k)
        M.close()
    A = W.powerlaw_rows(30_000, 480_000, seed=6, cap=20_000)
    B = np.random.default_rng(k).uniform(-1, 1, A.ncols * k)
    ref = oracle.spmm(A.rowptr, A.rowind, A.rowval, B, ncols=A.ncols, bncols=k)
    M = gb.CsrMatrix.from_host(A)
    C = M.spmm(_dev(torch, B), k).cpu().numpy()
    for j in range(k):
        assert cond_scaled_err(C[j::k], ref[j::k], A.rowptr, A.rowind, A.rowval,
                               B[j * A.ncols:(j + 1) * A.ncols]) <= TOL64


def test_csr_read_to_device(torch, tmp_path):
    """gb_csr_read parses a CSR text file into a device matrix; its SpMV equals
    the one of the same arrays uploaded from the host reader's output."""
    A = W.powerlaw_rows(50_000, 600_000, seed=51, cap=5000)
    p = tmp_path / "a.csr"
    gb.write_csr(p, A.rowptr, A.rowind, A.rowval, A.ncols)
    rp, ri, rv, nc = gb.read_csr(p)
    M1 = gb.CsrMatrix.read(p)
    M2 = gb.CsrMatrix.from_host(rowptr=rp, rowind=ri, rowval=rv, ncols=nc)
    assert (M1.nrows, M1.ncols, M1.nnz) == (len(rp) - 1, nc, len(ri))
    x = _dev(torch, W.dense_x(nc, 51))
    M1.set_schedule(gb.SCHED_ROW)
    M2.set_schedule(gb.SCHED_ROW)
    assert np.array_equal(M1.spmv(x).cpu().numpy(), M2.spmv(x).cpu().numpy())
