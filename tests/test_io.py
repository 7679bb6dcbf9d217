"""CSR and grid text files (gooseberry_read_* / _write_*, the reference's
src/io.c formats) against the reference's own readers and writers compiled
into oracle/_ref: the same arrays bit for bit on edge-case and large files,
byte-identical written files, the same error classes.  Host-only (no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import gooseberry_b200 as gb
import oracle
from gooseberry_b200 import workloads as W

pytestmark = pytest.mark.skipif(not oracle.ref_available("f64"), reason="reference build absent")

CSR_CASES = {
    "basic": "1 2.5 3 -1\n\n% comment\n2 4e-3\n3 1.5 1 7",
    "zero_based": "0 1.0 2 2.0\n1 3.5\n",
    "comments": "# head\n' q\n\" d\n/ s\n1 1\n% mm\n",
    "crlf": "1 1.5 2 2.5\r\n3 3.5\r\n",
    "odd_tokens": "1 2 3\n4 5.5 6\n",
    "signs_exp": "1 +1e3 2 -2.5E-2 5 .5\n",
    "blank_only": "\n\n\n",
    "empty": "",
    "no_trailing_newline": "2 1\n1 2",
    "tabs": "1\t2.0\t3\t4.0\n",
}


def _csr_equal(path, f64=True):
    real = "f64" if f64 else "f32"
    rc, n, nc, rp, ri, rv = oracle.ref_read_csr(path, real=real)
    assert rc == 1
    grp, gri, grv, gnc = gb.read_csr(path, f64=f64)
    assert gnc == nc and len(grp) == n + 1
    assert np.array_equal(grp, rp) and np.array_equal(gri, ri)
    assert np.array_equal(grv, rv)


@pytest.mark.parametrize("name", sorted(CSR_CASES))
def test_csr_edge_cases_match_reference(tmp_path, name):
    p = tmp_path / f"{name}.csr"
    p.write_text(CSR_CASES[name])
    _csr_equal(p, f64=True)
    _csr_equal(p, f64=False)


def test_large_csr_round_trip_matches_reference(tmp_path):
    """A 20k-row power-law matrix with some empty rows, written by both writers
    (byte-identical) and read back by both readers (the same arrays)."""
    A = W.powerlaw_rows(20_000, 200_000, seed=21, cap=2000)
    lengths = np.diff(A.rowptr.astype(np.int64))
    keep = np.ones(A.nnz, bool)
    for r in range(0, A.nrows, 997):  # empty rows
        keep[A.rowptr[r]:A.rowptr[r + 1]] = False
        lengths[r] = 0
    rp = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint32)
    ri, rv = A.rowind[keep], A.rowval[keep]
    p_ref, p_ours = tmp_path / "ref.csr", tmp_path / "ours.csr"
    assert oracle.ref_write_csr(p_ref, rp, ri, rv, A.ncols) == 1
    gb.write_csr(p_ours, rp, ri, rv, A.ncols)
    assert p_ref.read_bytes() == p_ours.read_bytes()
    _csr_equal(p_ref)
    _csr_equal(p_ref, f64=False)


GRID_CASES = {
    "basic": "1 2 3\n# c\n4 5 6\n",
    "leading_blank": "\n1 2\n3 4\n",
    "one_col": "1\n2\n3",
    "exp": "1e-3 -2E+4\n+5 .25\n",
}


@pytest.mark.parametrize("name", sorted(GRID_CASES))
def test_grid_cases_match_reference(tmp_path, name):
    p = tmp_path / f"{name}.grid"
    p.write_text(GRID_CASES[name])
    rc, n, nc, vals = oracle.ref_read_grid(p)
    assert rc == 1
    g = gb.read_grid(p)
    assert g.shape == (n, nc)
    # values fill the grid in order; a leading blank line counts as a row
    # whose slots the reference leaves unwritten, so compare what was read
    nvals = sum(len(line.split()) for line in GRID_CASES[name].splitlines()
                if line and line[0] not in "#%'\"/")
    assert np.array_equal(g.reshape(-1)[:nvals], vals[:nvals])


def test_ragged_grid_is_invalid_like_reference(tmp_path):
    for text in ("1 2\n3\n", "1 2\n\n3 4\n"):
        p = tmp_path / "bad.grid"
        p.write_text(text)
        assert oracle.ref_read_grid(p)[0] == 3  # GOOSEBERRY_ERROR_INVALIDINPUT
        with pytest.raises(gb.GooseberryError) as e:
            gb.read_grid(p)
        assert e.value.code == 3


def test_grid_writer_is_byte_identical(tmp_path):
    v = np.random.default_rng(3).uniform(-1e6, 1e6, (57, 13))
    v[3, 4] = 0.0
    v[5, 6] = 1e-300
    pr, po = tmp_path / "ref.grid", tmp_path / "ours.grid"
    assert oracle.ref_write_grid(pr, v.reshape(-1), 57, 13) == 1
    gb.write_grid(po, v)
    assert pr.read_bytes() == po.read_bytes()
    back = gb.read_grid(po)
    assert np.allclose(back, v, rtol=1e-5)  # %g keeps 6 significant digits


def test_error_codes(tmp_path):
    with pytest.raises(gb.GooseberryError) as e:
        gb.read_csr(tmp_path / "missing.csr")
    assert e.value.code == 6  # GOOSEBERRY_ERROR_FILENOTFOUND
    p = tmp_path / "a.csr"
    p.write_text("1 1\n")
    L = gb.lib()
    out = [np.zeros(1, np.uint64) for _ in range(5)]
    rc = L.gooseberry_read_sparse_matrix_f64(5, str(p).encode(), *[o.ctypes.data for o in out])
    assert rc == 2  # GOOSEBERRY_ERROR_UNIMPLEMENTED (GRAPH format)
    rc = L.gooseberry_read_sparse_matrix_f64(42, str(p).encode(), *[o.ctypes.data for o in out])
    assert rc == 3  # unknown format


def _odd_values(rng, m):
    """Values whose %g spelling has edge cases: non-finite, signed zero,
    subnormal, rounding ties at the sixth digit, the %f/%e switch points."""
    v = rng.uniform(-1, 1, m) * 10.0 ** rng.integers(-12, 12, m)
    special = [np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0, 5e-324, 2.2250738585072014e-308,
               1.7976931348623157e308, 999999.5, 9999995.0, 1e-5, 9.999995e-5, 0.0001,
               123456.5, 1e6, 100000.0, 0.5, 2.5]
    v[: len(special)] = special
    return v


def test_writers_byte_identical_on_odd_values_and_shapes(tmp_path):
    """A row longer than the writer's 8 MiB formatting chunk, empty rows,
    non-finite / subnormal / tie values, both value widths; and empty files."""
    rng = np.random.default_rng(17)
    lengths = np.array([0, 3, 400_000, 0, 1, 25, 0], np.int64)
    rp = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint32)
    nnz = int(rp[-1])
    ri = rng.integers(0, 2**32 - 2, nnz, dtype=np.uint64).astype(np.uint32)
    rv = _odd_values(rng, nnz)
    with np.errstate(over="ignore"):  # DBL_MAX becomes inf in float
        rv32 = rv.astype(np.float32)
    for real, vals in (("f64", rv), ("f32", rv32)):
        pr, po = tmp_path / f"ref_{real}.csr", tmp_path / f"ours_{real}.csr"
        assert oracle.ref_write_csr(pr, rp, ri, vals, 2**32 - 1, real=real) == 1
        gb.write_csr(po, rp, ri, vals, 2**32 - 1)
        assert pr.read_bytes() == po.read_bytes(), real
    g = _odd_values(rng, 300 * 7).reshape(300, 7)
    with np.errstate(over="ignore"):
        g32 = g.astype(np.float32)
    for real, vals in (("f64", g), ("f32", g32)):
        pr, po = tmp_path / f"ref_{real}.grid", tmp_path / f"ours_{real}.grid"
        assert oracle.ref_write_grid(pr, vals.reshape(-1), 300, 7, real=real) == 1
        gb.write_grid(po, vals)
        assert pr.read_bytes() == po.read_bytes(), real
    # nothing to write: an empty file, like the reference
    pe = tmp_path / "empty.csr"
    gb.write_csr(pe, np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0), 0)
    assert pe.read_bytes() == b""
    pe = tmp_path / "empty_rows.csr"
    gb.write_csr(pe, np.zeros(4, np.uint32), np.zeros(0, np.uint32), np.zeros(0), 0)
    assert pe.read_bytes() == b"\n\n\n"


@pytest.mark.skipif(not __import__("os").path.exists("/dev/full"), reason="no /dev/full")
def test_writer_reports_a_full_device():
    """Every formatting chunk still takes its turn after a failed write, so the
    call returns GOOSEBERRY_ERROR_WRITE instead of blocking."""
    A = W.powerlaw_rows(50_000, 1_000_000, seed=4, cap=5000)
    with pytest.raises(gb.GooseberryError) as e:
        gb.write_csr("/dev/full", A.rowptr, A.rowind, A.rowval, A.ncols)
    assert e.value.code == 5  # GOOSEBERRY_ERROR_WRITE


# Tokens strtoull (indices) and strtod (values) read whole.  On these the
# reference's CSR reader is well defined: it sizes each row by its token count
# over two (src/io.c:414) and copies that many entries (:457), which equals
# the pairs it parsed only when every token reads whole.
_IDX_TOKENS = ["1", "2", "3", "17", "0", "+3", "-1", "007", "4294967295", "4294967296",
               "99999999999999999999", "5"]
_VAL_TOKENS = ["1.5", "-2e-3", ".5", "5.", "1e400", "-1e400", "1e-400", "inf", "-inf", "nan",
               "NaN", "-INF", "infinity", "nan(123)", "0x1p3", "+.5", "1E5", "0.1",
               "123456789012345678901234567890", "4.9e-324", "-0", "7"]
_SEPS = [" ", "  ", "\t", " \t "]


def _fuzz_csr_text(rng):
    lines = []
    for _ in range(int(rng.integers(0, 30))):
        kind = rng.random()
        if kind < 0.1:
            lines.append(str(rng.choice(list("#%'\"/"))) + " note 1 2")
        elif kind < 0.15:
            lines.append(str(rng.choice(["", " ", "\t"])))
        else:
            toks = []
            for _ in range(int(rng.integers(0, 9))):
                toks.append(str(rng.choice(_IDX_TOKENS if len(toks) % 2 == 0 else _VAL_TOKENS)))
            sep = [str(rng.choice(_SEPS)) for _ in toks]
            line = "".join(s + t for s, t in zip(sep, toks))
            if rng.random() < 0.7:
                line = line.lstrip(" \t")
            if rng.random() < 0.2:
                line += str(rng.choice([" ", "\r", " \r", "\t"]))
            lines.append(line)
    text = "\n".join(lines)
    if rng.random() < 0.5:
        text += "\n"
    return text


def test_csr_reader_fuzz_matches_reference(tmp_path):
    """Seeded random CSR text (odd token counts, signs, wrap-around and
    overflowing indices, 0-based files, inf/nan/hex/subnormal values,
    comments, blank and whitespace-only lines, CR line ends): the same status,
    shape and arrays (bytes, so NaN payloads count) as the reference's reader,
    both widths."""
    rng = np.random.default_rng(2024)
    p = tmp_path / "fuzz.csr"
    for case in range(400):
        p.write_text(_fuzz_csr_text(rng))
        for f64, real in ((True, "f64"), (False, "f32")):
            rc, n, nc, rp, ri, rv = oracle.ref_read_csr(p, real=real)
            ctx = (case, real, p.read_text())
            assert rc == 1, ctx
            grp, gri, grv, gnc = gb.read_csr(p, f64=f64)
            assert gnc == nc and len(grp) == n + 1, ctx
            assert grp.tobytes() == rp.tobytes() and gri.tobytes() == ri.tobytes(), ctx
            assert grv.tobytes() == rv.tobytes(), ctx


def test_csr_reader_keeps_the_pairs_that_parse(tmp_path):
    """Tokens that do not read whole.  The reference overruns its arrays on
    these (rows sized by token count, src/io.c:414,457); here a row holds the
    pairs strtoull/strtod read, in the reference's loop order (src/io.c:423-437):
    the row ends at the first value that does not parse."""
    cases = {
        "1 2.5 12abc 3.0 4 5\n": ([0, 1], [0], [2.5]),          # value "abc" fails
        "0x1f 2.0\n": ([0, 0], [], []),                         # index 0, value "x1f" fails
        "3-1 4 5\n": ([0, 2], [2, 3], [-1.0, 5.0]),             # one token, one pair
        "2 1e 3 4\n": ([0, 1], [1], [1.0]),                     # "e" ends the row
        "1 1\n2 abc\n3 3\n": ([0, 1, 1, 2], [0, 2], [1.0, 3.0]),
    }
    p = tmp_path / "bad.csr"
    for text, (rp, ri, rv) in cases.items():
        p.write_text(text)
        grp, gri, grv, _ = gb.read_csr(p)
        assert grp.tolist() == rp and gri.tolist() == ri and grv.tolist() == rv, text


def test_grid_reader_fuzz_matches_reference(tmp_path):
    """Seeded random grids, some ragged, with any of the tokens above or
    tokens that read in part ("2.5e+3x", "1e", "abc"): the same status and
    values as the reference's reader (whose two passes parse alike)."""
    partial = ["2.5e+3x", "1e", "abc", "-.e1", "3-1", "1,5", "12abc", "0x1f"]
    rng = np.random.default_rng(7)
    p = tmp_path / "fuzz.grid"
    for case in range(300):
        ncols = int(rng.integers(1, 5))
        lines = [" ".join(str(rng.choice(_VAL_TOKENS)) for _ in range(ncols))]
        for _ in range(int(rng.integers(0, 7))):
            if rng.random() < 0.1:
                lines.append("# c")
                continue
            k = ncols if rng.random() < 0.85 else int(rng.integers(0, ncols + 2))
            toks = [str(rng.choice(_VAL_TOKENS if rng.random() < 0.9 else partial))
                    for _ in range(k)]
            lines.append(str(rng.choice(_SEPS)).join(toks))
        p.write_text("\n".join(lines) + ("\n" if rng.random() < 0.5 else ""))
        for f64, real in ((True, "f64"), (False, "f32")):
            rc, n, nc, vals = oracle.ref_read_grid(p, real=real)
            ctx = (case, real, p.read_text())
            if rc != 1:
                with pytest.raises(gb.GooseberryError) as e:
                    gb.read_grid(p, f64=f64)
                assert e.value.code == rc, ctx
                continue
            g = gb.read_grid(p, f64=f64)
            assert g.shape == (n, nc), ctx
            assert g.reshape(-1).tobytes() == vals[: n * nc].tobytes(), ctx
