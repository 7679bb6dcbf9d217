"""Seeded synthetic CSR workloads for the SpMV / CG hot path.

Every random draw comes from a counter-based generator: value ``i`` of stream
``s`` under seed ``seed`` is SplitMix64 (Steele, Lea & Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014) applied to
``key(seed, s) + (i + 1) * 0x9E3779B97F4A7C15``.  Draws are therefore
independent of batch size and order, so the CUDA path, the CPU oracle and the
CPU baseline all see identical bytes for the same (seed, stream, index).

Matrices are plain CSR as gooseberry stores them (``src/matrix.h:37-45``):
``rowptr`` uint32[n+1], ``rowind`` uint32[nnz] (sorted within each row),
``rowval`` float64[nnz].  Shapes follow the five benchmark workloads:

* ``uniform_rows``      -- n rows, exactly k distinct uniform columns per row.
* ``laplacian_2d``      -- 5-point Laplacian, diagonal 4, off-diagonals -1.
* ``powerlaw_rows``     -- row lengths from a discrete power law, exact nnz.
* ``diffusion_3d``      -- 7-point variable-coefficient SPD operator.
* ``diffusion_2d``      -- 5-point variable-coefficient SPD operator.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    """SplitMix64 output function (finaliser), vectorised over uint64."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _key(seed: int, stream: int) -> np.uint64:
    with np.errstate(over="ignore"):
        a = _mix(np.array([np.uint64(seed & 0xFFFFFFFFFFFFFFFF)]))[0]
        b = _mix(np.array([np.uint64((stream * 0x632BE59BD9B4E019) & 0xFFFFFFFFFFFFFFFF)]))[0]
    return np.uint64(a ^ b)


def rand_u64(seed: int, stream: int, start: int, count: int) -> np.ndarray:
    """Draws [start, start+count) of stream ``stream`` as uint64."""
    idx = np.arange(start + 1, start + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix(_key(seed, stream) + idx * _GOLDEN)


def rand_unit(seed: int, stream: int, count: int, start: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1): the top 53 bits of each draw."""
    u = rand_u64(seed, stream, start, count) >> np.uint64(11)
    return u.astype(np.float64) * (1.0 / 9007199254740992.0)


def rand_uniform(seed: int, stream: int, count: int, lo: float, hi: float,
                 start: int = 0) -> np.ndarray:
    return lo + (hi - lo) * rand_unit(seed, stream, count, start)


def rand_loguniform(seed: int, stream: int, count: int, lo: float, hi: float) -> np.ndarray:
    return np.exp(rand_uniform(seed, stream, count, np.log(lo), np.log(hi)))


# Stream ids: one per quantity so workloads never share draws.
S_COLS, S_VALS, S_X, S_B, S_LEN, S_FIX, S_FACE, S_BFACE, S_SIDE, S_ARRIVAL = range(1, 11)


@dataclass
class Csr:
    """CSR matrix in gooseberry's layout (``src/matrix.h:37-45``)."""
    nrows: int
    ncols: int
    rowptr: np.ndarray  # uint32[nrows+1]
    rowind: np.ndarray  # uint32[nnz]
    rowval: np.ndarray  # float64[nnz]

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.rowptr.astype(np.int64))

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.rowval, self.rowind.astype(np.int64),
                              self.rowptr.astype(np.int64)), shape=(self.nrows, self.ncols))


def _sorted_subset_rows(seed: int, lengths: np.ndarray, n: int) -> np.ndarray:
    """Per row, ``lengths[i]`` distinct columns uniform over [0, n), sorted.

    A sorted multiset of size L drawn iid-uniform from [0, n-L+1) plus the
    offsets 0..L-1 is a uniform L-subset of [0, n) in increasing order
    (stars and bars).  The sorted multiset is the floor of L sorted continuous
    uniforms, obtained as normalised partial sums of L+1 exponential spacings
    (so no per-row sort is needed).
    """
    lengths = lengths.astype(np.int64)
    nnz = int(lengths.sum())
    if nnz == 0:
        return np.zeros(0, dtype=np.uint32)
    nrows = len(lengths)
    seg = lengths + 1                              # L+1 spacings per row
    total = int(seg.sum())
    e = -np.log1p(-rand_unit(seed, S_COLS, total))  # Exp(1) spacings, > 0 a.s.
    e = np.maximum(e, 1e-300)
    cs = np.cumsum(e)
    seg_end = np.cumsum(seg)                       # exclusive ends
    seg_start = seg_end - seg
    base = np.where(seg_start > 0, cs[np.maximum(seg_start - 1, 0)], 0.0)
    row_total = cs[seg_end - 1] - base
    # position of the first L spacings of each row inside the spacing array
    row_of = np.repeat(np.arange(nrows, dtype=np.int64), lengths)
    within = np.arange(nnz, dtype=np.int64) - np.repeat(np.cumsum(lengths) - lengths, lengths)
    pos = seg_start[row_of] + within
    u = (cs[pos] - base[row_of]) / row_total[row_of]   # sorted in [0,1)
    span = (n - lengths + 1)[row_of].astype(np.float64)
    m = np.minimum(np.floor(u * span), span - 1).astype(np.int64)
    cols = m + within
    return cols.astype(np.uint32)


def uniform_rows(n: int = 100_000, k: int = 10, seed: int = 1) -> Csr:
    """n x n, exactly k distinct columns per row, uniform without replacement
    and sorted; values U[-1, 1]."""
    lengths = np.full(n, k, dtype=np.int64)
    cols = _sorted_subset_rows(seed, lengths, n)
    rowptr = np.arange(0, (n + 1) * k, k, dtype=np.uint64).astype(np.uint32)
    vals = rand_uniform(seed, S_VALS, n * k, -1.0, 1.0)
    return Csr(n, n, rowptr, cols, vals)


def powerlaw_lengths(n: int, nnz: int, seed: int, exponent: float = 2.1,
                     cap: int = 200_000, mean_z: float = 4.893) -> np.ndarray:
    """Row lengths: Z ~ P(k) ∝ k^-exponent on [1, cap] (inverse-CDF draw),
    L = min(cap, max(1, round(Z * (nnz/n) / mean_z))), then +-1 on distinct
    seeded rows until sum(L) == nnz exactly."""
    k = np.arange(1, cap + 1, dtype=np.float64)
    pmf = k ** (-exponent)
    cdf = np.cumsum(pmf)
    cdf /= cdf[-1]
    u = rand_unit(seed, S_LEN, n)
    z = np.searchsorted(cdf, u, side="right") + 1
    z = np.minimum(z, cap)
    target_mean = nnz / n
    L = np.minimum(cap, np.maximum(1, np.rint(z * target_mean / mean_z))).astype(np.int64)
    order = np.argsort(rand_u64(seed, S_FIX, 0, n), kind="stable")
    for _ in range(10_000):  # +-1 passes over distinct seeded rows
        diff = nnz - int(L.sum())
        if diff == 0:
            break
        if diff > 0:
            elig = order[L[order] < min(cap, n)]
            if len(elig) == 0:
                break
            L[elig[:diff]] += 1
        else:
            elig = order[L[order] > 1]
            if len(elig) == 0:
                break
            L[elig[:-diff]] -= 1
    if int(L.sum()) != nnz:
        raise ValueError("cannot hit the requested nnz with these constraints")
    return L


def powerlaw_rows(n: int = 8_000_000, nnz: int = 128_000_000, seed: int = 3,
                  cap: int = 200_000) -> Csr:
    """Power-law row lengths (exponent 2.1, capped), uniform sorted columns,
    values U[-1, 1]."""
    cap = min(cap, n)
    L = powerlaw_lengths(n, nnz, seed, cap=cap)
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(L, out=rowptr[1:])
    cols = _sorted_subset_rows(seed, L, n)
    vals = rand_uniform(seed, S_VALS, nnz, -1.0, 1.0)
    return Csr(n, n, rowptr.astype(np.uint32), cols, vals)


def _assemble_stencil(shape, coef_of_face, bcoef_of_face):
    """Symmetric M-matrix assembly on a structured grid (lexicographic order,
    last axis fastest).  ``coef_of_face(axis)`` gives the coefficient of every
    interior face normal to ``axis`` (array of shape with that axis one
    shorter); ``bcoef_of_face(axis, side)`` the Dirichlet boundary faces.
    Off-diagonals are -c; the diagonal sums every adjacent face coefficient.

    The CSR is written directly, without sorting: with strides s_0 > s_1 >
    ... the columns of a row in increasing order are r - s_0, ..., r - s_{d-1},
    r, r + s_{d-1}, ..., r + s_0 (the ones that exist)."""
    dims = len(shape)
    n = int(np.prod(shape))
    diag = np.zeros(shape, dtype=np.float64)
    coefs = []
    for ax in range(dims):
        c = coef_of_face(ax)
        coefs.append(c)
        lo = [slice(None)] * dims
        hi = [slice(None)] * dims
        lo[ax] = slice(0, shape[ax] - 1)
        hi[ax] = slice(1, shape[ax])
        diag[tuple(lo)] += c
        diag[tuple(hi)] += c
        for side in (0, 1):
            sl = [slice(None)] * dims
            sl[ax] = slice(0, 1) if side == 0 else slice(shape[ax] - 1, shape[ax])
            diag[tuple(sl)] += bcoef_of_face(ax, side)
    strides = [int(np.prod(shape[ax + 1:])) for ax in range(dims)]
    ridx = np.arange(n, dtype=np.int64)
    coords = np.unravel_index(ridx, shape)
    cols, vals, valid = [], [], []
    # lower neighbours, slowest axis first (largest stride -> smallest column)
    for ax in range(dims):
        ok = coords[ax] > 0
        face = np.zeros(n)
        sub = tuple(np.where(ok, coords[a] - (1 if a == ax else 0), 0) for a in range(dims))
        face[ok] = -coefs[ax][tuple(s_[ok] for s_ in sub)]
        cols.append(ridx - strides[ax])
        vals.append(face)
        valid.append(ok)
    cols.append(ridx)
    vals.append(diag.ravel())
    valid.append(np.ones(n, dtype=bool))
    # upper neighbours, fastest axis first
    for ax in reversed(range(dims)):
        ok = coords[ax] < shape[ax] - 1
        face = np.zeros(n)
        sub = tuple(np.where(ok, coords[a], 0) for a in range(dims))
        face[ok] = -coefs[ax][tuple(s_[ok] for s_ in sub)]
        cols.append(ridx + strides[ax])
        vals.append(face)
        valid.append(ok)
    C = np.stack(cols, axis=1)
    V = np.stack(vals, axis=1)
    M = np.stack(valid, axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(M.sum(axis=1))
    return Csr(n, n, rowptr.astype(np.uint32), C[M].astype(np.uint32), V[M])


def laplacian_2d(side: int = 1024) -> Csr:
    """5-point Laplacian on a side x side grid, Dirichlet: diagonal 4, -1 to
    each existing neighbour (missing neighbours dropped)."""
    shape = (side, side)

    def coef(ax):
        s = list(shape)
        s[ax] -= 1
        return np.ones(s, dtype=np.float64)

    def bcoef(ax, side_):
        s = list(shape)
        s[ax] = 1
        return np.ones(s, dtype=np.float64)

    return _assemble_stencil(shape, coef, bcoef)


def diffusion(shape, seed: int, lo: float, hi: float) -> Csr:
    """Variable-coefficient diffusion on a structured grid: one log-uniform
    coefficient in [lo, hi] per interior face (off-diagonal -c) and per
    boundary face (Dirichlet, diagonal only).  Symmetric, diagonally
    dominant, SPD."""
    shape = tuple(int(s) for s in shape)
    dims = len(shape)
    counts = []
    for ax in range(dims):
        s = list(shape)
        s[ax] -= 1
        counts.append(int(np.prod(s)))
    offs = np.concatenate([[0], np.cumsum(counts)])
    allc = rand_loguniform(seed, S_FACE, int(offs[-1]), lo, hi)
    bcounts = []
    for ax in range(dims):
        s = list(shape)
        s[ax] = 1
        bcounts += [int(np.prod(s))] * 2
    boffs = np.concatenate([[0], np.cumsum(bcounts)])
    allb = rand_loguniform(seed, S_BFACE, int(boffs[-1]), lo, hi)

    def coef(ax):
        s = list(shape)
        s[ax] -= 1
        return allc[offs[ax]:offs[ax + 1]].reshape(s)

    def bcoef(ax, side_):
        s = list(shape)
        s[ax] = 1
        k = 2 * ax + side_
        return allb[boffs[k]:boffs[k + 1]].reshape(s)

    return _assemble_stencil(shape, coef, bcoef)


def diffusion_3d(side: int = 160, seed: int = 4) -> Csr:
    return diffusion((side, side, side), seed, 1e-2, 1e2)


def diffusion_2d(side: int, seed: int) -> Csr:
    return diffusion((side, side), seed, 1e-1, 1e1)


def rhs(n: int, seed: int) -> np.ndarray:
    """b uniform in [-1, 1]."""
    return rand_uniform(seed, S_B, n, -1.0, 1.0)


def dense_x(n: int, seed: int) -> np.ndarray:
    """x uniform in [-1, 1]."""
    return rand_uniform(seed, S_X, n, -1.0, 1.0)


def serving_sides(count: int, seed: int, lo: int = 32, hi: int = 512) -> np.ndarray:
    """Grid sides round(exp(U[ln lo, ln hi])) for a request stream."""
    return np.rint(rand_loguniform(seed, S_SIDE, count, lo, hi)).astype(np.int64)


def poisson_arrivals(count: int, rate_per_s: float, seed: int) -> np.ndarray:
    """Arrival times (seconds) of a Poisson process with the given rate."""
    gaps = -np.log1p(-rand_unit(seed, S_ARRIVAL, count)) / rate_per_s
    return np.cumsum(gaps)
