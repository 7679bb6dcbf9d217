"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
code (``src/blas.c``, ``src/cgd.c``, ``src/matrix.c`` compiled unmodified into
``oracle/_ref/libgbref_{f64,f32}.so`` by ``oracle/Makefile``).

The reference ships no test vectors for this path, so these fixtures are the
pin: the oracle restatement and the CUDA path are both checked against them.
Run from the repo root (needs the reference sources at build time only):

    make -C oracle ref && OMP_NUM_THREADS=8 python tests/golden/make_golden.py
    python tests/golden/make_golden.py --only rcm     # just rcm_cases.npz

Fixtures
  spmv_cases.npz  small SpMV cases (inputs + reference outputs, f64 and f32)
  cg_cases.npz    small CG cases (inputs + reference x, iteration counts;
                  reference run on one OpenMP thread)
  rcm_cases.npz   Cuthill-McKee orders (src/permute.c:288-337, compiled with
                  the oracle shim's priority queue: equal degrees smaller
                  id first) and permute_sparse results (src/permute.c:120-205)
  full_sizes.json checksums of the reference SpMV on the full 100k x 100k
                  uniform matrix, and the reference CG iteration count /
                  final ||r|| on the full 1024x1024 Laplacian; with
                  ``--only large``: the reference SpMV checksums (both
                  widths) on the full 8M-row power-law matrix, and the
                  reference CG on the 160^3 3D operator (iterations, norms,
                  and a sample of x in cg_diffusion_160_xsample.npz)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gooseberry_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tridiag(n):
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i)
                cols.append(j)
                vals.append(v)
    rp = np.zeros(n + 1, np.uint32)
    np.add.at(rp, np.array(rows) + 1, 1)
    return W.Csr(n, n, np.cumsum(rp).astype(np.uint32), np.array(cols, np.uint32),
                 np.array(vals))


def ragged(seed):
    """Empty rows, a dense row, a row longer than one SpMV tile, singletons."""
    n = 5000
    lengths = np.zeros(n, np.int64)
    rng_len = W.rand_u64(seed, 20, 0, n) % np.uint64(40)
    lengths[:] = rng_len.astype(np.int64)
    lengths[::7] = 0           # empty rows
    lengths[10] = n            # a fully dense row
    lengths[11] = 3000         # longer than a 2048-item tile
    lengths[4999] = 9000 % n   # long last row
    lengths[12:20] = 1
    rowptr = np.zeros(n + 1, np.uint64)
    np.cumsum(lengths, out=rowptr[1:])
    cols = W._sorted_subset_rows(seed, lengths, n)
    vals = W.rand_uniform(seed, W.S_VALS, int(lengths.sum()), -1.0, 1.0)
    return W.Csr(n, n, rowptr.astype(np.uint32), cols, vals)


def spmv_cases():
    cases = {
        "tridiag5": (tridiag(5), np.arange(1, 6, dtype=np.float64)),
        "uniform300": (W.uniform_rows(300, 10, seed=11), W.dense_x(300, 11)),
        "uniform_k1": (W.uniform_rows(1000, 1, seed=12), W.dense_x(1000, 12)),
        "powerlaw4k": (W.powerlaw_rows(4000, 64000, seed=13, cap=4000), W.dense_x(4000, 13)),
        "ragged5k": (ragged(14), W.dense_x(5000, 14)),
        "laplace16": (W.laplacian_2d(16), W.dense_x(256, 15)),
        "diffusion3d8": (W.diffusion_3d(8, seed=16), W.dense_x(512, 16)),
    }
    out = {}
    for name, (A, x) in cases.items():
        y64 = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, x, real="f64")
        y32 = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval.astype(np.float32),
                              x.astype(np.float32), real="f32")
        out[f"{name}/rowptr"] = A.rowptr
        out[f"{name}/rowind"] = A.rowind
        out[f"{name}/rowval"] = A.rowval
        out[f"{name}/x"] = x
        out[f"{name}/y64"] = y64
        out[f"{name}/y32"] = y32
    # a multi-column product (bncols = 3) and a blocks call on uniform300
    A, _ = cases["uniform300"]
    B = W.rand_uniform(17, W.S_X, 300 * 3, -1.0, 1.0)
    out["spmm3/B"] = B
    out["spmm3/C"] = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, B, bncols=3, real="f64")
    blocks = np.array([0, 50, 50, 120, 300], np.uint32)
    init = np.full(300, 7.0)
    out["blocks/blocks"] = blocks
    out["blocks/C"] = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, cases["uniform300"][1],
                                      blocks=np.array([0, 50, 120], np.uint32),
                                      out=init.copy(), real="f64")
    out["blocks/blocks_partial"] = np.array([0, 50, 120], np.uint32)
    out["blocks/init"] = init
    np.savez_compressed(os.path.join(OUT, "spmv_cases.npz"), **out)
    return sorted(cases)


def cg_cases():
    # one thread: the reference's dots then sum in index order, so its CG is
    # bit-reproducible and pins the restatement exactly
    oracle.ref_set_threads(1)
    cases = {
        "laplace32": (W.laplacian_2d(32), W.rhs(1024, 21), 1e-8, 5000),
        "laplace64": (W.laplacian_2d(64), W.rhs(4096, 22), 1e-8, 5000),
        "diffusion2d40": (W.diffusion_2d(40, seed=23), W.rhs(1600, 23), 1e-10, 5000),
        "diffusion3d12": (W.diffusion_3d(12, seed=24), W.rhs(1728, 24), 1e-10, 5000),
        "maxiter": (W.laplacian_2d(48), W.rhs(2304, 25), 1e-14, 37),
    }
    out = {}
    for name, (A, b, rtol, niter) in cases.items():
        err = rtol * float(np.linalg.norm(b))
        x, it, last = oracle.ref_cgd(A.rowptr, A.rowind, A.rowval, b, err, niter)
        out[f"{name}/rowptr"] = A.rowptr
        out[f"{name}/rowind"] = A.rowind
        out[f"{name}/rowval"] = A.rowval
        out[f"{name}/b"] = b
        out[f"{name}/error"] = np.float64(err)
        out[f"{name}/niter"] = np.int64(niter)
        out[f"{name}/x"] = x
        out[f"{name}/iterations"] = np.int64(it)
    np.savez_compressed(os.path.join(OUT, "cg_cases.npz"), **out)
    oracle.ref_set_threads(int(os.environ.get("OMP_NUM_THREADS", "8") or 8))
    return sorted(cases)


def scrambled_band(n, half, seed):
    """A symmetric band matrix (|i-j| <= half) with its rows and columns
    renumbered by a seeded permutation: bandwidth ~n until reordered."""
    p = np.argsort(W.rand_u64(seed, 30, 0, n), kind="stable").astype(np.int64)
    inv = np.empty(n, np.int64)
    inv[p] = np.arange(n)
    rows, cols = [], []
    for d in range(-half, half + 1):
        i = np.arange(max(0, -d), min(n, n - d))
        rows.append(inv[i])
        cols.append(inv[i + d])
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    o = np.lexsort((c, r))
    r, c = r[o], c[o]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    vals = W.rand_uniform(seed, W.S_VALS, len(c), -1.0, 1.0)
    return W.Csr(n, n, np.cumsum(rp).astype(np.uint32), c.astype(np.uint32), vals)


def isolated(n, seed):
    """Mostly isolated vertices (diagonal only) with a few short chains: many
    one-vertex components."""
    rows, cols = list(range(n)), list(range(n))
    for a in range(0, n - 3, 97):
        rows += [a, a + 1, a + 1, a + 2]
        cols += [a + 1, a, a + 2, a + 1]
    r = np.array(rows)
    c = np.array(cols)
    o = np.lexsort((c, r))
    r, c = r[o], c[o]
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    vals = W.rand_uniform(seed, W.S_VALS, len(c), -1.0, 1.0)
    return W.Csr(n, n, np.cumsum(rp).astype(np.uint32), c.astype(np.uint32), vals)


def rcm_cases():
    cases = {
        "laplace16": (W.laplacian_2d(16), None),
        "band2000": (scrambled_band(2000, 4, 31), None),
        "uniform300": (W.uniform_rows(300, 10, seed=11), None),
        "uniform300_blocks": (W.uniform_rows(300, 10, seed=11),
                              np.array([0, 50, 50, 120, 300], np.uint32)),
        "powerlaw4k": (W.powerlaw_rows(4000, 64000, seed=13, cap=4000), None),
        "ragged5k": (ragged(14), None),
        "isolated3000": (isolated(3000, 32), None),
    }
    out = {}
    for name, (A, blocks) in cases.items():
        # values = entry numbers: distinct, so a permuted copy shows where
        # every entry went (and the file compresses)
        A = W.Csr(A.nrows, A.ncols, A.rowptr, A.rowind,
                  np.arange(len(A.rowind), dtype=np.float64))
        cases[name] = (A, blocks)
        rc, perm = oracle.ref_cuthillmckee(A.rowptr, A.rowind, A.nrows, blocks=blocks)
        assert rc == 1, (name, rc)
        out[f"{name}/rowptr"] = A.rowptr
        out[f"{name}/rowind"] = A.rowind
        if blocks is not None:
            out[f"{name}/blocks"] = blocks
        out[f"{name}/perm"] = perm
        # the reordered matrix P A P^T (the CLI's `permute -p bandwidth`)
        rc, prp, pri, prv = oracle.ref_permute_sparse(A.rowptr, A.rowind, A.rowval, A.ncols,
                                                      perm, perm)
        assert rc == 1, (name, rc)
        assert np.array_equal(prv, A.rowval[prv.astype(np.int64)])
        out[f"{name}/p_rowptr"] = prp
        out[f"{name}/p_rowind"] = pri
        out[f"{name}/p_source"] = prv.astype(np.uint32)  # entry numbers
    # rows only, and columns only, with seeded permutations
    A = cases["uniform300"][0]
    rperm = np.argsort(W.rand_u64(33, 30, 0, 300), kind="stable").astype(np.uint32)
    cperm = np.argsort(W.rand_u64(34, 30, 0, 300), kind="stable").astype(np.uint32)
    for tag, rp_, cp_ in (("rows", rperm, None), ("cols", None, cperm)):
        rc, prp, pri, prv = oracle.ref_permute_sparse(A.rowptr, A.rowind, A.rowval, A.ncols,
                                                      rp_, cp_)
        assert rc == 1
        out[f"perm_{tag}/rowptr"] = A.rowptr
        out[f"perm_{tag}/rowind"] = A.rowind
        out[f"perm_{tag}/rowperm"] = rp_ if rp_ is not None else np.zeros(0, np.uint32)
        out[f"perm_{tag}/colperm"] = cp_ if cp_ is not None else np.zeros(0, np.uint32)
        out[f"perm_{tag}/p_rowptr"] = prp
        out[f"perm_{tag}/p_rowind"] = pri
        out[f"perm_{tag}/p_source"] = prv.astype(np.uint32)
    np.savez_compressed(os.path.join(OUT, "rcm_cases.npz"), **out)
    return sorted(cases)


def full_sizes():
    res = {}
    t = time.time()
    A = W.uniform_rows(100_000, 10, seed=1)
    x = W.dense_x(100_000, 1)
    y = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, x, real="f64")
    res["spmv_uniform_100k"] = {
        "seed": 1, "n": 100_000, "k": 10,
        "y_sha256": hashlib.sha256(y.tobytes()).hexdigest(),
        "y_sum": float(y.sum()), "y_abs_sum": float(np.abs(y).sum()),
        "y_head": y[:8].tolist(),
    }
    print(f"spmv 100k: {time.time() - t:.1f}s", flush=True)
    t = time.time()
    A = W.laplacian_2d(1024)
    b = W.rhs(A.nrows, 2)
    bn = float(np.linalg.norm(b))
    x, it, last = oracle.ref_cgd(A.rowptr, A.rowind, A.rowval, b, 1e-8 * bn, 5000)
    r = b - A.to_scipy() @ x
    res["cg_laplace_1024"] = {
        "seed": 2, "side": 1024, "rtol": 1e-8, "niter": 5000,
        "iterations": it, "bnorm": bn,
        "true_rel_residual": float(np.linalg.norm(r) / bn),
        "x_sum": float(x.sum()),
        "omp_threads": int(os.environ.get("OMP_NUM_THREADS", "0") or 0),
    }
    print(f"cg 1024^2: {it} iterations, {time.time() - t:.1f}s", flush=True)
    with open(os.path.join(OUT, "full_sizes.json"), "w") as f:
        json.dump(res, f, indent=1)


def full_sizes_large():
    """The power-law SpMV (8M rows, 128M nonzeros) through the reference's
    blas_spmult, both value widths, and the reference cgd on the 160^3
    variable-coefficient 3D operator.  Merged into full_sizes.json; a sample
    of the reference CG solution (every (n // 65536)-th entry) goes to
    cg_diffusion_160_xsample.npz."""
    path = os.path.join(OUT, "full_sizes.json")
    res = json.load(open(path)) if os.path.exists(path) else {}
    t = time.time()
    A = W.powerlaw_rows(8_000_000, 128_000_000, seed=3, cap=200_000)
    x = W.dense_x(A.ncols, 3)
    y = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, x, real="f64")
    y32 = oracle.ref_spmm(A.rowptr, A.rowind, A.rowval.astype(np.float32),
                          x.astype(np.float32), real="f32")
    res["spmv_powerlaw_8m"] = {
        "seed": 3, "n": A.nrows, "nnz": int(A.rowptr[-1]), "cap": 200_000,
        "rowptr_sha256": hashlib.sha256(A.rowptr.tobytes()).hexdigest(),
        "y_sha256": hashlib.sha256(y.tobytes()).hexdigest(),
        "y32_sha256": hashlib.sha256(y32.tobytes()).hexdigest(),
        "y_sum": float(y.sum()), "y_abs_sum": float(np.abs(y).sum()),
    }
    print(f"spmv powerlaw 8M: {time.time() - t:.1f}s", flush=True)
    del A, y, y32
    t = time.time()
    A = W.diffusion_3d(160, seed=4)
    b = W.rhs(A.nrows, 4)
    bn = float(np.linalg.norm(b))
    # the reference's dot products reduce in OpenMP thread order, so on this
    # ill-conditioned system its iteration count depends on the thread count:
    # record the range over 1, 2, 4 and 8 threads (the golden x is the 8-thread one)
    by_threads, xs = {}, {}
    for nt in (1, 2, 4, 8):
        oracle.ref_set_threads(nt)
        xs[nt], by_threads[str(nt)], last = oracle.ref_cgd(A.rowptr, A.rowind, A.rowval, b,
                                                           1e-10 * bn, 50000)
    x, it = xs[8], by_threads["8"]
    spread = max(float(np.linalg.norm(xs[p] - xs[q]) / np.linalg.norm(xs[q]))
                 for p in xs for q in xs if p < q)
    r = b - A.to_scipy() @ x
    step = A.nrows // 65536
    np.savez_compressed(os.path.join(OUT, "cg_diffusion_160_xsample.npz"),
                        step=step, x=x[::step].copy())
    res["cg_diffusion_160"] = {
        "seed": 4, "side": 160, "b_seed": 4, "rtol": 1e-10, "niter": 50000,
        "iterations": it, "bnorm": bn, "last_rnorm": last,
        "true_rel_residual": float(np.linalg.norm(r) / bn),
        "x_norm": float(np.linalg.norm(x)), "x_sum": float(x.sum()),
        "x_sample_step": step,
        "omp_threads": 8,
        "reference_iterations_by_threads": by_threads,
        "reference_iterations_range": [min(by_threads.values()), max(by_threads.values())],
        "reference_solution_spread": spread,
        # a solve that stops at rel-res 1e-10 on this operator can sit this far
        # from another that does (mixed precision takes a different path there)
        "solution_tolerance": 1e-8,
    }
    print(f"cg 160^3: {it} iterations, {time.time() - t:.1f}s", flush=True)
    with open(path, "w") as f:
        json.dump(res, f, indent=1)


if __name__ == "__main__":
    if not oracle.ref_available("f64") or not oracle.ref_available("f32"):
        sys.exit("build the reference oracle first: make -C oracle ref")
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "rcm":
        print("rcm:", rcm_cases())
        sys.exit(0)
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "large":
        full_sizes_large()
        sys.exit(0)
    print("spmv:", spmv_cases())
    print("rcm:", rcm_cases())
    print("cg:", cg_cases())
    if "--skip-full" not in sys.argv:
        full_sizes()
