"""Writes the oracle fixtures of tests/golden (run from the repository root):

    python tests/golden/make_golden.py            # small workloads (seconds)
    python tests/golden/make_golden.py --full     # + the 64^3 work figure
    python tests/golden/make_golden.py --configs [name ...]   # full-size configurations

Each fixture holds the oracle's column permutation, event log and Krylov
result for a seeded workload, and pins the oracle against regressions. The
reference itself cannot be built in this image, so these are not reference
outputs. The full-size 3D work figure (work_advdiff3d_64.json) is the oracle's
algorithmic flop count for the benchmark workload.

--configs writes config_<name>.npz for the full-size configurations the
benchmark and the GPU parity tests use: the event log (every elimination
shape, scaling, RRQR rank, merge size and nnz counter), the Krylov iteration
count and residual, and seeded projections of the one-shot preconditioner
solve and of the Krylov solution (PROJ_ROWS seeded N(0,1) rows, seed
PROJ_SEED), so the GPU test compares vectors without storing them.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle_py as O  # noqa: E402
from spaqr_public_b200 import matgen, work  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
PROJ_ROWS = 8
PROJ_SEED = 77

# full-size configurations: (fixture name, workload, tol override)
CONFIGS = {
    "advdiff3d_64": ("advdiff3d_64", None),
    "contrast2d_512_t1e-1": ("contrast2d_512", 1e-1),
    "contrast2d_512_t1e-2": ("contrast2d_512", 1e-2),
    "contrast2d_512_t1e-3": ("contrast2d_512", 1e-3),
    "lsq2d_256": ("lsq2d_256", None),
}


def projections(x, seed=PROJ_SEED, rows=PROJ_ROWS):
    """rows seeded N(0, 1) projections of x (the GPU tests rebuild the rows)."""
    rng = np.random.default_rng(seed)
    out = np.zeros(rows)
    for i in range(rows):
        out[i] = rng.standard_normal(x.size) @ x
    return out


def spmv_t(A, y):
    """A^T y for A in CSC form."""
    m, n, cp, ri, va = A
    cols = np.repeat(np.arange(n), np.diff(cp))
    out = np.zeros(n)
    np.add.at(out, cols, va * y[ri])
    return out


def fixture(name):
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    t, x, its, r = O.run(A, w["b"], w["n"], w["d"], w["levels"], w["tol"], w["skip"], res=w["res"])
    cp, rp = t.perms()
    return dict(workload=name, levels=w["levels"], tol=w["tol"], skip=w["skip"], cperm=cp.tolist(),
                log=t.log().ravel().tolist(), gmres_its=its, gmres_res=r)


def config_fixture(key):
    name, tol = CONFIGS[key]
    w = matgen.workload(name)
    if tol is not None:
        w["tol"] = tol
    A = matgen.column_normalize(w["A"])
    square = int(A[0] == A[1])
    t0 = time.perf_counter()
    t = O.OracleTree(w["levels"], w["skip"], w["tol"], 1, 1.0, square)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    t1 = time.perf_counter()
    b = np.asarray(w["b"], dtype=np.float64)
    if square:
        xs = t.solve(b)
        x, its, res = t.gmres(A, b, iters=300, tol=w["res"])
    else:
        xs = t.solve_nrml(spmv_t(A, b))
        x, its, res = t.cgls(A, b, iters=300, tol=w["res"])
    t2 = time.perf_counter()
    true = float(np.linalg.norm(matgen.spmv(A, x) - b) / np.linalg.norm(b))
    np.savez_compressed(os.path.join(HERE, f"config_{key}.npz"), log=t.log().astype(np.int64),
                        its=np.int64(its), res=np.float64(res), true_res=np.float64(true),
                        solve_proj=projections(xs), solve_norm=np.float64(np.linalg.norm(xs)),
                        x_proj=projections(x), x_norm=np.float64(np.linalg.norm(x)),
                        levels=np.int64(w["levels"]), skip=np.int64(w["skip"]), tol=np.float64(w["tol"]),
                        res_target=np.float64(w["res"]))
    print(json.dumps(dict(fixture=key, factor_s=round(t1 - t0, 2), krylov_s=round(t2 - t1, 2), its=its, res=res,
                          true_res=true, log_rows=int(t.log().shape[0]))), flush=True)


def main(argv):
    if "--configs" in argv:
        keys = [a for a in argv[argv.index("--configs") + 1:] if not a.startswith("--")] or list(CONFIGS)
        for k in keys:
            config_fixture(k)
        return
    for name in ["advdiff2d_32", "advdiff3d_16"]:
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(fixture(name), f)
        print("wrote", name)
    if "--full" in argv:
        g = fixture("advdiff3d_64")
        out = dict(workload="advdiff3d_64", reference_flops=work.total_flops(g["log"], reference=True),
                   device_flops=work.total_flops(g["log"]), phases_reference=work.phase_flops(g["log"], True),
                   gmres_its=g["gmres_its"], gmres_res=g["gmres_res"],
                   final=[r for r in zip(*[iter(g["log"])] * 8) if r[0] == 6][0])
        with open(os.path.join(HERE, "work_advdiff3d_64.json"), "w") as f:
            json.dump(out, f, indent=1)
        print("wrote work_advdiff3d_64")


if __name__ == "__main__":
    main(sys.argv[1:])
