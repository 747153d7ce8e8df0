"""Writes the oracle fixtures of tests/golden (run from the repository root):

    python tests/golden/make_golden.py

Each fixture holds the oracle's column permutation, event log and GMRES
result for a small seeded workload, and pins the oracle against regressions.
The reference itself cannot be built in this image, so these are not
reference outputs. The full-size 3D work figure (work_advdiff3d_64.json) is the
oracle's algorithmic flop count for the benchmark workload, used to scale the
CPU baseline's bounded sample.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle_py as O  # noqa: E402
from spaqr_public_b200 import matgen, work  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture(name):
    w = matgen.workload(name)
    A = matgen.column_normalize(w["A"])
    t, x, its, r = O.run(A, w["b"], w["n"], w["d"], w["levels"], w["tol"], w["skip"], res=w["res"])
    cp, rp = t.perms()
    return dict(workload=name, levels=w["levels"], tol=w["tol"], skip=w["skip"], cperm=cp.tolist(),
                log=t.log().ravel().tolist(), gmres_its=its, gmres_res=r)


def main(full=False):
    for name in ["advdiff2d_32", "advdiff3d_16"]:
        with open(os.path.join(HERE, f"{name}.json"), "w") as f:
            json.dump(fixture(name), f)
        print("wrote", name)
    if full:
        g = fixture("advdiff3d_64")
        out = dict(workload="advdiff3d_64", reference_flops=work.total_flops(g["log"], reference=True),
                   device_flops=work.total_flops(g["log"]), phases_reference=work.phase_flops(g["log"], True),
                   gmres_its=g["gmres_its"], gmres_res=g["gmres_res"],
                   final=[r for r in zip(*[iter(g["log"])] * 8) if r[0] == 6][0])
        with open(os.path.join(HERE, "work_advdiff3d_64.json"), "w") as f:
            json.dump(out, f, indent=1)
        print("wrote work_advdiff3d_64")


if __name__ == "__main__":
    main(full="--full" in sys.argv)
