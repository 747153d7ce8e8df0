"""The full-size oracle fixtures (tests/golden/config_*.npz) against what is
known of them without a GPU: the 64^3 fixture's final counters and GMRES
iterations equal the oracle's separately recorded work figure
(work_advdiff3d_64.json, an independent oracle run), and the contrast sweep
records the oracle's behaviour at each tolerance (no convergence within 300
iterations at tol 1e-1)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _f(key):
    return dict(np.load(os.path.join(GOLDEN, f"config_{key}.npz")))


def test_advdiff3d_64_fixture_agrees_with_work_figure():
    f = _f("advdiff3d_64")
    work = json.load(open(os.path.join(GOLDEN, "work_advdiff3d_64.json")))
    log = f["log"]
    final = log[log[:, 0] == 6]
    assert final.shape[0] == 1
    assert final[0].tolist() == work["final"]
    assert int(f["its"]) == work["gmres_its"] == 11
    assert float(f["true_res"]) <= 1e-10
    # per-level records: 12 levels, the top separator collapses
    lv = log[log[:, 0] == 5]
    assert lv.shape[0] == 12


def test_contrast_sweep_fixtures():
    its = {k: int(_f(f"contrast2d_512_t{k}")["its"]) for k in ("1e-1", "1e-2", "1e-3")}
    assert its["1e-1"] == 300  # the oracle does not converge at tol 1e-1 either
    assert its["1e-2"] < 300 and its["1e-3"] < its["1e-2"]
    logs = [_f(f"contrast2d_512_t{k}")["log"] for k in ("1e-1", "1e-2", "1e-3")]
    # ranks shrink with the tolerance: fewer nonzeros in the factors at 1e-1
    nnz = [int(l[l[:, 0] == 6][0][4]) for l in logs]
    assert nnz[0] < nnz[1] < nnz[2]


def test_lsq_fixture():
    f = _f("lsq2d_256")
    assert 86 <= int(f["its"]) <= 88
    assert float(f["res"]) <= 1e-10
