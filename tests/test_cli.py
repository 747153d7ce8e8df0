"""The `spaqr` command-line driver (reference spaQR.cpp flags and flow).

CPU: help, argument errors, and the MatrixMarket reading printed before any
GPU work (symmetric storage expanded, more columns than rows transposed).
GPU: a square advection-diffusion system through the CLI with --rhs gives the
same GMRES iteration count as the library's own gmres on the column-normalised
matrix, and a residual at the requested tolerance; the FP32 form with --target
reaches the target; a least-squares system runs CGLS.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from spaqr_public_b200 import FP64, Tree, gmres, matgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "spaqr_public_b200", "_build", "spaqr")


def run(*args, timeout=600):
    p = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    return p.returncode, p.stdout, p.stderr


def write_vec(path, b):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix array real general\n")
        f.write(f"{len(b)} 1\n")
        for v in b:
            f.write(f"{float(v)!r}\n")


def test_help_and_argument_errors(tmp_path):
    rc, out, _ = run("--help")
    assert rc == 0 and "--matrix" in out and "--coordinates_n" in out and "--precision" in out
    rc, out, _ = run()
    assert "--matrix is mandatory" in out
    rc, out, _ = run("-m", "x.mtx", "-n", "4")
    assert rc == 1 and "cn and cd should be both provided" in out
    rc, _, err = run("-m", "x.mtx", "--bogus", "1")
    assert rc == 1 and "unknown option --bogus" in err
    rc, _, err = run("-m", "x.mtx", "--useEigenQR", "1")
    assert rc == 1 and "not part of this build" in err
    rc, _, err = run("-m", tmp_path / "missing.mtx")
    assert rc == 1 and "cannot read" in err
    bad = tmp_path / "bad.mtx"
    bad.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n")
    rc, _, err = run("-m", bad)
    assert rc == 1 and "entry count" in err


def test_matrix_market_reading(tmp_path):
    # 2 x 2 grid Laplacian in symmetric (lower) storage: 4 + 2 * 4 = 12 entries after expansion
    sym = tmp_path / "sym.mtx"
    sym.write_text("%%MatrixMarket matrix coordinate real symmetric\n% comment\n4 4 8\n"
                   "1 1 4\n2 1 -1\n3 1 -1\n2 2 4\n4 2 -1\n3 3 4\n4 3 -1\n4 4 4\n")
    # --hsl 1 stops the run at the tree setters, before any device work
    rc, out, err = run("-m", sym, "-n", 2, "-d", 2, "-l", 2, "-t", 0, "--hsl", 1)
    assert "Matrix %s with 4 rows,  4 columns loaded" % sym in out
    assert "Tensor coordinate matrix of size 2^2 built" in out
    assert rc == 1 and "hsl failed (6)" in err
    wide = tmp_path / "wide.mtx"
    wide.write_text("%%MatrixMarket matrix coordinate pattern general\n2 3 3\n1 1\n2 2\n1 3\n")
    rc, out, _ = run("-m", wide, "-n", 1, "-d", 2)
    assert "Finding QR on A.transpose() instead" in out
    assert "with 3 rows,  2 columns loaded" in out
    assert "Scaling necessary" not in out
    assert "cn^cd != N" in out and rc == 1


def _gmres_count(out):
    m = re.search(r"<<<<GMRES=(\d+)", out)
    assert m, out
    return int(m.group(1))


@pytest.mark.gpu
def test_cli_square_matches_library(gpu, tmp_path):
    w = matgen.workload("advdiff2d_64")
    A = w["A"]
    mtx, rhs = tmp_path / "A.mtx", tmp_path / "b.mtx"
    matgen.write_mm(mtx, A)
    write_vec(rhs, w["b"])
    rc, out, err = run("-m", mtx, "-n", 64, "-d", 2, "-l", w["levels"], "-t", w["tol"], "--skip", w["skip"],
                       "--rhs", rhs, "--res", 1e-12)
    assert rc == 0, err
    assert "lvl: 0" in out and "Time to factorize" in out and "<<<<tsolv=" in out
    its = _gmres_count(out)
    res = float(re.search(r"residual \|Ax-b\|/\|b\|: ([0-9.eE+-]+)", out).group(1))
    # the library on the same column-normalised system
    An = matgen.column_normalize(A)
    t = Tree(w["levels"], w["skip"], precision=FP64)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(64, 2)
    t.partition(An)
    t.assemble(An)
    t.factorize()
    _, its_lib, _ = gmres(An, w["b"], t, iters=300, tol=1e-12)
    t.close()
    assert its == its_lib
    assert res <= 1e-11

    rc, out, err = run("-m", mtx, "-n", 64, "-d", 2, "-l", w["levels"], "-t", w["tol"], "--rhs", rhs,
                       "--precision", "fp32", "--target", 1e-10)
    assert rc == 0, err
    res = float(re.search(r"residual \|Ax-b\|/\|b\|: ([0-9.eE+-]+)", out).group(1))
    assert res <= 1e-10 and "target not reached" not in out


@pytest.mark.gpu
def test_cli_least_squares_runs_cgls(gpu, tmp_path):
    A, b, _ = matgen.lsq2d(32, seed=3)
    mtx, rhs = tmp_path / "A.mtx", tmp_path / "b.mtx"
    matgen.write_mm(mtx, A)
    write_vec(rhs, b)
    rc, out, err = run("-m", mtx, "-n", 32, "-d", 2, "-l", 5, "-t", 1e-2, "--rhs", rhs, "--res", 1e-10)
    assert rc == 0, err
    m = re.search(r"CGLS: #iterations: (\d+), residual \|A'\(Ax-b\)\|/\|A'\(b\)\|: ([0-9.eE+-]+)", out)
    assert m, out
    assert int(m.group(1)) <= 300 and float(m.group(2)) <= 1e-9
    assert np.isfinite(float(m.group(2)))


@pytest.mark.gpu
def test_cli_order15(gpu, tmp_path):
    w = matgen.workload("advdiff2d_64")
    mtx, rhs = tmp_path / "A.mtx", tmp_path / "b.mtx"
    matgen.write_mm(mtx, w["A"])
    write_vec(rhs, w["b"])
    its = {}
    for order in ("1", "1.5"):
        rc, out, err = run("-m", mtx, "-n", 64, "-d", 2, "-l", w["levels"], "-t", 1e-1, "--order", order,
                           "--rhs", rhs, "--res", 1e-12)
        assert rc == 0, err
        its[order] = _gmres_count(out)
    assert its["1.5"] < its["1"]
