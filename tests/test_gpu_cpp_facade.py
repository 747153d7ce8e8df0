"""The header-only C++ facade (include/spaqr_tree.hpp) on the GPU: a C++ caller
written against the reference's names (Tree::partition / assemble / factorize /
solve and gmres, include/tree.h:139-147, include/is.h:14-15) factors and
solves the same seeded system as the Python path, with the same event-log
size, the same one-shot solve (bitwise: same library, same inputs) and the same
GMRES iteration count and solution."""
import os
import subprocess

import numpy as np
import pytest

from spaqr_public_b200 import Tree, _abi, gmres, matgen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "spaqr_tree.hpp"

static std::vector<char> slurp(const char* path) {
    std::vector<char> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    char buf[1 << 16];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + k);
    std::fclose(f);
    return v;
}
template <class T>
static std::vector<T> as(const std::vector<char>& v) {
    std::vector<T> out(v.size() / sizeof(T));
    std::copy(v.data(), v.data() + out.size() * sizeof(T), reinterpret_cast<char*>(out.data()));
    return out;
}

int main(int argc, char** argv) {
    // argv: dir n levels tol
    const std::string dir = argv[1];
    const int n = std::atoi(argv[2]), levels = std::atoi(argv[3]);
    const double tol = std::atof(argv[4]);
    auto cp = as<int>(slurp((dir + "/cp.bin").c_str()));
    auto ri = as<int>(slurp((dir + "/ri.bin").c_str()));
    auto va = as<double>(slurp((dir + "/va.bin").c_str()));
    auto b = as<double>(slurp((dir + "/b.bin").c_str()));
    const int N = (int)cp.size() - 1;
    spq::CscView A{N, N, cp.data(), ri.data(), va.data()};
    spq::Tree t(levels, 0);
    t.set_tol(tol);
    t.set_scale(1);
    t.set_square(1);
    t.set_grid(n, 2);
    t.partition(A);
    t.assemble(A);
    t.factorize();
    std::vector<double> x;
    t.solve(b, x);
    std::vector<double> xg;
    double res = 1e-12;
    const int its = spq::gmres(A, b, xg, t, 100, 100, res);
    FILE* f = std::fopen((dir + "/x.bin").c_str(), "wb");
    std::fwrite(x.data(), sizeof(double), x.size(), f);
    std::fclose(f);
    f = std::fopen((dir + "/xg.bin").c_str(), "wb");
    std::fwrite(xg.data(), sizeof(double), xg.size(), f);
    std::fclose(f);
    std::printf("its %d res %.6e\n", its, res);
    return 0;
}
"""


def test_cpp_facade_factorize_solve_gmres_match_python(gpu, tmp_path):
    w = matgen.workload("advdiff2d_32")
    A = matgen.column_normalize(w["A"])
    m, n, cp, ri, va = A
    b = np.asarray(w["b"], dtype=np.float64)
    for name, arr, dt in (("cp", cp, np.int32), ("ri", ri, np.int32), ("va", va, np.float64), ("b", b, np.float64)):
        np.ascontiguousarray(arr, dtype=dt).tofile(tmp_path / f"{name}.bin")
    libdir = os.path.dirname(_abi.LIB_PATH)
    src, exe = tmp_path / "facade.cpp", tmp_path / "facade"
    src.write_text(SRC)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lspaqr_b200", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe), str(tmp_path), str(w["n"]), str(w["levels"]), str(w["tol"])],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    its_cpp = int(out.stdout.split()[1])
    x_cpp = np.fromfile(tmp_path / "x.bin", dtype=np.float64)
    xg_cpp = np.fromfile(tmp_path / "xg.bin", dtype=np.float64)
    # the Python path on the same inputs
    t = Tree(w["levels"], 0)
    t.set_tol(w["tol"])
    t.set_scale(1)
    t.set_square(1)
    t.set_coords_grid(w["n"], w["d"])
    t.partition(A)
    t.assemble(A)
    t.factorize()
    x = t.solve(b)
    xg, its, res = gmres(A, b, t, iters=100, tol=1e-12)
    assert np.array_equal(x_cpp, x)
    assert its_cpp == its
    assert np.linalg.norm(xg_cpp - xg) <= 1e-12 * np.linalg.norm(xg)
    assert np.linalg.norm(matgen.spmv(A, xg_cpp) - b) <= 1e-11 * np.linalg.norm(b)
