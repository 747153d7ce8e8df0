"""The header-only C++ facade (include/spaqr_tree.hpp) compiles against the C
ABI, links the library and drives the host steps a C++ caller of the
reference would: Tree construction and setters, partition of a 2D Laplacian
in compressed-column form, and the error path of a solve before factorize
(no GPU needed)."""
import os
import subprocess
import tempfile

from spaqr_public_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cstdio>
#include <vector>
#include "spaqr_tree.hpp"

int main() {
    const int n = 16, N = n * n;
    std::vector<int> cp(1, 0), ri;
    std::vector<double> va;
    for (int j = 0; j < N; ++j) {  // 5-point Laplacian, lexicographic unknowns
        const int x = j / n, y = j % n;
        const int nb[5] = {j - n, j - 1, j, j + 1, j + n};
        const bool ok[5] = {x > 0, y > 0, true, y < n - 1, x < n - 1};
        for (int q = 0; q < 5; ++q)
            if (ok[q]) { ri.push_back(nb[q]); va.push_back(q == 2 ? 4.0 : -1.0); }
        cp.push_back((int)ri.size());
    }
    spq::CscView A{N, N, cp.data(), ri.data(), va.data()};
    spq::Tree t(4, 0);
    t.set_tol(1e-2);
    t.set_scale(1);
    t.set_square(1);
    t.set_grid(n, 2);
    t.partition(A);
    std::vector<double> b(N, 1.0), x;
    try {
        t.solve(b, x);
        std::printf("no error\n");
        return 1;
    } catch (const spq::Error& e) {
        std::printf("code %d\n", e.code);
    }
    return 0;
}
"""


def test_cpp_facade_compiles_links_and_partitions():
    libdir = os.path.dirname(_abi.LIB_PATH)
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "facade.cpp")
        exe = os.path.join(d, "facade")
        open(src, "w").write(SRC)
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
                        "-L", libdir, "-lspaqr_b200", "-Wl,-rpath," + libdir], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "code 2" in out.stdout  # SPQ_ERR_STATE: solve before factorize
