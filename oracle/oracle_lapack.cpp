// TEST INFRASTRUCTURE ONLY: run-time binding of the LAPACKE/CBLAS symbols used by
// the oracle. The reference links LAPACKE/CBLAS from OpenBLAS at build time
// (Makefile:31-36); this image ships OpenBLAS 0.3.15 only inside a Python wheel,
// so the oracle opens it with dlopen.
#include "oracle_lapack.h"

#include <dlfcn.h>
#include <glob.h>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace orc {

static Lapack g_lapack;
static bool g_ok = false;
static std::string g_err;
static std::once_flag g_once;

static std::vector<std::string> candidates() {
    std::vector<std::string> out;
    if (const char* e = std::getenv("SPQ_ORACLE_BLAS")) out.push_back(e);
    const char* pats[] = {
        "/opt/prime-rl/.venv/lib/python3*/site-packages/opencv_python_headless.libs/libopenblas*.so*",
        "/usr/lib/x86_64-linux-gnu/libopenblas*.so*",
        "/usr/lib/x86_64-linux-gnu/openblas*/liblapack.so*",
    };
    for (const char* p : pats) {
        glob_t g;
        if (glob(p, 0, nullptr, &g) == 0) {
            for (size_t i = 0; i < g.gl_pathc; ++i) out.push_back(g.gl_pathv[i]);
        }
        globfree(&g);
    }
    return out;
}

template <class F>
static bool bind(void* h, const char* name, F& fn) {
    fn = reinterpret_cast<F>(dlsym(h, name));
    return fn != nullptr;
}

// Wheel-bundled OpenBLAS finds its Fortran runtime next to itself only through
// the wheel's loader path, so the runtime libraries in the same folder are opened
// first (RTLD_GLOBAL) to satisfy the dependency.
static void preload_siblings(const std::string& p) {
    std::string dir = p.substr(0, p.find_last_of('/') + 1);
    for (const char* pat : {"libquadmath*.so*", "libgfortran*.so*"}) {
        glob_t g;
        if (glob((dir + pat).c_str(), 0, nullptr, &g) == 0)
            for (size_t i = 0; i < g.gl_pathc; ++i) dlopen(g.gl_pathv[i], RTLD_NOW | RTLD_GLOBAL);
        globfree(&g);
    }
}

static void load() {
    for (const auto& p : candidates()) {
        void* h = dlopen(p.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            preload_siblings(p);
            h = dlopen(p.c_str(), RTLD_NOW | RTLD_LOCAL);
        }
        if (!h) continue;
        Lapack L;
        bool ok = bind(h, "LAPACKE_dgeqrf", L.dgeqrf) && bind(h, "LAPACKE_dlarft", L.dlarft) &&
                  bind(h, "LAPACKE_dlarfb", L.dlarfb) && bind(h, "LAPACKE_dgeqp3", L.dgeqp3) &&
                  bind(h, "LAPACKE_dormqr", L.dormqr) && bind(h, "LAPACKE_dgesvd", L.dgesvd) &&
                  bind(h, "cblas_dtrsm", L.dtrsm) && bind(h, "cblas_dtrsv", L.dtrsv);
        if (!ok) { dlclose(h); continue; }
        bind(h, "openblas_set_num_threads", L.set_threads);
        bind(h, "openblas_get_num_threads", L.get_threads);
        L.path = p;
        g_lapack = L;
        g_ok = true;
        return;
    }
    g_err = "no OpenBLAS/LAPACKE shared library found (set SPQ_ORACLE_BLAS)";
}

const Lapack* lapack(std::string* err) {
    std::call_once(g_once, load);
    if (!g_ok) {
        if (err) *err = g_err;
        return nullptr;
    }
    return &g_lapack;
}

}  // namespace orc
