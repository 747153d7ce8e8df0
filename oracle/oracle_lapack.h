// LAPACKE / CBLAS entry points resolved at run time from an OpenBLAS shared
// library. TEST INFRASTRUCTURE ONLY (the oracle's numerical kernels are the
// same LAPACK routines the reference calls in src/util.cpp:233-816).
#pragma once
#include <string>

namespace orc {

enum { kColMajor = 102, kNoTrans = 111, kTrans = 112, kUpper = 121, kLower = 122,
       kNonUnit = 131, kUnit = 132, kLeft = 141, kRight = 142 };

struct Lapack {
    int (*dgeqrf)(int, int, int, double*, int, double*) = nullptr;
    int (*dlarft)(int, char, char, int, int, const double*, int, const double*, double*, int) = nullptr;
    int (*dlarfb)(int, char, char, char, char, int, int, int, const double*, int, const double*, int,
                  double*, int) = nullptr;
    int (*dgeqp3)(int, int, int, double*, int, int*, double*) = nullptr;
    int (*dormqr)(int, char, char, int, int, int, const double*, int, const double*, double*, int) = nullptr;
    int (*dgesvd)(int, char, char, int, int, double*, int, double*, double*, int, double*, int,
                  double*) = nullptr;
    void (*dtrsm)(int, int, int, int, int, int, int, double, const double*, int, double*, int) = nullptr;
    void (*dtrsv)(int, int, int, int, int, const double*, int, double*, int) = nullptr;
    void (*set_threads)(int) = nullptr;
    int (*get_threads)() = nullptr;
    std::string path;
};

// Loads the library once (path from $SPQ_ORACLE_BLAS, else the image's
// OpenBLAS 0.3.15). Returns nullptr and fills *err on failure.
const Lapack* lapack(std::string* err = nullptr);

}  // namespace orc
