// MatrixMarket input for the command-line driver, with the reader semantics of
// the reference (include/mmio.hpp:175-320):
//   * sparse: "matrix coordinate {real|integer|pattern} {general|symmetric|
//     skew-symmetric|hermitian}"; pattern entries are 1; a symmetric entry
//     off the diagonal also lands at its mirror (negated when skew-symmetric);
//     duplicate entries are summed (Eigen's setFromTriplets); the result is CSC
//     with strictly increasing row indices per column;
//   * dense: "matrix array real general", column-major (a vector is n x 1).
#pragma once

#include <algorithm>
#include <cctype>
#include <fstream>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace spq {
namespace mm {

struct Csc {
    int m = 0, n = 0;
    std::vector<int> colptr, rowind;
    std::vector<double> val;
};

inline std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Header line tokens after "%%MatrixMarket": object, format, field, symmetry.
inline std::vector<std::string> header(std::ifstream& f) {
    std::string line;
    if (!std::getline(f, line)) throw std::runtime_error("empty file");
    std::istringstream h(line);
    std::string tag;
    std::vector<std::string> tok;
    h >> tag;
    if (tag != "%%MatrixMarket") throw std::runtime_error("missing %%MatrixMarket header");
    for (std::string t; h >> t;) tok.push_back(lower(t));
    if (tok.size() < 4 || tok[0] != "matrix") throw std::runtime_error("unsupported MatrixMarket header");
    return tok;
}

// Next line that is neither empty nor a comment.
inline bool data_line(std::ifstream& f, std::string& line) {
    while (std::getline(f, line)) {
        size_t p = line.find_first_not_of(" \t\r");
        if (p == std::string::npos || line[p] == '%') continue;
        return true;
    }
    return false;
}

inline Csc from_triplets(int m, int n, std::vector<int>& r, std::vector<int>& c, std::vector<double>& v) {
    std::vector<size_t> ord(r.size());
    std::iota(ord.begin(), ord.end(), size_t(0));
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return c[a] != c[b] ? c[a] < c[b] : r[a] < r[b]; });
    Csc A;
    A.m = m;
    A.n = n;
    A.colptr.assign(n + 1, 0);
    for (size_t k = 0; k < ord.size(); ++k) {
        const size_t e = ord[k];
        if (!A.rowind.empty() && k > 0 && c[ord[k - 1]] == c[e] && r[ord[k - 1]] == r[e]) {
            A.val.back() += v[e];  // duplicate: summed
            continue;
        }
        A.rowind.push_back(r[e]);
        A.val.push_back(v[e]);
        A.colptr[c[e] + 1] += 1;
    }
    for (int j = 0; j < n; ++j) A.colptr[j + 1] += A.colptr[j];
    return A;
}

inline Csc read_sparse(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw std::runtime_error("cannot open file");
    const std::vector<std::string> h = header(f);
    if (h[1] != "coordinate") throw std::runtime_error("a sparse matrix must be in coordinate format");
    const std::string field = h[2], sym = h[3];
    if (field != "real" && field != "integer" && field != "pattern" && field != "double")
        throw std::runtime_error("unsupported field " + field);
    if (sym != "general" && sym != "symmetric" && sym != "skew-symmetric" && sym != "hermitian")
        throw std::runtime_error("unsupported symmetry " + sym);
    std::string line;
    if (!data_line(f, line)) throw std::runtime_error("missing size line");
    long long M = 0, N = 0, K = 0;
    {
        std::istringstream s(line);
        if (!(s >> M >> N >> K) || M < 0 || N < 0 || K < 0 || M > 2000000000LL || N > 2000000000LL)
            throw std::runtime_error("bad size line");
    }
    std::vector<int> r, c;
    std::vector<double> v;
    r.reserve(sym == "general" ? K : 2 * K);
    long long read = 0;
    while (data_line(f, line)) {
        std::istringstream s(line);
        long long i = 0, j = 0;
        double x = 1.0;
        if (!(s >> i >> j)) throw std::runtime_error("bad entry line");
        if (field != "pattern" && !(s >> x)) throw std::runtime_error("bad entry value");
        if (i < 1 || i > M || j < 1 || j > N) throw std::runtime_error("entry index out of range");
        r.push_back((int)(i - 1));
        c.push_back((int)(j - 1));
        v.push_back(x);
        if (sym != "general") {
            if (i < j) throw std::runtime_error("symmetric storage holds the lower triangle only");
            if (sym == "skew-symmetric" && i == j) throw std::runtime_error("skew-symmetric diagonal entry");
            if (i != j) {
                r.push_back((int)(j - 1));
                c.push_back((int)(i - 1));
                v.push_back(sym == "skew-symmetric" ? -x : x);
            }
        }
        ++read;
    }
    if (read != K) throw std::runtime_error("entry count does not match the size line");
    return from_triplets((int)M, (int)N, r, c, v);
}

// Dense array, column-major; rows and cols returned.
inline std::vector<double> read_dense(const std::string& path, int& rows, int& cols) {
    std::ifstream f(path);
    if (!f.is_open()) throw std::runtime_error("cannot open file");
    const std::vector<std::string> h = header(f);
    if (h[1] != "array" || h[3] != "general" || h[2] == "pattern")
        throw std::runtime_error("a dense matrix must be 'array <real> general'");
    std::string line;
    if (!data_line(f, line)) throw std::runtime_error("missing size line");
    long long M = 0, N = 0;
    {
        std::istringstream s(line);
        if (!(s >> M >> N) || M < 0 || N < 0 || M * N > 4000000000LL) throw std::runtime_error("bad size line");
    }
    std::vector<double> a;
    a.reserve((size_t)(M * N));
    while (data_line(f, line)) {
        std::istringstream s(line);
        double x;
        if (!(s >> x)) throw std::runtime_error("bad value line");
        a.push_back(x);
    }
    if ((long long)a.size() != M * N) throw std::runtime_error("value count does not match the size line");
    rows = (int)M;
    cols = (int)N;
    return a;
}

inline Csc transpose(const Csc& A) {
    std::vector<int> r, c;
    std::vector<double> v;
    for (int j = 0; j < A.n; ++j)
        for (int q = A.colptr[j]; q < A.colptr[j + 1]; ++q) {
            r.push_back(j);
            c.push_back(A.rowind[q]);
            v.push_back(A.val[q]);
        }
    return from_triplets(A.n, A.m, r, c, v);
}

}  // namespace mm
}  // namespace spq
