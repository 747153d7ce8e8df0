// Geometric nested dissection ordering, bit-exact with the reference.
//
// Reference steps and where they live:
//   A^T A pattern, recursive geometric bisection     src/partition.cpp:241-304
//   separator sweep, top level first                  src/partition.cpp:306-332
//   leaves                                            src/partition.cpp:334-341
//   rows -> clusters (rectangular input)              src/partition.cpp:103-134, src/tree.cpp:57-98
//   interface (left/right) inference on A             src/partition.cpp:506-578
//   hierarchical column sort                          src/tree.cpp:46-55
//   row permutation (rectangular input)               src/tree.cpp:100-163
#include "symbolic.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>

namespace spq {

Csc csc_from(int m, int n, const int* cp, const int* ri, const double* va) {
    Csc A;
    A.m = m;
    A.n = n;
    A.p.assign(cp, cp + n + 1);
    size_t nnz = (size_t)cp[n];
    A.i.assign(ri, ri + nnz);
    A.v.assign(va, va + nnz);
    return A;
}

Csc csc_transpose(const Csc& A) {
    Csc T;
    T.m = A.n;
    T.n = A.m;
    T.p.assign((size_t)A.m + 1, 0);
    for (int r : A.i) ++T.p[(size_t)r + 1];
    std::partial_sum(T.p.begin(), T.p.end(), T.p.begin());
    T.i.resize(A.i.size());
    T.v.resize(A.v.size());
    std::vector<int> next(T.p.begin(), T.p.end() - 1);
    for (int j = 0; j < A.n; ++j)
        for (int q = A.p[j]; q < A.p[j + 1]; ++q) {
            int dst = next[A.i[q]]++;
            T.i[dst] = j;
            T.v[dst] = A.v[q];
        }
    return T;
}

Csc csc_gather_cols(const Csc& A, const std::vector<int>& perm) {
    Csc B;
    B.m = A.m;
    B.n = A.n;
    B.p.resize((size_t)A.n + 1);
    B.p[0] = 0;
    for (int k = 0; k < A.n; ++k) B.p[k + 1] = B.p[k] + (A.p[perm[k] + 1] - A.p[perm[k]]);
    B.i.resize(A.i.size());
    B.v.resize(A.v.size());
    for (int k = 0; k < A.n; ++k) {
        int s = A.p[perm[k]], len = A.p[perm[k] + 1] - s;
        std::copy_n(A.i.begin() + s, len, B.i.begin() + B.p[k]);
        std::copy_n(A.v.begin() + s, len, B.v.begin() + B.p[k]);
    }
    return B;
}

Csc csc_gather_rows(const Csc& A, const std::vector<int>& perm) {
    std::vector<int> inv(perm.size());
    for (size_t k = 0; k < perm.size(); ++k) inv[perm[k]] = (int)k;
    Csc B = A;
    std::vector<std::pair<int, double>> tmp;
    for (int j = 0; j < A.n; ++j) {
        tmp.clear();
        for (int q = A.p[j]; q < A.p[j + 1]; ++q) tmp.emplace_back(inv[A.i[q]], A.v[q]);
        std::sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t t = 0; t < tmp.size(); ++t) {
            B.i[A.p[j] + t] = tmp[t].first;
            B.v[A.p[j] + t] = tmp[t].second;
        }
    }
    return B;
}

Cid lift(const Cid& c, int lvl) {
    auto up = [lvl](const Sep& s) { return s.lvl < lvl ? Sep(s.lvl + 1, s.sep / 2) : s; };
    Cid o;
    o.self = c.self;
    o.l = up(c.l);
    o.r = up(c.r);
    o.section = lvl > 0 ? c.section / 2 : c.section;
    o.part = (c.self.lvl == lvl) ? 2 : c.part;
    return o;
}

namespace {

// Sides of a separator at tree level lvl >= 1: the leaf index shifted by lvl-1.
inline int side_at(int leaf, int lvl) { return lvl >= 1 ? (leaf >> (lvl - 1)) : leaf; }

Sep common_ancestor(Sep a, Sep b) {
    while (a.lvl < b.lvl) { a.lvl++; a.sep /= 2; }
    while (b.lvl < a.lvl) { b.lvl++; b.sep /= 2; }
    while (a.sep != b.sep) { a.lvl++; b.lvl++; a.sep /= 2; b.sep /= 2; }
    return a;
}

// Neighbour lists of A^T A (structural, ascending).
struct Adjacency {
    std::vector<int64_t> p;
    std::vector<int> i;
};

Adjacency ata_adjacency(const Csc& A, const Csc& At) {
    Adjacency G;
    G.p.assign((size_t)A.n + 1, 0);
    std::vector<int> stamp(A.n, -1), list;
    G.i.reserve(A.i.size() * 4);
    for (int j = 0; j < A.n; ++j) {
        list.clear();
        for (int q = A.p[j]; q < A.p[j + 1]; ++q) {
            int r = A.i[q];
            for (int t = At.p[r]; t < At.p[r + 1]; ++t) {
                int c = At.i[t];
                if (stamp[c] != j) { stamp[c] = j; list.push_back(c); }
            }
        }
        std::sort(list.begin(), list.end());
        G.i.insert(G.i.end(), list.begin(), list.end());
        G.p[j + 1] = (int64_t)G.i.size();
    }
    return G;
}

// Recursive geometric bisection: at each depth every part is split at the
// (N/2)-th smallest coordinate along its widest coordinate (ties: lowest dim).
std::vector<int> bisect(int n, int nlevels, int d, const std::vector<double>& X) {
    std::vector<int> part(n, 0);
    std::vector<double> vals;
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int nparts = 1 << depth;
        std::vector<std::vector<int>> members(nparts);
        for (int i = 0; i < n; ++i) members[part[i]].push_back(i);
        for (int k = 0; k < nparts; ++k) {
            const auto& mem = members[k];
            if (mem.empty()) continue;
            int best = -1;
            double widest = -1.0;
            for (int a = 0; a < d; ++a) {
                double lo = std::numeric_limits<double>::max(), hi = std::numeric_limits<double>::lowest();
                for (int i : mem) {
                    double x = X[(size_t)i * d + a];
                    lo = std::min(lo, x);
                    hi = std::max(hi, x);
                }
                if (hi - lo > widest) { widest = hi - lo; best = a; }
            }
            vals.resize(mem.size());
            for (size_t t = 0; t < mem.size(); ++t) vals[t] = X[(size_t)mem[t] * d + best];
            std::nth_element(vals.begin(), vals.begin() + mem.size() / 2, vals.end());
            const double cut = vals[mem.size() / 2];
            for (int i : mem) part[i] = (X[(size_t)i * d + best] <= cut) ? 2 * k : 2 * k + 1;
        }
    }
    return part;
}

// Rows -> cluster ids by the largest squared norm of a run of equal ids along
// the row (permuted column order); empty rows go to the last cluster.
void rows_by_norm(const Csc& At_perm, const std::vector<Cid>& cid_of_pos, std::vector<Cid>& rmap) {
    const Cid last = cid_of_pos.back();
    for (int r = 0; r < At_perm.n; ++r) {
        if (rmap[r] != Cid()) continue;
        double best = -1;
        Cid pick;
        int q = At_perm.p[r], e = At_perm.p[r + 1];
        while (q < e) {
            const Cid cur = cid_of_pos[At_perm.i[q]];
            double acc = At_perm.v[q] * At_perm.v[q];
            int t = q + 1;
            while (t < e && cid_of_pos[At_perm.i[t]] == cur) { acc += At_perm.v[t] * At_perm.v[t]; ++t; }
            if (acc > best) { best = acc; pick = cur; }
            q = t;
        }
        rmap[r] = (pick == Cid()) ? last : pick;
    }
}

}  // namespace

Ordering geometric_ordering(const Csc& A, int nlevels, int d, const std::vector<double>& X, bool square) {
    if (nlevels < 1) throw std::invalid_argument("nlevels must be >= 1");
    if ((int64_t)X.size() != (int64_t)d * A.n) throw std::invalid_argument("coordinates must be d x ncols");
    const int n = A.n, m = A.m;
    const Csc At = csc_transpose(A);
    const Adjacency G = ata_adjacency(A, At);
    const std::vector<int> part = bisect(n, nlevels, d, X);

    // Separators, top level first; a column on the even side of a cut that
    // touches an unassigned column on the odd side joins that separator. The
    // sweep is sequential in column order (assignments feed later tests).
    std::vector<Cid> cmap(n);
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int l = nlevels - depth - 1;
        for (int i = 0; i < n; ++i) {
            if (cmap[i].self.lvl != -1) continue;
            const int pi = side_at(part[i], l);
            if (pi & 1) continue;
            for (int64_t q = G.p[i]; q < G.p[i + 1]; ++q) {
                const int j = G.i[q];
                if (cmap[j].self.lvl == -1 && side_at(part[j], l) == pi + 1) {
                    cmap[i].self = Sep(l, pi / 2);
                    break;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i)
        if (cmap[i].self.lvl == -1) cmap[i].self = cmap[i].l = cmap[i].r = Sep(0, part[i]);

    // Rows inherit ids: identity for square input, max-norm run otherwise.
    std::vector<Cid> rmap(m);
    if (m == n) {
        rmap = cmap;
    } else {
        std::vector<int> perm(n);
        std::iota(perm.begin(), perm.end(), 0);
        std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return cmap[a] < cmap[b]; });
        std::vector<Cid> cid_of_pos(n);
        for (int k = 0; k < n; ++k) cid_of_pos[k] = cmap[perm[k]];
        rows_by_norm(csc_transpose(csc_gather_cols(A, perm)), cid_of_pos, rmap);
    }

    // Interface sides of separator rows from their lower-level neighbours
    // (lowest level wins, first seen wins on ties).
    for (int r = 0; r < m; ++r) {
        const Sep self = rmap[r].self;
        if (self.lvl <= 0) continue;
        Sep left, right;
        for (int q = At.p[r]; q < At.p[r + 1]; ++q) {
            const Sep nb = cmap[At.i[q]].self;
            if (nb.lvl >= self.lvl) continue;
            int pj = (int)(nb.sep / std::pow(2.0, self.lvl - nb.lvl - 1));
            Sep& side = (pj % 2 == 0) ? left : right;
            if (side.lvl == -1 || nb.lvl < side.lvl) side = nb;
        }
        rmap[r].l = left;
        rmap[r].r = right;
    }
    // Columns take the ids of the rows with the same index (identity matching);
    // a missing side is completed from same-separator neighbours.
    std::vector<Cid> cm2(rmap);
    for (int r = 0; r < m; ++r) {
        const Sep self = rmap[r].self;
        Sep left = rmap[r].l, right = rmap[r].r;
        if (right == Sep()) {
            for (int q = At.p[r]; q < At.p[r + 1]; ++q) {
                const Cid& c = cm2[At.i[q]];
                if (c.self == self && c.r != Sep()) right = (right == Sep()) ? c.r : common_ancestor(right, c.r);
            }
        } else if (left == Sep()) {
            for (int q = At.p[r]; q < At.p[r + 1]; ++q) {
                const Cid& c = cm2[At.i[q]];
                if (c.self == self && c.l != Sep()) left = (left == Sep()) ? c.l : common_ancestor(left, c.l);
            }
        }
        rmap[r].l = left;
        rmap[r].r = right;
    }
    for (int r = 0; r < m; ++r) {
        if (rmap[r].l == Sep()) rmap[r].l = rmap[r].self;
        if (rmap[r].r == Sep()) rmap[r].r = rmap[r].self;
    }
    // cmap = rmap (first n entries are the ones the column sort reads)

    // Hierarchical column sort: by id, then by the id lifted to each level.
    Ordering o;
    o.cperm.resize(n);
    std::iota(o.cperm.begin(), o.cperm.end(), 0);
    std::vector<Cid> key(rmap.begin(), rmap.begin() + n);
    auto by_key = [&key](int a, int b) { return key[a] < key[b]; };
    std::stable_sort(o.cperm.begin(), o.cperm.end(), by_key);
    for (int lvl = 1; lvl < nlevels; ++lvl) {
        for (auto& k : key) k = lift(k, lvl);
        std::stable_sort(o.cperm.begin(), o.cperm.end(), by_key);
    }
    o.cid_of_pos.resize(n);
    for (int k = 0; k < n; ++k) o.cid_of_pos[k] = rmap[o.cperm[k]];

    if (square) {
        if (m != n) throw std::invalid_argument("identity row matching needs a square matrix");
        o.rperm = o.cperm;
        o.rows_of_col.assign(n, 1);
    } else {
        // Each row goes to the first column (permuted order) of its max-norm run.
        const Csc Atp = csc_transpose(csc_gather_cols(A, o.cperm));
        o.rows_of_col.assign(n, 0);
        std::vector<std::vector<int>> owned(n);
        for (int r = 0; r < m; ++r) {
            double best = -1;
            int pick = -1;
            int q = Atp.p[r], e = Atp.p[r + 1];
            while (q < e) {
                const Cid cur = o.cid_of_pos[Atp.i[q]];
                double acc = Atp.v[q] * Atp.v[q];
                int t = q + 1;
                while (t < e && o.cid_of_pos[Atp.i[t]] == cur) { acc += Atp.v[t] * Atp.v[t]; ++t; }
                if (acc > best) { best = acc; pick = Atp.i[q]; }
                q = t;
            }
            if (pick < 0) pick = n - 1;
            o.rows_of_col[pick]++;
            owned[pick].push_back(r);
        }
        o.rperm.clear();
        o.rperm.reserve(m);
        for (int k = 0; k < n; ++k) o.rperm.insert(o.rperm.end(), owned[k].begin(), owned[k].end());
    }
    return o;
}

}  // namespace spq
