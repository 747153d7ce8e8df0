// Nested-dissection orderings: geometric (bit-exact with the reference) and,
// without coordinates, a graph bisection of A^T A whose part vector goes
// through the reference's MetisPartition steps.
//
// Reference steps and where they live:
//   A^T A pattern, recursive geometric bisection     src/partition.cpp:241-304
//   separator sweep, top level first                  src/partition.cpp:306-332
//   leaves                                            src/partition.cpp:334-341
//   rows -> clusters (rectangular input)              src/partition.cpp:103-134, src/tree.cpp:57-98
//   interface (left/right) inference on A             src/partition.cpp:506-578
//   hierarchical column sort                          src/tree.cpp:46-55
//   row permutation (rectangular input)               src/tree.cpp:100-163
//   separators from a part vector (no coordinates)    src/partition.cpp:374-426
//   interfaces on A^T A (no coordinates)              src/partition.cpp:628-675
#include "symbolic.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <set>
#include <stdexcept>
#include <thread>
#include <unordered_map>

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

// Column r of the result lists the columns j of A with A(r, j) != 0 in
// increasing j. On host threads for large matrices: each thread counts its
// column range's entries per row, a prefix over (row, thread) places every
// thread's entries of a row after those of the lower ranges, and each thread
// scatters its own range: the same arrays as one pass in column order.
Csc csc_transpose(const Csc& A) {
    Csc T;
    T.m = A.n;
    T.n = A.m;
    T.p.assign((size_t)A.m + 1, 0);
    T.i.resize(A.i.size());
    T.v.resize(A.v.size());
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = A.i.size() < (size_t)(1 << 18) ? 1 : std::max(1, std::min({hw, 8, A.n / 2048}));
    if (nt == 1) {
        for (int r : A.i) ++T.p[(size_t)r + 1];
        std::partial_sum(T.p.begin(), T.p.end(), T.p.begin());
        std::vector<int> next(T.p.begin(), T.p.end() - 1);
        for (int j = 0; j < A.n; ++j)
            for (int q = A.p[j]; q < A.p[j + 1]; ++q) {
                int dst = next[A.i[q]]++;
                T.i[dst] = j;
                T.v[dst] = A.v[q];
            }
        return T;
    }
    std::vector<std::vector<int>> cnt(nt, std::vector<int>(A.m, 0));
    auto range = [&](int t, int& lo, int& hi) {
        lo = (int)((int64_t)A.n * t / nt);
        hi = (int)((int64_t)A.n * (t + 1) / nt);
    };
    std::vector<std::thread> th;
    auto run = [&](auto&& fn) {
        th.clear();
        for (int t = 1; t < nt; ++t) th.emplace_back([&, t] { fn(t); });
        fn(0);
        for (auto& x : th) x.join();
    };
    run([&](int t) {
        int lo, hi;
        range(t, lo, hi);
        auto& c = cnt[t];
        for (int q = A.p[lo]; q < A.p[hi]; ++q) ++c[A.i[q]];
    });
    // row pointers, then each thread's first slot in every row
    for (int r = 0; r < A.m; ++r) {
        int64_t s = T.p[r];
        for (int t = 0; t < nt; ++t) {
            const int c = cnt[t][r];
            cnt[t][r] = (int)s;
            s += c;
        }
        T.p[(size_t)r + 1] = s;
    }
    run([&](int t) {
        int lo, hi;
        range(t, lo, hi);
        auto& next = cnt[t];
        for (int j = lo; j < hi; ++j)
            for (int q = A.p[j]; q < A.p[j + 1]; ++q) {
                int dst = next[A.i[q]]++;
                T.i[dst] = j;
                T.v[dst] = A.v[q];
            }
    });
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

// fn(t, begin, end) over [0, n) in contiguous ranges on up to 8 host threads,
// at least min_items items per thread (one call on this thread below that).
template <class F>
void par_ranges(int n, F&& fn, int min_items = 2048) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min({hw, 8, n / std::max(1, min_items)}));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t)
        th.emplace_back([&, t] { fn(t, (int)((int64_t)n * t / nt), (int)((int64_t)n * (t + 1) / nt)); });
    fn(0, 0, (int)((int64_t)n / nt));
    for (auto& x : th) x.join();
}

// Column adjacency of A^T A (sorted neighbour lists), built in column ranges
// on host threads and concatenated.
Adjacency ata_adjacency(const Csc& A, const Csc& At) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min({hw, 8, A.n / 2048}));
    std::vector<std::vector<int>> li(nt);
    std::vector<std::vector<int64_t>> lp(nt);
    std::vector<int> lo(nt + 1);
    par_ranges(A.n, [&](int t, int b, int e) {
        lo[t] = b;
        if (t == nt - 1) lo[nt] = e;
        std::vector<int> stamp(A.n, -1), list;
        auto& gi = li[t];
        auto& gp = lp[t];
        gi.reserve((size_t)(A.p[e] - A.p[b]) * 4);
        gp.reserve((size_t)(e - b));
        for (int j = b; j < e; ++j) {
            list.clear();
            for (int q = A.p[j]; q < A.p[j + 1]; ++q) {
                int r = A.i[q];
                for (int t2 = At.p[r]; t2 < At.p[r + 1]; ++t2) {
                    int c = At.i[t2];
                    if (stamp[c] != j) { stamp[c] = j; list.push_back(c); }
                }
            }
            std::sort(list.begin(), list.end());
            gi.insert(gi.end(), list.begin(), list.end());
            gp.push_back((int64_t)gi.size());
        }
    });
    Adjacency G;
    G.p.assign((size_t)A.n + 1, 0);
    size_t tot = 0;
    for (auto& v : li) tot += v.size();
    G.i.reserve(tot);
    for (int t = 0; t < nt; ++t) {
        const int64_t base = (int64_t)G.i.size();
        for (int j = lo[t]; j < lo[t + 1]; ++j) G.p[j + 1] = base + lp[t][j - lo[t]];
        G.i.insert(G.i.end(), li[t].begin(), li[t].end());
    }
    return G;
}

// Recursive geometric bisection: at each depth every part is split at the
// (N/2)-th smallest coordinate along its widest coordinate (ties: lowest dim).
// The members of every part are kept as one ascending range of `order`; a
// split is a stable partition of the range (ascending on both sides, as a
// scan of all indices would list them), and the parts of a depth are split on
// host threads.
std::vector<int> bisect(int n, int nlevels, int d, const std::vector<double>& X) {
    std::vector<int> part(n, 0), order(n), tmp(n);
    std::iota(order.begin(), order.end(), 0);
    std::vector<int> st{0, n};  // part k: order[st[k], st[k + 1])
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int nparts = 1 << depth;
        std::vector<int> mid(nparts);
        auto split = [&](int k, std::vector<double>& vals) {
            const int b = st[k], e = st[k + 1];
            mid[k] = b;
            if (b == e) return;
            int best = -1;
            double widest = -1.0;
            for (int a = 0; a < d; ++a) {
                double lo = std::numeric_limits<double>::max(), hi = std::numeric_limits<double>::lowest();
                for (int t = b; t < e; ++t) {
                    double x = X[(size_t)order[t] * d + a];
                    lo = std::min(lo, x);
                    hi = std::max(hi, x);
                }
                if (hi - lo > widest) { widest = hi - lo; best = a; }
            }
            const int cnt = e - b;
            vals.resize(cnt);
            for (int t = 0; t < cnt; ++t) vals[t] = X[(size_t)order[b + t] * d + best];
            std::nth_element(vals.begin(), vals.begin() + cnt / 2, vals.end());
            const double cut = vals[cnt / 2];
            int l = b, r = 0;
            for (int t = b; t < e; ++t) {
                const int i = order[t];
                if (X[(size_t)i * d + best] <= cut) {
                    part[i] = 2 * k;
                    order[l++] = i;
                } else {
                    part[i] = 2 * k + 1;
                    tmp[b + r++] = i;
                }
            }
            std::copy(tmp.begin() + b, tmp.begin() + b + r, order.begin() + l);
            mid[k] = l;
        };
        if (nparts < 8) {
            std::vector<double> vals;
            for (int k = 0; k < nparts; ++k) split(k, vals);
        } else {
            par_ranges(
                nparts,
                [&](int, int kb, int ke) {
                    std::vector<double> vals;
                    for (int k = kb; k < ke; ++k) split(k, vals);
                },
                1);
        }
        std::vector<int> nst(2 * nparts + 1);
        for (int k = 0; k < nparts; ++k) {
            nst[2 * k] = st[k];
            nst[2 * k + 1] = mid[k];
        }
        nst[2 * nparts] = n;
        st.swap(nst);
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

// Hierarchical column sort (initPermutation, src/tree.cpp:46-55) of the column
// ids, then the rows: identity for square input, else each row joins the first
// column of its largest-norm run of equal ids (form_rmap, src/tree.cpp:57-98).
Ordering finish_ordering(const Csc& A, int nlevels, const std::vector<Cid>& ids, bool square) {
    const int n = A.n, m = A.m;
    // Hierarchical column sort: stable by id, then stable by the id lifted to
    // each level in turn. Every key is a function of the id, so the columns of
    // one id keep their order and the ids' relative order is that of the same
    // sorts run on the distinct ids: those (a few per bottom cluster) are
    // sorted, and the columns follow by a stable counting sort on their id's
    // rank. Same permutation as the sorts over all columns.
    Ordering o;
    std::vector<int> slot(n);
    std::vector<Cid> uniq;
    {
        struct CidHash {
            size_t operator()(const Cid& c) const {
                uint64_t h = 1469598103934665603ull;
                for (int v : {c.self.lvl, c.self.sep, c.l.lvl, c.l.sep, c.r.lvl, c.r.sep, c.part, c.section})
                    h = (h ^ (uint32_t)v) * 1099511628211ull;
                return (size_t)h;
            }
        };
        std::unordered_map<Cid, int, CidHash> at;
        at.reserve(1024);
        for (int j = 0; j < n; ++j) {
            auto it = at.find(ids[j]);
            if (it == at.end()) {
                it = at.emplace(ids[j], (int)uniq.size()).first;
                uniq.push_back(ids[j]);
            }
            slot[j] = it->second;
        }
    }
    const int D = (int)uniq.size();
    std::vector<int> ord(D);
    std::iota(ord.begin(), ord.end(), 0);
    std::vector<Cid> key(uniq);
    auto by_key = [&key](int a, int b) { return key[a] < key[b]; };
    std::stable_sort(ord.begin(), ord.end(), by_key);
    for (int lvl = 1; lvl < nlevels; ++lvl) {
        for (auto& k : key) k = lift(k, lvl);
        std::stable_sort(ord.begin(), ord.end(), by_key);
    }
    std::vector<int> rank(D), start(D + 1, 0);
    for (int q = 0; q < D; ++q) rank[ord[q]] = q;
    for (int j = 0; j < n; ++j) ++start[rank[slot[j]] + 1];
    for (int q = 0; q < D; ++q) start[q + 1] += start[q];
    o.cperm.resize(n);
    for (int j = 0; j < n; ++j) o.cperm[start[rank[slot[j]]]++] = j;
    o.cid_of_pos.resize(n);
    for (int k = 0; k < n; ++k) o.cid_of_pos[k] = ids[o.cperm[k]];

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
    // A column can join the separator of level l only if some neighbour lies on
    // the odd sibling side at l (sides part >> (l - 1) differing in the last
    // bit only: the highest differing bit of the two parts is l - 1, and the
    // column's is 0); one pass marks those levels per column (bit l), and each
    // sweep visits only the marked columns, in column order as before.
    std::vector<std::vector<int>> cand(nlevels);
    {
        std::vector<uint32_t> mask(n, 0);
        for (int i = 0; i < n; ++i)
            for (int64_t q = G.p[i]; q < G.p[i + 1]; ++q) {
                const unsigned x = (unsigned)(part[i] ^ part[G.i[q]]);
                if (x == 0) continue;
                const int h = 31 - __builtin_clz(x);
                if (h + 1 < nlevels && !((part[i] >> h) & 1)) mask[i] |= 1u << (h + 1);
            }
        for (int i = 0; i < n; ++i)
            for (int l = 1; l < nlevels; ++l)
                if (mask[i] >> l & 1) cand[l].push_back(i);
    }
    std::vector<Cid> cmap(n);
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int l = nlevels - depth - 1;
        for (int i : cand[l]) {
            if (cmap[i].self.lvl != -1) continue;
            const int pi = side_at(part[i], l);
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
    // (threads: each row reads cmap and writes its own entry)
    par_ranges(m, [&](int, int rb, int re) {
        for (int r = rb; r < re; ++r) {
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
    });
    // Columns take the ids of the rows with the same index (identity matching);
    // a missing side is completed from same-separator neighbours (threads: each
    // row reads the copy cm2 and writes its own entry).
    std::vector<Cid> cm2(rmap);
    par_ranges(m, [&](int, int rb, int re) {
        for (int r = rb; r < re; ++r) {
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
    });
    for (int r = 0; r < m; ++r) {
        if (rmap[r].l == Sep()) rmap[r].l = rmap[r].self;
        if (rmap[r].r == Sep()) rmap[r].r = rmap[r].self;
    }
    // cmap = rmap (first n entries are the ones the column sort reads)

    return finish_ordering(A, nlevels, std::vector<Cid>(rmap.begin(), rmap.begin() + n), square);
}

// ---------------------------------------------------------------- graph ordering
namespace {

// One bisection of the vertex set `mem` (ascending) of the A^T A graph: a
// breadth-first level structure from a pseudo-peripheral vertex gives the
// first ceil(|mem|/2) vertices side 0, then Fiduccia-Mattheyses passes move
// boundary vertices to lower the edge cut while |side 0| stays within
// |mem|/200 + 1 of that size. Deterministic: every tie goes to the lowest index.
void bisect_graph(const Adjacency& G, const std::vector<int>& mem, std::vector<int>& loc, std::vector<char>& side) {
    const int N = (int)mem.size();
    side.assign(N, 0);
    if (N < 2) return;
    for (int t = 0; t < N; ++t) loc[mem[t]] = t;
    // local adjacency (members only, no self loops)
    std::vector<int> lp(N + 1, 0), li;
    li.reserve((size_t)N * 8);
    for (int t = 0; t < N; ++t) {
        const int v = mem[t];
        for (int64_t q = G.p[v]; q < G.p[v + 1]; ++q) {
            const int u = G.i[q];
            const int lu = loc[u];
            if (u != v && lu >= 0 && lu < N && mem[lu] == u) li.push_back(lu);
        }
        lp[t + 1] = (int)li.size();
    }
    // breadth-first search from r; returns the visit order, dist filled (-1 unvisited)
    std::vector<int> dist(N, -1), order;
    order.reserve(N);
    auto bfs = [&](int r) {
        order.clear();
        std::fill(dist.begin(), dist.end(), -1);
        dist[r] = 0;
        order.push_back(r);
        for (size_t h = 0; h < order.size(); ++h) {
            const int v = order[h];
            for (int q = lp[v]; q < lp[v + 1]; ++q)
                if (dist[li[q]] < 0) { dist[li[q]] = dist[v] + 1; order.push_back(li[q]); }
        }
    };
    // pseudo-peripheral start (George-Liu): move to a minimum-degree vertex of
    // the last level while the eccentricity grows
    int r = 0, ecc = -1;
    for (int it = 0; it < 16; ++it) {
        bfs(r);
        const int e = dist[order.back()];
        if (e <= ecc) break;
        ecc = e;
        int best = -1;
        for (int v : order)
            if (dist[v] == e && (best < 0 || lp[v + 1] - lp[v] < lp[best + 1] - lp[best] ||
                                 (lp[v + 1] - lp[v] == lp[best + 1] - lp[best] && v < best)))
                best = v;
        r = best;
    }
    bfs(r);
    for (int v = 0; (int)order.size() < N; ++v) {  // other components, in index order
        if (dist[v] >= 0) continue;
        size_t h = order.size();
        dist[v] = 0;
        order.push_back(v);
        for (; h < order.size(); ++h) {
            const int x = order[h];
            for (int q = lp[x]; q < lp[x + 1]; ++q)
                if (dist[li[q]] < 0) { dist[li[q]] = dist[x] + 1; order.push_back(li[q]); }
        }
    }
    const int target = (N + 1) / 2, slack = N / 200 + 1;
    for (int t = target; t < N; ++t) side[order[t]] = 1;
    int w0 = target;

    // Fiduccia-Mattheyses refinement of the edge cut
    std::vector<int> gain(N);
    auto compute_gain = [&](int v) {
        int g = 0;
        for (int q = lp[v]; q < lp[v + 1]; ++q) g += side[li[q]] != side[v] ? 1 : -1;
        return g;
    };
    std::vector<char> locked(N), queued(N);
    std::vector<int> moves;
    for (int pass = 0; pass < 6; ++pass) {
        for (int v = 0; v < N; ++v) gain[v] = compute_gain(v);
        std::set<std::pair<int, int>> pq[2];  // (-gain, v) per side
        std::fill(locked.begin(), locked.end(), 0);
        std::fill(queued.begin(), queued.end(), 0);
        for (int v = 0; v < N; ++v) {
            bool boundary = false;
            for (int q = lp[v]; q < lp[v + 1] && !boundary; ++q) boundary = side[li[q]] != side[v];
            if (boundary) { pq[(int)side[v]].insert({-gain[v], v}); queued[v] = 1; }
        }
        moves.clear();
        int cum = 0, best = 0, best_len = 0, best_imb = std::abs(w0 - target), idle = 0;
        const int max_idle = std::max(64, N / 50);
        while (idle < max_idle) {
            int pick = -1;
            for (int sd = 0; sd < 2; ++sd) {
                if (pq[sd].empty()) continue;
                const int w_after = w0 + (sd == 0 ? -1 : 1);
                if (std::abs(w_after - target) > slack) continue;
                const auto& top = *pq[sd].begin();
                if (pick < 0 || top.first < -gain[pick] || (top.first == -gain[pick] && top.second < pick))
                    pick = top.second;
            }
            if (pick < 0) break;
            const int sd = side[pick];
            pq[sd].erase({-gain[pick], pick});
            queued[pick] = 0;
            locked[pick] = 1;
            cum += gain[pick];
            side[pick] = (char)(1 - sd);
            w0 += sd == 0 ? -1 : 1;
            gain[pick] = -gain[pick];
            moves.push_back(pick);
            for (int q = lp[pick]; q < lp[pick + 1]; ++q) {
                const int u = li[q];
                if (locked[u]) continue;
                if (queued[u]) pq[(int)side[u]].erase({-gain[u], u});
                gain[u] += side[u] == side[pick] ? -2 : 2;
                pq[(int)side[u]].insert({-gain[u], u});
                queued[u] = 1;
            }
            const int imb = std::abs(w0 - target);
            if (cum > best || (cum == best && imb < best_imb)) {
                best = cum;
                best_len = (int)moves.size();
                best_imb = imb;
                idle = 0;
            } else {
                ++idle;
            }
        }
        for (int t = (int)moves.size() - 1; t >= best_len; --t) {  // undo past the best prefix
            const int v = moves[t];
            w0 += side[v] == 0 ? -1 : 1;
            side[v] = (char)(1 - side[v]);
        }
        if (best <= 0) break;
    }
    for (int t = 0; t < N; ++t) loc[mem[t]] = -1;
}

}  // namespace

std::vector<int> graph_bisection(const Csc& A, int nlevels) {
    if (nlevels < 1) throw std::invalid_argument("nlevels must be >= 1");
    const int n = A.n;
    const Adjacency G = ata_adjacency(A, csc_transpose(A));
    std::vector<int> part(n, 0), next(n, 0), loc(n, -1);
    std::vector<char> side;
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int nparts = 1 << depth;
        std::vector<std::vector<int>> members(nparts);
        for (int i = 0; i < n; ++i) members[part[i]].push_back(i);
        for (int k = 0; k < nparts; ++k) {
            bisect_graph(G, members[k], loc, side);
            for (size_t t = 0; t < members[k].size(); ++t) next[members[k][t]] = 2 * k + side[t];
        }
        part.swap(next);
    }
    return part;
}

Ordering graph_ordering(const Csc& A, int nlevels, const std::vector<int>& parts, bool square) {
    if (nlevels < 1) throw std::invalid_argument("nlevels must be >= 1");
    const int n = A.n;
    if ((int)parts.size() != n) throw std::invalid_argument("parts must have one entry per column");
    const int nleaves = nlevels >= 2 ? 1 << (nlevels - 1) : 1;
    for (int p : parts)
        if (p < 0 || p >= nleaves) throw std::invalid_argument("part index out of range for nlevels");
    const Adjacency G = ata_adjacency(A, csc_transpose(A));

    // Separators, top level first (src/partition.cpp:384-414): a column on the
    // even side of a cut with an unassigned neighbour on the odd side joins it.
    std::vector<Cid> cmap(n);
    for (int depth = 0; depth + 1 < nlevels; ++depth) {
        const int l = nlevels - depth - 1;
        for (int i = 0; i < n; ++i) {
            if (cmap[i].self.lvl != -1) continue;
            const int pi = side_at(parts[i], l);
            if (pi & 1) continue;
            for (int64_t q = G.p[i]; q < G.p[i + 1]; ++q) {
                const int j = G.i[q];
                if (cmap[j].self.lvl == -1 && side_at(parts[j], l) == pi + 1) {
                    cmap[i].self = Sep(l, pi / 2);
                    break;
                }
            }
        }
    }
    // Leaves (src/partition.cpp:416-423), then the two sides of every separator
    // column from its lower-level neighbours: the left side starts at the
    // column's own leaf, both sides climb to the highest common ancestor
    // (getInterfacesUsingATA, src/partition.cpp:628-675). Every column's
    // section is its leaf part.
    for (int i = 0; i < n; ++i)
        if (cmap[i].self.lvl == -1) cmap[i].self = cmap[i].l = cmap[i].r = Sep(0, parts[i]);
    for (int i = 0; i < n; ++i) {
        const Sep self = cmap[i].self;
        cmap[i].section = parts[i];
        if (self.lvl <= 0) continue;
        Sep left(0, parts[i]), right;
        const int pi = side_at(parts[i], self.lvl);
        for (int64_t q = G.p[i]; q < G.p[i + 1]; ++q) {
            const int j = G.i[q];
            const Sep nb = cmap[j].self;
            if (nb.lvl >= self.lvl) continue;
            if (side_at(parts[j], self.lvl) <= pi) left = common_ancestor(nb, left);
            else right = (right.lvl == -1) ? nb : common_ancestor(nb, right);
        }
        if (right.lvl == -1) throw std::logic_error("graph ordering: separator column without a right side");
        cmap[i].l = left;
        cmap[i].r = right;
    }
    return finish_ordering(A, nlevels, cmap, square);
}

}  // namespace spq
