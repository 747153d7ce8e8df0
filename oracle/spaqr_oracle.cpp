// CPU oracle for spaQR. TEST INFRASTRUCTURE ONLY.
//
// A restatement, in plain C++ on std containers, of the reference algorithm of
// Abeynaya/spaQR_public. Every function cites the reference file:line it
// follows. Dense arithmetic goes through the same LAPACK/CBLAS routines the
// reference calls (src/util.cpp:233-816), resolved from OpenBLAS at run time.
//
// PARITY UNPINNED: the reference cannot be compiled in this image (Eigen, PaToH
// and METIS are absent), and it ships no tests or golden vectors; the README
// transcript (README.md:48-84) uses a matrix that is not distributed. Where the
// reference iterates a std::set<Cluster*> (pointer order, i.e. heap addresses)
// this restatement iterates in cluster creation order instead.
//
// Event log: records of 8 long longs [type, ilvl, order, a, b, c, d, e]
//   1 ELIM   a=stacked rows b=cols c=#updated column clusters d=#stacked blocks
//            e=total width of the updated columns
//   2 SCALE  a=rows b=cols c=#row blocks (larfb) d=#column blocks (trsm)
//            e=100000 * (width of the row blocks) + (height of the column blocks)
//   3 SPARS  a=cols before b=cols after c=width of C d=rows after
//   4 MERGE  a=rows b=cols c=#children
//   5 LEVEL  a=top-separator rows b=top-separator cols c=#clusters in the next bottom
//   6 FINAL  a=nnzA b=nnzR c=nnzH d=nnzQ
//   7 SHIFT  a=extra rows moved (rectangular reassign_rows)
//   8 EXTRA  a=rows before b=rows after (rectangular sparsify_extra)
#include "spaqr_oracle.h"
#include "oracle_lapack.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstring>
#include <limits>
#include <list>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

static thread_local std::string g_last_error;

static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static const Lapack& L() {
    std::string err;
    const Lapack* l = lapack(&err);
    if (!l) throw std::runtime_error(err);
    return *l;
}

// ---------------------------------------------------------------------------
// Sparse matrices (Eigen::SparseMatrix<double, ColMajor, int> semantics: sorted
// inner indices, structural entries kept).
// ---------------------------------------------------------------------------
struct Csc {
    int m = 0, n = 0;
    std::vector<int> p, i;
    std::vector<double> v;
};

static Csc make_csc(int m, int n, const int* cp, const int* ri, const double* va) {
    Csc A;
    A.m = m;
    A.n = n;
    A.p.assign(cp, cp + n + 1);
    A.i.assign(ri, ri + cp[n]);
    A.v.assign(va, va + cp[n]);
    return A;
}

static Csc transpose(const Csc& A) {
    Csc T;
    T.m = A.n;
    T.n = A.m;
    T.p.assign(A.m + 1, 0);
    for (int k : A.i) T.p[k + 1]++;
    for (int r = 0; r < A.m; ++r) T.p[r + 1] += T.p[r];
    T.i.resize(A.i.size());
    T.v.resize(A.v.size());
    std::vector<int> pos(T.p.begin(), T.p.end() - 1);
    for (int j = 0; j < A.n; ++j)
        for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
            int q = pos[A.i[k]]++;
            T.i[q] = j;
            T.v[q] = A.v[k];
        }
    return T;
}

// col_perm (src/util.cpp:912-940): column j of A moves to position pinv[j].
static Csc col_perm(const Csc& A, const std::vector<int>& p) {
    Csc B;
    B.m = A.m;
    B.n = A.n;
    B.p.assign(A.n + 1, 0);
    for (int k = 0; k < A.n; ++k) B.p[k + 1] = B.p[k] + (A.p[p[k] + 1] - A.p[p[k]]);
    B.i.resize(A.i.size());
    B.v.resize(A.v.size());
    for (int k = 0; k < A.n; ++k) {
        int s = A.p[p[k]], e = A.p[p[k] + 1];
        std::copy(A.i.begin() + s, A.i.begin() + e, B.i.begin() + B.p[k]);
        std::copy(A.v.begin() + s, A.v.begin() + e, B.v.begin() + B.p[k]);
    }
    return B;
}

// Structural pattern of A^T A with sorted inner indices
// (SpMat AtA = A.transpose()*A, src/partition.cpp:283).
static Csc ata_pattern(const Csc& A) {
    Csc At = transpose(A);  // column r of At = row r of A
    Csc P;
    P.m = P.n = A.n;
    P.p.assign(A.n + 1, 0);
    std::vector<int> mark(A.n, -1), buf;
    for (int j = 0; j < A.n; ++j) {
        buf.clear();
        for (int k = A.p[j]; k < A.p[j + 1]; ++k) {
            int r = A.i[k];
            for (int q = At.p[r]; q < At.p[r + 1]; ++q) {
                int c = At.i[q];
                if (mark[c] != j) {
                    mark[c] = j;
                    buf.push_back(c);
                }
            }
        }
        std::sort(buf.begin(), buf.end());
        P.i.insert(P.i.end(), buf.begin(), buf.end());
        P.p[j + 1] = (int)P.i.size();
    }
    P.v.assign(P.i.size(), 1.0);
    return P;
}

// ---------------------------------------------------------------------------
// SepID / ClusterID (include/cluster.h:22-111, src/cluster.cpp:19-32)
// ---------------------------------------------------------------------------
struct SepID {
    int lvl = -1, sep = 0;
    SepID() = default;
    SepID(int l, int s) : lvl(l), sep(s) {}
    bool operator==(const SepID& o) const { return lvl == o.lvl && sep == o.sep; }
    bool operator!=(const SepID& o) const { return !(*this == o); }
    bool operator<(const SepID& o) const { return lvl < o.lvl || (lvl == o.lvl && sep < o.sep); }
};

struct ClusterID {
    SepID self, l, r;
    int part = 2, section = 0;
    bool operator==(const ClusterID& o) const {
        return self == o.self && l == o.l && r == o.r && part == o.part && section == o.section;
    }
    bool operator!=(const ClusterID& o) const { return !(*this == o); }
    bool operator<(const ClusterID& o) const {
        if (self != o.self) return self < o.self;
        if (l != o.l) return l < o.l;
        if (r != o.r) return r < o.r;
        if (section != o.section) return section < o.section;
        return part < o.part;
    }
};

static SepID merge_sep(const SepID& s) { return SepID(s.lvl + 1, s.sep / 2); }

static ClusterID merge_if(const ClusterID& c, int lvl) {
    ClusterID o;
    o.self = c.self;
    o.l = c.l.lvl < lvl ? merge_sep(c.l) : c.l;
    o.r = c.r.lvl < lvl ? merge_sep(c.r) : c.r;
    o.section = lvl > 0 ? c.section / 2 : c.section;
    o.part = c.self.lvl == lvl ? 2 : c.part;
    return o;
}

// ---------------------------------------------------------------------------
// Geometric partition (src/partition.cpp:54-157, 241-348, 506-578)
// ---------------------------------------------------------------------------
static int part_at_lvl(int part_leaf, int lvl) {
    for (int l = 0; l < lvl - 1; ++l) part_leaf /= 2;
    return part_leaf;
}

static SepID find_highest_common(SepID n1, SepID n2) {
    int l1 = n1.lvl, l2 = n2.lvl, s1 = n1.sep, s2 = n2.sep;
    while (l1 < l2) { l1++; s1 /= 2; }
    while (l2 < l1) { l2++; s2 /= 2; }
    while (s1 != s2) { l1++; l2++; s1 /= 2; s2 /= 2; }
    return SepID(l1, s1);
}

static SepID find_lowest_common(SepID n1, SepID n2) { return n1.lvl < n2.lvl ? n1 : n2; }

// X is d x N column-major.
static void bissect_geo(const std::vector<int>& dofs, std::vector<int>& parts, const std::vector<double>& X,
                        int d, int start) {
    int N = (int)dofs.size();
    if (N == 0) return;
    int bestdim = -1;
    double maxrange = -1.0;
    for (int k = 0; k < d; ++k) {
        double maxi = std::numeric_limits<double>::lowest(), mini = std::numeric_limits<double>::max();
        for (int idof : dofs) {
            maxi = std::max(maxi, X[(size_t)idof * d + k]);
            mini = std::min(mini, X[(size_t)idof * d + k]);
        }
        double range = maxi - mini;
        if (range > maxrange) { bestdim = k; maxrange = range; }
    }
    // Value of the (N/2)-th smallest coordinate (independent of sort stability).
    std::vector<double> vals(N);
    for (int q = 0; q < N; ++q) vals[q] = X[(size_t)dofs[q] * d + bestdim];
    std::nth_element(vals.begin(), vals.begin() + N / 2, vals.end());
    double midv = vals[N / 2];
    for (int q = 0; q < N; ++q) {
        int j = dofs[q];
        parts[j] = (X[(size_t)j * d + bestdim] <= midv) ? start : start + 1;
    }
}

// form_rmap, ClusterID form (src/tree.cpp:57-98); cmap here is "cpermed".
static void form_rmap_ids(const Csc& A, std::vector<ClusterID>& rmap, const std::vector<ClusterID>& cpermed,
                          const std::vector<int>& cperm) {
    Csc At = transpose(col_perm(A, cperm));
    ClusterID last = cpermed[A.n - 1];
    for (int i = 0; i < A.m; ++i) {
        double max_val = -1;
        ClusterID rid = rmap[i];
        if (rid == ClusterID()) {
            int k = At.p[i], e = At.p[i + 1];
            while (k < e) {
                ClusterID cid = cpermed[At.i[k]];
                double val = At.v[k] * At.v[k];
                int q = k + 1;
                while (q < e && cid == cpermed[At.i[q]]) { val += At.v[q] * At.v[q]; ++q; }
                if (val > max_val) { max_val = val; rid = cid; }
                k = q;
            }
            if (rid == ClusterID()) rid = last;
            rmap[i] = rid;
        }
    }
}

static void get_interfaces_using_A(const Csc& A, std::vector<ClusterID>& cmap, std::vector<ClusterID>& rmap) {
    const int nrows = A.m;
    Csc At = transpose(A);
    for (int i = 0; i < nrows; ++i) {
        SepID self = rmap[i].self;
        if (self.lvl > 0) {
            SepID left(-1, 0), right(-1, 0);
            for (int q = At.p[i]; q < At.p[i + 1]; ++q) {
                SepID nbr = cmap[At.i[q]].self;
                if (nbr.lvl < self.lvl) {
                    int pj = nbr.sep;
                    pj = (int)(pj / std::pow(2.0, self.lvl - nbr.lvl - 1));
                    if (pj % 2 == 0) left = (left.lvl == -1) ? nbr : find_lowest_common(nbr, left);
                    else right = (right.lvl == -1) ? nbr : find_lowest_common(nbr, right);
                }
            }
            rmap[i].l = left;
            rmap[i].r = right;
        }
    }
    cmap = rmap;  // rmap2cmap without matching (src/partition.cpp:150-156)
    for (int i = 0; i < nrows; ++i) {
        SepID self = rmap[i].self, left = rmap[i].l, right = rmap[i].r;
        if (right == SepID()) {
            for (int q = At.p[i]; q < At.p[i + 1]; ++q) {
                int j = At.i[q];
                if (self == cmap[j].self && cmap[j].r != SepID())
                    right = (right == SepID()) ? cmap[j].r : find_highest_common(right, cmap[j].r);
            }
        } else if (left == SepID()) {
            for (int q = At.p[i]; q < At.p[i + 1]; ++q) {
                int j = At.i[q];
                if (self == cmap[j].self && cmap[j].l != SepID())
                    left = (left == SepID()) ? cmap[j].l : find_highest_common(left, cmap[j].l);
            }
        }
        rmap[i].l = left;
        rmap[i].r = right;
    }
    for (int i = 0; i < nrows; ++i) {
        if (rmap[i].l == SepID()) rmap[i].l = rmap[i].self;
        if (rmap[i].r == SepID()) rmap[i].r = rmap[i].self;
    }
    cmap = rmap;
}

static std::vector<ClusterID> geometric_partition_ata(const Csc& A, int nlevels, const std::vector<double>& X,
                                                      int d) {
    Csc AtA = ata_pattern(A);
    const int c = AtA.n;
    std::vector<int> parts(c, 0);
    for (int depth = 0; depth < nlevels - 1; ++depth) {
        int np = 1 << depth;
        std::vector<std::vector<int>> dofs(np);
        for (int i = 0; i < c; ++i) dofs[parts[i]].push_back(i);
        for (int k = 0; k < np; ++k) bissect_geo(dofs[k], parts, X, d, 2 * k);
    }
    std::vector<ClusterID> cmap(c);
    for (int depth = 0; depth < nlevels - 1; ++depth) {
        int l = nlevels - depth - 1;
        for (int i = 0; i < c; ++i) {
            if (cmap[i].self.lvl != -1) continue;
            int pi = part_at_lvl(parts[i], l);
            if (pi % 2 != 0) continue;
            bool sep = false;
            for (int q = AtA.p[i]; q < AtA.p[i + 1]; ++q) {
                int j = AtA.i[q];
                if (cmap[j].self.lvl == -1 && part_at_lvl(parts[j], l) == pi + 1) { sep = true; break; }
            }
            if (sep) cmap[i].self = SepID(l, pi / 2);
        }
    }
    for (int i = 0; i < c; ++i)
        if (cmap[i].self.lvl == -1) cmap[i].self = cmap[i].l = cmap[i].r = SepID(0, parts[i]);

    std::vector<ClusterID> rmap(A.m);
    if (A.m != A.n) {  // rows2clusters (src/partition.cpp:103-134)
        std::vector<int> cperm(c);
        for (int i = 0; i < c; ++i) cperm[i] = i;
        std::stable_sort(cperm.begin(), cperm.end(), [&](int a, int b) { return cmap[a] < cmap[b]; });
        std::vector<ClusterID> cpermed(c);
        for (int k = 0; k < c; ++k) cpermed[k] = cmap[cperm[k]];
        form_rmap_ids(A, rmap, cpermed, cperm);
    } else {
        rmap = cmap;
    }
    get_interfaces_using_A(A, cmap, rmap);
    return cmap;
}

// MetisPartition after METIS_PartGraphRecursive (src/partition.cpp:374-426)
// and getInterfacesUsingATA (src/partition.cpp:628-675). METIS is absent, so
// the leaf part vector `parts` is an input (the reference gets it from
// partition_metis_RB, src/partition.cpp:354-372).
static std::vector<ClusterID> metis_partition(const Csc& A, int nlevels, const std::vector<int>& parts) {
    Csc AtA = ata_pattern(A);
    const int c = AtA.n;
    if ((int)parts.size() != c) throw std::runtime_error("parts must have one entry per column");
    std::vector<ClusterID> cmap(c);
    for (int depth = 0; depth < nlevels - 1; ++depth) {
        int l = nlevels - depth - 1;
        for (int i = 0; i < c; ++i) {
            if (cmap[i].self.lvl != -1) continue;
            int pi = part_at_lvl(parts[i], l);
            if (pi % 2 != 0) continue;
            bool sep = false;
            for (int q = AtA.p[i]; q < AtA.p[i + 1]; ++q) {
                int j = AtA.i[q];
                if (cmap[j].self.lvl == -1 && part_at_lvl(parts[j], l) == pi + 1) { sep = true; break; }
            }
            if (sep) cmap[i].self = SepID(l, pi / 2);
        }
    }
    for (int i = 0; i < c; ++i)
        if (cmap[i].self.lvl == -1) cmap[i].self = cmap[i].l = cmap[i].r = SepID(0, parts[i]);
    // getInterfacesUsingATA
    for (int i = 0; i < c; ++i) {
        SepID self = cmap[i].self;
        if (self.lvl > 0) {
            SepID left(0, parts[i]), right(-1, 0);
            int pi = part_at_lvl(parts[i], self.lvl);
            for (int q = AtA.p[i]; q < AtA.p[i + 1]; ++q) {
                int j = AtA.i[q];
                SepID nbr = cmap[j].self;
                if (nbr.lvl < self.lvl) {
                    int pj = part_at_lvl(parts[j], self.lvl);
                    if (pj <= pi) left = find_highest_common(nbr, left);
                    else right = (right.lvl == -1) ? nbr : find_highest_common(nbr, right);
                }
            }
            if (right.lvl == -1) throw std::runtime_error("separator without a right side");
            cmap[i].l = left;
            cmap[i].r = right;
            cmap[i].section = parts[i];
        }
    }
    for (int i = 0; i < c; ++i) {
        if (cmap[i].self.lvl == 0) {
            cmap[i].l = cmap[i].self;
            cmap[i].r = cmap[i].self;
            cmap[i].section = parts[i];
        }
    }
    return cmap;
}

// initPermutation (src/tree.cpp:46-55)
static void init_permutation(int nlevels, const std::vector<ClusterID>& cmap, std::vector<int>& cperm) {
    std::vector<ClusterID> pm = cmap;
    auto comp = [&pm](int a, int b) { return pm[a] < pm[b]; };
    std::stable_sort(cperm.begin(), cperm.end(), comp);
    for (int lvl = 1; lvl < nlevels; ++lvl) {
        for (auto& s : pm) s = merge_if(s, lvl);
        std::stable_sort(cperm.begin(), cperm.end(), comp);
    }
}

// ---------------------------------------------------------------------------
// Dense blocks, clusters, edges (include/cluster.h:118-248, include/edge.h)
// ---------------------------------------------------------------------------
struct Mat {
    int rows = 0, cols = 0;
    std::vector<double> a;  // column-major, ld = rows
    Mat() = default;
    Mat(int r, int c) : rows(r), cols(c), a((size_t)r * c, 0.0) {}
    double* data() { return a.data(); }
    const double* data() const { return a.data(); }
    double& operator()(int i, int j) { return a[(size_t)j * rows + i]; }
    double operator()(int i, int j) const { return a[(size_t)j * rows + i]; }
    // conservativeResize(nr, NoChange): keeps the overlapping top rows.
    void resize_rows(int nr) {
        Mat b(nr, cols);
        int k = std::min(nr, rows);
        for (int j = 0; j < cols; ++j)
            for (int i = 0; i < k; ++i) b(i, j) = (*this)(i, j);
        *this = std::move(b);
    }
    Mat top_rows(int k) const { return block(0, 0, k, cols); }
    Mat block(int i0, int j0, int r, int c) const {
        Mat b(r, c);
        for (int j = 0; j < c; ++j)
            for (int i = 0; i < r; ++i) b(i, j) = (*this)(i0 + i, j0 + j);
        return b;
    }
    void set_block(int i0, int j0, const Mat& s) {
        for (int j = 0; j < s.cols; ++j)
            for (int i = 0; i < s.rows; ++i) (*this)(i0 + i, j0 + j) = s(i, j);
    }
};

struct Cluster;
struct Edge {
    Cluster* n1;
    Cluster* n2;
    std::unique_ptr<Mat> A;  // A(rows of n2, cols of n1); null once freed
};

struct ByOrder {
    bool operator()(const Cluster* a, const Cluster* b) const;
};

struct Cluster {
    int cstart, csize, rstart, rsize;
    ClusterID id;
    int order;
    bool eliminated = false;
    int csize_org, rsize_org;
    Cluster* parent = nullptr;
    ClusterID parentid;
    std::vector<double> tau;
    Mat T;
    std::vector<double> x, xt;
    int rposparent = 0, cposparent = 0;
    std::vector<Cluster*> children;
    std::set<Cluster*, ByOrder> rsparsity, cnbrs;
    std::list<Edge*> edgesOut, edgesIn;
    Cluster(int cs, int cz, int rs, int rz, ClusterID i, int o)
        : cstart(cs), csize(cz), rstart(rs), rsize(rz), id(i), order(o), csize_org(cz), rsize_org(rz) {
        set_size(rz, cz);
    }
    int level() const { return id.self.lvl; }
    int cols() const { return csize; }
    int rows() const { return rsize; }
    void set_size(int r, int c) {  // src/cluster.cpp:79-89
        rsize = r;
        csize = c;
        x.assign(r, 0.0);
        xt.assign(r, 0.0);
    }
    void reset_size(int r, int c) { rsize = r; csize = c; }
    void resize_x(int r) {
        x.resize(x.size() + r, 0.0);
        xt.resize(xt.size() + r, 0.0);
    }
    Edge* self_edge() {
        for (Edge* e : edgesOut)
            if (e->n2 == this) return e;
        return nullptr;
    }
};

bool ByOrder::operator()(const Cluster* a, const Cluster* b) const { return a->order < b->order; }

static Edge* find_out(Cluster* c, Cluster* n2) {
    for (Edge* e : c->edgesOut)
        if (e->n2 == n2) return e;
    return nullptr;
}

// ---------------------------------------------------------------------------
// LAPACK wrappers (src/util.cpp:233-816)
// ---------------------------------------------------------------------------
static void geqrf(Mat& A, std::vector<double>& tau) {
    if (A.rows == 0 || A.cols == 0) return;
    L().dgeqrf(kColMajor, A.rows, A.cols, A.data(), A.rows, tau.data());
}
static void larft(const Mat& V, const std::vector<double>& tau, Mat& T) {
    if (V.rows == 0 || V.cols == 0) return;
    L().dlarft(kColMajor, 'F', 'C', V.rows, V.cols, V.data(), V.rows, tau.data(), T.data(), T.rows);
}
// C <- H^T C (src/util.cpp:421-443); V is C.rows x k.
static void larfb_lt(const Mat& V, const Mat& T, double* C, int m, int n) {
    if (m == 0 || n == 0 || V.cols == 0) return;
    L().dlarfb(kColMajor, 'L', 'T', 'F', 'C', m, n, V.cols, V.data(), m, T.data(), V.cols, C, m);
}
static void larfb_vec(const Mat& V, const Mat& T, double* x, int m, char trans) {
    if (m == 0 || V.cols == 0) return;
    L().dlarfb(kColMajor, 'L', trans, 'F', 'C', m, 1, V.cols, V.data(), m, T.data(), V.cols, x, m);
}
static void geqp3(Mat& A, std::vector<int>& jpvt, std::vector<double>& tau) {
    if (A.rows == 0 || A.cols == 0) return;
    L().dgeqp3(kColMajor, A.rows, A.cols, A.data(), A.rows, jpvt.data(), tau.data());
    for (int& j : jpvt) j--;
}
// gesvd_values (src/util.cpp:767-782): singular values only, same job flags.
static std::vector<double> gesvd_values(Mat A) {
    const int m = A.rows, n = A.cols, k = std::min(m, n);
    std::vector<double> S(k, 0.0);
    if (k == 0) return S;
    std::vector<double> U((size_t)m * m), VT((size_t)n * n), superb(std::max(1, k - 1));
    L().dgesvd(kColMajor, 'O', 'N', m, n, A.data(), m, S.data(), U.data(), m, VT.data(), n, superb.data());
    return S;
}
static void trsm_right_upper(const Mat& R, Mat& B) {
    if (B.rows == 0 || B.cols == 0) return;
    L().dtrsm(kColMajor, kRight, kUpper, kNoTrans, kNonUnit, B.rows, B.cols, 1.0, R.data(), R.rows, B.data(),
              B.rows);
}
static void trsv_upper(const Mat& R, double* x, int n, bool trans) {
    if (n == 0) return;
    L().dtrsv(kColMajor, kUpper, trans ? kTrans : kNoTrans, kNonUnit, n, R.data(), R.rows, x, 1);
}
// x <- Q^T x / Q x with Q from (v, tau) (src/util.cpp:306-329).
static void ormqr_vec(const Mat& v, const std::vector<double>& tau, double* x, int m, char trans) {
    if (m == 0 || v.cols == 0) return;
    L().dormqr(kColMajor, 'L', trans, m, 1, v.cols, v.data(), v.rows, tau.data(), x, m);
}

static int choose_rank(const std::vector<double>& s, double tol, bool rel = true) {
    // src/util.cpp:795-816
    if (tol == 0) return (int)s.size();
    if (tol >= 1.0) return 0;
    if (s.size() <= 1) return (int)s.size();
    double sref = rel ? std::abs(s[0]) : 1.0;
    int rank = 1;
    while (rank < (int)s.size() && std::abs(s[rank]) / sref >= tol) rank++;
    return rank;
}

// ---------------------------------------------------------------------------
// Operations (src/operations.cpp, src/toperations.cpp)
// ---------------------------------------------------------------------------
struct Op {
    virtual ~Op() = default;
    virtual void fwd() = 0;
    virtual void bwd() = 0;
    virtual const char* name() const = 0;
    // Solution segments (Cluster::x) the forward or backward part reads or
    // writes, for the wave-parallel solve; nullptr stands for "all of them"
    // (the op then runs alone, in tape order).
    virtual void touch(bool fwd, std::vector<const void*>& keys) const {
        (void)fwd;
        keys.push_back(nullptr);
    }
};

// QR (src/operations.cpp:12-57, include/operations.h:22-50)
struct OpQR : Op {
    Cluster* c;
    int nrows = 0, ncols, ccols;
    std::vector<int> a21, a12;
    explicit OpQR(Cluster* c_) : c(c_), ncols(c_->cols()), ccols(c_->cols()) {
        for (Edge* e : c->edgesOut)
            if (e->A) { a21.push_back(e->n2->rows()); nrows += e->A->rows; }
        for (Edge* e : c->edgesIn) a12.push_back(e->A->cols);
    }
    void fwd() override {
        Mat Q(nrows, ncols);
        std::vector<double> xc(nrows, 0.0);
        int cur = 0, i = 0;
        for (Edge* e : c->edgesOut) {
            if (!e->A) continue;
            int s = a21[i];
            for (int q = 0; q < s; ++q) xc[cur + q] = e->n2->x[q];
            Q.set_block(cur, 0, *e->A);
            cur += s;
            ++i;
        }
        larfb_vec(Q, c->T, xc.data(), nrows, 'T');
        cur = 0;
        i = 0;
        for (Edge* e : c->edgesOut) {
            if (!e->A) continue;
            int s = a21[i];
            for (int q = 0; q < s; ++q) e->n2->x[q] = xc[cur + q];
            cur += s;
            ++i;
        }
    }
    void bwd() override {
        double* xs = c->x.data();
        int i = 0;
        for (Edge* e : c->edgesIn) {
            int s = a12[i];
            const Mat& B = *e->A;
            const double* xn = e->n1->x.data();
            for (int j = 0; j < s; ++j)
                for (int r = 0; r < ccols; ++r) xs[r] -= B(r, j) * xn[j];
            ++i;
        }
        Mat R = c->edgesOut.front()->A->top_rows(ccols);
        trsv_upper(R, xs, ccols, false);
    }
    const char* name() const override { return "QR"; }
    void touch(bool f, std::vector<const void*>& keys) const override {
        if (f) {
            for (Edge* e : c->edgesOut)
                if (e->A) keys.push_back(e->n2);
        } else {
            keys.push_back(c);
            for (Edge* e : c->edgesIn) keys.push_back(e->n1);
        }
    }
};

// Reassign (src/operations.cpp:60-69)
struct OpReassign : Op {
    Cluster *c, *n;
    int nstart, nrows;
    std::vector<int> idx;
    OpReassign(Cluster* c_, const std::vector<int>& ind, Cluster* n_, int ns, int nr)
        : c(c_), n(n_), nstart(ns), nrows(nr) {
        for (int v : ind) idx.push_back(c_->cols() + v);
    }
    void fwd() override {
        for (int i = nstart; i < nstart + nrows; ++i) n->x[i] = c->x[idx[i - nstart]];
    }
    void bwd() override {}
    const char* name() const override { return "Reassign"; }
};

// ScaleD (src/operations.cpp:76-84): Q holds geqrf output (square) or R (rectangular).
struct OpScaleD : Op {
    Cluster* c;
    int hs, fs;  // head / full segment lengths at creation
    Mat Q;
    std::vector<double> t;
    bool has_t;
    OpScaleD(Cluster* c_, Mat Q_, std::vector<double> t_, bool ht)
        : c(c_), hs(c_->cols()), fs(c_->rows()), Q(std::move(Q_)), t(std::move(t_)), has_t(ht) {}
    void fwd() override { ormqr_vec(Q, t, c->x.data(), fs, 'T'); }
    void bwd() override {
        Mat R = Q.top_rows(hs);
        trsv_upper(R, c->x.data(), hs, false);
    }
    const char* name() const override { return "ScaleD"; }
    void touch(bool, std::vector<const void*>& keys) const override { keys.push_back(c); }
};

// OrthogonalD (src/operations.cpp:89-90)
struct OpOrthD : Op {
    Cluster* c;
    int hs;
    Mat V;
    std::vector<double> tau;
    OpOrthD(Cluster* c_, Mat V_, std::vector<double> tau_) : c(c_), hs(c_->cols()), V(std::move(V_)),
                                                             tau(std::move(tau_)) {}
    // c's column count before the split given explicitly (the wave-parallel
    // sparsification resizes c before the op is recorded)
    OpOrthD(Cluster* c_, Mat V_, std::vector<double> tau_, int hs_) : c(c_), hs(hs_), V(std::move(V_)),
                                                                      tau(std::move(tau_)) {}
    void fwd() override { ormqr_vec(V, tau, c->x.data(), hs, 'T'); }
    void bwd() override { ormqr_vec(V, tau, c->x.data(), V.rows, 'N'); }
    const char* name() const override { return "OrthogonalD"; }
    void touch(bool, std::vector<const void*>& keys) const override { keys.push_back(c); }
};

// Orthogonal (src/operations.cpp:87, include/operations.h:113-129): no forward
// part; backward x_head <- Q x_head over the cluster's columns before the split.
struct OpOrth : Op {
    Cluster* c;
    Mat V;
    std::vector<double> tau;
    OpOrth(Cluster* c_, Mat V_, std::vector<double> tau_) : c(c_), V(std::move(V_)), tau(std::move(tau_)) {}
    void fwd() override {}
    void bwd() override { ormqr_vec(V, tau, c->x.data(), V.rows, 'N'); }
    const char* name() const override { return "Orthogonal"; }
};

// Split (src/operations.cpp:118-119, include/operations.h:165-177): the fine
// cluster takes the last rows of the coarse one's full segment (forward) and
// gives its values back to the last entries of the coarse head (backward).
struct OpSplit : Op {
    Cluster *c, *f;
    int chead, cfull, fs;
    OpSplit(Cluster* c_, Cluster* f_) : c(c_), f(f_), chead(c_->cols()), cfull(c_->rows()), fs(f_->rows()) {}
    void fwd() override {
        for (int q = 0; q < fs; ++q) f->x[q] = c->x[cfull - fs + q];
    }
    void bwd() override {
        for (int q = 0; q < fs; ++q) c->x[chead - fs + q] = f->x[q];
    }
    const char* name() const override { return "Split"; }
};

// Merge (src/operations.cpp:94-115)
struct OpMerge : Op {
    Cluster* p;
    explicit OpMerge(Cluster* p_) : p(p_) {}
    void fwd() override {
        int k = 0;
        for (Cluster* c : p->children)
            for (int i = 0; i < c->rows(); ++i) p->x[k++] = c->x[i];
    }
    void bwd() override {
        int k = 0;
        for (Cluster* c : p->children)
            for (int i = 0; i < c->cols(); ++i) c->x[i] = p->x[k++];
    }
    const char* name() const override { return "Merge"; }
    void touch(bool, std::vector<const void*>& keys) const override {
        keys.push_back(p);
        for (Cluster* c : p->children) keys.push_back(c);
    }
};

// SplitD (src/operations.cpp:121-131); shared by the transposed tape.
static void splitd_fwd(double* xc, double* xf, int crows, int ccols, int rank) {
    for (int q = 0; q < ccols - rank; ++q) xf[q] = xc[rank + q];
    std::vector<double> rem(xc + ccols, xc + crows);
    for (int q = 0; q < crows - ccols; ++q) xc[rank + q] = rem[q];
    for (int q = 0; q < ccols - rank; ++q) xc[crows - (ccols - rank) + q] = xf[q];
}
static void splitd_bwd(double* xc, const double* xf, int crows, int ccols, int rank) {
    std::vector<double> rem(xc + rank, xc + rank + (crows - ccols));
    for (int q = 0; q < ccols - rank; ++q) xc[rank + q] = xf[q];
    for (int q = 0; q < crows - ccols; ++q) xc[ccols + q] = rem[q];
}

struct OpSplitD : Op {
    Cluster *c, *f;
    int crows, ccols, rank;
    OpSplitD(Cluster* c_, Cluster* f_, int r) : c(c_), f(f_), crows(c_->rows()), ccols(c_->cols()), rank(r) {}
    // c's sizes before the split given explicitly (the wave-parallel
    // sparsification resizes c before the op is recorded)
    OpSplitD(Cluster* c_, Cluster* f_, int r, int cr, int cc) : c(c_), f(f_), crows(cr), ccols(cc), rank(r) {}
    void fwd() override { splitd_fwd(c->x.data(), f->x.data(), crows, ccols, rank); }
    void bwd() override { splitd_bwd(c->x.data(), f->x.data(), crows, ccols, rank); }
    const char* name() const override { return "SplitD"; }
    void touch(bool, std::vector<const void*>& keys) const override {
        keys.push_back(c);
        keys.push_back(f);
    }
};

// Transposed tape (src/toperations.cpp)
struct TOpQR : Op {
    Cluster* c;
    int nrows = 0, ncols, ccols;
    std::vector<int> a21, a12;
    explicit TOpQR(Cluster* c_) : c(c_), ncols(c_->cols()), ccols(c_->cols()) {
        for (Edge* e : c->edgesOut)
            if (e->A) { a21.push_back(e->n2->rows()); nrows += e->A->rows; }
        for (Edge* e : c->edgesIn) a12.push_back(e->A->cols);
    }
    void fwd() override {
        double* xs = c->xt.data();
        Mat R = c->edgesOut.front()->A->top_rows(ccols);
        trsv_upper(R, xs, ccols, true);
        int i = 0;
        for (Edge* e : c->edgesIn) {
            int s = a12[i];
            const Mat& B = *e->A;
            double* xn = e->n1->xt.data();
            for (int j = 0; j < s; ++j) {
                double acc = 0.0;
                for (int r = 0; r < ccols; ++r) acc += B(r, j) * xs[r];
                xn[j] -= acc;
            }
            ++i;
        }
    }
    void bwd() override {
        Mat Q(nrows, ncols);
        std::vector<double> xc(nrows, 0.0);
        int cur = 0, i = 0;
        for (Edge* e : c->edgesOut) {
            if (!e->A) continue;
            int s = a21[i];
            for (int q = 0; q < s; ++q) xc[cur + q] = e->n2->xt[q];
            Q.set_block(cur, 0, *e->A);
            cur += s;
            ++i;
        }
        larfb_vec(Q, c->T, xc.data(), nrows, 'N');
        cur = 0;
        i = 0;
        for (Edge* e : c->edgesOut) {
            if (!e->A) continue;
            int s = a21[i];
            for (int q = 0; q < s; ++q) e->n2->xt[q] = xc[cur + q];
            cur += s;
            ++i;
        }
    }
    const char* name() const override { return "QR"; }
};

struct TOpReassign : Op {
    Cluster *c, *n;
    int nstart, nrows;
    std::vector<int> idx;
    TOpReassign(Cluster* c_, const std::vector<int>& ind, Cluster* n_, int ns, int nr)
        : c(c_), n(n_), nstart(ns), nrows(nr) {
        for (int v : ind) idx.push_back(c_->cols() + v);
    }
    void fwd() override {}
    void bwd() override {
        for (int i = nstart; i < nstart + nrows; ++i) c->xt[idx[i - nstart]] = n->xt[i];
    }
    const char* name() const override { return "Reassign"; }
};

struct TOpScaleD : Op {
    Cluster* c;
    int hs;
    Mat R;
    TOpScaleD(Cluster* c_, Mat R_) : c(c_), hs(c_->cols()), R(std::move(R_)) {}
    void fwd() override {
        Mat Rt = R.top_rows(hs);
        trsv_upper(Rt, c->xt.data(), hs, true);
    }
    void bwd() override {}
    const char* name() const override { return "ScaleD"; }
};

struct TOpOrthD : Op {
    Cluster* c;
    int hs;
    const Mat* V;
    const std::vector<double>* tau;
    TOpOrthD(Cluster* c_, const Mat* V_, const std::vector<double>* t_) : c(c_), hs(c_->cols()), V(V_), tau(t_) {}
    void fwd() override { ormqr_vec(*V, *tau, c->xt.data(), hs, 'T'); }
    void bwd() override { ormqr_vec(*V, *tau, c->xt.data(), V->rows, 'N'); }
    const char* name() const override { return "OrthogonalD"; }
};

struct TOpMerge : Op {
    Cluster* p;
    explicit TOpMerge(Cluster* p_) : p(p_) {}
    void fwd() override {
        int k = 0;
        for (Cluster* c : p->children)
            for (int i = 0; i < c->cols(); ++i) p->xt[k++] = c->xt[i];
    }
    void bwd() override {
        int k = 0;
        for (Cluster* c : p->children)
            for (int i = 0; i < c->rows(); ++i) c->xt[i] = p->xt[k++];
    }
    const char* name() const override { return "Merge"; }
};

struct TOpSplitD : Op {
    Cluster *c, *f;
    int crows, ccols, rank;
    TOpSplitD(Cluster* c_, Cluster* f_, int r) : c(c_), f(f_), crows(c_->rows()), ccols(c_->cols()), rank(r) {}
    void fwd() override { splitd_fwd(c->xt.data(), f->xt.data(), crows, ccols, rank); }
    void bwd() override { splitd_bwd(c->xt.data(), f->xt.data(), crows, ccols, rank); }
    const char* name() const override { return "SplitD"; }
};

// ---------------------------------------------------------------------------
// Tree (src/tree.cpp, include/tree.h)
// ---------------------------------------------------------------------------
// Fixed pool of host threads for the wave-parallel mode: run(n, k, f) calls
// f(0..n-1) on up to k threads (the caller included), each index once, and
// rethrows the first exception after all have finished.
class Pool {
public:
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& th : workers_) th.join();
    }
    void run(int n, int k, const std::function<void(int)>& f) {
        if (n <= 0) return;
        k = std::max(1, std::min(k, n));
        while ((int)workers_.size() < k - 1) workers_.emplace_back([this] { loop(); });
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &f;
            n_ = n;
            next_ = 0;
            tickets_ = k - 1;  // workers that may join this run
            running_ = 0;
            gen_++;
            err_.clear();
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(mu_);
        done_.wait(g, [&] { return tickets_ == 0 && running_ == 0; });
        job_ = nullptr;
        if (!err_.empty()) throw std::runtime_error(err_);
    }

private:
    void work() {
        for (;;) {
            const int i = next_.fetch_add(1);
            if (i >= n_) break;
            try {
                (*job_)(i);
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> g(mu_);
                if (err_.empty()) err_ = e.what();
            }
        }
    }
    void loop() {
        long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || (gen_ != seen && tickets_ > 0); });
                if (stop_) return;
                seen = gen_;
                --tickets_;
                ++running_;
            }
            work();
            {
                std::lock_guard<std::mutex> g(mu_);
                --running_;
            }
            done_.notify_all();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    std::atomic<int> next_{0};
    int n_ = 0, tickets_ = 0, running_ = 0;
    long long gen_ = 0;
    bool stop_ = false;
    std::string err_;
};

static Pool& pool() {
    static Pool p;
    return p;
}

class Tree {
public:
    Tree(int nlevels, int skip) : nlevels_(nlevels), skip_(skip), bottoms_(nlevels), fine_(nlevels) {}
    ~Tree() {
        for (auto& c : all_) {
            for (Edge* e : c->edgesOut) owned_edges_.insert(e);
        }
        for (Edge* e : owned_edges_) delete e;
    }
    int nlevels_, skip_;
    double tol_ = 0;
    int scale_ = 0, square_ = 0;
    float order_ = 1;
    int d_ = 0;
    std::vector<double> X_;
    std::vector<int> parts_;    // leaf parts for the partition without coordinates
    bool numeric_fill_ = true;  // without coordinates: the numeric fill test of src/tree.cpp:857-860
    int nrows_ = 0, ncols_ = 0, ilvl_ = -1, current_bottom_ = 0, max_order_ = 0;
    std::vector<int> cperm_, rperm_;
    std::vector<std::list<Cluster*>> bottoms_, fine_;
    std::vector<std::unique_ptr<Cluster>> all_;
    std::set<Edge*> owned_edges_;
    std::vector<std::unique_ptr<Op>> ops_, tops_;
    unsigned long long nnzA_ = 0, nnzR_ = 0, nnzH_ = 0, nnzQ_ = 0;
    std::vector<long long> log_;
    double t_part_ = 0, t_asm_ = 0, t_fact_ = 0;

    void rec(long long type, long long a, long long b = 0, long long c = 0, long long d = 0, long long e = 0,
             long long order = -1) {
        long long r[8] = {type, ilvl_, order, a, b, c, d, e};
        log_.insert(log_.end(), r, r + 8);
    }

    Cluster* new_cluster(int cs, int cz, int rs, int rz, ClusterID id) {
        all_.emplace_back(new Cluster(cs, cz, rs, rz, id, max_order_++));
        return all_.back().get();
    }
    const std::list<Cluster*>& bottom_current() const { return bottoms_[current_bottom_]; }
    const std::list<Cluster*>& bottom_original() const { return bottoms_[0]; }

    Edge* add_edge(Cluster* c1, Cluster* c2) {  // src/tree.cpp:251-261
        Edge* e = new Edge{c1, c2, std::unique_ptr<Mat>(new Mat(c2->rows(), c1->cols()))};
        owned_edges_.insert(e);
        c1->cnbrs.insert(c2);
        c1->edgesOut.push_back(e);
        if (c1 != c2) c2->edgesIn.push_back(e);
        return e;
    }

    std::pair<int, int> topsize() const {  // src/tree.cpp:27-37
        int tc = 0, tr = 0;
        for (Cluster* s : bottom_current())
            if (s->level() == nlevels_ - 1) { tc += s->cols(); tr += s->rows(); }
        return {tr, tc};
    }

    // -------- partition (src/tree.cpp:595-723) --------
    void partition(const Csc& A) {
        double t0 = now();
        const int r = A.m, c = A.n;
        nrows_ = r;
        ncols_ = c;
        if (X_.empty() && parts_.empty())
            throw std::runtime_error("set coordinates, or the leaf parts of the partition without them");
        std::vector<ClusterID> cmap =
            X_.empty() ? metis_partition(A, nlevels_, parts_) : geometric_partition_ata(A, nlevels_, X_, d_);
        rperm_.resize(r);
        cperm_.resize(c);
        for (int i = 0; i < r; ++i) rperm_[i] = i;
        for (int i = 0; i < c; ++i) cperm_[i] = i;
        init_permutation(nlevels_, cmap, cperm_);
        std::vector<ClusterID> cpermed(c);
        for (int k = 0; k < c; ++k) cpermed[k] = cmap[cperm_[k]];
        std::vector<int> c2r_count(c, 0);
        if (!square_) {
            Csc Ap = col_perm(A, cperm_);
            form_rmap_rows(Ap, cpermed, c2r_count);
        } else {
            std::fill(c2r_count.begin(), c2r_count.end(), 1);
            rperm_ = cperm_;
        }
        int k = 0, l = 0;
        while (k < c) {
            int kn = k + 1;
            ClusterID cid = cpermed[k];
            int nr2c = c2r_count[k];
            while (kn < c && cid == cpermed[kn]) { nr2c += c2r_count[kn]; kn++; }
            Cluster* self = new_cluster(k, kn - k, l, nr2c, cid);
            bottoms_[0].push_back(self);
            k = kn;
            l += nr2c;
        }
        if (l != r) throw std::runtime_error("row count mismatch in partition");
        for (int lvl = 1; lvl < nlevels_; ++lvl) {
            auto& prev = bottoms_[lvl - 1];
            auto begin = std::find_if(prev.begin(), prev.end(), [lvl](Cluster* s) { return s->level() >= lvl; });
            for (auto it = begin; it != prev.end(); ++it) (*it)->parentid = merge_if((*it)->id, lvl);
            for (auto it = begin; it != prev.end();) {
                ClusterID pid = (*it)->parentid;
                std::vector<Cluster*> ch{*it};
                int cs = (*it)->cols(), rs = (*it)->rows(), c0 = (*it)->cstart, r0 = (*it)->rstart;
                ++it;
                while (it != prev.end() && pid == (*it)->parentid) {
                    ch.push_back(*it);
                    cs += (*it)->cols();
                    rs += (*it)->rows();
                    ++it;
                }
                Cluster* p = new_cluster(c0, cs, r0, rs, pid);
                for (Cluster* x : ch) { x->parent = p; p->children.push_back(x); }
                bottoms_[lvl].push_back(p);
            }
        }
        t_part_ = now() - t0;
    }

    // form_rmap, row-permutation form (src/tree.cpp:100-163), unmatched.
    void form_rmap_rows(const Csc& Ap, const std::vector<ClusterID>& cpermed, std::vector<int>& c2r_count) {
        const int r = Ap.m, c = Ap.n;
        Csc At = transpose(Ap);
        std::vector<std::vector<int>> c2r(c);
        for (int i = 0; i < r; ++i) {
            double max_val = -1;
            int cidx = -1;
            int k = At.p[i], e = At.p[i + 1];
            while (k < e) {
                ClusterID cid = cpermed[At.i[k]];
                double val = At.v[k] * At.v[k];
                int q = k + 1;
                while (q < e && cid == cpermed[At.i[q]]) { val += At.v[q] * At.v[q]; ++q; }
                if (val > max_val) { max_val = val; cidx = At.i[k]; }
                k = q;
            }
            if (cidx == -1) cidx = c - 1;
            c2r_count[cidx]++;
            c2r[cidx].push_back(i);
        }
        int start = 0;
        for (int i = 0; i < c; ++i)
            for (int j = 0; j < c2r_count[i]; ++j) rperm_[start++] = c2r[i][j];
    }

    // -------- assemble (src/tree.cpp:725-778) --------
    void assemble(const Csc& A) {
        double t0 = now();
        const int r = A.m, c = A.n;
        nnzA_ = A.i.size();
        // App = A(rperm, cperm)
        Csc Ap = col_perm(A, cperm_);
        Csc ApT = transpose(Ap);
        Csc App = transpose(col_perm(ApT, rperm_));
        std::vector<Cluster*> cmap(c), rmap(r);
        for (Cluster* s : bottom_original()) {
            for (int k = s->cstart; k < s->cstart + s->cols(); ++k) cmap[k] = s;
            for (int i = s->rstart; i < s->rstart + s->rows(); ++i) rmap[i] = s;
        }
        for (Cluster* self : bottom_original()) {
            std::set<Cluster*, ByOrder> cn;
            for (int j = self->cstart; j < self->cstart + self->cols(); ++j)
                for (int q = App.p[j]; q < App.p[j + 1]; ++q) cn.insert(rmap[App.i[q]]);
            cn.insert(self);
            for (Cluster* nbr : cn) {
                Mat* sA = new Mat(nbr->rows(), self->cols());
                for (int col = 0; col < self->cols(); ++col) {
                    int j = self->cstart + col;
                    for (int q = App.p[j]; q < App.p[j + 1]; ++q) {
                        int row = App.i[q];
                        if (row >= nbr->rstart && row < nbr->rstart + nbr->rows())
                            (*sA)(row - nbr->rstart, col) = App.v[q];
                    }
                }
                Edge* e = new Edge{self, nbr, std::unique_ptr<Mat>(sA)};
                owned_edges_.insert(e);
                self->edgesOut.push_back(e);
                if (self != nbr) nbr->edgesIn.push_back(e);
            }
            self->edgesOut.sort([](Edge* a, Edge* b) { return a->n2->order < b->n2->order; });
            self->cnbrs = cn;
        }
        t_asm_ = now() - t0;
    }

    // -------- symbolic fill (src/tree.cpp:168-224, 834-870) --------
    bool check_if_valid(const ClusterID& cid, const ClusterID& nid, const std::set<SepID>& col_sparsity) const {
        SepID cself = cid.self, nself = nid.self;
        if (cself.lvl > nself.lvl) return false;
        int dd = nself.lvl - cself.lvl;
        int csep = cself.sep / (int)std::pow(2.0, dd);
        if (csep != nself.sep) return false;
        SepID nl = nid.l, nr = nid.r;
        int dl = nl.lvl - cself.lvl, dr = nr.lvl - cself.lvl;
        bool lyes, ryes;
        if (nl.lvl >= cself.lvl) lyes = (cself.sep / (int)std::pow(2.0, dl)) == nl.sep;
        else lyes = (nl.sep / (int)std::pow(2.0, -dl)) == cself.sep;
        if (nr.lvl >= cself.lvl) ryes = (cself.sep / (int)std::pow(2.0, dr)) == nr.sep;
        else ryes = (nr.sep / (int)std::pow(2.0, -dr)) == cself.sep;
        if (!lyes && !ryes) return false;
        if (X_.empty()) return true;  // the column-sparsity tests are geometric only
        if (!col_sparsity.count(nself)) return false;
        if (!col_sparsity.count(nl) && !col_sparsity.count(nr)) return false;
        return true;
    }

    // ||A1^T A2||_F (the numeric fill test's product, src/tree.cpp:858)
    static double product_norm(const Mat& A1, const Mat& A2) {
        double s = 0;
        for (int a = 0; a < A1.cols; ++a)
            for (int b = 0; b < A2.cols; ++b) {
                double dot = 0;
                for (int r = 0; r < A1.rows; ++r) dot += A1(r, a) * A2(r, b);
                s += dot * dot;
            }
        return std::sqrt(s);
    }

    void get_sparsity(Cluster* c) {
        std::set<Cluster*, ByOrder> rs;
        std::set<SepID> cs;
        for (Edge* e : c->edgesOut) cs.insert(e->n2->id.self);
        for (Edge* e : c->edgesOut) {
            if (!e->A) continue;
            Cluster* n = e->n2;
            rs.insert(n);
            for (Edge* ein : n->edgesIn) {
                if (ein->A && ein->n1 != c && !ein->n1->eliminated) {
                    Cluster* nin = ein->n1;
                    bool valid = check_if_valid(c->id, nin->id, cs);
                    if (X_.empty() && numeric_fill_ && valid && !(nin->id.l == c->id.self || nin->id.r == c->id.self))
                        valid = product_norm(*e->A, *ein->A) > 1e-14;
                    if (valid) rs.insert(nin);
                }
            }
        }
        c->rsparsity = rs;
    }

    // -------- elimination (src/tree.cpp:263-316, 780-832) --------
    void update_cluster(Cluster* c, Cluster* n, const Mat& Q) {
        std::vector<Mat*> N;
        Mat V(Q.rows, n->cols());
        int cur = 0;
        for (Edge* edge : c->edgesOut) {
            if (!edge->A) continue;
            Cluster* nbr = edge->n2;
            Edge* ecn = find_out(n, nbr);
            if (!ecn) ecn = add_edge(n, nbr);
            N.push_back(ecn->A.get());
            V.set_block(cur, 0, *ecn->A);
            cur += ecn->A->rows;
        }
        larfb_lt(Q, c->T, V.data(), V.rows, V.cols);
        cur = 0;
        for (Mat* b : N) {
            *b = V.block(cur, 0, b->rows, b->cols);
            cur += b->rows;
        }
    }

    void eliminate_cluster(Cluster* c) {
        if (c->cols() == 0) { c->eliminated = true; rec(1, 0, 0, 0, 0, 0, c->order); return; }
        std::vector<Mat*> H;
        int num_rows = 0, num_cols = 0;
        for (Edge* e : c->edgesOut)
            if (e->A) { H.push_back(e->A.get()); num_rows += e->A->rows; num_cols = e->A->cols; }
        Mat Q(num_rows, num_cols);
        int cur = 0;
        for (Mat* h : H) { Q.set_block(cur, 0, *h); cur += h->rows; }
        int k = std::min(num_rows, num_cols);
        c->tau.assign(k, 0.0);
        c->T = Mat(k, k);
        geqrf(Q, c->tau);
        if (square_) {
            cur = 0;
            for (Mat* h : H) { *h = Q.block(cur, 0, h->rows, h->cols); cur += h->rows; }
        } else {
            *H[0] = Q.top_rows(H[0]->cols);
        }
        larft(Q, c->tau, c->T);
        nnzH_ += (unsigned long long)(num_rows * num_cols);
        int nupd = 0, wtr = 0;
        for (Cluster* n : c->rsparsity) {
            if (!n->eliminated && c != n) {
                update_cluster(c, n, Q);
                nnzR_ += (unsigned long long)(c->cols() * n->cols());
                ++nupd;
                wtr += n->cols();
            }
        }
        if (!square_)
            for (Edge* e : c->edgesOut)
                if (e->n2 != c) e->A.reset();
        ops_.emplace_back(new OpQR(c));
        if (!square_) tops_.emplace_back(new TOpQR(c));
        c->eliminated = true;
        rec(1, num_rows, num_cols, nupd, (long long)H.size(), wtr, c->order);
    }

    // -------- rectangular row shift (src/tree.cpp:319-411) --------
    void reassign_rows(Cluster* c) {
        if (c->rows() == c->cols()) return;
        int rsize = c->rows() - c->cols();
        std::vector<std::pair<Cluster*, double>> r2c(rsize, {c, 0.0});
        for (Edge* edge : c->edgesIn) {
            Cluster* n = edge->n1;
            if (!find_out(c, n)) continue;
            const Mat& B = *edge->A;
            for (int i = 0; i < rsize; ++i) {
                double s = 0;
                for (int j = 0; j < B.cols; ++j) s += B(c->cols() + i, j) * B(c->cols() + i, j);
                double rn = std::sqrt(s);
                if (rn > r2c[i].second) r2c[i] = {n, rn};
            }
        }
        std::vector<int> row_perm(rsize);
        for (int i = 0; i < rsize; ++i) row_perm[i] = i;
        std::stable_sort(row_perm.begin(), row_perm.end(),
                         [&](int a, int b) { return r2c[a].first->order < r2c[b].first->order; });
        for (Edge* edge : c->edgesIn) {
            Cluster* nold = edge->n1;
            const Mat& B = *edge->A;
            Mat A12t(rsize, B.cols);
            for (int i = 0; i < rsize; ++i)
                for (int j = 0; j < B.cols; ++j) A12t(i, j) = B(c->cols() + row_perm[i], j);
            for (int i = 0; i < rsize;) {
                Cluster* nnew = r2c[row_perm[i]].first;
                int inext = i + 1;
                while (inext < rsize && nnew == r2c[row_perm[inext]].first) inext++;
                int rinc = inext - i;
                Edge* e = find_out(nold, nnew);
                if (nold == nnew) {
                    if (!e) throw std::runtime_error("reassign_rows: missing self edge");
                } else if (!e) {
                    e = add_edge(nold, nnew);
                }
                int old_r = e->A->rows;
                e->A->resize_rows(old_r + rinc);
                for (int q = 0; q < rinc; ++q)
                    for (int j = 0; j < e->A->cols; ++j) (*e->A)(old_r + q, j) = A12t(i + q, j);
                if (nold == nnew) {
                    int nstart = nnew->rows();
                    nnew->resize_x(rinc);
                    std::vector<int> ind(row_perm.begin() + i, row_perm.begin() + inext);
                    ops_.emplace_back(new OpReassign(c, ind, nnew, nstart, rinc));
                    if (!square_) tops_.emplace_back(new TOpReassign(c, ind, nnew, nstart, rinc));
                }
                i = inext;
            }
        }
        for (Edge* edge : c->edgesOut) {
            if (edge->n2 == c) continue;
            Cluster* n = edge->n2;
            Edge* fs = find_out(n, n);
            if (!fs) throw std::runtime_error("reassign_rows: neighbour without diagonal block");
            n->reset_size(fs->A->rows, fs->A->cols);
            for (Edge* e : n->edgesIn)
                if (!e->n1->eliminated && e->A && e->A->rows != n->rows()) e->A->resize_rows(n->rows());
        }
        rec(7, rsize, 0, 0, 0, 0, c->order);
    }

    // -------- merge (src/tree.cpp:414-475, 872-881) --------
    void update_size(Cluster* snew) {
        int rs = 0, cs = 0;
        for (Cluster* so : snew->children) {
            so->rposparent = rs;
            so->cposparent = cs;
            rs += so->rows();
            cs += so->cols();
        }
        snew->set_size(rs, cs);
        snew->csize_org = cs;
        snew->rsize_org = rs;
        ops_.emplace_back(new OpMerge(snew));
        if (!square_) tops_.emplace_back(new TOpMerge(snew));
        rec(4, rs, cs, (long long)snew->children.size(), 0, 0, snew->order);
    }

    void update_edges(Cluster* snew) {
        for (Cluster* so : snew->children)
            for (Edge* eo : so->edgesOut)
                if (!eo->n2->eliminated) snew->cnbrs.insert(eo->n2->parent);
        std::vector<Cluster*> nb(snew->cnbrs.begin(), snew->cnbrs.end());
        for (Cluster* n : nb) add_edge(snew, n);
        snew->edgesOut.sort([](Edge* a, Edge* b) { return a->n2->order < b->n2->order; });
        for (Cluster* so : snew->children) {
            for (Edge* eo : so->edgesOut) {
                Cluster* nold = eo->n2;
                if (nold->eliminated) continue;
                Edge* f = find_out(snew, nold->parent);
                if (!f) throw std::runtime_error("update_edges: missing parent edge");
                f->A->set_block(nold->rposparent, so->cposparent, *eo->A);
                eo->A.reset();  // the reference deletes the edge object
            }
        }
    }

    void merge_all() {
        current_bottom_++;
        for (Cluster* s : bottom_current()) update_size(s);
        for (Cluster* s : bottom_current()) update_edges(s);
    }

    // -------- scaling (src/tree.cpp:533-591) --------
    bool want_sparsify(Cluster* c) const {
        if (c->level() > ilvl_) return c->id.l.lvl <= ilvl_ && c->id.r.lvl <= ilvl_;
        return false;
    }

    void diag_scale(Cluster* c) {
        Edge* e = c->self_edge();
        Mat Q = *e->A;
        std::vector<double> t(c->cols(), 0.0);
        geqrf(Q, t);
        Mat T(c->cols(), c->cols());
        larft(Q, t, T);
        Mat R(c->cols(), c->cols());
        for (int j = 0; j < c->cols(); ++j)
            for (int i = 0; i <= j; ++i) R(i, j) = Q(i, j);
        Mat& D = *e->A;
        for (int j = 0; j < D.cols; ++j)
            for (int i = 0; i < D.rows; ++i) D(i, j) = (i == j) ? 1.0 : 0.0;
        nnzR_ = (unsigned long long)((double)nnzR_ + 0.5 * c->cols() * c->cols());
        nnzH_ += (unsigned long long)(c->rows() * c->cols());
        int nrow = 0, ncol = 0, wrow = 0, hcol = 0;
        for (Edge* ei : c->edgesIn)
            if (!ei->n1->eliminated) {
                larfb_lt(Q, T, ei->A->data(), ei->A->rows, ei->A->cols);
                ++nrow;
                wrow += ei->A->cols;
            }
        for (Edge* eo : c->edgesOut)
            if (!eo->n2->eliminated && eo->n2 != c) {
                trsm_right_upper(R, *eo->A);
                ++ncol;
                hcol += eo->A->rows;
            }
        rec(2, c->rows(), c->cols(), nrow, ncol, (long long)wrow * 100000 + hcol, c->order);
        if (square_) {
            ops_.emplace_back(new OpScaleD(c, std::move(Q), std::move(t), true));
        } else {
            ops_.emplace_back(new OpScaleD(c, R, {}, false));
            tops_.emplace_back(new TOpScaleD(c, R));
        }
    }

    // -------- sparsification (src/tree.cpp:992-1114, 1260-1307, 226-247) --------
    void sparsify_extra(Cluster* c) {
        if (c->cols() == 0 || c->rows() <= c->cols()) return;
        int rows_before = c->rows();
        std::vector<Mat*> Apm;
        int spm = 0;
        for (Edge* e : c->edgesIn)
            if (!e->n1->eliminated) { Apm.push_back(e->A.get()); spm += e->A->cols; }
        Mat Apmc(c->rows(), spm);
        int cur = 0;
        for (Mat* m : Apm) { Apmc.set_block(0, cur, *m); cur += m->cols; }
        Mat rest = Apmc.block(c->cols(), 0, c->rows() - c->cols(), spm);
        int rank = c->cols(), rank_rows = 0;
        if (rest.rows > 0) {
            std::vector<int> jpvt(rest.cols, 0);
            std::vector<double> t(std::min(rest.rows, rest.cols), 0.0);
            geqp3(rest, jpvt, t);
            std::vector<double> rii(std::min(rest.rows, rest.cols));
            for (size_t q = 0; q < rii.size(); ++q) rii[q] = rest(q, q);
            rank_rows = choose_rank(rii, tol_, true);
            Mat Cr(rank_rows, rest.cols);
            for (int q = 0; q < rest.cols; ++q)
                for (int i = 0; i < rank_rows && i <= q; ++i) Cr(i, jpvt[q]) = rest(i, q);
            rest = Cr;
            rank_rows += rank;
        }
        c->reset_size(rank_rows, rank);
        Edge* es = c->self_edge();
        *es->A = es->A->top_rows(rank_rows);
        cur = 0;
        for (Mat* m : Apm) {
            int w = m->cols;
            Mat nm(c->rows(), w);
            nm.set_block(0, 0, Apmc.block(0, cur, c->cols(), w));
            nm.set_block(c->cols(), 0, rest.block(0, cur, c->rows() - c->cols(), w));
            *m = nm;
            cur += w;
        }
        rec(8, rows_before, c->rows(), 0, 0, 0, c->order);
    }

    // -------- sparsify without block scaling (--scale 0, src/tree.cpp:887-989) --------
    // C = [A_mp^T | (1/s) A_pp^T A_pm] with s the smallest singular value of
    // [A_pp; A_mp]; the RRQR's reflectors Q rotate the cluster's columns
    // (A_pp <- A_pp Q, A_mp <- its rank rows of R), the last columns and rows
    // split off into a fine cluster, which is eliminated at once.
    void sparsify(Cluster* c) {
        int cols_before = c->cols();
        if (c->cols() == 0) { rec(3, 0, 0, 0, c->rows(), 0, c->order); return; }
        std::vector<Mat*> Apm, Amp;
        Mat* App = nullptr;
        int spm = 0, smp = 0;
        for (Edge* e : c->edgesIn)
            if (!e->n1->eliminated) { Apm.push_back(e->A.get()); spm += e->A->cols; }
        for (Edge* e : c->edgesOut) {
            if (e->n2->eliminated) continue;
            if (e->n2 != c) { Amp.push_back(e->A.get()); smp += e->A->rows; }
            else App = e->A.get();
        }
        if (!App) throw std::runtime_error("sparsify: cluster without its diagonal block");
        Mat Apmc(c->rows(), spm);
        int cur = 0;
        for (Mat* m : Apm) { Apmc.set_block(0, cur, *m); cur += m->cols; }
        Mat Ap(App->rows + smp, c->cols());
        Ap.set_block(0, 0, *App);
        Mat C(c->cols(), smp + spm);
        cur = 0;
        for (Mat* m : Amp) {
            Ap.set_block(App->rows + cur, 0, *m);
            for (int j = 0; j < m->cols; ++j)
                for (int i = 0; i < m->rows; ++i) C(j, cur + i) = (*m)(i, j);
            cur += m->rows;
        }
        const std::vector<double> S = gesvd_values(Ap);
        const double sinv = 1.0 / S[std::min(Ap.rows, Ap.cols) - 1];
        for (int j = 0; j < spm; ++j)
            for (int i = 0; i < c->cols(); ++i) {
                double acc = 0;
                for (int r = 0; r < App->rows; ++r) acc += (*App)(r, i) * Apmc(r, j);
                C(i, smp + j) = sinv * acc;
            }
        std::vector<int> jpvt(C.cols, 0);
        std::vector<double> t(std::min(C.rows, C.cols), 0.0);
        geqp3(C, jpvt, t);
        std::vector<double> rii(std::min(C.rows, C.cols));
        for (size_t q = 0; q < rii.size(); ++q) rii[q] = C(q, q);
        int rank = choose_rank(rii, tol_);
        if (rank >= C.rows) { rec(3, cols_before, c->cols(), C.cols, c->rows(), 0, c->order); return; }
        Mat v = C.block(0, 0, C.rows, rank);
        std::vector<double> h(t.begin(), t.begin() + rank);
        if (App->rows > 0)  // ormqr_notrans_right (src/util.cpp:358-369): A_pp <- A_pp Q
            L().dormqr(kColMajor, 'R', 'N', App->rows, App->cols, rank, v.data(), v.rows, h.data(), App->data(),
                       App->rows);
        ops_.emplace_back(new OpOrth(c, v, h));
        const int cf_csize = c->cols() - rank;
        Cluster* cf = new_cluster(c->cstart + rank, cf_csize, c->rstart + c->rows() - cf_csize, cf_csize, c->id);
        ops_.emplace_back(new OpSplit(c, cf));
        c->reset_size(c->rows() - cf_csize, rank);
        Mat Cr(rank, C.cols);  // upper(C.topRows(rank)) * P^T
        for (int q = 0; q < C.cols; ++q)
            for (int i = 0; i < rank && i <= q; ++i) Cr(i, jpvt[q]) = C(i, q);
        cur = 0;
        for (Mat* m : Amp) {
            Mat nb(m->rows, rank);
            for (int j = 0; j < rank; ++j)
                for (int i = 0; i < m->rows; ++i) nb(i, j) = Cr(j, cur + i);
            cur += m->rows;
            *m = std::move(nb);
        }
        split_edges(c, cf);
        fine_[ilvl_].push_back(cf);
        eliminate_cluster(cf);
        rec(3, cols_before, c->cols(), C.cols, c->rows(), 0, c->order);
    }

    // split_edges (src/tree.cpp:480-530): the fine cluster takes the last rows
    // of every block in the coarse cluster's row, and the diagonal block splits
    // into [A_cc A_cf; A_fc A_ff].
    void split_edges(Cluster* c, Cluster* f) {
        for (Edge* e : c->edgesIn) {
            if (e->n1->eliminated) continue;
            const Mat& A = *e->A;
            Edge* ef = new Edge{e->n1, f, std::unique_ptr<Mat>(new Mat(A.block(A.rows - f->rows(), 0, f->rows(), A.cols)))};
            owned_edges_.insert(ef);
            *e->A = A.top_rows(c->rows());
            f->edgesIn.push_back(ef);
            f->rsparsity.insert(e->n1);
            e->n1->edgesOut.push_back(ef);
        }
        Edge* es = c->self_edge();
        if (!es) throw std::runtime_error("split_edges: cluster without its diagonal block");
        const Mat S = *es->A;
        Edge* eff = new Edge{f, f, std::unique_ptr<Mat>(new Mat(S.block(S.rows - f->rows(), S.cols - f->cols(), f->rows(), f->cols())))};
        Edge* efc = new Edge{f, c, std::unique_ptr<Mat>(new Mat(S.block(0, S.cols - f->cols(), c->rows(), f->cols())))};
        Edge* ecf = new Edge{c, f, std::unique_ptr<Mat>(new Mat(S.block(S.rows - f->rows(), 0, f->rows(), c->cols())))};
        *es->A = S.block(0, 0, c->rows(), c->cols());
        for (Edge* e : {eff, efc, ecf}) owned_edges_.insert(e);
        f->edgesOut.push_back(eff);
        f->edgesOut.push_back(efc);
        f->edgesIn.push_back(ecf);
        c->edgesOut.push_back(ecf);
        f->cnbrs.insert(c);
        f->cnbrs.insert(f);
        f->rsparsity.insert(c);
        f->edgesOut.sort([](const Edge* a, const Edge* b) { return a->n2->order > b->n2->order; });
    }

    // sparsifyD (src/tree.cpp:992-1114) and, with imp, sparsifyD_imp (order 1.5,
    // src/tree.cpp:1117-1257): the same RRQR and block rewrite; imp also keeps
    // the E2 term, (Q^T A_pm_top)(rank:, :), as edges from the neighbours into
    // the fine cluster, whose QR op subtracts it in the backward sweep.
    void sparsifyD(Cluster* c, bool imp = false) {
        int cols_before = c->cols();
        if (c->cols() == 0) { rec(3, 0, 0, 0, c->rows(), 0, c->order); return; }
        std::vector<Mat*> Apm, Amp;
        Edge* e_self = nullptr;
        int spm = 0, smp = 0;
        for (Edge* e : c->edgesIn)
            if (!e->n1->eliminated) { Apm.push_back(e->A.get()); spm += e->A->cols; }
        for (Edge* e : c->edgesOut) {
            if (!e->n2->eliminated && e->n2 != c) { Amp.push_back(e->A.get()); smp += e->A->rows; }
            else if (e->n2 == c) e_self = e;
        }
        Mat C(c->cols(), spm + smp);
        Mat Apmc(c->rows(), spm);
        int cur = 0;
        for (Mat* m : Apm) { Apmc.set_block(0, cur, *m); cur += m->cols; }
        Mat rest;
        if (!square_) rest = Apmc.block(c->cols(), 0, c->rows() - c->cols(), spm);
        Mat Apmc_top;
        if (imp) Apmc_top = Apmc.block(0, 0, c->cols(), spm);
        cur = 0;
        for (Mat* m : Amp) {
            for (int j = 0; j < m->cols; ++j)
                for (int i = 0; i < m->rows; ++i) C(j, cur + i) = (*m)(i, j);
            cur += m->rows;
        }
        for (int j = 0; j < spm; ++j)
            for (int i = 0; i < c->cols(); ++i) C(i, smp + j) = Apmc(i, j);
        std::vector<int> jpvt(C.cols, 0);
        std::vector<double> t(std::min(C.rows, C.cols), 0.0);
        geqp3(C, jpvt, t);
        std::vector<double> rii(std::min(C.rows, C.cols));
        for (size_t q = 0; q < rii.size(); ++q) rii[q] = C(q, q);
        int rank = choose_rank(rii, tol_);
        if (rank >= C.rows) { rec(3, cols_before, c->cols(), C.cols, c->rows(), 0, c->order); return; }
        Mat v = C.block(0, 0, C.rows, rank);
        std::vector<double> h(t.begin(), t.begin() + rank);
        OpOrthD* od = new OpOrthD(c, v, h);
        ops_.emplace_back(od);
        if (!square_) tops_.emplace_back(new TOpOrthD(c, &od->V, &od->tau));
        nnzQ_ += (unsigned long long)(C.rows * rank);
        int cf_cstart = c->cstart + rank;
        int cf_csize = c->cols() - rank;
        int cf_rstart = c->rstart + c->cols() - cf_csize;
        Cluster* cf = new_cluster(cf_cstart, cf_csize, cf_rstart, cf_csize, c->id);
        ops_.emplace_back(new OpSplitD(c, cf, rank));
        if (!square_) tops_.emplace_back(new TOpSplitD(c, cf, rank));
        // Crank = upper(C.topRows(rank)) * P^T
        Mat Cr(rank, C.cols);
        for (int q = 0; q < C.cols; ++q)
            for (int i = 0; i < rank && i <= q; ++i) Cr(i, jpvt[q]) = C(i, q);
        Mat selfb(c->rows() - cf_csize, rank);
        for (int j = 0; j < rank; ++j)
            for (int i = 0; i < rank; ++i) selfb(i, j) = (*e_self->A)(i, j);
        const Mat self_old = imp ? *e_self->A : Mat();
        int rank_rows = rank + rest.rows;
        c->reset_size(rank_rows, rank);
        cur = 0;
        for (Mat* m : Amp) {
            Mat nm(m->rows, rank);
            for (int j = 0; j < rank; ++j)
                for (int i = 0; i < m->rows; ++i) nm(i, j) = Cr(j, cur + i);
            cur += m->rows;
            *m = nm;
        }
        int count = cur, cc = cur;
        for (Mat* m : Apm) {
            Mat nm(c->rows(), m->cols);
            for (int j = 0; j < m->cols; ++j)
                for (int i = 0; i < c->cols(); ++i) nm(i, j) = Cr(i, cc + j);
            if (!square_)
                for (int j = 0; j < m->cols; ++j)
                    for (int i = 0; i < c->rows() - c->cols(); ++i) nm(c->cols() + i, j) = rest(i, cc - count + j);
            cc += m->cols;
            *m = nm;
        }
        if (!imp) {
            *e_self->A = selfb.top_rows(c->rows());
        } else {
            // Aff = self(0:cf, 0:cf); self = its bottom-right rows x cols corner
            Mat* Aff = new Mat(self_old.block(0, 0, cf->cols(), cf->cols()));
            *e_self->A = self_old.block(self_old.rows - c->rows(), self_old.cols - c->cols(), c->rows(), c->cols());
            Edge* eff = new Edge{cf, cf, std::unique_ptr<Mat>(Aff)};
            owned_edges_.insert(eff);
            cf->edgesOut.push_back(eff);
            // E2: rows rank.. of Q^T A_pm_top (ormqr_trans_left, src/util.cpp:331-347)
            if (spm > 0 && rank > 0)
                L().dormqr(kColMajor, 'L', 'T', Apmc_top.rows, spm, rank, v.data(), v.rows, h.data(),
                           Apmc_top.data(), Apmc_top.rows);
            int cc2 = 0;
            for (Edge* e : c->edgesIn) {
                if (e->n1->eliminated) continue;
                Cluster* mm = e->n1;
                Mat* Afm = new Mat(Apmc_top.block(rank, cc2, cf->rows(), mm->cols()));
                Edge* e2 = new Edge{mm, cf, std::unique_ptr<Mat>(Afm)};
                owned_edges_.insert(e2);
                cf->edgesIn.push_back(e2);
                mm->edgesOut.push_back(e2);
                cc2 += mm->cols();
            }
        }
        fine_[ilvl_].push_back(cf);
        if (imp) {
            const int kk = std::min(cf->rows(), cf->cols());
            cf->tau.assign(kk, 0.0);
            cf->T = Mat(kk, kk);
            ops_.emplace_back(new OpQR(cf));
            if (!square_) tops_.emplace_back(new TOpQR(cf));
        }
        cf->eliminated = true;
        rec(3, cols_before, c->cols(), C.cols, c->rows(), 0, c->order);
    }

    // -------- wave-parallel execution (CPU baseline timing only) --------
    // With threads_ > 1 the square, scaled, order-1 factorization runs each
    // level's elimination, scaling and sparsification as conflict-free waves
    // on host threads, and the solve runs its op tape the same way. A task
    // joins the wave after the last earlier task that touched any of its
    // blocks (or solution segments), so every block sees its updates in the
    // sequential order: the event log and every number are bitwise those of
    // the sequential path (tests/test_oracle_parallel.py). Graph changes (fill
    // edges, new clusters, op records, counters, log records) are made on one
    // thread in the sequential order; only the dense arithmetic is spread.
    int threads_ = 1;
    bool par_ok() const { return threads_ > 1 && square_ && scale_ && order_ != 1.5f && tol_ != 0; }

    // wave of each of n tasks; touch(i, keys) lists task i's keys (nullptr: all)
    template <class Touch>
    static std::vector<int> waves_of(int n, Touch touch) {
        std::unordered_map<const void*, int> last;
        std::vector<int> w(n);
        std::vector<const void*> keys;
        int barrier = -1, top = -1;
        for (int i = 0; i < n; ++i) {
            keys.clear();
            touch(i, keys);
            int wv = barrier + 1;
            bool all = false;
            for (const void* k : keys) {
                if (!k) { all = true; break; }
                auto it = last.find(k);
                if (it != last.end()) wv = std::max(wv, it->second + 1);
            }
            if (all) {
                wv = top + 1;
                barrier = wv;
            } else {
                for (const void* k : keys) last[k] = wv;
            }
            w[i] = wv;
            top = std::max(top, wv);
        }
        return w;
    }

    // Runs f(i) for every task, wave by wave. A wave of one task keeps the
    // BLAS thread count the caller set (orc_blas_threads), a wider wave runs
    // one BLAS thread per task. OpenBLAS's threaded kernels round differently
    // from its one-thread kernels, so the results are bitwise the sequential
    // path's when BLAS runs one thread, and agree to rounding otherwise.
    template <class F>
    void run_waves(const std::vector<int>& wave, F f) {
        int nw = 0;
        for (int v : wave) nw = std::max(nw, v + 1);
        std::vector<std::vector<int>> by(nw);
        for (int i = 0; i < (int)wave.size(); ++i) by[wave[i]].push_back(i);
        const Lapack& l = L();
        const int blas = l.get_threads ? l.get_threads() : 1;
        for (auto& g : by) {
            if (g.empty()) continue;
            if (l.set_threads && blas > 1) l.set_threads(g.size() == 1 ? blas : 1);
            pool().run((int)g.size(), threads_, [&](int q) { f(g[q]); });
        }
        if (l.set_threads && blas > 1) l.set_threads(blas);
    }

    struct ElimTask {
        Cluster* c;
        std::vector<Edge*> col;                  // stacked column blocks
        std::vector<Cluster*> upd;               // updated clusters (rsparsity order)
        std::vector<std::vector<Edge*>> blocks;  // per updated cluster: its blocks in stacking order
        int num_rows = 0, num_cols = 0;
    };

    // eliminate_cluster over the level's interiors (src/tree.cpp:780-832)
    void eliminate_level_par() {
        std::vector<ElimTask> tasks;
        for (Cluster* c : bottom_current()) {
            if (c->level() != ilvl_) continue;
            ElimTask t;
            t.c = c;
            if (c->cols() > 0) {
                for (Edge* e : c->edgesOut)
                    if (e->A) { t.col.push_back(e); t.num_rows += e->A->rows; t.num_cols = e->A->cols; }
                for (Cluster* n : c->rsparsity) {
                    if (n->eliminated || c == n) continue;
                    std::vector<Edge*> bl;
                    for (Edge* e : t.col) {
                        Edge* ecn = find_out(n, e->n2);
                        if (!ecn) ecn = add_edge(n, e->n2);
                        bl.push_back(ecn);
                    }
                    t.upd.push_back(n);
                    t.blocks.push_back(std::move(bl));
                }
            }
            c->eliminated = true;
            tasks.push_back(std::move(t));
        }
        auto wave = waves_of((int)tasks.size(), [&](int i, std::vector<const void*>& k) {
            for (Edge* e : tasks[i].col) k.push_back(e);
            for (auto& bl : tasks[i].blocks)
                for (Edge* e : bl) k.push_back(e);
        });
        run_waves(wave, [&](int i) {
            ElimTask& t = tasks[i];
            Cluster* c = t.c;
            if (c->cols() == 0) return;
            Mat Q(t.num_rows, t.num_cols);
            int cur = 0;
            for (Edge* e : t.col) { Q.set_block(cur, 0, *e->A); cur += e->A->rows; }
            int k = std::min(t.num_rows, t.num_cols);
            c->tau.assign(k, 0.0);
            c->T = Mat(k, k);
            geqrf(Q, c->tau);
            cur = 0;
            for (Edge* e : t.col) { *e->A = Q.block(cur, 0, e->A->rows, e->A->cols); cur += e->A->rows; }
            larft(Q, c->tau, c->T);
            for (size_t u = 0; u < t.upd.size(); ++u) {
                Mat V(Q.rows, t.upd[u]->cols());
                cur = 0;
                for (Edge* e : t.blocks[u]) { V.set_block(cur, 0, *e->A); cur += e->A->rows; }
                larfb_lt(Q, c->T, V.data(), V.rows, V.cols);
                cur = 0;
                for (Edge* e : t.blocks[u]) { *e->A = V.block(cur, 0, e->A->rows, e->A->cols); cur += e->A->rows; }
            }
        });
        for (ElimTask& t : tasks) {
            Cluster* c = t.c;
            if (c->cols() == 0) { rec(1, 0, 0, 0, 0, 0, c->order); continue; }
            nnzH_ += (unsigned long long)(t.num_rows * t.num_cols);
            int wtr = 0;
            for (Cluster* n : t.upd) {
                nnzR_ += (unsigned long long)(c->cols() * n->cols());
                wtr += n->cols();
            }
            ops_.emplace_back(new OpQR(c));
            rec(1, t.num_rows, t.num_cols, (long long)t.upd.size(), (long long)t.col.size(), wtr, c->order);
        }
    }

    struct ScaleTask {
        Cluster* c;
        Edge* self;
        std::vector<Edge*> rowb, colb;
        Mat Q;
        std::vector<double> tau;
        int wrow = 0, hcol = 0;
    };

    // diag_scale over the level's interfaces (src/tree.cpp:533-580), square
    void scale_level_par() {
        std::vector<ScaleTask> tasks;
        for (Cluster* c : bottom_current()) {
            if (!want_sparsify(c)) continue;
            ScaleTask t;
            t.c = c;
            t.self = c->self_edge();
            for (Edge* ei : c->edgesIn)
                if (!ei->n1->eliminated) t.rowb.push_back(ei);
            for (Edge* eo : c->edgesOut)
                if (!eo->n2->eliminated && eo->n2 != c) t.colb.push_back(eo);
            tasks.push_back(std::move(t));
        }
        auto wave = waves_of((int)tasks.size(), [&](int i, std::vector<const void*>& k) {
            k.push_back(tasks[i].self);
            for (Edge* e : tasks[i].rowb) k.push_back(e);
            for (Edge* e : tasks[i].colb) k.push_back(e);
        });
        run_waves(wave, [&](int i) {
            ScaleTask& t = tasks[i];
            Cluster* c = t.c;
            t.Q = *t.self->A;
            t.tau.assign(c->cols(), 0.0);
            geqrf(t.Q, t.tau);
            Mat T(c->cols(), c->cols());
            larft(t.Q, t.tau, T);
            Mat R(c->cols(), c->cols());
            for (int j = 0; j < c->cols(); ++j)
                for (int r = 0; r <= j; ++r) R(r, j) = t.Q(r, j);
            Mat& D = *t.self->A;
            for (int j = 0; j < D.cols; ++j)
                for (int r = 0; r < D.rows; ++r) D(r, j) = (r == j) ? 1.0 : 0.0;
            for (Edge* ei : t.rowb) {
                larfb_lt(t.Q, T, ei->A->data(), ei->A->rows, ei->A->cols);
                t.wrow += ei->A->cols;
            }
            for (Edge* eo : t.colb) {
                trsm_right_upper(R, *eo->A);
                t.hcol += eo->A->rows;
            }
        });
        for (ScaleTask& t : tasks) {
            Cluster* c = t.c;
            nnzR_ = (unsigned long long)((double)nnzR_ + 0.5 * c->cols() * c->cols());
            nnzH_ += (unsigned long long)(c->rows() * c->cols());
            rec(2, c->rows(), c->cols(), (long long)t.rowb.size(), (long long)t.colb.size(),
                (long long)t.wrow * 100000 + t.hcol, c->order);
            ops_.emplace_back(new OpScaleD(c, std::move(t.Q), std::move(t.tau), true));
        }
    }

    struct SparsTask {
        Cluster* c;
        Edge* self = nullptr;
        std::vector<Edge*> in, out;  // Apm (row blocks) and Amp (column blocks)
        int cols_before = 0, rows_before = 0, ccols = 0, rank = 0;
        bool split = false;
        Mat v;
        std::vector<double> h;
    };

    // sparsifyD over the level's interfaces (src/tree.cpp:992-1114), square, order 1
    void sparsify_level_par() {
        std::vector<SparsTask> tasks;
        for (Cluster* c : bottom_current()) {
            if (!want_sparsify(c)) continue;
            SparsTask t;
            t.c = c;
            for (Edge* e : c->edgesIn)
                if (!e->n1->eliminated) t.in.push_back(e);
            for (Edge* e : c->edgesOut) {
                if (!e->n2->eliminated && e->n2 != c) t.out.push_back(e);
                else if (e->n2 == c) t.self = e;
            }
            tasks.push_back(std::move(t));
        }
        auto wave = waves_of((int)tasks.size(), [&](int i, std::vector<const void*>& k) {
            if (tasks[i].self) k.push_back(tasks[i].self);
            for (Edge* e : tasks[i].in) k.push_back(e);
            for (Edge* e : tasks[i].out) k.push_back(e);
        });
        // numbers and this task's own blocks and sizes; ops, the fine cluster
        // and the log record follow below in task order
        run_waves(wave, [&](int i) {
            SparsTask& t = tasks[i];
            Cluster* c = t.c;
            t.cols_before = c->cols();
            t.rows_before = c->rows();
            if (c->cols() == 0) return;
            int spm = 0, smp = 0;
            for (Edge* e : t.in) spm += e->A->cols;
            for (Edge* e : t.out) smp += e->A->rows;
            Mat C(c->cols(), spm + smp);
            Mat Apmc(c->rows(), spm);
            int cur = 0;
            for (Edge* e : t.in) { Apmc.set_block(0, cur, *e->A); cur += e->A->cols; }
            cur = 0;
            for (Edge* e : t.out) {
                const Mat& m = *e->A;
                for (int j = 0; j < m.cols; ++j)
                    for (int r = 0; r < m.rows; ++r) C(j, cur + r) = m(r, j);
                cur += m.rows;
            }
            for (int j = 0; j < spm; ++j)
                for (int r = 0; r < c->cols(); ++r) C(r, smp + j) = Apmc(r, j);
            std::vector<int> jpvt(C.cols, 0);
            std::vector<double> tt(std::min(C.rows, C.cols), 0.0);
            geqp3(C, jpvt, tt);
            std::vector<double> rii(std::min(C.rows, C.cols));
            for (size_t q = 0; q < rii.size(); ++q) rii[q] = C(q, q);
            const int rank = choose_rank(rii, tol_);
            t.rank = rank;
            t.ccols = C.cols;
            if (rank >= C.rows) return;
            t.split = true;
            t.v = C.block(0, 0, C.rows, rank);
            t.h.assign(tt.begin(), tt.begin() + rank);
            Mat Cr(rank, C.cols);
            for (int q = 0; q < C.cols; ++q)
                for (int r = 0; r < rank && r <= q; ++r) Cr(r, jpvt[q]) = C(r, q);
            const int cf_csize = c->cols() - rank;
            Mat selfb(c->rows() - cf_csize, rank);
            for (int j = 0; j < rank; ++j)
                for (int r = 0; r < rank; ++r) selfb(r, j) = (*t.self->A)(r, j);
            c->reset_size(rank, rank);  // square: rank rows
            cur = 0;
            for (Edge* e : t.out) {
                Mat& m = *e->A;
                Mat nm(m.rows, rank);
                for (int j = 0; j < rank; ++j)
                    for (int r = 0; r < m.rows; ++r) nm(r, j) = Cr(j, cur + r);
                cur += m.rows;
                m = std::move(nm);
            }
            int cc = cur;
            for (Edge* e : t.in) {
                Mat& m = *e->A;
                Mat nm(c->rows(), m.cols);
                for (int j = 0; j < m.cols; ++j)
                    for (int r = 0; r < c->cols(); ++r) nm(r, j) = Cr(r, cc + j);
                cc += m.cols;
                m = std::move(nm);
            }
            *t.self->A = selfb.top_rows(c->rows());
        });
        for (SparsTask& t : tasks) {
            Cluster* c = t.c;
            if (t.cols_before == 0) { rec(3, 0, 0, 0, c->rows(), 0, c->order); continue; }
            if (!t.split) { rec(3, t.cols_before, c->cols(), t.ccols, c->rows(), 0, c->order); continue; }
            ops_.emplace_back(new OpOrthD(c, std::move(t.v), std::move(t.h), t.cols_before));
            nnzQ_ += (unsigned long long)(t.cols_before * t.rank);
            const int cf_csize = t.cols_before - t.rank;
            Cluster* cf = new_cluster(c->cstart + t.rank, cf_csize, c->rstart + t.cols_before - cf_csize, cf_csize,
                                      c->id);
            ops_.emplace_back(new OpSplitD(c, cf, t.rank, t.rows_before, t.cols_before));
            fine_[ilvl_].push_back(cf);
            cf->eliminated = true;
            rec(3, t.cols_before, c->cols(), t.ccols, c->rows(), 0, c->order);
        }
    }

    // solve tape as waves: forward ops in order, backward ops in reverse order
    std::vector<int> fwd_wave_, bwd_wave_;
    void plan_solve_waves() {
        const int n = (int)ops_.size();
        fwd_wave_ = waves_of(n, [&](int i, std::vector<const void*>& k) { ops_[i]->touch(true, k); });
        std::vector<int> b = waves_of(n, [&](int i, std::vector<const void*>& k) { ops_[n - 1 - i]->touch(false, k); });
        bwd_wave_ = b;
    }
    void solve_par(const double* bin, double* xout) {
        if (fwd_wave_.size() != ops_.size()) plan_solve_waves();
        std::vector<double> b(nrows_);
        for (int k = 0; k < nrows_; ++k) b[k] = bin[rperm_[k]];
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->rsize_org; ++i) c->x[i] = b[c->rstart + i];
        const int n = (int)ops_.size();
        run_waves(fwd_wave_, [&](int i) { ops_[i]->fwd(); });
        run_waves(bwd_wave_, [&](int i) { ops_[n - 1 - i]->bwd(); });
        std::vector<double> x(ncols_);
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->csize_org; ++i) x[c->cstart + i] = c->x[i];
        for (int k = 0; k < ncols_; ++k) xout[cperm_[k]] = x[k];
    }

    // -------- factorize (src/tree.cpp:1309-1437) --------
    void factorize() {
        double t0 = now();
        for (ilvl_ = 0; ilvl_ < nlevels_; ++ilvl_) {
            for (Cluster* s : bottom_current())
                if (s->level() == ilvl_) get_sparsity(s);
            if (par_ok()) {
                eliminate_level_par();
            } else {
                for (Cluster* s : bottom_current())
                    if (s->level() == ilvl_) eliminate_cluster(s);
            }
            if (ilvl_ < nlevels_ - 1 && !square_)
                for (Cluster* s : bottom_current())
                    if (s->eliminated) reassign_rows(s);
            if (scale_ && ilvl_ < nlevels_ - 2 && ilvl_ >= skip_ && tol_ != 0) {
                if (par_ok()) {
                    scale_level_par();
                } else {
                    for (Cluster* s : bottom_current())
                        if (want_sparsify(s)) diag_scale(s);
                }
            }
            if (ilvl_ >= skip_ && ilvl_ < nlevels_ - 2 && tol_ != 0) {
                if (scale_ && !square_)
                    for (Cluster* s : bottom_current())
                        if (want_sparsify(s)) sparsify_extra(s);
                const bool par = par_ok();
                if (par) sparsify_level_par();
                for (Cluster* s : bottom_current()) {
                    if (par || !want_sparsify(s)) continue;
                    if (scale_) sparsifyD(s, order_ == 1.5f);
                    else if (square_) sparsify(s);
                    else throw std::runtime_error("--scale 0 is restated for square systems only");
                }
            }
            if (ilvl_ < nlevels_ - 1) merge_all();
            auto ts = topsize();
            rec(5, ts.first, ts.second, (long long)bottom_current().size());
        }
        rec(6, (long long)nnzA_, (long long)nnzR_, (long long)nnzH_, (long long)nnzQ_);
        t_fact_ = now() - t0;
    }

    // -------- solves (src/tree.cpp:1440-1517) --------
    void solve(const double* bin, double* xout) {
        if (threads_ > 1 && square_) { solve_par(bin, xout); return; }
        std::vector<double> b(nrows_);
        for (int k = 0; k < nrows_; ++k) b[k] = bin[rperm_[k]];
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->rsize_org; ++i) c->x[i] = b[c->rstart + i];
        for (auto& op : ops_) op->fwd();
        for (auto it = ops_.rbegin(); it != ops_.rend(); ++it) (*it)->bwd();
        std::vector<double> x(ncols_);
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->csize_org; ++i) x[c->cstart + i] = c->x[i];
        for (int k = 0; k < ncols_; ++k) xout[cperm_[k]] = x[k];
    }

    void solve_nrml(const double* bin, double* xout) {
        std::vector<double> b(ncols_);
        for (int k = 0; k < ncols_; ++k) b[k] = bin[cperm_[k]];
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->csize_org; ++i) c->xt[i] = b[c->cstart + i];
        auto skip = [](const Op* o) {
            return !std::strcmp(o->name(), "QR") || !std::strcmp(o->name(), "ScaleD") ||
                   !std::strcmp(o->name(), "OrthogonalD");
        };
        for (auto& op : tops_) op->fwd();
        for (auto it = tops_.rbegin(); it != tops_.rend(); ++it)
            if (!skip(it->get())) (*it)->bwd();
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->rsize_org; ++i) c->x[i] = c->xt[i];
        for (auto& op : ops_)
            if (!skip(op.get())) op->fwd();
        for (auto it = ops_.rbegin(); it != ops_.rend(); ++it) (*it)->bwd();
        std::vector<double> x(ncols_);
        for (Cluster* c : bottom_original())
            for (int i = 0; i < c->csize_org; ++i) x[c->cstart + i] = c->x[i];
        for (int k = 0; k < ncols_; ++k) xout[cperm_[k]] = x[k];
    }
};

// ---------------------------------------------------------------------------
// Krylov drivers (src/is.cpp:94-345)
// ---------------------------------------------------------------------------
static void spmv(const Csc& A, const double* x, double* y) {  // y = A x
    std::fill(y, y + A.m, 0.0);
    for (int j = 0; j < A.n; ++j) {
        double xj = x[j];
        for (int q = A.p[j]; q < A.p[j + 1]; ++q) y[A.i[q]] += A.v[q] * xj;
    }
}
static void spmv_t(const Csc& A, const double* x, double* y) {  // y = A^T x
    for (int j = 0; j < A.n; ++j) {
        double s = 0;
        for (int q = A.p[j]; q < A.p[j + 1]; ++q) s += A.v[q] * x[A.i[q]];
        y[j] = s;
    }
}
static double nrm2(const std::vector<double>& v) {
    double s = 0;
    for (double a : v) s += a * a;
    return std::sqrt(s);
}

// Elementary reflector H = I - tau [1; ess][1; ess]^T with H x = [beta; 0].
// Sign convention: beta = -sign(x0) ||x||; tau = (beta - x0)/beta; ess = x(1:)/(x0 - beta).
static void make_householder(const double* x, int n, double* ess, double& tau, double& beta) {
    double tail = 0;
    for (int i = 1; i < n; ++i) tail += x[i] * x[i];
    double c0 = x[0];
    if (tail <= std::numeric_limits<double>::min()) {
        tau = 0;
        beta = c0;
        for (int i = 1; i < n; ++i) ess[i - 1] = 0;
    } else {
        beta = std::sqrt(c0 * c0 + tail);
        if (c0 >= 0) beta = -beta;
        for (int i = 1; i < n; ++i) ess[i - 1] = x[i] / (c0 - beta);
        tau = (beta - c0) / beta;
    }
}
// v <- H v for H = I - tau [1; ess][1; ess]^T (v of length n, ess of length n-1).
static void apply_householder(double* v, int n, const double* ess, double tau) {
    if (n == 1) { v[0] *= (1.0 - tau); return; }
    if (tau == 0) return;
    double tmp = v[0];
    for (int i = 1; i < n; ++i) tmp += ess[i - 1] * v[i];
    v[0] -= tau * tmp;
    for (int i = 1; i < n; ++i) v[i] -= tau * ess[i - 1] * tmp;
}
// Givens (c, s) such that [c -s; s c] [p; q] = [r; 0].
static void make_givens(double p, double q, double& c, double& s) {
    if (q == 0) { c = p < 0 ? -1 : 1; s = 0; }
    else if (p == 0) { c = 0; s = q < 0 ? 1 : -1; }
    else if (std::abs(p) > std::abs(q)) {
        double t = q / p, u = std::sqrt(1 + t * t);
        if (p < 0) u = -u;
        c = 1 / u;
        s = -t * c;
    } else {
        double t = p / q, u = std::sqrt(1 + t * t);
        if (q < 0) u = -u;
        s = -1 / u;
        c = -t * s;
    }
}
static void rot(double& a, double& b, double c, double s) {  // G^T applied: [c -s; s c]
    double x = a, y = b;
    a = c * x - s * y;
    b = s * x + c * y;
}

static int gmres(const Csc& A, const double* rhs, double* x, Tree& P, int iters, int restart, double tol,
                 double* res_out) {
    const int m = A.m;
    std::vector<double> rhsv(rhs, rhs + m);
    if (nrm2(rhsv) <= std::numeric_limits<double>::min()) {
        std::fill(x, x + m, 0.0);
        *res_out = 0;
        return 0;
    }
    const int maxIters = iters;
    int it = 0;
    std::vector<double> p0(m), r0(m), t(m), v(m), xnew(m);
    spmv(A, x, t.data());
    for (int i = 0; i < m; ++i) p0[i] = rhs[i] - t[i];
    P.solve(p0.data(), r0.data());
    double r0Norm = nrm2(r0);
    if (r0Norm == 0) { *res_out = 0; return 0; }
    std::vector<double> H((size_t)m * (restart + 1), 0.0), w(restart + 1, 0.0), tau(restart + 1, 0.0);
    std::vector<double> Gc(restart, 0.0), Gs(restart, 0.0);
    auto col = [&](int j) { return H.data() + (size_t)j * m; };
    double beta;
    make_householder(r0.data(), m, col(0) + 1, tau[0], beta);
    w[0] = beta;
    double tol_error = 0;
    for (int k = 1; k <= restart; ++k) {
        ++it;
        std::fill(v.begin(), v.end(), 0.0);
        v[k - 1] = 1.0;
        for (int i = k - 1; i >= 0; --i) apply_householder(v.data() + i, m - i, col(i) + i + 1, tau[i]);
        spmv(A, v.data(), t.data());
        P.solve(t.data(), v.data());
        for (int i = 0; i < k; ++i) apply_householder(v.data() + i, m - i, col(i) + i + 1, tau[i]);
        double tn = 0;
        for (int i = k; i < m; ++i) tn += v[i] * v[i];
        if (std::sqrt(tn) != 0.0 && k < m) {
            make_householder(v.data() + k, m - k, col(k) + k + 1, tau[k], beta);
            apply_householder(v.data() + k, m - k, col(k) + k + 1, tau[k]);
        }
        for (int i = 0; i < k - 1; ++i) rot(v[i], v[i + 1], Gc[i], Gs[i]);
        if (k < m && v[k] != 0) {
            make_givens(v[k - 1], v[k], Gc[k - 1], Gs[k - 1]);
            rot(v[k - 1], v[k], Gc[k - 1], Gs[k - 1]);
            rot(w[k - 1], w[k], Gc[k - 1], Gs[k - 1]);
        }
        for (int i = 0; i < k; ++i) col(k - 1)[i] = v[i];
        tol_error = std::abs(w[k]) / r0Norm;
        bool stop = (k == m || tol_error < tol || it == maxIters);
        if (stop || k == restart) {
            std::vector<double> y(w.begin(), w.begin() + k);
            for (int i = k - 1; i >= 0; --i) {
                double s = y[i];
                for (int j = i + 1; j < k; ++j) s -= col(j)[i] * y[j];
                y[i] = s / col(i)[i];
            }
            std::fill(xnew.begin(), xnew.end(), 0.0);
            for (int i = k - 1; i >= 0; --i) {
                xnew[i] += y[i];
                apply_householder(xnew.data() + i, m - i, col(i) + i + 1, tau[i]);
            }
            for (int i = 0; i < m; ++i) x[i] += xnew[i];
            if (stop) { *res_out = tol_error; return it; }
            k = 0;
            spmv(A, x, t.data());
            for (int i = 0; i < m; ++i) p0[i] = rhs[i] - t[i];
            P.solve(p0.data(), r0.data());
            std::fill(H.begin(), H.end(), 0.0);
            std::fill(w.begin(), w.end(), 0.0);
            std::fill(tau.begin(), tau.end(), 0.0);
            make_householder(r0.data(), m, col(0) + 1, tau[0], beta);
            w[0] = beta;
        }
    }
    *res_out = tol_error;
    return it;
}

static int cgls(const Csc& A, const double* rhs, double* x, Tree& P, int maxIters, double tol, double* res_out) {
    const int m = A.m, n = A.n;
    std::vector<double> residual(m), nr(n), tmp(m), p(n), z(n), Atb(n);
    spmv(A, x, tmp.data());
    for (int i = 0; i < m; ++i) residual[i] = rhs[i] - tmp[i];
    spmv_t(A, residual.data(), nr.data());
    spmv_t(A, rhs, Atb.data());
    double rhsNorm2 = 0;
    for (double a : Atb) rhsNorm2 += a * a;
    if (rhsNorm2 == 0) { std::fill(x, x + n, 0.0); *res_out = 0; return 0; }
    double threshold = tol * tol * rhsNorm2;
    double rn2 = 0;
    for (double a : nr) rn2 += a * a;
    if (rn2 < threshold) { *res_out = std::sqrt(rn2 / rhsNorm2); return 0; }
    P.solve_nrml(nr.data(), p.data());
    double absNew = 0;
    for (int j = 0; j < n; ++j) absNew += nr[j] * p[j];
    int i = 0;
    while (i < maxIters) {
        spmv(A, p.data(), tmp.data());
        double tn = 0;
        for (double a : tmp) tn += a * a;
        double alpha = absNew / tn;
        for (int j = 0; j < n; ++j) x[j] += alpha * p[j];
        for (int q = 0; q < m; ++q) residual[q] -= alpha * tmp[q];
        spmv_t(A, residual.data(), nr.data());
        rn2 = 0;
        for (double a : nr) rn2 += a * a;
        if (rn2 < threshold) break;
        P.solve_nrml(nr.data(), z.data());
        double absOld = absNew;
        absNew = 0;
        for (int j = 0; j < n; ++j) absNew += nr[j] * z[j];
        double beta = absNew / absOld;
        for (int j = 0; j < n; ++j) p[j] = z[j] + beta * p[j];
        i++;
    }
    *res_out = std::sqrt(rn2 / rhsNorm2);
    return i;
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C interface
// ---------------------------------------------------------------------------
using namespace orc;
struct orc_tree {
    std::unique_ptr<Tree> t;
};

template <class F>
static int guarded(F f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

extern "C" {

orc_tree* orc_create(int nlevels, int skip, double tol, int scale, float order, int square) {
    if (nlevels < 1) { g_last_error = "nlevels must be >= 1"; return nullptr; }
    orc_tree* h = new orc_tree;
    h->t.reset(new Tree(nlevels, skip));
    h->t->tol_ = tol;
    h->t->scale_ = scale;
    h->t->order_ = order;
    h->t->square_ = square;
    return h;
}
void orc_destroy(orc_tree* t) { delete t; }
const char* orc_last_error(void) { return g_last_error.c_str(); }
int orc_blas_threads(int n) {
    std::string err;
    const Lapack* l = lapack(&err);
    if (!l) { g_last_error = err; return -1; }
    if (n > 0 && l->set_threads) l->set_threads(n);
    return l->get_threads ? l->get_threads() : 1;
}
int orc_set_threads(orc_tree* t, int n) {
    if (!t || n < 1) { g_last_error = "threads must be >= 1"; return -1; }
    t->t->threads_ = n;
    return 0;
}
int orc_set_coords(orc_tree* t, int d, int n, const double* X) {
    return guarded([&] {
        t->t->d_ = d;
        t->t->X_.assign(X, X + (size_t)d * n);
    });
}
int orc_set_parts(orc_tree* t, int n, const int* parts, int numeric_fill) {
    return guarded([&] {
        t->t->parts_.assign(parts, parts + n);
        t->t->numeric_fill_ = numeric_fill != 0;
    });
}
int orc_partition(orc_tree* t, int m, int n, const int* cp, const int* ri, const double* va) {
    return guarded([&] { t->t->partition(make_csc(m, n, cp, ri, va)); });
}
int orc_assemble(orc_tree* t, int m, int n, const int* cp, const int* ri, const double* va) {
    return guarded([&] { t->t->assemble(make_csc(m, n, cp, ri, va)); });
}
int orc_factorize(orc_tree* t) {
    return guarded([&] { t->t->factorize(); });
}
int orc_solve(orc_tree* t, const double* b, double* x) {
    return guarded([&] { t->t->solve(b, x); });
}
int orc_solve_nrml(orc_tree* t, const double* b, double* x) {
    return guarded([&] { t->t->solve_nrml(b, x); });
}
int orc_get_perm(orc_tree* t, int* cperm, int* rperm) {
    std::copy(t->t->cperm_.begin(), t->t->cperm_.end(), cperm);
    std::copy(t->t->rperm_.begin(), t->t->rperm_.end(), rperm);
    return 0;
}
long long orc_log_size(orc_tree* t) { return (long long)t->t->log_.size(); }
int orc_get_log(orc_tree* t, long long* out) {
    std::copy(t->t->log_.begin(), t->t->log_.end(), out);
    return 0;
}
int orc_num_bottom(orc_tree* t) { return (int)t->t->bottoms_[0].size(); }
int orc_get_bottom(orc_tree* t, int* out) {
    for (Cluster* c : t->t->bottoms_[0]) {
        int r[10] = {c->cstart, c->csize_org, c->rstart, c->rsize_org, c->id.self.lvl,
                     c->id.self.sep, c->id.l.lvl, c->id.l.sep, c->id.r.lvl, c->id.r.sep};
        std::copy(r, r + 10, out);
        out += 10;
    }
    return 0;
}
int orc_get_times(orc_tree* t, double* out) {
    out[0] = t->t->t_part_;
    out[1] = t->t->t_asm_;
    out[2] = t->t->t_fact_;
    return 0;
}
int orc_gmres(orc_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* b,
              double* x, int iters, int restart, double tol, int* its, double* res) {
    return guarded([&] {
        Csc A = make_csc(m, n, cp, ri, va);
        *its = gmres(A, b, x, *t->t, iters, restart, tol, res);
    });
}
int orc_cgls(orc_tree* t, int m, int n, const int* cp, const int* ri, const double* va, const double* b,
             double* x, int iters, double tol, int* its, double* res) {
    return guarded([&] {
        Csc A = make_csc(m, n, cp, ri, va);
        *its = cgls(A, b, x, *t->t, iters, tol, res);
    });
}
int orc_dgeqrf(int m, int n, double* a, int lda, double* tau) {
    return guarded([&] { L().dgeqrf(kColMajor, m, n, a, lda, tau); });
}
int orc_dlarft(int m, int k, const double* v, int ldv, const double* tau, double* t, int ldt) {
    return guarded([&] { L().dlarft(kColMajor, 'F', 'C', m, k, v, ldv, tau, t, ldt); });
}
int orc_dlarfb_lt(int m, int n, int k, const double* v, int ldv, const double* t, int ldt, double* c, int ldc) {
    return guarded([&] { L().dlarfb(kColMajor, 'L', 'T', 'F', 'C', m, n, k, v, ldv, t, ldt, c, ldc); });
}
int orc_dgeqp3(int m, int n, double* a, int lda, int* jpvt, double* tau) {
    return guarded([&] {
        L().dgeqp3(kColMajor, m, n, a, lda, jpvt, tau);
        for (int j = 0; j < n; ++j) jpvt[j]--;
    });
}
int orc_choose_rank(const double* rii, int n, double tol) {
    std::vector<double> s(rii, rii + n);
    return choose_rank(s, tol);
}

}  // extern "C"
