// Host symbolic layer: sparse patterns, separator/cluster identifiers, the
// geometric nested-dissection ordering (bit-exact with the reference's) and the
// ordering without coordinates (src/partition.cpp, src/tree.cpp:46-163,
// include/cluster.h:22-111).
#pragma once
#include <cstdint>
#include <vector>

namespace spq {

// Compressed-column matrix with sorted row indices (Eigen::SparseMatrix layout).
struct Csc {
    int m = 0, n = 0;
    std::vector<int> p, i;
    std::vector<double> v;
};

Csc csc_from(int m, int n, const int* colptr, const int* rowind, const double* val);
Csc csc_transpose(const Csc& A);
// B[:, k] = A[:, perm[k]] (the effect of col_perm, src/util.cpp:912-940).
Csc csc_gather_cols(const Csc& A, const std::vector<int>& perm);
// B[k, :] = A[perm[k], :].
Csc csc_gather_rows(const Csc& A, const std::vector<int>& perm);

// Separator id (lvl, sep); lvl = -1 is "unset".
struct Sep {
    int lvl = -1, sep = 0;
    Sep() = default;
    Sep(int l, int s) : lvl(l), sep(s) {}
    bool operator==(const Sep& o) const { return lvl == o.lvl && sep == o.sep; }
    bool operator!=(const Sep& o) const { return !(*this == o); }
    bool operator<(const Sep& o) const { return lvl != o.lvl ? lvl < o.lvl : sep < o.sep; }
};

// Cluster id: the separator it lives on and the two sides of the interface.
// Ordering key (self, l, r, section, part) as in include/cluster.h:104-110.
struct Cid {
    Sep self, l, r;
    int part = 2, section = 0;
    bool operator==(const Cid& o) const {
        return self == o.self && l == o.l && r == o.r && part == o.part && section == o.section;
    }
    bool operator!=(const Cid& o) const { return !(*this == o); }
    bool operator<(const Cid& o) const {
        if (self != o.self) return self < o.self;
        if (l != o.l) return l < o.l;
        if (r != o.r) return r < o.r;
        if (section != o.section) return section < o.section;
        return part < o.part;
    }
};

// One step up the separator tree (src/cluster.cpp:19-32).
Cid lift(const Cid& c, int lvl);

struct Ordering {
    std::vector<int> cperm, rperm;  // new position k holds original column/row cperm[k]/rperm[k]
    std::vector<Cid> cid_of_pos;    // cluster id of permuted column k
    std::vector<int> rows_of_col;   // rows attached to permuted column k (1 for square input)
};

// Geometric nested dissection on A^T A followed by the interface inference on A
// and the hierarchical column sort. X is d x n column-major (column j = the
// coordinates of unknown j). With square set (identity row matching, m == n)
// the rows follow the columns; otherwise every row joins the first column of
// its largest-norm run of equal cluster ids (src/tree.cpp:100-163).
Ordering geometric_ordering(const Csc& A, int nlevels, int d, const std::vector<double>& X, bool square = true);

// Ordering without coordinates. graph_bisection splits the A^T A graph
// recursively into 2^(nlevels-1) leaf parts (this library's own partitioner,
// standing in for METIS_PartGraphRecursive at src/partition.cpp:354-372); the
// leaf index holds the cuts from the top, first cut in the highest bit.
// graph_ordering turns any such part vector (this one, or one computed by
// METIS) into separators, interfaces and the permutations exactly as the
// reference's MetisPartition (src/partition.cpp:374-426) followed by
// getInterfacesUsingATA (src/partition.cpp:628-675) and Tree::partition.
std::vector<int> graph_bisection(const Csc& A, int nlevels);
Ordering graph_ordering(const Csc& A, int nlevels, const std::vector<int>& parts, bool square = true);

}  // namespace spq
