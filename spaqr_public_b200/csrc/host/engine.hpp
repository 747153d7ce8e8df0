// The spaQR factorization engine of one handle: the reference's cluster/edge
// graph kept on the host (symbolic, bit-exact), dense blocks in device memory,
// and every numerical step issued as batched sm_100a kernels.
//
// Reference map:
//   Tree state and API                  include/tree.h:36-152
//   partition / assemble                src/tree.cpp:595-778
//   get_sparsity / check_if_valid       src/tree.cpp:168-224, 834-870
//   eliminate_cluster / update_cluster  src/tree.cpp:263-316, 780-832
//   diagScale                           src/tree.cpp:533-580
//   sparsifyD                           src/tree.cpp:992-1114
//   merge_all / update_size / edges     src/tree.cpp:414-475, 872-881
//   factorize                           src/tree.cpp:1309-1437
//   solve                               src/tree.cpp:1440-1466, src/operations.cpp
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <set>
#include <string>
#include <vector>

#include "../kernels/kernels.hpp"
#include "device.hpp"
#include "symbolic.hpp"

namespace spq {

struct Config {
    int nlevels = 0, skip = 0, scale = 0, square = 0;
    double tol = 0;
    float order = 1.0f;
    int hsl = 0, verbose = 0, device = 0;
    int d = 0;
    std::vector<double> X;
    // Leaf part of every column for the ordering without coordinates (empty:
    // graph_bisection computes it); ignored when coordinates are set.
    std::vector<int> parts;
    // Ordering without coordinates: the reference's numeric fill test (a fill
    // candidate is kept only if ||A1^T A2|| > 1e-14, src/tree.cpp:856-859);
    // 0 keeps every candidate that passes the separator tests.
    int numeric_fill = 1;
};

// Event log record: [type, ilvl, order, a, b, c, d, e] (same layout as the
// CPU oracle): 1 ELIM, 2 SCALE, 3 SPARS, 4 MERGE, 5 LEVEL, 6 FINAL.
using Log = std::vector<long long>;

// Kernel families timed when profiling is on.
enum KernelFamily {
    KF_COPY = 0,      // batched block gather / scatter / merge copies
    KF_PANEL = 1,     // Householder panel factorization
    KF_TRAILING = 2,  // compact-WY trailing update
    KF_TRSM = 3,      // right triangular solve (scaling)
    KF_RRQR = 4,      // truncated column-pivoted QR (sparsification)
    KF_SPARS_WB = 5,  // sparsification write-back + T factors
    KF_ASSEMBLE = 6,  // value scatter into blocks
    KF_SOLVE = 7,     // one preconditioner application (CUDA graph of sweep waves)
    kNumFamilies = 8
};
struct KernelStat {
    long long launches = 0;
    double ms = 0, flops = 0, bytes = 0;  // summed over launches; flops/bytes algorithmic
};

class EngineBase {
public:
    virtual ~EngineBase() = default;
    virtual void set_profile(int level) = 0;  // 0 off, 1 per-family timing, 2 plus a launch timeline
    virtual KernelStat kernel_stat(int family) = 0;
    virtual void reset_kernel_stats() = 0;
    virtual void partition(const Csc& A) = 0;
    virtual void assemble(const Csc& A) = 0;
    virtual void factorize() = 0;
    virtual void solve_dev(const double* d_b, double* d_x) = 0;
    // y = M^T g with M the preconditioner of solve_dev (adjoint sweeps)
    virtual void solve_adjoint_dev(const double* d_g, double* d_y) = 0;
    // x = M_n b, M_n ~ (A^T A)^{-1} of a least-squares factorization (b, x of length n)
    virtual void solve_nrml_dev(const double* d_b, double* d_x) = 0;
    virtual bool least_squares() const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual const Log& log() const = 0;
    virtual const std::vector<int>& cperm() const = 0;
    virtual const std::vector<int>& rperm() const = 0;
    virtual int nrows() const = 0;
    virtual int ncols() const = 0;
    virtual bool factorized() const = 0;
    virtual std::vector<int> bottom_info() const = 0;
    virtual void stats(double* times, long long* counters) const = 0;
    virtual std::vector<double> level_times() const = 0;
    // Host side of the last factorize, seconds: [wall, waits for the device
    // readbacks (ranks, row norms), device allocations of the arenas, scratch
    // growth, solve-plan build, then the host time of each level phase summed
    // over levels: fill, elimination, row shift, scaling, sparsification,
    // merge] (waits and allocations are part of the phase times)
    virtual std::vector<double> host_times() const = 0;
    // One preconditioner application outside the CUDA graph with every sweep
    // wave timed: returns [ms, ops, smem elements] per wave (forward waves then
    // backward waves).
    virtual std::vector<double> profile_solve_waves() = 0;
    // True once the preconditioner's solve graph exists (built by the first
    // application); from then on an application allocates nothing.
    virtual bool solve_ready() = 0;  // the solve graph exists (waits for a capture in flight)
    // Device workspace of at least `elems` doubles on the handle's stream for a
    // Krylov solve (the factorization's scratch buffer, idle between
    // factorizations): valid until the next call or factorization.
    virtual double* krylov_workspace(size_t elems) = 0;
};

std::unique_ptr<EngineBase> make_engine(const Config& cfg, int precision);

}  // namespace spq
