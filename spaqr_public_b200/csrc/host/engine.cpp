// spaQR engine: host symbolic graph + batched device numerics. See engine.hpp
// for the reference map. The symbolic steps are performed in the reference's
// order on the host; the numerical work of each phase is collected into tasks,
// grouped into waves of tasks that touch disjoint blocks (so that running a
// wave concurrently gives the same result as the reference's sequential loop),
// and issued as batched kernels on the handle's stream.
#include "engine.hpp"
#include "krylov.hpp"

#include "autotune.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <exception>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <pthread.h>
#include <thread>
#include <unordered_map>

namespace spq {
namespace {

double wall() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline int npanels(int k) { return (k + kNB - 1) / kNB; }

// Grow-only storage with stable element addresses, in chunks of 4096 elements
// (a std::deque allocates one small block per few elements, which made the
// 189k fill blocks of a level cost a malloc each ten).
template <class E>
class ChunkedStore {
public:
    static constexpr size_t kChunk = 4096;
    size_t size() const { return n_; }
    E& operator[](size_t i) { return chunks_[i / kChunk][i % kChunk]; }
    E& back() { return (*this)[n_ - 1]; }
    void push_back(const E& e) {
        resize(n_ + 1);
        back() = e;
    }
    void resize(size_t n) {  // grows only
        while (chunks_.size() * kChunk < n) chunks_.emplace_back(new E[kChunk]);
        n_ = std::max(n_, n);
    }

private:
    std::vector<std::unique_ptr<E[]>> chunks_;
    size_t n_ = 0;
};

// Host worker threads for the engine's parallel passes, started once per
// process (a factorization makes hundreds of short passes, and starting
// threads for each costs 10-20 us per thread). One pass at a time: a pass
// submitted while another holds the pool (a second handle, the backward
// schedule's thread) runs its chunks on the calling thread, with the same
// chunk boundaries, so results do not depend on which thread ran a chunk. A
// child process forked after the workers started has none of them and runs
// every pass on its own thread.
class HostPool {
public:
    static HostPool& get() {
        static HostPool* p = new HostPool();  // never destroyed: the workers live until exit
        return *p;
    }
    // Calls body(t) for t in [0, nt) on the caller and the workers and returns
    // when all have returned; false (nothing called) if the pool is busy.
    bool run(size_t nt, const std::function<void(size_t)>& body) {
        if (forked_ || workers_ == 0) return false;
        std::unique_lock<std::mutex> busy(submit_, std::try_to_lock);
        if (!busy.owns_lock()) return false;
        Job job{&body, nt};
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &job;
            ++gen_;
        }
        cv_.notify_all();
        work(job);
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [&] { return job.done.load() == nt && job.active == 0; });
        job_ = nullptr;
        return true;
    }

private:
    struct Job {
        const std::function<void(size_t)>* body;
        size_t nt;
        std::atomic<size_t> next{0}, done{0};
        int active = 0;  // workers inside work(), under mu_
    };
    HostPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        workers_ = std::min(hw, 8u) - 1;
        for (unsigned i = 0; i < workers_; ++i) std::thread([this] { loop(); }).detach();
        pthread_atfork(nullptr, nullptr, [] { get().forked_ = true; });
    }
    void work(Job& j) {
        for (size_t t; (t = j.next.fetch_add(1)) < j.nt;) {
            (*j.body)(t);
            if (j.done.fetch_add(1) + 1 == j.nt) {
                std::lock_guard<std::mutex> g(mu_);
                done_cv_.notify_all();
            }
        }
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            Job* j;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return job_ != nullptr && gen_ != seen; });
                seen = gen_;
                j = job_;
                ++j->active;
            }
            work(*j);
            std::lock_guard<std::mutex> g(mu_);
            if (--j->active == 0) done_cv_.notify_all();
        }
    }
    unsigned workers_ = 0;
    bool forked_ = false;
    std::mutex submit_, mu_;
    std::condition_variable cv_, done_cv_;
    Job* job_ = nullptr;
    unsigned long long gen_ = 0;
};

// Greedy wave assignment in list order: a task runs one wave after the last
// task that touched any of its blocks.
std::vector<int> assign_waves(const std::vector<std::vector<int>>& touched, int nuid, int* nwaves) {
    std::vector<int> last(nuid, -1), wave(touched.size(), 0);
    int nw = 0;
    for (size_t t = 0; t < touched.size(); ++t) {
        int w = 0;
        for (int u : touched[t]) w = std::max(w, last[u] + 1);
        for (int u : touched[t]) last[u] = w;
        wave[t] = w;
        nw = std::max(nw, w + 1);
    }
    *nwaves = nw;
    return wave;
}

template <class T>
class Engine final : public EngineBase {
public:
    struct Cluster;
    struct Blk {
        T* p = nullptr;
        int ld = 0, rows = 0, cols = 0, uid = -1;
    };
    struct Edge {
        Cluster* n1;
        Cluster* n2;
        Blk A;
        bool live = true;
    };
    struct ByOrder {
        bool operator()(const Cluster* a, const Cluster* b) const { return a->order < b->order; }
    };
    struct Cluster {
        int cstart, csize, rstart, rsize;
        Cid id;
        int order;
        bool elim = false;
        int csize_org, rsize_org;
        Cluster* parent = nullptr;
        Cid parentid;
        int rposparent = 0, cposparent = 0;
        std::vector<Cluster*> children;
        std::vector<Cluster*> rsparsity;  // by order
        std::vector<Edge*> out, in;
        int xcap = 0;
        int64_t xoff = -1;
        int pos = -1;  // scratch: position in the current cluster list during a host pass
        int level() const { return id.self.lvl; }
    };
    enum TapeKind { TK_QR, TK_SCALED, TK_ORTHD, TK_SPLITD, TK_MERGE, TK_REASSIGN, TK_ORTH, TK_SPLIT0 };
    struct A12 {
        const T* B;
        int ld, s;
        Cluster* n1;
    };
    struct TapeOp {
        TapeKind kind;
        Cluster* c = nullptr;
        Cluster* f = nullptr;
        const T* fac = nullptr;
        const T* tp = nullptr;
        const T* rinv = nullptr;  // R^-1 (k x k) of a QR / ScaleD op, formed after the factorization
        const T* qt = nullptr;    // Q^T (m x m) of a ScaleD op, formed after the factorization
        int m = 0, k = 0, ld = 0;
        std::vector<std::pair<Cluster*, int>> segs;
        std::vector<A12> a12;
        int crows = 0, ccols = 0, rank = 0;
        std::vector<int> idx;  // TK_REASSIGN: positions in c's segment; f = destination, m = its start
    };

    // The host symbolic steps (partition) need no GPU; the device is opened by
    // the first step that uses it (assemble).
    Engine(const Config& cfg) : cfg_(cfg), bottoms_(std::max(cfg.nlevels, 1)), fine_(std::max(cfg.nlevels, 1)) {}
    ~Engine() override {
        if (!stream_) return;
        cudaSetDevice(cfg_.device);
        try {
            finish_capture();
        } catch (...) {
        }
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (graph_) cudaGraphDestroy(graph_);
        if (adj_exec_) cudaGraphExecDestroy(adj_exec_);
        if (adj_graph_) cudaGraphDestroy(adj_graph_);
        if (nrml_exec_) cudaGraphExecDestroy(nrml_exec_);
        if (nrml_graph_) cudaGraphDestroy(nrml_graph_);
        for (auto& e : events_) cudaEventDestroy(e);
        cudaStreamSynchronize(stream_);
        arena_.release();
        desc_arena_.release();
        scratch_.hand_off(stream_);
        cudaStreamSynchronize(stream_);
        for (Lanes* ln : {&lanes_, &cap_lanes_}) {
            if (ln->side) cudaStreamDestroy(ln->side);
            if (ln->side2) cudaStreamDestroy(ln->side2);
            if (ln->fork) cudaEventDestroy(ln->fork);
            if (ln->join) cudaEventDestroy(ln->join);
            if (ln->join2) cudaEventDestroy(ln->join2);
        }
        if (cap_lanes_.main) cudaStreamDestroy(cap_lanes_.main);
        for (int i = 0; i < kRqSide; ++i) {
            if (rq_side_[i]) cudaStreamDestroy(rq_side_[i]);
            if (rq_join_[i]) cudaEventDestroy(rq_join_[i]);
        }
        if (rq_fork_) cudaEventDestroy(rq_fork_);
        cudaStreamDestroy(stream_);
    }
    void open_device() {
        if (stream_) return;
        cuda_check(cudaSetDevice(cfg_.device), "cudaSetDevice");
        cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        lanes_.main = stream_;
        cuda_check(cudaStreamCreateWithFlags(&cap_lanes_.main, cudaStreamNonBlocking), "cudaStreamCreate");
        for (Lanes* ln : {&lanes_, &cap_lanes_}) {
            cuda_check(cudaStreamCreateWithFlags(&ln->side, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaStreamCreateWithFlags(&ln->side2, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&ln->fork, cudaEventDisableTiming), "event");
            cuda_check(cudaEventCreateWithFlags(&ln->join, cudaEventDisableTiming), "event");
            cuda_check(cudaEventCreateWithFlags(&ln->join2, cudaEventDisableTiming), "event");
        }
        cuda_check(cudaEventCreateWithFlags(&rq_fork_, cudaEventDisableTiming), "event");
        for (int i = 0; i < kRqSide; ++i) {
            cuda_check(cudaStreamCreateWithFlags(&rq_side_[i], cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&rq_join_[i], cudaEventDisableTiming), "event");
        }
        cudaMemPool_t pool = device_pool(cfg_.device);
        arena_.set_stream(stream_, pool);
        desc_arena_.set_stream(stream_, pool);
        scratch_.set_pool(pool, cfg_.device);
        prepare_kernels<T>();
        // The no-allocation GMRES must not make the driver place anything on
        // the device when it runs: with lazy module loading the fixed
        // workspace array and the Krylov kernels would otherwise be loaded
        // (device memory taken) by its first call. Bind time loads both.
        prepare_krylov_kernels();
        double* ws = nullptr;
        size_t ws_elems = 0;
        cuda_check(noalloc_scratch(&ws, &ws_elems), "no-allocation workspace address");
    }

    cudaStream_t stream() const override { return stream_; }
    const Log& log() const override { return log_; }
    const std::vector<int>& cperm() const override { return cperm_; }
    const std::vector<int>& rperm() const override { return rperm_; }
    int nrows() const override { return nrows_; }
    int ncols() const override { return ncols_; }
    bool factorized() const override { return factorized_; }

    // ------------------------------------------------------------- partition
    void partition(const Csc& A) override {
        double t0 = wall();
        if (A.m < A.n) throw std::invalid_argument("need rows >= cols");
        if (cfg_.square && A.m != A.n) throw std::invalid_argument("square (identity matching) needs m == n");
        nrows_ = A.m;
        ncols_ = A.n;
        rect_ = !cfg_.square;
        geo_ = !cfg_.X.empty();
        Ordering o = geo_ ? geometric_ordering(A, cfg_.nlevels, cfg_.d, cfg_.X, cfg_.square != 0)
                          : graph_ordering(A, cfg_.nlevels,
                                           cfg_.parts.empty() ? graph_bisection(A, cfg_.nlevels) : cfg_.parts,
                                           cfg_.square != 0);
        cperm_ = o.cperm;
        rperm_ = o.rperm;
        const int c = A.n;
        int k = 0, l = 0;
        while (k < c) {
            int kn = k + 1;
            const Cid cid = o.cid_of_pos[k];
            int nr = o.rows_of_col[k];
            while (kn < c && o.cid_of_pos[kn] == cid) { nr += o.rows_of_col[kn]; ++kn; }
            bottoms_[0].push_back(new_cluster(k, kn - k, l, nr, cid));
            k = kn;
            l += nr;
        }
        if (l != A.m) throw std::runtime_error("partition: row count mismatch");
        for (int lvl = 1; lvl < cfg_.nlevels; ++lvl) {
            auto& prev = bottoms_[lvl - 1];
            size_t b = 0;
            while (b < prev.size() && prev[b]->level() < lvl) ++b;
            for (size_t i = b; i < prev.size(); ++i) prev[i]->parentid = lift(prev[i]->id, lvl);
            for (size_t i = b; i < prev.size();) {
                const Cid pid = prev[i]->parentid;
                std::vector<Cluster*> ch{prev[i]};
                int cs = prev[i]->csize, rs = prev[i]->rsize, c0 = prev[i]->cstart, r0 = prev[i]->rstart;
                ++i;
                while (i < prev.size() && prev[i]->parentid == pid) {
                    ch.push_back(prev[i]);
                    cs += prev[i]->csize;
                    rs += prev[i]->rsize;
                    ++i;
                }
                Cluster* p = new_cluster(c0, cs, r0, rs, pid);
                for (Cluster* x : ch) {
                    x->parent = p;
                    p->children.push_back(x);
                }
                bottoms_[lvl].push_back(p);
            }
        }
        t_part_ = wall() - t0;
    }

    // ------------------------------------------------------------- assemble
    void assemble(const Csc& A) override {
        double t0 = wall();
        if (bottoms_[0].empty()) throw std::logic_error("assemble before partition");
        open_device();
        nnzA_ = A.i.size();
        // permuted matrix: its column k is column cperm_[k] of A, row irow[r] is row r of A
        std::vector<int> irow(A.m);
        for (int k = 0; k < A.m; ++k) irow[rperm_[k]] = k;
        std::vector<Cluster*> rowcl(A.m);
        for (Cluster* s : bottoms_[0])
            for (int i = s->rstart; i < s->rstart + s->rsize; ++i) rowcl[i] = s;
        // (this thread, cluster order) each bottom cluster's row-cluster
        // neighbours by order, their blocks and edges
        const auto& B = bottoms_[0];
        const size_t nb = B.size();
        std::vector<size_t> first(nb + 1, 0);
        std::vector<std::vector<std::pair<Cluster*, Blk>>> nblk(nb);
        std::vector<Cluster*> cn;
        for (size_t s = 0; s < nb; ++s) {
            Cluster* self = B[s];
            cn.clear();
            size_t cnt = 0;
            for (int j = self->cstart; j < self->cstart + self->csize; ++j) {
                const int oc = cperm_[j];
                for (int q = A.p[oc]; q < A.p[oc + 1]; ++q) cn.push_back(rowcl[irow[A.i[q]]]);
                cnt += (size_t)(A.p[oc + 1] - A.p[oc]);
            }
            cn.push_back(self);
            std::sort(cn.begin(), cn.end(), ByOrder());
            cn.erase(std::unique(cn.begin(), cn.end()), cn.end());
            for (Cluster* nbr : cn) {
                Blk b = new_block(nbr->rsize, self->csize);
                nblk[s].emplace_back(nbr, b);
                Edge* e = new_edge(self, nbr, b);
                self->out.push_back(e);
                if (self != nbr) nbr->in.push_back(e);
            }
            first[s + 1] = first[s] + cnt;
        }
        // (threads) the block address and value of every entry, straight into
        // pinned staging; the scatter is a permutation, so the order is free
        const size_t nnz = first[nb];
        char* h = pinned_.get(std::max<size_t>(nnz, 1) * 16);
        uint64_t* haddr = reinterpret_cast<uint64_t*>(h);
        double* hvals = reinterpret_cast<double*>(h + std::max<size_t>(nnz, 1) * 8);
        host_parallel_for(
            nb,
            [&](size_t b0, size_t e0) {
                for (size_t s = b0; s < e0; ++s) {
                    const Cluster* self = B[s];
                    const auto& nbl = nblk[s];
                    size_t o = first[s];
                    for (int col = 0; col < self->csize; ++col) {
                        const int oc = cperm_[self->cstart + col];
                        for (int q = A.p[oc]; q < A.p[oc + 1]; ++q) {
                            const int r = irow[A.i[q]];
                            const Cluster* nbr = rowcl[r];
                            size_t u = 0;
                            while (nbl[u].first != nbr) ++u;
                            const Blk& b = nbl[u].second;
                            haddr[o] = reinterpret_cast<uint64_t>(b.p + (r - nbr->rstart) + (size_t)col * b.ld);
                            hvals[o] = A.v[q];
                            ++o;
                        }
                    }
                }
            },
            64);
        if (nnz > 0) {
            uint64_t* d_addr = desc_arena_.alloc_n<uint64_t>(nnz);
            double* d_vals = desc_arena_.alloc_n<double>(nnz);
            cuda_check(cudaMemcpyAsync(d_addr, haddr, nnz * 8, cudaMemcpyHostToDevice, stream_), "upload");
            cuda_check(cudaMemcpyAsync(d_vals, hvals, nnz * 8, cudaMemcpyHostToDevice, stream_), "upload");
            timed(KF_ASSEMBLE, 0, (double)nnz * (16 + sizeof(T)),
                  [&] { launch_scatter_values<T>(d_addr, d_vals, (int64_t)nnz, stream_); });
            ++launches_fact_;
        }
        cuda_check(cudaStreamSynchronize(stream_), "assemble");
        pinned_.reset();
        assembled_ = true;
        t_asm_ = wall() - t0;
    }

    // ------------------------------------------------------------- factorize
    void factorize() override {
        if (!assembled_) throw std::logic_error("factorize before assemble");
        if (factorized_) throw std::logic_error("factorize called twice");
        if (cfg_.order != 1.0f && cfg_.order != 1.5f)
            throw std::invalid_argument("--order must be 1 or 1.5");
        if (!cfg_.scale && cfg_.tol != 0 && rect_)
            throw std::invalid_argument("--scale 0 is supported for square systems only");
        double t0 = wall();
        launches_fact_ = 0;
        t_rank_wait_ = 0;
        for (double& x : t_phase_) x = 0;
        alloc0_ = arena_.alloc_seconds() + desc_arena_.alloc_seconds();
        grow0_ = scratch_.grow_seconds();
        const int L = cfg_.nlevels;
        // numeric status word of this factorization (zeroed arena memory):
        // the QR and RRQR kernels OR kStat* bits into it
        d_status_ = arena_.template alloc_n<int>(1);
        level_ev_.assign((size_t)L * 7, nullptr);
        for (auto& e : level_ev_) {
            cuda_check(cudaEventCreate(&e), "event");
            events_.push_back(e);
        }
        for (ilvl_ = 0; ilvl_ < L; ++ilvl_) {
            cudaEvent_t* ev = &level_ev_[(size_t)ilvl_ * 7];
            cudaEventRecord(ev[0], stream_);
            double th = wall();
            auto lap = [&](int k) {
                const double now = wall();
                t_phase_[k] += now - th;
                th = now;
            };
            std::vector<Cluster*> fill;
            for (Cluster* s : cur())
                if (s->level() == ilvl_) fill.push_back(s);
            // (threads) each cluster's fill set reads the graph and writes only its own set
            const bool numeric = !geo_ && cfg_.numeric_fill;
            std::vector<std::vector<FillCand>> cand(numeric ? fill.size() : 0);
            host_parallel_for(
                fill.size(),
                [&](size_t b, size_t e) {
                    for (size_t i = b; i < e; ++i) get_sparsity(fill[i], numeric ? &cand[i] : nullptr);
                },
                16);
            if (numeric) numeric_fill(fill, cand);
            const size_t nfill = fill.size();
            if (cfg_.verbose >= 3)
                std::fprintf(stderr, "[lvl %d] fill host: %zu of %zu clusters, %.2f ms\n", ilvl_, nfill, cur().size(),
                             (wall() - th) * 1e3);
            lap(0);
            cudaEventRecord(ev[1], stream_);
            phase_ = 1;
            elim_phase();
            lap(1);
            cudaEventRecord(ev[2], stream_);
            if (rect_ && ilvl_ < L - 1) reassign_phase();
            lap(2);
            cudaEventRecord(ev[3], stream_);  // shift (rectangular only)
            phase_ = 3;
            const bool window = ilvl_ < L - 2 && ilvl_ >= cfg_.skip && cfg_.tol != 0;
            if (cfg_.scale && window) scale_phase();
            lap(3);
            cudaEventRecord(ev[4], stream_);
            phase_ = 4;
            if (rect_ && cfg_.scale && window) extra_phase();
            if (window) {
                if (cfg_.scale)
                    sparsify_phase();
                else
                    sparsify0_phase();
            }
            lap(4);
            cudaEventRecord(ev[5], stream_);
            phase_ = 5;
            if (ilvl_ < L - 1) merge_all();
            lap(5);
            cudaEventRecord(ev[6], stream_);
            auto ts = topsize();
            rec(5, ts.first, ts.second, (long long)cur().size());
            if (cfg_.verbose) print_level(ev, ts);
        }
        rec(6, (long long)nnzA_, (long long)nnzR_, (long long)nnzH_, (long long)nnzQ_);
        const double tp0 = wall();
        phase_ = 6;
        build_solve_plan();
        t_plan_ = wall() - tp0;
        int status = 0;
        cuda_check(cudaMemcpyAsync(&status, d_status_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "status");
        cuda_check(cudaStreamSynchronize(stream_), "factorize");
        status_ = status;
        pinned_.reset();
        factorized_ = true;
        t_fact_ = wall() - t0;
        if (status) {
            std::string what = "numeric failure in the factorization:";
            if (status & kStatNonFinite) what += " a QR or RRQR pivot is NaN or Inf (non-finite values in A or in a factor)";
            if (status & kStatRRQRNaN) what += "; a sparsification met columns without a finite norm";
            if (status & kStatZeroPivot) what += (status & kStatNonFinite) ? ";" : "";
            if (status & kStatZeroPivot) what += " an elimination or scaling QR has an exactly zero pivot (singular block)";
            throw std::runtime_error(what);
        }
        if (cfg_.verbose) {
            std::printf("Tolerance set: %.3e\nTime to factorize:  %.3e\n", cfg_.tol, t_fact_);
            std::printf("Size of top separator: %d\n", bottoms_[L - 1].empty() ? 0 : bottoms_[L - 1].front()->csize);
            std::printf("nnzA: %llu nnzR: %llu\nnnzH: %llu nnzQ: %llu\n", nnzA_, nnzR_, nnzH_, nnzQ_);
        }
    }

    // ------------------------------------------------------------- solve
    void solve_dev(const double* d_b, double* d_x) override {
        if (!factorized_) throw std::logic_error("solve before factorize");
        if (rect_) throw std::invalid_argument("least-squares factorization: use solve_nrml / cgls");
        double t0 = wall();
        phase_ = 7;
        cuda_check(cudaMemcpyAsync(d_bin_, d_b, sizeof(double) * nrows_, cudaMemcpyDeviceToDevice, stream_), "solve in");
        // Until the solve graph is ready an application launches its sweeps
        // directly (the same kernels in the same order as the graph: the same
        // result), so the device does not wait for the graph; a host thread
        // captures it after the first application's launches are issued.
        if (!graph_exec_ && cap_done_) finish_capture();
        if (graph_exec_) {
            timed(KF_SOLVE, 0, solve_bytes_,
                  [&] { cuda_check(cudaGraphLaunch(graph_exec_, stream_), "graph launch"); });
        } else {
            timed(KF_SOLVE, 0, solve_bytes_, [&] { launches_solve_ = run_solve_sweeps(lanes_); });
            if (!cap_thread_.joinable()) start_capture();
        }
        cuda_check(cudaMemcpyAsync(d_x, d_xout_, sizeof(double) * ncols_, cudaMemcpyDeviceToDevice, stream_),
                   "solve out");
        t_solve_ = wall() - t0;
        ++applications_;
    }

    // y = M^T g: the factors applied transposed (adjoint sweeps, own graph).
    void solve_adjoint_dev(const double* d_g, double* d_y) override {
        if (!factorized_) throw std::logic_error("adjoint solve before factorize");
        if (rect_) throw std::invalid_argument("least-squares factorization: the adjoint solve needs a square one");
        double t0 = wall();
        cuda_check(cudaMemcpyAsync(d_adj_in_, d_g, sizeof(double) * ncols_, cudaMemcpyDeviceToDevice, stream_),
                   "adjoint in");
        if (!adj_exec_) {
            if (adj_waves_.empty()) build_adjoint_plan();
            cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
            run_adjoint_sweeps();
            cuda_check(cudaStreamEndCapture(stream_, &adj_graph_), "capture end");
            cuda_check(cudaGraphInstantiate(&adj_exec_, adj_graph_, 0), "graph instantiate");
        }
        timed(KF_SOLVE, 0, solve_bytes_, [&] { cuda_check(cudaGraphLaunch(adj_exec_, stream_), "graph launch"); });
        cuda_check(cudaMemcpyAsync(d_y, d_adj_out_, sizeof(double) * nrows_, cudaMemcpyDeviceToDevice, stream_),
                   "adjoint out");
        t_solve_ = wall() - t0;
        ++applications_;
    }

    std::vector<int> bottom_info() const override {
        std::vector<int> out;
        for (Cluster* c : bottoms_[0]) {
            int r[10] = {c->cstart, c->csize_org, c->rstart, c->rsize_org, c->id.self.lvl,
                         c->id.self.sep, c->id.l.lvl, c->id.l.sep, c->id.r.lvl, c->id.r.sep};
            out.insert(out.end(), r, r + 10);
        }
        return out;
    }
    void stats(double* times, long long* counters) const override {
        times[0] = t_part_;
        times[1] = t_asm_;
        times[2] = t_fact_;
        times[3] = t_solve_;
        counters[0] = (long long)nnzA_;
        counters[1] = (long long)nnzR_;
        counters[2] = (long long)nnzH_;
        counters[3] = (long long)nnzQ_;
        counters[4] = launches_fact_;
        counters[5] = launches_solve_;
        counters[6] = (long long)(arena_.bytes_reserved() + desc_arena_.bytes_reserved() + scratch_.capacity());
        counters[7] = applications_;
    }
    std::vector<double> host_times() const override {
        return {t_fact_,     t_rank_wait_, arena_.alloc_seconds() + desc_arena_.alloc_seconds() - alloc0_,
                scratch_.grow_seconds() - grow0_, t_plan_, t_phase_[0], t_phase_[1], t_phase_[2], t_phase_[3],
                t_phase_[4], t_phase_[5]};
    }
    std::vector<double> level_times() const override {
        std::vector<double> out;
        for (size_t l = 0; l + 7 <= level_ev_.size(); l += 7) {
            for (int p = 0; p < 6; ++p) {
                float ms = 0;
                cudaEventElapsedTime(&ms, level_ev_[l + p], level_ev_[l + p + 1]);
                out.push_back(ms);
            }
        }
        return out;
    }

private:
    Config cfg_;
    cudaStream_t stream_ = nullptr;
    // The streams a solve sweep launches on: the origin stream and two branches
    // forked from and joined to it (tall Q applications, large triangular ops).
    // lanes_ runs on stream_; cap_lanes_ is a second set on which a host thread
    // captures the solve graph while stream_ runs the first applications.
    struct Lanes {
        cudaStream_t main = nullptr, side = nullptr, side2 = nullptr;
        cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
    };
    Lanes lanes_, cap_lanes_;
    // Branch streams of a sparsification wave's RRQR: the launches of one wave
    // (one per cluster size) are independent interfaces and run side by side,
    // forked from stream_ and joined to it before the rank readback.
    static constexpr int kRqSide = 3;
    cudaStream_t rq_side_[kRqSide] = {};
    cudaEvent_t rq_fork_ = nullptr, rq_join_[kRqSide] = {};
    std::thread cap_thread_;
    std::atomic<bool> cap_done_{false};
    std::exception_ptr cap_err_;
    cudaGraph_t cap_graph_ = nullptr;
    cudaGraphExec_t cap_exec_ = nullptr;
    Arena arena_;
    int* d_status_ = nullptr;  // device status word of the current factorization
    int status_ = 0;           // its value at the end of the factorization
    Arena desc_arena_{size_t(16) << 20};
    Scratch scratch_;
    PinnedStage pinned_;
    double t_rank_wait_ = 0, t_plan_ = 0, alloc0_ = 0, grow0_ = 0;
    double t_phase_[6] = {0, 0, 0, 0, 0, 0};  // host time per phase: fill, elim, shift, scale, sparsify, merge
    std::vector<std::vector<Cluster*>> bottoms_, fine_;
    std::vector<std::unique_ptr<Cluster>> clusters_;
    ChunkedStore<Edge> edges_;
    std::vector<TapeOp> tape_;
    std::vector<int> cperm_, rperm_;
    bool rect_ = false;  // least squares (no identity row matching): rows move, R^T R solves
    bool geo_ = true;    // ordering from coordinates (the fill test uses the column-sparsity checks)
    int nrows_ = 0, ncols_ = 0, ilvl_ = -1, cur_bottom_ = 0, max_order_ = 0, next_uid_ = 0;
    bool assembled_ = false, factorized_ = false;
    unsigned long long nnzA_ = 0, nnzR_ = 0, nnzH_ = 0, nnzQ_ = 0;
    Log log_;
    double t_part_ = 0, t_asm_ = 0, t_fact_ = 0, t_solve_ = 0;
    long long launches_fact_ = 0, launches_solve_ = 0, applications_ = 0;
    std::vector<cudaEvent_t> events_, level_ev_;
    // solve plan
    T* xbuf_ = nullptr;
    double* d_bin_ = nullptr;
    double* d_xout_ = nullptr;
    int* d_src_ = nullptr;
    int* d_dst_ = nullptr;
    int64_t* d_xin_ = nullptr;
    int64_t* d_xout_pos_ = nullptr;
    // a sweep op with the x segments it reads and writes (wave scheduling)
    struct POp {
        SolveOp op;
        std::vector<Cluster*> rd, wr;
        int smem;
    };
    struct WMeta {
        size_t off;
        int n, smem;
        double words;
        int hkind, ha, hb;
        size_t boff;  // tall Q applications (cluster kernel): ops [boff, boff + nbig)
        int nbig, bcl;
        size_t toff;  // large triangular ops (cluster kernel): ops [toff, toff + ntri)
        int ntri, tcl, tk;
    };
    std::vector<POp> plan_fwd_, plan_bwd_;  // host copies, kept for the adjoint plan
    std::vector<int> gemv_cols_;            // columns of every neighbour block (work counts)
    struct Wave {
        const SolveOp* ops;
        int nops, smem;
        double words;        // factor words the wave reads
        int hkind, ha, hb;   // kind and sizes of its largest op
        const SolveOp* big;  // tall Q applications, one cluster of bcl CTAs each
        int nbig, bcl;
        const SolveOp* tri;  // large triangular ops, one cluster of tcl CTAs each (k <= tk)
        int ntri, tcl, tk;
    };
    static constexpr int kApplyqBigRows = 192;
    // A backward triangular op goes to the cluster kernel from kTriClWords
    // words of R^-1 and neighbour blocks, on ceil(words / kTriClPerCta) CTAs
    // (the wave's largest op sets the launch's cluster size).
    static constexpr double kTriClWords = 16384, kTriClPerCta = 16384;
    Wave make_wave(const SolveOp* d_ops, const WMeta& mt) const {
        return Wave{d_ops + mt.off, mt.n,     mt.smem,  mt.words, mt.hkind, mt.ha,  mt.hb,
                    d_ops + mt.boff, mt.nbig, mt.bcl,  d_ops + mt.toff, mt.ntri, mt.tcl, mt.tk};
    }
    // One sweep wave: the one-CTA ops, the tall Q applications and the large
    // triangular ops (independent ops: each cluster launch runs on a branch
    // forked from the stream).
    int launch_wave(const Wave& w, T* xb) { return launch_wave(w, xb, lanes_); }
    int launch_wave(const Wave& w, T* xb, const Lanes& ln) {
        const bool fork = (w.nops > 0) + (w.nbig > 0) + (w.ntri > 0) > 1;
        if (fork) {
            cuda_check(cudaEventRecord(ln.fork, ln.main), "fork");
            if (w.nbig > 0) cuda_check(cudaStreamWaitEvent(ln.side, ln.fork, 0), "fork");
            if (w.ntri > 0) cuda_check(cudaStreamWaitEvent(ln.side2, ln.fork, 0), "fork");
        }
        if (w.nbig > 0)
            cuda_check(launch_applyq_cl<T>(w.big, w.nbig, w.bcl, d_segs_, xb, fork ? ln.side : ln.main),
                       "solve cluster launch");
        if (w.ntri > 0)
            cuda_check(launch_tri_cl<T>(w.tri, w.ntri, w.tcl, w.tk, d_gemv_, xb, fork ? ln.side2 : ln.main),
                       "solve cluster launch");
        if (w.nops > 0) launch_solve_step<T>(w.ops, w.nops, d_segs_, d_gemv_, nullptr, xb, w.smem, ln.main);
        if (fork) {
            if (w.nbig > 0) {
                cuda_check(cudaEventRecord(ln.join, ln.side), "join");
                cuda_check(cudaStreamWaitEvent(ln.main, ln.join, 0), "join");
            }
            if (w.ntri > 0) {
                cuda_check(cudaEventRecord(ln.join2, ln.side2), "join");
                cuda_check(cudaStreamWaitEvent(ln.main, ln.join2, 0), "join");
            }
        }
        return (w.nops > 0) + (w.nbig > 0) + (w.ntri > 0);
    }
    std::vector<Wave> fwd_waves_, bwd_waves_, adj_waves_;
    int64_t xtot_ = 0;
    double* d_adj_in_ = nullptr;
    double* d_adj_out_ = nullptr;
    cudaGraph_t adj_graph_ = nullptr;
    cudaGraphExec_t adj_exec_ = nullptr;
    const XSeg* d_segs_ = nullptr;
    const GemvRef<T>* d_gemv_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    double solve_bytes_ = 0;  // algorithmic bytes of one preconditioner application

    // ------------------------------------------------------------- kernel timing (optional)
    // With profiling on, every launch is bracketed by CUDA events on the
    // handle's stream and charged to its kernel family together with the
    // algorithmic flops and bytes of the tasks it served.
    struct Pending {
        int fam;
        cudaEvent_t a, b;
        double flops, bytes;
        std::string tag;
        int level, phase;
    };
    double tg_[5] = {0, 0, 0, 0, 0};  // elimination build: host time of the fill-block steps (verbose 3)
    int phase_ = 0;  // phase of the launches being issued (profiling trace): 0-5 level phases, 6 solve plan, 7 solve
    bool prof_ = false, timeline_ = false;
    std::vector<Pending> pend_;
    std::string tag_;  // launch shape printed beside its time (profiling with verbose >= 4)
    bool tracing() const { return prof_ && cfg_.verbose >= 4; }
    KernelStat fam_[kNumFamilies];

    template <class F>
    size_t timed(int fam, double flops, double bytes, F&& launch) {
        if (!prof_) {
            launch();
            return SIZE_MAX;
        }
        cudaEvent_t a, b;
        cuda_check(cudaEventCreate(&a), "event");
        cuda_check(cudaEventCreate(&b), "event");
        cudaEventRecord(a, stream_);
        launch();
        cudaEventRecord(b, stream_);
        pend_.push_back(Pending{fam, a, b, flops, bytes, std::move(tag_), ilvl_, phase_});
        tag_.clear();
        return pend_.size() - 1;
    }
    void flush_prof() {
        if (pend_.empty()) return;
        cuda_check(cudaStreamSynchronize(stream_), "profile sync");
        for (auto& p : pend_) {
            float ms = 0;
            cudaEventElapsedTime(&ms, p.a, p.b);
            fam_[p.fam].launches += 1;
            fam_[p.fam].ms += ms;
            fam_[p.fam].flops += p.flops;
            fam_[p.fam].bytes += p.bytes;
            if (prof_ && cfg_.verbose >= 4)
                std::fprintf(stderr, "    trace %d %.4f ms L%d P%d %s\n", p.fam, ms, p.level, p.phase, p.tag.c_str());
            if (timeline_) {
                float st = 0;
                cudaEventElapsedTime(&st, pend_.front().a, p.a);
                std::fprintf(stderr, "timeline %d %.4f %.4f L%d P%d\n", p.fam, st, ms, p.level, p.phase);
            }
        }
        for (auto& p : pend_) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        pend_.clear();
    }

public:
    void set_profile(int level) override {
        prof_ = level > 0;
        timeline_ = level > 1;
    }
    double* krylov_workspace(size_t elems) override {
        open_device();
        return static_cast<double*>(scratch_.get(std::max<size_t>(elems, 1) * sizeof(double), stream_));
    }
    KernelStat kernel_stat(int fam) override {
        flush_prof();
        return (fam >= 0 && fam < kNumFamilies) ? fam_[fam] : KernelStat{};
    }
    void reset_kernel_stats() override {
        flush_prof();
        for (auto& f : fam_) f = KernelStat{};
    }

private:
    // ------------------------------------------------------------- helpers
    const std::vector<Cluster*>& cur() const { return bottoms_[cur_bottom_]; }

    void rec(long long type, long long a, long long b = 0, long long c = 0, long long d = 0, long long e = 0,
             long long order = -1) {
        long long r[8] = {type, ilvl_, order, a, b, c, d, e};
        log_.insert(log_.end(), r, r + 8);
    }

    Cluster* new_cluster(int cs, int cz, int rs, int rz, const Cid& id) {
        Cluster* c = new Cluster{cs, cz, rs, rz, id, max_order_++};
        c->csize_org = cz;
        c->rsize_org = rz;
        c->xcap = rz;
        clusters_.emplace_back(c);
        return c;
    }
    static size_t block_elems(int rows, int cols) { return (size_t)std::max(rows, 1) * std::max(cols, 1); }
    Blk new_block(int rows, int cols) {
        Blk b;
        b.rows = rows;
        b.cols = cols;
        b.ld = std::max(rows, 1);
        b.p = arena_.alloc_n<T>(block_elems(rows, cols));
        b.uid = next_uid_++;
        return b;
    }
    Edge* new_edge(Cluster* n1, Cluster* n2, const Blk& b) {
        edges_.push_back(Edge{n1, n2, b, true});
        return &edges_.back();
    }
    Edge* add_edge(Cluster* c1, Cluster* c2) {  // src/tree.cpp:251-261
        Edge* e = new_edge(c1, c2, new_block(c2->rsize, c1->csize));
        c1->out.push_back(e);
        if (c1 != c2) c2->in.push_back(e);
        return e;
    }
    // fn(begin, end) over [0, n) on up to 8 host threads, in chunks of at least
    // min_chunk items (one call on this thread below that); the first exception
    // a chunk throws is rethrown after all have joined.
    template <class F>
    static void host_parallel_for(size_t n, F&& fn, size_t min_chunk = 256) {
        const size_t hw = std::max(1u, std::thread::hardware_concurrency());
        const size_t nt = std::min<size_t>(std::min<size_t>(hw, 8), n / min_chunk);
        if (nt <= 1) {
            fn(size_t(0), n);
            return;
        }
        std::vector<std::exception_ptr> err(nt);
        const std::function<void(size_t)> body = [&](size_t t) {
            try {
                fn(n * t / nt, n * (t + 1) / nt);
            } catch (...) {
                err[t] = std::current_exception();
            }
        };
        if (!HostPool::get().run(nt, body))
            for (size_t t = 0; t < nt; ++t) body(t);
        for (auto& e : err)
            if (e) std::rethrow_exception(e);
    }
    static Edge* find_out(Cluster* c, Cluster* n2) {
        for (Edge* e : c->out)
            if (e->n2 == n2) return e;
        return nullptr;
    }

    std::pair<int, int> topsize() const {
        int tr = 0, tc = 0;
        for (Cluster* s : cur())
            if (s->level() == cfg_.nlevels - 1) { tr += s->rsize; tc += s->csize; }
        return {tr, tc};
    }
    bool want_sparsify(const Cluster* c) const {
        return c->level() > ilvl_ && c->id.l.lvl <= ilvl_ && c->id.r.lvl <= ilvl_;
    }

    // src/tree.cpp:168-224. Without coordinates the reference skips the two
    // column-sparsity tests and instead drops a candidate whose coupling block
    // product has norm <= 1e-14 (src/tree.cpp:857-860); that numeric test is not
    // made here: every candidate that passes the separator tests is kept. The
    // blocks it would drop receive updates of rounding size, so the factors
    // agree to rounding, with more (near-zero) fill blocks.
    bool valid_fill(const Cid& cid, const Cid& nid, const std::vector<Sep>& cols) const {
        const Sep cs = cid.self, ns = nid.self;
        if (cs.lvl > ns.lvl) return false;
        auto pw = [](int e) { return 1 << e; };
        if (cs.sep / pw(ns.lvl - cs.lvl) != ns.sep) return false;
        auto side_ok = [&](const Sep& s) {
            const int dl = s.lvl - cs.lvl;
            return s.lvl >= cs.lvl ? (cs.sep / pw(dl)) == s.sep : (s.sep / pw(-dl)) == cs.sep;
        };
        if (!side_ok(nid.l) && !side_ok(nid.r)) return false;
        if (!geo_) return true;
        auto has = [&](const Sep& x) { return std::binary_search(cols.begin(), cols.end(), x); };
        if (!has(ns)) return false;
        if (!has(nid.l) && !has(nid.r)) return false;
        return true;
    }
    // src/tree.cpp:834-870 (purely symbolic, with or without coordinates)
    // A fill candidate left to the numeric test: nin joins c's fill set if
    // ||A(n, c)^T A(n, nin)|| > 1e-14 for some shared row cluster n.
    struct FillCand {
        Cluster* nin;
        Blk a1, a2;
    };
    void get_sparsity(Cluster* c, std::vector<FillCand>* numeric = nullptr) {
        std::vector<Cluster*> rs;
        std::vector<Sep> cols;
        for (Edge* e : c->out) cols.push_back(e->n2->id.self);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        for (Edge* e : c->out) {
            if (!e->live) continue;
            Cluster* n = e->n2;
            rs.push_back(n);
            for (Edge* ein : n->in) {
                if (!(ein->live && ein->n1 != c && !ein->n1->elim && valid_fill(c->id, ein->n1->id, cols))) continue;
                Cluster* nin = ein->n1;
                // without coordinates the reference also asks the coupling to be
                // numerically nonzero (src/tree.cpp:856-859), unless nin is one of
                // c's own interfaces
                if (numeric && !(nin->id.l == c->id.self || nin->id.r == c->id.self))
                    numeric->push_back(FillCand{nin, e->A, ein->A});
                else
                    rs.push_back(nin);
            }
        }
        std::sort(rs.begin(), rs.end(), [](const Cluster* a, const Cluster* b) { return a->order < b->order; });
        rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
        c->rsparsity = std::move(rs);
        if (numeric) {  // candidates already in the set need no test
            auto in_rs = [&](const Cluster* x) {
                return std::binary_search(c->rsparsity.begin(), c->rsparsity.end(), x,
                                          [](const Cluster* a, const Cluster* b) { return a->order < b->order; });
            };
            numeric->erase(std::remove_if(numeric->begin(), numeric->end(),
                                          [&](const FillCand& f) { return in_rs(f.nin); }),
                           numeric->end());
        }
    }

    // The numeric fill test of the level's candidates: one batched launch of
    // ||A1^T A2|| (FP64 sums) and one readback; passing candidates join their
    // cluster's fill set.
    void numeric_fill(const std::vector<Cluster*>& fill, std::vector<std::vector<FillCand>>& cand) {
        std::vector<ProdNormTask<T>> tasks;
        for (auto& v : cand)
            for (auto& f : v)
                tasks.push_back(ProdNormTask<T>{f.a1.p, f.a2.p, f.a1.ld, f.a2.ld, f.a1.rows, f.a1.cols, f.a2.cols, 0});
        if (tasks.empty()) return;
        double* d_out = desc_arena_.alloc_n<double>(tasks.size());
        Upload up;
        const size_t o = up.add(tasks);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        launch_product_norms<T>(reinterpret_cast<const ProdNormTask<T>*>(d + o), (int)tasks.size(), d_out, stream_);
        ++launches_fact_;
        std::vector<double> norms(tasks.size());
        cuda_check(cudaMemcpyAsync(norms.data(), d_out, norms.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_),
                   "fill norms");
        cuda_check(cudaStreamSynchronize(stream_), "fill norms");
        pinned_.reset();
        size_t q = 0;
        for (size_t i = 0; i < fill.size(); ++i) {
            bool added = false;
            for (auto& f : cand[i]) {
                if (norms[q++] > 1e-14) {
                    fill[i]->rsparsity.push_back(f.nin);
                    added = true;
                }
            }
            if (added) {
                auto& rs = fill[i]->rsparsity;
                std::sort(rs.begin(), rs.end(), [](const Cluster* a, const Cluster* b) { return a->order < b->order; });
                rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
            }
        }
    }

    // ------------------------------------------------------------- batched QR execution
    // One QR job: gathers into [fac | scratch], factors, scatters the trailing part back.
    struct QRJob {
        int m = 0, k = 0, ntr = 0;
        T* fac = nullptr;
        T* tau = nullptr;
        T* tp = nullptr;
        size_t tr_off = 0;  // element offset in the wave scratch
        std::vector<CopyDesc<T>> gather, scatter;  // tr pointers patched at issue time (relative)
    };

    // Issues the jobs of one wave (already built), then extra copies (after the QR).
    // One wave's descriptor arrays (host only), then its upload and launches.
    struct PanelLaunch {
        int kind = 0;  // 0 single-CTA, 1 shared-memory slabs, 2 register-resident
        int cluster = 0, max_slab = 0;
        std::vector<int> ids;
    };
    struct WaveBuild {
        std::vector<CopyDesc<T>> g, s;
        std::vector<QRTask<T>> qt;
        int maxk = 0, maxR = 0;
        std::vector<std::vector<int>> ids;
        std::vector<std::vector<TileRef>> tiles;
        std::vector<TileRef> trsm_tiles;
        std::vector<std::vector<PanelLaunch>> pgroups;
    };
    // Places each job's trailing block in the wave scratch; returns its element count.
    static size_t wave_scratch_elems(std::vector<QRJob>& jobs) {
        size_t tr_elems = 0;
        for (auto& j : jobs) {
            j.tr_off = tr_elems;
            tr_elems += (size_t)j.m * j.ntr;
        }
        return tr_elems;
    }
    // Pure host work: reads the jobs, writes B (safe on any host thread).
    static void build_wave(const std::vector<QRJob>& jobs, const std::vector<TrsmTask<T>>& trsm, T* trbase,
                           int* status, WaveBuild& B) {
        auto& g = B.g;
        auto& s = B.s;
        auto& qt = B.qt;
        {
            size_t ng = 0, ns = 0;
            for (auto& j : jobs) {
                ng += j.gather.size();
                ns += j.scatter.size();
            }
            g.reserve(ng);
            s.reserve(ns);
            qt.reserve(jobs.size());
        }
        int& maxk = B.maxk;
        int& maxR = B.maxR;
        for (auto& j : jobs) {
            T* tr = trbase + j.tr_off;
            for (auto c : j.gather) {
                if (c.dst == nullptr) c.dst = tr + c.pad;  // relative trailing destination
                c.pad = 0;
                g.push_back(c);
            }
            for (auto c : j.scatter) {
                c.src = tr + c.pad;
                c.pad = 0;
                s.push_back(c);
            }
            qt.push_back(QRTask<T>{j.fac, tr, j.tau, j.tp, j.m, j.k, j.ntr, 0, status});
            maxk = std::max(maxk, j.k);
            maxR = std::max(maxR, j.m);
        }
        // per-panel active lists and trailing tiles
        auto& ids = B.ids;
        auto& tiles = B.tiles;
        for (int p = 0; p < maxk; p += kNB) {
            std::vector<int> a;
            std::vector<TileRef> tl;
            for (size_t t = 0; t < qt.size(); ++t) {
                if (qt[t].k <= p) continue;
                a.push_back((int)t);
                const int w = std::min(kNB, qt[t].k - p);
                const int ntot = (qt[t].k - p - w) + qt[t].ntr;
                for (int c0 = 0, ti = 0; c0 < ntot; c0 += kTN, ++ti) tl.push_back(TileRef{(int)t, ti});
            }
            ids.push_back(std::move(a));
            tiles.push_back(std::move(tl));
        }
        auto& trsm_tiles = B.trsm_tiles;
        for (size_t t = 0; t < trsm.size(); ++t)
            for (int r0 = 0, ti = 0; r0 < trsm[t].rows; r0 += 128, ++ti) trsm_tiles.push_back(TileRef{(int)t, ti});
        // panel groups: cluster size by panel height (row slabs of about 256 rows, at
        // least 32), 0 = single-CTA kernel for panels beyond the clusters' shared memory
        auto panel_cluster = [](int R) {
            int c = std::max(1, std::min(16, (R + 255) / 256));
            while (c > 1 && R < 32 * c) --c;
            while (c < 16 && (size_t)R > panel_cl_max_rows<T>(c)) ++c;
            return (size_t)R > panel_cl_max_rows<T>(c) ? 0 : c;
        };
        // panel launches of each step: tasks beyond the clusters (single-CTA kernel)
        // apart; the cluster tasks in one launch whose cluster is the largest any of
        // them needs, unless the idle CTAs of the smaller tasks would cost more than
        // one more launch (the launch does not fit the SMs at once and a third or
        // more of its CTAs would idle); then one launch per class of cluster sizes
        // (1, 2, 3-4, 5-8, 9-16). ids: task indices then their cluster sizes.
        // Panels of at most 16 * kPanelRegRows rows run register-resident
        // (k_panel_reg, slabs of kPanelRegRows rows), taller ones from shared-memory
        // slabs (k_panel_cl).
        auto& pgroups = B.pgroups;
        pgroups.assign(ids.size(), {});
        for (size_t i = 0; i < ids.size(); ++i) {
            const int p = (int)i * kNB;
            PanelLaunch single;
            std::vector<std::pair<int, int>> clt[2];  // (cluster size, task) of kinds 1 and 2
            for (int t : ids[i]) {
                const int R = qt[t].m - p;
                if (R <= 16 * kPanelRegRows) {  // FP32 panels up to 512 rows: one CTA, no cluster barrier
                    const int c = (sizeof(T) == 4 && R <= 2 * kPanelRegRows)
                                      ? 1
                                      : std::max(1, (R + kPanelRegRows - 1) / kPanelRegRows);
                    clt[1].push_back({c, t});
                    continue;
                }
                const int c = panel_cluster(R);
                if (c == 0)
                    single.ids.push_back(t);
                else
                    clt[0].push_back({c, t});
            }
            if (!single.ids.empty()) pgroups[i].push_back(std::move(single));
            for (int kind = 1; kind <= 2; ++kind) {
                auto& list = clt[kind - 1];
                if (list.empty()) continue;
                int cmax = 0;
                long long used = 0;
                for (auto& e : list) {
                    cmax = std::max(cmax, e.first);
                    used += e.first;
                }
                const long long total = (long long)cmax * (long long)list.size();
                const bool one = total <= 2 * 148 || 3 * used >= 2 * total;
                auto cls = [&](int c) { return one ? 0 : (c <= 2 ? c : c <= 4 ? 3 : c <= 8 ? 4 : 5); };
                std::map<int, std::vector<std::pair<int, int>>> by;
                for (auto& e : list) by[-cls(e.first)].push_back(e);
                for (auto& kv : by) {
                    // tallest panels first: clusters start in list order, so a launch
                    // with more clusters than fit at once does not end on a tall one
                    // started last (tasks are independent: no result changes)
                    std::stable_sort(kv.second.begin(), kv.second.end(),
                                     [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                                         return qt[a.second].m > qt[b.second].m;
                                     });
                    PanelLaunch L;
                    L.kind = kind;
                    for (auto& e : kv.second) {
                        L.cluster = std::max(L.cluster, e.first);
                        L.max_slab = std::max(L.max_slab, (qt[e.second].m - p + e.first - 1) / e.first);
                        L.ids.push_back(e.second);
                    }
                    for (auto& e : kv.second) L.ids.push_back(e.first);
                    pgroups[i].push_back(std::move(L));
                }
            }
        }
    }

    void run_qr_wave(std::vector<QRJob>& jobs, const std::vector<TrsmTask<T>>& trsm,
                     const std::vector<CopyDesc<T>>& post) {
        const double tw_wave = wall();
        const size_t tr_elems = wave_scratch_elems(jobs);
        T* trbase = static_cast<T*>(scratch_.get(std::max<size_t>(tr_elems, 1) * sizeof(T), stream_));
        WaveBuild B;
        build_wave(jobs, trsm, trbase, d_status_, B);
        issue_wave(B, trsm, post, tw_wave);
    }

    void issue_wave(WaveBuild& B, const std::vector<TrsmTask<T>>& trsm, const std::vector<CopyDesc<T>>& post,
                    double tw_wave) {
        const double pin0 = pinned_.alloc_seconds(), grow0 = scratch_.grow_seconds(),
                     ar0 = arena_.alloc_seconds() + desc_arena_.alloc_seconds();
        auto& g = B.g;
        auto& s = B.s;
        auto& qt = B.qt;
        const int maxR = B.maxR;
        auto& ids = B.ids;
        auto& tiles = B.tiles;
        auto& trsm_tiles = B.trsm_tiles;
        auto& pgroups = B.pgroups;
        const double tw_built = wall();
        // One CTA per tile, independent of the others: the tiles of the tallest
        // tasks (trailing update) and of the widest R (TRSM) first, so that a
        // launch of more CTAs than fit at once does not end on a long one
        // started last. The order changes no result.
        for (auto& tl : tiles)
            std::stable_sort(tl.begin(), tl.end(),
                             [&](const TileRef& a, const TileRef& b) { return qt[a.task].m > qt[b.task].m; });
        std::stable_sort(trsm_tiles.begin(), trsm_tiles.end(),
                         [&](const TileRef& a, const TileRef& b) { return trsm[a.task].k > trsm[b.task].k; });
        Upload up;
        size_t o_g = up.add(g), o_s = up.add(s), o_q = up.add(qt), o_tr = up.add(trsm), o_tt = up.add(trsm_tiles),
               o_post = up.add(post);
        std::vector<size_t> o_ids, o_tiles;
        std::vector<std::vector<size_t>> o_pg(ids.size());
        for (size_t i = 0; i < ids.size(); ++i) {
            o_ids.push_back(up.add(ids[i]));
            o_tiles.push_back(up.add(tiles[i]));
            for (auto& L : pgroups[i]) o_pg[i].push_back(up.add(L.ids));
        }
        char* d = up.commit(desc_arena_, stream_, pinned_);
        const double tw_up = wall();
        issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o_g), g);
        const int smem_limit = (int)((160 * 1024) / (kNB * sizeof(T)));
        for (size_t i = 0; i < ids.size(); ++i) {
            const int p = (int)i * kNB;
            int rows = 0;
            double pf = 0, pb = 0, tf = 0, tb = 0;
            for (int t : ids[i]) {
                const double R = qt[t].m - p, w = std::min(kNB, qt[t].k - p);
                rows = std::max(rows, qt[t].m - p);
                pf += 2 * R * w * w - 2.0 / 3.0 * w * w * w + R * w * w;  // geqrf + larft of the panel
                pb += 2 * R * w * sizeof(T);
            }
            for (const TileRef& tr : tiles[i]) {
                const QRTask<T>& q = qt[tr.task];
                const double R = q.m - p, w = std::min(kNB, q.k - p);
                const int ntot = (q.k - p - (int)w) + q.ntr;
                const double tn = std::min(kTN, ntot - tr.tile * kTN);
                tf += 4 * R * tn * w;
                tb += (2 * R * tn + R * w) * sizeof(T);
            }
            const int smem_rows = std::min(rows, smem_limit);
            if (tracing()) {
                tag_ = "panel p " + std::to_string(p);
                for (auto& L : pgroups[i])
                    tag_ += " | kind " + std::to_string(L.kind) + " cl " + std::to_string(L.cluster) + " n " +
                            std::to_string(L.kind ? L.ids.size() / 2 : L.ids.size()) + " slab " +
                            std::to_string(L.max_slab);
            }
            timed(KF_PANEL, pf, pb, [&] {
                for (size_t g = 0; g < pgroups[i].size(); ++g) {
                    const PanelLaunch& L = pgroups[i][g];
                    const int* gids = reinterpret_cast<const int*>(d + o_pg[i][g]);
                    const QRTask<T>* dq = reinterpret_cast<const QRTask<T>*>(d + o_q);
                    if (L.kind == 0)
                        launch_panel<T>(dq, gids, (int)L.ids.size(), p, smem_rows, stream_);
                    else if (L.kind == 1)
                        cuda_check(launch_panel_cl<T>(dq, gids, (int)L.ids.size() / 2, L.cluster, L.max_slab, p,
                                                      stream_),
                                   "panel launch");
                    else
                        cuda_check(launch_panel_reg<T>(dq, gids, (int)L.ids.size() / 2, L.cluster, L.max_slab, p,
                                                       stream_),
                                   "panel launch");
                    ++launches_fact_;
                }
            });
            if (!tiles[i].empty()) {
                if (tracing())
                    tag_ = "trailing p " + std::to_string(p) + " tiles " + std::to_string(tiles[i].size()) + " R " +
                           std::to_string(rows);
                timed(KF_TRAILING, tf, tb, [&] {
                    launch_trailing<T>(reinterpret_cast<const QRTask<T>*>(d + o_q),
                                       reinterpret_cast<const TileRef*>(d + o_tiles[i]), (int)tiles[i].size(), p,
                                       stream_);
                });
                ++launches_fact_;
            }
        }
        issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o_s), s);
        if (!trsm_tiles.empty()) {
            double f = 0, by = 0;
            for (auto& t : trsm) {
                f += (double)t.rows * t.k * t.k;
                by += (2.0 * t.rows * t.k + 0.5 * t.k * t.k) * sizeof(T);
            }
            timed(KF_TRSM, f, by, [&] {
                launch_trsm<T>(reinterpret_cast<const TrsmTask<T>*>(d + o_tr),
                               reinterpret_cast<const TileRef*>(d + o_tt), (int)trsm_tiles.size(), stream_);
            });
            ++launches_fact_;
        }
        issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o_post), post);
        if (cfg_.verbose >= 3) {  // diagnostics: the wave's shape and its time (synchronizes)
            const double tsub = wall();
            cuda_check(cudaStreamSynchronize(stream_), "wave sync");
            int mk = 0, mn = 0;
            size_t nt = 0;
            double work = 0;
            for (auto& q : qt) {
                mk = std::max(mk, q.k);
                mn = std::max(mn, q.ntr);
                work += (double)q.m * q.k * (q.k + q.ntr);
            }
            for (auto& tl : tiles) nt += tl.size();
            std::fprintf(stderr, "    qr wave: %zu tasks, max m %d, max k %d, max ntr %d, %zu panel steps, %zu tiles, "
                         "m k (k + ntr) %.3e, %zu trsm tasks, %.2f ms (host %.2f: build %.2f upload %.2f launch %.2f "
                         "pinned %.2f scratch %.2f arena %.2f, %zu pinned chunks)\n",
                         qt.size(), maxR, mk, mn, ids.size(), nt, work, trsm.size(), (wall() - tw_wave) * 1e3,
                         (tsub - tw_wave) * 1e3, (tw_built - tw_wave) * 1e3, (tw_up - tw_built) * 1e3,
                         (tsub - tw_up) * 1e3, (pinned_.alloc_seconds() - pin0) * 1e3,
                         (scratch_.grow_seconds() - grow0) * 1e3,
                         (arena_.alloc_seconds() + desc_arena_.alloc_seconds() - ar0) * 1e3, pinned_.chunks());
        }
    }

    void issue_copies(const CopyDesc<T>* d, const std::vector<CopyDesc<T>>& h) {
        if (h.empty()) return;
        double by = 0;
        int maxc = 0;
        for (auto& c : h) {
            by += (c.src ? 2.0 : 1.0) * c.rows * c.cols * sizeof(T);
            maxc = std::max(maxc, c.cols);
        }
        timed(KF_COPY, 0, by, [&] { launch_copy<T>(d, (int)h.size(), maxc, stream_); });
        ++launches_fact_;
    }

    static CopyDesc<T> cp(const T* src, T* dst, int sld, int dld, int rows, int cols, int mode = 0, int pad = 0) {
        return CopyDesc<T>{src, dst, sld, dld, rows, cols, mode, pad};
    }

    // ------------------------------------------------------------- elimination (src/tree.cpp:780-832)
    void elim_phase() {
        const double te0 = wall();
        struct Task {
            QRJob job;
            std::vector<int> uids;
        };
        // The level's interiors in order. Graph changes (fill blocks: arena
        // addresses, uids, edge order) are made on this thread in that order;
        // the read-only block search and the descriptor lists, which are most of
        // the host work, run on host threads. Same blocks, same order, same
        // descriptors as one task after another.
        std::vector<Cluster*> lv;
        for (Cluster* c : cur())
            if (c->level() == ilvl_) lv.push_back(c);
        const size_t nl = lv.size();
        std::unordered_map<const Cluster*, int> pos_in_level;
        pos_in_level.reserve(nl * 2);
        for (size_t i = 0; i < nl; ++i) pos_in_level[lv[i]] = (int)i;
        struct Plan {
            std::vector<Edge*> H;           // stacked column blocks
            std::vector<Cluster*> upd;      // updated clusters, rsparsity order
            std::vector<Edge*> blk;         // upd.size() x H.size(): the block of (upd, H row cluster), null if missing
            int m = 0, k = 0;
        };
        std::vector<Plan> plans(nl);
        // The split below relies on no interior of this level lying in another's
        // column or fill set (true of nested dissection, whose interiors are cut
        // apart by separators): then no task's fill lands in another task's
        // column. Otherwise the tasks are built one after another.
        std::atomic<bool> coupled{false};
        // 1. (threads) blocks that already exist: a neighbour n is updated unless
        //    eliminated before this phase or earlier in it (lower position)
        host_parallel_for(
            nl,
            [&](size_t b, size_t e) {
                std::vector<std::pair<const Cluster*, int>> hs;
                for (size_t i = b; i < e; ++i) {
                    Cluster* c = lv[i];
                    Plan& P = plans[i];
                    if (c->csize == 0) continue;
                    for (Edge* ed : c->out)
                        if (ed->live) {
                            P.H.push_back(ed);
                            P.m += ed->A.rows;
                            if (ed->n2 != c && pos_in_level.count(ed->n2)) coupled = true;
                        }
                    P.k = P.H.front()->A.cols;
                    // H's row clusters by address: one pass over a neighbour's edges
                    // finds all of its blocks in those rows (the first edge per row
                    // cluster, as a scan per row cluster would)
                    hs.clear();
                    for (size_t h = 0; h < P.H.size(); ++h) hs.emplace_back(P.H[h]->n2, (int)h);
                    std::sort(hs.begin(), hs.end());
                    for (size_t h = 1; h < hs.size(); ++h)
                        if (hs[h].first == hs[h - 1].first) coupled = true;  // two blocks in one row cluster
                    const size_t nh = P.H.size();
                    for (Cluster* n : c->rsparsity) {
                        if (n == c || n->elim) continue;
                        auto it = pos_in_level.find(n);
                        if (it != pos_in_level.end()) {
                            coupled = true;
                            if (it->second < (int)i) continue;
                        }
                        P.upd.push_back(n);
                        const size_t base = P.blk.size();
                        P.blk.resize(base + nh, nullptr);
                        for (Edge* e2 : n->out) {
                            auto f = std::lower_bound(hs.begin(), hs.end(), std::make_pair((const Cluster*)e2->n2, -1));
                            if (f != hs.end() && f->first == e2->n2 && !P.blk[base + f->second])
                                P.blk[base + f->second] = e2;
                        }
                    }
                }
            },
            16);
        const double ts1 = wall();
        double ts2 = ts1, ts3 = ts1;
        const size_t nedges0 = edges_.size();
        std::vector<Task> tasks;
        if (!coupled) {
        // 2. arena memory of every job and the missing fill blocks, the same
        //    blocks, uids, edges and list orders as a task-by-task elimination
        //    (a block is made by the first task that misses it, in level order,
        //    and found by the later ones):
        //    a. (threads) each task's missing (updated cluster n, row cluster r)
        //       slots in (u, h) order, at its prefix-sum position
        const std::vector<Cluster*>& all_c = cur();
        for (size_t q = 0; q < all_c.size(); ++q) all_c[q]->pos = (int)q;
        struct Miss {
            int task, slot, n, r;  // n, r: positions in cur()
        };
        std::vector<size_t> mbase(nl + 1, 0);
        host_parallel_for(
            nl,
            [&](size_t b, size_t e) {
                for (size_t i = b; i < e; ++i)
                    mbase[i + 1] = (size_t)std::count(plans[i].blk.begin(), plans[i].blk.end(), nullptr);
            },
            64);
        for (size_t i = 0; i < nl; ++i) mbase[i + 1] += mbase[i];
        const size_t nm = mbase[nl];
        std::vector<Miss> miss(nm);
        host_parallel_for(
            nl,
            [&](size_t b, size_t e) {
                for (size_t i = b; i < e; ++i) {
                    const Plan& P = plans[i];
                    const size_t nh = P.H.size();
                    size_t q = mbase[i];
                    for (size_t s = 0; s < P.blk.size(); ++s)
                        if (!P.blk[s]) miss[q++] = Miss{(int)i, (int)s, P.upd[s / nh]->pos, P.H[s % nh]->n2->pos};
                }
            },
            64);
        const double tg1 = wall();
        //    b. the slots of each n in that order; (threads) per n, the first
        //       slot of each r makes the block (creator[m] == m), the rest use it
        const size_t ncl = all_c.size();
        std::vector<size_t> nb0(ncl + 1, 0);
        for (const Miss& m : miss) ++nb0[m.n + 1];
        for (size_t q = 0; q < ncl; ++q) nb0[q + 1] += nb0[q];
        std::vector<int> byn(nm), creator(nm);
        {
            std::vector<size_t> cur_n(nb0.begin(), nb0.end() - 1);
            for (size_t m = 0; m < nm; ++m) byn[cur_n[miss[m].n]++] = (int)m;
        }
        host_parallel_for(
            ncl,
            [&](size_t b, size_t e) {
                std::vector<std::pair<int, int>> rs;
                for (size_t q = b; q < e; ++q) {
                    if (nb0[q] == nb0[q + 1]) continue;
                    rs.clear();
                    for (size_t x = nb0[q]; x < nb0[q + 1]; ++x) rs.emplace_back(miss[byn[x]].r, byn[x]);
                    std::sort(rs.begin(), rs.end());
                    for (size_t x = 0; x < rs.size(); ++x)
                        creator[rs[x].second] = (x && rs[x].first == rs[x - 1].first) ? creator[rs[x - 1].second]
                                                                                       : rs[x].second;
                }
            },
            256);
        const double tg2 = wall();
        //    c. (level order) job memory, then the task's new blocks: uids and
        //       arena addresses in creation order
        std::vector<Task> all(nl);
        std::vector<int> rank(nm, -1);
        std::vector<T*> bptr;
        bptr.reserve(nm);
        const size_t e0 = edges_.size();
        const int uid0 = next_uid_;
        for (size_t i = 0; i < nl; ++i) {
            Cluster* c = lv[i];
            const Plan& P = plans[i];
            if (c->csize == 0) continue;
            QRJob& j = all[i].job;
            j.m = P.m;
            j.k = P.k;
            j.fac = arena_.alloc_n<T>((size_t)P.m * P.k);
            j.tau = arena_.alloc_n<T>(P.k);
            j.tp = arena_.alloc_n<T>((size_t)npanels(P.k) * kNB * kNB);
            for (size_t m = mbase[i]; m < mbase[i + 1]; ++m)
                if (creator[m] == (int)m) {
                    rank[m] = (int)bptr.size();
                    bptr.push_back(arena_.alloc_n<T>(block_elems(all_c[miss[m].r]->rsize, all_c[miss[m].n]->csize)));
                }
        }
        const size_t nnew = bptr.size();
        if (nnew > size_t(std::numeric_limits<int>::max() - next_uid_))
            throw std::runtime_error("elimination: block uid overflow");
        next_uid_ += (int)nnew;
        const double tg3 = wall();
        edges_.resize(e0 + nnew);
        std::vector<int> cr(nnew);  // the new block's row cluster (position in cur()), -1 on the diagonal
        //    d. (threads) the new edges, each n's out list and the tasks' slots;
        //       then each r's in list, in creation order
        host_parallel_for(
            ncl,
            [&](size_t b, size_t e) {
                for (size_t q = b; q < e; ++q) {
                    Cluster* n = all_c[q];
                    for (size_t x = nb0[q]; x < nb0[q + 1]; ++x) {
                        const int m = byn[x];
                        if (creator[m] != m) continue;
                        Cluster* r = all_c[miss[m].r];
                        Blk bk;
                        bk.rows = r->rsize;
                        bk.cols = n->csize;
                        bk.ld = std::max(bk.rows, 1);
                        bk.p = bptr[rank[m]];
                        bk.uid = uid0 + rank[m];
                        Edge& ed = edges_[e0 + rank[m]];
                        ed = Edge{n, r, bk, true};
                        n->out.push_back(&ed);
                        cr[rank[m]] = r == n ? -1 : miss[m].r;
                    }
                    for (size_t x = nb0[q]; x < nb0[q + 1]; ++x) {
                        const int m = byn[x];
                        plans[miss[m].task].blk[miss[m].slot] = &edges_[e0 + rank[creator[m]]];
                    }
                }
            },
            256);
        const double tg4 = wall();
        {
            const size_t hw = std::max(1u, std::thread::hardware_concurrency());
            const size_t nth = std::max<size_t>(1, std::min<size_t>({hw, 8, nnew / 4096}));
            host_parallel_for(
                nth,
                [&](size_t b, size_t e) {
                    for (size_t k = b; k < e; ++k) {  // row clusters [ncl k / nth, ncl (k + 1) / nth)
                        const int lo = (int)(ncl * k / nth), hi = (int)(ncl * (k + 1) / nth);
                        for (size_t x = 0; x < nnew; ++x)
                            if (cr[x] >= lo && cr[x] < hi) all_c[cr[x]]->in.push_back(&edges_[e0 + x]);
                    }
                },
                1);
        }
        for (size_t i = 0; i < nl; ++i) lv[i]->elim = true;
        ts2 = wall();
        tg_[0] = tg1 - ts1;
        tg_[1] = tg2 - tg1;
        tg_[2] = tg3 - tg2;
        tg_[3] = tg4 - tg3;
        tg_[4] = ts2 - tg4;
        // 3. (threads) each job's copy descriptors and block uids
        host_parallel_for(
            nl,
            [&](size_t b, size_t e) {
                for (size_t i = b; i < e; ++i) {
                    Cluster* c = lv[i];
                    Plan& P = plans[i];
                    if (c->csize == 0) continue;
                    Task& t = all[i];
                    QRJob& j = t.job;
                    const int m = P.m, k = P.k;
                    const size_t nh = P.H.size();
                    j.gather.reserve(nh * (1 + P.upd.size()));
                    j.scatter.reserve(nh * P.upd.size());
                    t.uids.reserve(nh * (1 + P.upd.size()));
                    int off = 0;
                    for (Edge* ed : P.H) {
                        j.gather.push_back(cp(ed->A.p, j.fac + off, ed->A.ld, m, ed->A.rows, k));
                        t.uids.push_back(ed->A.uid);
                        off += ed->A.rows;
                    }
                    int co = 0;
                    for (size_t u = 0; u < P.upd.size(); ++u) {
                        Cluster* n = P.upd[u];
                        off = 0;
                        for (size_t h = 0; h < nh; ++h) {
                            Edge* ecn = P.blk[u * nh + h];
                            const int pad = off + co * m;  // relative to the wave scratch of this job
                            j.gather.push_back(cp(ecn->A.p, nullptr, ecn->A.ld, m, ecn->A.rows, n->csize, 0, pad));
                            j.scatter.push_back(cp(nullptr, ecn->A.p, m, ecn->A.ld, ecn->A.rows, n->csize, 0, pad));
                            t.uids.push_back(ecn->A.uid);
                            off += ecn->A.rows;
                        }
                        co += n->csize;
                    }
                    j.ntr = co;
                }
            },
            64);
        ts3 = wall();
        // 4. (threads) each task's tape op; then (this thread, level order) the
        //    tape, counters, log and, for least squares, the column blocks a
        //    finished elimination drops
        std::vector<TapeOp> qops(nl);
        host_parallel_for(
            nl,
            [&](size_t b, size_t e) {
                for (size_t i = b; i < e; ++i) {
                    Cluster* c = lv[i];
                    const Plan& P = plans[i];
                    if (c->csize == 0) continue;
                    TapeOp& op = qops[i];
                    op.kind = TK_QR;
                    op.c = c;
                    op.fac = all[i].job.fac;
                    op.tp = all[i].job.tp;
                    op.m = P.m;
                    op.k = P.k;
                    op.ld = P.m;
                    op.segs.reserve(P.H.size());
                    for (Edge* ed : P.H) op.segs.emplace_back(ed->n2, ed->n2->rsize);
                    op.a12.reserve(c->in.size());
                    for (Edge* ed : c->in) op.a12.push_back(A12{ed->A.p, ed->A.ld, ed->A.cols, ed->n1});
                }
            },
            64);
        for (size_t i = 0; i < nl; ++i) {
            Cluster* c = lv[i];
            Plan& P = plans[i];
            if (c->csize == 0) {
                rec(1, 0, 0, 0, 0, 0, c->order);
                continue;
            }
            const int m = P.m, k = P.k;
            int co = 0;
            for (Cluster* n : P.upd) {
                nnzR_ += (unsigned long long)(c->csize * n->csize);
                co += n->csize;
            }
            nnzH_ += (unsigned long long)(m * k);
            tape_.push_back(std::move(qops[i]));
            if (rect_) {  // least squares keeps R only: the self block shrinks to k rows, the rest goes
                for (Edge* ed : c->out) {
                    if (ed->n2 == c)
                        ed->A.rows = std::min(ed->A.rows, k);
                    else
                        ed->live = false;
                }
            }
            rec(1, m, k, (long long)P.upd.size(), (long long)P.H.size(), co, c->order);
            tasks.push_back(std::move(all[i]));
        }
        } else {
            for (Cluster* c : cur()) {
                if (c->level() != ilvl_) continue;
                if (c->csize == 0) {
                    c->elim = true;
                    rec(1, 0, 0, 0, 0, 0, c->order);
                    continue;
                }
                std::vector<Edge*> H;
                int m = 0;
                for (Edge* e : c->out)
                    if (e->live) { H.push_back(e); m += e->A.rows; }
                const int k = H.front()->A.cols;
                Task t;
                QRJob& j = t.job;
                j.m = m;
                j.k = k;
                j.fac = arena_.alloc_n<T>((size_t)m * k);
                j.tau = arena_.alloc_n<T>(k);
                j.tp = arena_.alloc_n<T>((size_t)npanels(k) * kNB * kNB);
                int off = 0;
                for (Edge* e : H) {
                    j.gather.push_back(cp(e->A.p, j.fac + off, e->A.ld, m, e->A.rows, k));
                    t.uids.push_back(e->A.uid);
                    off += e->A.rows;
                }
                int nupd = 0, co = 0;
                // H's row clusters by address: one pass over a neighbour's edges finds
                // all of its blocks in those rows (the first edge per row cluster, as a
                // scan per row cluster would); missing ones are added in H's order
                std::vector<std::pair<const Cluster*, int>> hs;
                hs.reserve(H.size());
                for (size_t i = 0; i < H.size(); ++i) hs.emplace_back(H[i]->n2, (int)i);
                std::sort(hs.begin(), hs.end());
                std::vector<Edge*> found(H.size());
                for (Cluster* n : c->rsparsity) {
                    if (n->elim || n == c) continue;
                    std::fill(found.begin(), found.end(), nullptr);
                    for (Edge* e2 : n->out) {
                        auto it = std::lower_bound(hs.begin(), hs.end(), std::make_pair((const Cluster*)e2->n2, -1));
                        if (it != hs.end() && it->first == e2->n2 && !found[it->second]) found[it->second] = e2;
                    }
                    off = 0;
                    for (size_t hi = 0; hi < H.size(); ++hi) {
                        Edge* e = H[hi];
                        Edge* ecn = found[hi];
                        if (!ecn) ecn = add_edge(n, e->n2);
                        const int pad = off + co * m;  // relative to the wave scratch of this job
                        j.gather.push_back(cp(ecn->A.p, nullptr, ecn->A.ld, m, ecn->A.rows, n->csize, 0, pad));
                        j.scatter.push_back(cp(nullptr, ecn->A.p, m, ecn->A.ld, ecn->A.rows, n->csize, 0, pad));
                        t.uids.push_back(ecn->A.uid);
                        off += ecn->A.rows;
                    }
                    co += n->csize;
                    nnzR_ += (unsigned long long)(c->csize * n->csize);
                    ++nupd;
                }
                j.ntr = co;
                nnzH_ += (unsigned long long)(m * k);
                TapeOp op;
                op.kind = TK_QR;
                op.c = c;
                op.fac = j.fac;
                op.tp = j.tp;
                op.m = m;
                op.k = k;
                op.ld = m;
                for (Edge* e : H) op.segs.emplace_back(e->n2, e->n2->rsize);
                for (Edge* e : c->in) op.a12.push_back(A12{e->A.p, e->A.ld, e->A.cols, e->n1});
                tape_.push_back(std::move(op));
                c->elim = true;
                if (rect_) {  // least squares keeps R only: the self block shrinks to k rows, the rest goes
                    for (Edge* e : c->out) {
                        if (e->n2 == c)
                            e->A.rows = std::min(e->A.rows, k);
                        else
                            e->live = false;
                    }
                }
                rec(1, m, k, nupd, (long long)H.size(), co, c->order);
                tasks.push_back(std::move(t));
            }
        }
        if (tasks.empty()) return;
        const double te1 = wall();
        std::vector<std::vector<int>> touched;
        for (auto& t : tasks) touched.push_back(std::move(t.uids));
        int nw = 0;
        auto wave = assign_waves(touched, next_uid_, &nw);
        print_waves("elim", wave, nw);
        if (cfg_.verbose >= 3)
            std::fprintf(stderr,
                         "[lvl %d] elim host: tasks %.2f ms%s (plans %.2f, graph %.2f with %zu fill blocks "
                         "[slots %.2f, first makers %.2f, memory %.2f, edges %.2f, in lists %.2f], "
                         "descriptors %.2f, tape %.2f), waves %.2f ms\n",
                         ilvl_, (te1 - te0) * 1e3, coupled ? " (coupled: serial build)" : "", (ts1 - te0) * 1e3,
                         (ts2 - ts1) * 1e3, edges_.size() - nedges0, tg_[0] * 1e3, tg_[1] * 1e3, tg_[2] * 1e3,
                         tg_[3] * 1e3, tg_[4] * 1e3, (ts3 - ts2) * 1e3, (te1 - ts3) * 1e3, (wall() - te1) * 1e3);
        // every wave's descriptors first (host threads, one scratch sized for the
        // largest wave), then the uploads and launches in wave order
        std::vector<std::vector<QRJob>> wjobs(nw);
        for (size_t t = 0; t < tasks.size(); ++t) wjobs[wave[t]].push_back(std::move(tasks[t].job));
        const double tw0 = wall();
        size_t maxe = 1;
        for (auto& jobs : wjobs) maxe = std::max(maxe, wave_scratch_elems(jobs));
        T* trbase = static_cast<T*>(scratch_.get(maxe * sizeof(T), stream_));
        std::vector<WaveBuild> builds(nw);
        const std::vector<TrsmTask<T>> no_trsm;
        const std::vector<CopyDesc<T>> no_post;
        // The wave builds (pure functions of their jobs) run on host threads,
        // wave w on lane w mod lanes so that they finish about in wave order,
        // while this thread uploads and launches each wave as soon as it is
        // built, in wave order: the device starts on the first wave instead of
        // waiting for the last build.
        const size_t lanes = std::min<size_t>(std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 8),
                                              (size_t)nw);
        std::unique_ptr<std::atomic<bool>[]> ready(new std::atomic<bool>[nw]);
        for (int w = 0; w < nw; ++w) ready[w] = false;
        std::atomic<bool> failed{false};
        std::exception_ptr berr;
        std::thread producer([&] {
            try {
                host_parallel_for(
                    lanes,
                    [&](size_t b, size_t e) {
                        for (size_t l = b; l < e; ++l)
                            for (size_t w = l; w < (size_t)nw && !failed; w += lanes) {
                                build_wave(wjobs[w], no_trsm, trbase, d_status_, builds[w]);
                                ready[w].store(true, std::memory_order_release);
                            }
                    },
                    1);
            } catch (...) {
                berr = std::current_exception();
                failed = true;
            }
        });
        try {
            for (int w = 0; w < nw; ++w) {
                while (!ready[w].load(std::memory_order_acquire)) {
                    if (failed) break;
                    std::this_thread::yield();
                }
                if (failed) break;
                issue_wave(builds[w], no_trsm, no_post, wall());
            }
        } catch (...) {
            failed = true;
            producer.join();
            throw;
        }
        producer.join();
        if (berr) std::rethrow_exception(berr);
        if (cfg_.verbose >= 3)
            std::fprintf(stderr, "[lvl %d] elim host: %d wave builds and launches %.2f ms\n", ilvl_, nw,
                         (wall() - tw0) * 1e3);
    }

    // ------------------------------------------------------------- scaling (src/tree.cpp:533-580)
    void scale_phase() {
        struct Task {
            QRJob job;
            std::vector<TrsmTask<T>> trsm;
            CopyDesc<T> ident;
            std::vector<int> uids;
        };
        std::vector<Task> tasks;
        for (Cluster* c : cur()) {
            if (!want_sparsify(c)) continue;
            Edge* es = find_out(c, c);
            if (!es) throw std::runtime_error("diagScale: cluster without diagonal block");
            const int rows = c->rsize, cols = c->csize;
            nnzR_ = (unsigned long long)((double)nnzR_ + 0.5 * cols * cols);
            nnzH_ += (unsigned long long)(rows * cols);
            Task t;
            QRJob& j = t.job;
            j.m = rows;
            j.k = cols;
            j.fac = arena_.alloc_n<T>((size_t)rows * std::max(cols, 1));
            j.tau = arena_.alloc_n<T>(std::max(cols, 1));
            j.tp = arena_.alloc_n<T>((size_t)std::max(npanels(cols), 1) * kNB * kNB);
            j.gather.push_back(cp(es->A.p, j.fac, es->A.ld, rows, rows, cols));
            t.uids.push_back(es->A.uid);
            int co = 0, nrow = 0, ncol = 0;
            for (Edge* e : c->in) {
                if (e->n1->elim) continue;
                const int pad = co * rows;
                j.gather.push_back(cp(e->A.p, nullptr, e->A.ld, rows, rows, e->A.cols, 0, pad));
                j.scatter.push_back(cp(nullptr, e->A.p, rows, e->A.ld, rows, e->A.cols, 0, pad));
                t.uids.push_back(e->A.uid);
                co += e->A.cols;
                ++nrow;
            }
            j.ntr = co;
            int hcol = 0;
            for (Edge* e : c->out) {
                if (e->n2->elim || e->n2 == c) continue;
                t.trsm.push_back(TrsmTask<T>{j.fac, e->A.p, rows, cols, e->A.ld, e->A.rows});
                t.uids.push_back(e->A.uid);
                ++ncol;
                hcol += e->A.rows;
            }
            t.ident = cp(nullptr, es->A.p, 0, es->A.ld, rows, cols, 1);
            TapeOp op;
            op.kind = TK_SCALED;
            op.c = c;
            op.fac = j.fac;
            op.tp = j.tp;
            op.m = rows;  // full segment
            op.k = cols;  // head / reflectors
            op.ld = rows;
            tape_.push_back(std::move(op));
            rec(2, rows, cols, nrow, ncol, (long long)co * 100000 + hcol, c->order);
            if (cols == 0) continue;
            tasks.push_back(std::move(t));
        }
        if (tasks.empty()) return;
        std::vector<std::vector<int>> touched;
        for (auto& t : tasks) touched.push_back(std::move(t.uids));
        int nw = 0;
        auto wave = assign_waves(touched, next_uid_, &nw);
        print_waves("scale", wave, nw);
        for (int w = 0; w < nw; ++w) {
            std::vector<QRJob> jobs;
            std::vector<TrsmTask<T>> tr;
            std::vector<CopyDesc<T>> post;
            for (size_t t = 0; t < tasks.size(); ++t) {
                if (wave[t] != w) continue;
                jobs.push_back(std::move(tasks[t].job));
                tr.insert(tr.end(), tasks[t].trsm.begin(), tasks[t].trsm.end());
                post.push_back(tasks[t].ident);
            }
            run_qr_wave(jobs, tr, post);
        }
    }

    // ------------------------------------------------------------- sparsification (src/tree.cpp:992-1114)
    // ------------------------------------------------------------- --scale 0 (sparsify, src/tree.cpp:887-989)
    // Per interface c (square systems): sinv = 1 / sigma_min([A_pp; A_mp]) (QR
    // of the stacked column, then one-sided Jacobi on its R); the RRQR of
    // C = [A_mp^T | sinv A_pp^T A_pm]; A_mp <- rows of R P^T (the same
    // write-back as sparsifyD), A_pp <- A_pp Q (the reflectors applied to
    // A_pp^T, transposed back); the fine cluster takes the last rows of every
    // block in c's row and the corners of the diagonal block (split_edges,
    // src/tree.cpp:480-530), and is eliminated at once. Waves as sparsifyD:
    // every block a task touches lies in its interface's own row or column.
    void sparsify0_phase() {
        std::vector<Cluster*> list;
        std::vector<std::vector<int>> touched;
        for (Cluster* c : cur()) {
            if (!want_sparsify(c)) continue;
            std::vector<int> u;
            for (Edge* e : c->in)
                if (!e->n1->elim) u.push_back(e->A.uid);
            for (Edge* e : c->out)
                if (!e->n2->elim) u.push_back(e->A.uid);
            list.push_back(c);
            touched.push_back(std::move(u));
        }
        if (list.empty()) return;
        int nw = 0;
        auto wave = assign_waves(touched, next_uid_, &nw);
        print_waves("sparsify0", wave, nw);
        std::vector<std::vector<std::vector<long long>>> recs(list.size());
        const int order0 = max_order_;
        fine_of_.assign(list.size(), nullptr);
        for (int w = 0; w < nw; ++w) {
            std::vector<Spars0Job> jobs;
            size_t celems = 0, ielems = 0;
            for (size_t t = 0; t < list.size(); ++t) {
                if (wave[t] != w) continue;
                Cluster* c = list[t];
                if (c->csize == 0) {
                    recs[t] = {{3, 0, 0, 0, c->rsize, 0, c->order}};
                    continue;
                }
                Spars0Job j;
                j.idx = t;
                j.c = c;
                for (Edge* e : c->in)
                    if (!e->n1->elim) { j.apm.push_back(e); j.spm += e->A.cols; }
                for (Edge* e : c->out) {
                    if (e->n2->elim) continue;
                    if (e->n2 != c) { j.amp.push_back(e); j.smp += e->A.rows; }
                    else j.self = e;
                }
                if (!j.self) throw std::runtime_error("sparsify (scale 0): interface without its diagonal block");
                j.m = c->csize;
                j.n = j.smp + j.spm;
                j.ld = std::max((j.n + 3) & ~3, 4);
                j.c_off = celems;
                celems += (size_t)j.m * j.ld;
                j.i_off = ielems;
                ielems += 3 * (size_t)std::max(j.n, 1) + 1;
                celems += 3 * (size_t)std::max(j.n, 1);
                celems = (celems + 31) & ~size_t(31);
                jobs.push_back(std::move(j));
            }
            if (!jobs.empty()) run_sparsify0_wave(jobs, celems, ielems, recs);
        }
        // The fine clusters were created wave by wave; the reference creates them
        // in the interfaces' order, and the order is what its records show: the
        // k-th compressed interface of the list gets the k-th new order.
        int next = order0;
        for (size_t t = 0; t < list.size(); ++t) {
            Cluster* cf = fine_of_[t];
            if (!cf) continue;
            cf->order = next++;
            recs[t][0][6] = cf->order;  // the fine cluster's elimination record
        }
        if (next != max_order_) throw std::logic_error("sparsify (scale 0): fine cluster count");
        for (size_t t = 0; t < list.size(); ++t)
            for (const auto& r : recs[t]) rec(r[0], r[1], r[2], r[3], r[4], r[5], r[6]);
    }
    std::vector<Cluster*> fine_of_;  // sparsify0_phase: the fine cluster of each listed interface

    struct Spars0Job {
        size_t idx = 0;
        Cluster* c = nullptr;
        std::vector<Edge*> apm, amp;
        Edge* self = nullptr;
        int m = 0, n = 0, smp = 0, spm = 0, ld = 0;
        size_t c_off = 0, i_off = 0;
    };

    // One elimination QR job of the listed column blocks H (stacked in order)
    // updating the blocks blk[u][h] of every cluster upd[u]; the tape op and
    // the counters as elim_phase. Returns the job (its descriptors built).
    QRJob fine_elim_job(Cluster* c, const std::vector<Edge*>& H, const std::vector<Cluster*>& upd,
                        const std::vector<std::vector<Edge*>>& blk, std::vector<int>& uids) {
        QRJob j;
        int m = 0;
        for (Edge* e : H) m += e->A.rows;
        const int k = H.front()->A.cols;
        j.m = m;
        j.k = k;
        j.fac = arena_.alloc_n<T>((size_t)m * k);
        j.tau = arena_.alloc_n<T>(k);
        j.tp = arena_.alloc_n<T>((size_t)npanels(k) * kNB * kNB);
        int off = 0;
        for (Edge* e : H) {
            j.gather.push_back(cp(e->A.p, j.fac + off, e->A.ld, m, e->A.rows, k));
            uids.push_back(e->A.uid);
            off += e->A.rows;
        }
        int co = 0;
        for (size_t u = 0; u < upd.size(); ++u) {
            Cluster* n = upd[u];
            off = 0;
            for (Edge* ecn : blk[u]) {
                const int pad = off + co * m;
                j.gather.push_back(cp(ecn->A.p, nullptr, ecn->A.ld, m, ecn->A.rows, n->csize, 0, pad));
                j.scatter.push_back(cp(nullptr, ecn->A.p, m, ecn->A.ld, ecn->A.rows, n->csize, 0, pad));
                uids.push_back(ecn->A.uid);
                off += ecn->A.rows;
            }
            co += n->csize;
            nnzR_ += (unsigned long long)(c->csize * n->csize);
        }
        j.ntr = co;
        nnzH_ += (unsigned long long)(m * k);
        TapeOp op;
        op.kind = TK_QR;
        op.c = c;
        op.fac = j.fac;
        op.tp = j.tp;
        op.m = m;
        op.k = k;
        op.ld = m;
        for (Edge* e : H) op.segs.emplace_back(e->n2, e->n2->rsize);
        for (Edge* e : c->in) op.a12.push_back(A12{e->A.p, e->A.ld, e->A.cols, e->n1});
        tape_.push_back(std::move(op));
        c->elim = true;
        return j;
    }

    // Runs a set of conflict-free QR jobs (the elimination machinery).
    void run_qr_jobs(std::vector<QRJob>& jobs) {
        if (jobs.empty()) return;
        const size_t e = wave_scratch_elems(jobs);
        T* trbase = static_cast<T*>(scratch_.get(std::max<size_t>(e, 1) * sizeof(T), stream_));
        WaveBuild B;
        const std::vector<TrsmTask<T>> no_trsm;
        const std::vector<CopyDesc<T>> no_post;
        build_wave(jobs, no_trsm, trbase, d_status_, B);
        issue_wave(B, no_trsm, no_post, wall());
    }

    void run_sparsify0_wave(std::vector<Spars0Job>& jobs, size_t celems, size_t ielems,
                            std::vector<std::vector<std::vector<long long>>>& recs) {
        const size_t nj = jobs.size();
        // 1. QR of every stacked [A_pp; A_mp] (copies, the factor kept in the arena)
        std::vector<QRJob> apq(nj);
        std::vector<int> ra(nj, 0);
        for (size_t q = 0; q < nj; ++q) {
            auto& j = jobs[q];
            Cluster* c = j.c;
            int rows = j.self->A.rows;
            for (Edge* e : j.amp) rows += e->A.rows;
            ra[q] = rows;
            QRJob& a = apq[q];
            a.m = rows;
            a.k = j.m;
            a.fac = arena_.alloc_n<T>((size_t)rows * j.m);
            a.tau = arena_.alloc_n<T>(j.m);
            a.tp = arena_.alloc_n<T>((size_t)npanels(j.m) * kNB * kNB);
            int off = 0;
            a.gather.push_back(cp(j.self->A.p, a.fac, j.self->A.ld, rows, j.self->A.rows, j.m));
            off += j.self->A.rows;
            for (Edge* e : j.amp) {
                a.gather.push_back(cp(e->A.p, a.fac + off, e->A.ld, rows, e->A.rows, j.m));
                off += e->A.rows;
            }
            (void)c;
        }
        run_qr_jobs(apq);
        // 2. sinv per job (one-sided Jacobi on R), 3. A_pm gathered column-major
        double* d_sinv = desc_arena_.alloc_n<double>(nj);
        std::vector<SigmaTask<T>> sig;
        std::vector<AtbTask<T>> atb;
        std::vector<TileRef> atb_tiles;
        std::vector<CopyDesc<T>> pmg;
        for (size_t q = 0; q < nj; ++q) {
            auto& j = jobs[q];
            T* work = arena_.alloc_n<T>((size_t)j.m * j.m);
            sig.push_back(SigmaTask<T>{apq[q].fac, work, d_sinv + q, ra[q], j.m});
            const int rows = j.self->A.rows;
            T* bpm = j.spm > 0 ? arena_.alloc_n<T>((size_t)rows * j.spm) : nullptr;
            int off = 0;
            for (Edge* e : j.apm) {
                pmg.push_back(cp(e->A.p, bpm + (size_t)off * rows, e->A.ld, rows, rows, e->A.cols));
                off += e->A.cols;
            }
            if (j.spm > 0) {
                const int id = (int)atb.size();
                atb.push_back(AtbTask<T>{j.self->A.p, bpm, nullptr, d_sinv + q, j.self->A.ld, rows, j.ld, rows, j.m,
                                         j.spm, j.smp, 0});
                for (int t0 = 0; t0 < j.spm; t0 += 32) atb_tiles.push_back(TileRef{id, t0 / 32});
            }
        }
        {
            Upload u;
            const size_t o_s = u.add(sig), o_c = u.add(pmg);
            char* d = u.commit(desc_arena_, stream_, pinned_);
            launch_sigma_min<T>(reinterpret_cast<const SigmaTask<T>*>(d + o_s), (int)sig.size(), stream_);
            ++launches_fact_;
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o_c), pmg);
        }
        // 4. C = [A_mp^T | sinv A_pp^T A_pm] and its RRQR
        std::vector<RRQRTaskRM<T>> rt;
        const std::vector<int> ranks = rrqr_batch(
            jobs, celems, ielems, rt,
            [&](const Spars0Job& j, T* C, std::vector<CopyDesc<T>>& g) {
                int cur = 0;
                for (Edge* e : j.amp) {
                    g.push_back(cp(e->A.p, C + cur, e->A.ld, j.ld, e->A.rows, e->A.cols));
                    cur += e->A.rows;
                }
            },
            [&](T* cb) {
                if (atb.empty()) return;
                for (auto& a : atb) {
                    const size_t q = (size_t)(a.sinv - d_sinv);
                    a.C = cb + jobs[q].c_off;
                }
                Upload u;
                const size_t o_a = u.add(atb), o_t = u.add(atb_tiles);
                char* d = u.commit(desc_arena_, stream_, pinned_);
                launch_atb_scaled<T>(reinterpret_cast<const AtbTask<T>*>(d + o_a),
                                     reinterpret_cast<const TileRef*>(d + o_t), (int)atb_tiles.size(), stream_);
                ++launches_fact_;
            });
        // 5. write-back of A_mp, reflectors of C; A_pp <- A_pp Q; split; fine eliminations
        std::vector<SparsWBRM<T>> wb;
        std::vector<SpBlock<T>> blocks;
        std::vector<CopyDesc<T>> tr_in, tr_out, splits;
        std::vector<QRTask<T>> rq;  // A_pp^T <- Q^T A_pp^T
        struct Fine {
            size_t q;
            Cluster* cf;
            int r, rows_old, cols_old;
            T* V;
            T* tp;
        };
        std::vector<Fine> fines;
        double wb_bytes = 0;
        for (size_t q = 0; q < nj; ++q) {
            auto& j = jobs[q];
            Cluster* c = j.c;
            const int r = ranks[q], m = j.m;
            if (r < 0) throw std::runtime_error("sparsify: invalid rank from device");
            if (r >= m) {
                recs[j.idx] = {{3, m, c->csize, j.n, c->rsize, 0, c->order}};
                continue;
            }
            T* V = arena_.alloc_n<T>((size_t)m * std::max(r, 1));
            T* tau = arena_.alloc_n<T>(std::max(r, 1));
            T* tp = arena_.alloc_n<T>((size_t)std::max(npanels(r), 1) * kNB * kNB);
            SparsWBRM<T> w{rt[q].C, rt[q].pos, rt[q].colat, rt[q].tau, V, tau, tp, m, j.ld, r, 0, (int)blocks.size(), 0};
            int cur = 0;
            for (Edge* e : j.amp) {
                blocks.push_back(SpBlock<T>{e->A.p, e->A.ld, e->A.rows, e->A.cols, cur, 0});
                cur += e->A.rows;
            }
            w.nblk = (int)blocks.size() - w.blk0;
            wb.push_back(w);
            wb_bytes += ((double)r * j.n + 2.0 * m * r) * sizeof(T);
            const int rows = j.self->A.rows;
            T* At = arena_.alloc_n<T>((size_t)m * rows);  // A_pp^T (m x rows)
            tr_in.push_back(cp(j.self->A.p, At, j.self->A.ld, m, rows, m, 2));
            rq.push_back(QRTask<T>{V, At, tau, tp, m, r, rows, 1, d_status_});
            tr_out.push_back(cp(At, j.self->A.p, m, j.self->A.ld, m, rows, 2));
            const int nf = m - r;
            Cluster* cf = new_cluster(c->cstart + r, nf, c->rstart + rows - nf, nf, c->id);
            fines.push_back(Fine{q, cf, r, rows, m, V, tp});
        }
        if (!wb.empty()) {
            Upload u2;
            size_t o_w = u2.add(wb), o_b = u2.add(blocks), o_i = u2.add(tr_in), o_q = u2.add(rq);
            int maxr = 0;
            for (auto& x : rq) maxr = std::max(maxr, x.k);
            std::vector<std::vector<TileRef>> tl;
            for (int p = 0; p < maxr; p += kNB) {
                std::vector<TileRef> v;
                for (size_t t = 0; t < rq.size(); ++t) {
                    if (rq[t].k <= p) continue;
                    for (int c0 = 0, ti = 0; c0 < rq[t].ntr; c0 += kTN, ++ti) v.push_back(TileRef{(int)t, ti});
                }
                tl.push_back(std::move(v));
            }
            std::vector<size_t> o_t;
            for (auto& v : tl) o_t.push_back(u2.add(v));
            const size_t o_o = u2.add(tr_out);
            char* d2 = u2.commit(desc_arena_, stream_, pinned_);
            int parts = 1;
            for (const auto& x : wb) parts = std::max(parts, std::max(x.nblk, (x.r + kNB - 1) / kNB));
            timed(KF_SPARS_WB, 0, wb_bytes, [&] {
                launch_spars_wb_rm<T>(reinterpret_cast<const SparsWBRM<T>*>(d2 + o_w),
                                      reinterpret_cast<const SpBlock<T>*>(d2 + o_b), (int)wb.size(), parts, stream_);
            });
            ++launches_fact_;
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d2 + o_i), tr_in);
            for (size_t i = 0; i < tl.size(); ++i) {
                if (tl[i].empty()) continue;
                timed(KF_TRAILING, 0, 0, [&] {
                    launch_trailing<T>(reinterpret_cast<const QRTask<T>*>(d2 + o_q),
                                       reinterpret_cast<const TileRef*>(d2 + o_t[i]), (int)tl[i].size(), (int)i * kNB,
                                       stream_);
                });
                ++launches_fact_;
            }
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d2 + o_o), tr_out);
        }
        // split_edges and the fine clusters' eliminations
        std::vector<QRJob> fjobs;
        for (const Fine& F : fines) {
            auto& j = jobs[F.q];
            Cluster* c = j.c;
            Cluster* cf = F.cf;
            const int r = F.r, nf = F.cols_old - r, rows_new = F.rows_old - nf;
            // tape: Orthogonal (backward part only), Split (with c's sizes before the
            // split), then the fine cluster's QR below, as the reference records them
            TapeOp ot;
            ot.kind = TK_ORTH;
            ot.c = c;
            ot.fac = F.V;
            ot.tp = F.tp;
            ot.m = F.cols_old;
            ot.k = r;
            ot.ld = F.cols_old;
            tape_.push_back(std::move(ot));
            TapeOp st;
            st.kind = TK_SPLIT0;
            st.c = c;
            st.f = cf;
            st.crows = F.rows_old;
            st.ccols = F.cols_old;
            st.rank = nf;
            tape_.push_back(std::move(st));
            // the fine cluster's rows of every block in c's row (A_pm): new blocks
            for (Edge* e : j.apm) {
                Blk b = new_block(nf, e->A.cols);
                splits.push_back(cp(e->A.p + rows_new, b.p, e->A.ld, b.ld, nf, e->A.cols));
                e->A.rows = rows_new;
                Edge* ef = new_edge(e->n1, cf, b);
                cf->in.push_back(ef);
                e->n1->out.push_back(ef);
            }
            // the diagonal block's corners (A_pp after A_pp Q)
            Edge* es = j.self;
            Blk bff = new_block(nf, nf), bfc = new_block(rows_new, nf), bcf = new_block(nf, r);
            splits.push_back(cp(es->A.p + rows_new + (size_t)r * es->A.ld, bff.p, es->A.ld, bff.ld, nf, nf));
            splits.push_back(cp(es->A.p + (size_t)r * es->A.ld, bfc.p, es->A.ld, bfc.ld, rows_new, nf));
            splits.push_back(cp(es->A.p + rows_new, bcf.p, es->A.ld, bcf.ld, nf, r));
            es->A.rows = rows_new;
            es->A.cols = r;
            Edge* eff = new_edge(cf, cf, bff);
            Edge* efc = new_edge(cf, c, bfc);
            Edge* ecf = new_edge(c, cf, bcf);
            cf->out.push_back(eff);  // by order, descending: the fine cluster first, then c
            cf->out.push_back(efc);
            cf->in.push_back(ecf);
            c->out.push_back(ecf);
            // new shapes of c and its column blocks
            for (Edge* e : j.amp) e->A.cols = r;
            c->rsize = rows_new;
            c->csize = r;
            fine_[ilvl_].push_back(cf);
            // eliminate_cluster(cf): H = [cf rows; c rows], updates of its fill set
            std::vector<Cluster*> upd;
            std::vector<std::vector<Edge*>> blk;
            for (Edge* e : j.apm) upd.push_back(e->n1);
            upd.push_back(c);
            std::vector<size_t> order(upd.size());
            for (size_t i = 0; i < upd.size(); ++i) order[i] = i;
            std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return upd[a]->order < upd[b]->order; });
            std::vector<Cluster*> upd_s;
            for (size_t i : order) {
                Cluster* n = upd[i];
                if (n->elim || n == cf) continue;
                if (!upd_s.empty() && upd_s.back() == n) continue;
                upd_s.push_back(n);
                Edge* to_f = n == c ? ecf : find_edge(n, cf);
                Edge* to_c = n == c ? es : find_edge(n, c);
                if (!to_f || !to_c) throw std::runtime_error("sparsify (scale 0): missing block of the fine elimination");
                blk.push_back({to_f, to_c});
            }
            std::vector<int> uids;
            fjobs.push_back(fine_elim_job(cf, {eff, efc}, upd_s, blk, uids));
            int wtr = 0;
            for (Cluster* n : upd_s) wtr += n->csize;
            recs[j.idx] = {{1, cf->rsize + rows_new, nf, (long long)upd_s.size(), 2, wtr, cf->order},
                           {3, F.cols_old, r, j.n, rows_new, 0, c->order}};
            fine_of_[j.idx] = cf;
        }
        if (!splits.empty()) {
            Upload u3;
            const size_t o = u3.add(splits);
            char* d3 = u3.commit(desc_arena_, stream_, pinned_);
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d3 + o), splits);
        }
        run_qr_jobs(fjobs);
    }

    // The first edge of n's out list into the row cluster r.
    static Edge* find_edge(Cluster* n, Cluster* r) {
        for (Edge* e : n->out)
            if (e->n2 == r) return e;
        return nullptr;
    }

    void sparsify_phase() {
        std::vector<Cluster*> list;
        std::vector<std::vector<int>> touched;
        for (Cluster* c : cur()) {
            if (!want_sparsify(c)) continue;
            std::vector<int> u;
            for (Edge* e : c->in)
                if (!e->n1->elim) u.push_back(e->A.uid);
            for (Edge* e : c->out)
                if (!e->n2->elim) u.push_back(e->A.uid);
            list.push_back(c);
            touched.push_back(std::move(u));
        }
        if (list.empty()) return;
        int nw = 0;
        auto wave = assign_waves(touched, next_uid_, &nw);
        print_waves("sparsify", wave, nw);
        std::vector<std::vector<long long>> recs(list.size());
        for (int w = 0; w < nw; ++w) {
            struct Job {
                size_t idx;
                Cluster* c;
                std::vector<Edge*> apm, amp;
                Edge* self;
                int m, n, smp, ld;
                size_t c_off, i_off;
            };
            std::vector<Job> jobs;
            size_t celems = 0, ielems = 0;
            for (size_t t = 0; t < list.size(); ++t) {
                if (wave[t] != w) continue;
                Cluster* c = list[t];
                if (c->csize == 0) {
                    recs[t] = {0, 0, 0, c->rsize};
                    continue;
                }
                Job j;
                j.idx = t;
                j.c = c;
                j.self = nullptr;
                int spm = 0, smp = 0;
                for (Edge* e : c->in)
                    if (!e->n1->elim) { j.apm.push_back(e); spm += e->A.cols; }
                for (Edge* e : c->out) {
                    if (!e->n2->elim && e->n2 != c) { j.amp.push_back(e); smp += e->A.rows; }
                    else if (e->n2 == c) j.self = e;
                }
                j.m = c->csize;
                j.n = smp + spm;
                j.smp = smp;
                j.ld = std::max((j.n + 3) & ~3, 4);  // row stride: 16-byte rows for column vectors
                j.c_off = celems;
                celems += (size_t)j.m * j.ld;
                j.i_off = ielems;
                ielems += 3 * (size_t)std::max(j.n, 1) + 1;
                celems += 3 * (size_t)std::max(j.n, 1);  // tau, vn1, vn2
                celems = (celems + 31) & ~size_t(31);     // next C starts 128-byte aligned (vector loads)
                jobs.push_back(std::move(j));
            }
            const double tw = wall();
            if (!jobs.empty()) run_sparsify_wave(jobs, celems, ielems, recs);
            if (cfg_.verbose >= 2 && !jobs.empty()) {
                int mm = 0, mn = 0;
                for (auto& j : jobs) { mm = std::max(mm, j.m); mn = std::max(mn, j.n); }
                std::fprintf(stderr, "    sparsify wave %d: %zu tasks, max m %d, max n %d, %.2f ms\n", w, jobs.size(),
                             mm, mn, (wall() - tw) * 1e3);
            }
        }
        for (size_t t = 0; t < list.size(); ++t) {
            const auto& r = recs[t];
            rec(3, r[0], r[1], r[2], r[3], 0, list[t]->order);
        }
    }

    // Gathers every job's interface into a row-major C in the wave scratch (row
    // stride j.ld, rows j.m, columns j.n; gather(job, C, descriptors) lists the
    // copies), runs the cluster RRQR on all of them (one launch per cluster
    // size; larger interfaces get more CTAs) and reads the ranks back. rt
    // receives the device task descriptors (C, positions, tau) for the
    // write-back.
    struct NoPre {
        void operator()(T*) const {}
    };
    template <class Job, class Gather, class Pre = NoPre>
    std::vector<int> rrqr_batch(std::vector<Job>& jobs, size_t celems, size_t ielems, std::vector<RRQRTaskRM<T>>& rt,
                                Gather&& gather, Pre&& pre = Pre()) {
        const size_t ibytes = (((ielems + jobs.size()) * sizeof(int)) + 255) & ~size_t(255);
        char* base = static_cast<char*>(scratch_.get(ibytes + celems * sizeof(T), stream_));
        int* ib = reinterpret_cast<int*>(base);
        T* cb = reinterpret_cast<T*>(base + ibytes);
        std::vector<CopyDesc<T>> g;
        rt.clear();
        for (auto& j : jobs) {
            T* C = cb + j.c_off;
            gather(j, C, g);
            const size_t nn = std::max(j.n, 1);
            T* tail = C + (size_t)j.m * j.ld;  // tau, vn1, vn2
            int* ii = ib + jobs.size() + j.i_off;
            int* rk = ib + rt.size();
            rt.push_back(RRQRTaskRM<T>{C, ii, ii + nn, tail, tail + nn, tail + 2 * nn, rk, j.m, j.n, j.ld, 0, cfg_.tol,
                                         d_status_});
        }
        auto cluster_of = [](const Job& j) {
            const double w = (double)j.m * j.n;
            int c = w <= 32768 ? 1 : w <= 131072 ? 2 : w <= 524288 ? 4 : w <= 2097152 ? 8 : 16;
            while (c < 16 && (j.n + c - 1) / c > 4096) c *= 2;  // keep each CTA's slab <= 4096 columns
            return c;
        };
        // Interfaces that fit a 16-CTA cluster take the blocked kernel (its result
        // is the same for every cluster size, so the size is the autotuner's
        // choice); wider ones the unblocked kernel with the cluster size above.
        // Groups: (blocked, size class).
        std::map<std::pair<int, int>, std::vector<int>> groups;
        for (size_t q = 0; q < jobs.size(); ++q) {
            const int blk = rrqr_blk_fits<T>(jobs[q].m, jobs[q].n, 16) ? 1 : 0;
            groups[{blk, cluster_of(jobs[q])}].push_back((int)q);
        }
        // Within a launch, clusters start in task order: the largest interfaces
        // first, so that a launch with more clusters than fit at once does not
        // end on a large one started last. Each task is independent: the order
        // changes no result.
        for (auto& kv : groups)
            std::stable_sort(kv.second.begin(), kv.second.end(), [&](int a, int b) {
                const auto w = [&](int q) {
                    return (double)jobs[q].m * jobs[q].n * std::min(jobs[q].m, jobs[q].n);
                };
                return w(a) > w(b);
            });
        Upload up;
        size_t o_g = up.add(g), o_r = up.add(rt);
        std::map<std::pair<int, int>, size_t> o_ids;
        for (auto& kv : groups) o_ids[kv.first] = up.add(kv.second);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o_g), g);
        pre(cb);  // device work that completes the C matrices (in stream order, before the RRQR)
        Autotuner& tuner = Autotuner::get();
        const bool tuning = tuner.mode() == 1;
        int dev = 0;
        cudaGetDevice(&dev);
        struct Tuned {
            TuneKey key;
            int cluster;
            cudaEvent_t a, b;
            const std::vector<int>* q;
        };
        std::vector<Tuned> tuned;
        std::vector<size_t> rqs;
        // The groups are disjoint sets of interfaces. Without per-launch
        // profiling they run side by side, stream_ and the branch streams taking
        // them in turn, the group with the most work first (its clusters are
        // placed while the SMs are still free); with profiling one after another
        // on stream_ in map order, so that each launch's events time it alone.
        // Neither the order nor the stream changes a result.
        std::vector<decltype(&*groups.begin())> order;
        for (auto& kv : groups) order.push_back(&kv);
        const bool conc = !prof_ && order.size() > 1;
        const int nside = conc ? std::min<int>(kRqSide, (int)order.size() - 1) : 0;
        if (conc) {
            auto work = [&](const std::vector<int>& qs) {
                double w = 0;
                for (int q : qs) w += (double)jobs[q].m * jobs[q].n * std::min(jobs[q].m, jobs[q].n);
                return w;
            };
            std::stable_sort(order.begin(), order.end(),
                             [&](const auto* a, const auto* b) { return work(a->second) > work(b->second); });
            cuda_check(cudaEventRecord(rq_fork_, stream_), "fork");
            for (int i = 0; i < nside; ++i) cuda_check(cudaStreamWaitEvent(rq_side_[i], rq_fork_, 0), "fork");
        }
        for (size_t gi = 0; gi < order.size(); ++gi) {
            auto& kv = *order[gi];
            const int lane_of = conc ? (int)(gi % (size_t)(nside + 1)) : 0;
            cudaStream_t ls = lane_of == 0 ? stream_ : rq_side_[lane_of - 1];
            int maxm = 0, maxn = 0;
            for (int q : kv.second) {
                maxm = std::max(maxm, jobs[q].m);
                maxn = std::max(maxn, jobs[q].n);
            }
            const int nt = (int)kv.second.size();
            const RRQRTaskRM<T>* dt = reinterpret_cast<const RRQRTaskRM<T>*>(d + o_r);
            const int* di = reinterpret_cast<const int*>(d + o_ids[kv.first]);
            if (kv.first.first == 1) {
                // candidates: every cluster size whose slab fits; default: the smallest
                // that puts at least one CTA on every SM, else the largest
                std::vector<int> cands;
                for (int c = 1; c <= 16; c *= 2)
                    if (rrqr_blk_fits<T>(maxm, maxn, c)) cands.push_back(c);
                int dflt = cands.back();
                for (int c : cands)
                    if ((long long)c * nt >= 148) {
                        dflt = c;
                        break;
                    }
                const TuneKey key{0, dev, (int)sizeof(T), Autotuner::bucket(maxm), Autotuner::bucket(maxn),
                                  Autotuner::bucket(nt)};
                int cl = tuner.choose(key, cands, dflt);
                cudaEvent_t ea = nullptr, eb = nullptr;
                if (tuning) {
                    cuda_check(cudaEventCreate(&ea), "event");
                    cuda_check(cudaEventCreate(&eb), "event");
                    cudaEventRecord(ea, ls);
                }
                if (tracing())
                    tag_ = "rrqr_blk n " + std::to_string(nt) + " cl " + std::to_string(cl) + " m " +
                           std::to_string(maxm) + " k " + std::to_string(maxn);
                rqs.push_back(timed(KF_RRQR, 0, 0, [&] {
                    cudaError_t e = launch_rrqr_blk<T>(dt, di, nt, cl, maxm, maxn, ls);
                    while (e != cudaSuccess && cl > 1 && rrqr_blk_fits<T>(maxm, maxn, cl / 2)) {
                        cudaGetLastError();  // a cluster this large did not launch here: halve it
                        cl /= 2;
                        e = launch_rrqr_blk<T>(dt, di, nt, cl, maxm, maxn, ls);
                    }
                    cuda_check(e, "rrqr launch");
                }));
                if (tuning) {
                    cudaEventRecord(eb, ls);
                    tuned.push_back(Tuned{key, cl, ea, eb, &kv.second});
                }
            } else {
                const int cl = kv.first.second;
                rqs.push_back(timed(KF_RRQR, 0, 0, [&] {
                    cudaError_t e = launch_rrqr_rm<T>(dt, di, nt, cl, maxm, maxn, ls);
                    if (e != cudaSuccess && cl > 8) {  // 16-CTA clusters are an opt-in; fall back to 8
                        cudaGetLastError();
                        e = launch_rrqr_rm<T>(dt, di, nt, 8, maxm, maxn, ls);
                    }
                    cuda_check(e, "rrqr launch");
                }));
            }
            ++launches_fact_;
        }
        for (int i = 0; i < nside; ++i) {
            cuda_check(cudaEventRecord(rq_join_[i], rq_side_[i]), "join");
            cuda_check(cudaStreamWaitEvent(stream_, rq_join_[i], 0), "join");
        }
        std::vector<int> ranks(jobs.size());
        const double tw0 = wall();
        cuda_check(cudaMemcpyAsync(ranks.data(), ib, sizeof(int) * jobs.size(), cudaMemcpyDeviceToHost, stream_),
                   "rank");
        cuda_check(cudaStreamSynchronize(stream_), "rank readback");
        t_rank_wait_ += wall() - tw0;
        pinned_.reset();  // every staged upload before the readback has landed
        for (auto& tu : tuned) {  // device time per unit of work (m n (r + 1)) of each tuned launch
            float ms = 0;
            if (cudaEventElapsedTime(&ms, tu.a, tu.b) == cudaSuccess) {
                double work = 0;
                for (int q : *tu.q) {
                    const double r = std::min(std::max(ranks[q], 0), std::min(jobs[q].m, jobs[q].n));
                    work += (double)jobs[q].m * jobs[q].n * (r + 1);
                }
                if (work > 0) tuner.record(tu.key, tu.cluster, ms / work);
            }
            cudaEventDestroy(tu.a);
            cudaEventDestroy(tu.b);
        }
        // rqs is in map order when profiling (the only case with entries to fill)
        size_t gi = 0;
        for (auto& kv : groups) {  // algorithmic work of each launch, now that the ranks are known
            const size_t rq = rqs[gi++];
            if (rq == SIZE_MAX) continue;
            // algorithmic work: the flops of dgeqp3 stopped at rank r, and the
            // bytes of reading C once and writing its factor once (R's first r
            // rows, the r reflectors); the kernels' per-step passes over C run
            // from L2 and shared memory, so they are not counted as HBM bytes
            double f = 0, by = 0;
            for (int q : kv.second) {
                const double m = jobs[q].m, n = jobs[q].n;
                const int r = ranks[q] >= jobs[q].m ? std::min(jobs[q].m, jobs[q].n) : ranks[q];
                f += 4 * m * n * r - 2.0 * r * r * (m + n) + 4.0 / 3.0 * r * r * r;
                by += (m * n + r * n + m * r) * sizeof(T);
            }
            pend_[rq].flops = f;
            pend_[rq].bytes = by;
        }
        return ranks;
    }

    template <class Job>
    void run_sparsify_wave(std::vector<Job>& jobs, size_t celems, size_t ielems,
                           std::vector<std::vector<long long>>& recs) {
        std::vector<RRQRTaskRM<T>> rt;
        const std::vector<int> ranks = rrqr_batch(jobs, celems, ielems, rt, [&](const Job& j, T* C,
                                                                                 std::vector<CopyDesc<T>>& g) {
            // C(i, cur + r) = A_mp(r, i), C(i, smp + c) = A_pm(i, c) (top csize rows of A_pm)
            int cur = 0;
            for (Edge* e : j.amp) {
                g.push_back(cp(e->A.p, C + cur, e->A.ld, j.ld, e->A.rows, e->A.cols));
                cur += e->A.rows;
            }
            for (Edge* e : j.apm) {
                g.push_back(cp(e->A.p, C + cur, e->A.ld, j.ld, j.m, e->A.cols, 2));
                cur += e->A.cols;
            }
        });
        std::vector<SparsWBRM<T>> wb;
        std::vector<SpBlock<T>> blocks;
        std::vector<CopyDesc<T>> pre, post;  // least squares: extra rows of A_pm move up under the new top
        double wb_bytes = 0;
        // order 1.5 (sparsifyD_imp, src/tree.cpp:1117-1257): the E2 term (Q^T A_pm_top)(rank:, :)
        // of every sparsified interface, computed after the write-back from a copy of its
        // block-start A_pm_top (taken with the pre copies) by the panel trailing kernel
        const bool imp = cfg_.order == 1.5f;
        std::vector<QRTask<T>> e2q;
        for (size_t q = 0; q < jobs.size(); ++q) {
            auto& j = jobs[q];
            Cluster* c = j.c;
            const int r = ranks[q];
            const int m = j.m;
            const int nr = c->rsize - c->csize;  // rows beyond the columns (0 for square problems)
            if (r >= m) {
                recs[j.idx] = {m, c->csize, j.n, c->rsize};
                continue;
            }
            if (r < 0) throw std::runtime_error("sparsify: invalid rank from device");
            T* V = arena_.alloc_n<T>((size_t)m * std::max(r, 1));
            T* tau = arena_.alloc_n<T>(std::max(r, 1));
            T* tp = arena_.alloc_n<T>((size_t)std::max(npanels(r), 1) * kNB * kNB);
            SparsWBRM<T> s{rt[q].C, rt[q].pos, rt[q].colat, rt[q].tau, V, tau, tp, m, j.ld, r, 0,
                           (int)blocks.size(), 0};
            int cur = 0;
            for (Edge* e : j.amp) {
                blocks.push_back(SpBlock<T>{e->A.p, e->A.ld, e->A.rows, e->A.cols, cur, 0});
                cur += e->A.rows;
            }
            for (Edge* e : j.apm) {
                blocks.push_back(SpBlock<T>{e->A.p, e->A.ld, e->A.rows, e->A.cols, cur, 1});
                cur += e->A.cols;
            }
            s.nblk = (int)blocks.size() - s.blk0;
            wb.push_back(s);
            wb_bytes += ((double)r * j.n + 2.0 * m * r) * sizeof(T);
            // tape: OrthogonalD then SplitD (pushed before the size change)
            TapeOp od;
            od.kind = TK_ORTHD;
            od.c = c;
            od.fac = V;
            od.tp = tp;
            od.m = m;
            od.k = r;
            od.ld = m;
            tape_.push_back(std::move(od));
            nnzQ_ += (unsigned long long)(m * r);
            const int nf = m - r;
            Cluster* cf = new_cluster(c->cstart + r, nf, c->rstart + c->csize - nf, nf, c->id);
            TapeOp sd;
            sd.kind = TK_SPLITD;
            sd.c = c;
            sd.f = cf;
            sd.crows = c->rsize;
            sd.ccols = c->csize;
            sd.rank = r;
            tape_.push_back(std::move(sd));
            if (nr > 0) {
                // rows [m, m + nr) of every A_pm block become rows [r, r + nr) (through a
                // staging copy: the ranges overlap); the diagonal block's rows [r, r + nr) are zero
                for (Edge* e : j.apm) {
                    T* st = arena_.alloc_n<T>((size_t)nr * std::max(e->A.cols, 1));
                    pre.push_back(cp(e->A.p + m, st, e->A.ld, nr, nr, e->A.cols));
                    post.push_back(cp(st, e->A.p + r, nr, e->A.ld, nr, e->A.cols));
                }
                pre.push_back(cp(nullptr, j.self->A.p + r, 0, j.self->A.ld, nr, r));
            }
            if (imp) {
                int spm = 0;
                for (Edge* e : j.apm) spm += e->A.cols;
                T* G = spm > 0 ? arena_.alloc_n<T>((size_t)m * spm) : nullptr;
                int coff = 0;
                TapeOp fq;
                fq.kind = TK_QR;
                fq.c = cf;
                fq.k = nf;
                for (Edge* e : j.apm) {
                    pre.push_back(cp(e->A.p, G + (size_t)coff * m, e->A.ld, m, m, e->A.cols));
                    Blk b{G + r + (size_t)coff * m, m, nf, e->A.cols, next_uid_++};
                    Edge* e2 = new_edge(e->n1, cf, b);
                    cf->in.push_back(e2);
                    e->n1->out.push_back(e2);
                    fq.a12.push_back(A12{b.p, m, e->A.cols, e->n1});
                    coff += e->A.cols;
                }
                if (spm > 0) e2q.push_back(QRTask<T>{V, G, tau, tp, m, r, spm, 1, d_status_});
                tape_.push_back(std::move(fq));  // QR(cf) right after the SplitD, as the reference
            }
            // new shapes
            for (Edge* e : j.amp) e->A.cols = r;
            for (Edge* e : j.apm) e->A.rows = r + nr;
            j.self->A.rows = r + nr;
            j.self->A.cols = r;
            c->rsize = r + nr;
            c->csize = r;
            fine_[ilvl_].push_back(cf);
            cf->elim = true;
            recs[j.idx] = {m, r, j.n, r + nr};
        }
        if (!pre.empty()) {
            Upload u1;
            const size_t o = u1.add(pre);
            char* d1 = u1.commit(desc_arena_, stream_, pinned_);
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d1 + o), pre);
        }
        if (!wb.empty()) {
            Upload u2;
            size_t o_w = u2.add(wb), o_b = u2.add(blocks);
            char* d2 = u2.commit(desc_arena_, stream_, pinned_);
            int parts = 1;  // CTAs per task: enough for its blocks and its 32-reflector panels
            for (const auto& x : wb) parts = std::max(parts, std::max(x.nblk, (x.r + kNB - 1) / kNB));
            timed(KF_SPARS_WB, 0, wb_bytes, [&] {
                launch_spars_wb_rm<T>(reinterpret_cast<const SparsWBRM<T>*>(d2 + o_w),
                                      reinterpret_cast<const SpBlock<T>*>(d2 + o_b), (int)wb.size(), parts,
                                      stream_);
            });
            ++launches_fact_;
        }
        if (!e2q.empty()) {  // E2 = Q^T A_pm_top, panel by panel (tiles of the copy only)
            int maxr = 0;
            for (auto& q : e2q) maxr = std::max(maxr, q.k);
            std::vector<std::vector<TileRef>> tl;
            for (int p = 0; p < maxr; p += kNB) {
                std::vector<TileRef> v;
                for (size_t t = 0; t < e2q.size(); ++t) {
                    if (e2q[t].k <= p) continue;
                    for (int c0 = 0, ti = 0; c0 < e2q[t].ntr; c0 += kTN, ++ti) v.push_back(TileRef{(int)t, ti});
                }
                tl.push_back(std::move(v));
            }
            Upload u4;
            const size_t o_q = u4.add(e2q);
            std::vector<size_t> o_t;
            for (auto& v : tl) o_t.push_back(u4.add(v));
            char* d4 = u4.commit(desc_arena_, stream_, pinned_);
            for (size_t i = 0; i < tl.size(); ++i) {
                if (tl[i].empty()) continue;
                timed(KF_TRAILING, 0, 0, [&] {
                    launch_trailing<T>(reinterpret_cast<const QRTask<T>*>(d4 + o_q),
                                       reinterpret_cast<const TileRef*>(d4 + o_t[i]), (int)tl[i].size(),
                                       (int)i * kNB, stream_);
                });
                ++launches_fact_;
            }
        }
        if (!post.empty()) {
            Upload u3;
            const size_t o = u3.add(post);
            char* d3 = u3.commit(desc_arena_, stream_, pinned_);
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d3 + o), post);
        }
    }

    // ------------------------------------------------------------- rectangular row shift (src/tree.cpp:319-411)
    // The rows of every cluster eliminated at this level beyond its columns move
    // to the neighbour whose block carries the largest row norm. The norms come
    // from one batched kernel and one readback; the moves are replayed on the
    // host in the reference's order, and every block that grows is rebuilt
    // once (old rows, appended rows, zero padding) by one batched copy.
    void reassign_phase() {
        struct Item {
            Cluster* c;
            std::vector<std::pair<Edge*, int64_t>> normed;  // in-edge, offset of its row norms
        };
        std::vector<Item> items;
        std::vector<RowNormTask<T>> tasks;
        int64_t tot = 0;
        for (Cluster* c : cur()) {
            if (!c->elim || c->rsize == c->csize) continue;
            if (c->rsize < c->csize) throw std::runtime_error("reassign_rows: fewer rows than columns");
            Item it{c, {}};
            const int rs = c->rsize - c->csize;
            for (Edge* e : c->in) {
                if (!find_out(c, e->n1)) continue;  // only column neighbours vote
                tasks.push_back(RowNormTask<T>{e->A.p, e->A.ld, c->csize, rs, e->A.cols, tot});
                it.normed.emplace_back(e, tot);
                tot += rs;
            }
            items.push_back(std::move(it));
        }
        if (items.empty()) return;
        std::vector<double> norms((size_t)std::max<int64_t>(tot, 1), 0.0);
        if (tot > 0) {
            double* d_norms = static_cast<double*>(scratch_.get(sizeof(double) * (size_t)tot, stream_));
            Upload up;
            const size_t o_t = up.add(tasks);
            char* d = up.commit(desc_arena_, stream_, pinned_);
            launch_row_norms<T>(reinterpret_cast<const RowNormTask<T>*>(d + o_t), (int)tasks.size(), (int)tot, d_norms,
                                stream_);
            ++launches_fact_;
            const double tw0 = wall();
            cuda_check(cudaMemcpyAsync(norms.data(), d_norms, sizeof(double) * (size_t)tot, cudaMemcpyDeviceToHost,
                                       stream_),
                       "row norms");
            cuda_check(cudaStreamSynchronize(stream_), "row norm readback");
            t_rank_wait_ += wall() - tw0;
            pinned_.reset();
        }
        // host replay; blocks that change are described as row segments of their final layout
        struct Seg {
            const T* src;  // null: zeros
            int ld, rows;
        };
        std::map<Edge*, std::vector<Seg>> plan;
        std::set<Edge*> fresh;
        auto segs_of = [&](Edge* e) -> std::vector<Seg>& {
            auto f = plan.find(e);
            if (f == plan.end()) {
                std::vector<Seg> v;
                v.push_back(Seg{fresh.count(e) ? nullptr : e->A.p, e->A.ld, e->A.rows});
                f = plan.emplace(e, std::move(v)).first;
            }
            return f->second;
        };
        for (Item& it : items) {
            Cluster* c = it.c;
            const int rs = c->rsize - c->csize;
            std::vector<std::pair<Cluster*, double>> r2c(rs, {c, 0.0});
            for (auto& ne : it.normed)
                for (int i = 0; i < rs; ++i) {
                    const double v = norms[ne.second + i];
                    if (v > r2c[i].second) r2c[i] = {ne.first->n1, v};
                }
            std::vector<int> perm(rs);
            std::iota(perm.begin(), perm.end(), 0);
            std::stable_sort(perm.begin(), perm.end(),
                             [&](int a, int b) { return r2c[a].first->order < r2c[b].first->order; });
            for (Edge* e : c->in) {
                Cluster* nold = e->n1;
                const T* extra = e->A.p + c->csize;  // extra row q of this block: extra + q (ld e->A.ld)
                for (int i = 0; i < rs;) {
                    Cluster* nnew = r2c[perm[i]].first;
                    int inext = i + 1;
                    while (inext < rs && r2c[perm[inext]].first == nnew) ++inext;
                    const int rinc = inext - i;
                    Edge* te = find_out(nold, nnew);
                    if (nold == nnew) {
                        if (!te) throw std::runtime_error("reassign_rows: missing self edge");
                    } else if (!te) {
                        te = add_edge(nold, nnew);
                        fresh.insert(te);
                    }
                    // rows that stay with the eliminated c only extend its own in-block,
                    // of which later steps read the top c->csize rows: not materialised
                    if (nnew != c) {
                        auto& sg = segs_of(te);
                        for (int q = i; q < inext; ++q) sg.push_back(Seg{extra + perm[q], e->A.ld, 1});
                        te->A.rows += rinc;
                    }
                    if (nold == nnew) {
                        TapeOp op;
                        op.kind = TK_REASSIGN;
                        op.c = c;
                        op.f = nnew;
                        op.m = nnew->rsize;  // first new row of nnew's segment
                        op.k = rinc;
                        for (int q = i; q < inext; ++q) op.idx.push_back(c->csize + perm[q]);
                        tape_.push_back(std::move(op));
                        nnew->xcap += rinc;
                    }
                    i = inext;
                }
            }
            for (Edge* eo : c->out) {  // neighbours take their diagonal block's rows; pad their row blocks
                if (eo->n2 == c) continue;
                Cluster* n = eo->n2;
                Edge* fs = find_out(n, n);
                if (!fs) throw std::runtime_error("reassign_rows: neighbour without diagonal block");
                n->rsize = fs->A.rows;
                n->csize = fs->A.cols;
                for (Edge* ei : n->in) {
                    if (ei->n1->elim || !ei->live || ei->A.rows == n->rsize) continue;
                    if (ei->A.rows > n->rsize) throw std::runtime_error("reassign_rows: block taller than its cluster");
                    auto& sg = segs_of(ei);
                    sg.push_back(Seg{nullptr, 0, n->rsize - ei->A.rows});
                    ei->A.rows = n->rsize;
                }
            }
            rec(7, rs, 0, 0, 0, 0, c->order);
        }
        // rebuild every changed block once (fresh storage reads as zeros)
        std::vector<CopyDesc<T>> copies;
        std::map<const T*, Blk> moved;
        for (auto& kv : plan) {
            Edge* e = kv.first;
            const int uid = e->A.uid;
            Blk nb = new_block(e->A.rows, e->A.cols);
            nb.uid = uid;
            moved[e->A.p] = nb;
            int r0 = 0;
            for (const Seg& sg : kv.second) {
                if (sg.src && sg.rows > 0 && e->A.cols > 0)
                    copies.push_back(cp(sg.src, nb.p + r0, sg.ld, nb.ld, sg.rows, e->A.cols));
                r0 += sg.rows;
            }
            if (r0 != e->A.rows) throw std::runtime_error("reassign_rows: row plan mismatch");
            e->A = nb;
        }
        for (TapeOp& t : tape_)  // back-substitutions recorded earlier read the rebuilt blocks
            for (A12& a : t.a12) {
                auto f = moved.find(a.B);
                if (f != moved.end()) {
                    a.B = f->second.p;
                    a.ld = f->second.ld;
                }
            }
        if (!copies.empty()) {
            Upload up;
            const size_t o = up.add(copies);
            char* d = up.commit(desc_arena_, stream_, pinned_);
            issue_copies(reinterpret_cast<const CopyDesc<T>*>(d + o), copies);
        }
    }

    // ------------------------------------------------------------- sparsify_extra (src/tree.cpp:1260-1307)
    // The rows of an interface beyond its columns are compressed by a truncated
    // column-pivoted QR of [A_pm extra rows] (rank by the same rule as
    // sparsifyD); only upper(R) P^T is kept, no op. The interfaces' blocks are
    // disjoint, so all compressions of a level run as one batch.
    void extra_phase() {
        struct Job {
            size_t idx;
            Cluster* c;
            std::vector<Edge*> apm;
            int m, n, ld, csize;
            size_t c_off, i_off;
        };
        std::vector<Job> jobs;
        size_t celems = 0, ielems = 0;
        for (Cluster* c : cur()) {
            if (!want_sparsify(c) || c->csize == 0 || c->rsize <= c->csize) continue;
            Job j;
            j.idx = jobs.size();
            j.c = c;
            j.csize = c->csize;
            int spm = 0;
            for (Edge* e : c->in)
                if (!e->n1->elim) { j.apm.push_back(e); spm += e->A.cols; }
            j.m = c->rsize - c->csize;
            j.n = spm;
            j.ld = std::max((j.n + 3) & ~3, 4);
            j.c_off = celems;
            celems += (size_t)j.m * j.ld + 3 * (size_t)std::max(j.n, 1);
            celems = (celems + 31) & ~size_t(31);
            j.i_off = ielems;
            ielems += 3 * (size_t)std::max(j.n, 1) + 1;
            jobs.push_back(std::move(j));
        }
        if (jobs.empty()) return;
        std::vector<RRQRTaskRM<T>> rt;
        const std::vector<int> ranks = rrqr_batch(jobs, celems, ielems, rt, [&](const Job& j, T* C, std::vector<CopyDesc<T>>& g) {
            int cur = 0;
            for (Edge* e : j.apm) {  // C(i, cur + c) = A_pm(csize + i, c)
                g.push_back(cp(e->A.p + j.csize, C + cur, e->A.ld, j.ld, j.m, e->A.cols, 2));
                cur += e->A.cols;
            }
        });
        std::vector<SparsWBRM<T>> wb;
        std::vector<SpBlock<T>> blocks;
        for (size_t q = 0; q < jobs.size(); ++q) {
            Job& j = jobs[q];
            Cluster* c = j.c;
            const int kmax = std::min(j.m, j.n);
            const int r = std::min(ranks[q], kmax);
            if (r < 0) throw std::runtime_error("sparsify_extra: invalid rank from device");
            const int rows_before = c->rsize;
            if (r > 0) {
                SparsWBRM<T> w{rt[q].C, rt[q].pos, rt[q].colat, rt[q].tau, nullptr, nullptr, nullptr, j.m, j.ld, r, 0,
                               (int)blocks.size(), 0};
                int cur = 0;
                for (Edge* e : j.apm) {
                    blocks.push_back(SpBlock<T>{e->A.p + j.csize, e->A.ld, r, e->A.cols, cur, 1});
                    cur += e->A.cols;
                }
                w.nblk = (int)blocks.size() - w.blk0;
                wb.push_back(w);
            }
            const int rows_after = j.csize + r;
            for (Edge* e : j.apm) e->A.rows = rows_after;
            Edge* es = find_out(c, c);
            if (!es) throw std::runtime_error("sparsify_extra: cluster without diagonal block");
            es->A.rows = rows_after;
            c->rsize = rows_after;
            rec(8, rows_before, rows_after, 0, 0, 0, c->order);
        }
        if (!wb.empty()) {
            Upload u2;
            const size_t o_w = u2.add(wb), o_b = u2.add(blocks);
            char* d2 = u2.commit(desc_arena_, stream_, pinned_);
            int parts = 1;
            for (const auto& x : wb) parts = std::max(parts, x.nblk);
            timed(KF_SPARS_WB, 0, 0, [&] {
                launch_spars_wb_rm<T>(reinterpret_cast<const SparsWBRM<T>*>(d2 + o_w),
                                      reinterpret_cast<const SpBlock<T>*>(d2 + o_b), (int)wb.size(), parts, stream_);
            });
            ++launches_fact_;
        }
    }

    // ------------------------------------------------------------- merge (src/tree.cpp:414-475, 872-881)
    void merge_all() {
        const double tm0 = wall();
        ++cur_bottom_;
        for (Cluster* s : cur()) {
            int rs = 0, cs = 0;
            for (Cluster* so : s->children) {
                so->rposparent = rs;
                so->cposparent = cs;
                rs += so->rsize;
                cs += so->csize;
            }
            s->rsize = rs;
            s->csize = cs;
            s->rsize_org = rs;
            s->csize_org = cs;
            s->xcap = rs;
            TapeOp op;
            op.kind = TK_MERGE;
            op.c = s;
            tape_.push_back(std::move(op));
            rec(4, rs, cs, (long long)s->children.size(), 0, 0, s->order);
        }
        const double tm1 = wall();
        double t_nb = 0, t_add = 0, t_sort = 0, t_cp = 0;
        struct Move {  // one child block into its parent block
            Edge* eo;
            Cluster* so;
            Cluster* np;  // the parent of the block's row cluster
            int roff;     // row offset of that row cluster in its parent
        };
        const std::vector<Cluster*>& par = cur();
        const size_t np = par.size();
        std::unordered_map<const Cluster*, int> pidx;  // parent -> position in par
        pidx.reserve(np * 2);
        for (size_t pi = 0; pi < np; ++pi) pidx[par[pi]] = (int)pi;
        std::vector<std::vector<Cluster*>> nbs(np);
        std::vector<std::vector<Move>> moves(np);
        std::vector<std::vector<std::pair<Cluster*, Edge*>>> pes(np);  // parent edges by neighbour address
        std::vector<size_t> pbytes(np, 0);
        // 1. (threads) each parent's neighbour parents, the bytes of its new blocks
        //    and its child-block moves: reads only its own children's edges
        host_parallel_for(np, [&](size_t b, size_t e) {
            for (size_t pi = b; pi < e; ++pi) {
                Cluster* s = par[pi];
                std::vector<Cluster*>& nb = nbs[pi];
                for (Cluster* so : s->children)
                    for (Edge* eo : so->out) {
                        const Cluster* nold = eo->n2;
                        if (nold->elim) continue;
                        nb.push_back(nold->parent);
                        if (!eo->live) continue;
                        if (eo->A.rows != nold->rsize || eo->A.cols != so->csize)
                            throw std::runtime_error("merge: block shape mismatch");
                        moves[pi].push_back(Move{eo, so, nold->parent, nold->rposparent});
                    }
                std::sort(nb.begin(), nb.end(),
                          [](const Cluster* a, const Cluster* b) { return a->order < b->order; });
                nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
                for (Cluster* n : nb) pbytes[pi] += Arena::rounded(block_elems(n->rsize, s->csize) * sizeof(T));
            }
        });
        const double tb = wall();
        t_nb = tb - tm1;
        // 2. the parent edges in the reference's order (parents in order, each
        //    parent's neighbours by order): uids and edge slots by prefix sums,
        //    each parent's blocks from one arena range in that order. Then (threads)
        //    the edges and out lists per parent, and the in lists per neighbour,
        //    each list in the order one parent after another gives it.
        std::vector<size_t> ebase(np + 1, 0);
        for (size_t pi = 0; pi < np; ++pi) ebase[pi + 1] = ebase[pi] + nbs[pi].size();
        const size_t ne = ebase[np], e0 = edges_.size();
        if (ne > size_t(std::numeric_limits<int>::max() - next_uid_))
            throw std::runtime_error("merge: block uid overflow");
        const int uid0 = next_uid_;
        next_uid_ += (int)ne;
        std::vector<char*> pbase(np, nullptr);
        for (size_t pi = 0; pi < np; ++pi)
            if (pbytes[pi]) pbase[pi] = static_cast<char*>(arena_.alloc(pbytes[pi]));
        edges_.resize(e0 + ne);
        std::vector<int> tgt(ne);  // the neighbour's position in par
        host_parallel_for(np, [&](size_t b, size_t e) {
            for (size_t pi = b; pi < e; ++pi) {
                Cluster* s = par[pi];
                char* p = pbase[pi];
                s->out.reserve(s->out.size() + nbs[pi].size());
                pes[pi].reserve(nbs[pi].size());
                for (size_t j = 0; j < nbs[pi].size(); ++j) {
                    Cluster* n = nbs[pi][j];
                    const size_t q = ebase[pi] + j;
                    Blk bk;
                    bk.rows = n->rsize;
                    bk.cols = s->csize;
                    bk.ld = std::max(bk.rows, 1);
                    bk.p = reinterpret_cast<T*>(p);
                    bk.uid = uid0 + (int)q;
                    p += Arena::rounded(block_elems(bk.rows, bk.cols) * sizeof(T));
                    Edge& ed = edges_[e0 + q];
                    ed = Edge{s, n, bk, true};
                    s->out.push_back(&ed);
                    pes[pi].emplace_back(n, &ed);
                    const auto it = pidx.find(n);
                    if (it == pidx.end()) throw std::runtime_error("merge: neighbour outside the level");
                    tgt[q] = n == s ? -1 : it->second;
                }
            }
        });
        {
            std::vector<int> nin(np, 0);
            for (int t : tgt)
                if (t >= 0) ++nin[t];
            for (size_t t = 0; t < np; ++t) par[t]->in.reserve(par[t]->in.size() + nin[t]);
            const size_t hw = std::max(1u, std::thread::hardware_concurrency());
            const size_t nth = std::max<size_t>(1, std::min<size_t>({hw, 8, np / 256}));
            host_parallel_for(nth, [&](size_t b, size_t e) {
                for (size_t k = b; k < e; ++k) {  // neighbours [np k / nth, np (k + 1) / nth)
                    const int lo = (int)(np * k / nth), hi = (int)(np * (k + 1) / nth);
                    for (size_t q = 0; q < ne; ++q)
                        if (tgt[q] >= lo && tgt[q] < hi) par[tgt[q]]->in.push_back(&edges_[e0 + q]);
                }
            }, 1);
        }
        const double tc = wall();
        t_add = tc - tb;
        // 3. (threads) each parent sorts its out list and writes its copies into
        //    the pinned stage at its prefix-sum position
        std::vector<size_t> cbase(np + 1, 0);
        for (size_t pi = 0; pi < np; ++pi) cbase[pi + 1] = cbase[pi] + moves[pi].size();
        const size_t ncp = cbase[np];
        CopyDesc<T>* hcp = ncp ? reinterpret_cast<CopyDesc<T>*>(pinned_.get(ncp * sizeof(CopyDesc<T>))) : nullptr;
        std::vector<double> pby(np, 0);
        std::vector<int> pmaxc(np, 0);
        host_parallel_for(np, [&](size_t b, size_t e) {
            for (size_t pi = b; pi < e; ++pi) {
                Cluster* s = par[pi];
                std::stable_sort(s->out.begin(), s->out.end(),
                                 [](Edge* a, Edge* b) { return a->n2->order < b->n2->order; });
                auto& pe = pes[pi];
                std::sort(pe.begin(), pe.end());
                CopyDesc<T>* o = hcp + cbase[pi];
                for (const Move& mv : moves[pi]) {
                    auto it = std::lower_bound(pe.begin(), pe.end(), std::make_pair(mv.np, (Edge*)nullptr));
                    if (it == pe.end() || it->first != mv.np) throw std::runtime_error("merge: missing parent edge");
                    Edge* f = it->second;
                    Edge* eo = mv.eo;
                    *o++ = cp(eo->A.p, f->A.p + mv.roff + (size_t)mv.so->cposparent * f->A.ld, eo->A.ld, f->A.ld,
                              eo->A.rows, eo->A.cols);
                    pby[pi] += 2.0 * eo->A.rows * eo->A.cols * sizeof(T);
                    pmaxc[pi] = std::max(pmaxc[pi], eo->A.cols);
                    eo->live = false;
                }
            }
        });
        const double td = wall();
        t_sort = td - tc;
        t_cp = 0;
        const double tm2 = wall();
        if (ncp) {
            double by = 0;
            int maxc = 0;
            for (size_t pi = 0; pi < np; ++pi) {
                by += pby[pi];
                maxc = std::max(maxc, pmaxc[pi]);
            }
            const size_t bytes = ncp * sizeof(CopyDesc<T>);
            auto* d = static_cast<CopyDesc<T>*>(desc_arena_.alloc(bytes));
            cuda_check(cudaMemcpyAsync(d, hcp, bytes, cudaMemcpyHostToDevice, stream_), "merge copy list upload");
            timed(KF_COPY, 0, by, [&] { launch_copy<T>(d, (int)ncp, maxc, stream_); });
            ++launches_fact_;
        }
        if (cfg_.verbose >= 3)
            std::fprintf(stderr,
                         "[lvl %d] merge host: %zu clusters, %zu copies, sizes %.2f ms, neighbours %.2f, edges %.2f, "
                         "sort + copy list %.2f, concatenate %.2f, upload+launch %.2f\n",
                         ilvl_, cur().size(), ncp, (tm1 - tm0) * 1e3, t_nb * 1e3, t_add * 1e3,
                         t_sort * 1e3, t_cp * 1e3, (wall() - tm2) * 1e3);
    }

    // Diagnostic (verbose >= 2): tasks and waves of one phase.
    void print_waves(const char* phase, const std::vector<int>& wave, int nw) {
        if (cfg_.verbose < 2) return;
        std::vector<int> cnt(nw, 0);
        for (int w : wave) cnt[w]++;
        int mx = 0;
        for (int c : cnt) mx = std::max(mx, c);
        std::fprintf(stderr, "[lvl %d] %-8s tasks %zu waves %d max/wave %d\n", ilvl_, phase, wave.size(), nw, mx);
    }

    void print_level(cudaEvent_t* ev, std::pair<int, int> ts) {
        cudaEventSynchronize(ev[6]);
        float ms[6];
        for (int p = 0; p < 6; ++p) cudaEventElapsedTime(&ms[p], ev[p], ev[p + 1]);
        std::printf(
            "lvl: %d    update fill-in: %.3f  elmn: %.3f  shift: %.3f  scale: %.3f  sprsfy: %.3f  merge: %.3f  "
            "size top_sep: %d, %d   a.r top_sep: %.3f\n",
            ilvl_, ms[0] * 1e-3, ms[1] * 1e-3, ms[2] * 1e-3, ms[3] * 1e-3, ms[4] * 1e-3, ms[5] * 1e-3, ts.first,
            ts.second, ts.second ? (double)ts.first / ts.second : 0.0);
    }

    // ------------------------------------------------------------- solve plan
    // R^-1 of every QR and ScaleD op with k <= kRinvMax: the identity (zeroed
    // arena memory plus a unit diagonal) run through the TRSM, X <- X R^-1,
    // once per factorization. The solve's triangular ops then apply R^-1 (or
    // R^-T) as one product instead of a chain of diagonal blocks.
    void form_rinv() {
        std::vector<TrsmTask<T>> tasks;
        std::vector<TileRef> tiles;
        double f = 0, by = 0;
        for (TapeOp& t : tape_) {
            if (!((t.kind == TK_QR || t.kind == TK_SCALED) && t.fac != nullptr)) continue;
            if (t.k < 1 || t.k > kRinvMax) continue;
            T* X = arena_.template alloc_n<T>((size_t)t.k * t.k);
            t.rinv = X;
            const int id = (int)tasks.size();
            tasks.push_back(TrsmTask<T>{t.fac, X, t.ld, t.k, t.k, t.k});
            for (int r = 0; r < t.k; r += 128) tiles.push_back(TileRef{id, r / 128});
            f += (double)t.k * t.k * t.k;
            by += (1.5 * t.k * t.k) * sizeof(T);
        }
        if (tasks.empty()) return;
        Upload up;
        const size_t o_t = up.add(tasks), o_l = up.add(tiles);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        const TrsmTask<T>* dt = reinterpret_cast<const TrsmTask<T>*>(d + o_t);
        launch_unit_diag<T>(dt, (int)tasks.size(), stream_);
        timed(KF_TRSM, f, by, [&] {
            launch_trsm<T>(dt, reinterpret_cast<const TileRef*>(d + o_l), (int)tiles.size(), stream_);
        });
        launches_fact_ += 2;
    }

    // Q^T of every ScaleD and OrthD op, and of every elimination QR op whose
    // rows are one cluster's segment, of kDenseQMin..kRinvMax rows with at
    // least half as many reflectors as rows: the identity run through the
    // compact-WY update (the elimination's trailing kernel, panel by panel),
    // once per factorization. The solve's sweeps then apply Q^T (and OrthD's
    // Q, as its transpose) as one dense product split over a thread-block
    // cluster, instead of a chain of one reduction per reflector panel.
    static constexpr int kDenseQMin = 64;
    void form_qt() {
        std::vector<QRTask<T>> tasks;
        std::vector<TrsmTask<T>> diag;
        double f = 0, by = 0;
        int maxk = 0;
        for (TapeOp& t : tape_) {
            // elimination QR ops qualify when their rows are one cluster's segment
            const bool qr1 = t.kind == TK_QR && t.segs.size() == 1 && t.segs[0].second == t.m;
            if (!((t.kind == TK_SCALED || t.kind == TK_ORTHD || qr1) && t.fac != nullptr && t.k >= 1)) continue;
            if (t.m < kDenseQMin || t.m > kRinvMax || 2 * t.k < t.m || t.ld != t.m) continue;
            T* M = arena_.alloc_n<T>((size_t)t.m * t.m);
            t.qt = M;
            tasks.push_back(QRTask<T>{const_cast<T*>(t.fac), M, nullptr, const_cast<T*>(t.tp), t.m, t.k, t.m, 1,
                                      nullptr});
            diag.push_back(TrsmTask<T>{nullptr, M, t.m, t.m, t.m, t.m});
            maxk = std::max(maxk, t.k);
            f += 4.0 * t.m * t.m * t.k - 2.0 * t.m * t.k * t.k;
            by += (2.0 * t.m * t.m + (double)t.m * t.k) * sizeof(T);
        }
        if (tasks.empty()) return;
        Upload up;
        const size_t o_q = up.add(tasks), o_d = up.add(diag);
        // the tile lists of every panel step (alive until the commit: add()
        // records where they lie)
        std::vector<std::vector<TileRef>> tl;
        for (int p = 0; p < maxk; p += kNB) {
            std::vector<TileRef> v;
            for (size_t i = 0; i < tasks.size(); ++i) {
                if (tasks[i].k <= p) continue;
                for (int c0 = 0, ti = 0; c0 < tasks[i].ntr; c0 += kTN, ++ti) v.push_back(TileRef{(int)i, ti});
            }
            tl.push_back(std::move(v));
        }
        std::vector<size_t> o_t;
        for (const auto& v : tl) {
            o_t.push_back(v.empty() ? size_t(0) : up.add(v));
            o_t.push_back(v.size());
        }
        char* d = up.commit(desc_arena_, stream_, pinned_);
        launch_unit_diag<T>(reinterpret_cast<const TrsmTask<T>*>(d + o_d), (int)diag.size(), stream_);
        ++launches_fact_;
        const double per = f / std::max<size_t>(1, o_t.size() / 2), pby = by / std::max<size_t>(1, o_t.size() / 2);
        for (size_t i = 0; i < o_t.size(); i += 2) {
            if (o_t[i + 1] == 0) continue;
            timed(KF_TRAILING, per, pby, [&] {
                launch_trailing<T>(reinterpret_cast<const QRTask<T>*>(d + o_q),
                                   reinterpret_cast<const TileRef*>(d + o_t[i]), (int)o_t[i + 1], (int)(i / 2) * kNB,
                                   stream_);
            });
            ++launches_fact_;
        }
    }

    void build_solve_plan() {
        if (rect_) {
            build_nrml_plan();
            return;
        }
        const double tq0 = wall();
        form_rinv();
        form_qt();
        int64_t xtot = 0;
        for (auto& c : clusters_) {
            c->xoff = xtot;
            xtot += std::max(c->xcap, 1);
        }
        xbuf_ = arena_.alloc_n<T>(xtot);
        xtot_ = xtot;
        d_bin_ = arena_.alloc_n<double>(nrows_);
        d_xout_ = arena_.alloc_n<double>(ncols_);
        d_adj_in_ = arena_.alloc_n<double>(ncols_);
        d_adj_out_ = arena_.alloc_n<double>(nrows_);
        std::vector<int> src, dst;
        std::vector<int64_t> xin, xo;
        src.reserve(nrows_);
        xin.reserve(nrows_);
        dst.reserve(ncols_);
        xo.reserve(ncols_);
        for (Cluster* c : bottoms_[0]) {
            for (int i = 0; i < c->rsize_org; ++i) {
                src.push_back(rperm_[c->rstart + i]);
                xin.push_back(c->xoff + i);
            }
            for (int i = 0; i < c->csize_org; ++i) {
                dst.push_back(cperm_[c->cstart + i]);
                xo.push_back(c->xoff + i);
            }
        }
        const double tq1 = wall();
        std::vector<XSeg> segs;
        std::vector<GemvRef<T>> gemv;
        std::vector<POp> fwd, bwd;
        fwd.reserve(tape_.size());
        bwd.reserve(tape_.size());
        auto ptr = [](const T* p) { return (int64_t)reinterpret_cast<uintptr_t>(p); };
        // every op's segment and GEMV entries at offsets fixed in tape order, so
        // the ops are built on host threads into the same arrays
        const size_t ntape = tape_.size();
        std::vector<size_t> seg_off(ntape + 1, 0), gemv_off(ntape + 1, 0);
        for (size_t i = 0; i < ntape; ++i) {
            const TapeOp& t = tape_[i];
            seg_off[i + 1] = seg_off[i] + (t.kind == TK_QR ? t.segs.size() : t.kind == TK_MERGE ? t.c->children.size() : 0);
            gemv_off[i + 1] = gemv_off[i] + (t.kind == TK_QR ? t.a12.size() : 0);
        }
        segs.resize(seg_off[ntape]);
        gemv.resize(gemv_off[ntape]);
        std::vector<POp> F(ntape), B(ntape);
        host_parallel_for(ntape, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            const TapeOp& t = tape_[i];
            POp& f = F[i];
            POp& b = B[i];
            size_t sq = seg_off[i], gq = gemv_off[i];
            switch (t.kind) {
                case TK_QR: {
                    f.op = SolveOp{SK_APPLYQ, 0, t.m, t.k, t.ld, 0, 0, 0, ptr(t.fac), ptr(t.tp), 0,
                                   (int)seg_off[i], (int)t.segs.size()};
                    f.rd.reserve(t.segs.size());
                    f.wr.reserve(t.segs.size());
                    b.rd.reserve(t.a12.size() + 1);
                    for (auto& s : t.segs) {
                        segs[sq++] = XSeg{s.first->xoff, s.second, 0};
                        f.rd.push_back(s.first);
                        f.wr.push_back(s.first);
                    }
                    if (t.qt) {  // one segment (form_qt): contiguous x, Q^T formed
                        f.op.x0 = t.segs[0].first->xoff;
                        f.op.nseg = 0;
                        f.op.p2 = ptr(t.qt);
                    }
                    f.smem = t.m;
                    b.op = SolveOp{SK_TRI, 0, t.k, 0, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.rinv), 0,
                                   (int)gemv_off[i], (int)t.a12.size()};
                    for (auto& a : t.a12) {
                        gemv[gq++] = GemvRef<T>{ptr(a.B), a.n1->xoff, a.ld, a.s};
                        b.rd.push_back(a.n1);
                    }
                    b.rd.push_back(t.c);
                    b.wr.push_back(t.c);
                    b.smem = t.rinv ? 2 * t.k : t.k;
                    break;
                }
                case TK_SCALED:
                    f.op = SolveOp{SK_APPLYQ, 0, t.m, t.k, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.tp), ptr(t.qt),
                                   0, 0};
                    f.rd = f.wr = {t.c};
                    f.smem = t.m;
                    b.op = SolveOp{SK_TRI, 0, t.k, 0, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.rinv), 0, 0, 0};
                    b.rd = b.wr = {t.c};
                    b.smem = t.rinv ? 2 * t.k : t.k;
                    break;
                case TK_ORTHD:
                    f.op = SolveOp{SK_APPLYQ, 0, t.m, t.k, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.tp), ptr(t.qt),
                                   0, 0};
                    f.rd = f.wr = {t.c};
                    f.smem = t.m;
                    b.op = f.op;
                    b.op.dir = 1;
                    b.rd = b.wr = {t.c};
                    b.smem = t.m;
                    break;
                case TK_SPLITD:
                    f.op = SolveOp{SK_SPLIT, 0, t.crows, t.ccols, t.rank, 0, t.c->xoff, t.f->xoff, 0, 0, 0, 0, 0};
                    f.rd = {t.c};
                    f.wr = {t.c, t.f};
                    f.smem = t.crows;
                    b.op = f.op;
                    b.op.dir = 1;
                    b.rd = {t.c, t.f};
                    b.wr = {t.c};
                    b.smem = t.crows;
                    break;
                case TK_ORTH:  // backward only: x(c)[0, m) <- Q x(c)[0, m)
                    b.op = SolveOp{SK_APPLYQ, 1, t.m, t.k, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.tp), 0, 0, 0};
                    b.rd = b.wr = {t.c};
                    b.smem = t.m;
                    break;
                case TK_SPLIT0:
                    f.op = SolveOp{SK_SPLIT0, 0, t.crows, t.ccols, t.rank, 0, t.c->xoff, t.f->xoff, 0, 0, 0, 0, 0};
                    f.rd = {t.c};
                    f.wr = {t.f};
                    f.smem = 0;
                    b.op = f.op;
                    b.op.dir = 1;
                    b.rd = {t.f};
                    b.wr = {t.c};
                    b.smem = 0;
                    break;
                case TK_MERGE: {
                    f.op = SolveOp{SK_MERGE, 0, 0, 0, 0, 0, t.c->xoff, 0, 0, 0, 0, (int)seg_off[i],
                                   (int)t.c->children.size()};
                    for (Cluster* ch : t.c->children) {
                        segs[sq++] = XSeg{ch->xoff, ch->rsize, ch->csize};
                        f.rd.push_back(ch);
                        b.wr.push_back(ch);
                    }
                    f.wr = {t.c};
                    b.rd = {t.c};
                    b.op = f.op;
                    b.op.dir = 1;
                    f.smem = b.smem = 0;
                    break;
                }
                default:  // TK_REASSIGN: least squares only
                    break;
            }
        }
        }, 256);
        for (size_t i = 0; i < ntape; ++i) {
            // the QR op of an order-1.5 fine cluster has no forward part (its T is zero),
            // and neither has the Orthogonal op of --scale 0
            if (!(tape_[i].kind == TK_QR && tape_[i].fac == nullptr) && tape_[i].kind != TK_ORTH)
                fwd.push_back(std::move(F[i]));
            bwd.push_back(std::move(B[i]));
        }
        std::reverse(bwd.begin(), bwd.end());
        const double tq2 = wall();
        gemv_cols_.clear();
        for (auto& g : gemv) gemv_cols_.push_back(g.s);
        std::vector<std::vector<int>> fw, bw;
        {  // the two sweeps are scheduled independently: the backward one on a second thread
            std::exception_ptr err;
            std::thread tb([&] {
                try {
                    schedule_ops(bwd, bw);
                } catch (...) {
                    err = std::current_exception();
                }
            });
            schedule_ops(fwd, fw);
            tb.join();
            if (err) std::rethrow_exception(err);
        }
        std::vector<SolveOp> all;
        std::vector<WMeta> fm, bm;
        pack_waves(fwd, fw, all, fm);
        pack_waves(bwd, bw, all, bm);
        const double tq3 = wall();
        Upload up;
        size_t o_ops = up.add(all), o_segs = up.add(segs), o_gemv = up.add(gemv), o_src = up.add(src),
               o_dst = up.add(dst), o_xin = up.add(xin), o_xo = up.add(xo);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        const SolveOp* d_ops = reinterpret_cast<const SolveOp*>(d + o_ops);
        d_segs_ = reinterpret_cast<const XSeg*>(d + o_segs);
        d_gemv_ = reinterpret_cast<const GemvRef<T>*>(d + o_gemv);
        d_src_ = reinterpret_cast<int*>(d + o_src);
        d_dst_ = reinterpret_cast<int*>(d + o_dst);
        d_xin_ = reinterpret_cast<int64_t*>(d + o_xin);
        d_xout_pos_ = reinterpret_cast<int64_t*>(d + o_xo);
        fwd_waves_.clear();
        bwd_waves_.clear();
        for (auto& mt : fm) fwd_waves_.push_back(make_wave(d_ops, mt));
        for (auto& mt : bm) bwd_waves_.push_back(make_wave(d_ops, mt));
        adj_waves_.clear();  // built on the first adjoint solve
        plan_fwd_ = std::move(fwd);
        plan_bwd_ = std::move(bwd);
        nin_ = (int)src.size();
        nout_ = (int)dst.size();
        // one application reads every stored factor word once (nnzH + nnzR + nnzQ) plus the
        // right-hand side and solution vectors
        solve_bytes_ = (double)(nnzH_ + nnzR_ + nnzQ_) * sizeof(T) + 8.0 * (nrows_ + ncols_);
        if (cfg_.verbose >= 3)
            std::fprintf(stderr,
                         "solve plan host: %zu tape ops, buffers + maps %.2f ms, ops %.2f, waves %.2f, upload %.2f\n",
                         tape_.size(), (tq1 - tq0) * 1e3, (tq2 - tq1) * 1e3, (tq3 - tq2) * 1e3, (wall() - tq3) * 1e3);
        const size_t smem_cap = (200 * 1024) / sizeof(T);
        for (auto* ws : {&fwd_waves_, &bwd_waves_})
            for (auto& w : *ws)
                if ((size_t)w.smem > smem_cap)
                    throw std::runtime_error("solve: a cluster exceeds the shared-memory vector capacity");
    }
    int nin_ = 0, nout_ = 0;

    // Least-squares preconditioner (Tree::solve_nrml, src/tree.cpp:1471-1517):
    // x = M_n b with M_n ~ (A^T A)^{-1}, applied as four sweeps of the tape:
    // (A) the transposed ops forward on xt (R^T solves with x_n -= A12^T z,
    // Q^T of the sparsifications, transposed merges and splits), (B) the
    // transposed ops backward without QR / ScaleD / OrthogonalD (reassignments,
    // merges, splits), then xt -> x on the leaves, (C) the ops forward without
    // QR / ScaleD / OrthogonalD, and (D) the ops backward (R solves, Q of the
    // sparsifications, merges, splits). One CUDA graph.
    void build_nrml_plan() {
        int64_t xtot = 0;
        for (auto& c : clusters_) {
            c->xoff = xtot;
            xtot += std::max(c->xcap, 1);
        }
        xtot_ = xtot;
        xbuf_ = arena_.alloc_n<T>(xtot);
        xtbuf_ = arena_.alloc_n<T>(xtot);
        d_bin_ = arena_.alloc_n<double>(ncols_);
        d_xout_ = arena_.alloc_n<double>(ncols_);
        std::vector<int> src, dst;
        std::vector<int64_t> xin, xo, leaf;
        for (Cluster* c : bottoms_[0]) {
            for (int i = 0; i < c->csize_org; ++i) {
                src.push_back(cperm_[c->cstart + i]);  // b (length n) enters xt
                xin.push_back(c->xoff + i);
                dst.push_back(cperm_[c->cstart + i]);
                xo.push_back(c->xoff + i);
            }
            for (int i = 0; i < c->rsize_org; ++i) leaf.push_back(c->xoff + i);
        }
        // reassignment index lists first (the ops carry their device addresses)
        std::vector<int> idx;
        std::vector<size_t> idx_off(tape_.size(), 0);
        for (size_t q = 0; q < tape_.size(); ++q)
            if (tape_[q].kind == TK_REASSIGN) {
                idx_off[q] = idx.size();
                idx.insert(idx.end(), tape_[q].idx.begin(), tape_[q].idx.end());
            }
        const int* d_idx = nullptr;
        if (!idx.empty()) {
            Upload ui;
            const size_t o = ui.add(idx);
            d_idx = reinterpret_cast<const int*>(ui.commit(desc_arena_, stream_, pinned_) + o);
        }
        auto ptr = [](const void* p) { return (int64_t)reinterpret_cast<uintptr_t>(p); };
        std::vector<XSeg> segs;
        std::vector<GemvRef<T>> gemv;
        std::vector<POp> sa, sb, sc, sd;
        auto merge_segs = [&](Cluster* c, bool transposed) {
            const int s0 = (int)segs.size();
            for (Cluster* ch : c->children)
                segs.push_back(transposed ? XSeg{ch->xoff, ch->csize, ch->rsize} : XSeg{ch->xoff, ch->rsize, ch->csize});
            return s0;
        };
        for (size_t q = 0; q < tape_.size(); ++q) {
            const TapeOp& t = tape_[q];
            switch (t.kind) {
                case TK_QR: {
                    POp a{};
                    a.op = SolveOp{SK_TRI, 1, t.k, 0, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.rinv), 0,
                                   (int)gemv.size(), (int)t.a12.size()};
                    for (auto& e : t.a12) {
                        gemv.push_back(GemvRef<T>{ptr(e.B), e.n1->xoff, e.ld, e.s});
                        a.rd.push_back(e.n1);
                    }
                    a.rd.push_back(t.c);
                    a.wr = a.rd;
                    a.smem = t.rinv ? 2 * t.k : t.k;
                    POp d = a;
                    d.op.dir = 0;
                    d.wr = {t.c};
                    sa.push_back(a);
                    sd.push_back(d);
                    break;
                }
                case TK_SCALED: {
                    POp a{};
                    a.op = SolveOp{SK_TRI, 1, t.k, 0, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.rinv), 0, 0, 0};
                    a.rd = a.wr = {t.c};
                    a.smem = t.rinv ? 2 * t.k : t.k;
                    POp d = a;
                    d.op.dir = 0;
                    sa.push_back(a);
                    sd.push_back(d);
                    break;
                }
                case TK_ORTHD: {
                    POp a{};
                    a.op = SolveOp{SK_APPLYQ, 0, t.m, t.k, t.ld, 0, t.c->xoff, 0, ptr(t.fac), ptr(t.tp), 0, 0, 0};
                    a.rd = a.wr = {t.c};
                    a.smem = t.m;
                    POp d = a;
                    d.op.dir = 1;
                    sa.push_back(a);
                    sd.push_back(d);
                    break;
                }
                case TK_SPLITD: {
                    POp f{};
                    f.op = SolveOp{SK_SPLIT, 0, t.crows, t.ccols, t.rank, 0, t.c->xoff, t.f->xoff, 0, 0, 0, 0, 0};
                    f.rd = f.wr = {t.c, t.f};
                    f.smem = t.crows;
                    POp b = f;
                    b.op.dir = 1;
                    sa.push_back(f);
                    sb.push_back(b);
                    sc.push_back(f);
                    sd.push_back(b);
                    break;
                }
                case TK_MERGE: {
                    POp tf{}, tb{}, f{}, b{};
                    std::vector<Cluster*> all{t.c};
                    all.insert(all.end(), t.c->children.begin(), t.c->children.end());
                    tf.op = SolveOp{SK_MERGE, 0, 0, 0, 0, 0, t.c->xoff, 0, 0, 0, 0, merge_segs(t.c, true),
                                    (int)t.c->children.size()};
                    tb.op = tf.op;
                    tb.op.dir = 1;
                    f.op = SolveOp{SK_MERGE, 0, 0, 0, 0, 0, t.c->xoff, 0, 0, 0, 0, merge_segs(t.c, false),
                                   (int)t.c->children.size()};
                    b.op = f.op;
                    b.op.dir = 1;
                    for (POp* o : {&tf, &tb, &f, &b}) {
                        o->rd = o->wr = all;
                        o->smem = 0;
                    }
                    sa.push_back(tf);
                    sb.push_back(tb);
                    sc.push_back(f);
                    sd.push_back(b);
                    break;
                }
                case TK_REASSIGN: {
                    POp f{};
                    f.op = SolveOp{SK_REASSIGN, 0, t.k, 0, 0, 0, t.c->xoff, t.f->xoff + t.m, ptr(d_idx + idx_off[q]), 0,
                                   0, 0, 0};
                    f.rd = f.wr = {t.c, t.f};
                    f.smem = 0;
                    POp b = f;
                    b.op.dir = 1;
                    sb.push_back(b);
                    sc.push_back(f);
                    break;
                }
                default:  // TK_ORTH, TK_SPLIT0: --scale 0 runs on square systems only
                    break;
            }
        }
        std::reverse(sb.begin(), sb.end());
        std::reverse(sd.begin(), sd.end());
        gemv_cols_.clear();
        for (auto& g : gemv) gemv_cols_.push_back(g.s);
        std::vector<SolveOp> all;
        std::vector<WMeta> meta[4];
        std::vector<POp>* lists[4] = {&sa, &sb, &sc, &sd};
        for (int L = 0; L < 4; ++L) {
            std::vector<std::vector<int>> w;
            schedule_ops(*lists[L], w);
            pack_waves(*lists[L], w, all, meta[L]);
        }
        Upload up;
        size_t o_ops = up.add(all), o_segs = up.add(segs), o_gemv = up.add(gemv), o_src = up.add(src),
               o_dst = up.add(dst), o_xin = up.add(xin), o_xo = up.add(xo), o_leaf = up.add(leaf);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        const SolveOp* d_ops = reinterpret_cast<const SolveOp*>(d + o_ops);
        d_segs_ = reinterpret_cast<const XSeg*>(d + o_segs);
        d_gemv_ = reinterpret_cast<const GemvRef<T>*>(d + o_gemv);
        d_src_ = reinterpret_cast<int*>(d + o_src);
        d_dst_ = reinterpret_cast<int*>(d + o_dst);
        d_xin_ = reinterpret_cast<int64_t*>(d + o_xin);
        d_xout_pos_ = reinterpret_cast<int64_t*>(d + o_xo);
        d_leaf_ = reinterpret_cast<int64_t*>(d + o_leaf);
        const size_t smem_cap = (200 * 1024) / sizeof(T);
        for (int L = 0; L < 4; ++L) {
            nrml_waves_[L].clear();
            for (auto& mt : meta[L]) {
                if ((size_t)mt.smem > smem_cap)
                    throw std::runtime_error("solve_nrml: a cluster exceeds the shared-memory vector capacity");
                nrml_waves_[L].push_back(make_wave(d_ops, mt));
            }
        }
        nin_ = (int)src.size();
        nout_ = (int)dst.size();
        nleaf_ = (int)leaf.size();
        solve_bytes_ = (double)(nnzH_ + nnzR_ + nnzQ_) * sizeof(T) + 16.0 * ncols_;
    }
    std::vector<Wave> nrml_waves_[4];
    T* xtbuf_ = nullptr;
    int64_t* d_leaf_ = nullptr;
    int nleaf_ = 0;
    cudaGraph_t nrml_graph_ = nullptr;
    cudaGraphExec_t nrml_exec_ = nullptr;

    void run_nrml_sweeps() {
        launches_solve_ = 0;
        cuda_check(cudaMemsetAsync(xtbuf_, 0, sizeof(T) * (size_t)xtot_, stream_), "nrml zero");
        cuda_check(cudaMemsetAsync(xbuf_, 0, sizeof(T) * (size_t)xtot_, stream_), "nrml zero");
        launch_gather_in<T>(d_bin_, d_src_, d_xin_, xtbuf_, nin_, stream_);
        ++launches_solve_;
        for (int L = 0; L < 4; ++L) {
            if (L == 2) {
                launch_seg_copy<T>(xtbuf_, xbuf_, d_leaf_, nleaf_, stream_);
                ++launches_solve_;
            }
            T* xb = L < 2 ? xtbuf_ : xbuf_;
            for (auto& w : nrml_waves_[L]) launches_solve_ += launch_wave(w, xb);
        }
        launch_scatter_out<T>(xbuf_, d_xout_pos_, d_dst_, d_xout_, nout_, stream_);
        ++launches_solve_;
    }

public:
    void solve_nrml_dev(const double* d_b, double* d_x) override {
        if (!factorized_) throw std::logic_error("solve_nrml before factorize");
        if (!rect_) throw std::invalid_argument("solve_nrml needs a least-squares factorization (square matching off)");
        double t0 = wall();
        cuda_check(cudaMemcpyAsync(d_bin_, d_b, sizeof(double) * ncols_, cudaMemcpyDeviceToDevice, stream_),
                   "nrml in");
        if (!nrml_exec_) {
            cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
            run_nrml_sweeps();
            cuda_check(cudaStreamEndCapture(stream_, &nrml_graph_), "capture end");
            cuda_check(cudaGraphInstantiate(&nrml_exec_, nrml_graph_, 0), "graph instantiate");
        }
        timed(KF_SOLVE, 0, solve_bytes_, [&] { cuda_check(cudaGraphLaunch(nrml_exec_, stream_), "graph launch"); });
        cuda_check(cudaMemcpyAsync(d_x, d_xout_, sizeof(double) * ncols_, cudaMemcpyDeviceToDevice, stream_),
                   "nrml out");
        t_solve_ = wall() - t0;
        ++applications_;
    }
    bool least_squares() const override { return rect_; }

private:

    // Wave scheduling on x segments (RAW, WAR, WAW): an op runs one wave after
    // the last op that wrote a segment it touches, or read one it writes.
    void schedule_ops(const std::vector<POp>& ops, std::vector<std::vector<int>>& waves) const {
        std::vector<int> lw(max_order_, -1), lr(max_order_, -1);  // by cluster order
        std::vector<int> wv(ops.size());
        int nw = 0;
        for (size_t i = 0; i < ops.size(); ++i) {
            int w = 0;
            for (Cluster* c : ops[i].rd) w = std::max(w, lw[c->order] + 1);
            for (Cluster* c : ops[i].wr) w = std::max(w, std::max(lw[c->order], lr[c->order]) + 1);
            for (Cluster* c : ops[i].wr) lw[c->order] = w;
            for (Cluster* c : ops[i].rd) lr[c->order] = std::max(lr[c->order], w);
            wv[i] = w;
            nw = std::max(nw, w + 1);
        }
        waves.assign(nw, {});
        for (size_t i = 0; i < ops.size(); ++i) waves[wv[i]].push_back((int)i);
    }
    double op_words(const SolveOp& o) const {
        if (o.kind == SK_APPLYQ) return (double)o.a * o.b - 0.5 * (double)o.b * (o.b - 1);
        if (o.kind != SK_TRI) return 0.0;
        double w = 0.5 * (double)o.a * (o.a + 1);
        for (int q = 0; q < o.nseg; ++q) w += (double)o.a * gemv_cols_[o.seg0 + q];
        return w;
    }
    void pack_waves(const std::vector<POp>& ops, const std::vector<std::vector<int>>& waves,
                    std::vector<SolveOp>& all, std::vector<WMeta>& meta) const {
        // Every op goes to exactly one of three launches (after the wave's
        // one-CTA ops in the array: the tall Q applications, then the dense ops).
        // Backward triangular ops with R^-1 formed (or R = I) and large enough
        // neighbour blocks or R^-1, and ScaleD / OrthD steps with Q^T formed, go
        // to the dense cluster kernel
        auto cl_words = [&](const SolveOp& o) {
            return o.kind == SK_TRI ? op_words(o) : (double)o.a * o.a;
        };
        auto tri = [&](const SolveOp& o) {
            if (o.a < 1 || o.a > kRinvMax) return false;
            if (o.kind == SK_APPLYQ) return o.p2 != 0 && o.nseg == 0;  // Q^T x (dir 0) or Q x (dir 1)
            if (o.kind != SK_TRI || o.dir != 0 || o.nseg > kTriMaxRefs) return false;
            if (!(o.p1 != 0 || o.p0 == 0)) return false;
            return op_words(o) >= kTriClWords;
        };
        // other Q applications of at least kApplyqBigRows rows go to the tall-Q
        // cluster kernel
        auto big = [&](const SolveOp& o) {
            return o.kind == SK_APPLYQ && o.b > 0 && o.a >= kApplyqBigRows && o.a <= 16 * kApplyqClRows && !tri(o);
        };
        for (auto& w : waves) {
            WMeta mt{all.size(), 0, 0, 0.0, -1, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            double hw = -1, tw = 0;
            int maxm = 0;
            for (int i : w)
                if (!big(ops[i].op) && !tri(ops[i].op)) {
                    all.push_back(ops[i].op);
                    mt.smem = std::max(mt.smem, ops[i].smem);
                    ++mt.n;
                }
            mt.boff = all.size();
            for (int i : w)
                if (big(ops[i].op)) {
                    all.push_back(ops[i].op);
                    maxm = std::max(maxm, ops[i].op.a);
                    ++mt.nbig;
                }
            mt.bcl = mt.nbig ? (maxm + kApplyqClRows - 1) / kApplyqClRows : 0;
            mt.toff = all.size();
            for (int i : w)
                if (tri(ops[i].op)) {
                    all.push_back(ops[i].op);
                    tw = std::max(tw, cl_words(ops[i].op));
                    mt.tk = std::max(mt.tk, ops[i].op.a);
                    ++mt.ntri;
                }
            mt.tcl = mt.ntri ? std::min(kTriMaxCl, std::max(2, (int)std::ceil(tw / kTriClPerCta))) : 0;
            if ((size_t)(mt.n + mt.nbig + mt.ntri) != w.size())
                throw std::logic_error("solve plan: an op was routed to more or fewer than one launch");
            for (int i : w) {
                const double ow = op_words(ops[i].op);
                mt.words += ow;
                if (ow > hw) {
                    hw = ow;
                    mt.hkind = ops[i].op.kind;
                    mt.ha = ops[i].op.a;
                    mt.hb = ops[i].op.kind == SK_TRI ? ops[i].op.nseg : ops[i].op.b;
                }
            }
            meta.push_back(mt);
        }
    }

    // Adjoint sweeps, built on the first adjoint solve. One application is
    // M = B_0 ... B_{n-1} F_{n-1} ... F_0 (F forward ops in tape order, then the
    // backward ops in reverse), so M^T applies B_0^T ... B_{n-1}^T and then
    // F_{n-1}^T ... F_0^T: Q^T and Q swap, R^{-1} (x - A12 x_n) becomes R^{-T}
    // with x_n -= A12^T z, and the index maps of SplitD and Merge become their
    // transposes. Every transposed op reads and writes all the segments it
    // touches.
    void build_adjoint_plan() {
        auto transpose_op = [](const POp& o) {
            POp t = o;
            std::vector<Cluster*> touch = o.rd;
            touch.insert(touch.end(), o.wr.begin(), o.wr.end());
            std::sort(touch.begin(), touch.end(), ByOrder());
            touch.erase(std::unique(touch.begin(), touch.end()), touch.end());
            switch (o.op.kind) {
                case SK_APPLYQ:
                case SK_TRI:
                    t.op.dir ^= 1;
                    break;
                case SK_SPLIT:
                    t.op.kind = SK_SPLIT_T;
                    break;
                case SK_MERGE:
                    t.op.kind = SK_MERGE_T;
                    break;
                case SK_SPLIT0:
                    t.op.kind = SK_SPLIT0_T;
                    break;
                default:
                    throw std::logic_error("adjoint: op without a transpose");
            }
            t.rd = touch;
            t.wr = touch;
            return t;
        };
        std::vector<POp> adj;
        adj.reserve(plan_fwd_.size() + plan_bwd_.size());
        for (auto it = plan_bwd_.rbegin(); it != plan_bwd_.rend(); ++it) adj.push_back(transpose_op(*it));
        for (auto it = plan_fwd_.rbegin(); it != plan_fwd_.rend(); ++it) adj.push_back(transpose_op(*it));
        std::vector<std::vector<int>> aw;
        schedule_ops(adj, aw);
        std::vector<SolveOp> all;
        std::vector<WMeta> am;
        pack_waves(adj, aw, all, am);
        Upload up;
        const size_t o_ops = up.add(all);
        char* d = up.commit(desc_arena_, stream_, pinned_);
        const SolveOp* d_ops = reinterpret_cast<const SolveOp*>(d + o_ops);
        adj_waves_.clear();
        const size_t smem_cap = (200 * 1024) / sizeof(T);
        for (auto& mt : am) {
            if ((size_t)mt.smem > smem_cap)
                throw std::runtime_error("adjoint solve: a cluster exceeds the shared-memory vector capacity");
            adj_waves_.push_back(make_wave(d_ops, mt));
        }
        cuda_check(cudaStreamSynchronize(stream_), "adjoint plan upload");
        pinned_.reset();
    }

public:
    bool solve_ready() override {
        finish_capture();
        return graph_exec_ != nullptr;
    }

    std::vector<double> profile_solve_waves() override {
        if (!factorized_) throw std::logic_error("profile before factorize");
        std::vector<double> out;
        std::vector<cudaEvent_t> ev;
        auto rec_ev = [&]() {
            cudaEvent_t e;
            cuda_check(cudaEventCreate(&e), "event");
            cudaEventRecord(e, stream_);
            ev.push_back(e);
        };
        launch_gather_in<T>(d_bin_, d_src_, d_xin_, xbuf_, nin_, stream_);
        rec_ev();
        std::vector<const Wave*> all;
        for (auto& w : fwd_waves_) all.push_back(&w);
        for (auto& w : bwd_waves_) all.push_back(&w);
        std::vector<cudaEvent_t> mid;
        for (const Wave* w : all) {
            Wave a = *w, b = *w;
            a.nbig = 0;
            a.ntri = 0;
            b.nops = 0;
            launch_wave(a, xbuf_);
            cudaEvent_t e;
            cuda_check(cudaEventCreate(&e), "event");
            cudaEventRecord(e, stream_);
            mid.push_back(e);
            launch_wave(b, xbuf_);
            rec_ev();
        }
        cuda_check(cudaStreamSynchronize(stream_), "profile solve");
        for (size_t i = 0; i < all.size(); ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[i], ev[i + 1]);
            if (cfg_.verbose >= 3 && all[i]->nbig + all[i]->ntri > 0) {
                float m1 = 0;
                cudaEventElapsedTime(&m1, ev[i], mid[i]);
                std::fprintf(stderr,
                             "solve wave %zu: %d ops %.4f ms, %d tall Q ops (cluster %d) and %d triangular ops "
                             "(cluster %d) %.4f ms\n",
                             i, all[i]->nops, m1, all[i]->nbig, all[i]->bcl, all[i]->ntri, all[i]->tcl, ms - m1);
            }
            out.push_back(ms);
            out.push_back(all[i]->nops);
            out.push_back(all[i]->smem);
            out.push_back(all[i]->words);
            out.push_back(all[i]->hkind);
            out.push_back(all[i]->ha);
            out.push_back(all[i]->hb);
        }
        for (auto e : ev) cudaEventDestroy(e);
        for (auto e : mid) cudaEventDestroy(e);
        if (cfg_.verbose >= 4) profile_solve_ops(all);
        return out;
    }

    // Diagnostics: every op of every sweep wave launched alone (5 times between
    // two events), one line per op on stderr: wave, kind, dir, sizes, neighbour
    // columns (triangular ops), the cluster size (tall Q ops, else 0) and the
    // time of one launch. x is scratch here.
    void profile_solve_ops(const std::vector<const Wave*>& all) {
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        constexpr int kRep = 5;
        std::vector<SolveOp> h;
        for (size_t i = 0; i < all.size(); ++i) {
            const Wave& w = *all[i];
            for (int part = 0; part < 3; ++part) {
                const int n = part == 0 ? w.nops : part == 1 ? w.nbig : w.ntri;
                if (n == 0) continue;
                const SolveOp* d = part == 0 ? w.ops : part == 1 ? w.big : w.tri;
                h.resize(n);
                cuda_check(cudaMemcpy(h.data(), d, n * sizeof(SolveOp), cudaMemcpyDeviceToHost), "profile ops");
                for (int j = 0; j < n; ++j) {
                    const SolveOp& o = h[j];
                    cudaEventRecord(e0, stream_);
                    for (int r = 0; r < kRep; ++r) {
                        if (part == 0)
                            launch_solve_step<T>(d + j, 1, d_segs_, d_gemv_, nullptr, xbuf_, w.smem, stream_);
                        else if (part == 1)
                            cuda_check(launch_applyq_cl<T>(d + j, 1, w.bcl, d_segs_, xbuf_, stream_), "profile op");
                        else
                            cuda_check(launch_tri_cl<T>(d + j, 1, w.tcl, w.tk, d_gemv_, xbuf_, stream_), "profile op");
                    }
                    cudaEventRecord(e1, stream_);
                    cuda_check(cudaEventSynchronize(e1), "profile op");
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    long long gc = 0;
                    if (o.kind == SK_TRI)
                        for (int q = 0; q < o.nseg; ++q) gc += gemv_cols_[o.seg0 + q];
                    std::fprintf(stderr, "op %zu kind %d dir %d a %d b %d c %d nseg %d gcols %lld cl %d us %.2f\n", i,
                                 o.kind, o.dir, o.a, o.b, o.c, o.nseg, gc, part == 0 ? 0 : part == 1 ? w.bcl : w.tcl,
                                 ms * 1e3 / kRep);
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }

private:
    // One application's launches on ln; returns how many kernels it launched.
    int run_solve_sweeps(const Lanes& ln) {
        int n = 0;
        launch_gather_in<T>(d_bin_, d_src_, d_xin_, xbuf_, nin_, ln.main);
        ++n;
        for (auto& w : fwd_waves_) n += launch_wave(w, xbuf_, ln);
        for (auto& w : bwd_waves_) n += launch_wave(w, xbuf_, ln);
        launch_scatter_out<T>(xbuf_, d_xout_pos_, d_dst_, d_xout_, nout_, ln.main);
        return n + 1;
    }
    // The solve graph: captured from the same launches on cap_lanes_ by a host
    // thread (capture records, it does not run), instantiated and uploaded
    // there, while the first applications run their launches on stream_.
    void start_capture() {
        cap_done_ = false;
        cap_err_ = nullptr;
        cap_thread_ = std::thread([this] {
            try {
                cuda_check(cudaSetDevice(cfg_.device), "cudaSetDevice");
                cuda_check(cudaStreamBeginCapture(cap_lanes_.main, cudaStreamCaptureModeThreadLocal), "capture");
                run_solve_sweeps(cap_lanes_);
                cuda_check(cudaStreamEndCapture(cap_lanes_.main, &cap_graph_), "capture end");
                cuda_check(cudaGraphInstantiate(&cap_exec_, cap_graph_, 0), "graph instantiate");
                // placed on the device here, not by its first launch
                cuda_check(cudaGraphUpload(cap_exec_, cap_lanes_.main), "graph upload");
                cuda_check(cudaStreamSynchronize(cap_lanes_.main), "graph upload");
            } catch (...) {
                cap_err_ = std::current_exception();
                cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
                if (cudaStreamIsCapturing(cap_lanes_.main, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(cap_lanes_.main, &g);
                    if (g) cudaGraphDestroy(g);
                }
            }
            cap_done_ = true;
        });
    }
    // Waits for a capture in flight and adopts its graph (a capture error is
    // rethrown here).
    void finish_capture() {
        if (!cap_thread_.joinable()) return;
        cap_thread_.join();
        graph_ = cap_graph_;
        graph_exec_ = cap_exec_;
        cap_graph_ = nullptr;
        cap_exec_ = nullptr;
        if (cap_err_) {
            std::exception_ptr e = cap_err_;
            cap_err_ = nullptr;
            std::rethrow_exception(e);
        }
    }
    // M^T = G_in^T (sweeps)^T S_out^T: start from zero, place g where the solve
    // reads x out, run the transposed waves, read y where the solve puts b in.
    void run_adjoint_sweeps() {
        cuda_check(cudaMemsetAsync(xbuf_, 0, sizeof(T) * (size_t)xtot_, stream_), "adjoint zero");
        launch_gather_in<T>(d_adj_in_, d_dst_, d_xout_pos_, xbuf_, nout_, stream_);
        for (auto& w : adj_waves_) launch_wave(w, xbuf_);
        launch_scatter_out<T>(xbuf_, d_xin_, d_src_, d_adj_out_, nin_, stream_);
    }
};

}  // namespace

std::unique_ptr<EngineBase> make_engine(const Config& cfg, int precision) {
    if (precision == 1) return std::unique_ptr<EngineBase>(new Engine<float>(cfg));
    return std::unique_ptr<EngineBase>(new Engine<double>(cfg));
}

}  // namespace spq
