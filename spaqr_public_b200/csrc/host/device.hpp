// Device memory for one factorization handle: a zero-initialised bump arena
// for blocks and factors (nothing is freed before the handle), a growable
// scratch buffer for per-wave workspaces, and descriptor uploads.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace spq {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

inline double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Process-wide stream-ordered memory pool of one device, shared by every
// handle on it. Freed memory stays in the pool (unlimited release threshold),
// so a later factorization is served without new device allocations and a
// growing scratch buffer needs no stream synchronisation. trim_device_pools()
// returns the cached memory to the device.
inline std::mutex& pool_mutex() {
    static std::mutex mu;
    return mu;
}
inline std::map<int, cudaMemPool_t>& pool_table() {
    static std::map<int, cudaMemPool_t> pools;
    return pools;
}
inline cudaMemPool_t device_pool(int dev) {
    std::lock_guard<std::mutex> g(pool_mutex());
    auto& pools = pool_table();
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    cuda_check(cudaMemPoolCreate(&p, &props), "cudaMemPoolCreate");
    uint64_t thr = UINT64_MAX;
    cuda_check(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &thr), "pool release threshold");
    pools[dev] = p;
    return p;
}
// Buffers a destroyed handle leaves for the next one (its stream drained
// first, so they are idle): the device scratch buffer of each device, and
// the pinned staging chunks. A new handle takes them instead of growing a
// scratch buffer and pinning host pages again, which costs tens of ms per
// 8 MiB chunk on a busy host.
struct HandoffCache {
    std::mutex mu;
    std::map<int, std::pair<void*, size_t>> scratch;  // device -> (buffer, bytes)
    std::vector<std::pair<char*, size_t>> pinned;     // free pinned chunks
};
inline HandoffCache& handoff_cache() {
    static HandoffCache c;
    return c;
}
inline void trim_device_pools() {
    {
        HandoffCache& c = handoff_cache();
        std::lock_guard<std::mutex> g(c.mu);
        int cur = 0;
        cudaGetDevice(&cur);
        for (auto& kv : c.scratch) {
            cudaSetDevice(kv.first);
            cudaFree(kv.second.first);
        }
        cudaSetDevice(cur);
        c.scratch.clear();
        for (auto& ch : c.pinned) cudaFreeHost(ch.first);
        c.pinned.clear();
    }
    std::lock_guard<std::mutex> g(pool_mutex());
    for (auto& kv : pool_table()) cudaMemPoolTrimTo(kv.second, 0);
}
inline void* pool_alloc(cudaMemPool_t pool, size_t bytes, cudaStream_t s, const char* what) {
    void* p = nullptr;
    cuda_check(cudaMallocFromPoolAsync(&p, bytes, pool, s), what);
    return p;
}

// Chunked bump allocator. Every chunk is zeroed when it is allocated and memory
// is never reused, so a fresh allocation always reads as zeros (the reference
// allocates fill-in and merged blocks with setZero).
class Arena {
public:
    explicit Arena(size_t chunk = size_t(256) << 20) : chunk_(chunk) {}
    ~Arena() { release(); }
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;

    void set_stream(cudaStream_t s, cudaMemPool_t pool) {
        stream_ = s;
        pool_ = pool;
    }
    // The bytes alloc(bytes) takes from a chunk: whole 128-byte lines, at least one.
    static size_t rounded(size_t bytes) { return bytes ? (bytes + 127) & ~size_t(127) : 128; }
    void* alloc(size_t bytes) {
        bytes = rounded(bytes);
        if (chunks_.empty() || used_ + bytes > cap_) {
            const double t0 = wall_seconds();
            size_t sz = bytes > chunk_ ? bytes : chunk_;
            void* p = pool_alloc(pool_, sz, stream_, "arena allocation");
            cuda_check(cudaMemsetAsync(p, 0, sz, stream_), "arena memset");
            chunks_.push_back(p);
            cap_ = sz;
            used_ = 0;
            total_ += sz;
            alloc_seconds_ += wall_seconds() - t0;
        }
        char* p = static_cast<char*>(chunks_.back()) + used_;
        used_ += bytes;
        return p;
    }
    template <class U>
    U* alloc_n(size_t n) {
        return static_cast<U*>(alloc(n * sizeof(U)));
    }
    size_t bytes_reserved() const { return total_; }
    double alloc_seconds() const { return alloc_seconds_; }
    // Returns the chunks to the pool in stream order (call before the stream
    // is destroyed).
    void release() {
        for (void* p : chunks_) cudaFreeAsync(p, stream_);
        chunks_.clear();
        cap_ = used_ = total_ = 0;
    }

private:
    size_t chunk_;
    cudaStream_t stream_ = nullptr;
    cudaMemPool_t pool_ = nullptr;
    std::vector<void*> chunks_;
    size_t cap_ = 0, used_ = 0, total_ = 0;
    double alloc_seconds_ = 0;
};

// Reusable device scratch on one stream. Growing frees the old buffer and
// allocates the new one in stream order, so work already queued on the old
// buffer finishes first without a host wait.
class Scratch {
public:
    void set_pool(cudaMemPool_t pool, int device) {
        pool_ = pool;
        dev_ = device;
    }
    void* get(size_t bytes, cudaStream_t s) {
        if (!p_) {  // the buffer a destroyed handle left on this device
            HandoffCache& c = handoff_cache();
            std::lock_guard<std::mutex> g(c.mu);
            auto it = c.scratch.find(dev_);
            if (it != c.scratch.end()) {
                p_ = it->second.first;
                cap_ = it->second.second;
                c.scratch.erase(it);
            }
        }
        if (bytes > cap_) {
            const double t0 = wall_seconds();
            if (p_) cudaFreeAsync(p_, s);
            p_ = nullptr;
            cap_ = 0;
            const size_t nc = bytes + bytes / 4 + (size_t(1) << 20);
            p_ = pool_alloc(pool_, nc, s, "scratch allocation");
            cap_ = nc;
            grow_seconds_ += wall_seconds() - t0;
        }
        return p_;
    }
    void release(cudaStream_t s) {
        if (p_) cudaFreeAsync(p_, s);
        p_ = nullptr;
        cap_ = 0;
    }
    // Leaves the buffer for the next handle on the device (the stream must be
    // drained); the smaller of two buffers goes back to the pool.
    void hand_off(cudaStream_t s) {
        if (!p_) return;
        HandoffCache& c = handoff_cache();
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.scratch.find(dev_);
        if (it != c.scratch.end() && it->second.second >= cap_) {
            cudaFreeAsync(p_, s);
        } else {
            if (it != c.scratch.end()) cudaFreeAsync(it->second.first, s);
            c.scratch[dev_] = {p_, cap_};
        }
        p_ = nullptr;
        cap_ = 0;
    }
    size_t capacity() const { return cap_; }
    double grow_seconds() const { return grow_seconds_; }

private:
    int dev_ = 0;
    cudaMemPool_t pool_ = nullptr;
    void* p_ = nullptr;
    size_t cap_ = 0;
    double grow_seconds_ = 0;
};

// Pinned host staging for descriptor uploads. A cudaMemcpyAsync from pageable
// memory may wait for the stream before staging the bytes; from pinned memory
// it returns at once, so the host builds the next wave while the device runs
// the current one. Bump allocation in pinned chunks; reset() is legal only
// when the stream has drained every copy issued from the stage.
class PinnedStage {
public:
    // The chunks go to the handoff cache (the owner drained its stream first).
    ~PinnedStage() {
        HandoffCache& c = handoff_cache();
        std::lock_guard<std::mutex> g(c.mu);
        for (auto& ch : chunks_) c.pinned.push_back(ch);
    }
    char* get(size_t bytes) {
        bytes = (bytes + 15) & ~size_t(15);
        while (ci_ < chunks_.size() && used_ + bytes > chunks_[ci_].second) {
            ++ci_;
            used_ = 0;
        }
        if (ci_ == chunks_.size()) {
            const size_t sz = bytes > kChunk ? bytes : kChunk;
            char* p = nullptr;
            size_t got = 0;
            {  // a chunk a destroyed handle left, else newly pinned pages
                HandoffCache& c = handoff_cache();
                std::lock_guard<std::mutex> g(c.mu);
                for (size_t i = 0; i < c.pinned.size(); ++i)
                    if (c.pinned[i].second >= sz) {
                        p = c.pinned[i].first;
                        got = c.pinned[i].second;
                        c.pinned.erase(c.pinned.begin() + (long)i);
                        break;
                    }
            }
            if (!p) {
                const double t0 = wall_seconds();
                void* q = nullptr;
                cuda_check(cudaHostAlloc(&q, sz, cudaHostAllocPortable), "pinned staging");
                alloc_seconds_ += wall_seconds() - t0;
                p = static_cast<char*>(q);
                got = sz;
            }
            chunks_.emplace_back(p, got);
            used_ = 0;
        }
        char* p = chunks_[ci_].first + used_;
        used_ += bytes;
        return p;
    }
    void reset() {
        ci_ = 0;
        used_ = 0;
    }
    double alloc_seconds() const { return alloc_seconds_; }
    size_t chunks() const { return chunks_.size(); }

private:
    static constexpr size_t kChunk = size_t(8) << 20;
    double alloc_seconds_ = 0;
    std::vector<std::pair<char*, size_t>> chunks_;
    size_t ci_ = 0, used_ = 0;
};

// One batch of heterogeneous descriptor arrays, uploaded with one copy into
// arena memory that stays valid for the handle's lifetime. add() records where
// an array lies; commit() packs the arrays straight into the pinned stage, so
// every array passed to add() must stay alive and unchanged until commit().
class Upload {
public:
    template <class U>
    size_t add(const std::vector<U>& v) {
        const size_t off = (size_ + 15) & ~size_t(15);
        const size_t bytes = v.size() * sizeof(U);
        if (bytes) spans_.push_back(Span{reinterpret_cast<const char*>(v.data()), bytes, off});
        size_ = off + bytes;
        return off;
    }
    // Returns the device base; element arrays are at base + offset. The bytes
    // go through the pinned stage, so the copy does not wait for the stream.
    char* commit(Arena& arena, cudaStream_t s, PinnedStage& stage) {
        if (size_ == 0) return nullptr;
        char* d = static_cast<char*>(arena.alloc(size_));
        char* h = stage.get(size_);
        for (const Span& sp : spans_) std::memcpy(h + sp.off, sp.p, sp.bytes);
        cuda_check(cudaMemcpyAsync(d, h, size_, cudaMemcpyHostToDevice, s), "descriptor upload");
        return d;
    }
    bool empty() const { return size_ == 0; }

private:
    struct Span {
        const char* p;
        size_t bytes, off;
    };
    std::vector<Span> spans_;
    size_t size_ = 0;
};

}  // namespace spq
