// Device memory for one factorization handle: a zero-initialised bump arena
// for blocks and factors (nothing is freed before the handle), a growable
// scratch buffer for per-wave workspaces, and descriptor uploads.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
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

// Chunked bump allocator. Every chunk is zeroed when it is allocated and memory
// is never reused, so a fresh allocation always reads as zeros (the reference
// allocates fill-in and merged blocks with setZero).
class Arena {
public:
    explicit Arena(size_t chunk = size_t(256) << 20) : chunk_(chunk) {}
    ~Arena() { release(); }
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;

    void set_stream(cudaStream_t s) { stream_ = s; }
    void* alloc(size_t bytes) {
        bytes = (bytes + 127) & ~size_t(127);
        if (bytes == 0) bytes = 128;
        if (chunks_.empty() || used_ + bytes > cap_) {
            size_t sz = bytes > chunk_ ? bytes : chunk_;
            void* p = nullptr;
            cuda_check(cudaMalloc(&p, sz), "arena cudaMalloc");
            cuda_check(cudaMemsetAsync(p, 0, sz, stream_), "arena memset");
            chunks_.push_back(p);
            cap_ = sz;
            used_ = 0;
            total_ += sz;
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
    void release() {
        for (void* p : chunks_) cudaFree(p);
        chunks_.clear();
        cap_ = used_ = total_ = 0;
    }

private:
    size_t chunk_;
    cudaStream_t stream_ = nullptr;
    std::vector<void*> chunks_;
    size_t cap_ = 0, used_ = 0, total_ = 0;
};

// Reusable device scratch. grow() waits for the stream before replacing the
// buffer, so work queued on the old buffer is finished.
class Scratch {
public:
    ~Scratch() {
        if (p_) cudaFree(p_);
    }
    void* get(size_t bytes, cudaStream_t s) {
        if (bytes > cap_) {
            cuda_check(cudaStreamSynchronize(s), "scratch sync");
            if (p_) cudaFree(p_);
            p_ = nullptr;
            size_t nc = bytes + bytes / 4 + (size_t(1) << 20);
            cuda_check(cudaMalloc(&p_, nc), "scratch cudaMalloc");
            cap_ = nc;
        }
        return p_;
    }
    size_t capacity() const { return cap_; }

private:
    void* p_ = nullptr;
    size_t cap_ = 0;
};

// Host staging of one batch of heterogeneous descriptor arrays, uploaded with
// one copy into arena memory that stays valid for the handle's lifetime.
class Upload {
public:
    template <class U>
    size_t add(const std::vector<U>& v) {
        size_t off = (buf_.size() + 15) & ~size_t(15);
        buf_.resize(off + v.size() * sizeof(U));
        if (!v.empty()) std::memcpy(buf_.data() + off, v.data(), v.size() * sizeof(U));
        return off;
    }
    // Returns the device base; element arrays are at base + offset.
    char* commit(Arena& arena, cudaStream_t s) {
        if (buf_.empty()) return nullptr;
        char* d = static_cast<char*>(arena.alloc(buf_.size()));
        cuda_check(cudaMemcpyAsync(d, buf_.data(), buf_.size(), cudaMemcpyHostToDevice, s), "descriptor upload");
        // pageable source: the copy is staged before return, buf_ may be reused
        return d;
    }
    void clear() { buf_.clear(); }
    bool empty() const { return buf_.empty(); }

private:
    std::vector<char> buf_;
};

}  // namespace spq
