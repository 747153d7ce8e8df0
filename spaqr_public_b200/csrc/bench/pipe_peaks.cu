// Measured arithmetic peaks of the pipes the factorization kernels use, for
// their compute rooflines: FP32 and FP64 FMA (SIMT), and the warp-level
// tensor-core MMAs (TF32 m16n8k8 with FP32 accumulation, FP64 m8n8k4).
//
//   spaqr_public_b200/_build/spq_pipe_peaks [device]
//
// prints one JSON line {"fp32_fma_tflops", "fp64_fma_tflops",
// "tf32_mma_tflops", "fp64_mma_tflops", "sm_count", ...}. Each figure is the
// best of 5 timed launches (CUDA events, after one warm-up launch) of a grid
// of 8 CTAs per SM running independent dependency chains, long enough
// (tens of ms) that launch overhead is negligible. Flops: 2 per FMA, 2*M*N*K
// per MMA. The inputs live in registers and the results are stored once (so
// the compiler keeps the chains), so no memory traffic enters the timing.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

template <class T>
__global__ void __launch_bounds__(kThreads) k_fma(T* out, int iters, T a, T b) {
    T acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = T(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc[c] = acc[c] * a + b;
    }
    T s = T(0);
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += acc[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// TF32 mma.sync m16n8k8 (row.col), four independent accumulator chains per warp.
__global__ void __launch_bounds__(kThreads) k_mma_tf32(float* out, int iters) {
    unsigned a[4], b[2];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = __float_as_uint(1.0f + 1e-3f * (threadIdx.x + i));
#pragma unroll
    for (int i = 0; i < 2; ++i) b[i] = __float_as_uint(1e-6f * (threadIdx.x + i));
    float d[4][4] = {};
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < 4; ++c)
            asm volatile(
                "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+f"(d[c][0]), "+f"(d[c][1]), "+f"(d[c][2]), "+f"(d[c][3])
                : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) s += d[c][0] + d[c][1] + d[c][2] + d[c][3];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64 mma.sync m8n8k4 (row.col), four independent accumulator chains per warp.
__global__ void __launch_bounds__(kThreads) k_mma_f64(double* out, int iters) {
    double a = 1.0 + 1e-3 * threadIdx.x, b = 1e-6 * threadIdx.x;
    double d[4][2] = {};
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < 4; ++c)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(d[c][0]), "+d"(d[c][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) s += d[c][0] + d[c][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "spq_pipe_peaks: %s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}

// Best TFLOP/s over 5 timed launches of `launch` doing `flops` each.
template <class F>
double best_tflops(F launch, double flops) {
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    launch();  // warm-up
    check(cudaDeviceSynchronize(), "warm-up");
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        check(cudaEventRecord(e0), "record");
        launch();
        check(cudaEventRecord(e1), "record");
        check(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        if (ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace

int main(int argc, char** argv) {
    const int dev = argc > 1 ? std::atoi(argv[1]) : 0;
    check(cudaSetDevice(dev), "cudaSetDevice");
    cudaDeviceProp prop;
    check(cudaGetDeviceProperties(&prop, dev), "properties");
    const int sms = prop.multiProcessorCount;
    const int grid = sms * 8;
    const double threads = double(grid) * kThreads;
    void* buf = nullptr;
    check(cudaMalloc(&buf, size_t(grid) * kThreads * sizeof(double)), "cudaMalloc");
    const int it_fma = 1 << 14, it_mma = 1 << 12;
    const double f32 = best_tflops([&] { k_fma<float><<<grid, kThreads>>>((float*)buf, it_fma, 0.999f, 1e-3f); },
                                   threads * it_fma * kChains * 2.0);
    const double f64 = best_tflops([&] { k_fma<double><<<grid, kThreads>>>((double*)buf, it_fma / 4, 0.999, 1e-3); },
                                   threads * (it_fma / 4) * kChains * 2.0);
    const double warps = threads / 32;
    const double t32 = best_tflops([&] { k_mma_tf32<<<grid, kThreads>>>((float*)buf, it_mma); },
                                   warps * it_mma * 4 * (2.0 * 16 * 8 * 8));
    const double d64 = best_tflops([&] { k_mma_f64<<<grid, kThreads>>>((double*)buf, it_mma / 4); },
                                   warps * (it_mma / 4) * 4 * (2.0 * 8 * 8 * 4));
    check(cudaGetLastError(), "launch");
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, dev);
    std::printf(
        "{\"fp32_fma_tflops\": %.2f, \"fp64_fma_tflops\": %.2f, \"tf32_mma_tflops\": %.2f, \"fp64_mma_tflops\": %.2f, "
        "\"sm_count\": %d, \"device\": \"%s\", \"how\": \"best of 5 CUDA-event launches, %d CTAs x %d threads, "
        "independent register chains (2 flops per FMA, 2MNK per mma.sync)\"}\n",
        f32, f64, t32, d64, sms, prop.name, grid, kThreads);
    cudaFree(buf);
    return 0;
}
