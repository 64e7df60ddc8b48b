// Arithmetic peaks of this device's CUDA cores, measured: FP32 FFMA, packed
// FP32 FFMA2 and FP64 DFMA throughput (no counterpart in the reference).  The
// row march is bound by instruction issue and its floating-point pipes, not by
// HBM, so its second roofline is the measured fused-multiply-add rate.
//
// Each thread runs kChains independent multiply-add chains (a = a*b + c with
// |b| < 1, so the values settle and never overflow or go subnormal); the grid
// fills every SM several times over.  Best of three timed launches after one
// warm-up launch, CUDA events on a private stream.
#include <cuda_runtime.h>

#include <string>

#include "cfs.h"

namespace cfs {
void record_global_error(int code, const std::string& msg);  // cfs_api.cpp
}

namespace {

constexpr int kThreads = 256;
constexpr int kChains = 8;
constexpr int kUnroll = 8;

template <class T>
__global__ void __launch_bounds__(kThreads) fma_chains(T* sink, int iters, T b, T c) {
    T a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = T(threadIdx.x + k) * T(1e-3);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u)
#pragma unroll
            for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == T(-1)) sink[blockIdx.x * kThreads + threadIdx.x] = s;  // never true: keeps the chains live
}

__global__ void __launch_bounds__(kThreads) ffma2_chains(float* sink, int iters, float b, float c) {
    float2 a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = make_float2(float(threadIdx.x + k) * 1e-3f, float(k) * 1e-3f);
    const float2 bb = make_float2(b, b), cc = make_float2(c, c);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u)
#pragma unroll
            for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], bb, cc);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
    if (s == -1.0f) sink[blockIdx.x * kThreads + threadIdx.x] = s;
}

// Times `launch` (best of three after a warm-up); returns ms or a negative value on error.
template <class F>
float best_ms(F launch, cudaStream_t st) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return -1.0f;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return -1.0f;
    }
    float best = -1.0f;
    launch();
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0, st);
        launch();
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best < 0.0f || ms < best) best = ms;
    }
    if (cudaGetLastError() != cudaSuccess) best = -1.0f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

}  // namespace

extern "C" int cfs_fp_peaks(int device, double* fp32_tflops, double* fp32x2_tflops, double* fp64_tflops) {
    if (!fp32_tflops || !fp32x2_tflops || !fp64_tflops) {
        cfs::record_global_error(CFS_ERR_INVALID, "cfs_fp_peaks: null output");
        return CFS_ERR_INVALID;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cfs::record_global_error(CFS_ERR_CUDA, "cfs_fp_peaks: cudaSetDevice failed");
        return CFS_ERR_CUDA;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = (sms > 0 ? sms : 148) * 8;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cfs::record_global_error(CFS_ERR_CUDA, "cfs_fp_peaks: stream creation failed");
        return CFS_ERR_CUDA;
    }
    void* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(double) * blocks * kThreads) != cudaSuccess) {
        cudaStreamDestroy(st);
        cfs::record_global_error(CFS_ERR_NOMEM, "cfs_fp_peaks: device allocation failed");
        return CFS_ERR_NOMEM;
    }
    const int it32 = 4096, it64 = 1024;
    const double fma_per_iter = double(blocks) * kThreads * kUnroll * kChains;
    const float m32 = best_ms([&] { fma_chains<float><<<blocks, kThreads, 0, st>>>(static_cast<float*>(sink), it32, 0.9999f, 1e-3f); }, st);
    const float m2 = best_ms([&] { ffma2_chains<<<blocks, kThreads, 0, st>>>(static_cast<float*>(sink), it32, 0.9999f, 1e-3f); }, st);
    const float m64 = best_ms([&] { fma_chains<double><<<blocks, kThreads, 0, st>>>(static_cast<double*>(sink), it64, 0.9999, 1e-3); }, st);
    cudaFree(sink);
    cudaStreamDestroy(st);
    if (m32 <= 0.0f || m2 <= 0.0f || m64 <= 0.0f) {
        cfs::record_global_error(CFS_ERR_CUDA, "cfs_fp_peaks: a timing launch failed");
        return CFS_ERR_CUDA;
    }
    // 2 flops per FMA; FFMA2 carries two FMAs
    *fp32_tflops = 2.0 * fma_per_iter * it32 / (m32 * 1e-3) / 1e12;
    *fp32x2_tflops = 4.0 * fma_per_iter * it32 / (m2 * 1e-3) / 1e12;
    *fp64_tflops = 2.0 * fma_per_iter * it64 / (m64 * 1e-3) / 1e12;
    return CFS_OK;
}
