// pg_peaks.cu -- on-chip ceilings measured on the device the solver runs on,
// for the secondary rooflines of the sweep: shared-memory read bandwidth,
// read bandwidth of an L2-resident buffer, and FP32 FMA throughput.  Each is
// a plain streaming kernel timed with CUDA events; every access stays inside
// the buffers this file allocates.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "pg_types.h"

namespace {

constexpr int kPeakThreads = 512;
constexpr int kSmemFloats = 8192;  // 32 KB per block

// Conflict-free 16-byte shared-memory reads: consecutive lanes read
// consecutive 16-byte words, so a warp's 32 reads cover 512 bytes.
__global__ void __launch_bounds__(kPeakThreads) k_peak_smem(int iters, float* out) {
    __shared__ __align__(16) float s[kSmemFloats];
    for (int i = threadIdx.x; i < kSmemFloats; i += blockDim.x) s[i] = (float)(i & 7);
    __syncthreads();
    const float4* s4 = reinterpret_cast<const float4*>(s);
    constexpr int n4 = kSmemFloats / 4;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    int idx = threadIdx.x % n4;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float4 v = s4[(idx + k * 64) & (n4 - 1)];
            a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
        }
        idx = (idx + 32) & (n4 - 1);
    }
    if (a.x + a.y + a.z + a.w == -1.0f) out[blockIdx.x] = a.x;  // never true; keeps the reads
}

// Grid-stride 16-byte reads over a buffer that fits in L2, `passes` times.
__global__ void __launch_bounds__(kPeakThreads)
    k_peak_l2(const float4* __restrict__ buf, int64_t n4, int passes, float* out) {
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int p = 0; p < passes; ++p)
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 v = __ldcg(buf + i);
            a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
        }
    if (a.x + a.y + a.z + a.w == -1.0f) out[blockIdx.x] = a.x;
}

// Eight independent FMA chains per thread.
__global__ void __launch_bounds__(kPeakThreads) k_peak_fma(int iters, float* out) {
    float r[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = (float)(threadIdx.x + k);
    const float a = 0.999f, b = 1.0e-3f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += r[k];
    if (s == -1.0f) out[blockIdx.x] = s;
}

template <typename F>
cudaError_t time_best(F launch, int reps, float* best_ms) {
    cudaEvent_t e0, e1;
    cudaError_t e = cudaEventCreate(&e0);
    if (e != cudaSuccess) return e;
    e = cudaEventCreate(&e1);
    if (e != cudaSuccess) { cudaEventDestroy(e0); return e; }
    *best_ms = 1e30f;
    launch();  // warm-up
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        *best_ms = std::min(*best_ms, ms);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e;
}

}  // namespace

extern "C" int pg_measure_peaks(int device, double* smem_gbs, double* l2_gbs,
                                double* fma_tflops) {
    if (cudaSetDevice(device) != cudaSuccess)
        return pg::set_last_error(PG_ECUDA, "cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms <= 0) return pg::set_last_error(PG_ECUDA, "no multiprocessors reported");
    const int blocks = sms * 4;
    float* out = nullptr;
    float4* buf = nullptr;
    const int64_t l2_bytes = (int64_t)64 << 20;
    cudaError_t e = cudaMalloc(&out, sizeof(float) * blocks);
    if (e == cudaSuccess) e = cudaMalloc(&buf, l2_bytes);
    if (e == cudaSuccess) e = cudaMemset(buf, 0, l2_bytes);
    float ms = 0.f;
    if (e == cudaSuccess && smem_gbs) {
        const int iters = 4096;
        e = time_best([&] { k_peak_smem<<<blocks, kPeakThreads>>>(iters, out); }, 5, &ms);
        *smem_gbs = (double)blocks * kPeakThreads * iters * 8 * 16 / (ms * 1e-3) / 1e9;
    }
    if (e == cudaSuccess && l2_gbs) {
        const int passes = 16;
        const int64_t n4 = l2_bytes / 16;
        e = time_best([&] { k_peak_l2<<<blocks, kPeakThreads>>>(buf, n4, passes, out); }, 5, &ms);
        *l2_gbs = (double)l2_bytes * passes / (ms * 1e-3) / 1e9;
    }
    if (e == cudaSuccess && fma_tflops) {
        const int iters = 16384;
        e = time_best([&] { k_peak_fma<<<blocks, kPeakThreads>>>(iters, out); }, 5, &ms);
        *fma_tflops = 2.0 * blocks * kPeakThreads * iters * 8 / (ms * 1e-3) / 1e12;
    }
    if (out) cudaFree(out);
    if (buf) cudaFree(buf);
    if (e != cudaSuccess)
        return pg::set_last_error(PG_ECUDA, std::string("pg_measure_peaks: ") + cudaGetErrorString(e));
    return PG_OK;
}
