// peaks.cu -- microbenchmarks for the roofline denominators the stepping
// kernels are measured against, besides the HBM copy bandwidth the pool
// measures: L2 read bandwidth (the 64^3 and 128^3 Grid3f workloads are
// L2-resident), FP32 FMA and FP64 FMA throughput, and the throughput of the
// hardware cosine (__cosf, the special-function unit) that the plane-wave
// mode sums run on.  Built into its own library (libcrp_peaks.so), used by
// the benchmark only.
#include <cuda_runtime.h>

#include <stdint.h>

namespace {

// Each thread reads float4 elements of a buffer that fits in L2, strided by
// the whole grid, `reps` times over.
__global__ void l2_read_kernel(const float4 *__restrict__ buf, uint64_t n4, int reps, float *sink) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (int r = 0; r < reps; r++) {
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
            float4 v = __ldcg(buf + i);  // cache at L2 only: L1 does not serve repeats
            acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
        }
    }
    if (acc.x + acc.y + acc.z + acc.w == 1234.5f) sink[0] = acc.x;
}

// 8 independent FMA chains per thread, `iters` rounds of 8 FMAs.
__global__ void fp32_fma_kernel(int iters, float *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-3f + k;
    const float m = 0.999999f, c = 1e-6f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 1234.5f) sink[0] = s;
}

__global__ void fp64_fma_kernel(int iters, double *sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-3 + k;
    const double m = 0.999999, c = 1e-6;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
    }
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 1234.5) sink[0] = s;
}

// 8 independent cosine chains per thread: x <- __cosf(x) (values stay in
// [cos 1, 1]), `iters` rounds of 8.
__global__ void cos_kernel(int iters, float *sink) {
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-4f + 0.1f * k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __cosf(a[k]);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 1234.5f) sink[0] = s;
}

template <class F>
cudaError_t time_ms(F launch, int repeats, float *ms) {
    cudaEvent_t e0, e1;
    cudaError_t e = cudaEventCreate(&e0);
    if (e != cudaSuccess) return e;
    e = cudaEventCreate(&e1);
    if (e != cudaSuccess) return e;
    launch();  // warm-up
    cudaEventRecord(e0);
    for (int r = 0; r < repeats; r++) launch();
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / repeats;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

}  // namespace

extern "C" {

// Measured peaks of the current device.  Returns 0 or a cudaError_t.
//   l2_gbs       L2 read bandwidth [GB/s] over a 32 MB buffer
//   fp32_tflops  FP32 FMA throughput [TFLOP/s, 2 flop per FMA]
//   fp64_tflops  FP64 FMA throughput [TFLOP/s]
//   cos_gops     __cosf throughput [10^9 cosines/s]
typedef struct crp_peaks {
    double l2_gbs, fp32_tflops, fp64_tflops, cos_gops;
    int32_t sm_count, _pad;
} crp_peaks;

int crp_peaks_measure(crp_peaks *out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    out->sm_count = sms;
    const uint64_t bytes = 32ull << 20;
    const uint64_t n4 = bytes / 16;
    float4 *buf = nullptr;
    float *sink = nullptr;
    if ((e = cudaMalloc(&buf, bytes)) != cudaSuccess) return (int)e;
    if ((e = cudaMalloc(&sink, 64)) != cudaSuccess) { cudaFree(buf); return (int)e; }
    cudaMemset(buf, 0, bytes);
    const int grid = sms * 8, block = 256, reps = 20;
    float ms = 0.f;
    e = time_ms([&] { l2_read_kernel<<<grid, block>>>(buf, n4, reps, sink); }, 5, &ms);
    if (e == cudaSuccess) out->l2_gbs = (double)bytes * reps / (ms * 1e-3) / 1e9;
    const int iters = 4096;
    const double threads = (double)sms * 8 * 256;
    if (e == cudaSuccess) {
        e = time_ms([&] { fp32_fma_kernel<<<sms * 8, 256>>>(iters, sink); }, 5, &ms);
        out->fp32_tflops = threads * iters * 8 * 2 / (ms * 1e-3) / 1e12;
    }
    if (e == cudaSuccess) {
        e = time_ms([&] { fp64_fma_kernel<<<sms * 8, 256>>>(iters / 8, (double *)sink); }, 5, &ms);
        out->fp64_tflops = threads * (iters / 8) * 8 * 2 / (ms * 1e-3) / 1e12;
    }
    if (e == cudaSuccess) {
        e = time_ms([&] { cos_kernel<<<sms * 8, 256>>>(iters / 4, sink); }, 5, &ms);
        out->cos_gops = threads * (iters / 4) * 8 / (ms * 1e-3) / 1e9;
    }
    cudaFree(buf);
    cudaFree(sink);
    return (int)e;
}

}  // extern "C"
