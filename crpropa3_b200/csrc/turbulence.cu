// turbulence.cu -- turbulent Grid3f generation on the device:
// GridTurbulence (GridTurbulence.cpp:29-123), SimpleGridTurbulence
// (SimpleGridTurbulence.cpp:19-115), HelicalGridTurbulence
// (HelicalGridTurbulence.cpp:19-127).
//
// The reference fills the half-spectrum B(k) mode by mode in one loop that
// draws from a single MT19937 stream, runs FFTW's inverse real transform on
// each component and rescales the grid to Brms.  Here:
//   1. one thread per half-spectrum mode flags the modes in the turbulent
//      range (kMin <= |k| <= kMax, |k| of the float wave vector as the
//      reference forms it) and an exclusive scan (CUB) numbers them in the
//      reference's loop order;
//   2. the host draws the reference's sequence for that many modes
//      (crp_turbulence_draws) and one copy takes it to the device;
//   3. one thread per mode builds the orthogonal base and the complex
//      amplitude from its own draws, in the reference's float / double
//      arithmetic;
//   4. cuFFT's C2R (unnormalised like FFTW's) transforms each component;
//   5. one kernel interleaves the components into Vector3f cells and sums
//      |b|^2 per block in double (squares included); the host finishes the sum and one kernel
//      scales the cells by Brms / rms rounded to float (scaleGrid,
//      GridTools.cpp:16, rmsFieldStrength :59).
// Traffic is a few passes over the grid; the FFT dominates.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdio>
#include <vector>

#include "crp_gpu.h"

namespace crp {
void set_last_error(const char *msg);
}

namespace {

crp_status turb_fail(crp_status st, const char *msg) {
    crp::set_last_error(msg);
    return st;
}

#define TURB_CUDA(call)                                                        \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            char b_[256];                                                      \
            snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_)); \
            crp::set_last_error(b_);                                           \
            return CRP_ERR_CUDA;                                               \
        }                                                                      \
    } while (0)

struct KSpace {
    uint64_t n, n2;
    double kmin, kmax;
};

// wave number of index i: (double)i / n - i / (n / 2) (GridTurbulence.cpp:47)
__host__ __device__ __forceinline__ double wave_number(uint64_t i, uint64_t n) {
    return (double)i / (double)n - (double)(i / (n / 2));
}

// |ek| of the Vector3f wave vector, float arithmetic (Vector3.h getR)
__host__ __device__ __forceinline__ float k_length(float x, float y, float z) {
#ifdef __CUDA_ARCH__
    return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
#else
    return std::sqrt(x * x + y * y + z * z);
#endif
}

__host__ __device__ __forceinline__ bool kept(const KSpace &K, uint64_t i, float &ex, float &ey, float &ez,
                                              double &k) {
    const uint64_t ix = i / (K.n * K.n2), iy = (i / K.n2) % K.n, iz = i % K.n2;
    ex = (float)wave_number(ix, K.n);
    ey = (float)wave_number(iy, K.n);
    ez = (float)wave_number(iz, K.n);
    k = (double)k_length(ex, ey, ez);
    return !((k < K.kmin) || (k > K.kmax));
}

__global__ void flag_kernel(KSpace K, uint64_t total, unsigned int *flags) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float ex, ey, ez;
    double k;
    flags[i] = kept(K, i, ex, ey, ez, k) ? 1u : 0u;
}

struct Amp {
    int kind;
    double lambda, lbendover, sindex, qindex, alpha, helicity, mu0;
};

struct f3v { float x, y, z; };

__device__ __forceinline__ f3v fcross(f3v a, f3v b) {  // Vector3::cross (Vector3.h:268)
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(b.y, a.z)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(b.z, a.x)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(b.x, a.y))};
}
__device__ __forceinline__ float flen(f3v a) {
    return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z)));
}
__device__ __forceinline__ f3v fdiv(f3v a, float s) { return {__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)}; }

// Vector3f::getAngleTo(n0) < limit with n0 = (1, 1, 1) (Vector3.h:172-186);
// the limit is float(1e-3) in GridTurbulence and SimpleGridTurbulence
// (isParallelTo), the double 1e-3 in HelicalGridTurbulence
__device__ __forceinline__ bool parallel_to_111(f3v e, double limit) {
    const f3v n0 = {1.f, 1.f, 1.f};
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(e.x, n0.x), __fmul_rn(e.y, n0.y)), __fmul_rn(e.z, n0.z));
    const float c = __fdiv_rn(__fdiv_rn(dot, flen(n0)), flen(e));
    float angle;
    if (c >= 1.f) angle = 0.f;
    else if (c <= -1.f) angle = (float)M_PI;
    else angle = acosf(c);
    return (double)angle < limit;
}

// TurbulenceSpectrum::energySpectrum (TurbulentField.h:75)
__device__ __forceinline__ double energy_spectrum(double k, const Amp &A) {
    const double kHat = k * A.lbendover;
    return pow(kHat, A.qindex) / pow(1.0 + kHat * kHat, (A.sindex + A.qindex) / 2.0 + 1.0);
}

__global__ void amplitude_kernel(KSpace K, Amp A, uint64_t total, const unsigned int *flags,
                                 const unsigned int *index, const double *draws, float2 *bx, float2 *by,
                                 float2 *bz) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    if (!flags[i]) {
        bx[i] = by[i] = bz[i] = make_float2(0.f, 0.f);
        return;
    }
    float ex, ey, ez;
    double k;
    kept(K, i, ex, ey, ez, k);
    const f3v ek = {ex, ey, ez};
    f3v e1, e2;
    if (parallel_to_111(ek, A.kind == CRP_TURBULENCE_HELICAL ? 1e-3 : (double)1e-3f)) {
        e1 = {-1.f, 1.f, 0.f};
        e2 = {1.f, 1.f, -2.f};
    } else {
        e1 = fcross({1.f, 1.f, 1.f}, ek);
        e2 = fcross(ek, e1);
    }
    e1 = fdiv(e1, flen(e1));
    e2 = fdiv(e2, flen(e2));
    const uint64_t j = index[i];
    if (A.kind == CRP_TURBULENCE_HELICAL) {  // HelicalGridTurbulence.cpp:87-116
        const double *d = draws + 3 * j;
        const double pre = A.mu0 / (4 * M_PI * pow(k, 3));
        const double tot = fabs(d[0] * pow(k, A.alpha / 2));
        const double bp = pre * sqrt((1 + A.helicity) / 2) * tot;
        const double bm = pre * sqrt((1 - A.helicity) / 2) * tot;
        const double tp = 2 * M_PI * d[1], tm = 2 * M_PI * d[2];
        const double ctp = cos(tp), stp = sin(tp), ctm = cos(tm), stm = sin(tm);
        const double s2 = sqrt(2.);
        const double re1 = bp * ctp + bm * ctm, re2 = -bp * stp + bm * stm;
        const double im1 = bp * stp + bm * stm, im2 = bp * ctp - bm * ctm;
        bx[i] = make_float2((float)((re1 * e1.x + re2 * e2.x) / s2), (float)((im1 * e1.x + im2 * e2.x) / s2));
        by[i] = make_float2((float)((re1 * e1.y + re2 * e2.y) / s2), (float)((im1 * e1.y + im2 * e2.y) / s2));
        bz[i] = make_float2((float)((re1 * e1.z + re2 * e2.z) / s2), (float)((im1 * e1.z + im2 * e2.z) / s2));
        return;
    }
    double theta, phase, scale;
    if (A.kind == CRP_TURBULENCE_SIMPLE) {  // SimpleGridTurbulence.cpp:88-93
        const double *d = draws + 3 * j;
        theta = 2 * M_PI * d[0];
        scale = d[1] * pow(k, A.alpha / 2);
        phase = 2 * M_PI * d[2];
    } else {                                // GridTurbulence.cpp:96-104
        const double *d = draws + 2 * j;
        theta = 2 * M_PI * d[0];
        scale = sqrt(energy_spectrum(k * A.lambda, A));
        phase = 2 * M_PI * d[1];
    }
    // b = e1 cos(theta) + e2 sin(theta) in float; b *= scale (rounded to float)
    const float ct = (float)cos(theta), st = (float)sin(theta), sc = (float)scale;
    const float b[3] = {__fmul_rn(__fadd_rn(__fmul_rn(e1.x, ct), __fmul_rn(e2.x, st)), sc),
                        __fmul_rn(__fadd_rn(__fmul_rn(e1.y, ct), __fmul_rn(e2.y, st)), sc),
                        __fmul_rn(__fadd_rn(__fmul_rn(e1.z, ct), __fmul_rn(e2.z, st)), sc)};
    const double cp = cos(phase), sp = sin(phase);
    bx[i] = make_float2((float)(b[0] * cp), (float)(b[0] * sp));
    by[i] = make_float2((float)(b[1] * cp), (float)(b[1] * sp));
    bz[i] = make_float2((float)(b[2] * cp), (float)(b[2] * sp));
}

// interleave the three real components into Vector3f cells, per-block sum of |b|^2
__global__ void interleave_kernel(const float *rx, const float *ry, const float *rz, uint64_t cells, float *out,
                                  double *partial) {
    __shared__ double red[256];
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double v2 = 0;
    if (i < cells) {
        const float x = rx[i], y = ry[i], z = rz[i];
        out[3 * i] = x;
        out[3 * i + 1] = y;
        out[3 * i + 2] = z;
        // |b|^2 in double: the float squares of rmsFieldStrength (getR2, GridTools.cpp:59) underflow
        // to zero for the tiny amplitudes of SI spectra with a small bend-over scale
        v2 = (double)x * x + (double)y * y + (double)z * z;
    }
    red[threadIdx.x] = v2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void scale_kernel(float *v, uint64_t count, float a) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) v[i] = __fmul_rn(v[i], a);
}

struct Scratch {
    std::vector<void *> p;
    cufftHandle plan = 0;
    bool has_plan = false;
    ~Scratch() {
        if (has_plan) cufftDestroy(plan);
        for (void *q : p) cudaFree(q);
    }
    template <typename T>
    cudaError_t alloc(T **out, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, sizeof(T) * (count ? count : 1));
        if (e == cudaSuccess) p.push_back(q);
        *out = static_cast<T *>(q);
        return e;
    }
};

crp_status check_desc(const crp_turbulence_desc *d, KSpace &K) {
    if (!d) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulence descriptor is NULL");
    if (d->kind < CRP_TURBULENCE_GRID || d->kind > CRP_TURBULENCE_HELICAL)
        return turb_fail(CRP_ERR_INVALID_ARGUMENT, "unknown turbulence kind");
    // n <= 1024 keeps the half-spectrum below 2^31 modes (the scan's count)
    if (d->n < 2 || d->n > 1024) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulence grid size must be in [2, 1024]");
    if (!(d->spacing > 0)) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulence spacing must be > 0");
    // GridTurbulence::checkGridRequirements (GridTurbulence.cpp:126)
    if (d->lmin < 2 * d->spacing) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulentField: lMin < 2 * spacing");
    if (d->lmax > d->n * d->spacing) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulentField: lMax > size");
    if (d->lmax < d->lmin) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "lMax < lMin");
    if (d->kind == CRP_TURBULENCE_HELICAL && !(d->helicity >= -1 && d->helicity <= 1))
        return turb_fail(CRP_ERR_INVALID_ARGUMENT, "HelicalGridTurbulence: H must be in [-1, 1]");
    K.n = d->n;
    K.n2 = d->n / 2 + 1;
    K.kmin = d->spacing / d->lmax;
    K.kmax = d->spacing / d->lmin;
    return CRP_OK;
}

}  // namespace

extern "C" {

crp_status crp_turbulence_modes(const crp_turbulence_desc *d, uint64_t *n_modes) {
    KSpace K;
    crp_status st = check_desc(d, K);
    if (st) return st;
    if (!n_modes) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "n_modes is NULL");
    uint64_t m = 0;
    const uint64_t total = K.n * K.n * K.n2;
    for (uint64_t i = 0; i < total; i++) {
        float ex, ey, ez;
        double k;
        m += kept(K, i, ex, ey, ez, k) ? 1 : 0;
    }
    *n_modes = m;
    return CRP_OK;
}

crp_status crp_turbulence_grid(const crp_turbulence_desc *d, float *out_device, void *stream) {
    KSpace K;
    crp_status st = check_desc(d, K);
    if (st) return st;
    if (!out_device) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "out_device is NULL");
    if (d->seed == 0) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "seed 0 is not reproducible; give a non-zero seed");
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, out_device) != cudaSuccess || attr.type != cudaMemoryTypeDevice)
        return turb_fail(CRP_ERR_INVALID_ARGUMENT, "out_device is not device memory");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t n = K.n, total = n * n * K.n2, cells = n * n * n;
    const unsigned threads = 256;
    const unsigned blocks_k = (unsigned)((total + threads - 1) / threads);
    const unsigned blocks_c = (unsigned)((cells + threads - 1) / threads);
    Scratch sc;
    unsigned int *flags, *index;
    TURB_CUDA(sc.alloc(&flags, total));
    TURB_CUDA(sc.alloc(&index, total));
    flag_kernel<<<blocks_k, threads, 0, s>>>(K, total, flags);
    TURB_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    TURB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flags, index, (int)total, s));
    unsigned char *tmp;
    TURB_CUDA(sc.alloc(&tmp, tmp_bytes));
    TURB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flags, index, (int)total, s));
    unsigned int last_flag = 0, last_index = 0;
    TURB_CUDA(cudaMemcpyAsync(&last_flag, flags + total - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    TURB_CUDA(cudaMemcpyAsync(&last_index, index + total - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    TURB_CUDA(cudaStreamSynchronize(s));
    const uint64_t modes = (uint64_t)last_flag + last_index;
    const int per = d->kind == CRP_TURBULENCE_GRID ? 2 : 3;
    std::vector<double> h_draws(per * modes);
    st = crp_turbulence_draws((uint32_t)d->seed, d->kind, modes, h_draws.data());
    if (st) return st;
    double *draws;
    TURB_CUDA(sc.alloc(&draws, h_draws.size()));
    TURB_CUDA(cudaMemcpyAsync(draws, h_draws.data(), sizeof(double) * h_draws.size(), cudaMemcpyHostToDevice, s));
    float2 *bk;
    TURB_CUDA(sc.alloc(&bk, 3 * total));
    Amp A;
    A.kind = d->kind;
    A.lambda = 1 / d->spacing * 2 * M_PI;  // GridTurbulence.cpp:55
    A.lbendover = d->lbendover;
    A.sindex = d->sindex;
    A.qindex = d->qindex;
    A.alpha = -d->sindex - 2;              // SimpleGridTurbulence.cpp:15
    A.helicity = d->helicity;
    A.mu0 = 4 * M_PI * 1e-7;               // Units.h mu0 (newton / ampere^2 = 1)
    amplitude_kernel<<<blocks_k, threads, 0, s>>>(K, A, total, flags, index, draws, bk, bk + total,
                                                  bk + 2 * total);
    TURB_CUDA(cudaGetLastError());
    float *real;
    TURB_CUDA(sc.alloc(&real, 3 * cells));
    if (cufftPlan3d(&sc.plan, (int)n, (int)n, (int)n, CUFFT_C2R) != CUFFT_SUCCESS)
        return turb_fail(CRP_ERR_CUDA, "cufftPlan3d failed");
    sc.has_plan = true;
    if (cufftSetStream(sc.plan, s) != CUFFT_SUCCESS) return turb_fail(CRP_ERR_CUDA, "cufftSetStream failed");
    for (int c = 0; c < 3; c++) {
        if (cufftExecC2R(sc.plan, reinterpret_cast<cufftComplex *>(bk + c * total), real + c * cells) != CUFFT_SUCCESS)
            return turb_fail(CRP_ERR_CUDA, "cufftExecC2R failed");
    }
    double *partial;
    TURB_CUDA(sc.alloc(&partial, blocks_c));
    interleave_kernel<<<blocks_c, threads, 0, s>>>(real, real + cells, real + 2 * cells, cells, out_device, partial);
    TURB_CUDA(cudaGetLastError());
    std::vector<double> h_partial(blocks_c);
    TURB_CUDA(cudaMemcpyAsync(h_partial.data(), partial, sizeof(double) * blocks_c, cudaMemcpyDeviceToHost, s));
    TURB_CUDA(cudaStreamSynchronize(s));
    double sum = 0;
    for (double v : h_partial) sum += v;
    const double rms = std::sqrt(sum / n / n / n);  // rmsFieldStrength (GridTools.cpp:59)
    if (!(rms > 0)) return turb_fail(CRP_ERR_INVALID_ARGUMENT, "turbulence: no mode in [kMin, kMax]");
    const float a = (float)(d->brms / rms);         // scaleGrid: Vector3f *= double -> float factor
    scale_kernel<<<(unsigned)((3 * cells + threads - 1) / threads), threads, 0, s>>>(out_device, 3 * cells, a);
    TURB_CUDA(cudaGetLastError());
    TURB_CUDA(cudaStreamSynchronize(s));
    return CRP_OK;
}

}  // extern "C"
