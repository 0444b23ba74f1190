// source.cu -- crp_source_sample_device: the source features of
// crp_source_sample (SourceParticleType / SourceMultipleParticleTypes,
// SourceEnergy / SourcePowerLawSpectrum, SourceIsotropicEmission /
// SourceDirection; Source.cpp:74-150, :742, :808) drawn on the device for
// throughput runs.  The draws come from a counter-based Philox4x32-10 stream
// (candidate index, block) instead of the reference's sequential MT19937, so
// any candidate can be drawn by any thread in any order and a run split over
// calls (first) or ranks gives the same candidates; the distributions are the
// reference's, the sequence is not.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "chain.cuh"
#include "engine_internal.h"

namespace crp {
void set_last_error(const char *msg);                            // crp_engine.cu
crp_status check_device_ptr(const void *ptr, const char *what);  // crp_engine.cu
}

namespace {

crp_status fail(crp_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    crp::set_last_error(buf);
    return st;
}

constexpr int kMaxTypes = 256;
constexpr uint32_t kSourceTag = 0x536f7572u;  // separates these counters from other Philox uses

// Everything one launch reads, passed by value (under the 4 KB parameter limit).
struct SourceParams {
    int32_t n_types, spectrum, log_uniform, isotropic;
    int32_t ids[kMaxTypes];
    double cdf[kMaxTypes];       // cumulative abundances (Random::randBin's table)
    double p1, p2, ex, energy;   // power law: pow(emax, index + 1), pow(emin, index + 1), 1 / (index + 1)
    double dir[3];
    uint64_t seed, first, n;
};
static_assert(sizeof(SourceParams) <= 4096, "kernel parameter limit");

// 53-bit uniform in [0, 1) from two 32-bit words
__device__ __forceinline__ double uniform53(uint32_t hi, uint32_t lo) {
    return (double)(((uint64_t)hi << 21) | (uint64_t)(lo >> 11)) * 0x1.0p-53;
}

__global__ void __launch_bounds__(256) source_kernel(const SourceParams P, int32_t *__restrict__ id,
                                                     double *__restrict__ energy, double *__restrict__ dir) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        const uint64_t c = P.first + i;
        // word w of candidate c: word w % 4 of Philox({lo(c), hi(c), tag + w / 4, 0}, seed)
        const uint4 a = crp::philox4x32_10(make_uint4((uint32_t)c, (uint32_t)(c >> 32), kSourceTag, 0u),
                                           (uint32_t)P.seed, (uint32_t)(P.seed >> 32));
        const uint4 b = crp::philox4x32_10(make_uint4((uint32_t)c, (uint32_t)(c >> 32), kSourceTag + 1u, 0u),
                                           (uint32_t)P.seed, (uint32_t)(P.seed >> 32));
        // SourceMultipleParticleTypes: Random::randBin, the first bin whose cumulative weight reaches u
        int32_t pid = P.ids[0];
        if (P.n_types > 1) {
            const double u = __dmul_rn(uniform53(a.x, a.y), P.cdf[P.n_types - 1]);
            int k = 0;
            while (k < P.n_types - 1 && P.cdf[k] < u) k++;
            pid = P.ids[k];
        }
        id[i] = pid;
        // SourcePowerLawSpectrum: Random::randPowerLaw
        double e = P.energy;
        if (P.spectrum) {
            const double u = uniform53(a.z, a.w);
            // products and sums rounded separately (no contraction), as the reference's host code
            const double v = __dadd_rn(__dmul_rn(__dsub_rn(P.p1, P.p2), u), P.p2);
            e = P.log_uniform ? exp(v) : pow(v, P.ex);
        }
        energy[i] = e;
        // SourceIsotropicEmission: Random::randVector; then ParticleState::setDirection's normalisation
        double x = P.dir[0], y = P.dir[1], z = P.dir[2];
        if (P.isotropic) {
            z = __dadd_rn(-1.0, __dmul_rn(2.0, uniform53(b.x, b.y)));
            const double t = __dadd_rn(-M_PI, __dmul_rn(M_PI - -M_PI, uniform53(b.z, b.w)));
            const double r = sqrt(__dsub_rn(1.0, __dmul_rn(z, z)));
            x = __dmul_rn(r, cos(t));
            y = __dmul_rn(r, sin(t));
        }
        const double nrm = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
        dir[i] = x / nrm;
        dir[P.n + i] = y / nrm;
        dir[2 * P.n + i] = z / nrm;
    }
}

}  // namespace

extern "C" crp_status crp_source_sample_device(const crp_source_desc *src, uint64_t seed, uint64_t first,
                                               uint64_t n, int32_t *id, double *energy, double *dir_xyz,
                                               void *stream) {
    if (!src) return fail(CRP_ERR_INVALID_ARGUMENT, "crp_source_sample_device: src is NULL");
    if (src->n_types < 1 || src->n_types > kMaxTypes || !src->ids)
        return fail(CRP_ERR_INVALID_ARGUMENT, "SourceMultipleParticleTypes: no nuclei set (1 to 256 types)");
    if (src->spectrum && ((src->emin < 0) || (src->emax < src->emin)))
        return fail(CRP_ERR_INVALID_ARGUMENT, "Power law distribution only possible for 0 <= min <= max");
    if (n == 0) return CRP_OK;
    const void *outs[3] = {id, energy, dir_xyz};
    for (const void *q : outs) {
        crp_status st = crp::check_device_ptr(q, "crp_source_sample_device: an output array");
        if (st) return st;
    }
    SourceParams P;
    std::memset(&P, 0, sizeof(P));
    P.n_types = src->n_types;
    P.spectrum = src->spectrum != 0;
    P.isotropic = src->isotropic != 0;
    double acc = 0;
    for (int i = 0; i < src->n_types; i++) {
        const double w = src->abundances ? src->abundances[i] : 1.0;
        if (!(w >= 0)) return fail(CRP_ERR_INVALID_ARGUMENT, "SourceMultipleParticleTypes: negative abundance");
        acc = acc + w;
        P.ids[i] = src->ids[i];
        P.cdf[i] = acc;
    }
    if (P.n_types > 1 && !(acc > 0))
        return fail(CRP_ERR_INVALID_ARGUMENT, "SourceMultipleParticleTypes: abundances sum to zero");
    if (P.spectrum) {  // Random::randPowerLaw's constants, with the host's libm
        if (std::fabs(src->index + 1.0) < 2.220446049250313e-16) {
            P.log_uniform = 1;
            P.p1 = std::log(src->emax);
            P.p2 = std::log(src->emin);
        } else {
            P.p1 = std::pow(src->emax, src->index + 1);
            P.p2 = std::pow(src->emin, src->index + 1);
            P.ex = 1 / (src->index + 1);
        }
    }
    P.energy = src->energy;
    for (int k = 0; k < 3; k++) P.dir[k] = src->direction[k];
    if (!P.isotropic && !(P.dir[0] * P.dir[0] + P.dir[1] * P.dir[1] + P.dir[2] * P.dir[2] > 0))
        return fail(CRP_ERR_INVALID_ARGUMENT, "SourceDirection: zero direction");
    P.seed = seed;
    P.first = first;
    P.n = n;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return fail(CRP_ERR_CUDA, "crp_source_sample_device: %s", cudaGetErrorString(e));
    const uint64_t blocks_needed = (n + 255) / 256;
    const uint64_t cap = (uint64_t)sms * 8;
    const unsigned grid = (unsigned)(blocks_needed < cap ? blocks_needed : cap);
    source_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(P, id, energy, dir_xyz);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CRP_ERR_CUDA, "crp_source_sample_device launch: %s", cudaGetErrorString(e));
    return CRP_OK;
}
