// mixed_device.cuh -- device code of the mixed-precision form shared by its
// translation units (step_mixed.cu, step_mixed_bp.cu): field evaluation,
// the propagation modules and the chunked stepping kernel template.
//
// Same modules and module order as the FP64 form (step_fp64.cu), with the
// arithmetic split by what each quantity needs:
//   * FP64: position, trajectory length, time, the step controller's error
//     sum and its pow(), grid coordinates before the cell split, wave phases
//     before range reduction, and the direction vector (accumulated as
//     u <- u + du with du formed in FP32);
//   * FP32: field interpolation and wave sums, the Boris rotation, the
//     Cash-Karp and DiffusionSDE stage derivatives and their weighted sums.
// Rounding errors of FP32 then enter only through increments that are small
// against the FP64 quantities they are added to, which keeps the
// accumulated error of 10^3-10^6 steps at the FP64 level of the increments'
// relative error times their size.
#pragma once

#include <type_traits>

#include "chain.cuh"
#include "engine_internal.h"
#include "grid_interp.cuh"
#include "uf23.cuh"
#include "pt11.cuh"
#include "tf17.cuh"
#include "jf12.cuh"
#include "kst24_cmz.cuh"
#include "advection.cuh"


// Resident blocks of 128 threads per SM the register budget of the
// fixed-step Boris and the Cash-Karp kernels is sized for (measured on the
// grid workloads: both are bound by gather latency, and more warps in
// flight pay until spills set in).
#ifndef CRP_BP_FIXED_MIN_BLOCKS
#define CRP_BP_FIXED_MIN_BLOCKS 6
#endif
#ifndef CRP_CK_MIN_BLOCKS
#define CRP_CK_MIN_BLOCKS 3
#endif

namespace crp {
namespace {

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 f3mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 cross(f3 a, f3 v) {
    return {a.y * v.z - v.y * a.z, a.z * v.x - v.z * a.x, a.x * v.y - v.x * a.y};
}
__device__ __forceinline__ float dot(f3 a, f3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double clipd(double x, double lo, double hi) { return dmax(lo, dmin(x, hi)); }

__device__ __forceinline__ int wrap(int i, int n, bool pow2) {
    return pow2 ? (i & (n - 1)) : (((i % n) + n) % n);
}

// Trilinear Grid3f interpolation: FP64 cell coordinates, FP32 weights and
// values (the reference's own interpolation arithmetic is FP32, Grid.h:571).
// With a cell cache (FS_GRID kernels) the 8 corners are loaded only when the
// cell changes.
// PER: the grid is periodic with power-of-two dimensions, has no clipVolume
// and has the padded copy (FS_GRID_PERIODIC): those branches are compiled out.
// The periodic power-of-two case in two parts: grid_cell_load finds the
// cell of (x, y, z) and, when it is not the cached one, loads its 8 corners
// into the candidate's cache; grid_cell_interp forms the trilinear sum from
// the cache.
struct CellFrac { float fx0, fy0, fz0; };

__device__ __forceinline__ CellFrac grid_cell_load(const DevGrid &g, double x, double y, double z, Cand &cc) {
    const double rx = (x - g.gox) * g.inv_sx, ry = (y - g.goy) * g.inv_sy, rz = (z - g.goz) * g.inv_sz;
    const double flx = floor(rx), fly = floor(ry), flz = floor(rz);
    const CellFrac f{(float)(rx - flx), (float)(ry - fly), (float)(rz - flz)};
    const int ix0 = wrap((int)flx, g.nx, true), ix1 = (ix0 + 1 == g.nx) ? 0 : ix0 + 1;
    const int iy0 = wrap((int)fly, g.ny, true), iy1 = (iy0 + 1 == g.ny) ? 0 : iy0 + 1;
    const int iz0 = wrap((int)flz, g.nz, true), iz1 = (iz0 + 1 == g.nz) ? 0 : iz0 + 1;
    // 32-bit cell indices (fewer than 2^31 cells)
    const unsigned sy = (unsigned)g.nz, sx = (unsigned)g.ny * (unsigned)g.nz;
    const unsigned b00 = (unsigned)ix0 * sx + (unsigned)iy0 * sy, b10 = (unsigned)ix1 * sx + (unsigned)iy0 * sy;
    const unsigned b01 = (unsigned)ix0 * sx + (unsigned)iy1 * sy, b11 = (unsigned)ix1 * sx + (unsigned)iy1 * sy;
    const unsigned idx[8] = {b00 + iz0, b10 + iz0, b01 + iz0, b00 + iz1, b10 + iz1, b01 + iz1, b11 + iz0, b11 + iz1};
    const long long k0 = (long long)idx[0], k7 = (long long)idx[7];
    if (k0 != cc.cell0 || k7 != cc.cell7) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const float4 v = __ldg(g.values4 + idx[k]);
            cc.corner[k][0] = v.x; cc.corner[k][1] = v.y; cc.corner[k][2] = v.z;
        }
        cc.cell0 = k0; cc.cell7 = k7;
    }
    return f;
}

__device__ __forceinline__ f3 grid_cell_interp(const CellFrac &f, const Cand &cc) {
    const float fx0 = f.fx0, fy0 = f.fy0, fz0 = f.fz0;
    const float fx1 = 1.f - fx0, fy1 = 1.f - fy0, fz1 = 1.f - fz0;
    const float w[8] = {fx1 * fy1 * fz1, fx0 * fy1 * fz1, fx1 * fy0 * fz1, fx1 * fy1 * fz0,
                        fx0 * fy1 * fz0, fx1 * fy0 * fz0, fx0 * fy0 * fz1, fx0 * fy0 * fz0};
    float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        bx = fmaf(cc.corner[k][0], w[k], bx);
        by = fmaf(cc.corner[k][1], w[k], by);
        bz = fmaf(cc.corner[k][2], w[k], bz);
    }
    return f3mk(bx, by, bz);
}

template <bool CACHE, bool PER = false>
__device__ __forceinline__ f3 grid_field_t(const DevGrid &g, double x, double y, double z, Cand *cc) {
    if (CACHE && PER) return grid_cell_interp(grid_cell_load(g, x, y, z, *cc), *cc);
    if (!PER && g.interp != CRP_INTERPOLATION_TRILINEAR) {  // tricubic, nearest (Grid.h:328-331)
        const gi3 v = gi_vector_other(g, x, y, z);
        return f3mk(v.x, v.y, v.z);
    }
    if (!PER && g.clip_volume) {
        bool in = (x >= g.ox) && (x <= g.ex) && (y >= g.oy) && (y <= g.ey) && (z >= g.oz) && (z <= g.ez);
        if (!in) return f3mk(0.f, 0.f, 0.f);
    }
    double rx = (x - g.gox) * g.inv_sx, ry = (y - g.goy) * g.inv_sy, rz = (z - g.goz) * g.inv_sz;
    double flx = floor(rx), fly = floor(ry), flz = floor(rz);
    float fx0 = (float)(rx - flx), fy0 = (float)(ry - fly), fz0 = (float)(rz - flz);
    int ix0, ix1, iy0, iy1, iz0, iz1;
    if (!PER && g.reflective) {
        double r[3] = {rx, ry, rz};
        int n[3] = {g.nx, g.ny, g.nz}, lo[3], hi[3];
        float f[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double v = r[a];
            int guard = 0;
            while (((v < -0.5) || (v > (n[a] - 0.5))) && guard < 64) {
                v = 2 * n[a] * (v > (n[a] - 0.5)) - v - 1;
                guard++;
            }
            lo[a] = (int)floor(v);
            hi[a] = lo[a] + (lo[a] < n[a] - 1);
            if (v < 0) { lo[a] = 0; hi[a] = 0; }
            if (lo[a] < 0 || lo[a] >= n[a]) { lo[a] = 0; hi[a] = 0; }
            f[a] = (float)(v - floor(v));
        }
        ix0 = lo[0]; ix1 = hi[0]; iy0 = lo[1]; iy1 = hi[1]; iz0 = lo[2]; iz1 = hi[2];
        fx0 = f[0]; fy0 = f[1]; fz0 = f[2];
    } else {
        bool p2 = PER || g.pow2 != 0;
        ix0 = wrap((int)flx, g.nx, p2); ix1 = (ix0 + 1 == g.nx) ? 0 : ix0 + 1;
        iy0 = wrap((int)fly, g.ny, p2); iy1 = (iy0 + 1 == g.ny) ? 0 : iy0 + 1;
        iz0 = wrap((int)flz, g.nz, p2); iz1 = (iz0 + 1 == g.nz) ? 0 : iz0 + 1;
    }
    const float fx1 = 1.f - fx0, fy1 = 1.f - fy0, fz1 = 1.f - fz0;
    // cell indices: 32-bit for FS_GRID_PERIODIC grids (fewer than 2^31 cells)
    using Index = typename std::conditional<PER, unsigned, size_t>::type;
    const Index sy = (Index)g.nz, sx = (Index)g.ny * (Index)g.nz;
    const Index b00 = (Index)ix0 * sx + (Index)iy0 * sy, b10 = (Index)ix1 * sx + (Index)iy0 * sy;
    const Index b01 = (Index)ix0 * sx + (Index)iy1 * sy, b11 = (Index)ix1 * sx + (Index)iy1 * sy;
    const Index idx[8] = {b00 + iz0, b10 + iz0, b01 + iz0, b00 + iz1, b10 + iz1, b01 + iz1, b11 + iz0, b11 + iz1};
    const float w[8] = {fx1 * fy1 * fz1, fx0 * fy1 * fz1, fx1 * fy0 * fz1, fx1 * fy1 * fz0,
                        fx0 * fy1 * fz0, fx1 * fy0 * fz0, fx0 * fy0 * fz1, fx0 * fy0 * fz0};
    float lc[8][3];
    float (*c)[3] = CACHE ? cc->corner : lc;
    const long long k0 = (long long)idx[0], k7 = (long long)idx[7];
    if (!CACHE || k0 != cc->cell0 || k7 != cc->cell7) {
        if (PER || g.values4) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                float4 v = __ldg(g.values4 + idx[k]);
                c[k][0] = v.x; c[k][1] = v.y; c[k][2] = v.z;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const float *p = g.values + 3 * idx[k];
                c[k][0] = __ldg(p); c[k][1] = __ldg(p + 1); c[k][2] = __ldg(p + 2);
            }
        }
        if (CACHE) { cc->cell0 = k0; cc->cell7 = k7; }
    }
    float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        bx = fmaf(c[k][0], w[k], bx);
        by = fmaf(c[k][1], w[k], by);
        bz = fmaf(c[k][2], w[k], bz);
    }
    return f3mk(bx, by, bz);
}

__device__ f3 grid_field(const DevGrid &g, double x, double y, double z) {
    return grid_field_t<false>(g, x, y, z, nullptr);
}

// PlaneWaveTurbulence sum (PlaneWaveTurbulence.cpp:231).  The phase is
// taken in turns, p = (k kappa . x + beta) / 2 pi, in FP64 (|p| reaches 1e4
// turns at kpc distances and pc wavelengths, where FP32 would keep no
// fraction); its fraction f = p - rint(p) is exact in FP64, and the FP32
// hardware cosine takes 2 pi f.  Amplitudes A xi and the sums are FP32.
// The table holds the modes in pairs (a, b), 80 bytes = five 16-byte loads:
// {k kappa / 2 pi times 2^32} of a and b as six FP64, then beta / 2 pi of a
// and b as unsigned 32-bit fixed-point turns, then A xi of a and b as six
// FP32.  An odd mode count ends with a zero-amplitude mode.  The table is
// read from global memory (read-only path) or from a copy a kernel staged in
// shared memory.
struct PwTab {
    const float4 *pairs;
    int npairs;
    double fast_limit;
};

// cos(2 pi (p + beta)) for a phase p in turns given as p * 2^32 (the table's
// scale) and beta in 32-bit fixed-point turns.  FAST (|p * 2^32| < 2^50):
// adding 1.5 * 2^52 rounds p * 2^32 to an integer whose low 32 bits are the
// fraction of a turn in fixed point; beta is added there (mod 2^32), and the
// sum's top 23 bits, shifted by half a turn, become a float in [-1/2, 1/2)
// through the exponent bits of 1.0 (no conversion instruction, 2^-23-turn
// steps, rounded).  Otherwise the FP64 fraction of p + beta rounded to FP32.
template <bool FAST>
__device__ __forceinline__ float cos_turns(double ps, unsigned beta) {
    const float twopi = 6.28318530717958647692f;
    if (FAST) {
        const unsigned lo = (unsigned)__double2loint(ps + 6755399441055744.0) + beta;
        const float f = __int_as_float(0x3f800000u | (((lo + 256u) ^ 0x80000000u) >> 9)) - 1.5f;
        return __cosf(twopi * f);
    }
    const double p = (ps + (double)beta) * 2.3283064365386962890625e-10;  // 2^-32, exact
    return __cosf(twopi * (float)(p - rint(p)));
}

// One mode pair's contribution to a position's two accumulator sets.
template <bool FAST>
__device__ __forceinline__ void pw_pair_add(double2 k0, double2 k1, double2 k2, float4 u, float4 v, double x,
                                            double y, double z, float (&acc)[6]) {
    const double p0 = fma(k0.x, x, fma(k0.y, y, k1.x * z));
    const double p1 = fma(k1.y, x, fma(k2.x, y, k2.y * z));
    const float c0 = cos_turns<FAST>(p0, __float_as_uint(u.x));
    const float c1 = cos_turns<FAST>(p1, __float_as_uint(u.y));
    acc[0] = fmaf(u.z, c0, acc[0]); acc[1] = fmaf(u.w, c0, acc[1]); acc[2] = fmaf(v.x, c0, acc[2]);
    acc[3] = fmaf(v.y, c1, acc[3]); acc[4] = fmaf(v.z, c1, acc[4]); acc[5] = fmaf(v.w, c1, acc[5]);
}

// The modes are summed in kPwGroups groups of consecutive pairs (group g:
// pairs [g np / 4, (g + 1) np / 4)), each with two accumulator sets (one per
// mode of a pair, which halves the dependence chain), and the groups are
// added as (G0 + G1) + (G2 + G3).  This is the order in which the
// DiffusionSDE kernel's block evaluates the sum cooperatively (four warps,
// one group each), so the lane-by-lane sum here gives the same bits.
constexpr int kPwGroups = 4;

__device__ __forceinline__ int pw_group_begin(int npairs, int g) { return (g * npairs) / kPwGroups; }

template <bool SHARED, bool FAST>
__device__ __forceinline__ f3 pw_group_sum(const float4 *tab, int q0, int q1, double x, double y, double z) {
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
    for (int q = q0; q < q1; q++) {
        const double2 *kd = reinterpret_cast<const double2 *>(tab + 5 * q);
        double2 k0, k1, k2;
        float4 u, v;
        if (SHARED) {
            k0 = kd[0]; k1 = kd[1]; k2 = kd[2];
            u = tab[5 * q + 3]; v = tab[5 * q + 4];
        } else {
            k0 = __ldg(kd); k1 = __ldg(kd + 1); k2 = __ldg(kd + 2);
            u = __ldg(tab + 5 * q + 3); v = __ldg(tab + 5 * q + 4);
        }
        pw_pair_add<FAST>(k0, k1, k2, u, v, x, y, z, acc);
    }
    return f3mk(acc[0] + acc[3], acc[1] + acc[4], acc[2] + acc[5]);
}

__device__ __forceinline__ f3 pw_combine(f3 g0, f3 g1, f3 g2, f3 g3) {
    return f3mk((g0.x + g1.x) + (g2.x + g3.x), (g0.y + g1.y) + (g2.y + g3.y), (g0.z + g1.z) + (g2.z + g3.z));
}

template <bool SHARED, bool FAST>
__device__ __forceinline__ f3 pw_sum_t(const float4 *tab, int npairs, double x, double y, double z) {
    const f3 g0 = pw_group_sum<SHARED, FAST>(tab, pw_group_begin(npairs, 0), pw_group_begin(npairs, 1), x, y, z);
    const f3 g1 = pw_group_sum<SHARED, FAST>(tab, pw_group_begin(npairs, 1), pw_group_begin(npairs, 2), x, y, z);
    const f3 g2 = pw_group_sum<SHARED, FAST>(tab, pw_group_begin(npairs, 2), pw_group_begin(npairs, 3), x, y, z);
    const f3 g3 = pw_group_sum<SHARED, FAST>(tab, pw_group_begin(npairs, 3), npairs, x, y, z);
    return pw_combine(g0, g1, g2, g3);
}

template <bool SHARED>
__device__ __forceinline__ f3 pw_sum(const float4 *tab, int npairs, double lim, double x, double y, double z) {
    if (fmax(fabs(x), fmax(fabs(y), fabs(z))) < lim) return pw_sum_t<SHARED, true>(tab, npairs, x, y, z);
    return pw_sum_t<SHARED, false>(tab, npairs, x, y, z);
}

__device__ __forceinline__ f3 plane_wave_field(const DevPlaneWave &w, double x, double y, double z,
                                               const PwTab *sh = nullptr) {
    if (sh) return pw_sum<true>(sh->pairs, sh->npairs, sh->fast_limit, x, y, z);
    return pw_sum<false>(w.pairs, w.npairs, w.fast_limit, x, y, z);
}

// ---------------------------------------------------------------- JF12Field
// FP32 form of JF12Field::getField (JF12Field.cpp:199-346): lengths in kpc,
// fields in muG (squares of SI positions overflow FP32), the azimuth's sine
// and cosine as y/r and x/r, the X-field elevation's as ratios of the legs,
// fast exponentials.  Not inlined: one compiled body, so every kernel that
// calls it rounds the same way.

__device__ __forceinline__ float jf_logistic_f(float x, float x0, float w) {
    return __frcp_rn(1.f + __expf(__fdividef(-2.f * (fabsf(x) - x0), w)));
}

__device__ __forceinline__ float jf_r_negx_f(const DevJF12 &J, float r, float phi) {
    const float pi = 3.14159265358979f;
    const float inv = __frcp_rn(J.tan90mp);
    float r_negx = r * __expf(-(phi - pi) * inv);
    if (r_negx > J.rarms[7]) r_negx = r * __expf(-(phi + pi) * inv);
    if (r_negx > J.rarms[7]) r_negx = r * __expf(-(phi + 3.f * pi) * inv);
    return r_negx;
}

// JF12FieldSolenoidal's disk (JF12FieldSolenoidal.cpp:115) in FP32, kpc and
// muG: the arm of (r, phi) found at r1 along the spiral, the transition
// polynomial and its derivative (:197, :219), the azimuth integral H.
__device__ __forceinline__ f3 jf12s_disk_f(const DevJF12 &J, float r, float z, float phi, float sinPhi,
                                           float cosPhi) {
    if (!((J.s_r1 < r) && (r < J.s_r2))) return f3mk(0.f, 0.f, 0.f);
    const float lf = jf_logistic_f(z, J.hdisk, J.wdisk);
    float phi1 = phi - logf(r / J.s_r1) * J.s_cotp;
    float s1, c1;
    sincosf(phi1, &s1, &c1);
    phi1 = atan2f(s1, c1);
    int idx = 1;
    while (idx < 10 && phi1 < J.s_phi0[idx]) idx += 1;
    const float hint = phi1 * J.s_b[idx] + J.s_coeff[idx];
    const float mag1 = J.s_b[idx];
    float p, q;
    if ((r > J.s_r1s) && (r < J.s_r2s)) {
        p = J.s_r1 / r;
        q = 0.f;
    } else {
        float ra = J.s_r1, rb = J.s_r1s;
        if (r >= J.s_r2s) { ra = J.s_r2; rb = J.s_r2s; }
        const float fakt = (ra / rb - 2.f) / ((ra - rb) * (ra - rb));
        p = (J.s_r1 / rb) * (2.f - r / rb + fakt * (r - rb) * (r - rb));
        q = (J.s_r1 / rb) * (2.f - 2.f * r / rb + fakt * (3.f * r * r - 4.f * r * rb + rb * rb));
    }
    const float br = p * mag1 * J.sinp;
    const float bphi = p * mag1 * J.cosp - q * hint * J.sinp;
    const float s = 1.f - lf;
    return f3mk((br * cosPhi - bphi * sinPhi) * s, (br * sinPhi + bphi * cosPhi) * s, 0.f);
}

// JF12FieldSolenoidal's X field (JF12FieldSolenoidal.cpp:131) in FP32, kpc and muG.
__device__ __forceinline__ f3 jf12s_x_f(const DevJF12 &J, float r, float z, float sinPhi, float cosPhi) {
    const float zS = J.s_zs, rXc = J.rxc, rX = J.rx, bX = J.bx, tanT = J.tanthx0, az = fabsf(z);
    const float rc = rXc + az / tanT, r0c = rXc + zS / tanT;
    if (az > zS) {
        if (r == 0.f) {
            const float a = 1.f + az * J.s_cotx / rXc;
            return f3mk(0.f, 0.f, bX / (a * a));
        }
        float bMagX, sT, cT;
        if (r < rc) {
            const float rp = r * rXc / rc;
            bMagX = bX * expf(-rp / rX) * (rXc / rc) * (rXc / rc);
            const float th = atanf(az / (r - rp));
            sincosf(th, &sT, &cT);
        } else {
            const float rp = r - az / tanT;
            bMagX = bX * expf(-rp / rX) * (rp / r);
            sT = J.sinthx0;
            cT = J.costhx0;
        }
        const float zs = z < 0.f ? -bMagX : bMagX;
        return f3mk(zs * cT * cosPhi, zs * cT * sinPhi, bMagX * sT);
    }
    float r0 = r / (1.f - 1.f / (2.f * (zS + rXc * tanT)) * (zS - z * z / zS));
    float f;
    if (r0 >= r0c) {
        r0 = r + 1.f / (2.f * tanT) * (zS - z * z / zS);
        f = 1.f + 1.f / (2.f * r * tanT / zS) * (1.f - (z / zS) * (z / zS));
    } else {
        const float g = 1.f - 1.f / (2.f + 2.f * (rXc * tanT / zS)) * (1.f - (z / zS) * (z / zS));
        f = 1.f / (g * g);
    }
    float br0, bz0;
    if (r0 < r0c) {
        const float rp = r0 * rXc / r0c;
        float st, ct;
        sincosf(atanf(zS / (r0 - rp)), &st, &ct);
        const float m = bX * expf(-rp / rX) * (rXc / r0c) * (rXc / r0c);
        br0 = m * ct;
        bz0 = m * st;
    } else {
        const float rp = r0 - zS / tanT;
        const float m = bX * expf(-rp / rX) * (rp / r0);
        br0 = m * J.costhx0;
        bz0 = m * J.sinthx0;
    }
    const float br = z / zS * f * br0;
    return f3mk(br * cosPhi, br * sinPhi, bz0 * f);
}

// regular field [muG] at (x, y, z) [kpc]
__device__ f3 jf12_regular_f(const DevJF12 &J, float x, float y, float z) {
    f3 b = f3mk(0.f, 0.f, 0.f);
    const float r2 = x * x + y * y;
    if (!(r2 + z * z < 400.f)) return b;  // d < 20 kpc
    const float r = sqrtf(r2);
    float cosPhi = 1.f, sinPhi = 0.f;
    if (r > 0.f) {
        const float ir = __frcp_rn(r);
        cosPhi = x * ir;
        sinPhi = y * ir;
    }
    const bool sol = J.d.variant == CRP_JF12_SOLENOIDAL;
    if (sol) {
        if (J.d.use_disk) {
            const f3 d = jf12s_disk_f(J, r, z, (x == 0.f && y == 0.f) ? 0.f : atan2f(y, x), sinPhi, cosPhi);
            b.x += d.x; b.y += d.y;
        }
    } else if (J.d.use_disk && r > 3.f) {
        const float lf = jf_logistic_f(z, J.hdisk, J.wdisk);
        if (r < 5.f) {
            const float bMag = J.bring * __fdividef(5.f, r) * (1.f - lf);
            b.x += -bMag * sinPhi;
            b.y += bMag * cosPhi;
        } else {
            const float r_negx = jf_r_negx_f(J, r, atan2f(y, x));
            float bMag = 0.f;
#pragma unroll
            for (int i = 7; i >= 0; i--)
                if (r_negx < J.rarms[i]) bMag = J.bdisk[i];
            bMag *= __fdividef(5.f, r) * (1.f - lf);
            b.x += bMag * (J.sinp * cosPhi - J.cosp * sinPhi);
            b.y += bMag * (J.sinp * sinPhi + J.cosp * cosPhi);
        }
    }
    const bool outside1 = r2 + z * z > 1.f;
    const float az = fabsf(z);
    if (J.d.use_toroidal_halo && outside1) {
        float bMagH = __expf(__fdividef(-az, J.z0)) * jf_logistic_f(z, J.hdisk, J.wdisk);
        if (z >= 0.f)
            bMagH *= J.bnorth * (1.f - jf_logistic_f(r, J.rnorth, J.whalo));
        else
            bMagH *= J.bsouth * (1.f - jf_logistic_f(r, J.rsouth, J.whalo));
        b.x += -bMagH * sinPhi;
        b.y += bMagH * cosPhi;
    }
    if (sol) {
        if (J.d.use_x) {
            const f3 xf = jf12s_x_f(J, r, z, sinPhi, cosPhi);
            b.x += xf.x; b.y += xf.y; b.z += xf.z;
        }
    } else if (J.d.use_x && outside1) {
        float bMagX, sinT, cosT;
        const float rc = J.rxc + __fdividef(az, J.tanthx0);
        if (r < rc) {
            const float q = __fdividef(J.rxc, rc);
            const float rp = r * q;
            bMagX = J.bx * __expf(__fdividef(-rp, J.rx)) * q * q;
            if (z == 0.f) {
                sinT = 1.f;
                cosT = 0.f;
            } else {
                // r - rp = r (rc - rxc) / rc = r (|z| / tan thetaX0) / rc, without the
                // cancellation of r - rp near the plane
                const float dr = __fdividef(r * __fdividef(az, J.tanthx0), rc);
                const float ih = rsqrtf(az * az + dr * dr);
                sinT = az * ih;
                cosT = dr * ih;
            }
        } else {
            const float rp = r - __fdividef(az, J.tanthx0);
            bMagX = J.bx * __expf(__fdividef(-rp, J.rx)) * __fdividef(rp, r);
            sinT = J.sinthx0;
            cosT = J.costhx0;
        }
        const float zs = z < 0.f ? -bMagX : bMagX;
        b.x += zs * cosT * cosPhi;
        b.y += zs * cosT * sinPhi;
        b.z += bMagX * sinT;
    }
    return b;
}

// turbulent field strength [muG] (JF12Field.cpp:301)
__device__ float jf12_turbulent_strength_f(const DevJF12 &J, float x, float y, float z) {
    const float r2 = x * x + y * y;
    if (r2 + z * z > 400.f) return 0.f;
    const float r = sqrtf(r2);
    float bDisk;
    if (r < 5.f) {
        bDisk = J.bdturb5;
    } else {
        const float r_negx = jf_r_negx_f(J, r, atan2f(y, x));
        bDisk = 0.f;
#pragma unroll
        for (int i = 7; i >= 0; i--)
            if (r_negx < J.rarms[i]) bDisk = J.bdturb[i];
        bDisk *= __fdividef(5.f, r);
    }
    const float zd = __fdividef(z, J.zdturb), zh = __fdividef(z, J.zhturb);
    bDisk *= __expf(-0.5f * zd * zd);
    const float bHalo = J.bhturb * __expf(__fdividef(-r, J.rhturb) - 0.5f * zh * zh);
    return sqrtf(bDisk * bDisk + bHalo * bHalo);
}

__device__ __noinline__ f3 jf12_field_f(const DevComponent &f, double x, double y, double z) {
    const DevJF12 &J = *f.jf;
    const float xs = (float)(x * J.inv_kpc), ys = (float)(y * J.inv_kpc), zs = (float)(z * J.inv_kpc);
    const float unit = (float)J.muG;
    f3 b = f3mk(0.f, 0.f, 0.f);
    if (J.d.use_turbulent) {
        const f3 g = grid_field(f.grid, x, y, z);
        const float s = jf12_turbulent_strength_f(J, xs, ys, zs) * unit;
        b = f3mk(g.x * s, g.y * s, g.z * s);
    }
    if (J.d.use_striated || J.d.use_regular) {
        float m = unit;
        if (J.d.use_striated)
            m *= 1.f + J.sqrtbeta * __ldg(f.mod.values + gi_nearest_cell(f.mod, x, y, z));
        const f3 r = jf12_regular_f(J, xs, ys, zs);
        b.x += r.x * m;
        b.y += r.y * m;
        b.z += r.z * m;
    }
    return b;
}

// ---------------------------------------------------------------- PT11Field
// The mixed form of PT11Field::getField (PT11Field.cpp:80-128): FP32 in kpc
// and muG, the reference's formulas; r = 0 divides by zero as the reference
// does.
__device__ __noinline__ f3 pt11_field_f(const DevComponent &f, double px, double py, double pz) {
    const DevPT11 &P = *f.pt32;
    const float x = (float)(px * P.inv_kpc), y = (float)(py * P.inv_kpc), z = (float)(pz * P.inv_kpc);
    const float r = sqrtf(x * x + y * y);
    float bx = 0.f, by = 0.f, bz = 0.f;
    if (P.use_ass || P.use_bss) {
        // theta = pi - phi, phi of Vector3::getPhi (0 on the axis)
        const float theta = 3.14159265358979f - ((x == 0.f && y == 0.f) ? 0.f : atan2f(y, x));
        const float cos_theta = -x / r, sin_theta = y / r;
        bx = -(P.sinp * cos_theta - P.cosp * sin_theta);
        by = -(-P.sinp * sin_theta - P.cosp * cos_theta);
        float m = cosf(theta - P.cotp * logf(r / P.r_sun) + P.phi);
        if (P.use_ass) m = fabsf(m);
        const float rr = r < P.r_c ? P.r_c : r;  // std::max(r, R_c)
        m *= P.b0_d * P.r_sun / rr / P.cos_phi * expf(-fabsf(z) / P.z0_d);
        bx *= m;
        by *= m;
        bz = -0.f * m;  // NaN with m on the axis, as in the reference
    }
    if (P.use_halo) {
        const float az = fabsf(z);
        float m = z > 0.f ? P.b0_hn : -P.b0_hs;
        const float z1 = az < P.z0_h ? P.z11_h : P.z12_h;
        const float v = (az - P.z0_h) / z1;
        m *= r / P.r0_h * expf(1.f - r / P.r0_h) / (1.f + v * v);
        bx += m * (-y / r);
        by += m * (x / r);
        bz += m * 0.f;
    }
    return f3mk(bx * P.muG, by * P.muG, bz * P.muG);
}

// ---------------------------------------------------------------- UF23Field
// The mixed form of UF23Field::getField (UF23Field.cpp:269-558): FP32 in the
// model's units (kpc, microgauss), the reference's formulas, with three
// rewritings that keep FP32 digits: 1 - exp(-x) as -expm1(-x); the azimuth
// difference acos(cos a cos b + sin a sin b) as |a - b| reduced to [0, pi]
// (the same angle, without acos's loss near 0); and the poloidal halo's
// t1 + t0 as 4 A^P r^P / (t1 - t0) where t0 < 0 (the same value, from
// (t1 + t0)(t1 - t0) = 4 A^P r^P, without the cancellation).
constexpr float kUffMinNormal = 1.17549435e-38f;  // numeric_limits<float>::min()
constexpr float kUffTwoPi = 6.28318530717958648f;

__device__ __forceinline__ float uff_sigmoid(float x, float x0, float w) { return 1.f / (1.f + expf(-(x - x0) / w)); }

__device__ __forceinline__ float uff_delta_phi(float a, float b) { return fabsf(remainderf(a - b, kUffTwoPi)); }

// getSpiralField (UF23Field.cpp:510)
__device__ __forceinline__ f3 uff_spiral(const DevUF23 &W, float x, float y, float z) {
    const float r2 = x * x + y * y;
    if (r2 == 0.f) return f3mk(0.f, 0.f, 0.f);
    const float r = sqrtf(r2);
    const float phi = atan2f(y, x);
    const float hdz = 1.f - uff_sigmoid(fabsf(z), W.disk_h, W.disk_w);
    const float rFacI = uff_sigmoid(r, 5.f, 0.5f);
    const float rFacO = 1.f - uff_sigmoid(r, 20.f, 0.5f);
    const float rFac = r > 1e-8f ? -expm1f(-r2) / r : r;
    const float fac = hdz * 5.f * rFac * rFacO * rFacI;
    const float phi0 = phi - logf(r / 5.f) * W.inv_tanp;
    const float b = W.b1 * cosf(phi0 - W.ph1) + W.b2 * cosf(2.f * (phi0 - W.ph2)) +
                    W.b3 * cosf(3.f * (phi0 - W.ph3));
    const float br = b * fac * W.sinp, bphi = b * fac * W.cosp, cp = x / r, sp = y / r;
    return f3mk(br * cp - bphi * sp, br * sp + bphi * cp, 0.f);
}

// getSpurField (UF23Field.cpp:453)
__device__ __forceinline__ f3 uff_spur(const DevUF23 &W, float x, float y, float z, float r) {
    const float rRef = 8.2f;
    if (r < kUffMinNormal) return f3mk(0.f, 0.f, 0.f);
    float phi = atan2f(y, x);
    if (phi < 0.f) phi += kUffTwoPi;
    const float phiRef = W.ph1;
    int iBest = -2;
    float bestDist = -1.f;
    for (int i = -1; i <= 1; ++i) {
        const float rr = rRef * expf((phi - phiRef + i * kUffTwoPi) * W.tanp);
        if (bestDist < 0.f || fabsf(r - rr) < bestDist) {
            bestDist = fabsf(r - rr);
            iBest = i;
        }
    }
    if (iBest != 0) return f3mk(0.f, 0.f, 0.f);
    const float phi0 = phi - logf(r / rRef) * W.inv_tanp;
    const float delta = uff_delta_phi(phiRef, phi0) * W.spur_inv_width;
    const float B = W.b1 * expf(-0.5f * delta * delta);
    const float wS = 5.f * (3.14159265358979f / 180.f);
    const float gS = 1.f - uff_sigmoid(uff_delta_phi(W.spur_center, phi), W.spur_length, wS);
    const float hd = 1.f - uff_sigmoid(fabsf(z), W.disk_h, W.disk_w);
    const float bS = rRef / r * B * hd * gS;
    const float br = bS * W.sinp, bphi = bS * W.cosp, cp = x / r, sp = y / r;
    return f3mk(br * cp - bphi * sp, br * sp + bphi * cp, 0.f);
}

// getToroidalHaloField (UF23Field.cpp:361)
__device__ __forceinline__ f3 uff_toroidal(const DevUF23 &W, float x, float y, float z, float r) {
    const float absZ = fabsf(z);
    const float b0 = z >= 0.f ? W.tbn : W.tbs;
    const float bPhi = b0 * (1.f - uff_sigmoid(r, W.tr, W.tw)) * uff_sigmoid(absZ, W.disk_h, W.disk_w) *
                       expf(-absZ / W.tz);
    const float cp = r > kUffMinNormal ? x / r : 1.f, sp = r > kUffMinNormal ? y / r : 0.f;
    return f3mk(-bPhi * sp, bPhi * cp, 0.f);
}

// getPoloidalHaloField (UF23Field.cpp:385), scaled so that no power of r,
// |z| or A is formed (A^P and t0^2 overflow FP32 for the models' constants):
// with R = (r/A)^P, Zc = (|z|/Z)^P (c |z|^P = A^P Zc) and m = max(0, ln R,
// ln Zc), t0 = A^P e^m t0s and t1 = A^P e^m t1s, where t0s = e^-m + Zc e^-m -
// R e^-m and t1s = sqrt(t0s^2 + 4 R e^-2m) have every term in [0, 1].  Then,
// with s = t1s + t0s and g = ln(2 e^-m / s) / P: a = r e^g, a / rOverA =
// r e^2g and rOverA^(P-2) (a^P + A^P) / t1 = e^2g (s / 2 + R e^-m) / t1s.
__device__ __forceinline__ f3 uff_poloidal(const DevUF23 &W, int model, float x, float y, float z, float r) {
    const float ln2 = 0.693147180559945309f, az = fabsf(z);
    const float lr = W.pp * logf(r / W.pa), lz = W.pp * logf(az / W.pzz);  // ln R, ln Zc (-inf at 0)
    const float m = fmaxf(0.f, fmaxf(lr, lz));
    const float eR = expf(lr - m), eZ = expf(lz - m), q = expf(lr - 2.f * m);
    const float t0 = expf(-m) + eZ - eR;
    const float t1 = sqrtf(t0 * t0 + 4.f * q);
    const float s = t0 >= 0.f ? t1 + t0 : 4.f * q / (t1 - t0);  // (t1 + t0)(t1 - t0) = 4 R e^-2m
    const float g = (ln2 - m - logf(s)) * W.inv_pp;
    const float a = r * expf(g);
    const float radial = model == CRP_UF23_EXPX ? expf(-a / W.pr) : 1.f - uff_sigmoid(a, W.pr, W.pw);
    const float Bzz = W.pb * radial, e2g = expf(2.f * g);
    const float signZ = z < 0.f ? -1.f : 1.f;
    // c |z|^(P-1) / t1 = Zc e^-m / (|z| t1s)
    const float zt = az > 0.f ? eZ / (az * t1) : 0.f;
    const float Br = Bzz * r * e2g * signZ * zt;
    const float Bz = Bzz * e2g * (0.5f * s + eR) / t1;
    if (r < kUffMinNormal) return f3mk(0.f, 0.f, Bz);
    return f3mk(Br * (x / r), Br * (y / r), Bz);
}

// getTwistedHaloField (UF23Field.cpp:318)
__device__ __forceinline__ f3 uff_twisted(const DevUF23 &W, float x, float y, float z, float r) {
    const float cp = r > kUffMinNormal ? x / r : 1.f, sp = r > kUffMinNormal ? y / r : 0.f;
    const f3 bX = uff_poloidal(W, CRP_UF23_TWISTX, x, y, z, r);
    const float bR = bX.x * cp + bX.y * sp, bZ = bX.z;
    float bPhi = 0.f;
    if (W.twist != 0.f && r != 0.f) {
        // -240 km/s in kpc/Myr
        constexpr float v0 = (float)(-240 * (1 / 3.0856775807e+16) / (1 / (1e6 * 60 * 60 * 24 * 365.25)));
        const float r0 = 1.6f, z0 = 10.f;
        const float e = expf(-r / r0), fr = -expm1f(-r / r0);
        const float t0 = expf(2.f * fabsf(z) / z0);
        const float gz = 2.f / (1.f + t0);
        const float signZ = z < 0.f ? -1.f : 1.f;
        const float deltaZ = -signZ * v0 * fr / z0 * t0 * gz * gz;
        const float deltaR = v0 * (e / r0 - fr / r) * gz;
        bPhi = (bZ * deltaZ + bR * deltaR) * W.twist;
    }
    return f3mk(bR * cp - bPhi * sp, bR * sp + bPhi * cp, bZ);
}

// UF23Field::getField (UF23Field.cpp:269) and operator() (:277), [T]
__device__ __noinline__ f3 uf23_field_f(const DevComponent &f, double px, double py, double pz) {
    const DevUF23 &W = *f.uf;
    const int model = W.d.model;
    const float x = (float)(px * W.inv_kpc), y = (float)(py * W.inv_kpc), z = (float)(pz * W.inv_kpc);
    if (x * x + y * y + z * z > W.r2max) return f3mk(0.f, 0.f, 0.f);
    const float r = sqrtf(x * x + y * y);
    const f3 d = model == CRP_UF23_SPUR ? uff_spur(W, x, y, z, r) : uff_spiral(W, x, y, z);
    f3 h;
    if (model == CRP_UF23_TWISTX) {
        h = uff_twisted(W, x, y, z, r);
    } else {
        const f3 t = uff_toroidal(W, x, y, z, r), p = uff_poloidal(W, model, x, y, z, r);
        h = f3mk(t.x + p.x, t.y + p.y, t.z + p.z);
    }
    return f3mk((d.x + h.x) * W.muG, (d.y + h.y) * W.muG, (d.z + h.z) * W.muG);
}

// ---------------------------------------------------------------- TF17Field
// The mixed form of TF17Field::getField (TF17Field.cpp:197-303): FP32 in kpc
// and muG, the reference's formulas, with 1 - exp(-x) formed as -expm1(-x)
// (no cancellation near the axis in single precision).
__device__ __forceinline__ float tf17f_zscale(const DevTF17 &T, float z) { return 1.f + z * z / T.h_p / T.h_p; }

__device__ __forceinline__ float tf17f_winding(const DevTF17 &T, float r, float z) {
    return T.cot_p0 * logf(-expm1f(-r / T.l_p) + T.eps) / tf17f_zscale(T, z);
}

__device__ __forceinline__ float tf17f_radial_scale(const DevTF17 &T, float B1, float phi_star, float z1, float phi,
                                                   float r, float z) {
    return B1 * expf(-fabsf(z1) / T.h_disk) * cosf(phi - tf17f_winding(T, r, z) - phi_star);
}

__device__ __forceinline__ float tf17f_azimuthal(const DevTF17 &T, float r, float z, float B_r, float B_z) {
    const float r_ = r / T.l_p;
    const float rscale = r > T.eps ? r_ * expf(-r_) / (-expm1f(-r_)) : 1.f - r_ / 2.f - r_ * r_ / 12.f;
    const float zs = tf17f_zscale(T, z);
    return T.cot_p0 / zs * rscale * B_r - 2.f * z * r / (T.h_p * T.h_p) / zs * tf17f_winding(T, r, z) * B_z;
}

__device__ __noinline__ f3 tf17_field_f(const DevComponent &f, double px, double py, double pz) {
    const DevTF17 &T = *f.tf32;
    const float x = (float)(px * T.inv_kpc), y = (float)(py * T.inv_kpc), z = (float)(pz * T.inv_kpc);
    const float r = sqrtf(x * x + y * y);
    const float phi = 3.14159265358979f - ((x == 0.f && y == 0.f) ? 0.f : atan2f(y, x));
    float sinPhi, cosPhi;
    sincosf(phi, &sinPhi, &cosPhi);
    float bx = 0.f, by = 0.f, bz = 0.f;
    if (T.use_disk) {
        float B_r = 0.f, B_phi = 0.f, B_z = 0.f;
        if (T.disk_model == CRP_TF17_AD1) {
            if (r > T.r1_disk) {
                const float z1z = (1.f + T.a_disk * T.r1_disk * T.r1_disk) / (1.f + T.a_disk * r * r);
                const float B_r0 = tf17f_radial_scale(T, T.b1_disk, T.phi_star_disk, z1z * z, phi, r, z);
                B_r = (T.r1_disk / r) * z1z * B_r0;
                B_z = 2.f * T.a_disk * T.r1_disk * z1z * z / (1.f + T.a_disk * r * r) * B_r0;
                B_phi = tf17f_azimuthal(T, r, z, B_r, B_z);
            } else {
                const float phi1 = tf17f_winding(T, T.r1_disk, z) + T.phi_star_disk;
                const float B_amp = T.b1_disk * expf(-fabsf(z) / T.h_disk);
                float s1, c1;
                sincosf(phi1 - phi, &s1, &c1);
                B_r = c1 * B_amp;
                B_phi = s1 * B_amp;
            }
        } else if (T.disk_model == CRP_TF17_BD1) {
            if (r > T.eps) {
                const float rr = T.r1_disk / r;
                const float z1z = 5.f / (rr * rr + 4.f / sqrtf(rr));
                const float B_r0 = tf17f_radial_scale(T, T.b1_disk, T.phi_star_disk, z1z * z, phi, r, z);
                B_r = rr * z1z * B_r0;
                B_z = -0.4f * rr / r * z1z * z1z * z * (rr * rr - 1.f / sqrtf(rr)) * B_r0;
            } else {
                const float z1z = 5.f * r * r / (T.r1_disk * T.r1_disk);
                const float B_r0 = tf17f_radial_scale(T, T.b1_disk, T.phi_star_disk, z1z * z, phi, r, z);
                B_r = 5.f * r / T.r1_disk * B_r0;
                B_z = -10.f * z / T.r1_disk * B_r0;
            }
            B_phi = tf17f_azimuthal(T, r, z, B_r, B_z);
        } else {  // CRP_TF17_DD1
            const float zsg = z >= 0.f ? 1.f : -1.f;
            const float za = fabsf(z);
            const float wind = tf17f_winding(T, r, z);
            if (za > T.eps) {
                const float z1z = T.z1_disk / za;
                const float rr = 1.5f / (sqrtf(z1z) + 0.5f / z1z);
                const float F_r = rr * r <= T.l_disk ? 1.f : expf(1.f - rr * r / T.l_disk);
                const float B_z0 = zsg * T.b1_disk * F_r * cosf(phi - wind - T.phi_star_disk);
                B_r = -0.5f / 1.5f * rr * rr * rr * r / za * (sqrtf(z1z) - 1.f / z1z) * B_z0;
                B_z = zsg * rr * rr * B_z0;
            } else {
                const float zz = za / T.z1_disk;
                const float rr = 1.5f * sqrtf(za / T.z1_disk);
                const float F_r = rr * r <= T.l_disk ? 1.f : expf(1.f - rr * r / T.l_disk);
                const float B_z0 = zsg * T.b1_disk * F_r * cosf(phi - wind - T.phi_star_disk);
                B_r = -1.125f * r / T.z1_disk * (1.f - 2.5f * zz * sqrtf(zz)) * B_z0;
                B_z = zsg * rr * rr * B_z0;
            }
            B_phi = tf17f_azimuthal(T, r, z, B_r, B_z);
        }
        bx += -(B_r * cosPhi - B_phi * sinPhi);
        by += B_r * sinPhi + B_phi * cosPhi;
        bz += B_z;
    }
    if (T.use_halo) {
        const float r1h = (1.f + T.a_halo * T.z1_halo * T.z1_halo) / (1.f + T.a_halo * z * z);
        float B_z0 = T.b1_halo * expf(-r1h * r / T.l_halo);
        if (T.halo_model == CRP_TF17_C1) B_z0 *= cosf(phi - tf17f_winding(T, r, z) - T.phi_star_halo);
        const float B_r = 2.f * T.a_halo * r1h * r1h * r * z / (1.f + T.a_halo * z * z) * B_z0;
        const float B_z = r1h * r1h * B_z0;
        const float B_phi = tf17f_azimuthal(T, r, z, B_r, B_z);
        bx += -(B_r * cosPhi - B_phi * sinPhi);
        by += B_r * sinPhi + B_phi * cosPhi;
        bz += B_z;
    }
    return f3mk(bx * T.muG, by * T.muG, bz * T.muG);
}

// ---------------------------------------------------------------- KST24Field
// The mixed form of KST24Field::getField (KST24Field.cpp:128-374): FP32 in
// the model's units (kpc, gauss), each arm's trigonometric constants formed
// once on the host.
__device__ __forceinline__ void kst24f_toroidal(float x, float y, float z, float B, float zmin, float zmax,
                                                float rmin, float rmax, f3 &v) {
    if ((z <= zmin) || (zmax <= z)) return;
    const float cR = sqrtf(x * x + y * y);
    if ((rmin <= cR) && (cR <= rmax)) {
        const float th = atan2f(y, x);
        float s, c;
        sincosf(th, &s, &c);
        v.x += B * s;
        v.y += -B * c;
    }
}

__device__ __forceinline__ void kst24f_x(const DevKST24 &K, float x, float y, float z, f3 &v) {
    const float sign = z < 0.f ? -1.f : 1.f;
    if (fabsf(z) > 10.f) return;
    const float cR = sqrtf(x * x + y * y);
    const float cR_0 = cR - z * sign * K.tan_x;
    if ((cR_0 < K.x_rmin) || (K.x_rmax < cR_0)) return;
    const float m = K.x_b * (cR_0 / cR);
    const float th = atan2f(y, x);
    float s, c;
    sincosf(th, &s, &c);
    v.x += m * c * sign * K.sin_x;
    v.y += m * s * sign * K.sin_x;
    v.z += m * K.cos_x;
}

__device__ __forceinline__ void kst24f_arm(const DevKST24Arm &A, float x, float y, float z, f3 &v) {
    if ((z < A.zmin) || (A.zmax < z)) return;
    const float p0 = x + A.x_shift, p1 = y + A.y_shift;
    const float r = sqrtf(p0 * p0 + p1 * p1);
    if ((r < A.rmin) || (A.rmax < r)) return;
    const float a_kpc = 3.f, k = A.k, twopi = 6.28318530717959f;
    const float phi = atan2f(p1, p0);
    int nn = (int)floorf((logf(r / a_kpc) - k * (phi + A.phi0)) / (twopi * k));
    float r1 = a_kpc * expf(k * (phi + A.phi0 + twopi * nn));
    const float r2 = r1 * expf(k * twopi);
    if (fabsf(r - r1) > fabsf(r - r2)) {
        r1 = r2;
        nn++;
    }
    float s, c;
    sincosf(phi, &s, &c);
    float xi = r1 * c, yi = r1 * s;
    float d1x = k * xi - yi, d1y = k * yi + xi;
    float dn = rsqrtf(d1x * d1x + d1y * d1y);
    d1x *= dn; d1y *= dn;
    const float dphi = -((xi - p0) * d1x + (yi - p1) * d1y) / (r1 / A.cos_pitch);
    r1 = a_kpc * expf(k * (phi + A.phi0 + dphi + twopi * nn));
    sincosf(phi + dphi, &s, &c);
    xi = r1 * c; yi = r1 * s;
    d1x = k * xi - yi; d1y = k * yi + xi;
    dn = rsqrtf(d1x * d1x + d1y * d1y);
    d1x *= dn; d1y *= dn;
    const float d1 = sqrtf((xi - p0) * (xi - p0) + (yi - p1) * (yi - p1));
    const float L1 = r1 / A.sin_pitch, L1s = 5.f / A.sin_pitch;
    const float gp = A.arc_radius2 * (1.f + (L1 - L1s) * A.arc_div);
    const float gz = A.arc_radius1 * (1.f + (L1 - L1s) * A.arc_div);
    float arp = (A.arc_radius2 < gp) ? gp : A.arc_radius2;
    float arz = (A.arc_radius1 < gz) ? gz : A.arc_radius1;
    if (arp > 1.2f) arp = 1.2f;
    if (arz > 1.2f) arz = 1.2f;
    const float d_at = sqrtf(powf(fabsf(d1 / arp), A.arc_eps) + powf(fabsf(z / arz), A.arc_eps));
    if ((d_at > 1.f) || (d_at < 0.f)) return;
    const float sf = (A.arc_radius1 * A.arc_radius2) / (arp * arz);
    v.x += A.b * d1x * sf;
    v.y += A.b * d1y * sf;
}

__device__ __noinline__ f3 kst24_field_f(const DevComponent &f, double px, double py, double pz) {
    const DevKST24 &K = *f.kst32;
    const float x = (float)(px * K.inv_kpc), y = (float)(py * K.inv_kpc), z = (float)(pz * K.inv_kpc);
    f3 v = f3mk(0.f, 0.f, 0.f);
    if (z > K.north_zmin) {
        kst24f_toroidal(x, y, z, K.north_b, K.north_zmin, K.north_zmax, K.north_rmin, K.north_rmax, v);
        kst24f_x(K, x, y, z, v);
    } else if (z < K.south_zmax) {
        kst24f_toroidal(x, y, z, K.south_b, K.south_zmin, K.south_zmax, K.south_rmin, K.south_rmax, v);
        kst24f_x(K, x, y, z, v);
    } else {
        const float ex = x - K.lb_x0, ey = y - K.lb_y0, ez = z - K.lb_z0;
        const float cR = sqrtf(ex * ex + ey * ey + ez * ez);
        if (cR < K.lb_rmin + K.lb_dr) {  // the Local Bubble: its shell field only
            if (!((cR < K.lb_rmin) || (K.lb_rmin + K.lb_dr < cR))) {
                const float ux = ex / cR, uy = ey / cR, uz = ez / cR;
                const float ct = ux * K.lb_dir[0] + uy * K.lb_dir[1] + uz * K.lb_dir[2];
                const float m = K.lb_b * K.lb_ampl;
                v = f3mk(m * (K.lb_dir[0] - ux * ct), m * (K.lb_dir[1] - uy * ct), m * (K.lb_dir[2] - uz * ct));
            }
        } else {
#pragma unroll 1
            for (int i = 0; i < 5; i++) kst24f_arm(K.arms[i], x, y, z, v);
            kst24f_x(K, x, y, z, v);
        }
    }
    return f3mk(v.x * K.gauss, v.y * K.gauss, v.z * K.gauss);
}

// Multiply-adds here are written out (fma) so that the result does not
// depend on how the compiler contracts the expression in each kernel that
// inlines it: the chunked and persistent launches must agree bit for bit.
// PeriodicMagneticField's map of a position into the component's cell
// (MagneticField.cpp:41-58).
__device__ __forceinline__ void component_position(const DevComponent &f, double &x, double &y, double &z) {
    if (f.periodic) {
        double qx = x - f.po[0], qy = y - f.po[1], qz = z - f.po[2];
        double nx = floor(qx / f.pe[0]), ny = floor(qy / f.pe[1]), nz = floor(qz / f.pe[2]);
        x = fma(-nx, f.pe[0], qx); y = fma(-ny, f.pe[1], qy); z = fma(-nz, f.pe[2], qz);
        if (f.periodic_reflective) {
            if ((long long)fabs(nx) % 2 == 1) x = f.pe[0] - x;
            if ((long long)fabs(ny) % 2 == 1) y = f.pe[1] - y;
            if ((long long)fabs(nz) % 2 == 1) z = f.pe[2] - z;
        }
    }
}

__device__ __forceinline__ f3 component_field(const DevComponent &f, double x, double y, double z,
                                             const PwTab *sh = nullptr) {
    component_position(f, x, y, z);
    switch (f.kind) {
    case CRP_FIELD_GRID: return grid_field(f.grid, x, y, z);
    case CRP_FIELD_MODULATED_GRID: {  // MagneticFieldGrid.cpp:51
        const float m = gi_scalar(f.mod, x, y, z);
        const f3 b = grid_field(f.grid, x, y, z);
        return f3mk(b.x * m, b.y * m, b.z * m);
    }
    case CRP_FIELD_PLANE_WAVE: return plane_wave_field(f.pw, x, y, z, sh);
    case CRP_FIELD_UNIFORM: return f3mk((float)f.uniform[0], (float)f.uniform[1], (float)f.uniform[2]);
    case CRP_FIELD_JF12: return jf12_field_f(f, x, y, z);
    case CRP_FIELD_UF23: return uf23_field_f(f, x, y, z);  // FP32 in kpc and microgauss
    case CRP_FIELD_PT11: return pt11_field_f(f, x, y, z);  // FP32 in kpc and muG
    case CRP_FIELD_ARCHIMEDEAN_SPIRAL: {  // FP64 evaluation, FP32 result
        const u3 b = archimedean_field(f.arch, x, y, z);
        return f3mk((float)b.x, (float)b.y, (float)b.z);
    }
    case CRP_FIELD_TF17: return tf17_field_f(f, x, y, z);  // FP32 in kpc and muG
    case CRP_FIELD_SINGLE_MODE: {  // FP64 evaluation (the phase reaches many turns), FP32 result
        const u3 b = single_mode_field(f.mode, x, y, z);
        return f3mk((float)b.x, (float)b.y, (float)b.z);
    }
    case CRP_FIELD_KST24: return kst24_field_f(f, x, y, z);  // FP32 in kpc and gauss
    case CRP_FIELD_CMZ: {  // FP64 evaluation, FP32 result
        const u3 b = cmz_field(*f.cmz, x, y, z);
        return f3mk((float)b.x, (float)b.y, (float)b.z);
    }
    default: {
        double r = sqrt(fma(x, x, y * y));
        double s = f.b0 / r;
        return f3mk((float)(-y * s), (float)(x * s), 0.f);
    }
    }
}

// sh: the plan's plane-wave table staged in shared memory (at most one
// plane-wave component), or null.
template <int FS>
__device__ __forceinline__ f3 field_at(const DevPlan &P, double x, double y, double z,
                                       Cand *cc = nullptr, const PwTab *sh = nullptr) {
    if (FS == FS_GRID) return grid_field_t<true>(P.fields[0].grid, x, y, z, cc);
    if (FS == FS_GRID_PERIODIC) return grid_field_t<true, true>(P.fields[0].grid, x, y, z, cc);
    if (FS == FS_PLANE_WAVE) return plane_wave_field(P.fields[0].pw, x, y, z, sh);
    if (P.n_fields == 1) return component_field(P.fields[0], x, y, z, sh);
    f3 b = f3mk(0.f, 0.f, 0.f);
#pragma unroll 1
    for (int i = 0; i < P.n_fields; i++) {
        f3 c = component_field(P.fields[i], x, y, z, sh);
        b.x += c.x; b.y += c.y; b.z += c.z;
    }
    return b;
}

// Candidate::setCurrentStep (Candidate.cpp:92): the time increment s / c is
// taken as s times the correctly rounded 1 / c (within one ulp of the
// increment; the FP64 form divides).
constexpr double kInvCLight = 1.0 / kCLight;
__device__ __forceinline__ void set_current_step(Cand &c, double s) {
    c.cur = s;
    c.len += s;
    c.time = fma(s, kInvCLight, c.time);
}

// Renormalise an FP64 direction that is within rounding of unit length:
// one Newton step of 1/sqrt(n2) from 1.
__device__ __forceinline__ void renorm(double &x, double &y, double &z) {
    double n2 = fma(x, x, fma(y, y, z * z));
    double f = fma(-0.5, n2, 1.5);
    if (fabs(n2 - 1.0) > 1e-6) f = rsqrt(n2);  // far from unit length: plain rescale
    x *= f; y *= f; z *= f;
}

// ---------------------------------------------------------------- Boris push
// The rotation and second drift of one Boris step, given the field at the
// midpoint (x, y, z) and kt = q c step / (2 E) in FP32.
__device__ __forceinline__ void bp_rotate_drift(double &x, double &y, double &z, double &ux, double &uy,
                                                double &uz, f3 B, float kt, double hh) {
    f3 t = f3mk(B.x * kt, B.y * kt, B.z * kt);   // t = B q step / (2 m c)
    float sf = __fdividef(2.f, 1.f + dot(t, t));
    f3 s = f3mk(t.x * sf, t.y * sf, t.z * sf);
    f3 u = f3mk((float)ux, (float)uy, (float)uz);
    f3 ut = cross(u, t);
    f3 v = f3mk(u.x + ut.x, u.y + ut.y, u.z + ut.z);
    f3 du = cross(v, s);
    ux += (double)du.x; uy += (double)du.y; uz += (double)du.z;
    x = fma(ux, hh, x); y = fma(uy, hh, y); z = fma(uz, hh, z);
}

// One PropagationBP::dY (PropagationBP.cpp:19) with FP32 rotation increment.
template <int FS>
__device__ __forceinline__ void bp_dy(const DevPlan &P, double &x, double &y, double &z, double &ux,
                                      double &uy, double &uz, double step, float kt, Cand *cc) {
    double hh = 0.5 * step;
    x = fma(ux, hh, x); y = fma(uy, hh, y); z = fma(uz, hh, z);
    f3 B = field_at<FS>(P, x, y, z, cc);
    bp_rotate_drift(x, y, z, ux, uy, uz, B, kt, hh);
}

template <int FS, int MODE = 0>
struct BP {
    static constexpr bool kReadsStepCount = false;
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        c.px = c.x; c.py = c.y; c.pz = c.z;
        double q = c.q, step = m.max_step;
        if (q == 0) {
            step = clipd(c.next, m.min_step, m.max_step);
            c.x = fma(c.dx, step, c.x); c.y = fma(c.dy, step, c.y); c.z = fma(c.dz, step, c.z);
            set_current_step(c, step);
            c.next = m.max_step;
            return;
        }
        double newStep = step;
        // t = B * q / 2 / m * step / c with m = E/c^2  ->  B * (q c step / (2 E)),
        // formed in FP32 like the rotation it scales
        const float kq = __fdividef((float)(q * (0.5 * kCLight)), (float)c.E);
        double xo = c.x, yo = c.y, zo = c.z, uxo = c.dx, uyo = c.dy, uzo = c.dz;
        if (MODE == 1 || (MODE == 0 && m.min_step == m.max_step)) {
            bp_dy<FS>(P, xo, yo, zo, uxo, uyo, uzo, step, kq * (float)step, &c);
            sc.tries++; sc.evals++;
        } else {
            step = clipd(c.next, m.min_step, m.max_step);
            newStep = step;
            for (int guard = 0; guard < 4096; guard++) {
                double x1 = c.x, y1 = c.y, z1 = c.z, u1x = c.dx, u1y = c.dy, u1z = c.dz;
                double x2 = c.x, y2 = c.y, z2 = c.z, u2x = c.dx, u2y = c.dy, u2z = c.dz;
                const float kts = kq * (float)step;
                bp_dy<FS>(P, x1, y1, z1, u1x, u1y, u1z, step, kts, &c);
                bp_dy<FS>(P, x2, y2, z2, u2x, u2y, u2z, step / 2, 0.5f * kts, &c);
                bp_dy<FS>(P, x2, y2, z2, u2x, u2y, u2z, step / 2, 0.5f * kts, &c);
                sc.tries++; sc.evals += 3;
                double ex = x1 - x2, ey = y1 - y2, ez = z1 - z2;
                double S = sqrt(ex * ex + ey * ey + ez * ez) / (step * 0.75);
                xo = x1; yo = y1; zo = z1; uxo = u1x; uyo = u1y; uzo = u1z;
                double r = sqrt(3.0 * S * S) / m.tolerance;
                if (r > 1) {
                    if (step == m.min_step) break;
                    newStep = step * 0.95 * pow(r, -0.2);
                    newStep = dmax(newStep, 0.1 * step);
                    newStep = dmax(newStep, m.min_step);
                    step = newStep;
                } else {
                    if (step != m.max_step) {
                        newStep = step * 0.95 * pow(r, -0.2);
                        newStep = dmin(newStep, 5 * step);
                        newStep = dmin(newStep, m.max_step);
                    }
                    break;
                }
            }
        }
        renorm(uxo, uyo, uzo);
        c.x = xo; c.y = yo; c.z = zo;
        c.dx = uxo; c.dy = uyo; c.dz = uzo;
        set_current_step(c, step);
        c.next = newStep;
    }
};

// --------------------------------------------------------------- Cash-Karp
__constant__ float ck_af[36] = {
    0.f, 0.f, 0.f, 0.f, 0.f, 0.f,
    1.f / 5.f, 0.f, 0.f, 0.f, 0.f, 0.f,
    3.f / 40.f, 9.f / 40.f, 0.f, 0.f, 0.f, 0.f,
    3.f / 10.f, -9.f / 10.f, 6.f / 5.f, 0.f, 0.f, 0.f,
    -11.f / 54.f, 5.f / 2.f, -70.f / 27.f, 35.f / 27.f, 0.f, 0.f,
    1631.f / 55296.f, 175.f / 512.f, 575.f / 13824.f, 44275.f / 110592.f, 253.f / 4096.f, 0.f};
__constant__ float ck_bf[6] = {37.f / 378.f, 0.f, 250.f / 621.f, 125.f / 594.f, 0.f, 512.f / 1771.f};
__constant__ double ck_eb[6] = {37. / 378. - 2825. / 27648., 0. - 0., 250. / 621. - 18575. / 48384.,
                                125. / 594. - 13525. / 55296., 0. - 277. / 14336., 512. / 1771. - 1. / 4.};

// One Cash-Karp try in time h (PropagationCK::tryStep): stage derivatives in
// FP32, stage positions as FP64 base + FP32 offset, error sum in FP64.
// Returns the position / direction increments and the direction error norm.
template <int FS>
__device__ __forceinline__ double ck_try(const DevPlan &P, Cand &c, double h, float qc2E,
                                         double &ddx, double &ddy, double &ddz, double &dux,
                                         double &duy, double &duz) {
    // stage derivative kx_i = c * unit(u_i) (as a unit vector, the factor c
    // is applied to the sums), ku_i = (q c / E) (v_i x B_i)
    f3 kx[6], ku[6];
    const float hf = (float)h;
    const float hc = (float)(h * kCLight);  // h * c, metres per unit velocity
    const f3 u0 = f3mk((float)c.dx, (float)c.dy, (float)c.dz);
    double eux = 0, euy = 0, euz = 0;
    float sxx = 0.f, sxy = 0.f, sxz = 0.f, sux = 0.f, suy = 0.f, suz = 0.f;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        float ox = 0.f, oy = 0.f, oz = 0.f, vx = u0.x, vy = u0.y, vz = u0.z;
#pragma unroll
        for (int j = 0; j < i; j++) {
            float a = ck_af[i * 6 + j];
            ox = fmaf(kx[j].x, a, ox); oy = fmaf(kx[j].y, a, oy); oz = fmaf(kx[j].z, a, oz);
            vx = fmaf(ku[j].x, a * hf, vx); vy = fmaf(ku[j].y, a * hf, vy); vz = fmaf(ku[j].z, a * hf, vz);
        }
        float inv = rsqrtf(vx * vx + vy * vy + vz * vz);
        f3 vel = f3mk(vx * inv, vy * inv, vz * inv);  // unit velocity
        f3 B = field_at<FS>(P, c.x + (double)(ox * hc), c.y + (double)(oy * hc), c.z + (double)(oz * hc), &c);
        f3 d = cross(vel, B);
        kx[i] = vel;
        ku[i] = f3mk(d.x * qc2E, d.y * qc2E, d.z * qc2E);  // (q c / E) (c vel x B)
        float b = ck_bf[i];
        sxx = fmaf(kx[i].x, b, sxx); sxy = fmaf(kx[i].y, b, sxy); sxz = fmaf(kx[i].z, b, sxz);
        sux = fmaf(ku[i].x, b, sux); suy = fmaf(ku[i].y, b, suy); suz = fmaf(ku[i].z, b, suz);
        double e = ck_eb[i] * h;
        eux = fma((double)ku[i].x, e, eux); euy = fma((double)ku[i].y, e, euy); euz = fma((double)ku[i].z, e, euz);
    }
    ddx = (double)sxx * (h * kCLight); ddy = (double)sxy * (h * kCLight); ddz = (double)sxz * (h * kCLight);
    dux = (double)(sux * hf); duy = (double)(suy * hf); duz = (double)(suz * hf);
    return sqrt(eux * eux + euy * euy + euz * euz);
}

template <int FS, int MODE = 0>
struct CK {
    static constexpr bool kReadsStepCount = false;
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        c.px = c.x; c.py = c.y; c.pz = c.z;
        double step = m.max_step;
        if (c.q == 0) {
            step = clipd(c.next, m.min_step, m.max_step);
            c.x = fma(c.dx, step, c.x); c.y = fma(c.dy, step, c.y); c.z = fma(c.dz, step, c.z);
            set_current_step(c, step);
            c.next = m.max_step;
            return;
        }
        const float qc2E = __fdividef((float)(c.q * (kCLight * kCLight)), (float)c.E);
        double ddx, ddy, ddz, dux, duy, duz;
        double newStep = step;
        if (MODE == 1 || (MODE == 0 && m.min_step == m.max_step)) {
            ck_try<FS>(P, c, step * kInvCLight, qc2E, ddx, ddy, ddz, dux, duy, duz);
            sc.tries++; sc.evals += 6;
        } else {
            step = clipd(c.next, m.min_step, m.max_step);
            newStep = step;
            for (int guard = 0; guard < 4096; guard++) {
                double err = ck_try<FS>(P, c, step * kInvCLight, qc2E, ddx, ddy, ddz, dux, duy, duz);
                sc.tries++; sc.evals += 6;
                double r = err / m.tolerance;
                if (r > 1) {
                    if (step == m.min_step) break;
                    newStep = step * 0.95 * pow(r, -0.2);
                    newStep = dmax(newStep, 0.1 * step);
                    newStep = dmax(newStep, m.min_step);
                    step = newStep;
                } else {
                    if (step != m.max_step) {
                        newStep = step * 0.95 * pow(r, -0.2);
                        newStep = dmin(newStep, 5 * step);
                        newStep = dmin(newStep, m.max_step);
                    }
                    break;
                }
            }
        }
        c.x += ddx; c.y += ddy; c.z += ddz;
        double ux = c.dx + dux, uy = c.dy + duy, uz = c.dz + duz;
        double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
        c.dx = ux * inv; c.dy = uy * inv; c.dz = uz * inv;
        set_current_step(c, step);
        c.next = newStep;
    }
};

// ------------------------------------------------------------ DiffusionSDE
__device__ __forceinline__ double s_rand(Stream &s) { return (double)s.next_u32() * (1.0 / 4294967295.0); }
__device__ __forceinline__ double s_uniform(Stream &s, double a, double b) { return fma(b - a, s_rand(s), a); }
__device__ __forceinline__ double s_norm(Stream &s) {
    double dblexc = ((double)s.next_u32() + 0.5) * (1.0 / 4294967296.0);
    double r = sqrt(-2.0 * log(1.0 - dblexc));
    double phi = 2.0 * kPi * ((double)s.next_u32() * (1.0 / 4294967296.0));
    return r * cos(phi);
}

// Explicit multiply-adds: the coroutine below is inlined into two kernels,
// and contraction left to the compiler can differ between them.
__device__ __forceinline__ double ddot(double ax, double ay, double az, double bx, double by, double bz) {
    return fma(ax, bx, fma(ay, by, az * bz));
}
__device__ __forceinline__ double dcross_c(double a1, double b2, double a2, double b1) {
    return fma(a1, b2, -(a2 * b1));  // a1 b2 - a2 b1
}

// ------------------------------------------------------------ DiffusionSDE
// DiffusionSDE::process (DiffusionSDE.cpp:47) written as a coroutine that
// stops at every field evaluation: the step-size halving tries of the
// field-line trace (DiffusionSDE::tryStep, :233, Cash-Karp stages of the unit
// field direction in FP32, FP64 base position and error), the 2^n sub-steps,
// then the perpendicular and drift displacements (:120-200).  Every lane
// runs its own number of six-stage traces, so a warp that evaluated fields
// lane by lane would spend most of its time with one or a few lanes inside a
// plane-wave mode sum; mixed_sde_coop_kernel instead evaluates the field
// for all lanes waiting for one in a single converged pass, and a lane whose
// step is done starts its next chain iteration at once.  SDE<FS> (the
// persistent kernels) runs the same coroutine lane by lane, so both give
// the same bits.  Stage i's offset gets a_ij k_j as soon as k_j is known.
struct SdeCo {
    double h, sh, TStep, NStep, BStep;
    double propTime, allowedTime;
    unsigned long long stepNumber, j;
    unsigned counter;
    int phase;                 // 0: step-halving tries, 1: sub-steps
    int stage;                 // next stage of the current try
    double bx, by, bz;         // base position of the current try
    double t;                  // time of the current try
    float tc;
    f3 a1, a2, a3, a4, a5;     // offsets of stages 1..5 (units of tc)
    float sx, sy, sz;
    double ex, ey, ez;
    double ox, oy, oz;         // end point of the last finished try
    double qx, qy, qz;         // position the lane waits for a field at
};

__device__ __forceinline__ void sde_co_start_try(SdeCo &co, double x, double y, double z, double t) {
    co.bx = x; co.by = y; co.bz = z;
    co.t = t;
    co.tc = (float)(t * kCLight);
    co.stage = 0;
    co.a1 = co.a2 = co.a3 = co.a4 = co.a5 = f3mk(0.f, 0.f, 0.f);
    co.sx = co.sy = co.sz = 0.f;
    co.ex = co.ey = co.ez = 0.0;
    co.qx = x; co.qy = y; co.qz = z;
}

// DiffusionSDE::driftStep (DiffusionSDE.cpp:255): the advection drift over
// the step time h at the step's start position (zero without a field).
__device__ __forceinline__ void sde_lin_prop(const DevModule &m, double x, double y, double z, double t, double h,
                                             double &lx, double &ly, double &lz) {
    lx = ly = lz = 0.;
    if (m.n_adv) {
        const u3 v = advection_at(m.adv, m.n_adv, x, y, z, t);
        lx = v.x * h; ly = v.y * h; lz = v.z * h;
    }
}

// First part of SDE::process up to the first field evaluation.  Returns
// false when the step needs no field (neutral candidate): it is then done.
template <int FS>
__device__ __forceinline__ bool sde_co_begin(const DevPlan &P, const DevModule &m, Cand &c, SdeCo &co) {
    c.px = c.x; c.py = c.y; c.pz = c.z;
    const double h = clipd(c.next, m.min_step, m.max_step) * kInvCLight;
    if (c.q == 0) {
        double lx, ly, lz;
        sde_lin_prop(m, c.x, c.y, c.z, c.time, h, lx, ly, lz);
        c.x = fma(c.dx, h * kCLight, c.x + lx); c.y = fma(c.dy, h * kCLight, c.y + ly);
        c.z = fma(c.dz, h * kCLight, c.z + lz);
        set_current_step(c, h * kCLight);
        c.next = m.max_step;
        return false;
    }
    const double rig = c.E / c.q;
    const double D = m.scale * 6.1e24 * pow(fabs(rig) / 4.0e9, m.alpha);
    const double BT0 = sqrt(2 * D), BT4 = sqrt(2 * m.eps * D);
    Stream s{P.seed, c.index, c.steps, make_uint4(0, 0, 0, 0), 0};
    const double eta0 = s_norm(s), eta1 = s_norm(s), eta2 = s_norm(s);
    co.h = h;
    co.TStep = BT0 * eta0; co.NStep = BT4 * eta1; co.BStep = BT4 * eta2;
    co.sh = sqrt(h);
    co.propTime = co.TStep * co.sh * kInvCLight;
    co.counter = 0;
    co.phase = 0;
    sde_co_start_try(co, c.x, c.y, c.z, co.propTime);
    return true;
}

// Rest of SDE::process after the last field-line trace (o = its end point).
__device__ __forceinline__ void sde_co_finish(const DevPlan &P, const DevModule &m, Cand &c, const SdeCo &co) {
    const double h = co.h, sh = co.sh;
    double tx = co.ox - c.x, ty = co.oy - c.y, tz = co.oz - c.z;
    double tn = sqrt(ddot(tx, ty, tz, tx, ty, tz));
    tx /= tn; ty /= tn; tz /= tn;
    double lx, ly, lz;
    sde_lin_prop(m, c.x, c.y, c.z, c.time, h, lx, ly, lz);
    if (!(tn == tn) || tn == 0.0) {
        if (m.n_adv) {  // only the advection drift
            c.x += lx; c.y += ly; c.z += lz;
        } else {
            c.x = fma(c.dx, h * kCLight, c.x); c.y = fma(c.dy, h * kCLight, c.y); c.z = fma(c.dz, h * kCLight, c.z);
        }
        set_current_step(c, h * kCLight);
        c.next = clipd(5 * h * kCLight, m.min_step, m.max_step);
        return;
    }
    Stream s{P.seed, c.index, c.steps, make_uint4(0, 0, 0, 0), 0};
    s.seek(6);  // the three normals took words 0-5
    double nx = 0, ny = 0, nz = 0;
    for (int guard = 0; nx == 0 && ny == 0 && nz == 0 && guard < 3; guard++) {
        double zr = s_uniform(s, -1.0, 1.0), tr = s_uniform(s, -kPi, kPi);
        double rr = sqrt(fma(-zr, zr, 1.0)), sn, cs;
        sincos(tr, &sn, &cs);
        double rx = rr * cs, ry = rr * sn, rz = zr;
        nx = dcross_c(ty, rz, ry, tz); ny = dcross_c(tz, rx, rz, tx); nz = dcross_c(tx, ry, rx, ty);
    }
    double nn = sqrt(ddot(nx, ny, nz, nx, ny, nz));
    if (nn == 0.0) { c.active = false; c.flags |= CRP_FLAG_NAN; return; }
    nx /= nn; ny /= nn; nz /= nn;
    double bx = dcross_c(ty, nz, ny, tz), by = dcross_c(tz, nx, nz, tx), bz = dcross_c(tx, ny, nx, ty);
    double bn = sqrt(ddot(bx, by, bz, bx, by, bz));
    bx /= bn; by /= bn; bz /= bn;
    double POx = fma(fma(nx, co.NStep, bx * co.BStep), sh, co.ox + lx);
    double POy = fma(fma(ny, co.NStep, by * co.BStep), sh, co.oy + ly);
    double POz = fma(fma(nz, co.NStep, bz * co.BStep), sh, co.oz + lz);
    if (isnan(POx + POy + POz)) { c.active = false; c.flags |= CRP_FLAG_NAN; return; }
    s.cursor = 12;
    double theta = acos(s_uniform(s, 1, cos(kPi / 2.)));
    double zr = s_uniform(s, -1.0, 1.0), tr = s_uniform(s, -kPi, kPi);
    double rr = sqrt(fma(-zr, zr, 1.0)), sn, cs;
    sincos(tr, &sn, &cs);
    double rx = rr * cs, ry = rr * sn, rz = zr;
    double ax = dcross_c(ty, rz, ry, tz), ay = dcross_c(tz, rx, rz, tx), az = dcross_c(tx, ry, rx, ty);
    double an = sqrt(ddot(ax, ay, az, ax, ay, az));
    if (an != 0.) { ax /= an; ay /= an; az /= an; }
    double st, ct;
    sincos(theta, &st, &ct);
    double adt = ddot(ax, ay, az, tx, ty, tz);
    double cx_ = dcross_c(ay, tz, az, ty), cy_ = dcross_c(az, tx, ax, tz), cz_ = dcross_c(ax, ty, ay, tx);
    const double omc = 1 - ct;
    double dx = fma(tx, ct, fma(cx_, st, (ax * adt) * omc));
    double dy = fma(ty, ct, fma(cy_, st, (ay * adt) * omc));
    double dz = fma(tz, ct, fma(cz_, st, (az * adt) * omc));
    double dn = 1.0 / sqrt(ddot(dx, dy, dz, dx, dy, dz));
    c.x = POx; c.y = POy; c.z = POz;
    c.dx = dx * dn; c.dy = dy * dn; c.dz = dz * dn;
    set_current_step(c, h * kCLight);
    c.next = (co.stepNumber > 1) ? h / ((double)co.stepNumber * (double)co.stepNumber) * kCLight
                                 : 4 * h * kCLight;
}

// Take the field at co.q for the current stage.  Returns true while the
// step waits for another field (co.q set), false when the step is done.
__device__ __forceinline__ bool sde_co_consume(const DevPlan &P, const DevModule &m, Cand &c, SdeCo &co,
                                               f3 B, StepCount &sc) {
    const int jst = co.stage;
    const float inv = rsqrtf(dot(B, B));
    const f3 k = f3mk(B.x * inv, B.y * inv, B.z * inv);
    const float b = ck_bf[jst];
    co.sx = fmaf(k.x, b, co.sx); co.sy = fmaf(k.y, b, co.sy); co.sz = fmaf(k.z, b, co.sz);
    const double e = ck_eb[jst];
    co.ex = fma((double)k.x, e, co.ex); co.ey = fma((double)k.y, e, co.ey); co.ez = fma((double)k.z, e, co.ez);
    // stage i's offset gets a_ij k_j for every later stage i
    auto add = [&](f3 &acc, int i) {
        const float a = ck_af[i * 6 + jst];
        acc.x = fmaf(k.x, a, acc.x); acc.y = fmaf(k.y, a, acc.y); acc.z = fmaf(k.z, a, acc.z);
    };
    if (jst < 1) add(co.a1, 1);
    if (jst < 2) add(co.a2, 2);
    if (jst < 3) add(co.a3, 3);
    if (jst < 4) add(co.a4, 4);
    if (jst < 5) add(co.a5, 5);
    co.stage = jst + 1;
    if (co.stage < 6) {
        const int st = co.stage;
        const f3 a = st == 1 ? co.a1 : st == 2 ? co.a2 : st == 3 ? co.a3 : st == 4 ? co.a4 : co.a5;
        co.qx = co.bx + (double)(a.x * co.tc);
        co.qy = co.by + (double)(a.y * co.tc);
        co.qz = co.bz + (double)(a.z * co.tc);
        return true;
    }
    // the try is complete: end point and error of the trace
    sc.tries++;
    sc.evals += 6;
    const double tcd = co.t * kCLight;
    co.ox = fma((double)co.sx, tcd, co.bx); co.oy = fma((double)co.sy, tcd, co.by); co.oz = fma((double)co.sz, tcd, co.bz);
    const double err = sqrt(ddot(co.ex, co.ey, co.ez, co.ex, co.ey, co.ez)) * fabs(tcd) / CRP_KPC;
    if (co.phase == 0) {
        const double r = err / m.tolerance;
        co.propTime *= 0.5;
        co.counter += 1;
        if (r > 1 && fabs(co.propTime) >= m.min_step * kInvCLight && co.counter < 60) {
            sde_co_start_try(co, c.x, c.y, c.z, co.propTime);
            return true;
        }
        co.stepNumber = 1ull << (co.counter - 1);
        co.allowedTime = co.TStep * co.sh * kInvCLight / (double)co.stepNumber;
        co.phase = 1;
        co.j = 0;
        sde_co_start_try(co, c.x, c.y, c.z, co.allowedTime);
        return true;
    }
    co.j++;
    if (co.j < co.stepNumber) {
        sde_co_start_try(co, co.ox, co.oy, co.oz, co.allowedTime);
        return true;
    }
    sde_co_finish(P, m, c, co);
    return false;
}

// DiffusionSDE::process (DiffusionSDE.cpp:47) for one lane: the coroutine
// run to completion, field evaluations in place.
template <int FS>
struct SDE {
    static constexpr bool kReadsStepCount = true;  // the Philox counter
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        SdeCo co;
        if (!sde_co_begin<FS>(P, m, c, co)) return;
        while (sde_co_consume(P, m, c, co, field_at<FS>(P, co.qx, co.qy, co.qz, &c), sc)) {
        }
    }
};


// The non-propagation modules mi in [from, to) of one chain iteration.
__device__ __forceinline__ void chain_part(const DevPlan &P, Cand &c, const DevRecords &rec, int from, int to) {
#pragma unroll 1
    for (int mi = from; mi < to; mi++) {
        const DevModule &m = P.modules[mi];
        if (m.kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH) max_trajectory_length(m, c, rec, mi);
        else if (m.kind == CRP_MODULE_OBSERVER) observer(P, m, c, rec, mi);
        else if (m.kind == CRP_MODULE_BOUNDARY) boundary(m, c, rec, mi);
    }
}

// step-mode variants selected by the launcher from min_step == max_step, so
// that a fixed-step kernel carries no adaptive-controller registers
template <int FS> using BPFixed = BP<FS, 1>;
// resident blocks of 128 threads per SM the register budget is sized for:
// the fixed-step Boris push is latency bound on its gathers and wants warps
template <class T> struct MinBlocks { static constexpr int value = 1; };
template <int FS, int MODE> struct MinBlocks<BP<FS, MODE>> { static constexpr int value = MODE == 1 ? CRP_BP_FIXED_MIN_BLOCKS : 1; };
template <int FS, int MODE> struct MinBlocks<CK<FS, MODE>> { static constexpr int value = CRP_CK_MIN_BLOCKS; };
template <int FS> using BPAdaptive = BP<FS, 2>;
template <int FS> using CKFixed = CK<FS, 1>;
template <int FS> using CKAdaptive = CK<FS, 2>;

template <template <int> class Prop, int FS, int CS>
__global__ void __launch_bounds__(128, MinBlocks<Prop<FS>>::value) mixed_chunk_kernel(const __grid_constant__ DevPlan P, DevState s, uint64_t n,
                                                          int max_steps, uint64_t step_cap,
                                                          DevCounters *cnt, DevRecords rec,
                                                          const uint32_t *perm, uint32_t *perm_out) {
    chunk_body<Prop<FS>, CS>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out);
}

template <template <int> class Prop>
cudaError_t launch_prop(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                        uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                        const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                        cudaStream_t st) {
    unsigned grid = (unsigned)((n + block - 1) / block);
#define CRP_CHUNK(FSV, CSV) mixed_chunk_kernel<Prop, FSV, CSV><<<grid, block, 0, st>>>(P, s, n, max_steps, \
        step_cap, cnt, rec, perm, perm_out)
    // compiled chain shapes for the single-field signatures; the generic
    // field sum walks the module list
    if (fs == FS_GRID_PERIODIC) {
        if (P.shape == CS_PM) CRP_CHUNK(FS_GRID_PERIODIC, CS_PM);
        else if (P.shape == CS_PMO) CRP_CHUNK(FS_GRID_PERIODIC, CS_PMO);
        else CRP_CHUNK(FS_GRID_PERIODIC, CS_GENERIC);
    } else if (fs == FS_GRID) {
        CRP_CHUNK(FS_GRID, CS_GENERIC);
    } else if (fs == FS_PLANE_WAVE) {
        if (P.shape == CS_PM) CRP_CHUNK(FS_PLANE_WAVE, CS_PM);
        else if (P.shape == CS_PMO) CRP_CHUNK(FS_PLANE_WAVE, CS_PMO);
        else CRP_CHUNK(FS_PLANE_WAVE, CS_GENERIC);
    } else {
        CRP_CHUNK(FS_GENERIC, CS_GENERIC);
    }
#undef CRP_CHUNK
    return cudaGetLastError();
}

}  // namespace
}  // namespace crp
