// step_fp64.cu -- the FP64 form of the stepping path.
//
// Operation for operation the reference's arithmetic, in the reference's
// order: PropagationBP::dY (PropagationBP.cpp:19), PropagationCK::tryStep /
// dYdt (PropagationCK.cpp:28, :51), DiffusionSDE::process / tryStep
// (DiffusionSDE.cpp:47, :233), Grid<Vector3f>::trilinearInterpolate in float
// (Grid.h:540), PeriodicMagneticField (MagneticField.cpp:41) and the scalar
// PlaneWaveTurbulence sum (PlaneWaveTurbulence.cpp:233).  This translation
// unit is compiled with -fmad=false so that no multiply-add is contracted:
// where the reference uses only + - * / sqrt floor (the Boris push over a
// Grid3f) the device result is bit-identical to the reference built without
// FMA.  pow in the step controllers and DiffusionSDE is cr_pow (crmath.cuh),
// correctly rounded, which agrees with glibc's pow except where glibc itself
// misrounds (about 1e-3 of inputs); cos in the wave sum and log/cos in the
// normal draws are CUDA's, within a few ulp of glibc's.
#include <type_traits>

#include "chain.cuh"
#include "crmath.cuh"
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

struct d3 { double x, y, z; };
__device__ __forceinline__ d3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ d3 add(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 muls(d3 a, double f) { return {a.x * f, a.y * f, a.z * f}; }
__device__ __forceinline__ d3 divs(d3 a, double f) { return {a.x / f, a.y / f, a.z / f}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 v) {
    return {a.y * v.z - v.y * a.z, a.z * v.x - v.z * a.x, a.x * v.y - v.x * a.y};
}
__device__ __forceinline__ double norm(d3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ d3 unit(d3 a) { return divs(a, norm(a)); }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double clipd(double x, double lo, double hi) { return dmax(lo, dmin(x, hi)); }

// Grid<Vector3f>::interpolate (Grid.h:318) -> trilinearInterpolate (:540).
// With a cell cache (FS_GRID kernels) the 8 corners are loaded only when the
// cell changes.
// PER: the grid is periodic with power-of-two dimensions and has no
// clipVolume (FS_GRID_PERIODIC): those branches are compiled out and the
// periodic clamp is a mask (equal to the double modulo of Grid.h:31 there).
template <bool CACHE, bool PER = false>
__device__ __forceinline__ d3 grid_field_t(const DevGrid &g, d3 pos, Cand *cc) {
    if (!PER && g.interp != CRP_INTERPOLATION_TRILINEAR) {  // tricubic, nearest (Grid.h:328-331)
        const gi3 v = gi_vector_other(g, pos.x, pos.y, pos.z);
        return mk(v.x, v.y, v.z);
    }
    if (!PER && g.clip_volume) {
        bool in = (pos.x >= g.ox) && (pos.x <= g.ex);
        in &= (pos.y >= g.oy) && (pos.y <= g.ey);
        in &= (pos.z >= g.oz) && (pos.z <= g.ez);
        if (!in) return mk(0, 0, 0);
    }
    double rx = (pos.x - g.gox) / g.sx;
    double ry = (pos.y - g.goy) / g.sy;
    double rz = (pos.z - g.goz) / g.sz;
    int ix0, ix1, iy0, iy1, iz0, iz1;
    double fX0, fY0, fZ0;
    if (!PER && g.reflective) {  // reflectiveClamp (Grid.h:49)
        double r[3] = {rx, ry, rz}, res[3];
        int n[3] = {g.nx, g.ny, g.nz}, lo[3], hi[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            double x = r[a];
            int guard = 0;
            while (((x < -0.5) || (x > (n[a] - 0.5))) && guard < 64) {
                x = 2 * n[a] * (x > (n[a] - 0.5)) - x - 1;
                guard++;
            }
            res[a] = x;
            lo[a] = (int)floor(x);
            hi[a] = lo[a] + (lo[a] < n[a] - 1);
            if (x < 0) { lo[a] = 0; hi[a] = 0; }
            // positions beyond 64 reflections are outside any physical use
            if (lo[a] < 0 || lo[a] >= n[a]) { lo[a] = 0; hi[a] = 0; }
        }
        ix0 = lo[0]; ix1 = hi[0]; iy0 = lo[1]; iy1 = hi[1]; iz0 = lo[2]; iz1 = hi[2];
        fX0 = res[0] - floor(res[0]);
        fY0 = res[1] - floor(res[1]);
        fZ0 = res[2] - floor(res[2]);
    } else if (PER) {  // periodicClamp (Grid.h:31), power-of-two dimensions
        ix0 = (int)floor(rx) & (g.nx - 1); ix1 = (ix0 + 1) & (g.nx - 1);
        iy0 = (int)floor(ry) & (g.ny - 1); iy1 = (iy0 + 1) & (g.ny - 1);
        iz0 = (int)floor(rz) & (g.nz - 1); iz1 = (iz0 + 1) & (g.nz - 1);
        fX0 = rx - floor(rx);
        fY0 = ry - floor(ry);
        fZ0 = rz - floor(rz);
    } else {  // periodicClamp (Grid.h:31)
        ix0 = (((int)floor(rx) % g.nx) + g.nx) % g.nx; ix1 = (ix0 + 1) % g.nx;
        iy0 = (((int)floor(ry) % g.ny) + g.ny) % g.ny; iy1 = (iy0 + 1) % g.ny;
        iz0 = (((int)floor(rz) % g.nz) + g.nz) % g.nz; iz1 = (iz0 + 1) % g.nz;
        fX0 = rx - floor(rx);
        fY0 = ry - floor(ry);
        fZ0 = rz - floor(rz);
    }
    const float fx1 = (float)(1 - fX0), fy1 = (float)(1 - fY0), fz1 = (float)(1 - fZ0);
    const float fx0 = (float)fX0, fy0 = (float)fY0, fz0 = (float)fZ0;
    // cell indices: 32-bit for FS_GRID_PERIODIC grids (fewer than 2^31 cells)
    using Index = typename std::conditional<PER, unsigned, size_t>::type;
    const Index sy = (Index)g.nz, sx = (Index)g.ny * (Index)g.nz;
    const float *v = g.values;
    const Index b00 = (Index)ix0 * sx + (Index)iy0 * sy, b10 = (Index)ix1 * sx + (Index)iy0 * sy;
    const Index b01 = (Index)ix0 * sx + (Index)iy1 * sy, b11 = (Index)ix1 * sx + (Index)iy1 * sy;
    // the corner order of Grid.h:571-578
    const float *p0 = v + 3 * (size_t)(b00 + iz0), *p1 = v + 3 * (size_t)(b10 + iz0),
                *p2 = v + 3 * (size_t)(b01 + iz0), *p3 = v + 3 * (size_t)(b00 + iz1),
                *p4 = v + 3 * (size_t)(b10 + iz1), *p5 = v + 3 * (size_t)(b01 + iz1),
                *p6 = v + 3 * (size_t)(b11 + iz0), *p7 = v + 3 * (size_t)(b11 + iz1);
    float lc[8][3];
    float (*c)[3] = CACHE ? cc->corner : lc;
    const long long k0 = (long long)(b00 + iz0), k7 = (long long)(b11 + iz1);
    if (!CACHE || k0 != cc->cell0 || k7 != cc->cell7) {
#define LD3(k, p) c[k][0] = __ldg(p); c[k][1] = __ldg(p + 1); c[k][2] = __ldg(p + 2);
        LD3(0, p0) LD3(1, p1) LD3(2, p2) LD3(3, p3) LD3(4, p4) LD3(5, p5) LD3(6, p6) LD3(7, p7)
#undef LD3
        if (CACHE) { cc->cell0 = k0; cc->cell7 = k7; }
    }
    const float wx[8] = {fx1, fx0, fx1, fx1, fx0, fx1, fx0, fx0};
    const float wy[8] = {fy1, fy1, fy0, fy1, fy1, fy0, fy0, fy0};
    const float wz[8] = {fz1, fz1, fz1, fz0, fz0, fz0, fz1, fz0};
    float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        bx += c[k][0] * wx[k] * wy[k] * wz[k];
        by += c[k][1] * wx[k] * wy[k] * wz[k];
        bz += c[k][2] * wx[k] * wy[k] * wz[k];
    }
    return mk(bx, by, bz);
}

__device__ d3 grid_field(const DevGrid &g, d3 pos) { return grid_field_t<false>(g, pos, nullptr); }

// PlaneWaveTurbulence::getField, scalar branch (PlaneWaveTurbulence.cpp:233).
__device__ d3 plane_wave_field(const DevPlaneWave &w, d3 pos) {
    d3 B = mk(0, 0, 0);
    const double *m = w.modes;
#pragma unroll 1
    for (int i = 0; i < w.n; i++, m += 9) {
        d3 xi = mk(__ldg(m), __ldg(m + 1), __ldg(m + 2));
        d3 kap = mk(__ldg(m + 3), __ldg(m + 4), __ldg(m + 5));
        double k = __ldg(m + 6), beta = __ldg(m + 7), ak = __ldg(m + 8);
        double z_ = dot(pos, kap);
        B = add(B, muls(muls(xi, ak), cos(k * z_ + beta)));
    }
    return B;
}

// ---------------------------------------------------------------- JF12Field
// The reference's arithmetic operation for operation (JF12Field.cpp:195-346);
// the regular field (JF12Field, PlanckJF12bField and JF12FieldSolenoidal) is
// in jf12.cuh.

__device__ __forceinline__ d3 jf12_regular(const crp_jf12_desc &J, d3 pos) {
    const u3 b = jf12_regular_fp64(J, pos.x, pos.y, pos.z);
    return mk(b.x, b.y, b.z);
}

// JF12Field::getTurbulentStrength (JF12Field.cpp:301)
__device__ double jf12_turbulent_strength(const crp_jf12_desc &J, d3 pos) {
    const double kpc = J.kpc;
    if (sqrt(pos.x * pos.x + pos.y * pos.y + pos.z * pos.z) > 20 * kpc) return 0;
    const double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    const double phi = jf_phi(pos.x, pos.y);
    double bDisk = 0;
    if (r < 5 * kpc) {
        bDisk = J.b_disk_turb5;
    } else {
        const double r_negx = jf_r_negx(J, r, phi);
        for (int i = 7; i >= 0; i--)
            if (r_negx < J.r_arms[i]) bDisk = J.b_disk_turb[i];
        bDisk *= (5 * kpc) / r;
    }
    bDisk *= exp(-0.5 * jf_sq(pos.z / J.z_disk_turb));
    const double bHalo = J.b_halo_turb * exp(-r / J.r_halo_turb) * exp(-0.5 * jf_sq(pos.z / J.z_halo_turb));
    return sqrt(jf_sq(bDisk) + jf_sq(bHalo));
}

// JF12Field::getField (JF12Field.cpp:346): turbulent + (striated or regular).
// Not inlined: the generic-field kernels keep their register budget.
__device__ __noinline__ d3 jf12_field(const DevComponent &f, d3 pos) {
    const crp_jf12_desc &J = f.jf->d;
    d3 b = mk(0., 0., 0.);
    if (J.use_turbulent) {
        // Vector3f * double: the strength is rounded to float, the product is float
        const d3 g = grid_field(f.grid, pos);
        const float s = (float)jf12_turbulent_strength(J, pos);
        b = add(b, mk((double)__fmul_rn((float)g.x, s), (double)__fmul_rn((float)g.y, s),
                      (double)__fmul_rn((float)g.z, s)));
    }
    if (J.use_striated) {  // JF12Field.cpp:296, closestValue of the striated Grid1f
        const double v = (double)__ldg(f.mod.values + gi_nearest_cell(f.mod, pos.x, pos.y, pos.z));
        b = add(b, muls(jf12_regular(J, pos), 1. + J.sqrt_beta * v));
    } else if (J.use_regular) {
        b = add(b, jf12_regular(J, pos));
    }
    return b;
}

__device__ d3 component_field(const DevComponent &f, d3 position) {
    d3 pos = position;
    if (f.periodic) {  // PeriodicMagneticField::getField (MagneticField.cpp:41)
        d3 o = mk(f.po[0], f.po[1], f.po[2]), e = mk(f.pe[0], f.pe[1], f.pe[2]);
        d3 q = sub(position, o);
        d3 n = mk(floor(q.x / e.x), floor(q.y / e.y), floor(q.z / e.z));
        d3 p = sub(q, mk(n.x * e.x, n.y * e.y, n.z * e.z));
        if (f.periodic_reflective) {
            if ((long long)fabs(n.x) % 2 == 1) p.x = e.x - p.x;
            if ((long long)fabs(n.y) % 2 == 1) p.y = e.y - p.y;
            if ((long long)fabs(n.z) % 2 == 1) p.z = e.z - p.z;
        }
        pos = p;
    }
    switch (f.kind) {
    case CRP_FIELD_GRID: return grid_field(f.grid, pos);
    case CRP_FIELD_MODULATED_GRID: {  // ModulatedMagneticFieldGrid::getField (MagneticFieldGrid.cpp:51)
        const float m = gi_scalar(f.mod, pos.x, pos.y, pos.z);
        return muls(grid_field(f.grid, pos), (double)m);
    }
    case CRP_FIELD_PLANE_WAVE: return plane_wave_field(f.pw, pos);
    case CRP_FIELD_UNIFORM: return mk(f.uniform[0], f.uniform[1], f.uniform[2]);
    case CRP_FIELD_JF12: return jf12_field(f, pos);
    case CRP_FIELD_UF23: {
        const u3 b = uf23_field(*f.uf, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_PT11: {
        const u3 b = pt11_field(*f.pt, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_ARCHIMEDEAN_SPIRAL: {
        const u3 b = archimedean_field(f.arch, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_TF17: {
        const u3 b = tf17_field(*f.tf, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_SINGLE_MODE: {
        const u3 b = single_mode_field(f.mode, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_KST24: {
        const u3 b = kst24_field(*f.kst, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    case CRP_FIELD_CMZ: {
        const u3 b = cmz_field(*f.cmz, pos.x, pos.y, pos.z);
        return mk(b.x, b.y, b.z);
    }
    default: {
        double r = sqrt(pos.x * pos.x + pos.y * pos.y);
        return muls(mk(-pos.y, pos.x, 0.), f.b0 / r);
    }
    }
}

// MagneticFieldList::getField (MagneticField.cpp:64) or the single field.
template <int FS>
__device__ __forceinline__ d3 field_at(const DevPlan &P, d3 pos, Cand *cc = nullptr) {
    if (FS == FS_GRID) return grid_field_t<true>(P.fields[0].grid, pos, cc);
    if (FS == FS_GRID_PERIODIC) return grid_field_t<true, true>(P.fields[0].grid, pos, cc);
    if (FS == FS_PLANE_WAVE) return plane_wave_field(P.fields[0].pw, pos);
    if (P.n_fields == 1) return component_field(P.fields[0], pos);
    d3 b = mk(0, 0, 0);
#pragma unroll 1
    for (int i = 0; i < P.n_fields; i++) b = add(b, component_field(P.fields[i], pos));
    return b;
}

__device__ __forceinline__ void set_current_step(Cand &c, double s) {  // Candidate.cpp:92
    c.cur = s;
    c.len += s;
    c.time += s / kCLight;
}

// ---------------------------------------------------------------- Boris push
template <int FS>
__device__ __forceinline__ void bp_dy(const DevPlan &P, d3 &x, d3 &u, double step, double q,
                                      double m, Cand *cc) {
    x = add(x, divs(muls(u, step), 2.));
    d3 B = field_at<FS>(P, x, cc);
    d3 t = divs(muls(divs(divs(muls(B, q), 2), m), step), kCLight);
    d3 s = divs(muls(t, 2), (1 + dot(t, t)));
    d3 vh = add(u, cross(u, t));
    u = add(u, cross(vh, s));
    x = add(x, divs(muls(u, step), 2.));
}

template <int FS, int MODE = 0>
struct BP {
    static constexpr bool kReadsStepCount = false;
    // PropagationBP::process (PropagationBP.cpp:62)
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        c.px = c.x; c.py = c.y; c.pz = c.z;
        double q = c.q, step = m.max_step;
        if (q == 0) {
            step = clipd(c.next, m.min_step, m.max_step);
            c.x = c.x + c.dx * step; c.y = c.y + c.dy * step; c.z = c.z + c.dz * step;
            set_current_step(c, step);
            c.next = m.max_step;
            return;
        }
        double newStep = step;
        double mass = c.E / (kCLight * kCLight);
        d3 xo = mk(c.x, c.y, c.z), uo = mk(c.dx, c.dy, c.dz);
        if (MODE == 1 || (MODE == 0 && m.min_step == m.max_step)) {
            bp_dy<FS>(P, xo, uo, step, q, mass, &c);
            sc.tries++; sc.evals++;
        } else {
            step = clipd(c.next, m.min_step, m.max_step);
            newStep = step;
            for (int guard = 0; guard < 4096; guard++) {
                d3 x1 = mk(c.x, c.y, c.z), u1 = mk(c.dx, c.dy, c.dz), xh = x1, uh = u1;
                bp_dy<FS>(P, x1, u1, step, q, mass, &c);
                bp_dy<FS>(P, xh, uh, step / 2, q, mass, &c);
                bp_dy<FS>(P, xh, uh, step / 2, q, mass, &c);
                sc.tries++; sc.evals += 3;
                double S = norm(sub(x1, xh)) / (step * (1 - 1 / 4.));
                xo = x1; uo = u1;
                double r = norm(mk(S, S, S)) / m.tolerance;
                if (r > 1) {
                    if (step == m.min_step) break;
                    newStep = step * 0.95 * cr_pow(r, -0.2);
                    newStep = dmax(newStep, 0.1 * step);
                    newStep = dmax(newStep, m.min_step);
                    step = newStep;
                } else {
                    if (step != m.max_step) {
                        newStep = step * 0.95 * cr_pow(r, -0.2);
                        newStep = dmin(newStep, 5 * step);
                        newStep = dmin(newStep, m.max_step);
                    }
                    break;
                }
            }
        }
        c.x = xo.x; c.y = xo.y; c.z = xo.z;
        d3 u = unit(uo);
        u = divs(u, norm(u));  // ParticleState::setDirection normalises again
        c.dx = u.x; c.dy = u.y; c.dz = u.z;
        set_current_step(c, step);
        c.next = newStep;
    }
};

// --------------------------------------------------------------- Cash-Karp
__constant__ double ck_a[36] = {
    0., 0., 0., 0., 0., 0.,
    1. / 5., 0., 0., 0., 0., 0.,
    3. / 40., 9. / 40., 0., 0., 0., 0.,
    3. / 10., -9. / 10., 6. / 5., 0., 0., 0.,
    -11. / 54., 5. / 2., -70. / 27., 35. / 27., 0., 0.,
    1631. / 55296., 175. / 512., 575. / 13824., 44275. / 110592., 253. / 4096., 0.};
__constant__ double ck_b[6] = {37. / 378., 0, 250. / 621., 125. / 594., 0., 512. / 1771.};
__constant__ double ck_bs[6] = {2825. / 27648., 0., 18575. / 48384., 13525. / 55296.,
                                277. / 14336., 1. / 4.};

template <int FS>
__device__ __forceinline__ void ck_try(const DevPlan &P, d3 x, d3 u, double h, double q, double E,
                                       d3 &xo, d3 &uo, d3 &eu, Cand *cc) {
    d3 kx[6], ku[6];
    xo = x; uo = u;
    eu = mk(0, 0, 0);
#pragma unroll
    for (int i = 0; i < 6; i++) {
        d3 yx = x, yu = u;
#pragma unroll
        for (int j = 0; j < i; j++) {
            yx = add(yx, muls(muls(kx[j], ck_a[i * 6 + j]), h));
            yu = add(yu, muls(muls(ku[j], ck_a[i * 6 + j]), h));
        }
        d3 vel = muls(unit(yu), kCLight);
        d3 B = field_at<FS>(P, yx, cc);
        d3 dudt = muls(cross(vel, B), q * kCLight / E);
        kx[i] = vel; ku[i] = dudt;
        xo = add(xo, muls(muls(kx[i], ck_b[i]), h));
        uo = add(uo, muls(muls(ku[i], ck_b[i]), h));
        eu = add(eu, muls(muls(ku[i], ck_b[i] - ck_bs[i]), h));
    }
}

template <int FS, int MODE = 0>
struct CK {
    static constexpr bool kReadsStepCount = false;
    // PropagationCK::process (PropagationCK.cpp:77)
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        c.px = c.x; c.py = c.y; c.pz = c.z;
        double step = m.max_step;
        if (c.q == 0) {
            step = clipd(c.next, m.min_step, m.max_step);
            c.x = c.x + c.dx * step; c.y = c.y + c.dy * step; c.z = c.z + c.dz * step;
            set_current_step(c, step);
            c.next = m.max_step;
            return;
        }
        d3 xo, uo, eu;
        d3 x = mk(c.x, c.y, c.z), u = mk(c.dx, c.dy, c.dz);
        double newStep = step;
        if (MODE == 1 || (MODE == 0 && m.min_step == m.max_step)) {
            ck_try<FS>(P, x, u, step / kCLight, c.q, c.E, xo, uo, eu, &c);
            sc.tries++; sc.evals += 6;
        } else {
            step = clipd(c.next, m.min_step, m.max_step);
            newStep = step;
            for (int guard = 0; guard < 4096; guard++) {
                ck_try<FS>(P, x, u, step / kCLight, c.q, c.E, xo, uo, eu, &c);
                sc.tries++; sc.evals += 6;
                double r = norm(eu) / m.tolerance;
                if (r > 1) {
                    if (step == m.min_step) break;
                    newStep = step * 0.95 * cr_pow(r, -0.2);
                    newStep = dmax(newStep, 0.1 * step);
                    newStep = dmax(newStep, m.min_step);
                    step = newStep;
                } else {
                    if (step != m.max_step) {
                        newStep = step * 0.95 * cr_pow(r, -0.2);
                        newStep = dmin(newStep, 5 * step);
                        newStep = dmin(newStep, m.max_step);
                    }
                    break;
                }
            }
        }
        c.x = xo.x; c.y = xo.y; c.z = xo.z;
        d3 un = unit(uo);
        un = divs(un, norm(un));
        c.dx = un.x; c.dy = un.y; c.dz = un.z;
        set_current_step(c, step);
        c.next = newStep;
    }
};

// ------------------------------------------------------------ DiffusionSDE
__device__ __forceinline__ double s_rand(Stream &s) { return (double)s.next_u32() * (1.0 / 4294967295.0); }
__device__ __forceinline__ double s_uniform(Stream &s, double a, double b) { return a + (b - a) * s_rand(s); }
__device__ __forceinline__ double s_norm(Stream &s) {  // Random::randNorm (Random.cpp:104)
    double dblexc = ((double)s.next_u32() + 0.5) * (1.0 / 4294967296.0);
    double r = sqrt(-2.0 * log(1.0 - dblexc)) * 1.0;
    double phi = 2.0 * 3.14159265358979323846264338328 * ((double)s.next_u32() * (1.0 / 4294967296.0));
    return 0.0 + r * cos(phi);
}
__device__ __forceinline__ d3 s_vector(Stream &s) {  // Random::randVector (Random.cpp:141)
    double z = s_uniform(s, -1.0, 1.0);
    double t = s_uniform(s, -1.0 * kPi, kPi);
    double r = sqrt(1 - z * z);
    return mk(r * cos(t), r * sin(t), z);
}
__device__ __forceinline__ d3 rotated(d3 v, d3 axis, double angle) {  // Vector3.h:206
    d3 u = axis;
    if (norm(u) != 0.) u = divs(u, norm(u));
    double c = cos(angle), s = sin(angle);
    d3 Rx = mk(c + u.x * u.x * (1 - c), u.x * u.y * (1 - c) - u.z * s, u.x * u.z * (1 - c) + u.y * s);
    d3 Ry = mk(u.y * u.x * (1 - c) + u.z * s, c + u.y * u.y * (1 - c), u.y * u.z * (1 - c) - u.x * s);
    d3 Rz = mk(u.z * u.x * (1 - c) - u.y * s, u.z * u.y * (1 - c) + u.x * s, c + u.z * u.z * (1 - c));
    return mk(dot(v, Rx), dot(v, Ry), dot(v, Rz));
}

template <int FS>
__device__ __forceinline__ void sde_try(const DevPlan &P, d3 PosIn, d3 &POut, d3 &PosErr,
                                        double propStep, Cand *cc) {
    d3 k[6];
    POut = PosIn;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        d3 y_n = PosIn;
#pragma unroll
        for (int j = 0; j < i; j++) y_n = add(y_n, muls(muls(k[j], ck_a[i * 6 + j]), propStep));
        d3 B = field_at<FS>(P, y_n, cc);
        k[i] = muls(unit(B), kCLight);
        POut = add(POut, muls(muls(k[i], ck_b[i]), propStep));
        PosErr = add(PosErr, divs(muls(muls(k[i], ck_b[i] - ck_bs[i]), propStep), CRP_KPC));
    }
}

template <int FS>
struct SDE {
    static constexpr bool kReadsStepCount = true;  // the Philox counter
    // DiffusionSDE::process (DiffusionSDE.cpp:47); the advection drift of
    // driftStep (:255) is LinProp = 0 + v_adv(PosIn) h.
    __device__ static d3 lin_prop(const DevModule &m, d3 pos, double h, double t) {
        if (m.n_adv == 0) return mk(0, 0, 0);
        const u3 v = advection_at(m.adv, m.n_adv, pos.x, pos.y, pos.z, t);
        return add(mk(0, 0, 0), muls(mk(v.x, v.y, v.z), h));
    }
    __device__ static void process(const DevPlan &P, const DevModule &m, Cand &c, StepCount &sc) {
        c.px = c.x; c.py = c.y; c.pz = c.z;
        double h = clipd(c.next, m.min_step, m.max_step) / kCLight;
        d3 PosIn = mk(c.x, c.y, c.z);
        if (c.q == 0) {
            d3 p = add(add(PosIn, lin_prop(m, PosIn, h, c.time)), muls(muls(mk(c.dx, c.dy, c.dz), h), kCLight));
            c.x = p.x; c.y = p.y; c.z = p.z;
            set_current_step(c, h * kCLight);
            c.next = m.max_step;
            return;
        }
        double rig = c.E / c.q;
        double DifCoeff = m.scale * 6.1e24 * cr_pow((fabs(rig) / 4.0e9), m.alpha);
        double BT0 = cr_pow(2 * DifCoeff, 0.5);
        double BT4 = cr_pow(2 * m.eps * DifCoeff, 0.5);
        Stream s{P.seed, c.index, c.steps, make_uint4(0, 0, 0, 0), 0};
        double eta0 = s_norm(s), eta1 = s_norm(s), eta2 = s_norm(s);
        double TStep = BT0 * eta0, NStep = BT4 * eta1, BStep = BT4 * eta2;
        double propTime = TStep * sqrt(h) / kCLight;
        unsigned counter = 0;
        double r = 42.;
        do {
            d3 PosOut = mk(0, 0, 0), PosErr = mk(0, 0, 0);
            sde_try<FS>(P, PosIn, PosOut, PosErr, propTime, &c);
            sc.tries++; sc.evals += 6;
            r = norm(PosErr) / m.tolerance;
            propTime *= 0.5;
            counter += 1;
        } while (r > 1 && fabs(propTime) >= m.min_step / kCLight && counter < 60);
        unsigned long long stepNumber = (unsigned long long)pow(2.0, (double)(counter - 1));
        double allowedTime = TStep * sqrt(h) / kCLight / (double)stepNumber;
        d3 Start = PosIn, PosOut = mk(0, 0, 0), PosErr = mk(0, 0, 0);
        for (unsigned long long j = 0; j < stepNumber; j++) {
            sde_try<FS>(P, Start, PosOut, PosErr, allowedTime, &c);
            sc.tries++; sc.evals += 6;
            Start = PosOut;
        }
        d3 TVec = unit(sub(PosOut, PosIn));
        double tTest = norm(TVec);
        if (tTest != tTest) {
            if (m.n_adv) {  // only the advection drift
                const d3 p = add(PosIn, lin_prop(m, PosIn, h, c.time));
                c.x = p.x; c.y = p.y; c.z = p.z;
            } else {
                c.x = c.x + c.dx * h * kCLight; c.y = c.y + c.dy * h * kCLight; c.z = c.z + c.dz * h * kCLight;
            }
            set_current_step(c, h * kCLight);
            double newStep = 5 * h * kCLight;
            c.next = clipd(newStep, m.min_step, m.max_step);
            return;
        }
        d3 NVec = mk(0, 0, 0);
        for (int guard = 0; norm(NVec) == 0. && guard < 3; guard++) NVec = cross(TVec, s_vector(s));
        if (norm(NVec) == 0.) { c.active = false; c.flags |= CRP_FLAG_NAN; return; }
        NVec = unit(NVec);
        d3 BVec = unit(cross(TVec, NVec));
        d3 PO = add(add(PosOut, lin_prop(m, PosIn, h, c.time)), muls(add(muls(NVec, NStep), muls(BVec, BStep)), sqrt(h)));
        if (isnan(norm(PO))) { c.active = false; c.flags |= CRP_FLAG_NAN; return; }
        s.cursor = 12;  // the cone draw takes the fourth block of the step
        double theta = acos(s_uniform(s, 1, cos(kPi / 2.)));
        d3 axis = cross(TVec, s_vector(s));
        d3 DirOut = rotated(TVec, axis, theta);
        c.x = PO.x; c.y = PO.y; c.z = PO.z;
        DirOut = divs(DirOut, norm(DirOut));
        c.dx = DirOut.x; c.dy = DirOut.y; c.dz = DirOut.z;
        set_current_step(c, h * kCLight);
        double nextStep;
        if (stepNumber > 1) nextStep = h * pow((double)stepNumber, -2.) * kCLight;
        else nextStep = 4 * h * kCLight;
        c.next = nextStep;
    }
};

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
__global__ void __launch_bounds__(128, MinBlocks<Prop<FS>>::value) fp64_chunk_kernel(const __grid_constant__ DevPlan P, DevState s, uint64_t n,
                                                         int max_steps, uint64_t step_cap,
                                                         DevCounters *cnt, DevRecords rec,
                                                         const uint32_t *perm, uint32_t *perm_out) {
    chunk_body<Prop<FS>, CS>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out);
}

template <template <int> class Prop, int FS, int CS>
__global__ void __launch_bounds__(128, MinBlocks<Prop<FS>>::value) fp64_persistent_kernel(
    const __grid_constant__ DevPlan P, DevState s, PersistentArgs a, DevCounters *cnt, DevRecords rec) {
    // the queue is written only between launches (advance_kernel)
    const DevQueue q = *a.q;
    const uint32_t *pending_in = q.cur ? a.list_b : a.list_a;
    uint32_t *pending_out = q.cur ? a.list_a : a.list_b;
    persistent_body<Prop<FS>, CS>(P, s, pending_in, q.n_pending, q.main_base, q.n_main, pending_out,
                              a.burst, a.refill, a.budget_ns, a.step_cap, cnt, rec);
}

template <template <int> class Prop>
cudaError_t launch_persistent_prop(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                   DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                   cudaStream_t st) {
#define CRP_PERSIST(FSV, CSV) fp64_persistent_kernel<Prop, FSV, CSV><<<grid, 128, 0, st>>>(P, s, a, cnt, rec)
    if (fs == FS_GRID_PERIODIC) {
        if (P.shape == CS_PM) CRP_PERSIST(FS_GRID_PERIODIC, CS_PM);
        else if (P.shape == CS_PMO) CRP_PERSIST(FS_GRID_PERIODIC, CS_PMO);
        else CRP_PERSIST(FS_GRID_PERIODIC, CS_GENERIC);
    } else if (fs == FS_GRID) {
        CRP_PERSIST(FS_GRID, CS_GENERIC);
    } else if (fs == FS_PLANE_WAVE) {
        if (P.shape == CS_PM) CRP_PERSIST(FS_PLANE_WAVE, CS_PM);
        else if (P.shape == CS_PMO) CRP_PERSIST(FS_PLANE_WAVE, CS_PMO);
        else CRP_PERSIST(FS_PLANE_WAVE, CS_GENERIC);
    } else {
        CRP_PERSIST(FS_GENERIC, CS_GENERIC);
    }
#undef CRP_PERSIST
    return cudaGetLastError();
}

__global__ void fp64_field_kernel(const __grid_constant__ DevPlan P, uint64_t n, const double *pos, double *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d3 b = field_at<FS_GENERIC>(P, mk(pos[i], pos[n + i], pos[2 * n + i]));
    out[i] = b.x; out[n + i] = b.y; out[2 * n + i] = b.z;
}

template <template <int> class Prop>
cudaError_t launch_prop(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                        uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                        const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                        cudaStream_t st) {
    unsigned grid = (unsigned)((n + block - 1) / block);
#define CRP_CHUNK(FSV, CSV) fp64_chunk_kernel<Prop, FSV, CSV><<<grid, block, 0, st>>>(P, s, n, max_steps, \
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

cudaError_t launch_fp64_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                              uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                              const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    int prop = P.modules[P.prop_index].propagator;
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    if (prop == CRP_PROP_BP)
        return fixed ? launch_prop<BPFixed>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st)
                     : launch_prop<BPAdaptive>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
    if (prop == CRP_PROP_CK)
        return fixed ? launch_prop<CKFixed>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st)
                     : launch_prop<CKAdaptive>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
    return launch_prop<SDE>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
}

cudaError_t launch_fp64_persistent(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                   DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                   cudaStream_t st) {
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    if (pm.propagator == CRP_PROP_BP)
        return fixed ? launch_persistent_prop<BPFixed>(P, s, a, cnt, rec, fs, grid, st)
                     : launch_persistent_prop<BPAdaptive>(P, s, a, cnt, rec, fs, grid, st);
    if (pm.propagator == CRP_PROP_CK)
        return fixed ? launch_persistent_prop<CKFixed>(P, s, a, cnt, rec, fs, grid, st)
                     : launch_persistent_prop<CKAdaptive>(P, s, a, cnt, rec, fs, grid, st);
    return launch_persistent_prop<SDE>(P, s, a, cnt, rec, fs, grid, st);
}

cudaError_t launch_fp64_field(const DevPlan &P, uint64_t n, const double *pos, double *out,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    fp64_field_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(P, n, pos, out);
    return cudaGetLastError();
}

}  // namespace crp
