// grid_interp.cuh -- Grid3f and Grid1f interpolation beyond the trilinear
// vector path of the stepping kernels: tricubic and nearest-neighbour
// (Grid.h:383-537), and the scalar Grid1f interpolations a
// ModulatedMagneticFieldGrid (MagneticFieldGrid.cpp:51) multiplies with.
//
// The arithmetic is the reference's, operation for operation, in both
// precision forms: the vector tricubic is its SIMD form (four-lane FP32 with
// the weights rounded to float, Grid.h:435-456), the scalar one its double
// form (Grid.h:498-536), the scalar trilinear multiplies in double and
// accumulates into a float (Grid.h:568-577 with T = float).  Intrinsics keep
// every product and sum separately rounded in translation units that
// otherwise contract multiply-adds.
#pragma once

#include "device_plan.cuh"

namespace crp {

// periodicBoundary / reflectiveBoundary of a cell index (Grid.h:37-46).
__device__ __forceinline__ int gi_periodic(int i, int n) { return ((i % n) + n) % n; }
__device__ __forceinline__ int gi_reflective(int i, int n) {
    for (int guard = 0; ((i < -0.5) || (i > (n - 0.5))) && guard < 64; guard++)
        i = 2 * n * (i > (n - 0.5)) - i - 1;
    return (i < 0 || i >= n) ? 0 : i;  // beyond 64 reflections: outside any physical use
}

// Symmetrical round (Grid.h:61).
__device__ __forceinline__ double gi_round(double r) {
    return (r > 0.0) ? floor(__dadd_rn(r, 0.5)) : ceil(__dsub_rn(r, 0.5));
}

__device__ __forceinline__ size_t gi_cell(const DevGrid &g, int ix, int iy, int iz) {
    return ((size_t)ix * (size_t)g.ny + (size_t)iy) * (size_t)g.nz + (size_t)iz;
}

// get(ix, iy, iz) through the periodic or reflective continuation.
__device__ __forceinline__ size_t gi_cell_bc(const DevGrid &g, int ix, int iy, int iz) {
    if (g.reflective)
        return gi_cell(g, gi_reflective(ix, g.nx), gi_reflective(iy, g.ny), gi_reflective(iz, g.nz));
    return gi_cell(g, gi_periodic(ix, g.nx), gi_periodic(iy, g.ny), gi_periodic(iz, g.nz));
}

struct gi3 { float x, y, z; };

// CubicInterpolate, SIMD form (Grid.h:435): c1 = 1/2, c2 = 3/2, c3 = 2,
// c4 = 5/2; pos, pos^2, pos^3 formed in double and rounded to float.
__device__ __forceinline__ float gi_cubic_f(float p0, float p1, float p2, float p3, float pos, float pos2,
                                            float pos3) {
    const float c1 = 0.5f, c2 = 1.5f, c3 = 2.f, c4 = 2.5f;
    const float term = __fmul_rn(__fsub_rn(__fmul_rn(c1, p2), __fmul_rn(c1, p0)), pos);
    const float term2 = __fmul_rn(__fsub_rn(__fadd_rn(p0, __fmul_rn(c3, p2)), __fadd_rn(__fmul_rn(c4, p1), __fmul_rn(c1, p3))),
                                  pos2);
    const float term3 = __fmul_rn(__fsub_rn(__fadd_rn(__fmul_rn(c2, p1), __fmul_rn(c1, p3)),
                                            __fadd_rn(__fmul_rn(c1, p0), __fmul_rn(c2, p2))),
                                  pos3);
    return __fadd_rn(__fadd_rn(__fadd_rn(term3, term2), term), p1);
}

__device__ __forceinline__ gi3 gi_cubic3(const gi3 p[4], double position) {
    const float pos = (float)position;
    const float pos2 = (float)__dmul_rn(position, position);
    const float pos3 = (float)__dmul_rn(__dmul_rn(position, position), position);
    gi3 r;
    r.x = gi_cubic_f(p[0].x, p[1].x, p[2].x, p[3].x, pos, pos2, pos3);
    r.y = gi_cubic_f(p[0].y, p[1].y, p[2].y, p[3].y, pos, pos2, pos3);
    r.z = gi_cubic_f(p[0].z, p[1].z, p[2].z, p[3].z, pos, pos2, pos3);
    return r;
}

// Unit-grid coordinate r = (position - gridOrigin) / spacing (Grid.h:462).
__device__ __forceinline__ void gi_unit(const DevGrid &g, double x, double y, double z, double &rx, double &ry,
                                        double &rz) {
    rx = __ddiv_rn(__dsub_rn(x, g.gox), g.sx);
    ry = __ddiv_rn(__dsub_rn(y, g.goy), g.sy);
    rz = __ddiv_rn(__dsub_rn(z, g.goz), g.sz);
}

// Grid<Vector3f>::tricubicInterpolate, SIMD form (Grid.h:459).
__device__ __forceinline__ gi3 gi_tricubic3(const DevGrid &g, double x, double y, double z) {
    double rx, ry, rz;
    gi_unit(g, x, y, z, rx, ry, rz);
    const int ix0 = (int)floor(rx), iy0 = (int)floor(ry), iz0 = (int)floor(rz);
    const double fx = __dsub_rn(rx, (double)ix0), fy = __dsub_rn(ry, (double)iy0), fz = __dsub_rn(rz, (double)iz0);
    gi3 vx[4];
#pragma unroll 1
    for (int a = -1; a < 3; a++) {
        gi3 vy[4];
#pragma unroll 1
        for (int b = -1; b < 3; b++) {
            gi3 vz[4];
#pragma unroll
            for (int c = -1; c < 3; c++) {
                const float *v = g.values + 3 * gi_cell_bc(g, ix0 + a, iy0 + b, iz0 + c);
                vz[c + 1] = gi3{__ldg(v), __ldg(v + 1), __ldg(v + 2)};
            }
            vy[b + 1] = gi_cubic3(vz, fz);
        }
        vx[a + 1] = gi_cubic3(vy, fy);
    }
    return gi_cubic3(vx, fx);
}

// Grid::closestValue (Grid.h:383): the cell index of the nearest grid point.
__device__ __forceinline__ size_t gi_nearest_cell(const DevGrid &g, double x, double y, double z) {
    double rx, ry, rz;
    gi_unit(g, x, y, z, rx, ry, rz);
    int ix, iy, iz;
    if (g.reflective) {
        ix = (int)gi_round(rx);
        iy = (int)gi_round(ry);
        iz = (int)gi_round(rz);
        return gi_cell(g, gi_reflective(ix, g.nx), gi_reflective(iy, g.ny), gi_reflective(iz, g.nz));
    }
    ix = (int)gi_round(fmod(rx, (double)g.nx));
    iy = (int)gi_round(fmod(ry, (double)g.ny));
    iz = (int)gi_round(fmod(rz, (double)g.nz));
    ix = (ix + g.nx * (ix < 0)) % g.nx;
    iy = (iy + g.ny * (iy < 0)) % g.ny;
    iz = (iz + g.nz * (iz < 0)) % g.nz;
    return gi_cell(g, ix, iy, iz);
}

// clipVolume test of Grid::interpolate (Grid.h:319).
__device__ __forceinline__ bool gi_in_volume(const DevGrid &g, double x, double y, double z) {
    bool in = (x >= g.ox) && (x <= g.ex);
    in &= (y >= g.oy) && (y <= g.ey);
    in &= (z >= g.oz) && (z <= g.ez);
    return in;
}

// Grid<Vector3f>::interpolate for the tricubic and nearest-neighbour types.
__device__ __forceinline__ gi3 gi_vector_other(const DevGrid &g, double x, double y, double z) {
    if (g.clip_volume && !gi_in_volume(g, x, y, z)) return gi3{0.f, 0.f, 0.f};
    if (g.interp == CRP_INTERPOLATION_TRICUBIC) return gi_tricubic3(g, x, y, z);
    const float *v = g.values + 3 * gi_nearest_cell(g, x, y, z);
    return gi3{__ldg(v), __ldg(v + 1), __ldg(v + 2)};
}

// CubicInterpolateScalar (Grid.h:498), double.
__device__ __forceinline__ double gi_cubic_d(double p0, double p1, double p2, double p3, double pos) {
    const double a = __dadd_rn(__dsub_rn(__dadd_rn(__dmul_rn(-0.5, p0), __dmul_rn(1.5, p1)), __dmul_rn(1.5, p2)),
                               __dmul_rn(0.5, p3));
    const double b = __dsub_rn(__dadd_rn(__dsub_rn(p0, __dmul_rn(2.5, p1)), __dmul_rn(p2, 2.)), __dmul_rn(0.5, p3));
    const double c = __dadd_rn(__dmul_rn(-0.5, p0), __dmul_rn(0.5, p2));
    const double t3 = __dmul_rn(__dmul_rn(__dmul_rn(a, pos), pos), pos);
    const double t2 = __dmul_rn(__dmul_rn(b, pos), pos);
    const double t1 = __dmul_rn(c, pos);
    return __dadd_rn(__dadd_rn(__dadd_rn(t3, t2), t1), p1);
}

// Grid<float>::interpolate (Grid.h:317) of a scalar grid (values: one float
// per cell): trilinear with double weights accumulated into a float,
// tricubic in double, or the nearest value.
__device__ __forceinline__ float gi_scalar(const DevGrid &g, double x, double y, double z) {
    if (g.clip_volume && !gi_in_volume(g, x, y, z)) return 0.f;
    if (g.interp == CRP_INTERPOLATION_NEAREST_NEIGHBOUR) return __ldg(g.values + gi_nearest_cell(g, x, y, z));
    double rx, ry, rz;
    gi_unit(g, x, y, z, rx, ry, rz);
    if (g.interp == CRP_INTERPOLATION_TRICUBIC) {
        const int ix0 = (int)floor(rx), iy0 = (int)floor(ry), iz0 = (int)floor(rz);
        const double fx = __dsub_rn(rx, (double)ix0), fy = __dsub_rn(ry, (double)iy0),
                     fz = __dsub_rn(rz, (double)iz0);
        double vx[4];
#pragma unroll 1
        for (int a = -1; a < 3; a++) {
            double vy[4];
#pragma unroll 1
            for (int b = -1; b < 3; b++) {
                double vz[4];
#pragma unroll
                for (int c = -1; c < 3; c++) vz[c + 1] = (double)__ldg(g.values + gi_cell_bc(g, ix0 + a, iy0 + b, iz0 + c));
                vy[b + 1] = gi_cubic_d(vz[0], vz[1], vz[2], vz[3], fz);
            }
            vx[a + 1] = gi_cubic_d(vy[0], vy[1], vy[2], vy[3], fy);
        }
        return (float)gi_cubic_d(vx[0], vx[1], vx[2], vx[3], fx);
    }
    // trilinear (Grid.h:539) with periodicClamp / reflectiveClamp (Grid.h:29, 49)
    const double r[3] = {rx, ry, rz};
    const int n[3] = {g.nx, g.ny, g.nz};
    int lo[3], hi[3];
    double f0[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double v = r[a];
        if (g.reflective) {
            for (int guard = 0; ((v < -0.5) || (v > (n[a] - 0.5))) && guard < 64; guard++)
                v = __dsub_rn(__dsub_rn(2 * n[a] * (v > (n[a] - 0.5)), v), 1.);
            lo[a] = (int)floor(v);
            hi[a] = lo[a] + (lo[a] < n[a] - 1);
            if (v < 0) { lo[a] = 0; hi[a] = 0; }
            if (lo[a] < 0 || lo[a] >= n[a]) { lo[a] = 0; hi[a] = 0; }
        } else {
            lo[a] = (((int)floor(v) % n[a]) + n[a]) % n[a];
            hi[a] = (lo[a] + 1) % n[a];
        }
        f0[a] = __dsub_rn(v, floor(v));
    }
    const double f1[3] = {__dsub_rn(1., f0[0]), __dsub_rn(1., f0[1]), __dsub_rn(1., f0[2])};
    // corner order and weights of Grid.h:570-577
    const int sel[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, 1, 1}};
    float b = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int ix = sel[k][0] ? hi[0] : lo[0], iy = sel[k][1] ? hi[1] : lo[1], iz = sel[k][2] ? hi[2] : lo[2];
        const double w = __dmul_rn(__dmul_rn(__dmul_rn((double)__ldg(g.values + gi_cell(g, ix, iy, iz)),
                                                       sel[k][0] ? f0[0] : f1[0]),
                                             sel[k][1] ? f0[1] : f1[1]),
                                   sel[k][2] ? f0[2] : f1[2]);
        b = (float)__dadd_rn((double)b, w);
    }
    return b;
}

}  // namespace crp
