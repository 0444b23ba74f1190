// kst24_cmz.cuh -- KST24Field::getField (KST24Field.cpp:128-374), the
// galactic field of Korochkin, Semikoz & Tinyakov 2024, and CMZField::getField
// (CMZField.cpp:14-304), the Galactic-centre field of Guenduez et al.  FP64,
// the reference's operation order; exp, log, pow, tan, sin, cos, atan2 and
// floor are CUDA's (within two ulp of glibc's); pow(v, 2) is v * v, its
// correctly rounded value.
// Included by both stepping units: the FP64 unit compiles it without
// contraction; the mixed unit rounds the FP64 result to FP32.
#pragma once

#include "uf23.cuh"

namespace crp {

__device__ __forceinline__ void kst24_add(u3 &v, const u3 &a) { v = {v.x + a.x, v.y + a.y, v.z + a.z}; }

// KST24Field::get_toroidal (KST24Field.cpp:209)
__device__ __forceinline__ u3 kst24_toroidal(double x, double y, double z, double B, double zmin, double zmax,
                                             double rmin, double rmax) {
    if ((z <= zmin) || (zmax <= z)) return {0., 0., 0.};
    const double cR = sqrt(x * x + y * y);
    if ((rmin <= cR) && (cR <= rmax)) {
        const double theta = atan2(y, x);
        return {B * sin(theta), -B * cos(theta), 0.};
    }
    return {0., 0., 0.};
}

// KST24Field::get_Xfield (KST24Field.cpp:228)
__device__ __forceinline__ u3 kst24_x(const crp_kst24_desc &K, double x, double y, double z) {
    int sign = 1;
    if (z < 0) sign = -1;
    if (fabs(z) > 10) return {0., 0., 0.};
    const double cR = sqrt(x * x + y * y);
    const double cR_0 = cR - z * sign * tan(K.x_theta_rad);
    if ((cR_0 < K.x_rmin) || (K.x_rmax < cR_0)) return {0., 0., 0.};
    const double mgn_frc = cR_0 / cR;
    const double xy_theta = atan2(y, x);
    const double st = sin(K.x_theta_rad);
    return {K.x_b * mgn_frc * cos(xy_theta) * sign * st, K.x_b * mgn_frc * sin(xy_theta) * sign * st,
            K.x_b * mgn_frc * cos(K.x_theta_rad)};
}

// KST24Field::is_LB (KST24Field.cpp:194) and get_LB (KST24Field.cpp:252)
__device__ __forceinline__ bool kst24_in_lb(const crp_kst24_desc &K, double x, double y, double z) {
    const double ex = x - K.lb_x0, ey = y - K.lb_y0, ez = z - K.lb_z0;
    return sqrt(ex * ex + ey * ey + ez * ez) < K.lb_rmin + K.lb_dr;
}

__device__ __forceinline__ u3 kst24_lb(const crp_kst24_desc &K, double x, double y, double z) {
    double ex = x - K.lb_x0, ey = y - K.lb_y0, ez = z - K.lb_z0;
    const double cR = sqrt(ex * ex + ey * ey + ez * ez);
    if ((cR < K.lb_rmin) || (K.lb_rmin + K.lb_dr < cR)) return {0., 0., 0.};
    ex /= cR;
    ey /= cR;
    ez /= cR;
    const double cosTheta = ex * K.lb_dir[0] + ey * K.lb_dir[1] + ez * K.lb_dir[2];
    const double fx = K.lb_dir[0] - ex * cosTheta, fy = K.lb_dir[1] - ey * cosTheta, fz = K.lb_dir[2] - ez * cosTheta;
    const double ampl = (1 + (K.lb_rmin * K.lb_rmin) / (2 * K.lb_rmin * K.lb_dr + K.lb_dr * K.lb_dr));
    return {K.lb_b * ampl * fx, K.lb_b * ampl * fy, K.lb_b * ampl * fz};
}

// KST24Field::get_logspiral (KST24Field.cpp:282): the nearest turn of the
// arm's logarithmic spiral, one first-order correction of the foot point, and
// the super-elliptic cross-section around it.
__device__ __forceinline__ u3 kst24_arm(const crp_kst24_arm &A, double x, double y, double z) {
    if ((z < A.zmin) || (A.zmax < z)) return {0., 0., 0.};
    const double p0 = x + A.x_shift, p1 = y + A.y_shift, p2 = z;
    const double r = sqrt(p0 * p0 + p1 * p1);
    if ((r < A.rmin) || (A.rmax < r)) return {0., 0., 0.};
    const double a_kpc = 3;
    const double k = tan(A.pitch_deg * M_PI / 180.);
    const double cos_pitch = cos(A.pitch_deg * M_PI / 180.);
    const double sin_pitch = sin(A.pitch_deg * M_PI / 180.);
    const double phi0 = A.phi0_deg * M_PI / 180.;
    const double arc_div_rad = A.arc_div_deg * M_PI / 180.;
    const double phi = atan2(p1, p0);
    int nn = (int)floor((log(r / a_kpc) - k * (phi + phi0)) / (2 * M_PI * k));
    double r1 = a_kpc * exp(k * (phi + phi0 + 2 * M_PI * nn));
    const double r2 = r1 * exp(k * 2 * M_PI);
    if (fabs(r - r1) > fabs(r - r2)) {
        r1 = r2;
        nn++;
    }
    double xi = r1 * cos(phi), yi = r1 * sin(phi);
    double dir1 = k * xi - yi, dir2 = k * yi + xi;
    double dirtmp = sqrt(dir1 * dir1 + dir2 * dir2);
    dir1 /= dirtmp;
    dir2 /= dirtmp;
    const double delta_phi = -((xi - p0) * dir1 + (yi - p1) * dir2) / (r1 / cos_pitch);
    r1 = a_kpc * exp(k * (phi + phi0 + delta_phi + 2 * M_PI * nn));
    xi = r1 * cos(phi + delta_phi);
    yi = r1 * sin(phi + delta_phi);
    dir1 = k * xi - yi;
    dir2 = k * yi + xi;
    dirtmp = sqrt(dir1 * dir1 + dir2 * dir2);
    dir1 /= dirtmp;
    dir2 /= dirtmp;
    const double d1 = sqrt((xi - p0) * (xi - p0) + (yi - p1) * (yi - p1));
    const double L1 = r1 / sin_pitch;
    const double r_scale = 5;
    const double L1_at_r_scale = r_scale / sin_pitch;
    // std::max(a, b): (a < b) ? b : a
    const double grow_plane = A.arc_radius2 * (1 + (L1 - L1_at_r_scale) * arc_div_rad);
    const double grow_z = A.arc_radius1 * (1 + (L1 - L1_at_r_scale) * arc_div_rad);
    double arc_r_plane = (A.arc_radius2 < grow_plane) ? grow_plane : A.arc_radius2;
    double arc_r_z = (A.arc_radius1 < grow_z) ? grow_z : A.arc_radius1;
    if (arc_r_plane > 1.2) arc_r_plane = 1.2;
    if (arc_r_z > 1.2) arc_r_z = 1.2;
    const double d_at_L1 = sqrt(pow(fabs(d1 / arc_r_plane), A.arc_eps) + pow(fabs(p2 / arc_r_z), A.arc_eps));
    if ((d_at_L1 > 1) || (d_at_L1 < 0.)) return {0., 0., 0.};
    const double scaling_factor = (A.arc_radius1 * A.arc_radius2) / (arc_r_plane * arc_r_z);
    return {A.b * dir1 * scaling_factor, A.b * dir2 * scaling_factor, 0.};
}

// [T].  Not inlined: one compiled body per unit.
static __device__ __noinline__ u3 kst24_field(const crp_kst24_desc &K, double px, double py, double pz) {
    const double x = px / K.kpc, y = py / K.kpc, z = pz / K.kpc;
    u3 v = {0., 0., 0.};
    if (z > K.north_zmin) {
        kst24_add(v, kst24_toroidal(x, y, z, K.north_b, K.north_zmin, K.north_zmax, K.north_rmin, K.north_rmax));
        kst24_add(v, kst24_x(K, x, y, z));
    } else if (z < K.south_zmax) {
        kst24_add(v, kst24_toroidal(x, y, z, K.south_b, K.south_zmin, K.south_zmax, K.south_rmin, K.south_rmax));
        kst24_add(v, kst24_x(K, x, y, z));
    } else if (kst24_in_lb(K, x, y, z)) {
        kst24_add(v, kst24_lb(K, x, y, z));
    } else {
        for (int i = 0; i < 5; i++) kst24_add(v, kst24_arm(K.arms[i], x, y, z));
        kst24_add(v, kst24_x(K, x, y, z));
    }
    return {v.x * K.gauss, v.y * K.gauss, v.z * K.gauss};
}

// CMZField::BPol (CMZField.cpp:18): the X-shaped poloidal model;
// pow_integer<3>(r1) is (r1 r1) r1
__device__ __forceinline__ u3 cmz_bpol(const crp_cmz_poloidal &P, double px, double py, double pz) {
    const double x = px - P.mid[0], y = py - P.mid[1], z = pz - P.mid[2];
    const double r = sqrt(x * x + y * y);
    const double phi = atan2(y, x);
    const double r1 = 1 / (1 + P.a * z * z);
    const double Bs = P.b * exp(-r1 * r / P.l);
    const double Br = 2 * P.a * ((r1 * r1) * r1) * r * z * Bs;
    return {Br * cos(phi), Br * sin(phi), r1 * r1 * Bs};
}

// CMZField::BAz (CMZField.cpp:36): the azimuthal model of a molecular cloud
__device__ __forceinline__ u3 cmz_baz(const crp_cmz_cloud &C, double px, double py, double pz) {
    const double x = px - C.mid[0], y = py - C.mid[1], z = pz - C.mid[2];
    const double r = sqrt(x * x + y * y);
    const double phi = atan2(y, x);
    const double R = C.r, eta = C.eta;
    const double Hc = R / sqrt(log(2.));
    const double b = 1., m = 1;
    const double r1 = R / 10;
    const double v = m / eta * log((r + b) / (R + b));
    const double cosV = cos(v + m * phi);
    double Br, Bphi;
    if (r > r1) {
        const double Pre = C.b1 * cosV * exp(-z * z / Hc / Hc);
        Br = Pre * R / r;
        Bphi = -Pre / eta * R / (r + b);
    } else {
        const double Pre = C.b1 * exp(-z * z / Hc / Hc) * R / r1 * (3 * r / r1 - 2 * r * r / r1 / r1) * cosV;
        Br = Pre;
        Bphi = 1 + 6 * (r - r1) / (2 * r - 3 * r1) * (sin(v + m * phi) - sin(v)) / cosV;
        Bphi *= -Pre * r / eta / (r + b);
    }
    return {Br * cos(phi) - Bphi * sin(phi), Br * sin(phi) + Bphi * cos(phi), 0.};
}

// CMZField::getField (CMZField.cpp:289) with getMCField (:116), getICField
// (:202), getNTFField (:214) and getRadioArcField (:273).  [T]
static __device__ __noinline__ u3 cmz_field(const crp_cmz_desc &M, double px, double py, double pz) {
    u3 out = {0., 0., 0.};
    if (M.use_mc) {
        u3 b = {0., 0., 0.};
        for (int i = 0; i < 12; i++) kst24_add(b, cmz_baz(M.clouds[i], px, py, pz));
        // Sgr A*: azimuthal only
        const double x = px + M.sgra_shift[0], y = py + M.sgra_shift[1], z = pz + M.sgra_shift[2];
        const double R = M.sgra_r, B1 = M.sgra_b1;
        const double Hc = R / sqrt(log(2.));
        const double r = sqrt(x * x + y * y);
        const double r1 = R / 10;
        const double phi = atan2(y, x);
        double Bphi;
        if (r > r1)
            Bphi = -B1 * exp(-z * z / Hc / Hc) * R / r;
        else
            Bphi = -B1 * exp(-z * z / Hc / Hc) * R / r1 * (3 * r / r1 - 2 * r * r / r1 * r1);
        b.x -= Bphi * sin(phi);
        b.y += Bphi * cos(phi);
        kst24_add(out, {b.x * M.gauss, b.y * M.gauss, b.z * M.gauss});
    }
    if (M.use_ic) kst24_add(out, cmz_bpol(M.ic, px, py, pz));
    if (M.use_ntf) {
        u3 b = {0., 0., 0.};
        for (int i = 0; i < 6; i++) kst24_add(b, cmz_bpol(M.ntf[i], px, py, pz));
        const u3 p = cmz_bpol(M.ntf[6], px, py, pz);  // the Pelican: y and z swapped
        b.x += p.x;
        b.y += p.z;
        b.z += p.y;
        kst24_add(out, {b.x * M.gauss, b.y * M.gauss, b.z * M.gauss});
    }
    if (M.use_radio_arc) {
        const u3 b = cmz_bpol(M.radio_arc, px, py, pz);
        kst24_add(out, {b.x * M.gauss, b.y * M.gauss, b.z * M.gauss});
    }
    return out;
}

}  // namespace crp
