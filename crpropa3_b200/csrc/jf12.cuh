// jf12.cuh -- the regular field of JF12Field and PlanckJF12bField
// (JF12Field.cpp:195-298) and of JF12FieldSolenoidal, whose disk and X
// fields replace the JF12 ones (JF12FieldSolenoidal.cpp:115-302), in FP64, SI
// units, the reference's operation order.  exp, log, sin, cos, atan and atan2
// are CUDA's (within an ulp or two of glibc's); pow(v, 2) is v * v, its
// correctly rounded value.
// Included by both stepping units: the FP64 unit compiles it without
// contraction; the mixed unit evaluates JF12FieldSolenoidal with it and rounds
// the result to FP32.
#pragma once

#include "uf23.cuh"

namespace crp {

// JF12Field::logisticFunction (JF12Field.cpp:195)
__device__ __forceinline__ double jf_logistic(double x, double x0, double w) {
    return 1. / (1. + exp(-2. * (fabs(x) - x0) / w));
}

__device__ __forceinline__ double jf_sq(double v) { return v * v; }

// Vector3::getPhi (Vector3.h:136)
__device__ __forceinline__ double jf_phi(double x, double y) {
    if ((fabs(x) < kUfMinNormal) && (fabs(y) < kUfMinNormal)) return 0.0;
    return atan2(y, x);
}

// Radius of the spiral arm through (r, phi) where it crosses the negative x
// axis, the arm-region lookup of getDiskField / getTurbulentStrength
// (JF12Field.cpp:228-233, :315-320).
__device__ __forceinline__ double jf_r_negx(const crp_jf12_desc &J, double r, double phi) {
    double r_negx = r * exp(-(phi - M_PI) / J.tan90_minus_pitch);
    if (r_negx > J.r_arms[7]) r_negx = r * exp(-(phi + M_PI) / J.tan90_minus_pitch);
    if (r_negx > J.r_arms[7]) r_negx = r * exp(-(phi + 3 * M_PI) / J.tan90_minus_pitch);
    return r_negx;
}

// JF12FieldSolenoidal::getDiskTransitionPolynomial (:197) and its derivative
// (:219): r1/r between the transitions, a quadratic in each transition.
__device__ __forceinline__ void jf12s_transition(const crp_jf12_desc &J, double r, double &p, double &q) {
    if ((r < J.r1) || (r > J.r2)) { p = 0.; q = 0.; return; }
    if ((r > J.r1s) && (r < J.r2s)) { p = J.r1 / r; q = 0.; return; }
    double r_a = J.r1, r_b = J.r1s;
    if (r >= J.r2s) { r_a = J.r2; r_b = J.r2s; }
    const double fakt = (r_a / r_b - 2.) / ((r_a - r_b) * (r_a - r_b));
    p = (J.r1 / r_b) * (2. - r / r_b + fakt * (r - r_b) * (r - r_b));
    q = (J.r1 / r_b) * (2. - 2. * r / r_b + fakt * (3. * r * r - 4. * r * r_b + r_b * r_b));
}

// JF12FieldSolenoidal::getDiskField (:115) with getHPhiIntegral (:241) and
// getSpiralFieldStrengthConstant (:260): the arm of (r, phi) found at r1 along
// the logarithmic spiral; the bound on the arm index only matters for a NaN
// azimuth (atan2's range keeps it below 10 otherwise).
__device__ __forceinline__ u3 jf12s_disk(const crp_jf12_desc &J, double r, double z, double phi, double sinPhi,
                                         double cosPhi) {
    if (!J.use_disk) return {0., 0., 0.};
    const double lfDisk = jf_logistic(z, J.h_disk, J.w_disk);
    if (!((J.r1 < r) && (r < J.r2))) return {0., 0., 0.};
    double phi1 = phi - log(r / J.r1) * J.cot_pitch;
    phi1 = atan2(sin(phi1), cos(phi1));
    int idx = 1;
    while (idx < 10 && phi1 < J.phi0_arms[idx]) idx += 1;
    const double hint = phi1 * J.b_arms[idx] + J.phi_coeff[idx];
    const double mag1 = J.b_arms[idx];
    double pdelta, qdelta;
    jf12s_transition(J, r, pdelta, qdelta);
    const double br = pdelta * mag1 * J.sin_pitch;
    const double bphi = pdelta * mag1 * J.cos_pitch - qdelta * hint * J.sin_pitch;
    const double s = 1 - lfDisk;
    return {(0. + (br * cosPhi - bphi * sinPhi)) * s, (0. + (br * sinPhi + bphi * cosPhi)) * s, 0. * s};
}

// JF12FieldSolenoidal::getXField (:131): the JF12 X field above |z| = zS,
// parabolic field lines below it.
__device__ __forceinline__ u3 jf12s_x(const crp_jf12_desc &J, double r, double z, double sinPhi, double cosPhi) {
    if (!J.use_x) return {0., 0., 0.};
    const double zS = J.z_s, rXc = J.r_xc, rX = J.r_x, bX = J.b_x, tanT = J.tan_theta_x0;
    const double rc = rXc + fabs(z) / tanT;
    const double r0c = rXc + zS / tanT;
    if (fabs(z) > zS) {
        if (r == 0.) {
            const double a = 1. + fabs(z) * J.cot_theta_x0 / rXc;
            return {0., 0., bX / (a * a)};
        }
        double bMagX, sinThetaX, cosThetaX, rp;
        if (r < rc) {
            rp = r * rXc / rc;
            bMagX = bX * exp(-1 * rp / rX) * (rXc / rc) * (rXc / rc);
            double thetaX = atan(fabs(z) / (r - rp));
            if (z == 0) thetaX = M_PI / 2.;
            sinThetaX = sin(thetaX);
            cosThetaX = cos(thetaX);
        } else {
            rp = r - fabs(z) / tanT;
            bMagX = bX * exp(-rp / rX) * (rp / r);
            sinThetaX = J.sin_theta_x0;
            cosThetaX = J.cos_theta_x0;
        }
        const double zsign = z < 0 ? -1 : 1;
        return {0. + zsign * bMagX * cosThetaX * cosPhi, 0. + zsign * bMagX * cosThetaX * sinPhi,
                0. + bMagX * sinThetaX};
    }
    double r0 = r * 1. / (1. - 1. / (2. * (zS + rXc * tanT)) * (zS - z * z / zS));
    double f;
    if (r0 >= r0c) {
        r0 = r + 1. / (2. * tanT) * (zS - z * z / zS);
        f = 1. + 1 / (2 * r * tanT / zS) * (1. - (z / zS) * (z / zS));
    } else {
        const double g = 1. - 1. / (2. + 2. * (rXc * tanT / zS)) * (1. - (z / zS) * (z / zS));
        f = 1. / (g * g);
    }
    double br0, bz0;
    if (r0 < r0c) {
        const double rp = r0 * rXc / r0c;
        const double thetaX = atan(zS / (r0 - rp));
        br0 = bX * exp(-rp / rX) * (rXc / r0c) * (rXc / r0c) * cos(thetaX);
        bz0 = bX * exp(-rp / rX) * (rXc / r0c) * (rXc / r0c) * sin(thetaX);
    } else {
        const double rp = r0 - zS / tanT;
        br0 = bX * exp(-rp / rX) * (rp / r0) * J.cos_theta_x0;
        bz0 = bX * exp(-rp / rX) * (rp / r0) * J.sin_theta_x0;
    }
    const double br = z / zS * f * br0;
    const double bz = bz0 * f;
    return {0. + br * cosPhi, 0. + br * sinPhi, 0. + bz};
}

// JF12Field::getRegularField (JF12Field.cpp:199) with getDiskField (:216),
// getToroidalHaloField (:248) and getXField (:267); JF12FieldSolenoidal
// (variant 2) with its own disk and X fields.
__device__ __forceinline__ u3 jf12_regular_fp64(const crp_jf12_desc &J, double px, double py, double pz) {
    u3 b = {0., 0., 0.};
    const double kpc = J.kpc;
    const double d = sqrt(px * px + py * py + pz * pz);
    if (!(d < 20 * kpc)) return b;
    const double r = sqrt(px * px + py * py), z = pz;
    const double phi = jf_phi(px, py);
    const double sinPhi = sin(phi), cosPhi = cos(phi);
    const bool sol = J.variant == CRP_JF12_SOLENOIDAL;
    u3 bd = {0., 0., 0.};
    if (sol) {
        bd = jf12s_disk(J, r, z, phi, sinPhi, cosPhi);
    } else if (J.use_disk) {
        const double lfDisk = jf_logistic(z, J.h_disk, J.w_disk);
        if (r > 3 * kpc) {
            if (r < 5 * kpc) {  // molecular ring
                const double bMag = J.b_ring * (5 * kpc / r) * (1 - lfDisk);
                bd.x += -bMag * sinPhi;
                bd.y += bMag * cosPhi;
            } else {            // spiral region
                const double r_negx = jf_r_negx(J, r, phi);
                double bMag = 0;
                for (int i = 7; i >= 0; i--)
                    if (r_negx < J.r_arms[i]) bMag = J.b_disk[i];
                bMag *= (5 * kpc / r) * (1 - lfDisk);
                bd.x += bMag * (J.sin_pitch * cosPhi - J.cos_pitch * sinPhi);
                bd.y += bMag * (J.sin_pitch * sinPhi + J.cos_pitch * cosPhi);
            }
        }
    }
    b = {b.x + bd.x, b.y + bd.y, b.z + bd.z};
    const bool outside1 = r * r + z * z > 1 * kpc * kpc;
    u3 bh = {0., 0., 0.};
    if (J.use_toroidal_halo && outside1) {
        const double lfDisk = jf_logistic(z, J.h_disk, J.w_disk);
        double bMagH = exp(-fabs(z) / J.z0) * lfDisk;
        if (z >= 0)
            bMagH *= J.b_north * (1 - jf_logistic(r, J.r_north, J.w_halo));
        else
            bMagH *= J.b_south * (1 - jf_logistic(r, J.r_south, J.w_halo));
        bh.x += -bMagH * sinPhi;
        bh.y += bMagH * cosPhi;
    }
    b = {b.x + bh.x, b.y + bh.y, b.z + bh.z};
    u3 bx = {0., 0., 0.};
    if (sol) {
        bx = jf12s_x(J, r, z, sinPhi, cosPhi);
    } else if (J.use_x && outside1) {
        double bMagX, sinThetaX, cosThetaX, rp;
        const double rc = J.r_xc + fabs(z) / J.tan_theta_x0;
        if (r < rc) {  // varying elevation region
            rp = r * J.r_xc / rc;
            bMagX = J.b_x * exp(-1 * rp / J.r_x) * jf_sq(J.r_xc / rc);
            double thetaX = atan2(fabs(z), (r - rp));
            if (z == 0) thetaX = M_PI / 2.;
            sinThetaX = sin(thetaX);
            cosThetaX = cos(thetaX);
        } else {       // constant elevation region
            rp = r - fabs(z) / J.tan_theta_x0;
            bMagX = J.b_x * exp(-rp / J.r_x) * (rp / r);
            sinThetaX = J.sin_theta_x0;
            cosThetaX = J.cos_theta_x0;
        }
        const double zsign = z < 0 ? -1 : 1;
        bx.x += zsign * bMagX * cosThetaX * cosPhi;
        bx.y += zsign * bMagX * cosThetaX * sinPhi;
        bx.z += bMagX * sinThetaX;
    }
    return {b.x + bx.x, b.y + bx.y, b.z + bx.z};
}

}  // namespace crp
