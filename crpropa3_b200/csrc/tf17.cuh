// tf17.cuh -- TF17Field::getField (TF17Field.cpp:197-303), the galactic
// field of Terral & Ferriere 2017: disk models Ad1, Bd1, Dd1 and halo models
// C0, C1; and PolarizedSingleModeMagneticField::getField
// (PolarizedSingleModeMagneticField.cpp:59).  FP64, SI units, the reference's
// operation order; atan2, sin, cos, exp and log are CUDA's (within two ulp
// of glibc's).
// Included by both stepping units; the FP64 unit compiles it without
// contraction.
#pragma once

#include "uf23.cuh"

namespace crp {

// TF17Field::zscale (TF17Field.cpp:304)
__device__ __forceinline__ double tf17_zscale(const crp_tf17_desc &T, double z) {
    return 1 + z * z / T.h_p / T.h_p;
}

// TF17Field::shiftedWindingFunction (TF17Field.cpp:300)
__device__ __forceinline__ double tf17_winding(const crp_tf17_desc &T, double r, double z) {
    return T.cot_p0 * log(1 - exp(-r / T.l_p) + T.epsilon) / tf17_zscale(T, z);
}

// TF17Field::radialFieldScale (TF17Field.cpp:293)
__device__ __forceinline__ double tf17_radial_scale(const crp_tf17_desc &T, double B1, double phi_star, double z1,
                                                   double phi, double r, double z) {
    const double phi_prime = phi - tf17_winding(T, r, z) - phi_star;
    return B1 * exp(-fabs(z1) / T.h_disk) * cos(phi_prime);
}

// TF17Field::azimuthalFieldComponent (TF17Field.cpp:285)
__device__ __forceinline__ double tf17_azimuthal(const crp_tf17_desc &T, double r, double z, double B_r,
                                                double B_z) {
    const double r_ = r / T.l_p;
    const double rscale = r > T.epsilon ? r_ * exp(-r_) / (1 - exp(-r_)) : 1 - r_ / 2. - r_ * r_ / 12.;
    double B_phi = T.cot_p0 / tf17_zscale(T, z) * rscale * B_r;
    B_phi = B_phi - 2 * z * r / (T.h_p * T.h_p) / tf17_zscale(T, z) * tf17_winding(T, r, z) * B_z;
    return B_phi;
}

// (r, phi, z) components to (x, y, z), the x component flipped (TF17Field.cpp:253)
__device__ __forceinline__ u3 tf17_cartesian(double B_r, double B_phi, double B_z, double sinPhi, double cosPhi) {
    return {-(B_r * cosPhi - B_phi * sinPhi), B_r * sinPhi + B_phi * cosPhi, B_z};
}

// TF17Field::getDiskField (TF17Field.cpp:201)
__device__ __forceinline__ u3 tf17_disk(const crp_tf17_desc &T, double r, double z, double phi, double sinPhi,
                                        double cosPhi) {
    double B_r = 0, B_phi = 0, B_z = 0;
    if (T.disk_model == CRP_TF17_AD1) {
        if (r > T.r1_disk) {
            const double z1_disk_z = (1. + T.a_disk * T.r1_disk * T.r1_disk) / (1. + T.a_disk * r * r);
            const double B_r0 = tf17_radial_scale(T, T.b1_disk, T.phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = (T.r1_disk / r) * z1_disk_z * B_r0;
            B_z = 2 * T.a_disk * T.r1_disk * z1_disk_z * z / (1 + T.a_disk * r * r) * B_r0;
            B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
        } else {
            const double phi1_disk = tf17_winding(T, T.r1_disk, z) + T.phi_star_disk;
            const double B_amp = T.b1_disk * exp(-fabs(z) / T.h_disk);
            B_r = cos(phi1_disk - phi) * B_amp;
            B_phi = sin(phi1_disk - phi) * B_amp;
        }
    } else if (T.disk_model == CRP_TF17_BD1) {
        if (r > T.epsilon) {
            const double r1_disk_r = T.r1_disk / r;
            const double z1_disk_z = 5. / (r1_disk_r * r1_disk_r + 4. / sqrt(r1_disk_r));
            const double B_r0 = tf17_radial_scale(T, T.b1_disk, T.phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = r1_disk_r * z1_disk_z * B_r0;
            B_z = -0.4 * r1_disk_r / r * z1_disk_z * z1_disk_z * z * (r1_disk_r * r1_disk_r - 1. / sqrt(r1_disk_r)) *
                  B_r0;
        } else {
            const double z1_disk_z = 5. * r * r / (T.r1_disk * T.r1_disk);
            const double B_r0 = tf17_radial_scale(T, T.b1_disk, T.phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = 5. * r / T.r1_disk * B_r0;
            B_z = -10. * z / T.r1_disk * B_r0;
        }
        B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    } else {  // CRP_TF17_DD1
        const double z_sign = z >= 0 ? 1. : -1.;
        const double z_abs = fabs(z);
        if (z_abs > T.epsilon) {
            const double z1_disk_z = T.z1_disk / z_abs;
            const double r1_disk_r = 1.5 / (sqrt(z1_disk_z) + 0.5 / z1_disk_z);
            const double F_r = r1_disk_r * r <= T.l_disk ? 1. : exp(1. - r1_disk_r * r / T.l_disk);
            const double B_z0 = z_sign * T.b1_disk * F_r * cos(phi - tf17_winding(T, r, z) - T.phi_star_disk);
            B_r = -0.5 / 1.5 * r1_disk_r * r1_disk_r * r1_disk_r * r / z_abs * (sqrt(z1_disk_z) - 1 / z1_disk_z) *
                  B_z0;
            B_z = z_sign * r1_disk_r * r1_disk_r * B_z0;
        } else {
            const double z_z1_disk = z_abs / T.z1_disk;
            const double r1_disk_r = 1.5 * sqrt(z_abs / T.z1_disk);
            const double F_r = r1_disk_r * r <= T.l_disk ? 1. : exp(1. - r1_disk_r * r / T.l_disk);
            const double B_z0 = z_sign * T.b1_disk * F_r * cos(phi - tf17_winding(T, r, z) - T.phi_star_disk);
            B_r = -1.125 * r / T.z1_disk * (1 - 2.5 * z_z1_disk * sqrt(z_z1_disk)) * B_z0;
            B_z = z_sign * r1_disk_r * r1_disk_r * B_z0;
        }
        B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    }
    return tf17_cartesian(B_r, B_phi, B_z, sinPhi, cosPhi);
}

// TF17Field::getHaloField (TF17Field.cpp:259)
__device__ __forceinline__ u3 tf17_halo(const crp_tf17_desc &T, double r, double z, double phi, double sinPhi,
                                        double cosPhi) {
    const double r1_halo_r = (1. + T.a_halo * T.z1_halo * T.z1_halo) / (1. + T.a_halo * z * z);
    double B_z0;
    if (T.halo_model == CRP_TF17_C0) {
        B_z0 = T.b1_halo * exp(-r1_halo_r * r / T.l_halo);
    } else {  // CRP_TF17_C1
        const double phi_prime = phi - tf17_winding(T, r, z) - T.phi_star_halo;
        B_z0 = T.b1_halo * exp(-r1_halo_r * r / T.l_halo) * cos(phi_prime);
    }
    const double B_r = 2 * T.a_halo * r1_halo_r * r1_halo_r * r * z / (1. + T.a_halo * z * z) * B_z0;
    const double B_z = r1_halo_r * r1_halo_r * B_z0;
    const double B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    return tf17_cartesian(B_r, B_phi, B_z, sinPhi, cosPhi);
}

// [T].  Not inlined: one compiled body per unit.
static __device__ __noinline__ u3 tf17_field(const crp_tf17_desc &T, double x, double y, double z) {
    const double r = sqrt(x * x + y * y);
    // azimuth pi - phi, phi of Vector3::getPhi (0 when |x| and |y| are below the least normal)
    const double phi = 3.14159265358979323846 -
                       ((fabs(x) < kUfMinNormal && fabs(y) < kUfMinNormal) ? 0.0 : atan2(y, x));
    const double cosPhi = cos(phi), sinPhi = sin(phi);
    double bx = 0., by = 0., bz = 0.;
    if (T.use_disk) {
        const u3 d = tf17_disk(T, r, z, phi, sinPhi, cosPhi);
        bx = bx + d.x; by = by + d.y; bz = bz + d.z;
    }
    if (T.use_halo) {
        const u3 h = tf17_halo(T, r, z, phi, sinPhi, cosPhi);
        bx = bx + h.x; by = by + h.y; bz = bz + h.z;
    }
    return {bx, by, bz};
}

// PolarizedSingleModeMagneticField::getField: B_max (u1 cos(k.d) + (u2 sigma) sin(k.d)), d = x - r0
static __device__ __noinline__ u3 single_mode_field(const crp_single_mode_desc &S, double x, double y, double z) {
    const double dx = x - S.r0[0], dy = y - S.r0[1], dz = z - S.r0[2];
    const double ph = S.k[0] * dx + S.k[1] * dy + S.k[2] * dz;
    const double c = cos(ph), s = sin(ph);
    return {(S.u1[0] * c + S.u2[0] * S.sigma * s) * S.b_max, (S.u1[1] * c + S.u2[1] * S.sigma * s) * S.b_max,
            (S.u1[2] * c + S.u2[2] * S.sigma * s) * S.b_max};
}

}  // namespace crp
