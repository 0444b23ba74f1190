// pt11.cuh -- PT11Field::getField (PT11Field.cpp:80-128), the galactic field
// of Pshirkov et al. 2011 (ASS or BSS logarithmic-spiral disk, antisymmetric
// halo), and ArchimedeanSpiralField::getField, in FP64 in SI units, the
// reference's operation order.  atan2, sin, cos, log and exp are CUDA's
// (within two ulp of glibc's); pow(v, 2) is v * v.
// Included by both stepping units; the FP64 unit compiles it without
// contraction.  r = 0 divides by zero as the reference does.
#pragma once

#include "uf23.cuh"

namespace crp {

// [T].  Not inlined: one compiled body per unit, and the generic-field
// kernels keep their register budget.
static __device__ __noinline__ u3 pt11_field(const crp_pt11_desc &P, double x, double y, double z) {
    const double r = sqrt(x * x + y * y);
    double bx = 0, by = 0, bz = 0;
    if (P.use_ass || P.use_bss) {
        // azimuth clockwise and the Sun at +x in the paper: theta = pi - phi, phi of
        // Vector3::getPhi (Vector3.h:136: 0 when |x| and |y| are below the least normal)
        const double phi = (fabs(x) < kUfMinNormal && fabs(y) < kUfMinNormal) ? 0.0 : atan2(y, x);
        const double theta = 3.14159265358979323846 - phi;
        const double cos_theta = -x / r, sin_theta = y / r;
        bx = -(P.sin_pitch * cos_theta - P.cos_pitch * sin_theta);
        by = -(-P.sin_pitch * sin_theta - P.cos_pitch * cos_theta);
        bz = -0.0;
        double m = cos(theta - P.cos_pitch / P.sin_pitch * log(r / P.r_sun) + P.phi);
        if (P.use_ass) m = fabs(m);
        const double rr = r < P.r_c ? P.r_c : r;  // std::max(r, R_c)
        m *= P.b0_d * P.r_sun / rr / P.cos_phi * exp(-fabs(z) / P.z0_d);
        bx *= m; by *= m; bz *= m;
    }
    if (P.use_halo) {
        double m = z > 0 ? P.b0_hn : -P.b0_hs;
        const double z1 = fabs(z) < P.z0_h ? P.z11_h : P.z12_h;
        const double v = (fabs(z) - P.z0_h) / z1;
        m *= r / P.r0_h * exp(1 - r / P.r0_h) / (1 + v * v);
        bx += m * (-y / r);
        by += m * (x / r);
        bz += m * 0;
    }
    return {bx, by, bz};
}

// ArchimedeanSpiralField::getField (ArchimedeanSpiralField.cpp:12-46), [T]: a
// radial field falling as (R_0 / r)^2 wound up by the rotation, reversed below
// z = 0.  theta and phi of Vector3::getTheta / getPhi (Vector3.h:136-151).
static __device__ __noinline__ u3 archimedean_field(const crp_archimedean_desc &A, double x, double y, double z) {
    const double r = sqrt(x * x + y * y + z * z);
    const bool txy = fabs(x) < kUfMinNormal && fabs(y) < kUfMinNormal;
    const double theta = (txy && fabs(z) < kUfMinNormal) ? 0.0 : atan2(sqrt(x * x + y * y), z);
    const double phi = txy ? 0.0 : atan2(y, x);
    const double cos_phi = cos(phi), sin_phi = sin(phi), cos_theta = cos(theta), sin_theta = sin(theta);
    const double c1 = A.r0 * A.r0 / r / r;
    double bx = 0.0 + c1 * cos_phi * sin_theta;
    double by = 0.0 + c1 * sin_phi * sin_theta;
    double bz = 0.0 + c1 * cos_theta;
    const double c2 = -(A.omega * A.r0 * A.r0 * sin_theta) / (r * A.vw);
    bx += c2 * (-sin_phi);
    by += c2 * cos_phi;
    if (z < 0.) { bx *= -1; by *= -1; bz *= -1; }
    return {bx * A.b0, by * A.b0, bz * A.b0};
}

}  // namespace crp
