// advection.cuh -- the advection fields DiffusionSDE drifts with
// (AdvectionField::getField, AdvectionField.cpp:12-460), FP64, SI units, the
// reference's operation order; exp, pow, tanh, sin, cos and atan2 are CUDA's
// (within two ulp of glibc's); pow(v, 2) is v * v, its correctly rounded value.
// Included by both stepping units: the FP64 unit compiles it without
// contraction.
#pragma once

#include "uf23.cuh"

namespace crp {

// Vector3d::getUnitVector of (x, y, z) times f: f * (v / |v|)
__device__ __forceinline__ u3 adv_radial(double x, double y, double z, double f) {
    const double R = sqrt(x * x + y * y + z * z);
    return {f * (x / R), f * (y / R), f * (z / R)};
}

// pow_integer<8> (Common.h:58): ((x^2)^2)^2
__device__ __forceinline__ double adv_pow8(double x) {
    const double c = x * x, d = c * c;
    return d * d;
}

// One advection field (crp_advection_desc) at (x, y, z) and time t.
__device__ __forceinline__ u3 advection_one(const crp_advection_desc &A, double x, double y, double z, double t) {
    switch (A.kind) {
    case CRP_ADVECTION_TIME_SHOCK: {  // OneDimensionalTimeDependentShock::getField (TimeDependentAdvectionField.cpp:16)
        const double a = 0.5 * (A.v1 + A.v0), b = 0.5 * (A.v1 - A.v0);
        const double xsh = A.v * (t - A.t0) + A.x0;
        return {a - b * tanh((x - xsh) / A.length), 0., 0.};
    }
    case CRP_ADVECTION_SEDOV_TAYLOR: {  // SedovTaylorBlastWave::getField (TimeDependentAdvectionField.cpp:103)
        const double r = sqrt(x * x + y * y + z * z);
        if (t == 0) return adv_radial(x, y, z, 0.);
        const double ea = pow(A.energy / A.density, 1. / 5.);
        const double R = ea * pow(t, 2. / 5.);
        const double vs = 2. / 5. * ea * pow(t, -3. / 5.);
        const double xi = r / R;
        const double V = 3 * (adv_pow8(xi) + 1) / (3 * adv_pow8(xi) + 5);
        const double u = 0.5 * xi * vs * V * (1 - tanh((xi - 1) * R / A.length));
        return adv_radial(x, y, z, u);
    }
    case CRP_ADVECTION_UNIFORM:  // UniformAdvectionField::getField (:33)
        return {A.value[0], A.value[1], A.value[2]};
    case CRP_ADVECTION_CONSTANT_SPHERICAL:  // ConstantSphericalAdvectionField::getField (:54)
        return adv_radial(x - A.origin[0], y - A.origin[1], z - A.origin[2], A.v);
    case CRP_ADVECTION_SPHERICAL: {  // SphericalAdvectionField::getField (:101), getV (:120)
        const double px = x - A.origin[0], py = y - A.origin[1], pz = z - A.origin[2];
        const double R = sqrt(px * px + py * py + pz * pz);
        if (R > A.radius) return {0., 0., 0.};
        const double vR = A.v * (1 - exp(-(pow(R, A.alpha) / A.tau)));
        return adv_radial(px, py, pz, vR);
    }
    case CRP_ADVECTION_CARTESIAN_SHOCK:  // OneDimensionalCartesianShock::getField (:188)
    case CRP_ADVECTION_OBLIQUE_SHOCK: {  // ObliqueAdvectionShock::getField (:359)
        const double vDown = A.v / A.compression;
        const double a = (A.v + vDown) * 0.5, b = (A.v - vDown) * 0.5;
        const double vy = A.kind == CRP_ADVECTION_OBLIQUE_SHOCK ? A.vy : 0.;
        return {a - b * tanh(x / A.length), vy, 0.};
    }
    case CRP_ADVECTION_SPHERICAL_SHOCK_1D: {  // OneDimensionalSphericalShock::getField (:254)
        const double r = sqrt(x * x + y * y + z * z);
        const double vDown = A.v / A.compression;
        const double a = (A.v + vDown) * 0.5, b = (A.v - vDown) * 0.5;
        double v;
        if (A.cool_upstream && r <= A.radius)
            v = a - b * tanh((r - A.radius) / A.length);
        else
            v = (a - b * tanh((r - A.radius) / A.length)) * (A.radius / r) * (A.radius / r);
        return adv_radial(x, y, z, v);
    }
    default: {  // CRP_ADVECTION_SPHERICAL_SHOCK: SphericalAdvectionShock::getField (:441)
        const double px = x - A.origin[0], py = y - A.origin[1], pz = z - A.origin[2];
        const double r = sqrt(px * px + py * py + pz * pz);
        // Vector3::getUnitVectorPhi (Vector3.h:167), getPhi's zero below the least normal
        const double phi = (fabs(px) < kUfMinNormal && fabs(py) < kUfMinNormal) ? 0.0 : atan2(py, px);
        const double g = 1. / (1 + exp(-((r - A.radius) / A.length)));
        const double q = A.radius / (2 * r);
        const double v_r = A.v * (1 + (q * q - 1) * g);
        const double v_p = A.v_phi * (A.r_rot / r);
        const u3 er = adv_radial(px, py, pz, 1.0);
        const double ephx = -sin(phi), ephy = cos(phi);
        return {v_r * er.x + v_p * ephx, v_r * er.y + v_p * ephy, v_r * er.z + v_p * 0.};
    }
    }
}

// DiffusionSDE::driftStep's field (DiffusionSDE.cpp:255, :371) at the
// candidate's time t: one field, or the sum of the n fields in order
// (AdvectionFieldList::getField, :12, which passes them time 0).
__device__ __forceinline__ u3 advection_at(const crp_advection_desc *adv, int n, double x, double y, double z,
                                           double t) {
    if (n == 1) return advection_one(adv[0], x, y, z, t);
    u3 b = {0., 0., 0.};
    for (int i = 0; i < n; i++) {
        const u3 a = advection_one(adv[i], x, y, z, 0.);
        b = {b.x + a.x, b.y + a.y, b.z + a.z};
    }
    return b;
}

}  // namespace crp
