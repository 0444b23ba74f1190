// uf23.cuh -- UF23Field (UF23Field.cpp:269-558), the eight coherent
// galactic field models of Unger & Farrar 2023, in FP64 in the model's own
// units (kpc, microgauss), the reference's operation order.  exp, log, sin,
// cos, acos, atan2 and pow are CUDA's (within two ulp of glibc's), pow(v, 2)
// is v * v, and the two powers of model constants (A/Z)^P and A^P come
// precomputed from the host.  Included by both stepping units; the FP64 unit
// compiles it without contraction.
#pragma once

#include "device_plan.cuh"

namespace crp {

struct u3 { double x, y, z; };

__device__ __forceinline__ u3 uf_cyl_to_cart(double v0, double v1, double v2, double cosPhi, double sinPhi) {
    return {v0 * cosPhi - v1 * sinPhi, v0 * sinPhi + v1 * cosPhi, v2};  // uf23::CylToCart
}
__device__ __forceinline__ double uf_sigmoid(double x, double x0, double w) {
    return 1 / (1 + exp(-(x - x0) / w));  // uf23::Sigmoid
}
__device__ __forceinline__ double uf_delta_phi(double phi0, double phi1) {
    return acos(cos(phi1) * cos(phi0) + sin(phi1) * sin(phi0));  // uf23::DeltaPhi
}
__device__ __forceinline__ double uf_sq(double v) { return v * v; }
constexpr double kUfMinNormal = 2.2250738585072014e-308;  // numeric_limits<double>::min()
constexpr double kUfPi = 3.1415926535897932384626;

// getSpiralField (UF23Field.cpp:510)
__device__ __forceinline__ u3 uf_spiral(const crp_uf23_desc &U, double x, double y, double z) {
    const double rRef = 5, rInner = 5, wInner = 0.5, rOuter = 20, wOuter = 0.5;
    const double r2 = x * x + y * y;
    if (r2 == 0) return {0, 0, 0};
    const double r = sqrt(r2);
    const double phi = atan2(y, x);
    const double hdz = 1 - uf_sigmoid(fabs(z), U.disk_h, U.disk_w);
    const double rFacI = uf_sigmoid(r, rInner, wInner);
    const double rFacO = 1 - uf_sigmoid(r, rOuter, wOuter);
    const double rFac = r > 1e-5 * (1e-3 * 1) ? (1 - exp(-r * r)) / r : r * (1 - r2 / 2);
    const double gdrTimesRrefByR = rRef * rFac * rFacO * rFacI;
    const double phi0 = phi - log(r / rRef) / U.tan_pitch;
    const double b = U.disk_b1 * cos(1 * (phi0 - U.disk_phase1)) + U.disk_b2 * cos(2 * (phi0 - U.disk_phase2)) +
                     U.disk_b3 * cos(3 * (phi0 - U.disk_phase3));
    const double fac = hdz * gdrTimesRrefByR;
    return uf_cyl_to_cart(b * fac * U.sin_pitch, b * fac * U.cos_pitch, 0, x / r, y / r);
}

// getSpurField (UF23Field.cpp:453)
__device__ __forceinline__ u3 uf_spur(const crp_uf23_desc &U, double x, double y, double z) {
    const double rRef = 8.2, twoPi = 2 * kUfPi;
    const double r = sqrt(x * x + y * y);
    if (r < kUfMinNormal) return {0, 0, 0};
    double phi = atan2(y, x);
    if (phi < 0) phi += twoPi;
    const double phiRef = U.disk_phase1;
    int iBest = -2;
    double bestDist = -1;
    for (int i = -1; i <= 1; ++i) {
        const double pphi = phi - phiRef + i * twoPi;
        const double rr = rRef * exp(pphi * U.tan_pitch);
        if (bestDist < 0 || fabs(r - rr) < bestDist) {
            bestDist = fabs(r - rr);
            iBest = i;
        }
    }
    if (iBest != 0) return {0, 0, 0};
    const double phi0 = phi - log(r / rRef) / U.tan_pitch;
    const double delta = uf_delta_phi(phiRef, phi0) / U.spur_width;
    const double B = U.disk_b1 * exp(-0.5 * uf_sq(delta));
    const double wS = 5 * (kUfPi / 180.);
    const double gS = 1 - uf_sigmoid(fabs(uf_delta_phi(U.spur_center, phi)), U.spur_length, wS);
    const double hd = 1 - uf_sigmoid(fabs(z), U.disk_h, U.disk_w);
    const double bS = rRef / r * B * hd * gS;
    return uf_cyl_to_cart(bS * U.sin_pitch, bS * U.cos_pitch, 0, x / r, y / r);
}

// getToroidalHaloField (UF23Field.cpp:361)
__device__ __forceinline__ u3 uf_toroidal(const crp_uf23_desc &U, double x, double y, double z) {
    const double r = sqrt(x * x + y * y);
    const double absZ = fabs(z);
    const double b0 = z >= 0 ? U.toroidal_bn : U.toroidal_bs;
    const double sigmoidR = uf_sigmoid(r, U.toroidal_r, U.toroidal_w);
    const double sigmoidZ = uf_sigmoid(absZ, U.disk_h, U.disk_w);
    const double bPhi = b0 * (1. - sigmoidR) * sigmoidZ * exp(-absZ / U.toroidal_z);
    const double cosPhi = r > kUfMinNormal ? x / r : 1;
    const double sinPhi = r > kUfMinNormal ? y / r : 0;
    return uf_cyl_to_cart(0, bPhi, 0, cosPhi, sinPhi);
}

// getPoloidalHaloField (UF23Field.cpp:385)
__device__ __forceinline__ u3 uf_poloidal(const DevUF23 &W, double x, double y, double z) {
    const crp_uf23_desc &U = W.d;
    const double r = sqrt(x * x + y * y);
    const double P = U.poloidal_p;
    const double c = W.c_pol;
    const double a0p = W.a0p;
    const double rp = pow(r, P);
    const double cabszp = c * pow(fabs(z), P);
    const double t0 = a0p + cabszp - rp;
    const double t1 = sqrt(uf_sq(t0) + 4 * a0p * rp);
    const double ap = 2 * a0p * rp / (t1 + t0);
    double a = 0;
    if (ap < 0) {
        if (r > kUfMinNormal) a = __longlong_as_double(0x7ff8000000000000ll);  // the reference throws
    } else {
        a = pow(ap, 1 / P);
    }
    const double radialDependence =
        U.model == CRP_UF23_EXPX ? exp(-a / U.poloidal_r) : 1 - uf_sigmoid(a, U.poloidal_r, U.poloidal_w);
    const double Bzz = U.poloidal_b * radialDependence;
    const double rOverA = 1 / pow(2 * a0p / (t1 + t0), 1 / P);
    const double signZ = z < 0 ? -1 : 1;
    const double Br = Bzz * c * a / rOverA * signZ * pow(fabs(z), P - 1) / t1;
    const double Bz = Bzz * pow(rOverA, P - 2) * (ap + a0p) / t1;
    if (r < kUfMinNormal) return {0, 0, Bz};
    return uf_cyl_to_cart(Br, 0, Bz, x / r, y / r);
}

// getTwistedHaloField (UF23Field.cpp:318)
__device__ __forceinline__ u3 uf_twisted(const DevUF23 &W, double x, double y, double z) {
    const crp_uf23_desc &U = W.d;
    const double r = sqrt(x * x + y * y);
    const double cosPhi = r > kUfMinNormal ? x / r : 1;
    const double sinPhi = r > kUfMinNormal ? y / r : 0;
    const u3 bX = uf_poloidal(W, x, y, z);
    const double bR = bX.x * cosPhi + bX.y * sinPhi;  // uf23::CartToCyl
    const double bZ = bX.z;
    double bPhi = 0;
    if (U.twisting_time != 0 && r != 0) {
        const double kilometer = 1 / 3.0856775807e+16;
        const double second = 1 / (1e6 * 60 * 60 * 24 * 365.25);
        const double v0 = -240 * kilometer / second;
        const double r0 = 1.6, z0 = 10;
        const double fr = 1 - exp(-r / r0);
        const double t0 = exp(2 * fabs(z) / z0);
        const double gz = 2 / (1 + t0);
        const double signZ = z < 0 ? -1 : 1;
        const double deltaZ = -signZ * v0 * fr / z0 * t0 * uf_sq(gz);
        const double deltaR = v0 * ((1 - fr) / r0 - fr / r) * gz;
        bPhi = (bZ * deltaZ + bR * deltaR) * U.twisting_time;
    }
    return uf_cyl_to_cart(bR, bPhi, bZ, cosPhi, sinPhi);
}

// UF23Field::getField (UF23Field.cpp:269) and operator() (:277), [T].
// Not inlined: one compiled body per unit, and the generic-field kernels keep
// their register budget.
static __device__ __noinline__ u3 uf23_field(const DevUF23 &W, double px, double py, double pz) {
    const crp_uf23_desc &U = W.d;
    const double x = px / U.kpc * 1, y = py / U.kpc * 1, z = pz / U.kpc * 1;
    if (x * x + y * y + z * z > U.max_radius_squared) return {0, 0, 0};
    const u3 d = U.model == CRP_UF23_SPUR ? uf_spur(U, x, y, z) : uf_spiral(U, x, y, z);
    u3 h;
    if (U.model == CRP_UF23_TWISTX) {
        h = uf_twisted(W, x, y, z);
    } else {
        const u3 t = uf_toroidal(U, x, y, z), p = uf_poloidal(W, x, y, z);
        h = {t.x + p.x, t.y + p.y, t.z + p.z};
    }
    return {(d.x + h.x) * U.microgauss, (d.y + h.y) * U.microgauss, (d.z + h.z) * U.microgauss};
}

}  // namespace crp
