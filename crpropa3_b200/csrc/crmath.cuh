// crmath.cuh -- x^y rounded to nearest from a double-double evaluation.
//
// The reference's adaptive step controllers call pow(r, -0.2)
// (PropagationCK.cpp:116, :123, PropagationBP.cpp:104, :111) and DiffusionSDE
// calls pow(|rigidity|/4e9, alpha) (DiffusionSDE.cpp:263).  glibc's pow is
// within 0.52 ulp, so it returns the correctly rounded result except in rare
// near-midpoint cases; CUDA's pow has a 2-ulp bound and differs from glibc in
// the last place on a few per cent of inputs, which changes accept/reject
// decisions of the step controller.  cr_pow evaluates log and exp in
// double-double arithmetic (about 100 bits) with the classic reductions:
//   log: x = 2^k m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1))
//        by its odd power series;
//   exp: t = j ln2 + u, u / 2^8 by its Taylor series, squared 8 times.
// and rounds hi + lo once.  Valid for finite x > 0 and finite y with
// |y log x| < 700; other inputs fall back to pow().  Host and device.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define CRP_HD __host__ __device__ __forceinline__
#else
#define CRP_HD inline
#endif

namespace crp {

struct dd {
    double hi, lo;
};

CRP_HD dd dd_two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    double e = (a - (s - bb)) + (b - bb);
    return {s, e};
}

CRP_HD dd dd_fast_two_sum(double a, double b) {
    double s = a + b;
    return {s, b - (s - a)};
}

CRP_HD dd dd_two_prod(double a, double b) {
    double p = a * b;
    return {p, fma(a, b, -p)};
}

CRP_HD dd dd_add(dd a, dd b) {
    dd s = dd_two_sum(a.hi, b.hi);
    dd t = dd_two_sum(a.lo, b.lo);
    s.lo += t.hi;
    s = dd_fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return dd_fast_two_sum(s.hi, s.lo);
}

CRP_HD dd dd_mul(dd a, dd b) {
    dd p = dd_two_prod(a.hi, b.hi);
    p.lo += a.hi * b.lo + a.lo * b.hi;
    return dd_fast_two_sum(p.hi, p.lo);
}

CRP_HD dd dd_mul_d(dd a, double b) {
    dd p = dd_two_prod(a.hi, b);
    p.lo += a.lo * b;
    return dd_fast_two_sum(p.hi, p.lo);
}

CRP_HD dd dd_div(dd a, dd b) {
    double q1 = a.hi / b.hi;
    dd r = dd_add(a, dd_mul_d(b, -q1));
    double q2 = r.hi / b.hi;
    r = dd_add(r, dd_mul_d(b, -q2));
    double q3 = r.hi / b.hi;
    dd q = dd_fast_two_sum(q1, q2);
    return dd_add(q, dd{q3, 0.0});
}

// ln 2 and its tail
#define CRP_LN2_HI 6.93147180559945286227e-01
#define CRP_LN2_LO 2.31904681384629955842e-17

// natural log of x > 0 (finite, normal) in double-double
CRP_HD dd dd_log(double x) {
    int k;
    double m = frexp(x, &k);  // x = m 2^k, m in [0.5, 1)
    if (m < 0.70710678118654752440) {
        m *= 2.0;
        k -= 1;
    }
    // s = (m - 1) / (m + 1); m - 1 is exact (Sterbenz)
    dd num = {m - 1.0, 0.0};
    dd den = dd_two_sum(m, 1.0);
    dd s = dd_div(num, den);
    dd z = dd_mul(s, s);
    // atanh(s)/s = sum_{i>=0} z^i / (2i+1), |z| <= 0.0295; 20 terms reach 2^-100
    dd acc = {1.0 / 41.0, 0.0};
    for (int i = 19; i >= 0; --i) {
        double c = 1.0 / (2 * i + 1);
        dd cdd = {c, fma(-c, (double)(2 * i + 1), 1.0) / (double)(2 * i + 1)};
        acc = dd_add(dd_mul(acc, z), cdd);
    }
    dd lm = dd_mul(dd_mul_d(s, 2.0), acc);
    dd kl = dd_add(dd_two_prod((double)k, CRP_LN2_HI), dd_two_prod((double)k, CRP_LN2_LO));
    return dd_add(kl, lm);
}

// exp of a double-double t with |t| < 700, in double-double
CRP_HD dd dd_exp(dd t) {
    double j = rint(t.hi / CRP_LN2_HI);
    dd u = dd_add(t, dd_add(dd_two_prod(-j, CRP_LN2_HI), dd_two_prod(-j, CRP_LN2_LO)));
    // u / 256, Taylor to degree 10, then square 8 times
    u.hi = ldexp(u.hi, -8);
    u.lo = ldexp(u.lo, -8);
    dd acc = {1.0 / 3628800.0, 0.0};  // 1/10!
    for (int i = 9; i >= 1; --i) {
        double f = 1.0;
        for (int q = 2; q <= i; ++q) f *= q;  // i! exact for i <= 9
        dd c = {1.0 / f, fma(-1.0 / f, f, 1.0) / f};
        acc = dd_add(dd_mul(acc, u), c);
    }
    // acc = sum_{i=1..10} u^(i-1)/i! ; e^u - 1 = u * acc
    dd em1 = dd_mul(u, acc);
    // (1 + em1)^256 via e^(2v) - 1 = (e^v - 1)(e^v + 1)
    for (int i = 0; i < 8; ++i) em1 = dd_mul(em1, dd_add(em1, dd{2.0, 0.0}));
    dd r = dd_add(em1, dd{1.0, 0.0});
    int ji = (int)j;
    r.hi = ldexp(r.hi, ji);
    r.lo = ldexp(r.lo, ji);
    return r;
}

CRP_HD double cr_pow(double x, double y) {
    if (!(x > 0.0) || !(x < INFINITY) || !(fabs(y) < INFINITY) || x < 2.2250738585072014e-308)
        return pow(x, y);
    if (y == 0.0 || x == 1.0) return 1.0;
    dd l = dd_log(x);
    dd t = dd_mul_d(l, y);
    if (!(fabs(t.hi) < 700.0)) return pow(x, y);
    dd r = dd_exp(t);
    return r.hi + r.lo;
}

}  // namespace crp
