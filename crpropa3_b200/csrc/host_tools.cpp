// host_tools.cpp -- host-side set-up and output of the stepping engine:
//   * crpropa::Random (MT19937, src/Random.cpp) for the draws the reference
//     makes on the host: PlaneWaveTurbulence modes, Source features;
//   * PlaneWaveTurbulence mode set-up (PlaneWaveTurbulence.cpp:79-229);
//   * Source sampling for the stepping workloads (Source.cpp);
//   * particle charge (ParticleState::setId, ParticleState.cpp:50);
//   * the TextOutput line formatter (TextOutput.cpp:55, :166).
// No device is needed for any of these.
#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <zlib.h>

#include "crp_gpu.h"

namespace crp {
void set_last_error(const char *msg);  // crp_engine.cu
}

namespace {

crp_status host_fail(crp_status st, const char *msg) {
    crp::set_last_error(msg);
    return st;
}

// MT19937 with the seeding, tempering and real conversions of crpropa::Random.
class Mt {
    uint32_t s_[624];
    int left_ = 0, next_ = 0;
    static uint32_t twist(uint32_t m, uint32_t a, uint32_t b) {
        uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
        return m ^ (y >> 1) ^ ((0u - (b & 1u)) & 0x9908b0dfu);
    }
    void reload() {
        int i = 0;
        for (; i < 624 - 397; i++) s_[i] = twist(s_[i + 397], s_[i], s_[i + 1]);
        for (; i < 623; i++) s_[i] = twist(s_[i - (624 - 397)], s_[i], s_[i + 1]);
        s_[623] = twist(s_[396], s_[623], s_[0]);
        left_ = 624;
        next_ = 0;
    }

public:
    explicit Mt(uint32_t seed) {
        s_[0] = seed;
        for (int i = 1; i < 624; i++) s_[i] = 1812433253u * (s_[i - 1] ^ (s_[i - 1] >> 30)) + (uint32_t)i;
        reload();
    }
    uint32_t u32() {
        if (left_ == 0) reload();
        --left_;
        uint32_t y = s_[next_++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        return y ^ (y >> 18);
    }
    double rand() { return double(u32()) * (1.0 / 4294967295.0); }
    double exc() { return double(u32()) * (1.0 / 4294967296.0); }               // randExc
    double dbl_exc() { return (double(u32()) + 0.5) * (1.0 / 4294967296.0); }  // randDblExc
    // randNorm(0, 1) (Random.cpp:111): Box-Muller, one value per two draws
    double norm() {
        const double r = std::sqrt(-2.0 * std::log(1.0 - dbl_exc())) * 1.0;
        const double phi = 2.0 * 3.14159265358979323846264338328 * exc();
        return 0.0 + r * std::cos(phi);
    }
    double uniform(double a, double b) { return a + (b - a) * rand(); }
    void vector(double &x, double &y, double &z) {
        double zz = uniform(-1.0, 1.0);
        double t = uniform(-1.0 * M_PI, M_PI);
        double r = std::sqrt(1 - zz * zz);
        x = r * std::cos(t); y = r * std::sin(t); z = zz;
    }
    double power_law(double index, double mn, double mx) {
        if (std::fabs(index + 1.0) < 2.220446049250313e-16) {
            double p1 = std::log(mx), p2 = std::log(mn);
            return std::exp((p1 - p2) * rand() + p2);
        }
        double p1 = std::pow(mx, index + 1), p2 = std::pow(mn, index + 1);
        double ex = 1 / (index + 1);
        return std::pow((p1 - p2) * rand() + p2, ex);
    }
};

// HepPID nucleus test for +/-10LZZZAAAI ids (L = 0, A >= Z), 2212 and 2112.
bool nucleus(int32_t id, int &Z) {
    int64_t a = id < 0 ? -(int64_t)id : id;
    if (a == 2212) { Z = 1; return true; }
    if (a == 2112) { Z = 0; return true; }
    if (a >= 1000000000LL && a < 2000000000LL && (a / 100000000) % 10 == 0) {
        int z = (int)((a / 10000) % 1000), A = (int)((a / 10) % 1000);
        if (A >= z) { Z = z; return true; }
    }
    return false;
}

const double kEplus = 1.602176487e-19;  // Units.h:54

}  // namespace

extern "C" {

crp_status crp_particle_charge(int32_t id, double *charge) {
    if (!charge) return host_fail(CRP_ERR_INVALID_ARGUMENT, "charge is NULL");
    int Z;
    if (nucleus(id, Z)) {
        // ParticleState::setId: chargeNumber(id) * eplus, negated for anti-nuclei
        double q = Z * kEplus;
        if (id < 0) q *= -1;
        *charge = q;
        return CRP_OK;
    }
    switch (id) {
    case 11: case 13: case 15: *charge = -1 * kEplus; return CRP_OK;
    case -11: case -13: case -15: *charge = 1 * kEplus; return CRP_OK;
    case 22: case 12: case -12: case 14: case -14: case 16: case -16: *charge = 0; return CRP_OK;
    default: break;
    }
    return host_fail(CRP_ERR_UNSUPPORTED, "particle id outside the charge table of the device path");
}

crp_status crp_random_draws(uint32_t seed, int32_t kind, uint64_t n, double a, double b, double c,
                            double *out) {
    if (!out && n) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    Mt r(seed);
    for (uint64_t i = 0; i < n; i++) {
        switch (kind) {
        case 0: out[i] = r.rand(); break;
        case 1: out[i] = r.uniform(a, b); break;
        case 2: r.vector(out[3 * i], out[3 * i + 1], out[3 * i + 2]); break;
        case 3: out[i] = r.power_law(a, b, c); break;
        case 4: out[i] = r.norm(); break;
        case 6: out[i] = (double)r.u32(); break;
        default: return host_fail(CRP_ERR_INVALID_ARGUMENT, "unknown draw kind");
        }
    }
    return CRP_OK;
}

crp_status crp_turbulence_draws(uint32_t seed, int32_t kind, uint64_t n_modes, double *out) {
    if (!out && n_modes) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    if (seed == 0) return host_fail(CRP_ERR_INVALID_ARGUMENT, "seed 0 is not reproducible; give a non-zero seed");
    if (kind < CRP_TURBULENCE_GRID || kind > CRP_TURBULENCE_HELICAL)
        return host_fail(CRP_ERR_INVALID_ARGUMENT, "unknown turbulence kind");
    // The MT19937 stream is sequential, the conversions of its words are not: the words are
    // drawn first (rand takes one, randNorm two), then converted on all host threads, which
    // gives the same values as drawing the conversions one after another.
    const int words = kind == CRP_TURBULENCE_GRID ? 2 : 4;
    std::vector<uint32_t> u((size_t)words * n_modes);
    Mt r(seed);
    for (size_t i = 0; i < u.size(); i++) u[i] = r.u32();
    auto rand_of = [](uint32_t w) { return double(w) * (1.0 / 4294967295.0); };   // Random::rand
    auto norm_of = [](uint32_t w1, uint32_t w2) {                                   // randNorm(0, 1)
        const double r1 = std::sqrt(-2.0 * std::log(1.0 - (double(w1) + 0.5) * (1.0 / 4294967296.0))) * 1.0;
        const double phi = 2.0 * 3.14159265358979323846264338328 * (double(w2) * (1.0 / 4294967296.0));
        return 0.0 + r1 * std::cos(phi);
    };
    auto convert = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; i++) {
            const uint32_t *w = &u[(size_t)words * i];
            if (kind == CRP_TURBULENCE_GRID) {          // GridTurbulence.cpp:97, :104
                out[2 * i] = rand_of(w[0]);
                out[2 * i + 1] = rand_of(w[1]);
            } else if (kind == CRP_TURBULENCE_SIMPLE) { // SimpleGridTurbulence.cpp:88-93
                out[3 * i] = rand_of(w[0]);
                out[3 * i + 1] = norm_of(w[1], w[2]);
                out[3 * i + 2] = rand_of(w[3]);
            } else {                                    // HelicalGridTurbulence.cpp:88-92
                out[3 * i] = norm_of(w[0], w[1]);
                out[3 * i + 1] = rand_of(w[2]);
                out[3 * i + 2] = rand_of(w[3]);
            }
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = n_modes < (1u << 16) ? 1u : std::min(hw, 32u);
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; t++)
        pool.emplace_back(convert, n_modes * t / nt, n_modes * (t + 1) / nt);
    convert(0, n_modes / nt);
    for (auto &th : pool) th.join();
    return CRP_OK;
}

crp_status crp_jf12_defaults(int32_t variant, crp_jf12_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    if (variant == CRP_JF12_SOLENOIDAL) {  // the constructor's default arguments (JF12FieldSolenoidal.h:62)
        const double parsec = 648000 / M_PI * 149597870700.0;
        return crp_jf12_solenoidal(3 * (1e3 * parsec), 0.5 * (1e3 * parsec), out);
    }
    if (variant != 0 && variant != 1) return host_fail(CRP_ERR_INVALID_ARGUMENT, "JF12 variant must be 0, 1 or 2");
    // Units.h: tesla = 1, gauss = 1e-4 tesla, au = 149597870700 m, parsec = 648000 / pi au
    const double au = 149597870700.0, parsec = 648000 / M_PI * au, kpc = 1e3 * parsec;
    const double gauss = 1e-4, muG = 1e-6 * gauss;
    crp_jf12_desc &j = *out;
    std::memset(&j, 0, sizeof(j));
    j.use_regular = j.use_disk = j.use_toroidal_halo = j.use_x = 1;
    j.variant = variant;
    j.kpc = kpc;
    // the constructor evaluates sin, cos and tan at run time (JF12Field.cpp:17-22, 55-58); the
    // volatile angles keep this compiler from folding them with another rounding
    volatile double pitch_v = 11.5 * M_PI / 180, theta_v = 49.0 * M_PI / 180;
    const double pitch = pitch_v, thetaX0 = theta_v;
    j.sin_pitch = std::sin(pitch);
    j.cos_pitch = std::cos(pitch);
    j.tan90_minus_pitch = std::tan(M_PI / 2 - pitch);
    const double arms[8] = {5.1, 6.3, 7.1, 8.3, 9.8, 11.4, 12.7, 15.5};
    for (int i = 0; i < 8; i++) j.r_arms[i] = arms[i] * kpc;
    j.b_ring = 0.1 * muG;
    j.h_disk = 0.40 * kpc;
    j.w_disk = 0.27 * kpc;
    const double disk[8] = {0.1, 3.0, -0.9, -0.8, -2.0, -4.2, 0.0, 2.7};
    for (int i = 0; i < 8; i++) j.b_disk[i] = disk[i] * muG;
    j.b_north = 1.4 * muG;
    j.b_south = -1.1 * muG;
    j.r_north = 9.22 * kpc;
    j.r_south = 17 * kpc;
    j.w_halo = 0.20 * kpc;
    j.z0 = 5.3 * kpc;
    j.b_x = 4.6 * muG;
    j.sin_theta_x0 = std::sin(thetaX0);
    j.cos_theta_x0 = std::cos(thetaX0);
    j.tan_theta_x0 = std::tan(thetaX0);
    j.r_xc = 4.8 * kpc;
    j.r_x = 2.9 * kpc;
    volatile double beta_v = 1.36;
    j.sqrt_beta = std::sqrt((double)beta_v);
    const double turb[8] = {10.81, 6.96, 9.59, 6.96, 1.96, 16.34, 37.29, 10.35};
    for (int i = 0; i < 8; i++) j.b_disk_turb[i] = turb[i] * muG;
    j.b_disk_turb5 = 7.63 * muG;
    j.z_disk_turb = 0.61 * kpc;
    j.b_halo_turb = 4.68 * muG;
    j.r_halo_turb = 10.97 * kpc;
    j.z_halo_turb = 2.84 * kpc;
    if (variant == 1) {  // PlanckJF12bField (JF12Field.cpp:352-371)
        j.b_disk[5] = -3.5 * muG;
        j.b_x = 1.8 * muG;
        const double pturb[8] = {3.12, 6.24, 3.12, 6.24, 3.12, 6.24, 3.12, 6.24};
        for (int i = 0; i < 8; i++) j.b_disk_turb[i] = pturb[i] * muG;
        j.b_disk_turb5 = 3.90 * muG;
        j.b_halo_turb = 7.332 * muG;
    }
    return CRP_OK;
}

crp_status crp_jf12_solenoidal(double delta, double zs, crp_jf12_desc *out) {
    // JF12FieldSolenoidal::JF12FieldSolenoidal (JF12FieldSolenoidal.cpp:8-77) on JF12Field's state
    crp_status st = crp_jf12_defaults(CRP_JF12_JF12, out);
    if (st != CRP_OK) return st;
    crp_jf12_desc &j = *out;
    j.variant = CRP_JF12_SOLENOIDAL;
    const double kpc = j.kpc, muG = 1e-6 * 1e-4;
    // the constructor's tan and log run at run time; volatile operands keep them from folding
    volatile double pitch_v = 11.5 * M_PI / 180;
    const double pitch = pitch_v;
    j.cot_pitch = 1. / std::tan(pitch);
    j.cot_theta_x0 = 1. / j.tan_theta_x0;
    j.z_s = zs;
    j.delta = delta;
    j.r1 = 5 * kpc;
    j.r2 = 20 * kpc;
    j.r1s = j.r1 + delta;
    j.r2s = j.r2 - delta;
    const double phi0 = 0.;
    double *a = j.phi0_arms, *b = j.b_arms, *c = j.phi_coeff;
    for (int i = 1; i < 9; i++) {
        volatile double ratio = j.r_arms[i - 1] / j.r1;
        a[i] = M_PI - j.cot_pitch * std::log((double)ratio);
    }
    a[0] = a[8] + 2 * M_PI;
    a[9] = a[1] - 2 * M_PI;
    a[10] = a[2] - 2 * M_PI;
    int idx0 = 1;
    while (idx0 < 10 && phi0 < a[idx0]) idx0 += 1;
    const double arms[8] = {0, 0.1, 3.0, -0.9, -0.8, -2.0, -4.2, 0.0};
    for (int i = 1; i < 8; i++) b[i] = arms[i] * muG;
    double flux1to7 = 0.;  // the eighth arm closes the net flux through r1
    for (int i = 1; i < 8; i++) flux1to7 += (a[i - 1] - a[i]) * b[i];
    b[8] = -flux1to7 / (a[7] - a[8]);
    b[0] = b[8];
    b[9] = b[1];
    b[10] = b[2];
    c[0] = 0;
    for (int i = 1; i < 10; i++) c[i] = c[i - 1] + (b[i - 1] - b[i]) * a[i - 1];
    const double corr = c[idx0] + b[idx0] * phi0;  // H(phi0) = 0
    for (int i = 1; i < 10; i++) c[i] = c[i] - corr;
    return CRP_OK;
}

crp_status crp_uf23_defaults(int32_t model, crp_uf23_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    if (model < CRP_UF23_BASE || model > CRP_UF23_NEBCOR) return host_fail(CRP_ERR_INVALID_ARGUMENT, "unknown field model");
    // the model's units (UF23Field.cpp:48-57): kpc = 1, microgauss = 1, megayear = 1
    const double kPi = 3.1415926535897932384626, degree = kPi / 180.;
    // Table 3 of the UF23 paper as the constructor sets it (UF23Field.cpp:70-256), one row per
    // model: B1 B2 B3 H phase1 phase2 phase3 pitch W | poloidal B P R W Z | striation |
    // toroidal BN BS R W Z  (angles in degrees); spur, twistX and expX add their own below
    struct Row { double v[20]; };
    static const Row rows[8] = {
        /* base */ {{1.0878565e+00, 2.6605034e+00, 3.1166311e+00, 7.9408965e-01, 2.6316589e+02, 9.7782269e+01,
                     3.5112281e+01, 1.0106900e+01, 1.0720909e-01, 9.7775487e-01, 1.4266186e+00, 7.2925417e+00,
                     1.1188158e-01, 4.4597373e+00, 3.4557571e-01, 3.2556760e+00, -3.0914569e+00, 1.0193815e+01,
                     1.6936993e+00, 4.0242749e+00}},
        /* neCL */ {{1.4259645e+00, 1.3543223e+00, 3.4390669e+00, 6.7405199e-01, 1.9961898e+02, 1.3541461e+02,
                     6.4909767e+01, 1.1867859e+01, 6.1162799e-02, 9.8387831e-01, 1.6773615e+00, 7.4084361e+00,
                     1.4168192e-01, 3.6521188e+00, 3.3600213e-01, 2.6256593e+00, -2.5699466e+00, 1.0134257e+01,
                     1.1547728e+00, 4.5585463e+00}},
        /* expX */ {{9.9258148e-01, 2.1821124e+00, 3.1197345e+00, 7.1508681e-01, 2.4745741e+02, 9.8578879e+01,
                     3.4884485e+01, 1.0027070e+01, 9.8524736e-02, 5.8357990e+00, 1.9510779e+00, 2.4994376e+00,
                     0, 0, 5.1440500e-01, 2.7077434e+00, -2.5677104e+00, 1.0134022e+01, 2.0956159e+00,
                     5.4564991e+00}},
        /* spur */ {{-4.2993328e+00, 0, 0, 7.5019749e-01, 1.5589875e+02, 0, 0, 1.2074432e+01, 1.2263120e-01,
                     9.9302987e-01, 1.3982374e+00, 7.1973387e+00, 1.2262244e-01, 4.4853270e+00, 3.3022369e-01,
                     2.9286724e+00, -2.5979895e+00, 9.7536425e+00, 1.4210055e+00, 6.0941229e+00}},
        /* cre10 */ {{1.2035697e+00, 2.7478490e+00, 3.2104342e+00, 8.0844932e-01, 2.6515882e+02, 9.8211313e+01,
                      3.5944588e+01, 1.0162759e+01, 1.0824003e-01, 9.6938453e-01, 1.4150957e+00, 7.2987296e+00,
                      1.0923051e-01, 4.5748332e+00, 2.4950386e-01, 3.7308133e+00, -3.5039958e+00, 1.0407507e+01,
                      1.7398375e+00, 2.9272800e+00}},
        /* synCG */ {{8.1386878e-01, 2.0586930e+00, 2.9437335e+00, 6.2172353e-01, 2.2988551e+02, 9.7388282e+01,
                      3.2927367e+01, 9.9034844e+00, 6.6517521e-02, 8.0883734e-01, 1.5820957e+00, 7.4625235e+00,
                      1.5003765e-01, 3.5338550e+00, 6.3434763e-01, 2.3991193e+00, -2.0919944e+00, 9.4227834e+00,
                      9.1608418e-01, 5.5844594e+00}},
        /* twistX */ {{1.3741995e+00, 2.0089881e+00, 1.5212463e+00, 9.3806180e-01, 2.3560316e+02, 1.0189856e+02,
                       5.6187572e+01, 1.2100979e+01, 1.4933338e-01, 6.2793114e-01, 2.3292519e+00, 7.9212358e+00,
                       2.9056201e-01, 2.6274437e+00, 7.7616317e-01, 0, 0, 0, 0, 0}},
        /* nebCor */ {{1.4081935e+00, 3.5292400e+00, 4.1290147e+00, 8.1151971e-01, 2.6447529e+02, 9.7572660e+01,
                       3.6403798e+01, 1.0151183e+01, 1.1863734e-01, 1.3485916e+00, 1.3414395e+00, 7.2473841e+00,
                       1.4318227e-01, 4.8242603e+00, 3.8610837e-10, 4.6491142e+00, -4.5006610e+00, 1.0205288e+01,
                       1.7004868e+00, 3.5557767e+00}},
    };
    const double *v = rows[model].v;
    crp_uf23_desc &u = *out;
    std::memset(&u, 0, sizeof(u));
    u.model = model;
    // the a -> infinity of all but expX: "1 * Gpc" in the constructor names crpropa::Gpc
    // (Units.h:116, in metres), not uf23::Gpc, so a is 1 Gpc in metres read as kpc
    const double au_ = 149597870700.0, parsec_ = 648000 / M_PI * au_;
    u.poloidal_a = 1 * (1e9 * parsec_);
    u.disk_b1 = v[0]; u.disk_b2 = v[1]; u.disk_b3 = v[2]; u.disk_h = v[3];
    u.disk_phase1 = v[4] * degree; u.disk_phase2 = v[5] * degree; u.disk_phase3 = v[6] * degree;
    u.disk_pitch = v[7] * degree; u.disk_w = v[8];
    u.poloidal_b = v[9]; u.poloidal_p = v[10]; u.poloidal_r = v[11]; u.poloidal_w = v[12];
    u.poloidal_z = v[13]; u.striation = v[14];
    u.toroidal_bn = v[15]; u.toroidal_bs = v[16]; u.toroidal_r = v[17]; u.toroidal_w = v[18];
    u.toroidal_z = v[19];
    if (model == CRP_UF23_SPUR) {
        u.spur_center = 1.5718686e+02 * degree;
        u.spur_length = 3.1839577e+01 * degree;
        u.spur_width = 1.0318114e+01 * degree;
    }
    if (model == CRP_UF23_TWISTX) u.twisting_time = 5.4733549e+01;
    if (model == CRP_UF23_EXPX) {  // internally xi is fitted and z = tan(xi) a
        u.poloidal_a = 6.1938701e+00;
        volatile double xi = 2.0926122e+01 * degree;
        u.poloidal_xi = xi;
        u.poloidal_z = u.poloidal_a * std::tan(u.poloidal_xi);
    }
    volatile double pitch = u.disk_pitch;  // evaluated at run time, as the constructor does
    u.sin_pitch = std::sin((double)pitch);
    u.cos_pitch = std::cos((double)pitch);
    u.tan_pitch = std::tan((double)pitch);
    u.max_radius_squared = std::pow(30., 2);
    const double au = 149597870700.0, parsec = 648000 / M_PI * au;
    u.kpc = 1e3 * parsec;
    u.microgauss = 1e-6 * 1e-4;
    return CRP_OK;
}

// PT11Field::SetParams (PT11Field.cpp:28): the pitch's cosine and sine and the phase PHI of the
// first reversal, through the C library at run time (volatile: no compile-time folding)
static void pt11_set_params(crp_pt11_desc &p) {
    volatile double pitch = p.pitch, d = p.d, r_sun = p.r_sun;
    p.cos_pitch = std::cos(pitch);
    p.sin_pitch = std::sin(pitch);
    p.phi = p.cos_pitch / p.sin_pitch * std::log1p(d / r_sun) - M_PI / 2;
    volatile double phi = p.phi;
    p.cos_phi = std::cos(phi);
}

crp_status crp_pt11_defaults(crp_pt11_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    const double au = 149597870700.0, parsec = 648000 / M_PI * au, kpc = 1e3 * parsec;
    const double gauss = 1e-4, muG = 1e-6 * gauss;
    crp_pt11_desc &p = *out;
    std::memset(&p, 0, sizeof(p));
    // PT11Field() (PT11Field.cpp:8-26): ASS disk and halo
    p.use_ass = 1;
    p.use_halo = 1;
    p.d = -0.6 * kpc;
    p.r_sun = 8.5 * kpc;
    p.r_c = 5.0 * kpc;
    p.z0_d = 1.0 * kpc;
    p.b0_d = 2.0 * muG;
    p.z0_h = 1.3 * kpc;
    p.r0_h = 8.0 * kpc;
    p.b0_hn = 4.0 * muG;
    p.b0_hs = 4.0 * muG;
    p.z11_h = 0.25 * kpc;
    p.z12_h = 0.4 * kpc;
    return crp_pt11_use(out, CRP_PT11_ASS, 1);
}

// TF17Field(disk, halo) (TF17Field.cpp:10-118): the parameters of the six model combinations,
// formed with the constructor's own expressions, and set_p0's cotangent (TF17Field.cpp:146)
// through the C library at run time.
crp_status crp_tf17_defaults(int32_t disk, int32_t halo, crp_tf17_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    if (disk < CRP_TF17_AD1 || disk > CRP_TF17_DD1 || halo < CRP_TF17_C0 || halo > CRP_TF17_C1)
        return host_fail(CRP_ERR_INVALID_ARGUMENT, "TF17Field: unknown disk or halo model");
    const double au = 149597870700.0, parsec = 648000 / M_PI * au, kpc = 1e3 * parsec;
    const double muG = 1e-6 * 1e-4;
    crp_tf17_desc &t = *out;
    std::memset(&t, 0, sizeof(t));
    t.disk_model = disk;
    t.halo_model = halo;
    t.use_disk = 1;
    t.use_halo = 1;
    double p0 = 0;
    if (halo == CRP_TF17_C0 && disk == CRP_TF17_AD1) {
        t.r1_disk = 3 * kpc; t.b1_disk = 19.0 * muG; t.h_disk = 0.055 * kpc;
        t.phi_star_disk = -54 * M_PI / 180; t.a_disk = 0.9 / kpc / kpc;
        t.z1_halo = 0; t.b1_halo = 0.36 * muG; t.l_halo = 3.0 * kpc; t.a_halo = 1.17 / kpc / kpc;
        p0 = -7.9 * M_PI / 180; t.h_p = 5 * kpc; t.l_p = 50 * kpc;
    } else if (halo == CRP_TF17_C0 && disk == CRP_TF17_BD1) {
        t.r1_disk = 3 * kpc; t.b1_disk = 2.0 * muG; t.h_disk = 0.32 * kpc;
        t.phi_star_disk = 153 * M_PI / 180;
        t.z1_halo = 0; t.b1_halo = 0.29 * muG; t.l_halo = 3.4 * kpc; t.a_halo = 0.88 / kpc / kpc;
        p0 = -7.2 * M_PI / 180; t.h_p = 9 * kpc; t.l_p = 50 * kpc;
    } else if (halo == CRP_TF17_C0 && disk == CRP_TF17_DD1) {
        t.z1_disk = 1.5 * kpc; t.b1_disk = 0.065 * muG; t.l_disk = 9.8 * kpc;
        t.phi_star_disk = 14 * M_PI / 180;
        t.z1_halo = 0; t.b1_halo = 0.18 * muG; t.l_halo = 4.8 * kpc; t.a_halo = 0.61 / kpc / kpc;
        p0 = -7.4 * M_PI / 180; t.h_p = 4.2 * kpc; t.l_p = 50 * kpc;
    } else if (halo == CRP_TF17_C1 && disk == CRP_TF17_AD1) {
        t.r1_disk = 3 * kpc; t.b1_disk = 32.0 * muG; t.h_disk = 0.054 * kpc;
        t.phi_star_disk = -31 * M_PI / 180; t.a_disk = 0.031 / kpc / kpc;
        t.z1_halo = 0; t.b1_halo = 9.0 * muG; t.l_halo = 2.1 * kpc;
        t.phi_star_halo = 198 * M_PI / 180; t.a_halo = 0.33 / kpc / kpc;
        p0 = -9.1 * M_PI / 180; t.h_p = 1.2 * kpc; t.l_p = 50 * kpc;
    } else if (halo == CRP_TF17_C1 && disk == CRP_TF17_BD1) {
        t.r1_disk = 3 * kpc; t.b1_disk = 24 * muG; t.h_disk = 0.090 * kpc;
        t.phi_star_disk = -34 * M_PI / 180;
        t.z1_halo = 0; t.b1_halo = 8.2 * muG; t.l_halo = 2.2 * kpc;
        t.phi_star_halo = 197 * M_PI / 180; t.a_halo = 0.38 / kpc / kpc;
        p0 = -9.0 * M_PI / 180; t.h_p = 1.2 * kpc; t.l_p = 50 * kpc;
    } else {  // C1, Dd1
        t.z1_disk = 1.5 * kpc; t.b1_disk = 0.40 * muG; t.l_disk = 2.9 * kpc;
        t.phi_star_disk = 120 * M_PI / 180;
        t.z1_halo = 0; t.b1_halo = 9.5 * muG; t.l_halo = 2.1 * kpc;
        t.phi_star_halo = 179 * M_PI / 180; t.a_halo = 0.45 / kpc / kpc;
        p0 = -8.4 * M_PI / 180; t.h_p = 1.2 * kpc; t.l_p = 50 * kpc;
    }
    t.p0 = p0;
    volatile double vp0 = p0;
    t.cot_p0 = std::cos(vp0) / std::sin(vp0);
    t.epsilon = std::numeric_limits<double>::epsilon();
    return CRP_OK;
}

// PolarizedSingleModeMagneticField's constructor (PolarizedSingleModeMagneticField.cpp:5-52):
// its checks in its order, with its messages, and its derived values with Vector3's arithmetic
// (getR = sqrt(x*x + y*y + z*z), cross, componentwise scaling).
crp_status crp_kst24_defaults(crp_kst24_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    // KST24Field::KST24Field (KST24Field.cpp:15-124): the model's published parameters
    crp_kst24_desc &k = *out;
    std::memset(&k, 0, sizeof(k));
    k.north_b = -3.2e-6; k.north_zmin = 1.185; k.north_zmax = 2.1; k.north_rmin = 1.0; k.north_rmax = 9.1;
    k.south_b = 3.2e-6; k.south_zmin = -2.5; k.south_zmax = -1.22; k.south_rmin = 1.0; k.south_rmax = 14.0;
    k.x_b = 1.8e-6; k.x_rmin = 1.0; k.x_rmax = 6.2;
    k.x_theta_rad = 28.0 * M_PI / 180.;
    k.lb_b = -3.5e-6; k.lb_rmin = 0.2; k.lb_dr = 0.03; k.lb_x0 = -8.2; k.lb_y0 = 0.095; k.lb_z0 = -0.05;
    // the constructor's cos and sin run at run time; volatile angles keep them from folding
    volatile double lB = 50.0, bB = 2.0;
    const double l = lB * M_PI / 180, b = bB * M_PI / 180;
    k.lb_dir[0] = std::cos(b) * std::cos(l);
    k.lb_dir[1] = std::cos(b) * std::sin(l);
    k.lb_dir[2] = std::sin(b);
    // b, pitch, phi0, x_shift, y_shift, arc_radius1, arc_radius2, arc_eps, arc_div, rmin, rmax, zmin, zmax
    static const crp_kst24_arm arms[5] = {
        {4.9e-6, 20, -134.0, 1.0, 0.0, 0.8, 1.0, 2.0, 0.0, 3.0, 16.0, -1.0, 1.0},     // Scutum
        {1.3e-6, 20, -80.0, 1.37, 0.0, 1.0, 0.79, 2.3, 3.0, 3.0, 15.0, -1.2, 1.2},    // Carina-Sagittarius
        {-3.5e-6, 20, -2.2, -0.15, 0.0, 0.73, 1.0, 1.45, 0.0, 3.3, 14.0, -1.0, 1.0},  // Local
        {-2.0e-6, 20, 46.0, -1.0, 0.0, 0.4, 1.1, 2.0, 0.0, 3.0, 17.0, -1.0, 1.0},     // Perseus 1
        {-3.5e-6, 20, 46.0, -1.0, 0.0, 1.2, 1.1, 2.0, 0.0, 3.0, 17.0, -2.0, 2.0}};    // Perseus 2
    for (int i = 0; i < 5; i++) k.arms[i] = arms[i];
    // Units.h: kpc = 1e3 parsec, parsec = 648000 / pi au; gauss = 1e-4 tesla
    k.kpc = 1e3 * (648000 / M_PI * 149597870700.0);
    k.gauss = 1e-4;
    return CRP_OK;
}

crp_status crp_cmz_defaults(crp_cmz_desc *out) {
    if (!out) return host_fail(CRP_ERR_INVALID_ARGUMENT, "out is NULL");
    crp_cmz_desc &c = *out;
    std::memset(&c, 0, sizeof(c));
    c.use_ic = 1;  // CMZField::CMZField (CMZField.cpp:6)
    const double pc = 648000 / M_PI * 149597870700.0, gauss = 1e-4;
    volatile double two_v = 2;
    const double ln2 = std::log((double)two_v);
    // getMCField (CMZField.cpp:116-200): centre (y, z) [pc], R [pc], B1, eta
    const double N = 59;
    struct Cloud { double y, z, r, b1, eta; };
    const Cloud clouds[12] = {
        {-81.59, -16.32, 1.7, 2.1e-3 / N, 0.01},  // Sgr C
        {37.53, -2.37, 2.4, 2.5e-3 / N, 0.01},    // Dust Ridge A
        {50.44, 8.16, 1.9, 0.9e-3 / N, 0.01},     // B
        {56.37, 7.71, 1.9, 1.2e-3 / N, 0.01},     // C
        {60.82, 7.42, 3.3, 1.7e-3 / N, 0.01},     // D
        {70.91, 0.74, 3.5, 4.1e-3 / N, 0.01},     // E
        {73.58, 2.97, 2.4, 3.9e-3 / N, 0.01},     // F
        {166.14, -10.38, 1.8, 0.8e-3 / N, 0.01},  // Sgr D
        {97.01, -5.93, 14, 1.0e-3 / N, 0.01},     // Sgr B2
        {-8.3, -6.9, 5, 3.0e-3 / 0.91, 0.77},     // inner 5 pc
        {-19.29, -11.87, 9.4, 2.7e-3 / N, 0.01},  // 20 km/s cloud
        {-2.97, -10.38, 9.4, 3.7e-3 / N, 0.01}};  // 50 km/s cloud
    for (int i = 0; i < 12; i++)
        c.clouds[i] = {{0, clouds[i].y * pc, clouds[i].z * pc}, clouds[i].b1, clouds[i].eta, clouds[i].r * pc};
    c.sgra_shift[0] = 0;
    c.sgra_shift[1] = 8.3 * pc;
    c.sgra_shift[2] = 6.9 * pc;
    c.sgra_r = 1.2e12;
    c.sgra_b1 = 65. / 3.07;
    // getICField (CMZField.cpp:202)
    const double icB1 = 1e-5 * gauss;
    volatile double ic_len = 70 * pc;
    c.ic = {{0., -8.3 * pc, -6.9 * pc}, icB1 / 0.85, 4 * ln2 / std::pow((double)ic_len, 2), 158 * pc / ln2};
    // getNTFField (CMZField.cpp:214-271): centre (y, z) [pc], a1 [m], a2 [m], B1; getA and getL
    struct Filament { double y, z, a1, a2, b1; };
    const double eta = 0.48;
    const Filament f[7] = {
        {-81.59, -1.48, 27.44 * pc, 1.73 * pc, 1.e-4},         // Sgr C
        {-126.1, -25.22, 12.86 * pc, 2.22 * pc, 88.e-6},       // the Snake
        {-68.24, 25.22, 15.08 * pc, 2.72, 1.e-3},              // G359.54+0.18 (a2 as the reference gives it)
        {-31.15, 23.74, 16.07 * pc, 3.46 * pc, 1.e-3},         // G359.79+0.17
        {5.93, 16.32, 28.68 * pc, 1.73 * pc, 1.e-4},           // southern thread
        {13.35, 25.22, 29.42 * pc, 2.23 * pc, 140.e-6},        // northern thread
        {-22.25, 69.73, 11.37 * pc, 2.23 * pc, 70.e-6 / eta}}; // the Pelican
    for (int i = 0; i < 7; i++)
        c.ntf[i] = {{0, f[i].y * pc, f[i].z * pc}, f[i].b1 / eta, 4 * ln2 / f[i].a1 / f[i].a1, f[i].a2 / 2 * ln2};
    // getRadioArcField (CMZField.cpp:273)
    const double a1 = 70.47 * pc, a2 = 9.89 * pc;
    c.radio_arc = {{0, 26.7 * pc, 10.38 * pc}, 1.e-3 / eta, 4 * ln2 / a1 / a1, a2 / 2 * ln2};
    c.gauss = gauss;
    return CRP_OK;
}

crp_status crp_single_mode_field(double b0, double wavelength, double sigma, const double r0[3],
                                 const double e1[3], const double e2[3], int32_t amplitude_rms,
                                 int32_t polarization_helicity, int32_t mode, crp_single_mode_desc *out) {
    if (!out || !r0 || !e1 || !e2) return host_fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    const char *who = "PolarizedSingleModeMagneticField: ";
    auto bad = [&](const char *msg) { return host_fail(CRP_ERR_INVALID_ARGUMENT, (std::string(who) + msg).c_str()); };
    if (mode == CRP_SINGLE_MODE_ELLIPTICAL) {
        if (std::fabs(sigma) > 1)
            return bad("The value of the  polarization parameter has to lie in the range [-1;+1].");
    } else if (mode == CRP_SINGLE_MODE_CIRCULAR) {
        if (std::fabs(sigma) != 1)
            return bad("For circular polarization the value of the polarization parameter has to be equal to -1 or +1.");
    } else if (mode == CRP_SINGLE_MODE_LINEAR) {
        if (std::fabs(sigma) != 0)
            return bad("For linear polarization the value of the polarization parameter has to be equal to 0.");
    } else {
        return bad("Wrong value for flagMode. Please choose \"elliptical\" or \"circular\" or \"linear\".");
    }
    if (e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2] != 0)
        return bad("e_1 and e_2 have to be orthogonal to each other.");
    const double r1 = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    if (r1 == 0) return bad("Vector e_1 cannot be zero.");
    const double r2 = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    if (r2 == 0) return bad("Vector e_2 cannot be zero.");
    crp_single_mode_desc &d = *out;
    std::memset(&d, 0, sizeof(d));
    for (int a = 0; a < 3; a++) {
        d.u1[a] = e1[a] / r1;
        d.u2[a] = e2[a] / r2;
        d.r0[a] = r0[a];
    }
    // e_2 x e_1, normalised, times 2 pi / wavelength
    double k[3] = {e2[1] * e1[2] - e1[1] * e2[2], e2[2] * e1[0] - e1[2] * e2[0], e2[0] * e1[1] - e1[0] * e2[1]};
    const double rk = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    for (int a = 0; a < 3; a++) k[a] = k[a] / rk;
    if (wavelength == 0) return bad("The correlation length cannot be zero.");
    for (int a = 0; a < 3; a++) d.k[a] = k[a] * 2 * M_PI / wavelength;
    if (polarization_helicity != CRP_SINGLE_MODE_POLARIZATION && polarization_helicity != CRP_SINGLE_MODE_HELICITY)
        return bad("Wrong value for flagPolarizationHelicity. Please choose \"polarization\" or \"helicity\".");
    if (polarization_helicity == CRP_SINGLE_MODE_HELICITY && std::fabs(sigma) != 1)
        return bad("In helicity mode only the maximum helicity case (sigma = +1 or sigma = -1) may be chosen.");
    if (amplitude_rms == CRP_SINGLE_MODE_AMPLITUDE) {
        d.b_max = b0;
    } else if (amplitude_rms == CRP_SINGLE_MODE_RMS) {
        volatile double q = 2 / (1 + sigma * sigma);
        d.b_max = std::sqrt(q) * b0;
    } else {
        return bad("Wrong value for flagAmplitudeRms. Please choose \"amplitude\" or \"rms\".");
    }
    d.sigma = sigma;
    d.b0 = b0;
    d.wavelength = wavelength;
    for (int a = 0; a < 3; a++) { d.e1[a] = e1[a]; d.e2[a] = e2[a]; }
    d.amplitude_rms = amplitude_rms;
    d.polarization_helicity = polarization_helicity;
    d.mode = mode;
    return CRP_OK;
}

crp_status crp_pt11_use(crp_pt11_desc *io, int32_t which, int32_t use) {
    if (!io) return host_fail(CRP_ERR_INVALID_ARGUMENT, "io is NULL");
    const double muG = 1e-6 * 1e-4;
    crp_pt11_desc &p = *io;
    if (which == CRP_PT11_HALO) {  // setUseHalo (PT11Field.cpp:66)
        p.use_halo = use ? 1 : 0;
        return CRP_OK;
    }
    if (which != CRP_PT11_ASS && which != CRP_PT11_BSS) return host_fail(CRP_ERR_INVALID_ARGUMENT, "unknown PT11 switch");
    const bool ass = which == CRP_PT11_ASS;
    (ass ? p.use_ass : p.use_bss) = use ? 1 : 0;
    if (!use) return CRP_OK;
    (ass ? p.use_bss : p.use_ass) = 0;  // setUseASS (PT11Field.cpp:35) / setUseBSS (:50)
    p.pitch = (ass ? -5.0 : -6.0) * M_PI / 180;
    p.b0_hs = (ass ? 2.0 : 4.0) * muG;
    pt11_set_params(p);
    return CRP_OK;
}

crp_status crp_plane_wave_modes(double brms, double lmin, double lmax, double lbendover,
                                double sindex, double qindex, int32_t nm, int32_t seed,
                                double *xi, double *kappa, double *k, double *beta, double *ak) {
    if (nm <= 1)
        return host_fail(CRP_ERR_INVALID_ARGUMENT,
                         "PlaneWaveTurbulence: Nm <= 1. Specify at least two wavemodes in order to generate the k distribution properly.");
    if (lmin > lmax) return host_fail(CRP_ERR_INVALID_ARGUMENT, "TurbulenceSpectrum: lMin > lMax");
    if (lmin <= 0) return host_fail(CRP_ERR_INVALID_ARGUMENT, "TurbulenceSpectrum: lMin <= 0");
    if (!xi || !kappa || !k || !beta || !ak) return host_fail(CRP_ERR_INVALID_ARGUMENT, "NULL mode array");
    if (seed == 0)
        return host_fail(CRP_ERR_INVALID_ARGUMENT,
                         "PlaneWaveTurbulence: seed 0 draws from /dev/urandom; give a non-zero seed");
    Mt r((uint32_t)seed);
    const double kmax = 2 * M_PI / lmin, kmin = 2 * M_PI / lmax;
    const double delta = std::log10(kmax / kmin);
    for (int i = 0; i < nm; i++)
        k[i] = std::pow(10, std::log10(kmin) + ((double)i) / ((double)(nm - 1)) * delta);
    const double delta_k0 = (k[1] - k[0]) / k[1];
    double sum = 0;
    for (int i = 0; i < nm; i++) {
        double kk = k[i];
        double kHat = kk * lbendover;
        // TurbulenceSpectrum::energySpectrum (TurbulentField.h:75)
        double es = std::pow(kHat, qindex) / std::pow(1.0 + kHat * kHat, (sindex + qindex) / 2.0 + 1.0);
        double Gk = es * (1 + kHat * kHat);
        ak[i] = Gk * delta_k0 * kk;
        sum += ak[i];
        double phi = r.uniform(-M_PI, M_PI);
        double costheta = r.uniform(-1., 1.);
        double sintheta = std::sqrt(1 - costheta * costheta);
        double alpha = r.uniform(0, 2 * M_PI);
        double b = r.uniform(0, 2 * M_PI);
        kappa[3 * i] = sintheta * std::cos(phi);
        kappa[3 * i + 1] = sintheta * std::sin(phi);
        kappa[3 * i + 2] = costheta;
        xi[3 * i] = costheta * std::cos(phi) * std::cos(alpha) + std::sin(phi) * std::sin(alpha);
        xi[3 * i + 1] = costheta * std::sin(phi) * std::cos(alpha) - std::cos(phi) * std::sin(alpha);
        xi[3 * i + 2] = -sintheta * std::cos(alpha);
        beta[i] = b;
    }
    for (int i = 0; i < nm; i++) ak[i] = std::sqrt(2 * ak[i] / sum) * brms;
    return CRP_OK;
}

crp_status crp_source_sample(const crp_source_desc *src, uint32_t seed, uint64_t n, int32_t *id,
                             double *energy, double *dir_xyz) {
    if (!src || (n && (!id || !energy || !dir_xyz)))
        return host_fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    if (src->n_types < 1 || src->n_types > 256 || !src->ids)
        return host_fail(CRP_ERR_INVALID_ARGUMENT, "SourceMultipleParticleTypes: no nuclei set");
    if (src->spectrum && ((src->emin < 0) || (src->emax < src->emin)))
        return host_fail(CRP_ERR_INVALID_ARGUMENT, "Power law distribution only possible for 0 <= min <= max");
    std::vector<double> cdf((size_t)src->n_types);
    double acc = 0;
    for (int i = 0; i < src->n_types; i++) {
        acc = (i ? cdf[i - 1] : 0) + (src->abundances ? src->abundances[i] : 1.0);
        cdf[i] = acc;
    }
    Mt r(seed);
    for (uint64_t i = 0; i < n; i++) {
        int32_t pid = src->ids[0];
        if (src->n_types > 1) {  // Random::randBin: lower_bound over the CDF
            double u = r.rand() * cdf.back();
            int k = 0;
            while (k < src->n_types && cdf[k] < u) k++;
            pid = src->ids[k];
        }
        id[i] = pid;
        energy[i] = src->spectrum ? r.power_law(src->index, src->emin, src->emax) : src->energy;
        double x, y, z;
        if (src->isotropic) r.vector(x, y, z);
        else { x = src->direction[0]; y = src->direction[1]; z = src->direction[2]; }
        double nrm = std::sqrt(x * x + y * y + z * z);  // ParticleState::setDirection
        dir_xyz[i] = x / nrm; dir_xyz[n + i] = y / nrm; dir_xyz[2 * n + i] = z / nrm;
    }
    return CRP_OK;
}

// TextOutput line (TextOutput.cpp:166-292): the enabled columns of the
// Output column bitset in the reference's order and printf formats.
static void format_row(const crp_output_desc *d, const crp_output_rows *r, uint64_t i,
                       std::string &out) {
    char buf[2048];
    size_t p = 0;
    const uint32_t f = d->columns;
    auto on = [&](int c) { return (f >> c) & 1u; };
    auto put = [&](const char *fmt, double v) { p += snprintf(buf + p, sizeof(buf) - p, fmt, v); };
    auto put3 = [&](const double *v, double s) {
        p += snprintf(buf + p, sizeof(buf) - p, "%8.5E\t%8.5E\t%8.5E\t", v[3 * i] / s, v[3 * i + 1] / s, v[3 * i + 2] / s);
    };
    auto putu = [&](uint64_t v) { p += snprintf(buf + p, sizeof(buf) - p, "%10" PRIu64 "\t", v); };
    auto puti = [&](int v) { p += snprintf(buf + p, sizeof(buf) - p, "%10i\t", v); };
    const bool d1 = d->one_dimensional != 0;
    if (on(CRP_COL_TRAJECTORY_LENGTH)) put("%8.5E\t", r->trajectory_length[i] / d->length_scale);
    if (on(CRP_COL_TIME)) put("%8.5E\t", r->time[i] / d->time_scale);
    if (on(CRP_COL_REDSHIFT)) put("%1.5E\t", 0.0);
    if (on(CRP_COL_SERIAL_NUMBER)) putu(r->serial ? r->serial[i] : 0);
    if (on(CRP_COL_CURRENT_ID)) puti(r->id[i]);
    if (on(CRP_COL_CURRENT_ENERGY)) put("%8.5E\t", r->energy[i] / d->energy_scale);
    if (on(CRP_COL_CURRENT_POSITION)) {
        if (d1) put("%8.5E\t", r->position[3 * i] / d->length_scale);
        else put3(r->position, d->length_scale);
    }
    if (on(CRP_COL_CURRENT_DIRECTION) && !d1) put3(r->direction, 1.0);
    // primaries: source and created serial numbers are the candidate's own (Candidate.cpp:240-252)
    if (on(CRP_COL_SERIAL_NUMBER)) putu(r->serial ? r->serial[i] : 0);
    if (on(CRP_COL_SOURCE_ID)) puti(r->source_id[i]);
    if (on(CRP_COL_SOURCE_ENERGY)) put("%8.5E\t", r->source_energy[i] / d->energy_scale);
    if (on(CRP_COL_SOURCE_POSITION)) {
        if (d1) put("%8.5E\t", r->source_position[3 * i] / d->length_scale);
        else put3(r->source_position, d->length_scale);
    }
    if (on(CRP_COL_SOURCE_DIRECTION) && !d1) put3(r->source_direction, 1.0);
    if (on(CRP_COL_SERIAL_NUMBER)) putu(r->serial ? r->serial[i] : 0);
    if (on(CRP_COL_CREATED_ID)) puti(r->source_id[i]);
    if (on(CRP_COL_CREATED_ENERGY)) put("%8.5E\t", r->source_energy[i] / d->energy_scale);
    if (on(CRP_COL_CREATED_POSITION)) {
        if (d1) put("%8.5E\t", r->source_position[3 * i] / d->length_scale);
        else put3(r->source_position, d->length_scale);
    }
    if (on(CRP_COL_CREATED_DIRECTION) && !d1) put3(r->source_direction, 1.0);
    if (on(CRP_COL_WEIGHT)) put("%8.5E\t", r->weight ? r->weight[i] : 1.0);
    if (on(CRP_COL_CANDIDATE_TAG)) p += snprintf(buf + p, sizeof(buf) - p, "%s\t", "PRIM");
    if (p == 0) return;
    buf[p - 1] = '\n';
    out.append(buf, p);
}

// TextOutput::printHeader (TextOutput.cpp:55)
static void format_header(const crp_output_desc *d, std::string &o) {
    const uint32_t f = d->columns;
    auto on = [&](int c) { return (f >> c) & 1u; };
    const bool d1 = d->one_dimensional != 0;
    char buf[256];
    o += "#";
    if (on(CRP_COL_TRAJECTORY_LENGTH)) o += "\tD";
    if (on(CRP_COL_TIME)) o += "\ttime";
    if (on(CRP_COL_REDSHIFT)) o += "\tz";
    if (on(CRP_COL_SERIAL_NUMBER)) o += "\tSN";
    if (on(CRP_COL_CURRENT_ID)) o += "\tID";
    if (on(CRP_COL_CURRENT_ENERGY)) o += "\tE";
    if (on(CRP_COL_CURRENT_POSITION) && d1) o += "\tX";
    if (on(CRP_COL_CURRENT_POSITION) && !d1) o += "\tX\tY\tZ";
    if (on(CRP_COL_CURRENT_DIRECTION) && !d1) o += "\tPx\tPy\tPz";
    if (on(CRP_COL_SERIAL_NUMBER)) o += "\tSN0";
    if (on(CRP_COL_SOURCE_ID)) o += "\tID0";
    if (on(CRP_COL_SOURCE_ENERGY)) o += "\tE0";
    if (on(CRP_COL_SOURCE_POSITION) && d1) o += "\tX0";
    if (on(CRP_COL_SOURCE_POSITION) && !d1) o += "\tX0\tY0\tZ0";
    if (on(CRP_COL_SOURCE_DIRECTION) && !d1) o += "\tP0x\tP0y\tP0z";
    if (on(CRP_COL_SERIAL_NUMBER)) o += "\tSN1";
    if (on(CRP_COL_CREATED_ID)) o += "\tID1";
    if (on(CRP_COL_CREATED_ENERGY)) o += "\tE1";
    if (on(CRP_COL_CREATED_POSITION) && d1) o += "\tX1";
    if (on(CRP_COL_CREATED_POSITION) && !d1) o += "\tX1\tY1\tZ1";
    if (on(CRP_COL_CREATED_DIRECTION) && !d1) o += "\tP1x\tP1y\tP1z";
    if (on(CRP_COL_WEIGHT)) o += "\tW";
    if (on(CRP_COL_CANDIDATE_TAG)) o += "\ttag";
    o += "\n#\n";
    // the stream prints the scale ratios with the default ostream precision (6 significant digits)
    if (on(CRP_COL_TRAJECTORY_LENGTH)) {
        snprintf(buf, sizeof(buf), "# D             Trajectory length [%g Mpc]\n", d->length_scale / 3.0856775814913673e22);
        o += buf;
    }
    if (on(CRP_COL_TIME)) {
        snprintf(buf, sizeof(buf), "# time          Time [%g Myr]\n", d->time_scale / (1e6 * 365.25 * 24 * 3600));
        o += buf;
    }
    if (on(CRP_COL_REDSHIFT)) o += "# z             Redshift\n";
    if (on(CRP_COL_SERIAL_NUMBER)) o += "# SN/SN0/SN1    Serial number. Unique (within this run) id of the particle.\n";
    if (on(CRP_COL_CURRENT_ID) || on(CRP_COL_CREATED_ID) || on(CRP_COL_SOURCE_ID))
        o += "# ID/ID0/ID1    Particle type (PDG MC numbering scheme)\n";
    if (on(CRP_COL_CURRENT_ENERGY) || on(CRP_COL_CREATED_ENERGY) || on(CRP_COL_SOURCE_ENERGY)) {
        snprintf(buf, sizeof(buf), "# E/E0/E1       Energy [%g EeV]\n", d->energy_scale / (1e18 * 1.602176487e-19));
        o += buf;
    }
    if (on(CRP_COL_CURRENT_POSITION) || on(CRP_COL_CREATED_POSITION) || on(CRP_COL_SOURCE_POSITION)) {
        snprintf(buf, sizeof(buf), "# X/X0/X1...    Position [%g Mpc]\n", d->length_scale / 3.0856775814913673e22);
        o += buf;
    }
    if (on(CRP_COL_CURRENT_DIRECTION) || on(CRP_COL_CREATED_DIRECTION) || on(CRP_COL_SOURCE_DIRECTION))
        o += "# Px/P0x/P1x... Heading (unit vector of momentum)\n";
    if (on(CRP_COL_WEIGHT)) o += "# W             Weights \n";
    o += "# no index = current, 0 = at source, 1 = at point of creation\n#\n";
    o += "# CRPropa version: ";
    o += d->version ? d->version : "";
    o += "\n#\n";
}

crp_status crp_text_output_write(const char *path, int32_t append, int32_t header,
                                 const crp_output_desc *desc, uint64_t n,
                                 const crp_output_rows *rows) {
    if (!path || !desc || (n && !rows)) return host_fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    // a name ending in ".gz" writes gzip (TextOutput.cpp:41, :388: zstream over zlib); appending
    // adds a gzip member, which readers concatenate
    const size_t len = std::strlen(path);
    const bool gz = len >= 3 && std::strcmp(path + len - 3, ".gz") == 0;
    FILE *f = nullptr;
    gzFile g = nullptr;
    if (gz) g = gzopen(path, append ? "ab" : "wb");
    else f = fopen(path, append ? "ab" : "wb");
    if (!f && !g) return host_fail(CRP_ERR_INVALID_ARGUMENT, "Cannot create file");
    bool ok = true;
    auto flush = [&](const std::string &o) {
        if (o.empty()) return;
        if (gz) ok = ok && gzwrite(g, o.data(), (unsigned)o.size()) == (int)o.size();
        else ok = ok && fwrite(o.data(), 1, o.size(), f) == o.size();
    };
    std::string out;
    out.reserve(256 * (size_t)(n < 4096 ? n + 1 : 4096));
    if (header) format_header(desc, out);
    for (uint64_t i = 0; i < n; i++) {
        format_row(desc, rows, i, out);
        if (out.size() > (1u << 22)) {
            flush(out);
            out.clear();
        }
    }
    flush(out);
    if (gz) ok = gzclose(g) == Z_OK && ok;
    else ok = fclose(f) == 0 && ok;
    if (!ok) return host_fail(CRP_ERR_INVALID_ARGUMENT, "write to the output file failed");
    return CRP_OK;
}

}  // extern "C"
