/*
 * crp_oracle.c -- TEST INFRASTRUCTURE: the oracle.
 *
 * A plain-C restatement of CRPropa3's charged-particle stepping path, used
 * only as the checker of the CUDA path (by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg).  The product
 * never links, loads or calls it.
 *
 * Every function follows the reference operation for operation, so that the
 * FP64 device path can be compared bit for bit where the reference uses only
 * + - * / sqrt floor (Boris push over a Grid3f).  Build without FMA
 * contraction (-ffp-contract=off) and without -ffast-math.  Citations are to
 * files of the reference project (CRPropa3).
 *
 * Pinned against the reference itself: tests/test_oracle_vs_reference.py
 * runs this oracle and the reference compiled from its sources
 * (oracle/Makefile) on the same inputs, and tests/golden/ holds vectors
 * generated from the reference by tests/golden/make_golden.py.
 *
 * Randomness: crpropa::Random (MT19937, src/Random.cpp) is restated for the
 * host-side draws (source sampling, PlaneWaveTurbulence and GridTurbulence
 * set-up).  DiffusionSDE here draws from Philox4x32-10 (Salmon et al.,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed by the run seed
 * with counter (step, candidate), exactly as the device does, and transforms
 * the 32-bit words the way Random::randNorm / randUniform / randVector /
 * randConeVector do (src/Random.cpp:104-166); the reference's own MT stream
 * is compared with it only in distribution.
 */
#include "crp_gpu.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* The step controllers' and DiffusionSDE's pow (PropagationCK.cpp:116,
 * PropagationBP.cpp:104, DiffusionSDE.cpp:263).  The default build calls
 * glibc's pow, as the reference does.  The build with
 * -DORACLE_POW=oracle_cr_pow calls a correctly rounded pow instead (crpow.cpp),
 * to separate last-place differences of pow implementations from every other
 * operation when the device's FP64 form is compared with this oracle. */
#ifndef ORACLE_POW
#define ORACLE_POW pow
#else
double ORACLE_POW(double, double);
#endif

/* include/crpropa/Units.h:54-55, :114-115 */
static const double c_light = 2.99792458e8;
static const double kpc_unit = 1e3 * (648000 / M_PI * 149597870700.0);

/* ------------------------------------------------------------------------
 * Vector3d (include/crpropa/Vector3.h)
 * ---------------------------------------------------------------------- */
typedef struct { double x, y, z; } v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 muls(v3 a, double f) { return mk(a.x * f, a.y * f, a.z * f); }  /* :305 */
static inline v3 divs(v3 a, double f) { return mk(a.x / f, a.y / f, a.z / f); }  /* :317 */
static inline v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 divv(v3 a, v3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; } /* :259 */
static inline v3 cross(v3 a, v3 v) {  /* :264 */
    return mk(a.y * v.z - v.y * a.z, a.z * v.x - v.z * a.x, a.x * v.y - v.x * a.y);
}
static inline double norm(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); } /* :127 */
static inline v3 unit(v3 a) { return divs(a, norm(a)); }                           /* :157 */
static inline v3 vfloor(v3 a) { return mk(floor(a.x), floor(a.y), floor(a.z)); }
static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double clipd(double x, double lo, double hi) { return dmax(lo, dmin(x, hi)); } /* Common.h:30 */

/* ------------------------------------------------------------------------
 * MT19937 as crpropa::Random (src/Random.cpp)
 * ---------------------------------------------------------------------- */
typedef struct { uint32_t state[624]; int left; int next; } mt_t;

static uint32_t mt_twist(uint32_t m, uint32_t s0, uint32_t s1) {
    uint32_t y = (s0 & 0x80000000u) | (s1 & 0x7fffffffu);
    return m ^ (y >> 1) ^ ((uint32_t)(-(int32_t)(s1 & 1u)) & 0x9908b0dfu);
}

static void mt_reload(mt_t *r) { /* Random.cpp:379 */
    uint32_t *s = r->state;
    int i;
    for (i = 0; i < 624 - 397; i++) s[i] = mt_twist(s[i + 397], s[i], s[i + 1]);
    for (; i < 623; i++) s[i] = mt_twist(s[i + 397 - 624], s[i], s[i + 1]);
    s[623] = mt_twist(s[396], s[623], s[0]);
    r->left = 624;
    r->next = 0;
}

void oracle_mt_seed(mt_t *r, uint32_t seed) { /* Random.cpp:306, :367 */
    r->state[0] = seed;
    for (int i = 1; i < 624; i++)
        r->state[i] = 1812433253u * (r->state[i - 1] ^ (r->state[i - 1] >> 30)) + (uint32_t)i;
    mt_reload(r);
}

static uint32_t mt_int(mt_t *r) { /* Random.cpp:248 */
    if (r->left == 0) mt_reload(r);
    --r->left;
    uint32_t s1 = r->state[r->next++];
    s1 ^= (s1 >> 11);
    s1 ^= (s1 << 7) & 0x9d2c5680u;
    s1 ^= (s1 << 15) & 0xefc60000u;
    return s1 ^ (s1 >> 18);
}

static double mt_rand(mt_t *r) { return (double)mt_int(r) * (1.0 / 4294967295.0); } /* :75 */
static double mt_uniform(mt_t *r, double a, double b) { return a + (b - a) * mt_rand(r); } /* :117 */

static v3 mt_vector(mt_t *r) { /* Random.cpp:141 */
    double z = mt_uniform(r, -1.0, 1.0);
    double t = mt_uniform(r, -1.0 * M_PI, M_PI);
    double rr = sqrt(1 - z * z);
    return mk(rr * cos(t), rr * sin(t), z);
}

static double mt_power_law(mt_t *r, double index, double mn, double mx) { /* :189 */
    if (fabs(index + 1.0) < 2.220446049250313e-16) {
        double p1 = log(mx), p2 = log(mn);
        return exp((p1 - p2) * mt_rand(r) + p2);
    }
    double p1 = pow(mx, index + 1), p2 = pow(mn, index + 1);
    double ex = 1 / (index + 1);
    return pow((p1 - p2) * mt_rand(r) + p2, ex);
}

size_t oracle_mt_size(void) { return sizeof(mt_t); }

/* Draw n values the way ref_shim's ref_random() does (same kinds). */
int oracle_random(uint32_t seed, int kind, uint64_t n, double a, double b, double c, double *out) {
    mt_t r;
    oracle_mt_seed(&r, seed);
    for (uint64_t i = 0; i < n; i++) {
        if (kind == 0) out[i] = mt_rand(&r);
        else if (kind == 1) out[i] = mt_uniform(&r, a, b);
        else if (kind == 2) { v3 v = mt_vector(&r); out[3*i] = v.x; out[3*i+1] = v.y; out[3*i+2] = v.z; }
        else if (kind == 3) out[i] = mt_power_law(&r, a, b, c);
        else if (kind == 6) out[i] = (double)mt_int(&r);
        else return 1;
    }
    return 0;
}

/* Source of the stepping workloads (Source.cpp:22): SourcePosition,
 * SourceParticleType / SourceMultipleParticleTypes (randBin over the
 * abundance CDF, Random.cpp:128), SourcePowerLawSpectrum, SourceIsotropicEmission,
 * drawn in that order from one MT19937 stream. */
int oracle_sample_source(uint32_t seed, uint64_t n, int ntypes, const int32_t *ids,
                         const double *abundances, double emin, double emax, double index,
                         int32_t *id_out, double *e_out, double *dir_out) {
    mt_t r;
    oracle_mt_seed(&r, seed);
    double cdf[64];
    if (ntypes < 1 || ntypes > 64) return 1;
    double acc = 0;
    for (int i = 0; i < ntypes; i++) { acc = (i ? cdf[i - 1] : 0) + abundances[i]; cdf[i] = acc; }
    for (uint64_t i = 0; i < n; i++) {
        int32_t id = ids[0];
        if (ntypes > 1) {
            double u = mt_rand(&r) * cdf[ntypes - 1];
            int k = 0;
            while (k < ntypes && cdf[k] < u) k++;  /* std::lower_bound */
            id = ids[k];
        }
        id_out[i] = id;
        e_out[i] = mt_power_law(&r, index, emin, emax);
        v3 d = mt_vector(&r);
        d = divs(d, norm(d)); /* ParticleState::setDirection */
        dir_out[3*i] = d.x; dir_out[3*i+1] = d.y; dir_out[3*i+2] = d.z;
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Philox4x32-10 (published algorithm) and the reference's transforms
 * ---------------------------------------------------------------------- */
typedef struct { uint32_t v[4]; } u32x4;

u32x4 oracle_philox(u32x4 ctr, uint32_t k0, uint32_t k1) {
    for (int round = 0; round < 10; round++) {
        if (round) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr.v[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr.v[2];
        u32x4 o;
        o.v[0] = (uint32_t)(p1 >> 32) ^ ctr.v[1] ^ k0;
        o.v[1] = (uint32_t)p1;
        o.v[2] = (uint32_t)(p0 >> 32) ^ ctr.v[3] ^ k1;
        o.v[3] = (uint32_t)p0;
        ctr = o;
    }
    return ctr;
}

void oracle_philox_block(const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
    u32x4 c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    u32x4 o = oracle_philox(c, key[0], key[1]);
    memcpy(out, o.v, sizeof(o.v));
}

/* The source features of oracle_sample_source (Source.cpp:74-150, :742, :808)
 * drawn from the counter-based stream of the device sampler: candidate c's
 * words are those of Philox({lo(c), hi(c), 0x536f7572 + block, 0}, seed),
 * each uniform 53 bits of two words; Random::randBin, randPowerLaw and
 * randVector map them as the reference maps its MT19937 draws. */
static double philox_uniform53(uint32_t hi, uint32_t lo) {
    return (double)(((uint64_t)hi << 21) | (uint64_t)(lo >> 11)) * 0x1.0p-53;
}

int oracle_sample_source_philox(uint64_t seed, uint64_t first, uint64_t n, int ntypes, const int32_t *ids,
                                const double *abundances, int spectrum, double emin, double emax, double index,
                                double energy, int isotropic, const double *direction, int32_t *id_out,
                                double *e_out, double *dir_out) {
    double cdf[256];
    if (ntypes < 1 || ntypes > 256) return 1;
    double acc = 0;
    for (int i = 0; i < ntypes; i++) { acc = acc + (abundances ? abundances[i] : 1.0); cdf[i] = acc; }
    int log_uniform = fabs(index + 1.0) < 2.220446049250313e-16;
    double p1 = log_uniform ? log(emax) : pow(emax, index + 1), p2 = log_uniform ? log(emin) : pow(emin, index + 1);
    double ex = 1 / (index + 1);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t c = first + i;
        u32x4 ca = {{(uint32_t)c, (uint32_t)(c >> 32), 0x536f7572u, 0u}};
        u32x4 cb = {{(uint32_t)c, (uint32_t)(c >> 32), 0x536f7573u, 0u}};
        u32x4 a = oracle_philox(ca, (uint32_t)seed, (uint32_t)(seed >> 32));
        u32x4 b = oracle_philox(cb, (uint32_t)seed, (uint32_t)(seed >> 32));
        int32_t pid = ids[0];
        if (ntypes > 1) {
            double u = philox_uniform53(a.v[0], a.v[1]) * cdf[ntypes - 1];
            int k = 0;
            while (k < ntypes - 1 && cdf[k] < u) k++;
            pid = ids[k];
        }
        id_out[i] = pid;
        double e = energy;
        if (spectrum) {
            double u = philox_uniform53(a.v[2], a.v[3]);
            e = log_uniform ? exp((p1 - p2) * u + p2) : pow((p1 - p2) * u + p2, ex);
        }
        e_out[i] = e;
        double x = direction[0], y = direction[1], z = direction[2];
        if (isotropic) {
            z = -1.0 + 2.0 * philox_uniform53(b.v[0], b.v[1]);
            double t = -M_PI + (M_PI - -M_PI) * philox_uniform53(b.v[2], b.v[3]);
            double r = sqrt(1 - z * z);
            x = r * cos(t);
            y = r * sin(t);
        }
        double nrm = sqrt(x * x + y * y + z * z);
        dir_out[i] = x / nrm;
        dir_out[n + i] = y / nrm;
        dir_out[2 * n + i] = z / nrm;
    }
    return 0;
}

/* Per-step stream of a candidate: word w of step s of candidate i is word
 * (w % 4) of Philox(ctr = {lo(4s + w/4), hi(4s + w/4), lo(i), hi(i)},
 * key = {lo(seed), hi(seed)}). */
typedef struct {
    uint64_t seed, cand, step;
    u32x4 block;
    int cursor;
} stream_t;

static uint32_t stream_int(stream_t *s) {
    int w = s->cursor++;
    if ((w & 3) == 0) {
        uint64_t c = s->step * 4 + (uint64_t)(w >> 2);
        u32x4 ctr = {{(uint32_t)c, (uint32_t)(c >> 32), (uint32_t)s->cand, (uint32_t)(s->cand >> 32)}};
        s->block = oracle_philox(ctr, (uint32_t)s->seed, (uint32_t)(s->seed >> 32));
    }
    return s->block.v[w & 3];
}
static double stream_rand(stream_t *s) { return (double)stream_int(s) * (1.0 / 4294967295.0); }
static double stream_uniform(stream_t *s, double a, double b) { return a + (b - a) * stream_rand(s); }
static double stream_norm(stream_t *s) { /* Random.cpp:104 randNorm(0, 1) */
    double dblexc = ((double)stream_int(s) + 0.5) * (1.0 / 4294967296.0);
    double r = sqrt(-2.0 * log(1.0 - dblexc)) * 1.0;
    double phi = 2.0 * 3.14159265358979323846264338328 * ((double)stream_int(s) * (1.0 / 4294967296.0));
    return 0.0 + r * cos(phi);
}
static v3 stream_vector(stream_t *s) { /* Random.cpp:141 */
    double z = stream_uniform(s, -1.0, 1.0);
    double t = stream_uniform(s, -1.0 * M_PI, M_PI);
    double r = sqrt(1 - z * z);
    return mk(r * cos(t), r * sin(t), z);
}
static v3 rotated(v3 v, v3 axis, double angle) { /* Vector3.h:206 getRotated */
    v3 u = axis;
    if (norm(u) != 0.) u = divs(u, norm(u));
    double c = cos(angle), s = sin(angle);
    v3 Rx = mk(c + u.x * u.x * (1 - c), u.x * u.y * (1 - c) - u.z * s, u.x * u.z * (1 - c) + u.y * s);
    v3 Ry = mk(u.y * u.x * (1 - c) + u.z * s, c + u.y * u.y * (1 - c), u.y * u.z * (1 - c) - u.x * s);
    v3 Rz = mk(u.z * u.x * (1 - c) - u.y * s, u.z * u.y * (1 - c) + u.x * s, c + u.z * u.z * (1 - c));
    return mk(dot(v, Rx), dot(v, Ry), dot(v, Rz));
}
static v3 stream_cone(stream_t *s, v3 mean, double radius) { /* Random.cpp:159, :147 */
    double theta = acos(stream_uniform(s, 1, cos(radius)));
    v3 axis = cross(mean, stream_vector(s));
    return rotated(mean, axis, theta);
}

/* ------------------------------------------------------------------------
 * Fields
 * ---------------------------------------------------------------------- */

/* Grid<Vector3f>::interpolate / trilinearInterpolate (Grid.h:318, :540),
 * values and weights in float as Vector3f * double converts the weight to
 * float (Vector3.h:305). */
/* periodicBoundary / reflectiveBoundary of a cell index (Grid.h:37-46) and
 * the symmetrical round (Grid.h:61). */
static int periodic_boundary(int i, int n) { return ((i % n) + n) % n; }
static int reflective_boundary(int i, int n) {
    while ((i < -0.5) || (i > (n - 0.5))) i = 2 * n * (i > (n - 0.5)) - i - 1;
    return i;
}
static double sym_round(double r) { return (r > 0.0) ? floor(r + 0.5) : ceil(r - 0.5); }

static size_t grid_cell(const crp_grid3f_desc *g, int ix, int iy, int iz) {
    return ((size_t)ix * (size_t)g->ny + (size_t)iy) * (size_t)g->nz + (size_t)iz;
}
static size_t grid_cell_bc(const crp_grid3f_desc *g, int ix, int iy, int iz) {
    int nx = (int)g->nx, ny = (int)g->ny, nz = (int)g->nz;
    if (g->reflective)
        return grid_cell(g, reflective_boundary(ix, nx), reflective_boundary(iy, ny), reflective_boundary(iz, nz));
    return grid_cell(g, periodic_boundary(ix, nx), periodic_boundary(iy, ny), periodic_boundary(iz, nz));
}

/* clipVolume test of Grid::interpolate (Grid.h:319). */
static int grid_in_volume(const crp_grid3f_desc *g, v3 pos) {
    v3 origin = mk(g->origin[0], g->origin[1], g->origin[2]);
    v3 spacing = mk(g->spacing[0], g->spacing[1], g->spacing[2]);
    v3 edge = add(origin, mulv(mk((double)g->nx, (double)g->ny, (double)g->nz), spacing));
    int in = (pos.x >= origin.x) && (pos.x <= edge.x);
    in &= (pos.y >= origin.y) && (pos.y <= edge.y);
    in &= (pos.z >= origin.z) && (pos.z <= edge.z);
    return in;
}

/* r = (position - gridOrigin) / spacing, gridOrigin = origin + spacing / 2 (Grid.h:227). */
static v3 grid_unit(const crp_grid3f_desc *g, v3 pos) {
    v3 origin = mk(g->origin[0], g->origin[1], g->origin[2]);
    v3 spacing = mk(g->spacing[0], g->spacing[1], g->spacing[2]);
    return divv(sub(pos, add(origin, divs(spacing, 2))), spacing);
}

/* CubicInterpolate, SIMD form (Grid.h:435), one lane: float arithmetic,
 * pos^2 and pos^3 formed in double. */
static float cubic_f(float p0, float p1, float p2, float p3, double position) {
    const float c1 = 0.5f, c2 = 1.5f, c3 = 2.f, c4 = 2.5f;
    float pos = (float)position, pos2 = (float)(position * position),
          pos3 = (float)(position * position * position);
    float term = (c1 * p2 - c1 * p0) * pos;
    float term2 = ((p0 + c3 * p2) - (c4 * p1 + c1 * p3)) * pos2;
    float term3 = ((c2 * p1 + c1 * p3) - (c1 * p0 + c2 * p2)) * pos3;
    return ((term3 + term2) + term) + p1;
}

/* Grid<Vector3f>::tricubicInterpolate, SIMD form (Grid.h:459). */
static v3 grid_tricubic3(const crp_grid3f_desc *g, v3 pos) {
    v3 r = grid_unit(g, pos);
    int ix0 = (int)floor(r.x), iy0 = (int)floor(r.y), iz0 = (int)floor(r.z);
    double fx = r.x - ix0, fy = r.y - iy0, fz = r.z - iz0;
    float vx[4][3], vy[4][3], vz[4][3];
    for (int a = -1; a < 3; a++) {
        for (int b = -1; b < 3; b++) {
            for (int c = -1; c < 3; c++) {
                const float *v = g->values + 3 * grid_cell_bc(g, ix0 + a, iy0 + b, iz0 + c);
                vz[c + 1][0] = v[0]; vz[c + 1][1] = v[1]; vz[c + 1][2] = v[2];
            }
            for (int k = 0; k < 3; k++) vy[b + 1][k] = cubic_f(vz[0][k], vz[1][k], vz[2][k], vz[3][k], fz);
        }
        for (int k = 0; k < 3; k++) vx[a + 1][k] = cubic_f(vy[0][k], vy[1][k], vy[2][k], vy[3][k], fy);
    }
    float res[3];
    for (int k = 0; k < 3; k++) res[k] = cubic_f(vx[0][k], vx[1][k], vx[2][k], vx[3][k], fx);
    return mk(res[0], res[1], res[2]);
}

/* Grid::closestValue (Grid.h:383): cell of the nearest grid point. */
static size_t grid_nearest_cell(const crp_grid3f_desc *g, v3 pos) {
    v3 r = grid_unit(g, pos);
    int nx = (int)g->nx, ny = (int)g->ny, nz = (int)g->nz;
    int ix, iy, iz;
    if (g->reflective) {
        ix = (int)sym_round(r.x); iy = (int)sym_round(r.y); iz = (int)sym_round(r.z);
        return grid_cell(g, reflective_boundary(ix, nx), reflective_boundary(iy, ny), reflective_boundary(iz, nz));
    }
    ix = (int)sym_round(fmod(r.x, nx));
    iy = (int)sym_round(fmod(r.y, ny));
    iz = (int)sym_round(fmod(r.z, nz));
    ix = (ix + nx * (ix < 0)) % nx;
    iy = (iy + ny * (iy < 0)) % ny;
    iz = (iz + nz * (iz < 0)) % nz;
    return grid_cell(g, ix, iy, iz);
}

/* CubicInterpolateScalar (Grid.h:498): the Catmull-Rom polynomial in double,
 * terms grouped as the reference groups them (the sums round differently in
 * any other order). */
static double cubic_d(double p0, double p1, double p2, double p3, double pos) {
    double a = -0.5 * p0 + 1.5 * p1 - 1.5 * p2 + 0.5 * p3;
    double b = p0 - 2.5 * p1 + p2 * 2 - 0.5 * p3;
    double c = -0.5 * p0 + 0.5 * p2;
    return a * pos * pos * pos + b * pos * pos + c * pos + p1;
}

/* Grid<float>::interpolate (Grid.h:317) of a scalar grid (Grid1f). */
static float scalar_grid(const crp_grid3f_desc *g, v3 pos) {
    if (g->clip_volume && !grid_in_volume(g, pos)) return 0.f;
    if (g->interpolation == CRP_INTERPOLATION_NEAREST_NEIGHBOUR) return g->values[grid_nearest_cell(g, pos)];
    v3 r = grid_unit(g, pos);
    if (g->interpolation == CRP_INTERPOLATION_TRICUBIC) {
        int ix0 = (int)floor(r.x), iy0 = (int)floor(r.y), iz0 = (int)floor(r.z);
        double fx = r.x - ix0, fy = r.y - iy0, fz = r.z - iz0;
        double vx[4], vy[4], vz[4];
        for (int a = -1; a < 3; a++) {
            for (int b = -1; b < 3; b++) {
                for (int c = -1; c < 3; c++) vz[c + 1] = g->values[grid_cell_bc(g, ix0 + a, iy0 + b, iz0 + c)];
                vy[b + 1] = cubic_d(vz[0], vz[1], vz[2], vz[3], fz);
            }
            vx[a + 1] = cubic_d(vy[0], vy[1], vy[2], vy[3], fy);
        }
        return (float)cubic_d(vx[0], vx[1], vx[2], vx[3], fx);
    }
    int n[3] = {(int)g->nx, (int)g->ny, (int)g->nz}, lo[3], hi[3];
    double rr[3] = {r.x, r.y, r.z}, f0[3], f1[3];
    for (int a = 0; a < 3; a++) {
        double x = rr[a];
        if (g->reflective) { /* reflectiveClamp, Grid.h:49 */
            while ((x < -0.5) || (x > (n[a] - 0.5))) x = 2 * n[a] * (x > (n[a] - 0.5)) - x - 1;
            lo[a] = (int)floor(x);
            hi[a] = lo[a] + (lo[a] < n[a] - 1);
            if (x < 0) { lo[a] = 0; hi[a] = 0; }
        } else { /* periodicClamp, Grid.h:29 */
            lo[a] = (((int)floor(x) % n[a]) + n[a]) % n[a];
            hi[a] = (lo[a] + 1) % n[a];
        }
        f0[a] = x - floor(x);
        f1[a] = 1 - f0[a];
    }
    /* Grid.h:570-577 with T = float: products in double, sum into a float */
    const int sel[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, 1, 1}};
    float b = 0.f;
    for (int k = 0; k < 8; k++) {
        float v = g->values[grid_cell(g, sel[k][0] ? hi[0] : lo[0], sel[k][1] ? hi[1] : lo[1],
                                      sel[k][2] ? hi[2] : lo[2])];
        b += v * (sel[k][0] ? f0[0] : f1[0]) * (sel[k][1] ? f0[1] : f1[1]) * (sel[k][2] ? f0[2] : f1[2]);
    }
    return b;
}

static v3 grid_field(const crp_grid3f_desc *g, v3 pos) {
    v3 origin = mk(g->origin[0], g->origin[1], g->origin[2]);
    v3 spacing = mk(g->spacing[0], g->spacing[1], g->spacing[2]);
    int Nx = (int)g->nx, Ny = (int)g->ny, Nz = (int)g->nz;
    if (g->clip_volume && !grid_in_volume(g, pos)) return mk(0, 0, 0); /* Grid.h:320 */
    if (g->interpolation == CRP_INTERPOLATION_TRICUBIC) return grid_tricubic3(g, pos);
    if (g->interpolation == CRP_INTERPOLATION_NEAREST_NEIGHBOUR) {
        const float *v = g->values + 3 * grid_nearest_cell(g, pos);
        return mk(v[0], v[1], v[2]);
    }
    v3 gridOrigin = add(origin, divs(spacing, 2)); /* Grid.h:227 */
    v3 r = divv(sub(pos, gridOrigin), spacing);
    int ix0, ix1, iy0, iy1, iz0, iz1;
    double fX0, fY0, fZ0;
    if (g->reflective) { /* Grid.h:49 reflectiveClamp */
        double rr[3] = {r.x, r.y, r.z};
        int n[3] = {Nx, Ny, Nz}, lo[3], hi[3];
        double res[3];
        for (int a = 0; a < 3; a++) {
            double x = rr[a];
            while ((x < -0.5) || (x > (n[a] - 0.5)))
                x = 2 * n[a] * (x > (n[a] - 0.5)) - x - 1;
            res[a] = x;
            lo[a] = (int)floor(x);
            hi[a] = lo[a] + (lo[a] < n[a] - 1);
            if (x < 0) { lo[a] = 0; hi[a] = 0; }
        }
        ix0 = lo[0]; ix1 = hi[0]; iy0 = lo[1]; iy1 = hi[1]; iz0 = lo[2]; iz1 = hi[2];
        fX0 = res[0] - floor(res[0]);
        fY0 = res[1] - floor(res[1]);
        fZ0 = res[2] - floor(res[2]);
    } else { /* Grid.h:31 periodicClamp */
        ix0 = (((int)floor(r.x) % Nx) + Nx) % Nx; ix1 = (ix0 + 1) % Nx;
        iy0 = (((int)floor(r.y) % Ny) + Ny) % Ny; iy1 = (iy0 + 1) % Ny;
        iz0 = (((int)floor(r.z) % Nz) + Nz) % Nz; iz1 = (iz0 + 1) % Nz;
        fX0 = r.x - floor(r.x);
        fY0 = r.y - floor(r.y);
        fZ0 = r.z - floor(r.z);
    }
    float fx1 = (float)(1 - fX0), fy1 = (float)(1 - fY0), fz1 = (float)(1 - fZ0);
    float fx0 = (float)fX0, fy0 = (float)fY0, fz0 = (float)fZ0;
    const float *v = g->values;
    size_t sy = (size_t)Nz, sx = (size_t)Ny * (size_t)Nz;
#define CELL(i, j, k) (v + 3 * ((size_t)(i) * sx + (size_t)(j) * sy + (size_t)(k)))
    const int cx[8] = {ix0, ix1, ix0, ix0, ix1, ix0, ix1, ix1};
    const int cy[8] = {iy0, iy0, iy1, iy0, iy0, iy1, iy1, iy1};
    const int cz[8] = {iz0, iz0, iz0, iz1, iz1, iz1, iz0, iz1};
    const float wx[8] = {fx1, fx0, fx1, fx1, fx0, fx1, fx0, fx0};
    const float wy[8] = {fy1, fy1, fy0, fy1, fy1, fy0, fy0, fy0};
    const float wz[8] = {fz1, fz1, fz1, fz0, fz0, fz0, fz1, fz0};
    float bx = 0.f, by = 0.f, bz = 0.f;
    for (int c = 0; c < 8; c++) {
        const float *p = CELL(cx[c], cy[c], cz[c]);
        bx += p[0] * wx[c] * wy[c] * wz[c];
        by += p[1] * wx[c] * wy[c] * wz[c];
        bz += p[2] * wx[c] * wy[c] * wz[c];
    }
#undef CELL
    return mk(bx, by, bz);
}

/* PlaneWaveTurbulence::getField, scalar branch (PlaneWaveTurbulence.cpp:233-239). */
static v3 plane_wave_field(const crp_plane_wave_desc *p, v3 pos) {
    v3 B = mk(0, 0, 0);
    for (int i = 0; i < p->n_modes; i++) {
        v3 kap = mk(p->kappa[3*i], p->kappa[3*i+1], p->kappa[3*i+2]);
        v3 xi = mk(p->xi[3*i], p->xi[3*i+1], p->xi[3*i+2]);
        double z_ = dot(pos, kap);
        B = add(B, muls(muls(xi, p->ak[i]), cos(p->k[i] * z_ + p->beta[i])));
    }
    return B;
}

/* ---------------------------------------------------------------- JF12Field
 * JF12Field::getField and its parts (JF12Field.cpp:195-346) and
 * JF12FieldSolenoidal's disk and X fields (JF12FieldSolenoidal.cpp:115-302),
 * same operation order, glibc's exp, log, sin, cos, atan, atan2 and pow as the
 * reference calls them. */

/* JF12Field::logisticFunction (JF12Field.cpp:195) */
static double jf_logistic(double x, double x0, double w) { return 1. / (1. + exp(-2. * (fabs(x) - x0) / w)); }

/* Vector3::getPhi (Vector3.h:136) */
static double jf_phi(double x, double y) {
    if ((fabs(x) < DBL_MIN) && (fabs(y) < DBL_MIN)) return 0.0;
    return atan2(y, x);
}

/* arm radius at the negative x axis (JF12Field.cpp:228-233, :315-320) */
static double jf_r_negx(const crp_jf12_desc *J, double r, double phi) {
    double r_negx = r * exp(-(phi - M_PI) / J->tan90_minus_pitch);
    if (r_negx > J->r_arms[7]) r_negx = r * exp(-(phi + M_PI) / J->tan90_minus_pitch);
    if (r_negx > J->r_arms[7]) r_negx = r * exp(-(phi + 3 * M_PI) / J->tan90_minus_pitch);
    return r_negx;
}

/* JF12FieldSolenoidal: the spiral arm of (r, phi) at r1 along the logarithmic
 * spiral (getHPhiIntegral :241, getSpiralFieldStrengthConstant :260) */
static int jf12s_arm(const crp_jf12_desc *J, double r, double phi, double *phi1_out) {
    double phi1 = phi - log(r / J->r1) * J->cot_pitch;
    phi1 = atan2(sin(phi1), cos(phi1));
    int idx = 1;
    while (idx < 10 && phi1 < J->phi0_arms[idx]) idx += 1;
    *phi1_out = phi1;
    return idx;
}

/* getDiskTransitionPolynomial (:197) and its derivative (:219) */
static void jf12s_transition(const crp_jf12_desc *J, double r, double *p, double *q) {
    if ((r < J->r1) || (r > J->r2)) { *p = 0.; *q = 0.; return; }
    if ((r > J->r1s) && (r < J->r2s)) { *p = J->r1 / r; *q = 0.; return; }
    double r_a = J->r1, r_b = J->r1s;
    if (r >= J->r2s) { r_a = J->r2; r_b = J->r2s; }
    double fakt = (r_a / r_b - 2.) / ((r_a - r_b) * (r_a - r_b));
    *p = (J->r1 / r_b) * (2. - r / r_b + fakt * (r - r_b) * (r - r_b));
    *q = (J->r1 / r_b) * (2. - 2. * r / r_b + fakt * (3. * r * r - 4. * r * r_b + r_b * r_b));
}

/* JF12FieldSolenoidal::getDiskField (:115) */
static v3 jf12s_disk(const crp_jf12_desc *J, double r, double z, double phi, double sinPhi, double cosPhi) {
    v3 b = mk(0, 0, 0);
    if (!J->use_disk) return b;
    double lfDisk = jf_logistic(z, J->h_disk, J->w_disk);
    if (!((J->r1 < r) && (r < J->r2))) return b;
    double phi1;
    int idx = jf12s_arm(J, r, phi, &phi1);
    double hint = phi1 * J->b_arms[idx] + J->phi_coeff[idx];
    double mag1 = J->b_arms[idx];
    double pdelta, qdelta;
    jf12s_transition(J, r, &pdelta, &qdelta);
    double br = pdelta * mag1 * J->sin_pitch;
    double bphi = pdelta * mag1 * J->cos_pitch - qdelta * hint * J->sin_pitch;
    b.x += br * cosPhi - bphi * sinPhi;
    b.y += br * sinPhi + bphi * cosPhi;
    return muls(b, 1 - lfDisk);
}

/* JF12FieldSolenoidal::getXField (:131) */
static v3 jf12s_x(const crp_jf12_desc *J, double r, double z, double sinPhi, double cosPhi) {
    v3 b = mk(0, 0, 0);
    if (!J->use_x) return b;
    double zS = J->z_s, rXc = J->r_xc, rX = J->r_x, bX = J->b_x, tanT = J->tan_theta_x0;
    double rc = rXc + fabs(z) / tanT;
    double r0c = rXc + zS / tanT;
    if (fabs(z) > zS) {
        if (r == 0.) {
            b.z = bX / ((1. + fabs(z) * J->cot_theta_x0 / rXc) * (1. + fabs(z) * J->cot_theta_x0 / rXc));
            return b;
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
            sinThetaX = J->sin_theta_x0;
            cosThetaX = J->cos_theta_x0;
        }
        double zsign = z < 0 ? -1 : 1;
        b.x += zsign * bMagX * cosThetaX * cosPhi;
        b.y += zsign * bMagX * cosThetaX * sinPhi;
        b.z += bMagX * sinThetaX;
        return b;
    }
    double r0 = r * 1. / (1. - 1. / (2. * (zS + rXc * tanT)) * (zS - z * z / zS));
    double f, br0, bz0;
    if (r0 >= r0c) {
        r0 = r + 1. / (2. * tanT) * (zS - z * z / zS);
        f = 1. + 1 / (2 * r * tanT / zS) * (1. - (z / zS) * (z / zS));
    } else {
        double g = 1. - 1. / (2. + 2. * (rXc * tanT / zS)) * (1. - (z / zS) * (z / zS));
        f = 1. / (g * g);
    }
    if (r0 < r0c) {
        double rp = r0 * rXc / r0c;
        double thetaX = atan(zS / (r0 - rp));
        br0 = bX * exp(-rp / rX) * (rXc / r0c) * (rXc / r0c) * cos(thetaX);
        bz0 = bX * exp(-rp / rX) * (rXc / r0c) * (rXc / r0c) * sin(thetaX);
    } else {
        double rp = r0 - zS / tanT;
        br0 = bX * exp(-rp / rX) * (rp / r0) * J->cos_theta_x0;
        bz0 = bX * exp(-rp / rX) * (rp / r0) * J->sin_theta_x0;
    }
    double br = z / zS * f * br0;
    double bz = bz0 * f;
    b.x += br * cosPhi;
    b.y += br * sinPhi;
    b.z += bz;
    return b;
}

/* getRegularField (JF12Field.cpp:199): getDiskField (:216) + getToroidalHaloField
 * (:248) + getXField (:267) */
static v3 jf12_regular(const crp_jf12_desc *J, v3 pos) {
    v3 b = mk(0, 0, 0);
    double kpc = J->kpc;
    double d = sqrt(pos.x * pos.x + pos.y * pos.y + pos.z * pos.z);
    if (!(d < 20 * kpc)) return b;
    double r = sqrt(pos.x * pos.x + pos.y * pos.y), z = pos.z;
    double phi = jf_phi(pos.x, pos.y);
    double sinPhi = sin(phi), cosPhi = cos(phi);
    int sol = J->variant == CRP_JF12_SOLENOIDAL;
    v3 bd = mk(0, 0, 0);
    if (sol) {
        bd = jf12s_disk(J, r, z, phi, sinPhi, cosPhi);
    } else if (J->use_disk) {
        double lfDisk = jf_logistic(z, J->h_disk, J->w_disk);
        if (r > 3 * kpc) {
            double bMag = 0;
            if (r < 5 * kpc) {
                bMag = J->b_ring * (5 * kpc / r) * (1 - lfDisk);
                bd.x += -bMag * sinPhi;
                bd.y += bMag * cosPhi;
            } else {
                double r_negx = jf_r_negx(J, r, phi);
                for (int i = 7; i >= 0; i--)
                    if (r_negx < J->r_arms[i]) bMag = J->b_disk[i];
                bMag *= (5 * kpc / r) * (1 - lfDisk);
                bd.x += bMag * (J->sin_pitch * cosPhi - J->cos_pitch * sinPhi);
                bd.y += bMag * (J->sin_pitch * sinPhi + J->cos_pitch * cosPhi);
            }
        }
    }
    b = add(b, bd);
    int outside1 = r * r + z * z > 1 * kpc * kpc;
    v3 bh = mk(0, 0, 0);
    if (J->use_toroidal_halo && outside1) {
        double lfDisk = jf_logistic(z, J->h_disk, J->w_disk);
        double bMagH = exp(-fabs(z) / J->z0) * lfDisk;
        if (z >= 0)
            bMagH *= J->b_north * (1 - jf_logistic(r, J->r_north, J->w_halo));
        else
            bMagH *= J->b_south * (1 - jf_logistic(r, J->r_south, J->w_halo));
        bh.x += -bMagH * sinPhi;
        bh.y += bMagH * cosPhi;
    }
    b = add(b, bh);
    v3 bx = mk(0, 0, 0);
    if (sol) {
        bx = jf12s_x(J, r, z, sinPhi, cosPhi);
    } else if (J->use_x && outside1) {
        double bMagX, sinThetaX, cosThetaX, rp;
        double rc = J->r_xc + fabs(z) / J->tan_theta_x0;
        if (r < rc) {
            rp = r * J->r_xc / rc;
            bMagX = J->b_x * exp(-1 * rp / J->r_x) * pow(J->r_xc / rc, 2.);
            double thetaX = atan2(fabs(z), (r - rp));
            if (z == 0) thetaX = M_PI / 2.;
            sinThetaX = sin(thetaX);
            cosThetaX = cos(thetaX);
        } else {
            rp = r - fabs(z) / J->tan_theta_x0;
            bMagX = J->b_x * exp(-rp / J->r_x) * (rp / r);
            sinThetaX = J->sin_theta_x0;
            cosThetaX = J->cos_theta_x0;
        }
        double zsign = z < 0 ? -1 : 1;
        bx.x += zsign * bMagX * cosThetaX * cosPhi;
        bx.y += zsign * bMagX * cosThetaX * sinPhi;
        bx.z += bMagX * sinThetaX;
    }
    return add(b, bx);
}

/* getTurbulentStrength (JF12Field.cpp:301) */
static double jf12_turbulent_strength(const crp_jf12_desc *J, v3 pos) {
    double kpc = J->kpc;
    if (sqrt(pos.x * pos.x + pos.y * pos.y + pos.z * pos.z) > 20 * kpc) return 0;
    double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    double phi = jf_phi(pos.x, pos.y);
    double bDisk = 0;
    if (r < 5 * kpc) {
        bDisk = J->b_disk_turb5;
    } else {
        double r_negx = jf_r_negx(J, r, phi);
        for (int i = 7; i >= 0; i--)
            if (r_negx < J->r_arms[i]) bDisk = J->b_disk_turb[i];
        bDisk *= (5 * kpc) / r;
    }
    bDisk *= exp(-0.5 * pow(pos.z / J->z_disk_turb, 2));
    double bHalo = J->b_halo_turb * exp(-r / J->r_halo_turb) * exp(-0.5 * pow(pos.z / J->z_halo_turb, 2));
    return sqrt(pow(bDisk, 2) + pow(bHalo, 2));
}

/* getField (JF12Field.cpp:346): turbulent + (striated or regular); the
 * turbulent part is Vector3f * double, a float product (Vector3.h:305). */
static v3 jf12_field(const crp_field_component *f, v3 pos) {
    const crp_jf12_desc *J = &f->jf12;
    v3 b = mk(0, 0, 0);
    if (J->use_turbulent) {
        v3 g = grid_field(&f->grid, pos);
        float s = (float)jf12_turbulent_strength(J, pos);
        float gx = (float)g.x * s, gy = (float)g.y * s, gz = (float)g.z * s;
        b = add(b, mk(gx, gy, gz));
    }
    if (J->use_striated) { /* JF12Field.cpp:296 */
        double v = f->modulation.values[grid_nearest_cell(&f->modulation, pos)];
        b = add(b, muls(jf12_regular(J, pos), 1. + J->sqrt_beta * v));
    } else if (J->use_regular) {
        b = add(b, jf12_regular(J, pos));
    }
    return b;
}

/* ---------------------------------------------------------------- UF23Field
 * UF23Field::getField and its parts (UF23Field.cpp:269-558) in the model's
 * units (kpc, microgauss), same operation order, glibc's libm. */

static const double UF23_TWO_PI = 2 * 3.1415926535897932384626;

/* uf23::CylToCart (UF23Field.cpp:12) */
static v3 uf_cyl_to_cart(double v0, double v1, double v2, double cosPhi, double sinPhi) {
    return mk(v0 * cosPhi - v1 * sinPhi, v0 * sinPhi + v1 * cosPhi, v2);
}

/* uf23::Sigmoid (UF23Field.cpp:29) */
static double uf_sigmoid(double x, double x0, double w) { return 1 / (1 + exp(-(x - x0) / w)); }

/* uf23::DeltaPhi (UF23Field.cpp:37) */
static double uf_delta_phi(double phi0, double phi1) { return acos(cos(phi1) * cos(phi0) + sin(phi1) * sin(phi0)); }

/* getSpiralField (UF23Field.cpp:510) */
static v3 uf_spiral(const crp_uf23_desc *U, double x, double y, double z) {
    const double rRef = 5, rInner = 5, wInner = 0.5, rOuter = 20, wOuter = 0.5;
    double r2 = x * x + y * y;
    if (r2 == 0) return mk(0, 0, 0);
    double r = sqrt(r2);
    double phi = atan2(y, x);
    double hdz = 1 - uf_sigmoid(fabs(z), U->disk_h, U->disk_w);
    double rFacI = uf_sigmoid(r, rInner, wInner);
    double rFacO = 1 - uf_sigmoid(r, rOuter, wOuter);
    double rFac = r > 1e-5 * (1e-3 * 1) ? (1 - exp(-r * r)) / r : r * (1 - r2 / 2);
    double gdrTimesRrefByR = rRef * rFac * rFacO * rFacI;
    double phi0 = phi - log(r / rRef) / U->tan_pitch;
    double b = U->disk_b1 * cos(1 * (phi0 - U->disk_phase1)) + U->disk_b2 * cos(2 * (phi0 - U->disk_phase2)) +
               U->disk_b3 * cos(3 * (phi0 - U->disk_phase3));
    double fac = hdz * gdrTimesRrefByR;
    return uf_cyl_to_cart(b * fac * U->sin_pitch, b * fac * U->cos_pitch, 0, x / r, y / r);
}

/* getSpurField (UF23Field.cpp:453) */
static v3 uf_spur(const crp_uf23_desc *U, double x, double y, double z) {
    const double rRef = 8.2;
    double r2 = x * x + y * y;
    double r = sqrt(r2);
    if (r < DBL_MIN) return mk(0, 0, 0);
    double phi = atan2(y, x);
    if (phi < 0) phi += UF23_TWO_PI;
    double phiRef = U->disk_phase1;
    int iBest = -2;
    double bestDist = -1;
    for (int i = -1; i <= 1; ++i) {
        double pphi = phi - phiRef + i * UF23_TWO_PI;
        double rr = rRef * exp(pphi * U->tan_pitch);
        if (bestDist < 0 || fabs(r - rr) < bestDist) {
            bestDist = fabs(r - rr);
            iBest = i;
        }
    }
    if (iBest != 0) return mk(0, 0, 0);
    double phi0 = phi - log(r / rRef) / U->tan_pitch;
    double deltaPhi0 = uf_delta_phi(phiRef, phi0);
    double delta = deltaPhi0 / U->spur_width;
    double B = U->disk_b1 * exp(-0.5 * pow(delta, 2));
    double wS = 5 * (3.1415926535897932384626 / 180.);
    double deltaPhiC = uf_delta_phi(U->spur_center, phi);
    double gS = 1 - uf_sigmoid(fabs(deltaPhiC), U->spur_length, wS);
    double hd = 1 - uf_sigmoid(fabs(z), U->disk_h, U->disk_w);
    double bS = rRef / r * B * hd * gS;
    return uf_cyl_to_cart(bS * U->sin_pitch, bS * U->cos_pitch, 0, x / r, y / r);
}

/* getToroidalHaloField (UF23Field.cpp:361) */
static v3 uf_toroidal(const crp_uf23_desc *U, double x, double y, double z) {
    double r2 = x * x + y * y;
    double r = sqrt(r2);
    double absZ = fabs(z);
    double b0 = z >= 0 ? U->toroidal_bn : U->toroidal_bs;
    double sigmoidR = uf_sigmoid(r, U->toroidal_r, U->toroidal_w);
    double sigmoidZ = uf_sigmoid(absZ, U->disk_h, U->disk_w);
    double bPhi = b0 * (1. - sigmoidR) * sigmoidZ * exp(-absZ / U->toroidal_z);
    double cosPhi = r > DBL_MIN ? x / r : 1;
    double sinPhi = r > DBL_MIN ? y / r : 0;
    return uf_cyl_to_cart(0, bPhi, 0, cosPhi, sinPhi);
}

/* getPoloidalHaloField (UF23Field.cpp:385) */
static v3 uf_poloidal(const crp_uf23_desc *U, double x, double y, double z) {
    double r2 = x * x + y * y;
    double r = sqrt(r2);
    double P = U->poloidal_p;
    double c = pow(U->poloidal_a / U->poloidal_z, P);
    double a0p = pow(U->poloidal_a, P);
    double rp = pow(r, P);
    double abszp = pow(fabs(z), P);
    double cabszp = c * abszp;
    double t0 = a0p + cabszp - rp;
    double t1 = sqrt(pow(t0, 2) + 4 * a0p * rp);
    double ap = 2 * a0p * rp / (t1 + t0);
    double a = 0;
    if (ap < 0) {
        if (r > DBL_MIN) a = NAN; /* the reference throws: "this should never happen" */
    } else {
        a = pow(ap, 1 / P);
    }
    double radialDependence = U->model == CRP_UF23_EXPX ? exp(-a / U->poloidal_r)
                                                        : 1 - uf_sigmoid(a, U->poloidal_r, U->poloidal_w);
    double Bzz = U->poloidal_b * radialDependence;
    double rOverA = 1 / pow(2 * a0p / (t1 + t0), 1 / P);
    double signZ = z < 0 ? -1 : 1;
    double Br = Bzz * c * a / rOverA * signZ * pow(fabs(z), P - 1) / t1;
    double Bz = Bzz * pow(rOverA, P - 2) * (ap + a0p) / t1;
    if (r < DBL_MIN) return mk(0, 0, Bz);
    return uf_cyl_to_cart(Br, 0, Bz, x / r, y / r);
}

/* getTwistedHaloField (UF23Field.cpp:318) */
static v3 uf_twisted(const crp_uf23_desc *U, double x, double y, double z) {
    double r = sqrt(x * x + y * y);
    double cosPhi = r > DBL_MIN ? x / r : 1;
    double sinPhi = r > DBL_MIN ? y / r : 0;
    v3 bX = uf_poloidal(U, x, y, z);
    /* uf23::CartToCyl (UF23Field.cpp:20) */
    double bR = bX.x * cosPhi + bX.y * sinPhi;
    double bZ = bX.z;
    double bPhi = 0;
    if (U->twisting_time != 0 && r != 0) {
        const double kilometer = 1 / 3.0856775807e+16;
        const double second = 1 / (1e6 * 60 * 60 * 24 * 365.25);
        const double v0 = -240 * kilometer / second;
        const double r0 = 1.6, z0 = 10;
        double fr = 1 - exp(-r / r0);
        double t0 = exp(2 * fabs(z) / z0);
        double gz = 2 / (1 + t0);
        double signZ = z < 0 ? -1 : 1;
        double deltaZ = -signZ * v0 * fr / z0 * t0 * pow(gz, 2);
        double deltaR = v0 * ((1 - fr) / r0 - fr / r) * gz;
        bPhi = (bZ * deltaZ + bR * deltaR) * U->twisting_time;
    }
    return uf_cyl_to_cart(bR, bPhi, bZ, cosPhi, sinPhi);
}

/* UF23Field::getField (UF23Field.cpp:269) and operator() (:277) */
static v3 uf23_field(const crp_uf23_desc *U, v3 position) {
    double x = position.x / U->kpc * 1, y = position.y / U->kpc * 1, z = position.z / U->kpc * 1;
    if (x * x + y * y + z * z > U->max_radius_squared) return mk(0, 0, 0);
    v3 disk = U->model == CRP_UF23_SPUR ? uf_spur(U, x, y, z) : uf_spiral(U, x, y, z);
    v3 halo = U->model == CRP_UF23_TWISTX ? uf_twisted(U, x, y, z)
                                          : add(uf_toroidal(U, x, y, z), uf_poloidal(U, x, y, z));
    v3 b = divs(add(disk, halo), 1);
    return muls(divs(b, 1), U->microgauss);
}

/* ---------------------------------------------------------------- PT11Field
 * PT11Field::getField (PT11Field.cpp:80-128), SI units. */
static v3 pt11_field(const crp_pt11_desc *P, v3 pos) {
    double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    v3 b = mk(0, 0, 0);
    if (P->use_ass || P->use_bss) {
        /* Vector3::getPhi (Vector3.h:136) */
        double phi = (fabs(pos.x) < DBL_MIN && fabs(pos.y) < DBL_MIN) ? 0.0 : atan2(pos.y, pos.x);
        double theta = M_PI - phi;
        double cos_theta = -pos.x / r;
        double sin_theta = pos.y / r;
        b.x = P->sin_pitch * cos_theta - P->cos_pitch * sin_theta;
        b.y = -P->sin_pitch * sin_theta - P->cos_pitch * cos_theta;
        b = muls(b, -1);
        double bMag = cos(theta - P->cos_pitch / P->sin_pitch * log(r / P->r_sun) + P->phi);
        if (P->use_ass) bMag = fabs(bMag);
        bMag *= P->b0_d * P->r_sun / (r < P->r_c ? P->r_c : r) / P->cos_phi * exp(-fabs(pos.z) / P->z0_d);
        b = muls(b, bMag);
    }
    if (P->use_halo) {
        double bMag = pos.z > 0 ? P->b0_hn : -P->b0_hs;
        double z1 = fabs(pos.z) < P->z0_h ? P->z11_h : P->z12_h;
        double v = (fabs(pos.z) - P->z0_h) / z1;
        bMag *= r / P->r0_h * exp(1 - r / P->r0_h) / (1 + v * v); /* pow(v, 2.) is exact: v * v */
        b = add(b, muls(mk(-pos.y / r, pos.x / r, 0), bMag));
    }
    return b;
}

/* ArchimedeanSpiralField::getField (ArchimedeanSpiralField.cpp:12-46), with
 * Vector3::getR / getTheta / getPhi (Vector3.h:126-151). */
static v3 archimedean_field(const crp_archimedean_desc *A, v3 pos) {
    double r = sqrt(pos.x * pos.x + pos.y * pos.y + pos.z * pos.z);
    double theta = (fabs(pos.x) < DBL_MIN && fabs(pos.y) < DBL_MIN && fabs(pos.z) < DBL_MIN)
                       ? 0.0 : atan2(sqrt(pos.x * pos.x + pos.y * pos.y), pos.z);
    double phi = (fabs(pos.x) < DBL_MIN && fabs(pos.y) < DBL_MIN) ? 0.0 : atan2(pos.y, pos.x);
    double cos_phi = cos(phi), sin_phi = sin(phi), cos_theta = cos(theta), sin_theta = sin(theta);
    v3 B = mk(0, 0, 0);
    double C1 = A->r0 * A->r0 / r / r;
    B.x += C1 * cos_phi * sin_theta;
    B.y += C1 * sin_phi * sin_theta;
    B.z += C1 * cos_theta;
    double C2 = -(A->omega * A->r0 * A->r0 * sin_theta) / (r * A->vw);
    B.x += C2 * (-sin_phi);
    B.y += C2 * cos_phi;
    if (pos.z < 0.) B = muls(B, -1);
    return muls(B, A->b0);
}

/* ---------------------------------------------------------------- TF17Field
 * TF17Field::getField and its helpers (TF17Field.cpp:197-307), SI units, the
 * reference's operation order. */
static double tf17_zscale(const crp_tf17_desc *T, double z) { return 1 + z * z / T->h_p / T->h_p; }

static double tf17_winding(const crp_tf17_desc *T, double r, double z) {
    return T->cot_p0 * log(1 - exp(-r / T->l_p) + T->epsilon) / tf17_zscale(T, z);
}

static double tf17_radial_scale(const crp_tf17_desc *T, double B1, double phi_star, double z1, double phi,
                                double r, double z) {
    double phi_prime = phi - tf17_winding(T, r, z) - phi_star;
    return B1 * exp(-fabs(z1) / T->h_disk) * cos(phi_prime);
}

static double tf17_azimuthal(const crp_tf17_desc *T, double r, double z, double B_r, double B_z) {
    double r_ = r / T->l_p;
    double rscale = r > T->epsilon ? r_ * exp(-r_) / (1 - exp(-r_)) : 1 - r_ / 2. - r_ * r_ / 12.;
    double B_phi = T->cot_p0 / tf17_zscale(T, z) * rscale * B_r;
    B_phi = B_phi - 2 * z * r / (T->h_p * T->h_p) / tf17_zscale(T, z) * tf17_winding(T, r, z) * B_z;
    return B_phi;
}

static v3 tf17_xyz(double B_r, double B_phi, double B_z, double sinPhi, double cosPhi) {
    return mk(-(B_r * cosPhi - B_phi * sinPhi), B_r * sinPhi + B_phi * cosPhi, B_z);
}

static v3 tf17_disk(const crp_tf17_desc *T, double r, double z, double phi, double sinPhi, double cosPhi) {
    double B_r = 0, B_phi = 0, B_z = 0;
    if (T->disk_model == CRP_TF17_AD1) {
        if (r > T->r1_disk) {
            double z1_disk_z = (1. + T->a_disk * T->r1_disk * T->r1_disk) / (1. + T->a_disk * r * r);
            double B_r0 = tf17_radial_scale(T, T->b1_disk, T->phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = (T->r1_disk / r) * z1_disk_z * B_r0;
            B_z = 2 * T->a_disk * T->r1_disk * z1_disk_z * z / (1 + T->a_disk * r * r) * B_r0;
            B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
        } else {
            double phi1_disk = tf17_winding(T, T->r1_disk, z) + T->phi_star_disk;
            double B_amp = T->b1_disk * exp(-fabs(z) / T->h_disk);
            B_r = cos(phi1_disk - phi) * B_amp;
            B_phi = sin(phi1_disk - phi) * B_amp;
        }
    } else if (T->disk_model == CRP_TF17_BD1) {
        if (r > T->epsilon) {
            double r1_disk_r = T->r1_disk / r;
            double z1_disk_z = 5. / (r1_disk_r * r1_disk_r + 4. / sqrt(r1_disk_r));
            double B_r0 = tf17_radial_scale(T, T->b1_disk, T->phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = r1_disk_r * z1_disk_z * B_r0;
            B_z = -0.4 * r1_disk_r / r * z1_disk_z * z1_disk_z * z * (r1_disk_r * r1_disk_r - 1. / sqrt(r1_disk_r)) *
                  B_r0;
        } else {
            double z1_disk_z = 5. * r * r / (T->r1_disk * T->r1_disk);
            double B_r0 = tf17_radial_scale(T, T->b1_disk, T->phi_star_disk, z1_disk_z * z, phi, r, z);
            B_r = 5. * r / T->r1_disk * B_r0;
            B_z = -10. * z / T->r1_disk * B_r0;
        }
        B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    } else { /* Dd1 */
        double z_sign = z >= 0 ? 1. : -1.;
        double z_abs = fabs(z);
        if (z_abs > T->epsilon) {
            double z1_disk_z = T->z1_disk / z_abs;
            double r1_disk_r = 1.5 / (sqrt(z1_disk_z) + 0.5 / z1_disk_z);
            double F_r = r1_disk_r * r <= T->l_disk ? 1. : exp(1. - r1_disk_r * r / T->l_disk);
            double B_z0 = z_sign * T->b1_disk * F_r * cos(phi - tf17_winding(T, r, z) - T->phi_star_disk);
            B_r = -0.5 / 1.5 * r1_disk_r * r1_disk_r * r1_disk_r * r / z_abs * (sqrt(z1_disk_z) - 1 / z1_disk_z) * B_z0;
            B_z = z_sign * r1_disk_r * r1_disk_r * B_z0;
        } else {
            double z_z1_disk = z_abs / T->z1_disk;
            double r1_disk_r = 1.5 * sqrt(z_abs / T->z1_disk);
            double F_r = r1_disk_r * r <= T->l_disk ? 1. : exp(1. - r1_disk_r * r / T->l_disk);
            double B_z0 = z_sign * T->b1_disk * F_r * cos(phi - tf17_winding(T, r, z) - T->phi_star_disk);
            B_r = -1.125 * r / T->z1_disk * (1 - 2.5 * z_z1_disk * sqrt(z_z1_disk)) * B_z0;
            B_z = z_sign * r1_disk_r * r1_disk_r * B_z0;
        }
        B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    }
    return tf17_xyz(B_r, B_phi, B_z, sinPhi, cosPhi);
}

static v3 tf17_halo(const crp_tf17_desc *T, double r, double z, double phi, double sinPhi, double cosPhi) {
    double r1_halo_r = (1. + T->a_halo * T->z1_halo * T->z1_halo) / (1. + T->a_halo * z * z);
    double B_z0;
    if (T->halo_model == CRP_TF17_C0) {
        B_z0 = T->b1_halo * exp(-r1_halo_r * r / T->l_halo);
    } else {
        double phi_prime = phi - tf17_winding(T, r, z) - T->phi_star_halo;
        B_z0 = T->b1_halo * exp(-r1_halo_r * r / T->l_halo) * cos(phi_prime);
    }
    double B_r = 2 * T->a_halo * r1_halo_r * r1_halo_r * r * z / (1. + T->a_halo * z * z) * B_z0;
    double B_z = r1_halo_r * r1_halo_r * B_z0;
    double B_phi = tf17_azimuthal(T, r, z, B_r, B_z);
    return tf17_xyz(B_r, B_phi, B_z, sinPhi, cosPhi);
}

static v3 tf17_field(const crp_tf17_desc *T, v3 pos) {
    double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    /* pi - Vector3::getPhi (Vector3.h:136) */
    double phi = M_PI - ((fabs(pos.x) < DBL_MIN && fabs(pos.y) < DBL_MIN) ? 0.0 : atan2(pos.y, pos.x));
    double cosPhi = cos(phi), sinPhi = sin(phi);
    v3 b = mk(0., 0., 0.);
    if (T->use_disk) b = add(b, tf17_disk(T, r, pos.z, phi, sinPhi, cosPhi));
    if (T->use_halo) b = add(b, tf17_halo(T, r, pos.z, phi, sinPhi, cosPhi));
    return b;
}

/* PolarizedSingleModeMagneticField::getField (PolarizedSingleModeMagneticField.cpp:59) */
static v3 single_mode_field(const crp_single_mode_desc *S, v3 pos) {
    v3 d = mk(pos.x - S->r0[0], pos.y - S->r0[1], pos.z - S->r0[2]);
    double ph = S->k[0] * d.x + S->k[1] * d.y + S->k[2] * d.z;
    double c = cos(ph), s = sin(ph);
    v3 a = mk(S->u1[0] * c, S->u1[1] * c, S->u1[2] * c);
    v3 b = mk(S->u2[0] * S->sigma * s, S->u2[1] * S->sigma * s, S->u2[2] * S->sigma * s);
    return muls(add(a, b), S->b_max);
}

/* ---------------------------------------------------------------- KST24Field
 * KST24Field::getField and its parts (KST24Field.cpp:128-374) in the model's
 * units (kpc, gauss), same operation order, glibc's libm as the reference
 * calls it (pow(x, 2) included). */

/* get_toroidal (KST24Field.cpp:209) */
static v3 kst24_toroidal(v3 p, double B, double zmin, double zmax, double rmin, double rmax) {
    v3 v = mk(0, 0, 0);
    if ((p.z <= zmin) || (zmax <= p.z)) return v;
    double cR = sqrt(pow(p.x, 2) + pow(p.y, 2));
    if ((rmin <= cR) && (cR <= rmax)) {
        double theta = atan2(p.y, p.x);
        v.x = B * sin(theta);
        v.y = -B * cos(theta);
        v.z = 0;
    }
    return v;
}

/* get_Xfield (KST24Field.cpp:228) */
static v3 kst24_x(const crp_kst24_desc *K, v3 p) {
    v3 v = mk(0, 0, 0);
    int sign = 1;
    if (p.z < 0) sign = -1;
    if (fabs(p.z) > 10) return v;
    double cR = sqrt(p.x * p.x + p.y * p.y);
    double cR_0 = cR - p.z * sign * tan(K->x_theta_rad);
    if ((cR_0 < K->x_rmin) || (K->x_rmax < cR_0)) return v;
    double mgn_frc = cR_0 / cR;
    double xy_theta = atan2(p.y, p.x);
    v.x = K->x_b * mgn_frc * cos(xy_theta) * sign * sin(K->x_theta_rad);
    v.y = K->x_b * mgn_frc * sin(xy_theta) * sign * sin(K->x_theta_rad);
    v.z = K->x_b * mgn_frc * cos(K->x_theta_rad);
    return v;
}

/* is_LB (KST24Field.cpp:194) */
static int kst24_in_lb(const crp_kst24_desc *K, v3 p) {
    double ex = p.x - K->lb_x0, ey = p.y - K->lb_y0, ez = p.z - K->lb_z0;
    double cR = sqrt(ex * ex + ey * ey + ez * ez);
    return cR < K->lb_rmin + K->lb_dr;
}

/* get_LB (KST24Field.cpp:252) */
static v3 kst24_lb(const crp_kst24_desc *K, v3 p) {
    v3 v = mk(0, 0, 0);
    double ex = p.x - K->lb_x0, ey = p.y - K->lb_y0, ez = p.z - K->lb_z0;
    double cR = sqrt(ex * ex + ey * ey + ez * ez);
    if ((cR < K->lb_rmin) || (K->lb_rmin + K->lb_dr < cR)) return v;
    ex /= cR;
    ey /= cR;
    ez /= cR;
    double cosTheta = ex * K->lb_dir[0] + ey * K->lb_dir[1] + ez * K->lb_dir[2];
    double fx = K->lb_dir[0] - ex * cosTheta, fy = K->lb_dir[1] - ey * cosTheta, fz = K->lb_dir[2] - ez * cosTheta;
    double ampl = (1 + pow(K->lb_rmin, 2) / (2 * K->lb_rmin * K->lb_dr + K->lb_dr * K->lb_dr));
    v.x = K->lb_b * ampl * fx;
    v.y = K->lb_b * ampl * fy;
    v.z = K->lb_b * ampl * fz;
    return v;
}

/* get_logspiral (KST24Field.cpp:282) */
static v3 kst24_arm(const crp_kst24_arm *A, v3 p) {
    v3 v = mk(0, 0, 0);
    if ((p.z < A->zmin) || (A->zmax < p.z)) return v;
    double p0 = p.x + A->x_shift, p1 = p.y + A->y_shift, p2 = p.z;
    double r = sqrt(p0 * p0 + p1 * p1);
    if ((r < A->rmin) || (A->rmax < r)) return v;
    double a_kpc = 3;
    double k = tan(A->pitch_deg * M_PI / 180.);
    double cos_pitch = cos(A->pitch_deg * M_PI / 180.);
    double sin_pitch = sin(A->pitch_deg * M_PI / 180.);
    double phi0 = A->phi0_deg * M_PI / 180.;
    double arc_div_rad = A->arc_div_deg * M_PI / 180.;
    double phi = atan2(p1, p0);
    int nn = floor((log(r / a_kpc) - k * (phi + phi0)) / (2 * M_PI * k));
    double r1 = a_kpc * exp(k * (phi + phi0 + 2 * M_PI * nn));
    double r2 = r1 * exp(k * 2 * M_PI);
    if (fabs(r - r1) > fabs(r - r2)) {
        r1 = r2;
        nn++;
    }
    double xi = r1 * cos(phi), yi = r1 * sin(phi);
    double dir1 = k * xi - yi, dir2 = k * yi + xi;
    double dirtmp = sqrt(dir1 * dir1 + dir2 * dir2);
    dir1 /= dirtmp;
    dir2 /= dirtmp;
    double delta_phi = -((xi - p0) * dir1 + (yi - p1) * dir2) / (r1 / cos_pitch);
    r1 = a_kpc * exp(k * (phi + phi0 + delta_phi + 2 * M_PI * nn));
    xi = r1 * cos(phi + delta_phi);
    yi = r1 * sin(phi + delta_phi);
    dir1 = k * xi - yi;
    dir2 = k * yi + xi;
    dirtmp = sqrt(dir1 * dir1 + dir2 * dir2);
    dir1 /= dirtmp;
    dir2 /= dirtmp;
    double d1 = sqrt(pow((xi - p0), 2) + pow((yi - p1), 2));
    double L1 = r1 / sin_pitch;
    double r_scale = 5;
    double L1_at_r_scale = r_scale / sin_pitch;
    double g_plane = A->arc_radius2 * (1 + (L1 - L1_at_r_scale) * arc_div_rad);
    double g_z = A->arc_radius1 * (1 + (L1 - L1_at_r_scale) * arc_div_rad);
    double arc_r_plane = (A->arc_radius2 < g_plane) ? g_plane : A->arc_radius2; /* std::max */
    double arc_r_z = (A->arc_radius1 < g_z) ? g_z : A->arc_radius1;
    if (arc_r_plane > 1.2) arc_r_plane = 1.2;
    if (arc_r_z > 1.2) arc_r_z = 1.2;
    double d_at_L1 = sqrt(pow(fabs(d1 / arc_r_plane), A->arc_eps) + pow(fabs(p2 / arc_r_z), A->arc_eps));
    if ((d_at_L1 > 1) || (d_at_L1 < 0.)) return v;
    double scaling_factor = (A->arc_radius1 * A->arc_radius2) / (arc_r_plane * arc_r_z);
    v.x = A->b * dir1 * scaling_factor;
    v.y = A->b * dir2 * scaling_factor;
    v.z = 0;
    return v;
}

/* getField (KST24Field.cpp:128) */
static v3 kst24_field(const crp_kst24_desc *K, v3 pos) {
    v3 vals = mk(0, 0, 0);
    v3 p = divs(pos, K->kpc);
    if (p.z > K->north_zmin) {
        vals = add(vals, kst24_toroidal(p, K->north_b, K->north_zmin, K->north_zmax, K->north_rmin, K->north_rmax));
        vals = add(vals, kst24_x(K, p));
        return muls(vals, K->gauss);
    }
    if (p.z < K->south_zmax) {
        vals = add(vals, kst24_toroidal(p, K->south_b, K->south_zmin, K->south_zmax, K->south_rmin, K->south_rmax));
        vals = add(vals, kst24_x(K, p));
        return muls(vals, K->gauss);
    }
    if (kst24_in_lb(K, p)) {
        vals = add(vals, kst24_lb(K, p));
        return muls(vals, K->gauss);
    }
    for (int i = 0; i < 5; i++) vals = add(vals, kst24_arm(&K->arms[i], p));
    vals = add(vals, kst24_x(K, p));
    return muls(vals, K->gauss);
}

/* ---------------------------------------------------------------- CMZField
 * CMZField::getField and its parts (CMZField.cpp:14-304), SI units, same
 * operation order, glibc's libm. */

/* BPol (CMZField.cpp:18); pow_integer<3>(r1) is (r1 r1) r1 (Common.h:58) */
static v3 cmz_bpol(const crp_cmz_poloidal *P, v3 position) {
    v3 pos = sub(position, mk(P->mid[0], P->mid[1], P->mid[2]));
    double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    double phi = atan2(pos.y, pos.x);
    double r1 = 1 / (1 + P->a * pos.z * pos.z);
    double Bs = P->b * exp(-r1 * r / P->l);
    double Br = 2 * P->a * ((r1 * r1) * r1) * r * pos.z * Bs;
    v3 b = mk(0, 0, 0);
    b.z = r1 * r1 * Bs;
    b.x = Br * cos(phi);
    b.y = Br * sin(phi);
    return b;
}

/* BAz (CMZField.cpp:36) */
static v3 cmz_baz(const crp_cmz_cloud *C, v3 position) {
    v3 pos = sub(position, mk(C->mid[0], C->mid[1], C->mid[2]));
    double r = sqrt(pos.x * pos.x + pos.y * pos.y);
    double phi = atan2(pos.y, pos.x);
    double R = C->r, eta = C->eta, B1 = C->b1;
    double Hc = R / sqrt(log(2));
    double b = 1.;
    double m = 1;
    double r1 = R / 10;
    double v = m / eta * log((r + b) / (R + b));
    double cosV = cos(v + m * phi);
    double Br = 0, Bphi = 0;
    if (r > r1) {
        double Pre = B1 * cosV * exp(-pos.z * pos.z / Hc / Hc);
        Br = Pre * R / r;
        Bphi = -Pre / eta * R / (r + b);
    } else {
        double Pre = B1 * exp(-pos.z * pos.z / Hc / Hc) * R / r1 * (3 * r / r1 - 2 * r * r / r1 / r1) * cosV;
        Br = Pre;
        Bphi = 1 + 6 * (r - r1) / (2 * r - 3 * r1) * (sin(v + m * phi) - sin(v)) / cosV;
        Bphi *= -Pre * r / eta / (r + b);
    }
    return mk(Br * cos(phi) - Bphi * sin(phi), Br * sin(phi) + Bphi * cos(phi), 0);
}

/* getField (CMZField.cpp:289): getMCField (:116), getICField (:202),
 * getNTFField (:214), getRadioArcField (:273) */
static v3 cmz_field(const crp_cmz_desc *M, v3 pos) {
    v3 out = mk(0, 0, 0);
    if (M->use_mc) {
        v3 b = mk(0, 0, 0);
        for (int i = 0; i < 12; i++) b = add(b, cmz_baz(&M->clouds[i], pos));
        double x = pos.x + M->sgra_shift[0], y = pos.y + M->sgra_shift[1], z = pos.z + M->sgra_shift[2];
        double R = M->sgra_r, B1 = M->sgra_b1;
        double Hc = R / sqrt(log(2));
        double r = sqrt(x * x + y * y);
        double r1 = R / 10;
        double phi = atan2(y, x);
        double Bphi;
        if (r > r1)
            Bphi = -B1 * exp(-z * z / Hc / Hc) * R / r;
        else
            Bphi = -B1 * exp(-z * z / Hc / Hc) * R / r1 * (3 * r / r1 - 2 * r * r / r1 * r1);
        b.x -= Bphi * sin(phi);
        b.y += Bphi * cos(phi);
        out = add(out, muls(b, M->gauss));
    }
    if (M->use_ic) out = add(out, cmz_bpol(&M->ic, pos));
    if (M->use_ntf) {
        v3 b = mk(0, 0, 0);
        for (int i = 0; i < 6; i++) b = add(b, cmz_bpol(&M->ntf[i], pos));
        v3 pel = cmz_bpol(&M->ntf[6], pos);
        b.x += pel.x;
        b.y += pel.z;
        b.z += pel.y;
        out = add(out, muls(b, M->gauss));
    }
    if (M->use_radio_arc) out = add(out, muls(cmz_bpol(&M->radio_arc, pos), M->gauss));
    return out;
}

static v3 component_field(const crp_field_component *f, v3 position) {
    v3 pos = position;
    if (f->periodic) { /* MagneticField.cpp:41 */
        v3 o = mk(f->periodic_origin[0], f->periodic_origin[1], f->periodic_origin[2]);
        v3 e = mk(f->periodic_extends[0], f->periodic_extends[1], f->periodic_extends[2]);
        v3 n = vfloor(divv(sub(position, o), e));
        v3 p = sub(sub(position, o), mulv(n, e));
        if (f->periodic_reflective) {
            if ((long)fabs(n.x) % 2 == 1) p.x = e.x - p.x;
            if ((long)fabs(n.y) % 2 == 1) p.y = e.y - p.y;
            if ((long)fabs(n.z) % 2 == 1) p.z = e.z - p.z;
        }
        pos = p;
    }
    switch (f->kind) {
    case CRP_FIELD_GRID: return grid_field(&f->grid, pos);
    case CRP_FIELD_MODULATED_GRID: { /* ModulatedMagneticFieldGrid::getField, MagneticFieldGrid.cpp:51 */
        float m = scalar_grid(&f->modulation, pos);
        return muls(grid_field(&f->grid, pos), (double)m);
    }
    case CRP_FIELD_PLANE_WAVE: return plane_wave_field(&f->plane_wave, pos);
    case CRP_FIELD_UNIFORM: return mk(f->uniform[0], f->uniform[1], f->uniform[2]);
    case CRP_FIELD_JF12: return jf12_field(f, pos);
    case CRP_FIELD_UF23: return uf23_field(&f->uf23, pos);
    case CRP_FIELD_PT11: return pt11_field(&f->pt11, pos);
    case CRP_FIELD_ARCHIMEDEAN_SPIRAL: return archimedean_field(&f->archimedean, pos);
    case CRP_FIELD_TF17: return tf17_field(&f->tf17, pos);
    case CRP_FIELD_SINGLE_MODE: return single_mode_field(&f->single_mode, pos);
    case CRP_FIELD_KST24: return kst24_field(&f->kst24, pos);
    case CRP_FIELD_CMZ: return cmz_field(&f->cmz, pos);
    case CRP_FIELD_TOROIDAL: {
        double r = sqrt(pos.x * pos.x + pos.y * pos.y);
        return muls(mk(-pos.y, pos.x, 0.), f->toroidal_b0 / r);
    }
    }
    return mk(0, 0, 0);
}

/* MagneticFieldList::getField (MagneticField.cpp:64) or the single field. */
static v3 field_at(const crp_plan_desc *d, v3 pos) {
    if (d->n_fields == 1) return component_field(&d->fields[0], pos);
    v3 b = mk(0, 0, 0);
    for (int i = 0; i < d->n_fields; i++) b = add(b, component_field(&d->fields[i], pos));
    return b;
}

int oracle_field_eval(const crp_plan_desc *d, uint64_t n, const double *pos, double *out) {
    for (uint64_t i = 0; i < n; i++) {
        v3 b = field_at(d, mk(pos[i], pos[n + i], pos[2 * n + i]));
        out[i] = b.x; out[n + i] = b.y; out[2 * n + i] = b.z;
    }
    return 0;
}

/* PlaneWaveTurbulence constructor (PlaneWaveTurbulence.cpp:79-229) with
 * TurbulenceSpectrum::energySpectrum (TurbulentField.h:75). */
int oracle_plane_wave_modes(double brms, double lmin, double lmax, double lbendover,
                            double sindex, double qindex, int nm, uint32_t seed, double *xi,
                            double *kappa, double *k, double *beta, double *ak) {
    if (nm <= 1) return 1;
    mt_t r;
    oracle_mt_seed(&r, seed);
    double kmax = 2 * M_PI / lmin, kmin = 2 * M_PI / lmax;
    double delta = log10(kmax / kmin);
    for (int i = 0; i < nm; i++)
        k[i] = pow(10, log10(kmin) + ((double)i) / ((double)(nm - 1)) * delta);
    double delta_k0 = (k[1] - k[0]) / k[1];
    double sum = 0;
    for (int i = 0; i < nm; i++) {
        double kk = k[i];
        double kHat = kk * lbendover;
        double kh = kk * lbendover;
        double es = pow(kh, qindex) / pow(1.0 + kh * kh, (sindex + qindex) / 2.0 + 1.0);
        double Gk = es * (1 + kHat * kHat);
        ak[i] = Gk * delta_k0 * kk;
        sum += ak[i];
        double phi = mt_uniform(&r, -M_PI, M_PI);
        double costheta = mt_uniform(&r, -1., 1.);
        double sintheta = sqrt(1 - costheta * costheta);
        double alpha = mt_uniform(&r, 0, 2 * M_PI);
        double b = mt_uniform(&r, 0, 2 * M_PI);
        kappa[3*i] = sintheta * cos(phi);
        kappa[3*i+1] = sintheta * sin(phi);
        kappa[3*i+2] = costheta;
        xi[3*i] = costheta * cos(phi) * cos(alpha) + sin(phi) * sin(alpha);
        xi[3*i+1] = costheta * sin(phi) * cos(alpha) - cos(phi) * sin(alpha);
        xi[3*i+2] = -sintheta * cos(alpha);
        beta[i] = b;
    }
    for (int i = 0; i < nm; i++) ak[i] = sqrt(2 * ak[i] / sum) * brms;
    return 0;
}

/* ------------------------------------------------------------------------
 * Candidate (Candidate.cpp) and the modules
 * ---------------------------------------------------------------------- */
typedef struct {
    v3 pos, dir, prev;
    double E, q, len, time, cur, next, maxlen;
    int32_t id;
    int active;
    uint32_t flags;
    uint64_t index, steps;
} cand_t;

static void set_current_step(cand_t *c, double s) { /* Candidate.cpp:92 */
    c->cur = s;
    c->len += s;
    c->time += s / c_light;
}
static void limit_next_step(cand_t *c, double s) { c->next = dmin(c->next, s); } /* :102 */

/* PropagationBP::dY (PropagationBP.cpp:19) */
static void bp_dy(const crp_plan_desc *d, v3 *pos, v3 *dir, double step, double q, double m) {
    v3 x = *pos, u = *dir;
    x = add(x, divs(muls(u, step), 2.));
    v3 B = field_at(d, x);
    v3 t = divs(muls(divs(divs(muls(B, q), 2), m), step), c_light);
    v3 s = divs(muls(t, 2), (1 + dot(t, t)));
    v3 vh = add(u, cross(u, t));
    u = add(u, cross(vh, s));
    x = add(x, divs(muls(u, step), 2.));
    *pos = x; *dir = u;
}

/* PropagationBP::process (PropagationBP.cpp:62) */
static void bp_process(const crp_plan_desc *d, const crp_module_desc *m, cand_t *c, uint64_t *tries) {
    c->prev = c->pos;
    double q = c->q, step = m->max_step;
    if (q == 0) {
        step = clipd(c->next, m->min_step, m->max_step);
        c->pos = add(c->pos, muls(c->dir, step));
        set_current_step(c, step);
        c->next = m->max_step;
        return;
    }
    double newStep = step;
    double mass = c->E / (c_light * c_light);
    v3 xo = c->pos, uo = c->dir;
    if (m->min_step == m->max_step) {
        bp_dy(d, &xo, &uo, step, q, mass);
        (*tries)++;
    } else {
        step = clipd(c->next, m->min_step, m->max_step);
        newStep = step;
        while (1) {
            v3 x1 = c->pos, u1 = c->dir, xh = c->pos, uh = c->dir;
            bp_dy(d, &x1, &u1, step, q, mass);           /* tryStep :8 */
            bp_dy(d, &xh, &uh, step / 2, q, mass);
            bp_dy(d, &xh, &uh, step / 2, q, mass);
            (*tries)++;
            double S = norm(sub(x1, xh)) / (step * (1 - 1 / 4.)); /* :152 */
            xo = x1; uo = u1;
            double r = norm(mk(S, S, S)) / m->tolerance;
            if (r > 1) {
                if (step == m->min_step) break;
                newStep = step * 0.95 * ORACLE_POW(r, -0.2);
                newStep = dmax(newStep, 0.1 * step);
                newStep = dmax(newStep, m->min_step);
                step = newStep;
            } else {
                if (step != m->max_step) {
                    newStep = step * 0.95 * ORACLE_POW(r, -0.2);
                    newStep = dmin(newStep, 5 * step);
                    newStep = dmin(newStep, m->max_step);
                }
                break;
            }
        }
    }
    c->pos = xo;
    v3 u = unit(uo);
    c->dir = divs(u, norm(u)); /* ParticleState::setDirection */
    set_current_step(c, step);
    c->next = newStep;
}

/* Cash-Karp tableau (PropagationCK.cpp:11-26) */
static const double ck_a[36] = {
    0., 0., 0., 0., 0., 0.,
    1. / 5., 0., 0., 0., 0., 0.,
    3. / 40., 9. / 40., 0., 0., 0., 0.,
    3. / 10., -9. / 10., 6. / 5., 0., 0., 0.,
    -11. / 54., 5. / 2., -70. / 27., 35. / 27., 0., 0.,
    1631. / 55296., 175. / 512., 575. / 13824., 44275. / 110592., 253. / 4096., 0.};
static const double ck_b[6] = {37. / 378., 0, 250. / 621., 125. / 594., 0., 512. / 1771.};
static const double ck_bs[6] = {2825. / 27648., 0., 18575. / 48384., 13525. / 55296.,
                                277. / 14336., 1. / 4.};

/* PropagationCK::tryStep / dYdt (PropagationCK.cpp:28, :51) */
static void ck_try(const crp_plan_desc *d, v3 x, v3 u, double h, double q, double E,
                   v3 *xo, v3 *uo, v3 *ex, v3 *eu) {
    v3 kx[6], ku[6];
    *xo = x; *uo = u;
    *ex = mk(0, 0, 0); *eu = mk(0, 0, 0);
    for (int i = 0; i < 6; i++) {
        v3 yx = x, yu = u;
        for (int j = 0; j < i; j++) {
            yx = add(yx, muls(muls(kx[j], ck_a[i * 6 + j]), h));
            yu = add(yu, muls(muls(ku[j], ck_a[i * 6 + j]), h));
        }
        v3 vel = muls(unit(yu), c_light);
        v3 B = field_at(d, yx);
        v3 dudt = muls(cross(vel, B), q * c_light / E);
        kx[i] = vel; ku[i] = dudt;
        *xo = add(*xo, muls(muls(kx[i], ck_b[i]), h));
        *uo = add(*uo, muls(muls(ku[i], ck_b[i]), h));
        *ex = add(*ex, muls(muls(kx[i], ck_b[i] - ck_bs[i]), h));
        *eu = add(*eu, muls(muls(ku[i], ck_b[i] - ck_bs[i]), h));
    }
}

/* PropagationCK::process (PropagationCK.cpp:77) */
static void ck_process(const crp_plan_desc *d, const crp_module_desc *m, cand_t *c, uint64_t *tries) {
    c->prev = c->pos;
    double step = m->max_step;
    if (c->q == 0) {
        step = clipd(c->next, m->min_step, m->max_step);
        c->pos = add(c->pos, muls(c->dir, step));
        set_current_step(c, step);
        c->next = m->max_step;
        return;
    }
    v3 xo, uo, ex, eu;
    double newStep = step;
    if (m->min_step == m->max_step) {
        ck_try(d, c->pos, c->dir, step / c_light, c->q, c->E, &xo, &uo, &ex, &eu);
        (*tries)++;
    } else {
        step = clipd(c->next, m->min_step, m->max_step);
        newStep = step;
        while (1) {
            ck_try(d, c->pos, c->dir, step / c_light, c->q, c->E, &xo, &uo, &ex, &eu);
            (*tries)++;
            double r = norm(eu) / m->tolerance;
            if (r > 1) {
                if (step == m->min_step) break;
                newStep = step * 0.95 * ORACLE_POW(r, -0.2);
                newStep = dmax(newStep, 0.1 * step);
                newStep = dmax(newStep, m->min_step);
                step = newStep;
            } else {
                if (step != m->max_step) {
                    newStep = step * 0.95 * ORACLE_POW(r, -0.2);
                    newStep = dmin(newStep, 5 * step);
                    newStep = dmin(newStep, m->max_step);
                }
                break;
            }
        }
    }
    c->pos = xo;
    v3 u = unit(uo);
    c->dir = divs(u, norm(u));
    set_current_step(c, step);
    c->next = newStep;
}

/* DiffusionSDE::tryStep (DiffusionSDE.cpp:233) */
static void sde_try(const crp_plan_desc *d, v3 PosIn, v3 *POut, v3 *PosErr, double propStep) {
    v3 k[6];
    *POut = PosIn;
    for (int i = 0; i < 6; i++) {
        v3 y_n = PosIn;
        for (int j = 0; j < i; j++) y_n = add(y_n, muls(muls(k[j], ck_a[i * 6 + j]), propStep));
        v3 B = field_at(d, y_n);
        k[i] = muls(unit(B), c_light);
        *POut = add(*POut, muls(muls(k[i], ck_b[i]), propStep));
        *PosErr = add(*PosErr, divs(muls(muls(k[i], ck_b[i] - ck_bs[i]), propStep), kpc_unit));
    }
}

/* ------------------------------------------------------------ AdvectionField
 * getField of the advection fields (AdvectionField.cpp:12-460), glibc's libm
 * as the reference calls it. */
/* pow_integer<8> (Common.h:58) */
static double adv_pow8(double x) {
    double c = x * x, d = c * c;
    return (1 * (d * d));
}

static v3 advection_one(const crp_advection_desc *A, v3 pos, double time) {
    switch (A->kind) {
    case CRP_ADVECTION_TIME_SHOCK: { /* TimeDependentAdvectionField.cpp:16 */
        double Aa = 0.5 * (A->v1 + A->v0);
        double B = 0.5 * (A->v1 - A->v0);
        double x = pos.x;
        double xsh = A->v * (time - A->t0) + A->x0;
        v3 v = mk(0, 0, 0);
        v.x = Aa - B * tanh((x - xsh) / A->length);
        return v;
    }
    case CRP_ADVECTION_SEDOV_TAYLOR: { /* TimeDependentAdvectionField.cpp:103 */
        double r = norm(pos);
        v3 e_r = unit(pos);
        if (time == 0) return muls(e_r, 0.);
        double Aa = A->density;
        double R = pow(A->energy / Aa, 1. / 5.) * pow(time, 2. / 5.);
        double vs = 2. / 5. * pow(A->energy / Aa, 1. / 5.) * pow(time, -3. / 5.);
        double xi = r / R;
        double V = 3 * (adv_pow8(xi) + 1) / (3 * adv_pow8(xi) + 5);
        double u = 0.5 * xi * vs * V * (1 - tanh((xi - 1) * R / A->length));
        return muls(e_r, u);
    }
    case CRP_ADVECTION_UNIFORM: /* :33 */
        return mk(A->value[0], A->value[1], A->value[2]);
    case CRP_ADVECTION_CONSTANT_SPHERICAL: { /* :54 */
        v3 P = sub(pos, mk(A->origin[0], A->origin[1], A->origin[2]));
        v3 u = unit(P);
        return mk(A->v * u.x, A->v * u.y, A->v * u.z);
    }
    case CRP_ADVECTION_SPHERICAL: { /* :101, getV :120 */
        v3 P = sub(pos, mk(A->origin[0], A->origin[1], A->origin[2]));
        double R = norm(P);
        if (R > A->radius) return mk(0, 0, 0);
        double vR = A->v * (1 - exp(-(pow(R, A->alpha) / A->tau)));
        v3 u = unit(P);
        return mk(vR * u.x, vR * u.y, vR * u.z);
    }
    case CRP_ADVECTION_CARTESIAN_SHOCK: /* :188 */
    case CRP_ADVECTION_OBLIQUE_SHOCK: { /* :359 */
        double vDown = A->v / A->compression;
        double a = (A->v + vDown) * 0.5, b = (A->v - vDown) * 0.5;
        v3 v = mk(0, 0, 0);
        v.x = a - b * tanh(pos.x / A->length);
        if (A->kind == CRP_ADVECTION_OBLIQUE_SHOCK) v.y = A->vy;
        return v;
    }
    case CRP_ADVECTION_SPHERICAL_SHOCK_1D: { /* :254 */
        double r = norm(pos);
        v3 e_r = unit(pos);
        double vDown = A->v / A->compression;
        double a = (A->v + vDown) * 0.5, b = (A->v - vDown) * 0.5;
        double v;
        if (A->cool_upstream) {
            if (r <= A->radius) v = a - b * tanh((r - A->radius) / A->length);
            else v = (a - b * tanh((r - A->radius) / A->length)) * (A->radius / r) * (A->radius / r);
        } else {
            v = (a - b * tanh((r - A->radius) / A->length)) * (A->radius / r) * (A->radius / r);
        }
        return mk(v * e_r.x, v * e_r.y, v * e_r.z);
    }
    default: { /* CRP_ADVECTION_SPHERICAL_SHOCK, :441; g :463 */
        v3 R = sub(pos, mk(A->origin[0], A->origin[1], A->origin[2]));
        v3 e_r = unit(R);
        double phi = ((fabs(R.x) < DBL_MIN) && (fabs(R.y) < DBL_MIN)) ? 0.0 : atan2(R.y, R.x);
        v3 e_phi = mk(-sin(phi), cos(phi), 0);
        double r = norm(R);
        double g = 1. / (1 + exp(-((r - A->radius) / A->length)));
        double v_r = A->v * (1 + (pow(A->radius / (2 * r), 2.) - 1) * g);
        double v_p = A->v_phi * (A->r_rot / r);
        return add(muls(e_r, v_r), muls(e_phi, v_p));
    }
    }
}

/* DiffusionSDE::driftStep (DiffusionSDE.cpp:255): LinProp = 0 + v(pos) h;
 * several fields are an AdvectionFieldList (:12), summed in order. */
static v3 sde_lin_prop(const crp_module_desc *m, v3 pos, double h, double time) {
    if (m->n_advection == 0) return mk(0, 0, 0);
    v3 v;
    if (m->n_advection == 1) {
        v = advection_one(&m->advection[0], pos, time);
    } else { /* AdvectionFieldList::getField passes no time: 0 */
        v = mk(0, 0, 0);
        for (int i = 0; i < m->n_advection; i++) v = add(v, advection_one(&m->advection[i], pos, 0.));
    }
    return add(mk(0, 0, 0), muls(v, h));
}

/* DiffusionSDE::process (DiffusionSDE.cpp:47) with the advection drift of
 * driftStep. */
static void sde_process(const crp_plan_desc *d, const crp_module_desc *m, cand_t *c, uint64_t *tries) {
    c->prev = c->pos;
    double h = clipd(c->next, m->min_step, m->max_step) / c_light;
    v3 PosIn = c->pos, DirIn = c->dir;
    (void)DirIn;
    double time = c->time; /* candidate->getTime() at the step's start */
    if (c->q == 0) {
        c->pos = add(add(c->pos, sde_lin_prop(m, PosIn, h, time)), muls(muls(c->dir, h), c_light));
        set_current_step(c, h * c_light);
        c->next = m->max_step;
        return;
    }
    double rig = c->E / c->q;
    double DifCoeff = m->sde_scale * 6.1e24 * ORACLE_POW((fabs(rig) / 4.0e9), m->sde_alpha);
    double BT0 = ORACLE_POW(2 * DifCoeff, 0.5);
    double BT4 = ORACLE_POW(2 * m->sde_epsilon * DifCoeff, 0.5);
    double BT8 = BT4;
    stream_t s = {d->seed, c->index, c->steps, {{0, 0, 0, 0}}, 0};
    double eta0 = stream_norm(&s), eta1 = stream_norm(&s), eta2 = stream_norm(&s);
    double TStep = BT0 * eta0, NStep = BT4 * eta1, BStep = BT8 * eta2;
    double propTime = TStep * sqrt(h) / c_light;
    size_t counter = 0;
    double r = 42.;
    do {
        v3 PosOut = mk(0, 0, 0), PosErr = mk(0, 0, 0);
        sde_try(d, PosIn, &PosOut, &PosErr, propTime);
        (*tries)++;
        r = norm(PosErr) / m->tolerance;
        propTime *= 0.5;
        counter += 1;
    } while (r > 1 && fabs(propTime) >= m->min_step / c_light);
    size_t stepNumber = (size_t)pow(2, (double)(counter - 1));
    double allowedTime = TStep * sqrt(h) / c_light / (double)stepNumber;
    v3 Start = PosIn, PosOut = mk(0, 0, 0), PosErr = mk(0, 0, 0);
    for (size_t j = 0; j < stepNumber; j++) {
        sde_try(d, Start, &PosOut, &PosErr, allowedTime);
        (*tries)++;
        Start = PosOut;
    }
    v3 TVec = unit(sub(PosOut, PosIn));
    double tTest = norm(TVec);
    if (tTest != tTest) {
        if (m->n_advection) c->pos = add(c->pos, sde_lin_prop(m, PosIn, h, time));  /* advection only */
        else c->pos = add(c->pos, muls(muls(c->dir, h), c_light));
        set_current_step(c, h * c_light);
        double newStep = 5 * h * c_light;
        c->next = clipd(newStep, m->min_step, m->max_step);
        return;
    }
    v3 NVec = mk(0, 0, 0);
    int guard = 0;
    while (norm(NVec) == 0. && guard < 3) { NVec = cross(TVec, stream_vector(&s)); guard++; }
    if (norm(NVec) == 0.) { c->active = 0; c->flags |= CRP_FLAG_NAN; return; }
    NVec = unit(NVec);
    v3 BVec = unit(cross(TVec, NVec));
    v3 PO = add(add(PosOut, sde_lin_prop(m, PosIn, h, time)), muls(add(muls(NVec, NStep), muls(BVec, BStep)), sqrt(h)));
    if (isnan(norm(PO))) { c->active = 0; c->flags |= CRP_FLAG_NAN; return; }
    s.cursor = 12; /* the cone draw uses the fourth block of the step */
    v3 DirOut = stream_cone(&s, TVec, M_PI / 2.);
    c->pos = PO;
    c->dir = divs(DirOut, norm(DirOut));
    set_current_step(c, h * c_light);
    double nextStep;
    if (stepNumber > 1) nextStep = h * pow((double)stepNumber, -2.) * c_light;
    else nextStep = 4 * h * c_light;
    c->next = nextStep;
}

typedef struct {
    crp_records *rec;
} rec_ctx;

static void write_record(crp_records *rec, const cand_t *c, int module) {
    if (!rec) return;
    uint64_t slot;
#ifdef _OPENMP
#pragma omp atomic capture
#endif
    slot = (*rec->count)++;
    if (slot >= rec->capacity) return;
    rec->index[slot] = c->index;
    rec->module[slot] = module;
    rec->trajectory_length[slot] = c->len;
    rec->time[slot] = c->time;
    rec->x[slot] = c->pos.x; rec->y[slot] = c->pos.y; rec->z[slot] = c->pos.z;
    rec->dx[slot] = c->dir.x; rec->dy[slot] = c->dir.y; rec->dz[slot] = c->dir.z;
    rec->energy[slot] = c->E;
    rec->id[slot] = c->id;
}

static double std_min(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double std_max(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* ParticleID.cpp:37 isNucleus: the neutron, and HepPID::isNucleus
 * (ParticleIDMethods.cc:242): the proton, or +/-10LZZZAAAI with A >= Z. */
static int is_nucleus(int id) {
    if (id == 2112) return 1;
    int a = id < 0 ? -id : id;
    if (a == 2212) return 1;
    if ((a / 1000000000) % 10 == 1 && (a / 100000000) % 10 == 0)
        return (a / 10) % 1000 >= (a / 10000) % 1000;
    return 0;
}

/* Sphere / Plane / ParaxialBox ::distance (Geometry.cpp:41, 19, 64). */
static double surface_distance(const crp_observer_feature_desc *f, v3 p) {
    v3 a = mk(f->a[0], f->a[1], f->a[2]);
    if (f->kind == CRP_OBSERVER_SURFACE_SPHERE) return norm(sub(p, a)) - f->r;
    v3 dX = sub(p, a);
    if (f->kind == CRP_OBSERVER_SURFACE_PLANE) return f->b[0] * dX.x + f->b[1] * dX.y + f->b[2] * dX.z;
    double hx = f->b[0] / 2., hy = f->b[1] / 2., hz = f->b[2] / 2.;
    double X = dX.x - hx, Y = dX.y - hy, Z = dX.z - hz;
    if ((fabs(X) <= hx) && (fabs(Y) <= hy) && (fabs(Z) <= hz)) {
        double d = std_min(hx - fabs(X), std_min(hy - fabs(Y), hz - fabs(Z)));
        return -1. * d;
    }
    double qa = std_max(0., fabs(X) - hx), qb = std_max(0., fabs(Y) - hy), qc = std_max(0., fabs(Z) - hz);
    return sqrt(qa * qa + qb * qb + qc * qc);
}

enum { DET_NOTHING = 0, DET_DETECTED = 1, DET_VETO = 2 };

/* ObserverFeature::checkDetection of each feature (Observer.cpp:93-394). */
static int check_feature(const crp_observer_feature_desc *f, cand_t *c) {
    int a;
    switch (f->kind) {
    case CRP_OBSERVER_SURFACE_SPHERE:
    case CRP_OBSERVER_SURFACE_PLANE:
    case CRP_OBSERVER_SURFACE_BOX: { /* ObserverSurface, Observer.cpp:394 */
        double cd = surface_distance(f, c->pos), pd = surface_distance(f, c->prev);
        limit_next_step(c, fabs(cd));
        if (cd * pd > 0) return DET_NOTHING;
        if (pd == 0) return DET_NOTHING;
        return DET_DETECTED;
    }
    case CRP_OBSERVER_DETECT_ALL: return DET_DETECTED; /* :93 */
    case CRP_OBSERVER_TRACKING: { /* :109 */
        double d = norm(sub(c->pos, mk(f->a[0], f->a[1], f->a[2])));
        if (d > f->r) {
            limit_next_step(c, fabs(d - f->r));
            return DET_NOTHING;
        }
        limit_next_step(c, f->step);
        return DET_DETECTED;
    }
    case CRP_OBSERVER_1D: /* :137 */
        if (c->pos.x > 0) {
            limit_next_step(c, c->pos.x);
            return DET_NOTHING;
        }
        return DET_DETECTED;
    case CRP_OBSERVER_INACTIVE_VETO: return c->active ? DET_NOTHING : DET_VETO; /* :174 */
    case CRP_OBSERVER_NUCLEUS_VETO: return is_nucleus(c->id) ? DET_VETO : DET_NOTHING; /* :185 */
    case CRP_OBSERVER_NEUTRINO_VETO: /* :196 */
        a = c->id < 0 ? -c->id : c->id;
        return (a == 12 || a == 14 || a == 16) ? DET_VETO : DET_NOTHING;
    case CRP_OBSERVER_PHOTON_VETO: return c->id == 22 ? DET_VETO : DET_NOTHING; /* :208 */
    case CRP_OBSERVER_ELECTRON_VETO: return (c->id == 11 || c->id == -11) ? DET_VETO : DET_NOTHING;
    default: return c->id == f->particle_id ? DET_VETO : DET_NOTHING; /* :234 */
    }
}

/* Observer::process (Observer.cpp:27-52); the single legacy feature when
 * n_features is 0. */
static void observer_process(const crp_module_desc *m, cand_t *c, crp_records *rec, int i) {
    crp_observer_feature_desc legacy;
    memset(&legacy, 0, sizeof(legacy));
    legacy.kind = m->observer_feature;
    memcpy(legacy.a, m->sphere_center, sizeof(legacy.a));
    legacy.r = m->sphere_radius;
    const crp_observer_feature_desc *fs = m->n_features > 0 ? m->features : &legacy;
    int nf = m->n_features > 0 ? m->n_features : 1;
    int state = DET_NOTHING;
    for (int f = 0; f < nf; f++) {
        int st = check_feature(&fs[f], c);
        if (st == DET_VETO) state = DET_VETO;
        else if (st == DET_DETECTED && state != DET_VETO) state = DET_DETECTED;
    }
    if (state == DET_DETECTED) {
        if (m->record) write_record(rec, c, i);
        c->flags |= CRP_FLAG_DETECTED;
        if (m->deactivate_on_detection) c->active = 0;
    }
}

static void reject_candidate(const crp_module_desc *m, cand_t *c, crp_records *rec, int i) {
    if (m->record) write_record(rec, c, i); /* AbstractCondition::reject, Module.cpp:25 */
    c->flags |= CRP_FLAG_REJECTED;
    c->active = 0;
}

/* CubicBoundary / SphericalBoundary / EllipsoidalBoundary /
 * CylindricalBoundary ::process (Boundary.cpp:171, 216, 259, 303). */
static void boundary_process(const crp_module_desc *m, cand_t *c, crp_records *rec, int i) {
    v3 a = mk(m->boundary_a[0], m->boundary_a[1], m->boundary_a[2]);
    if (m->boundary == CRP_BOUNDARY_CUBIC) {
        v3 r = sub(c->pos, a);
        double lo = std_min(r.x, std_min(r.y, r.z)), hi = std_max(r.x, std_max(r.y, r.z));
        if ((lo <= 0) || (hi >= m->boundary_size)) reject_candidate(m, c, rec, i);
        if (m->boundary_limit_step) {
            limit_next_step(c, lo + m->boundary_margin);
            limit_next_step(c, m->boundary_size - hi + m->boundary_margin);
        }
    } else if (m->boundary == CRP_BOUNDARY_SPHERICAL) {
        double d = norm(sub(c->pos, a));
        if (d >= m->boundary_size) reject_candidate(m, c, rec, i);
        if (m->boundary_limit_step) limit_next_step(c, m->boundary_size - d + m->boundary_margin);
    } else if (m->boundary == CRP_BOUNDARY_ELLIPSOIDAL) {
        v3 b = mk(m->boundary_b[0], m->boundary_b[1], m->boundary_b[2]);
        double d = norm(sub(c->pos, a)) + norm(sub(c->pos, b));
        if (d >= m->boundary_size) reject_candidate(m, c, rec, i);
        if (m->boundary_limit_step) limit_next_step(c, m->boundary_size - d + m->boundary_margin);
    } else {
        v3 d = sub(c->pos, a);
        double R2 = ORACLE_POW(d.x, 2.) + ORACLE_POW(d.y, 2.);
        double Z = fabs(d.z);
        if (R2 < ORACLE_POW(m->boundary_radius, 2.) && Z < m->boundary_size / 2.) {
            if (m->boundary_limit_step)
                limit_next_step(c, std_min(m->boundary_radius - ORACLE_POW(R2, 0.5), m->boundary_size / 2. - Z) +
                                       m->boundary_margin);
            return;
        }
        reject_candidate(m, c, rec, i);
    }
}

/* One ModuleList::process (ModuleList.cpp.in:54): every module in order. */
static void chain_process(const crp_plan_desc *d, cand_t *c, crp_records *rec, uint64_t *tries) {
    for (int i = 0; i < d->n_modules; i++) {
        const crp_module_desc *m = &d->modules[i];
        if (m->kind == CRP_MODULE_PROPAGATION) {
            if (m->propagator == CRP_PROP_BP) bp_process(d, m, c, tries);
            else if (m->propagator == CRP_PROP_CK) ck_process(d, m, c, tries);
            else sde_process(d, m, c, tries);
        } else if (m->kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH) { /* BreakCondition.cpp:42 */
            double maxLength = m->per_candidate_length ? c->maxlen : m->max_length;
            if (c->len >= maxLength) {
                if (m->record) write_record(rec, c, i);
                c->flags |= CRP_FLAG_REJECTED;  /* AbstractCondition::reject, Module.cpp:25 */
                c->active = 0;
            } else {
                limit_next_step(c, maxLength - c->len);
            }
        } else if (m->kind == CRP_MODULE_OBSERVER) { /* Observer.cpp:27 */
            observer_process(m, c, rec, i);
        } else if (m->kind == CRP_MODULE_BOUNDARY) {
            boundary_process(m, c, rec, i);
        }
    }
}

/* ModuleList::run(candidate_vector) (ModuleList.cpp.in:97) over the arrays:
 * each active candidate is processed until inactive, or until it has taken
 * max_steps steps in this call (0: no cap). */
int oracle_run(const crp_plan_desc *d, const crp_candidates *a, uint64_t n, crp_records *rec,
               int nthreads, uint64_t max_steps, uint64_t *steps_out, uint64_t *tries_out) {
    uint64_t steps = 0, tries = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : steps, tries)
#endif
    for (int64_t ii = 0; ii < (int64_t)n; ii++) {
        uint64_t i = (uint64_t)ii;
        cand_t c;
        c.pos = mk(a->x[i], a->y[i], a->z[i]);
        c.dir = mk(a->dx[i], a->dy[i], a->dz[i]);
        c.prev = mk(a->px[i], a->py[i], a->pz[i]);
        c.E = a->energy[i]; c.q = a->charge[i]; c.id = a->id[i];
        c.len = a->trajectory_length[i]; c.time = a->time[i];
        c.cur = a->current_step[i]; c.next = a->next_step[i];
        c.maxlen = a->max_length ? a->max_length[i] : 0;
        c.active = a->active[i] != 0; c.flags = a->flags[i];
        c.index = i;
        c.steps = a->step_count ? a->step_count[i] : 0;
        uint64_t taken = 0, t = 0;
        while (c.active && (max_steps == 0 || taken < max_steps)) {
            chain_process(d, &c, rec, &t);
            c.steps++;
            taken++;
        }
        steps += taken;
        tries += t;
        a->x[i] = c.pos.x; a->y[i] = c.pos.y; a->z[i] = c.pos.z;
        a->dx[i] = c.dir.x; a->dy[i] = c.dir.y; a->dz[i] = c.dir.z;
        a->px[i] = c.prev.x; a->py[i] = c.prev.y; a->pz[i] = c.prev.z;
        a->trajectory_length[i] = c.len; a->time[i] = c.time;
        a->current_step[i] = c.cur; a->next_step[i] = c.next;
        a->active[i] = (uint8_t)c.active; a->flags[i] = c.flags;
        if (a->step_count) a->step_count[i] = c.steps;
    }
    if (steps_out) *steps_out = steps;
    if (tries_out) *tries_out = tries;
    return 0;
}

/* ------------------------------------------------------------------------
 * Adjoint of the fixed-step Boris push (no reference counterpart)
 *
 * Forward model (the differentiable one): PropagationBP::dY
 * (PropagationBP.cpp:19) with the Grid3f values taken as doubles and the
 * trilinear weights in double (the corner order of Grid.h:571), then the
 * direction normalised.  Loss per candidate: 1 - u_final . target.
 * ---------------------------------------------------------------------- */
typedef struct {
    const float *g;
    int nx, ny, nz;
    double go[3], s[3];
} adj_grid_t;

static void adj_cell(const adj_grid_t *G, v3 x, size_t idx[8], double w[8], double dw[8][3]) {
    double r[3] = {(x.x - G->go[0]) / G->s[0], (x.y - G->go[1]) / G->s[1], (x.z - G->go[2]) / G->s[2]};
    int n[3] = {G->nx, G->ny, G->nz}, lo[3], hi[3];
    double f0[3], f1[3];
    for (int a = 0; a < 3; a++) {
        double fl = floor(r[a]);
        lo[a] = (((int)fl % n[a]) + n[a]) % n[a];
        hi[a] = (lo[a] + 1) % n[a];
        f0[a] = r[a] - fl;
        f1[a] = 1 - f0[a];
    }
    const int sel[8][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},{1,0,1},{0,1,1},{1,1,0},{1,1,1}};
    for (int k = 0; k < 8; k++) {
        int ix = sel[k][0] ? hi[0] : lo[0], iy = sel[k][1] ? hi[1] : lo[1], iz = sel[k][2] ? hi[2] : lo[2];
        idx[k] = ((size_t)ix * G->ny + (size_t)iy) * G->nz + (size_t)iz;
        double wx = sel[k][0] ? f0[0] : f1[0], wy = sel[k][1] ? f0[1] : f1[1], wz = sel[k][2] ? f0[2] : f1[2];
        double sx = (sel[k][0] ? 1.0 : -1.0) / G->s[0], sy = (sel[k][1] ? 1.0 : -1.0) / G->s[1],
               sz = (sel[k][2] ? 1.0 : -1.0) / G->s[2];
        w[k] = wx * wy * wz;
        dw[k][0] = sx * wy * wz;
        dw[k][1] = wx * sy * wz;
        dw[k][2] = wx * wy * sz;
    }
}

static v3 adj_field(const adj_grid_t *G, v3 x) {
    size_t idx[8];
    double w[8], dw[8][3];
    adj_cell(G, x, idx, w, dw);
    v3 B = mk(0, 0, 0);
    for (int k = 0; k < 8; k++) {
        const float *c = G->g + 3 * idx[k];
        B.x += w[k] * (double)c[0];
        B.y += w[k] * (double)c[1];
        B.z += w[k] * (double)c[2];
    }
    return B;
}

static void adj_step(const adj_grid_t *G, v3 *x, v3 *u, double hh, double kappa) {
    v3 x1 = add(*x, muls(*u, hh));
    v3 B = adj_field(G, x1);
    v3 t = muls(B, kappa);
    double D = 1 + dot(t, t);
    v3 s = muls(t, 2 / D);
    v3 v = add(*u, cross(*u, t));
    v3 u2 = add(*u, cross(v, s));
    *x = add(x1, muls(u2, hh));
    *u = divs(u2, norm(u2));
}

/* Loss and gradients for n candidates (position, direction, energy,
 * charge, target interleaved xyz): fixed step h, n_steps steps.  grad_grid
 * (3 doubles per cell) is accumulated (+=), may be NULL. */
int oracle_bp_adjoint(const float *grid, int nx, int ny, int nz, const double *origin,
                      const double *spacing, double h, int n_steps, uint64_t n, const double *pos,
                      const double *dir, const double *energy, const double *charge,
                      const double *target, double *loss, double *grad_dir, double *grad_energy,
                      double *grad_grid) {
    adj_grid_t G = {grid, nx, ny, nz,
                    {origin[0] + spacing[0] / 2, origin[1] + spacing[1] / 2, origin[2] + spacing[2] / 2},
                    {spacing[0], spacing[1], spacing[2]}};
    const double hh = h / 2;
    v3 *xs = (v3 *)malloc(sizeof(v3) * (size_t)(n_steps + 1));
    v3 *us = (v3 *)malloc(sizeof(v3) * (size_t)(n_steps + 1));
    if (!xs || !us) { free(xs); free(us); return 1; }
    for (uint64_t i = 0; i < n; i++) {
        double kappa = charge[i] * h * c_light / (2 * energy[i]);
        xs[0] = mk(pos[3*i], pos[3*i+1], pos[3*i+2]);
        us[0] = mk(dir[3*i], dir[3*i+1], dir[3*i+2]);
        for (int k = 0; k < n_steps; k++) {
            xs[k + 1] = xs[k]; us[k + 1] = us[k];
            adj_step(&G, &xs[k + 1], &us[k + 1], hh, kappa);
        }
        v3 tg = mk(target[3*i], target[3*i+1], target[3*i+2]);
        if (loss) loss[i] = 1 - dot(us[n_steps], tg);
        v3 xb = mk(0, 0, 0), ub = muls(tg, -1.0);
        double kb = 0;
        for (int k = n_steps - 1; k >= 0; k--) {
            v3 x = xs[k], u = us[k];
            /* recompute the step's intermediates */
            v3 x1 = add(x, muls(u, hh));
            size_t idx[8];
            double w[8], dw[8][3];
            adj_cell(&G, x1, idx, w, dw);
            v3 B = mk(0, 0, 0);
            for (int q = 0; q < 8; q++) {
                const float *c = G.g + 3 * idx[q];
                B.x += w[q] * (double)c[0]; B.y += w[q] * (double)c[1]; B.z += w[q] * (double)c[2];
            }
            v3 t = muls(B, kappa);
            double D = 1 + dot(t, t);
            v3 s = muls(t, 2 / D);
            v3 v = add(u, cross(u, t));
            v3 u2 = add(u, cross(v, s));
            double nn = norm(u2);
            v3 un = divs(u2, nn);
            /* reverse */
            v3 u2b = divs(sub(ub, muls(un, dot(un, ub))), nn);
            v3 x1b = xb;
            u2b = add(u2b, muls(xb, hh));
            v3 ubar = u2b;
            v3 vb = cross(s, u2b);
            v3 sb = cross(u2b, v);
            ubar = add(ubar, add(vb, cross(t, vb)));
            v3 tb = cross(vb, u);
            tb = add(tb, sub(muls(sb, 2 / D), muls(t, 4 * dot(t, sb) / (D * D))));
            v3 Bb = muls(tb, kappa);
            kb += dot(tb, B);
            for (int q = 0; q < 8; q++) {
                const float *c = G.g + 3 * idx[q];
                double gdot = Bb.x * (double)c[0] + Bb.y * (double)c[1] + Bb.z * (double)c[2];
                x1b.x += gdot * dw[q][0]; x1b.y += gdot * dw[q][1]; x1b.z += gdot * dw[q][2];
                if (grad_grid) {
                    grad_grid[3 * idx[q]] += w[q] * Bb.x;
                    grad_grid[3 * idx[q] + 1] += w[q] * Bb.y;
                    grad_grid[3 * idx[q] + 2] += w[q] * Bb.z;
                }
            }
            xb = x1b;
            ubar = add(ubar, muls(x1b, hh));
            ub = ubar;
        }
        grad_dir[3*i] = ub.x; grad_dir[3*i+1] = ub.y; grad_dir[3*i+2] = ub.z;
        /* kappa = q h c / (2E): d kappa / dE = -kappa / E */
        grad_energy[i] = kb * (-kappa / energy[i]);
    }
    free(xs);
    free(us);
    return 0;
}

/* Loss only, same forward model (for central finite differences). */
double oracle_bp_loss(const float *grid, int nx, int ny, int nz, const double *origin,
                      const double *spacing, double h, int n_steps, uint64_t n, const double *pos,
                      const double *dir, const double *energy, const double *charge,
                      const double *target) {
    adj_grid_t G = {grid, nx, ny, nz,
                    {origin[0] + spacing[0] / 2, origin[1] + spacing[1] / 2, origin[2] + spacing[2] / 2},
                    {spacing[0], spacing[1], spacing[2]}};
    double L = 0;
    for (uint64_t i = 0; i < n; i++) {
        double kappa = charge[i] * h * c_light / (2 * energy[i]);
        v3 x = mk(pos[3*i], pos[3*i+1], pos[3*i+2]), u = mk(dir[3*i], dir[3*i+1], dir[3*i+2]);
        for (int k = 0; k < n_steps; k++) adj_step(&G, &x, &u, h / 2, kappa);
        L += 1 - dot(u, mk(target[3*i], target[3*i+1], target[3*i+2]));
    }
    return L;
}
