// device_plan.cuh -- device-side description of a stepping plan and the
// candidate state layout.  Plain structs passed by value as kernel
// parameters (they live in the constant bank, so every lane reads them as a
// uniform broadcast).
#pragma once

#include <cstdint>

#include "crp_gpu.h"

namespace crp {

constexpr int kMaxFields = 4;
constexpr int kMaxModules = 8;
constexpr int kMaxFeatures = 8;  // observer features of all modules of a plan

struct DevGrid {
    const float *values;   // packed Vector3f cells, 12 B each (Grid.h:338 order)
    const float4 *values4; // the same cells padded to 16 B (mixed form), or null
    int nx, ny, nz;
    int reflective;
    int clip_volume;
    int pow2;              // nx, ny, nz all powers of two (periodic wrap by mask)
    double gox, goy, goz;  // gridOrigin = origin + spacing/2 (Grid.h:227)
    double sx, sy, sz;     // spacing
    double inv_sx, inv_sy, inv_sz;  // 1/spacing (mixed form only)
    double ox, oy, oz;     // origin (clipVolume test)
    double ex, ey, ez;     // origin + N*spacing (clipVolume test, Grid.h:322)
    int interp;            // crp_interpolation
    int pad_;
};

struct DevPlaneWave {
    const double *modes;   // FP64 form: per mode {xi x y z, kappa x y z, k, beta, Ak} (9 doubles)
    const float4 *pairs;   // mixed form: the modes in pairs, 80 B = 5 x 16 B per pair (step_mixed.cu)
    int n;                 // modes
    int npairs;            // (n + 1) / 2; an odd count ends with a zero-amplitude mode
    double fast_limit;     // mixed form: max(|x|, |y|, |z|) below which every scaled phase stays under 2^50
};

// JF12Field parameters (crp_jf12_desc, SI) for the FP64 form, and the same
// parameters as floats with lengths in kpc and fields in muG for the mixed
// form (positions of ~1e20 m would overflow FP32 squares).
struct DevJF12 {
    crp_jf12_desc d;
    double inv_kpc, muG;
    float rarms[8], bdisk[8], bdturb[8];
    float bring, hdisk, wdisk, bnorth, bsouth, rnorth, rsouth, whalo, z0;
    float bx, sinthx0, costhx0, tanthx0, rxc, rx, sinp, cosp, tan90mp, sqrtbeta;
    float bdturb5, zdturb, bhturb, rhturb, zhturb;
    // JF12FieldSolenoidal (variant CRP_JF12_SOLENOIDAL), kpc and muG
    float s_cotp, s_cotx, s_zs, s_r1, s_r2, s_r1s, s_r2s;
    float s_phi0[11], s_b[11], s_coeff[10];
};

// TF17Field parameters as floats in kpc and muG for the mixed form (the FP64
// form reads crp_tf17_desc).
struct DevTF17 {
    int disk_model, halo_model, use_disk, use_halo;
    float a_disk, z1_disk, r1_disk, b1_disk, l_disk, phi_star_disk, h_disk;
    float a_halo, z1_halo, b1_halo, l_halo, phi_star_halo;
    float cot_p0, h_p, l_p, eps;
    double inv_kpc;  // 1/kpc [1/m]
    float muG;       // [T]
};

// PT11Field parameters as floats in kpc and muG for the mixed form (the FP64
// form reads crp_pt11_desc), cot of the pitch formed once.
struct DevPT11 {
    int use_ass, use_bss, use_halo, pad;
    float r_sun, r_c, z0_d, b0_d, z0_h, r0_h, b0_hn, b0_hs, z11_h, z12_h;
    float sinp, cosp, cotp, phi, cos_phi;
    double inv_kpc;  // 1/kpc [1/m]
    float muG;       // [T]
};

// KST24Field parameters as floats in the model's units (kpc, gauss) for the
// mixed form, with each arm's trigonometric constants formed once.
struct DevKST24Arm {
    float b, k, cos_pitch, sin_pitch, phi0, arc_div, x_shift, y_shift;
    float arc_radius1, arc_radius2, arc_eps, rmin, rmax, zmin, zmax;
};
struct DevKST24 {
    float north_b, north_zmin, north_zmax, north_rmin, north_rmax;
    float south_b, south_zmin, south_zmax, south_rmin, south_rmax;
    float x_b, x_rmin, x_rmax, tan_x, sin_x, cos_x;
    float lb_b, lb_rmin, lb_dr, lb_x0, lb_y0, lb_z0, lb_dir[3], lb_ampl;
    DevKST24Arm arms[5];
    double inv_kpc;  // 1/kpc [1/m]
    float gauss;     // [T]
};

// UF23Field parameters with the two powers the poloidal halo recomputes at
// every call from model constants, evaluated once on the host with the C
// library's pow (the reference's own values).
struct DevUF23 {
    crp_uf23_desc d;
    double c_pol;  // pow(A / Z, P)
    double a0p;    // pow(A, P)
    // the mixed form's floats, same units (kpc, microgauss, radians)
    float b1, b2, b3, disk_h, disk_w, ph1, ph2, ph3, sinp, cosp, inv_tanp, tanp;
    float spur_center, spur_length, spur_inv_width;
    float tbn, tbs, tr, tw, tz;
    float pa, pb, pp, pr, pw, pzz, inv_pp;  // poloidal A, B, P, R, W, Z and 1/P
    float twist, r2max;
    float muG;       // [T]
    double inv_kpc;  // 1/kpc [1/m]
};

struct DevComponent {
    int kind;       // crp_field_kind
    int periodic;
    int periodic_reflective;
    int pad;
    double po[3], pe[3];
    DevGrid grid;
    DevPlaneWave pw;
    double uniform[3];
    double b0;
    DevGrid mod;    // CRP_FIELD_MODULATED_GRID: the Grid1f modulation (values: one float per cell);
                    // CRP_FIELD_JF12: the striated grid (grid: the turbulent grid)
    const DevJF12 *jf;  // CRP_FIELD_JF12: device copy of the parameters
    const DevUF23 *uf;        // CRP_FIELD_UF23: device copy of the parameters
    const crp_pt11_desc *pt;  // CRP_FIELD_PT11: device copy of the parameters
    const DevPT11 *pt32;      // and their float form (mixed)
    const crp_tf17_desc *tf;  // CRP_FIELD_TF17: device copy of the parameters
    const DevTF17 *tf32;      // and their float form (mixed)
    crp_single_mode_desc mode;  // CRP_FIELD_SINGLE_MODE
    const crp_kst24_desc *kst;  // CRP_FIELD_KST24: device copy of the parameters
    const DevKST24 *kst32;      // and their float form (mixed)
    const crp_cmz_desc *cmz;    // CRP_FIELD_CMZ: device copy of the switches and objects
    crp_archimedean_desc arch;  // CRP_FIELD_ARCHIMEDEAN_SPIRAL
};

struct DevModule {
    int kind;        // crp_module_kind
    int propagator;  // crp_propagator
    double tolerance, min_step, max_step;
    double eps, alpha, scale;
    int n_adv;                        // DiffusionSDE: advection fields, summed (0: none)
    const crp_advection_desc *adv;    // device copy of the n_adv descriptors
    double max_length;
    int per_candidate;
    int observer;    // crp_observer_feature
    double cx, cy, cz, radius;
    int deactivate;
    int record;
    int feat0, nfeat;      // observer: features feat0 .. feat0 + nfeat - 1 of DevPlan::feat
    int boundary;          // crp_boundary_kind
    int limit_step;        // boundary setLimitStep
    double bx, by, bz;     // boundary: a = (cx, cy, cz), b
    double bsize, bradius, margin;
};

// One observer feature (crp_observer_feature_desc).
struct DevFeature {
    int kind;
    int pid;
    double ax, ay, az;
    double bx, by, bz;
    double r, step;
};

// Module sequences the stepping kernels are compiled for: CS_PM =
// [propagation, MaximumTrajectoryLength], CS_PMO = [propagation,
// MaximumTrajectoryLength, Observer]; any other chain walks the module list
// (CS_GENERIC).  The plan records which one its chain matches.
enum ChainShape { CS_GENERIC = 0, CS_PM = 1, CS_PMO = 2 };

struct DevPlan {
    int n_fields;
    int n_modules;
    int prop_index;  // position of the propagation module in the chain
    int shape;       // ChainShape (chain.cuh) the module sequence matches
    uint64_t seed;
    DevComponent fields[kMaxFields];
    DevModule modules[kMaxModules];
    DevFeature feat[kMaxFeatures];
};

// Candidate arrays (include/crp_gpu.h crp_candidates), device pointers.
struct DevState {
    int32_t *id;
    double *charge, *energy;
    double *x, *y, *z;
    double *dx, *dy, *dz;
    double *px, *py, *pz;
    double *len, *time, *cur, *next;
    uint8_t *active;
    uint32_t *flags;
    double *max_length;
    uint64_t *steps;
};

struct DevRecords {
    uint64_t capacity;
    unsigned long long *count;
    uint64_t *index;
    int32_t *module;
    double *len, *time, *x, *y, *z, *dx, *dy, *dz, *energy;
    int32_t *id;
};

// Run counters, accumulated with one atomic per warp.
// Work queue of the persistent mode, in device memory so that a sequence of
// persistent launches with their bookkeeping can be captured in one CUDA
// graph: the pending list (candidates a launch left unfinished when its
// time budget ran out) is list `cur` (0: a, 1: b); the untouched main range
// is [main_base, main_base + n_main).  advance_kernel updates it between
// launches and accumulates the run totals.
struct DevQueue {
    unsigned long long n_pending, main_base, n_main, remaining;
    unsigned long long steps, tries, field_evals, launches;
    unsigned int cur, pad;
    unsigned long long pad2;
};

struct DevCounters {
    unsigned long long steps;
    unsigned long long tries;
    unsigned long long field_evals;
    unsigned long long active_left;
    unsigned long long queue_head;   // persistent mode: next candidate to take
    unsigned long long pending_count;
    unsigned long long status;       // non-zero: a bounded wait ran out / bad state
    unsigned long long pad;
};

}  // namespace crp
