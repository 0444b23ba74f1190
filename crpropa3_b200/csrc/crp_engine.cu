// crp_engine.cu -- host side of the C-ABI in include/crp_gpu.h: plan
// validation and upload, the run loop over the stepping kernels, the
// host-array path, field evaluation.
//
// The run loop replaces ModuleList::run(candidate_vector)
// (src/ModuleList.cpp.in:97): instead of an OpenMP loop over heap
// candidates, the structure-of-arrays state stays resident on the device and
// the kernels advance every active candidate, one thread per candidate,
// until it is inactive.  Cancellation (the reference's SIGINT flag,
// ModuleList.cpp.in:110) is a host flag polled between launches.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "crp_gpu.h"
#include "engine_internal.h"

using namespace crp;

namespace {

thread_local std::string g_error;

crp_status fail(crp_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return st;
}

crp_status cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(CRP_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    return fail(CRP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CUDA_TRY(call)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }

}  // namespace

namespace crp {
void set_last_error(const char *msg) { g_error = msg; }

// Every array a device entry point reads or writes must be reachable from
// the device: device memory, managed memory, or host memory registered /
// allocated with CUDA (mapped).  Ordinary host memory would make the kernels
// fault.  A null pointer passes (optional arrays).
crp_status check_device_ptr(const void *ptr, const char *what) {
    if (!ptr) return CRP_OK;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(CRP_ERR_INVALID_ARGUMENT, "%s: not a CUDA-accessible pointer", what);
    }
    if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return CRP_OK;
    if (a.type == cudaMemoryTypeHost && a.devicePointer == ptr) return CRP_OK;
    return fail(CRP_ERR_INVALID_ARGUMENT,
                "%s is host memory the device cannot address: pass device arrays to crp_run_device "
                "(or host arrays to crp_run)", what);
}
}  // namespace crp

constexpr double kInv2Pi = 0.15915494309189533577;  // 1 / (2 pi)
constexpr double kTurnScale = 4294967296.0;          // 2^32: turns as 32-bit fixed point
// crp_run() on host arrays: input chunks overlapped with the first launch,
// for runs of at least kPipelineMinCandidates
constexpr int kInputChunks = 8;
constexpr uint64_t kPipelineMinCandidates = 1u << 18;

struct crp_plan {
    int device = 0;
    int precision = CRP_PRECISION_FP64;
    int fs = FS_GENERIC;
    DevPlan dev{};
    std::vector<void *> owned;  // device allocations of grids and tables
    DevCounters *d_cnt = nullptr;
    DevCounters *h_cnt = nullptr;  // pinned
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // persistent mode: device work queue, its pinned host mirror, and the
    // stream the launch graphs are captured on and run in
    DevQueue *d_queue = nullptr;
    DevQueue *h_queue = nullptr;
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // device copies for crp_run() on host arrays
    uint64_t scratch_n = 0;
    void *scratch = nullptr;
    // crp_run() on host arrays, chunked mode: the inputs are copied in
    // kInputChunks chunks on copy_stream, and the first launch starts on each
    // chunk (on its own stream, so that the chunks run side by side) as soon
    // as the chunk has arrived; ident is the identity index list those
    // first-launch parts read their candidates through
    cudaStream_t copy_stream = nullptr;
    cudaStream_t part_stream[kInputChunks] = {};
    cudaEvent_t ev_chunk[kInputChunks] = {}, ev_part[kInputChunks] = {};
    cudaEvent_t ev_ready = nullptr;
    uint64_t ident_cap = 0;
    uint32_t *ident = nullptr;
    uint64_t rec_cap = 0;
    void *rec_scratch = nullptr;
    // compaction lists of still-active candidate indices (ping-pong)
    uint64_t list_cap = 0;
    uint32_t *lists = nullptr;
    // cell ordering of grid runs: keys in / out, the ordered index list and
    // the radix sort's temporary storage
    uint64_t sort_cap = 0;
    uint32_t *sort_buf = nullptr;
    size_t sort_tmp_bytes = 0;
    void *sort_tmp = nullptr;
    int tuned_block = 0;
    // autotuned launch configuration (crp_autotune); mode 0: not tuned
    int tuned_mode = 0;
    int tuned_ctas = 0, tuned_refill = 0, tuned_burst = 0;
    int num_sms = 0;
    // device copy of a sample for the autotuner's trials
    uint64_t trial_n = 0;
    void *trial = nullptr;

    ~crp_plan() {
        for (void *p : owned) cudaFree(p);
        if (d_cnt) cudaFree(d_cnt);
        if (h_cnt) cudaFreeHost(h_cnt);
        if (scratch) cudaFree(scratch);
        if (rec_scratch) cudaFree(rec_scratch);
        if (lists) cudaFree(lists);
        if (sort_buf) cudaFree(sort_buf);
        if (sort_tmp) cudaFree(sort_tmp);
        if (trial) cudaFree(trial);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (d_queue) cudaFree(d_queue);
        if (h_queue) cudaFreeHost(h_queue);
        if (gstream) cudaStreamDestroy(gstream);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        if (ident) cudaFree(ident);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (ev_ready) cudaEventDestroy(ev_ready);
        for (int k = 0; k < kInputChunks; k++) {
            if (part_stream[k]) cudaStreamDestroy(part_stream[k]);
            if (ev_chunk[k]) cudaEventDestroy(ev_chunk[k]);
            if (ev_part[k]) cudaEventDestroy(ev_part[k]);
        }
    }
};

namespace {

template <class T>
crp_status upload(crp_plan *p, const T *host, size_t count, const T **out) {
    void *d = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(T) * count));
    p->owned.push_back(d);
    CUDA_TRY(cudaMemcpy(d, host, sizeof(T) * count, cudaMemcpyHostToDevice));
    *out = static_cast<const T *>(d);
    return CRP_OK;
}

crp_status validate_module(const crp_module_desc &m) {
    if (m.kind == CRP_MODULE_PROPAGATION) {
        const char *name = m.propagator == CRP_PROP_CK ? "PropagationCK"
                         : m.propagator == CRP_PROP_BP ? "PropagationBP"
                         : m.propagator == CRP_PROP_SDE ? "DiffusionSDE" : nullptr;
        if (!name) return fail(CRP_ERR_UNSUPPORTED, "unknown propagator %d", m.propagator);
        // setTolerance / setMinimumStep / setMaximumStep
        // (PropagationCK.cpp:160-179, PropagationBP.cpp, DiffusionSDE.cpp)
        if (m.tolerance > 1 || m.tolerance < 0)
            return fail(CRP_ERR_INVALID_ARGUMENT, m.propagator == CRP_PROP_SDE
                        ? "%s: tolerance error not in range 0-1" : "%s: target error not in range 0-1", name);
        if (m.min_step < 0) return fail(CRP_ERR_INVALID_ARGUMENT, "%s: minStep < 0 ", name);
        if (m.min_step > m.max_step) return fail(CRP_ERR_INVALID_ARGUMENT, "%s: minStep > maxStep", name);
        if (!(m.max_step > 0)) return fail(CRP_ERR_INVALID_ARGUMENT, "%s: maxStep must be > 0", name);
        if (m.propagator == CRP_PROP_SDE) {
            if (m.sde_epsilon > 1 || m.sde_epsilon < 0)
                return fail(CRP_ERR_INVALID_ARGUMENT, "DiffusionSDE: epsilon not in range 0-1");
            if (m.sde_alpha > 2. || m.sde_alpha < 0)
                return fail(CRP_ERR_INVALID_ARGUMENT, "DiffusionSDE: alpha not in range 0-2");
            if (m.sde_scale < 0)
                return fail(CRP_ERR_INVALID_ARGUMENT, "DiffusionSDE: Scale error: Scale < 0");
            if (m.n_advection < 0 || m.n_advection > CRP_MAX_ADVECTION)
                return fail(CRP_ERR_UNSUPPORTED, "DiffusionSDE: at most %d advection fields", CRP_MAX_ADVECTION);
            for (int a = 0; a < m.n_advection; a++)
                if (m.advection[a].kind < CRP_ADVECTION_UNIFORM || m.advection[a].kind > CRP_ADVECTION_SEDOV_TAYLOR)
                    return fail(CRP_ERR_INVALID_ARGUMENT, "DiffusionSDE: unknown advection field kind %d",
                                m.advection[a].kind);
        } else if (m.n_advection != 0) {
            return fail(CRP_ERR_INVALID_ARGUMENT, "%s: advection fields belong to DiffusionSDE", name);
        }
    } else if (m.kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH) {
    } else if (m.kind == CRP_MODULE_OBSERVER) {
        if (m.n_features < 0 || m.n_features > CRP_MAX_OBSERVER_FEATURES)
            return fail(CRP_ERR_UNSUPPORTED, "at most %d observer features (got %d)", CRP_MAX_OBSERVER_FEATURES,
                        m.n_features);
        if (m.n_features == 0) {
            if (m.observer_feature != CRP_OBSERVER_SURFACE_SPHERE && m.observer_feature != CRP_OBSERVER_DETECT_ALL)
                return fail(CRP_ERR_UNSUPPORTED, "unsupported observer feature %d", m.observer_feature);
        }
        for (int f = 0; f < m.n_features; f++)
            if (m.features[f].kind < CRP_OBSERVER_SURFACE_SPHERE || m.features[f].kind > CRP_OBSERVER_PARTICLE_ID_VETO)
                return fail(CRP_ERR_UNSUPPORTED, "unsupported observer feature %d", m.features[f].kind);
    } else if (m.kind == CRP_MODULE_BOUNDARY) {
        if (m.boundary < CRP_BOUNDARY_SPHERICAL || m.boundary > CRP_BOUNDARY_CYLINDRICAL)
            return fail(CRP_ERR_UNSUPPORTED, "unsupported boundary %d", m.boundary);
    } else {
        return fail(CRP_ERR_UNSUPPORTED, "unsupported module kind %d", m.kind);
    }
    return CRP_OK;
}

// A Grid3f (comps 3) or Grid1f (comps 1) on the device: the cell values, the
// padded copy of a Grid3f for the mixed form, and GridProperties (Grid.h:75).
crp_status build_grid(crp_plan *p, const crp_grid3f_desc &g, int comps, DevGrid &dg) {
    const char *name = comps == 3 ? "Grid3f" : "Grid1f";
    if (!g.values || g.nx == 0 || g.ny == 0 || g.nz == 0)
        return fail(CRP_ERR_INVALID_ARGUMENT, "%s: empty grid", name);
    if (g.nx > (1u << 20) || g.ny > (1u << 20) || g.nz > (1u << 20))
        return fail(CRP_ERR_CAPACITY, "%s: a dimension beyond 2^20 cells", name);
    if (g.interpolation < CRP_INTERPOLATION_TRILINEAR || g.interpolation > CRP_INTERPOLATION_NEAREST_NEIGHBOUR)
        return fail(CRP_ERR_INVALID_ARGUMENT, "%s: interpolation type not understood", name);
    size_t cells = (size_t)g.nx * g.ny * g.nz;
    crp_status st = upload(p, g.values, cells * comps, &dg.values);
    if (st) return st;
    dg.values4 = nullptr;
    if (comps == 3 && p->precision == CRP_PRECISION_MIXED) {
        // 16-byte cells: one aligned 128-bit load per corner
        std::vector<float4> pad(cells);
        for (size_t i = 0; i < cells; i++)
            pad[i] = make_float4(g.values[3 * i], g.values[3 * i + 1], g.values[3 * i + 2], 0.f);
        st = upload(p, pad.data(), cells, &dg.values4);
        if (st) return st;
    }
    dg.nx = (int)g.nx; dg.ny = (int)g.ny; dg.nz = (int)g.nz;
    dg.reflective = g.reflective;
    dg.clip_volume = g.clip_volume;
    dg.interp = g.interpolation;
    dg.pow2 = is_pow2(g.nx) && is_pow2(g.ny) && is_pow2(g.nz);
    // Grid::setOrigin (Grid.h:225): gridOrigin = origin + spacing/2
    dg.gox = g.origin[0] + g.spacing[0] / 2;
    dg.goy = g.origin[1] + g.spacing[1] / 2;
    dg.goz = g.origin[2] + g.spacing[2] / 2;
    dg.sx = g.spacing[0]; dg.sy = g.spacing[1]; dg.sz = g.spacing[2];
    dg.inv_sx = 1.0 / g.spacing[0]; dg.inv_sy = 1.0 / g.spacing[1]; dg.inv_sz = 1.0 / g.spacing[2];
    dg.ox = g.origin[0]; dg.oy = g.origin[1]; dg.oz = g.origin[2];
    // edge = origin + Vector3d(Nx, Ny, Nz) * spacing (Grid.h:322)
    dg.ex = g.origin[0] + (double)g.nx * g.spacing[0];
    dg.ey = g.origin[1] + (double)g.ny * g.spacing[1];
    dg.ez = g.origin[2] + (double)g.nz * g.spacing[2];
    return CRP_OK;
}

crp_status build_component(crp_plan *p, const crp_field_component &f, DevComponent &d) {
    d.kind = f.kind;
    d.periodic = f.periodic;
    d.periodic_reflective = f.periodic_reflective;
    for (int a = 0; a < 3; a++) {
        d.po[a] = f.periodic_origin[a];
        d.pe[a] = f.periodic_extends[a];
        d.uniform[a] = f.uniform[a];
    }
    d.b0 = f.toroidal_b0;
    if (f.periodic && !(f.periodic_extends[0] > 0 && f.periodic_extends[1] > 0 && f.periodic_extends[2] > 0))
        return fail(CRP_ERR_INVALID_ARGUMENT, "PeriodicMagneticField: extends must be > 0");
    if (f.kind == CRP_FIELD_GRID || f.kind == CRP_FIELD_MODULATED_GRID) {
        crp_status st = build_grid(p, f.grid, 3, d.grid);
        if (st) return st;
        if (f.kind == CRP_FIELD_MODULATED_GRID) {
            st = build_grid(p, f.modulation, 1, d.mod);
            if (st) return st;
        }
    } else if (f.kind == CRP_FIELD_PLANE_WAVE) {
        const crp_plane_wave_desc &w = f.plane_wave;
        if (w.n_modes <= 1)
            return fail(CRP_ERR_INVALID_ARGUMENT,
                        "PlaneWaveTurbulence: Nm <= 1. Specify at least two wavemodes in order to generate the k distribution properly.");
        if (!w.xi || !w.kappa || !w.k || !w.beta || !w.ak)
            return fail(CRP_ERR_INVALID_ARGUMENT, "PlaneWaveTurbulence: mode arrays missing");
        int n = w.n_modes;
        std::vector<double> m9((size_t)n * 9);
        // mixed form, per pair of modes (a, b): {kx_a, ky_a, kz_a, kx_b, ky_b, kz_b} as doubles
        // (k kappa / 2 pi times 2^32: the phase in turns as 32-bit fixed point, exact scaling),
        // then {beta_a, beta_b} as unsigned 32-bit fixed-point turns and {A xi_a, A xi_b} as
        // floats: 48 + 8 + 24 = 80 bytes, five 16-byte loads
        const int npairs = (n + 1) / 2;
        std::vector<float4> pairs((size_t)npairs * 5);
        std::memset(pairs.data(), 0, pairs.size() * sizeof(float4));
        double ksum = 0;
        for (int i = 0; i < n; i++) {
            for (int a = 0; a < 3; a++) {
                m9[9 * i + a] = w.xi[3 * i + a];
                m9[9 * i + 3 + a] = w.kappa[3 * i + a];
            }
            m9[9 * i + 6] = w.k[i];
            m9[9 * i + 7] = w.beta[i];
            m9[9 * i + 8] = w.ak[i];
            const int q = i / 2, h = i % 2;
            double *kd = reinterpret_cast<double *>(&pairs[(size_t)q * 5]);
            uint32_t *bu = reinterpret_cast<uint32_t *>(&pairs[(size_t)q * 5 + 3]);
            float *af = reinterpret_cast<float *>(&pairs[(size_t)q * 5 + 3]) + 2;
            double s = 0;
            for (int a = 0; a < 3; a++) {
                kd[3 * h + a] = w.k[i] * w.kappa[3 * i + a] * kInv2Pi * kTurnScale;
                s += std::fabs(kd[3 * h + a]);
                af[3 * h + a] = (float)(w.ak[i] * w.xi[3 * i + a]);
            }
            ksum = std::max(ksum, s);
            // beta / 2 pi in [0, 1) turns, as 32-bit fixed point
            double bt = w.beta[i] * kInv2Pi;
            bt -= std::floor(bt);
            bu[h] = (uint32_t)(int64_t)std::llround(bt * kTurnScale);
        }
        crp_status st = upload(p, m9.data(), m9.size(), &d.pw.modes);
        if (st) return st;
        st = upload(p, pairs.data(), pairs.size(), &d.pw.pairs);
        if (st) return st;
        d.pw.n = n;
        d.pw.npairs = npairs;
        // the fixed-point phase needs |k kappa . x * 2^32 / 2 pi| < 2^50 for every mode:
        // max_i (|kx| + |ky| + |kz|) max(|x|, |y|, |z|) < 2^50
        d.pw.fast_limit = ksum > 0 ? 1125899906842624.0 / ksum : INFINITY;
    } else if (f.kind == CRP_FIELD_JF12) {
        const crp_jf12_desc &J = f.jf12;
        if (!(J.kpc > 0)) return fail(CRP_ERR_INVALID_ARGUMENT, "JF12Field: parameters not set (crp_jf12_defaults)");
        if (J.variant < CRP_JF12_JF12 || J.variant > CRP_JF12_SOLENOIDAL)
            return fail(CRP_ERR_INVALID_ARGUMENT, "JF12Field: unknown variant");
        if (J.variant == CRP_JF12_SOLENOIDAL && !(J.r1 > 0 && J.r2 > J.r1))
            return fail(CRP_ERR_INVALID_ARGUMENT, "JF12FieldSolenoidal: parameters not set (crp_jf12_solenoidal)");
        DevJF12 h;
        std::memset(&h, 0, sizeof(h));
        h.d = J;
        h.inv_kpc = 1.0 / J.kpc;
        // Units.h: muG = 1e-6 gauss, gauss = 1e-4 tesla
        h.muG = 1e-6 * 1e-4;
        const double L = 1.0 / J.kpc, B = 1.0 / h.muG;
        for (int i = 0; i < 8; i++) {
            h.rarms[i] = (float)(J.r_arms[i] * L);
            h.bdisk[i] = (float)(J.b_disk[i] * B);
            h.bdturb[i] = (float)(J.b_disk_turb[i] * B);
        }
        h.bring = (float)(J.b_ring * B); h.hdisk = (float)(J.h_disk * L); h.wdisk = (float)(J.w_disk * L);
        h.bnorth = (float)(J.b_north * B); h.bsouth = (float)(J.b_south * B);
        h.rnorth = (float)(J.r_north * L); h.rsouth = (float)(J.r_south * L);
        h.whalo = (float)(J.w_halo * L); h.z0 = (float)(J.z0 * L);
        h.bx = (float)(J.b_x * B); h.sinthx0 = (float)J.sin_theta_x0; h.costhx0 = (float)J.cos_theta_x0;
        h.tanthx0 = (float)J.tan_theta_x0; h.rxc = (float)(J.r_xc * L); h.rx = (float)(J.r_x * L);
        h.sinp = (float)J.sin_pitch; h.cosp = (float)J.cos_pitch; h.tan90mp = (float)J.tan90_minus_pitch;
        h.sqrtbeta = (float)J.sqrt_beta;
        h.bdturb5 = (float)(J.b_disk_turb5 * B); h.zdturb = (float)(J.z_disk_turb * L);
        h.bhturb = (float)(J.b_halo_turb * B); h.rhturb = (float)(J.r_halo_turb * L);
        h.zhturb = (float)(J.z_halo_turb * L);
        h.s_cotp = (float)J.cot_pitch; h.s_cotx = (float)J.cot_theta_x0; h.s_zs = (float)(J.z_s * L);
        h.s_r1 = (float)(J.r1 * L); h.s_r2 = (float)(J.r2 * L); h.s_r1s = (float)(J.r1s * L);
        h.s_r2s = (float)(J.r2s * L);
        for (int i = 0; i < 11; i++) { h.s_phi0[i] = (float)J.phi0_arms[i]; h.s_b[i] = (float)(J.b_arms[i] * B); }
        for (int i = 0; i < 10; i++) h.s_coeff[i] = (float)(J.phi_coeff[i] * B);
        if (J.use_turbulent) {  // JF12Field::setTurbulentGrid (JF12Field.cpp:118)
            if (!f.grid.values)
                return fail(CRP_ERR_INVALID_ARGUMENT, "JF12Field: No turbulent field set (use_turbulent without a grid)");
            crp_status st = build_grid(p, f.grid, 3, d.grid);
            if (st) return st;
        }
        if (J.use_striated) {  // JF12Field::setStriatedGrid (JF12Field.cpp:113)
            if (!f.modulation.values)
                return fail(CRP_ERR_INVALID_ARGUMENT, "JF12Field: No striated field set (use_striated without a grid)");
            crp_status st = build_grid(p, f.modulation, 1, d.mod);
            if (st) return st;
        }
        crp_status st = upload(p, &h, 1, &d.jf);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_UF23) {
        const crp_uf23_desc &U = f.uf23;
        if (U.model < CRP_UF23_BASE || U.model > CRP_UF23_NEBCOR)
            return fail(CRP_ERR_INVALID_ARGUMENT, "UF23Field: unknown field model");
        if (!(U.kpc > 0) || !(U.microgauss > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "UF23Field: parameters not set (crp_uf23_defaults)");
        DevUF23 h;
        h.d = U;
        h.c_pol = std::pow(U.poloidal_a / U.poloidal_z, U.poloidal_p);  // UF23Field.cpp:392-393
        h.a0p = std::pow(U.poloidal_a, U.poloidal_p);
        h.b1 = (float)U.disk_b1; h.b2 = (float)U.disk_b2; h.b3 = (float)U.disk_b3;
        h.disk_h = (float)U.disk_h; h.disk_w = (float)U.disk_w;
        h.ph1 = (float)U.disk_phase1; h.ph2 = (float)U.disk_phase2; h.ph3 = (float)U.disk_phase3;
        h.sinp = (float)U.sin_pitch; h.cosp = (float)U.cos_pitch;
        h.inv_tanp = (float)(1.0 / U.tan_pitch); h.tanp = (float)U.tan_pitch;
        h.spur_center = (float)U.spur_center; h.spur_length = (float)U.spur_length;
        h.spur_inv_width = U.spur_width != 0 ? (float)(1.0 / U.spur_width) : 0.f;
        h.tbn = (float)U.toroidal_bn; h.tbs = (float)U.toroidal_bs; h.tr = (float)U.toroidal_r;
        h.tw = (float)U.toroidal_w; h.tz = (float)U.toroidal_z;
        h.pb = (float)U.poloidal_b; h.pp = (float)U.poloidal_p; h.pr = (float)U.poloidal_r;
        h.pw = (float)U.poloidal_w; h.pa = (float)U.poloidal_a; h.pzz = (float)U.poloidal_z;
        h.inv_pp = (float)(1.0 / U.poloidal_p);
        h.twist = (float)U.twisting_time; h.r2max = (float)U.max_radius_squared;
        h.muG = (float)U.microgauss;
        h.inv_kpc = 1.0 / U.kpc;
        crp_status st = upload(p, &h, 1, &d.uf);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_PT11) {
        const crp_pt11_desc &T = f.pt11;
        if (T.use_ass && T.use_bss)
            return fail(CRP_ERR_INVALID_ARGUMENT, "PT11Field: ASS and BSS disk both on (crp_pt11_use)");
        if ((T.use_ass || T.use_bss) && !(T.r_sun > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "PT11Field: parameters not set (crp_pt11_defaults)");
        if (T.use_halo && !(T.r0_h > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "PT11Field: parameters not set (crp_pt11_defaults)");
        crp_status st = upload(p, &T, 1, &d.pt);
        if (st) return st;
        // Units.h: kpc = 1e3 parsec, parsec = 648000 / pi au; muG = 1e-6 gauss, gauss = 1e-4 tesla
        const double kpc = 1e3 * (648000 / M_PI * 149597870700.0), muG = 1e-6 * 1e-4;
        const double L = 1.0 / kpc, B = 1.0 / muG;
        DevPT11 f32;
        std::memset(&f32, 0, sizeof(f32));
        f32.use_ass = T.use_ass; f32.use_bss = T.use_bss; f32.use_halo = T.use_halo;
        f32.r_sun = (float)(T.r_sun * L); f32.r_c = (float)(T.r_c * L); f32.z0_d = (float)(T.z0_d * L);
        f32.b0_d = (float)(T.b0_d * B);
        f32.z0_h = (float)(T.z0_h * L); f32.r0_h = (float)(T.r0_h * L); f32.b0_hn = (float)(T.b0_hn * B);
        f32.b0_hs = (float)(T.b0_hs * B); f32.z11_h = (float)(T.z11_h * L); f32.z12_h = (float)(T.z12_h * L);
        f32.sinp = (float)T.sin_pitch; f32.cosp = (float)T.cos_pitch;
        f32.cotp = T.sin_pitch != 0 ? (float)(T.cos_pitch / T.sin_pitch) : 0.f;
        f32.phi = (float)T.phi; f32.cos_phi = (float)T.cos_phi;
        f32.inv_kpc = L;
        f32.muG = (float)muG;
        st = upload(p, &f32, 1, &d.pt32);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_TF17) {
        const crp_tf17_desc &T = f.tf17;
        if (T.disk_model < CRP_TF17_AD1 || T.disk_model > CRP_TF17_DD1 || T.halo_model < CRP_TF17_C0 ||
            T.halo_model > CRP_TF17_C1)
            return fail(CRP_ERR_INVALID_ARGUMENT, "TF17Field: unknown disk or halo model");
        if (!(T.h_p > 0) || !(T.l_p > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "TF17Field: parameters not set (crp_tf17_defaults)");
        crp_status st = upload(p, &T, 1, &d.tf);
        if (st) return st;
        // Units.h: kpc = 1e3 parsec, parsec = 648000 / pi au; muG = 1e-6 gauss, gauss = 1e-4 tesla
        const double kpc = 1e3 * (648000 / M_PI * 149597870700.0), muG = 1e-6 * 1e-4;
        DevTF17 f32;
        std::memset(&f32, 0, sizeof(f32));
        f32.disk_model = T.disk_model; f32.halo_model = T.halo_model;
        f32.use_disk = T.use_disk; f32.use_halo = T.use_halo;
        const double L = 1.0 / kpc, B = 1.0 / muG;
        f32.a_disk = (float)(T.a_disk * kpc * kpc); f32.z1_disk = (float)(T.z1_disk * L);
        f32.r1_disk = (float)(T.r1_disk * L); f32.b1_disk = (float)(T.b1_disk * B);
        f32.l_disk = (float)(T.l_disk * L); f32.phi_star_disk = (float)T.phi_star_disk;
        f32.h_disk = (float)(T.h_disk * L);
        f32.a_halo = (float)(T.a_halo * kpc * kpc); f32.z1_halo = (float)(T.z1_halo * L);
        f32.b1_halo = (float)(T.b1_halo * B); f32.l_halo = (float)(T.l_halo * L);
        f32.phi_star_halo = (float)T.phi_star_halo;
        f32.cot_p0 = (float)T.cot_p0; f32.h_p = (float)(T.h_p * L); f32.l_p = (float)(T.l_p * L);
        f32.eps = (float)T.epsilon;
        f32.inv_kpc = L;
        f32.muG = (float)muG;
        st = upload(p, &f32, 1, &d.tf32);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_SINGLE_MODE) {
        d.mode = f.single_mode;
    } else if (f.kind == CRP_FIELD_KST24) {
        if (!(f.kst24.kpc > 0) || !(f.kst24.gauss > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "KST24Field: parameters not set (crp_kst24_defaults)");
        crp_status st = upload(p, &f.kst24, 1, &d.kst);
        if (st) return st;
        const crp_kst24_desc &K = f.kst24;
        DevKST24 k32;
        std::memset(&k32, 0, sizeof(k32));
        k32.north_b = (float)K.north_b; k32.north_zmin = (float)K.north_zmin; k32.north_zmax = (float)K.north_zmax;
        k32.north_rmin = (float)K.north_rmin; k32.north_rmax = (float)K.north_rmax;
        k32.south_b = (float)K.south_b; k32.south_zmin = (float)K.south_zmin; k32.south_zmax = (float)K.south_zmax;
        k32.south_rmin = (float)K.south_rmin; k32.south_rmax = (float)K.south_rmax;
        k32.x_b = (float)K.x_b; k32.x_rmin = (float)K.x_rmin; k32.x_rmax = (float)K.x_rmax;
        k32.tan_x = (float)std::tan(K.x_theta_rad); k32.sin_x = (float)std::sin(K.x_theta_rad);
        k32.cos_x = (float)std::cos(K.x_theta_rad);
        k32.lb_b = (float)K.lb_b; k32.lb_rmin = (float)K.lb_rmin; k32.lb_dr = (float)K.lb_dr;
        k32.lb_x0 = (float)K.lb_x0; k32.lb_y0 = (float)K.lb_y0; k32.lb_z0 = (float)K.lb_z0;
        for (int a = 0; a < 3; a++) k32.lb_dir[a] = (float)K.lb_dir[a];
        k32.lb_ampl = (float)(1 + (K.lb_rmin * K.lb_rmin) / (2 * K.lb_rmin * K.lb_dr + K.lb_dr * K.lb_dr));
        for (int a = 0; a < 5; a++) {
            const crp_kst24_arm &A = K.arms[a];
            DevKST24Arm &B = k32.arms[a];
            const double pr = A.pitch_deg * M_PI / 180.;
            B.b = (float)A.b; B.k = (float)std::tan(pr); B.cos_pitch = (float)std::cos(pr);
            B.sin_pitch = (float)std::sin(pr); B.phi0 = (float)(A.phi0_deg * M_PI / 180.);
            B.arc_div = (float)(A.arc_div_deg * M_PI / 180.);
            B.x_shift = (float)A.x_shift; B.y_shift = (float)A.y_shift;
            B.arc_radius1 = (float)A.arc_radius1; B.arc_radius2 = (float)A.arc_radius2; B.arc_eps = (float)A.arc_eps;
            B.rmin = (float)A.rmin; B.rmax = (float)A.rmax; B.zmin = (float)A.zmin; B.zmax = (float)A.zmax;
        }
        k32.inv_kpc = 1.0 / K.kpc;
        k32.gauss = (float)K.gauss;
        st = upload(p, &k32, 1, &d.kst32);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_CMZ) {
        if (!(f.cmz.gauss > 0))
            return fail(CRP_ERR_INVALID_ARGUMENT, "CMZField: parameters not set (crp_cmz_defaults)");
        crp_status st = upload(p, &f.cmz, 1, &d.cmz);
        if (st) return st;
    } else if (f.kind == CRP_FIELD_ARCHIMEDEAN_SPIRAL) {
        d.arch = f.archimedean;
    } else if (f.kind == CRP_FIELD_UNIFORM || f.kind == CRP_FIELD_TOROIDAL) {
    } else {
        return fail(CRP_ERR_UNSUPPORTED, "unsupported field kind %d", f.kind);
    }
    return CRP_OK;
}

crp_status ensure_counters(crp_plan *p) {
    if (!p->d_cnt) CUDA_TRY(cudaMalloc(&p->d_cnt, sizeof(DevCounters)));
    if (!p->h_cnt) CUDA_TRY(cudaMallocHost(&p->h_cnt, sizeof(DevCounters)));
    if (!p->ev0) CUDA_TRY(cudaEventCreate(&p->ev0));
    if (!p->ev1) CUDA_TRY(cudaEventCreate(&p->ev1));
    return CRP_OK;
}

DevState to_dev_state(const crp_candidates &c) {
    DevState s;
    s.id = c.id; s.charge = c.charge; s.energy = c.energy;
    s.x = c.x; s.y = c.y; s.z = c.z;
    s.dx = c.dx; s.dy = c.dy; s.dz = c.dz;
    s.px = c.px; s.py = c.py; s.pz = c.pz;
    s.len = c.trajectory_length; s.time = c.time; s.cur = c.current_step; s.next = c.next_step;
    s.active = c.active; s.flags = c.flags; s.max_length = c.max_length; s.steps = c.step_count;
    return s;
}

DevRecords to_dev_records(const crp_records *r) {
    DevRecords d{};
    if (!r) return d;
    d.capacity = r->capacity;
    d.count = reinterpret_cast<unsigned long long *>(r->count);
    d.index = r->index; d.module = r->module;
    d.len = r->trajectory_length; d.time = r->time;
    d.x = r->x; d.y = r->y; d.z = r->z;
    d.dx = r->dx; d.dy = r->dy; d.dz = r->dz;
    d.energy = r->energy; d.id = r->id;
    return d;
}

bool needs_per_candidate(const crp_plan *p) {
    for (int i = 0; i < p->dev.n_modules; i++)
        if (p->dev.modules[i].kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH && p->dev.modules[i].per_candidate)
            return true;
    return false;
}

bool needs_step_count(const crp_plan *p) {
    return p->dev.modules[p->dev.prop_index].propagator == CRP_PROP_SDE;
}

}  // namespace

extern "C" {

uint32_t crp_abi_version(void) { return CRP_ABI_VERSION; }

crp_status crp_last_error(char *buffer, size_t size) {
    if (!buffer || size == 0) return CRP_ERR_INVALID_ARGUMENT;
    snprintf(buffer, size, "%s", g_error.c_str());
    return CRP_OK;
}

crp_status crp_device_count(int32_t *count) {
    if (!count) return fail(CRP_ERR_INVALID_ARGUMENT, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(CRP_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *count = n;
    return CRP_OK;
}

crp_status crp_plan_create(const crp_plan_desc *desc, crp_plan **out) {
    if (!desc || !out) return fail(CRP_ERR_INVALID_ARGUMENT, "desc or plan pointer is NULL");
    *out = nullptr;
    if (desc->abi_version != CRP_ABI_VERSION)
        return fail(CRP_ERR_INVALID_ARGUMENT, "ABI version %u, library has %u", desc->abi_version, CRP_ABI_VERSION);
    if (desc->precision != CRP_PRECISION_FP64 && desc->precision != CRP_PRECISION_MIXED)
        return fail(CRP_ERR_INVALID_ARGUMENT, "unknown precision %d", desc->precision);
    if (desc->n_fields < 0 || desc->n_fields > kMaxFields)
        return fail(CRP_ERR_UNSUPPORTED, "at most %d field components (got %d)", kMaxFields, desc->n_fields);
    if (desc->n_modules < 1 || desc->n_modules > kMaxModules)
        return fail(CRP_ERR_UNSUPPORTED, "1 to %d modules (got %d)", kMaxModules, desc->n_modules);
    int nprop = 0, prop_index = -1;
    for (int i = 0; i < desc->n_modules; i++) {
        crp_status st = validate_module(desc->modules[i]);
        if (st) return st;
        if (desc->modules[i].kind == CRP_MODULE_PROPAGATION) { nprop++; prop_index = i; }
    }
    if (nprop != 1) return fail(CRP_ERR_UNSUPPORTED, "the device path needs exactly one propagation module (got %d)", nprop);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(CRP_ERR_NO_DEVICE, "no CUDA device visible");

    crp_plan *p = new crp_plan();
    cudaGetDevice(&p->device);
    p->precision = desc->precision;
    DevPlan &d = p->dev;
    d.n_fields = desc->n_fields;
    d.n_modules = desc->n_modules;
    d.prop_index = prop_index;
    d.seed = desc->seed;
    // module sequences with compiled kernels (chain.cuh ChainShape)
    const auto kind = [&](int i) { return desc->modules[i].kind; };
    d.shape = CS_GENERIC;
    if (desc->n_modules == 2 && kind(0) == CRP_MODULE_PROPAGATION && kind(1) == CRP_MODULE_MAX_TRAJECTORY_LENGTH)
        d.shape = CS_PM;
    else if (desc->n_modules == 3 && kind(0) == CRP_MODULE_PROPAGATION &&
             kind(1) == CRP_MODULE_MAX_TRAJECTORY_LENGTH && kind(2) == CRP_MODULE_OBSERVER)
        d.shape = CS_PMO;
    for (int i = 0; i < desc->n_fields; i++) {
        crp_status st = build_component(p, desc->fields[i], d.fields[i]);
        if (st) { delete p; return st; }
    }
    int nfeat_total = 0;
    for (int i = 0; i < desc->n_modules; i++) {
        const crp_module_desc &m = desc->modules[i];
        DevModule &dm = d.modules[i];
        dm.kind = m.kind; dm.propagator = m.propagator;
        dm.tolerance = m.tolerance; dm.min_step = m.min_step; dm.max_step = m.max_step;
        dm.eps = m.sde_epsilon; dm.alpha = m.sde_alpha; dm.scale = m.sde_scale;
        dm.n_adv = 0;
        dm.adv = nullptr;
        if (m.kind == CRP_MODULE_PROPAGATION && m.propagator == CRP_PROP_SDE && m.n_advection > 0) {
            crp_status st = upload(p, m.advection, (size_t)m.n_advection, &dm.adv);
            if (st) { delete p; return st; }
            dm.n_adv = m.n_advection;
        }
        dm.max_length = m.max_length; dm.per_candidate = m.per_candidate_length;
        dm.observer = m.observer_feature;
        dm.cx = m.sphere_center[0]; dm.cy = m.sphere_center[1]; dm.cz = m.sphere_center[2];
        dm.radius = m.sphere_radius;
        dm.deactivate = m.deactivate_on_detection; dm.record = m.record;
        if (m.kind == CRP_MODULE_OBSERVER) {
            // the single legacy feature becomes a one-entry feature list
            crp_observer_feature_desc legacy{};
            legacy.kind = m.observer_feature;
            for (int a = 0; a < 3; a++) legacy.a[a] = m.sphere_center[a];
            legacy.r = m.sphere_radius;
            const crp_observer_feature_desc *fs = m.n_features > 0 ? m.features : &legacy;
            const int nf = m.n_features > 0 ? m.n_features : 1;
            if (nfeat_total + nf > kMaxFeatures) {
                delete p;
                return fail(CRP_ERR_UNSUPPORTED, "at most %d observer features per chain", kMaxFeatures);
            }
            dm.feat0 = nfeat_total;
            dm.nfeat = nf;
            for (int f = 0; f < nf; f++) {
                DevFeature &df = d.feat[nfeat_total++];
                df.kind = fs[f].kind;
                df.pid = fs[f].particle_id;
                df.ax = fs[f].a[0]; df.ay = fs[f].a[1]; df.az = fs[f].a[2];
                df.bx = fs[f].b[0]; df.by = fs[f].b[1]; df.bz = fs[f].b[2];
                df.r = fs[f].r; df.step = fs[f].step;
            }
        }
        if (m.kind == CRP_MODULE_BOUNDARY) {
            dm.boundary = m.boundary;
            dm.limit_step = m.boundary_limit_step;
            dm.cx = m.boundary_a[0]; dm.cy = m.boundary_a[1]; dm.cz = m.boundary_a[2];
            dm.bx = m.boundary_b[0]; dm.by = m.boundary_b[1]; dm.bz = m.boundary_b[2];
            dm.bsize = m.boundary_size; dm.bradius = m.boundary_radius; dm.margin = m.boundary_margin;
        }
    }
    if (d.n_fields == 1 && !desc->fields[0].periodic && desc->fields[0].kind == CRP_FIELD_GRID) {
        const DevGrid &g = d.fields[0].grid;
        const bool padded = p->precision != CRP_PRECISION_MIXED || g.values4 != nullptr;
        const bool small = (uint64_t)g.nx * g.ny * g.nz < (1ull << 31);  // 32-bit cell indices
        const bool trilinear = g.interp == CRP_INTERPOLATION_TRILINEAR;
        p->fs = (!g.reflective && !g.clip_volume && g.pow2 && padded && small && trilinear) ? FS_GRID_PERIODIC
                                                                                           : FS_GRID;
    }
    else if (d.n_fields == 1 && !desc->fields[0].periodic && desc->fields[0].kind == CRP_FIELD_PLANE_WAVE)
        p->fs = FS_PLANE_WAVE;
    else
        p->fs = FS_GENERIC;
    crp_status st = ensure_counters(p);
    if (st) { delete p; return st; }
    if (cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess)
        p->num_sms = 148;
    *out = p;
    return CRP_OK;
}

crp_status crp_plan_destroy(crp_plan *plan) {
    delete plan;
    return CRP_OK;
}

static crp_status check_device_arrays(const crp_candidates *c, const crp_records *r) {
    const void *const ptrs[] = {c->id, c->charge, c->energy, c->x, c->y, c->z, c->dx, c->dy, c->dz,
                                c->px, c->py, c->pz, c->trajectory_length, c->time,
                                c->current_step, c->next_step, c->active, c->flags,
                                c->max_length, c->step_count};
    for (const void *q : ptrs) {
        crp_status st = check_device_ptr(q, "a candidate array");
        if (st) return st;
    }
    if (r) {
        const void *const rp[] = {r->count, r->index, r->module, r->trajectory_length, r->time,
                                  r->x, r->y, r->z, r->dx, r->dy, r->dz, r->energy, r->id};
        for (const void *q : rp) {
            crp_status st = check_device_ptr(q, "a record array");
            if (st) return st;
        }
    }
    return CRP_OK;
}

static crp_status ensure_lists(crp_plan *p, uint64_t n) {
    if (p->list_cap < n) {
        if (p->lists) { cudaFree(p->lists); p->lists = nullptr; p->list_cap = 0; }
        CUDA_TRY(cudaMalloc(&p->lists, sizeof(uint32_t) * 2 * n));
        p->list_cap = n;
    }
    return CRP_OK;
}

// ---------------------------------------------------------------------------
// Cell ordering of grid runs.  Candidates that share grid cells share the
// corner loads of the interpolation (L1 and L2 hits) and change cells at
// similar steps (less divergence in the gather), so between launches the
// still-active candidates are ordered by the cell they are in (the Morton
// code of its indices, or blocks of 8^3 cells for grids above 1024 cells in
// a dimension; cell_key_kernel), sorted with a radix sort.  The order is a scheduling choice only: every
// candidate's trajectory is the same whatever order the threads take them in.
constexpr int kSortedStepsPerLaunch = 512;
constexpr uint64_t kSortMinCandidates = 1u << 16;

__device__ __forceinline__ int cell_of(double x, double go, double inv_s, int n) {
    const double c = floor((x - go) * inv_s);
    long long i = (long long)c % n;
    return (int)(i < 0 ? i + n : i);
}

// The sort key of a candidate's cell: with mb > 0 (every dimension at most
// 2^mb <= 1024 cells) the Morton code of (ix, iy, iz), 3 mb bits, so that
// cells close in all three directions get close keys; larger grids: blocks
// of 8^3 cells in x-major order, cells x-major inside a block.
__global__ void cell_key_kernel(DevGrid g, const double *x, const double *y, const double *z,
                                const uint32_t *list, uint32_t n, int nby, int nbz, int mb, uint32_t *keys,
                                uint32_t *vals) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t i = list ? list[t] : t;
    const int ix = cell_of(x[i], g.gox, g.inv_sx, g.nx);
    const int iy = cell_of(y[i], g.goy, g.inv_sy, g.ny);
    const int iz = cell_of(z[i], g.goz, g.inv_sz, g.nz);
    if (mb > 0) {
        uint32_t key = 0;
        for (int b = mb - 1; b >= 0; b--)
            key = (key << 3) | ((((uint32_t)ix >> b) & 1u) << 2) | ((((uint32_t)iy >> b) & 1u) << 1) |
                  (((uint32_t)iz >> b) & 1u);
        keys[t] = key;
    } else {
        const uint32_t block = ((uint32_t)(ix >> 3) * nby + (uint32_t)(iy >> 3)) * nbz + (uint32_t)(iz >> 3);
        keys[t] = block * 512u + (uint32_t)(((ix & 7) * 8 + (iy & 7)) * 8 + (iz & 7));
    }
    vals[t] = i;
}

// Bits per dimension of the Morton key (0: the grid is larger than 1024
// cells in some dimension).
static int cell_morton_bits(const DevGrid &g) {
    const int m = std::max(g.nx, std::max(g.ny, g.nz));
    if (m > 1024) return 0;
    int b = 1;
    while ((1 << b) < m) b++;
    return b;
}

// Bits of the largest key, or 0 when the grid is too large for 32-bit keys.
static int cell_key_bits(const DevGrid &g) {
    if (const int mb = cell_morton_bits(g)) return 3 * mb;
    const uint64_t nb = (uint64_t)((g.nx + 7) / 8) * ((g.ny + 7) / 8) * ((g.nz + 7) / 8) * 512;
    if (nb > (1ull << 32)) return 0;
    int bits = 1;
    while (bits < 32 && (1ull << bits) < nb) bits++;
    return bits;
}

static crp_status ensure_sort(crp_plan *p, uint64_t n) {
    if (p->sort_cap < n) {
        if (p->sort_buf) { cudaFree(p->sort_buf); p->sort_buf = nullptr; p->sort_cap = 0; }
        if (p->sort_tmp) { cudaFree(p->sort_tmp); p->sort_tmp = nullptr; p->sort_tmp_bytes = 0; }
        CUDA_TRY(cudaMalloc(&p->sort_buf, sizeof(uint32_t) * 4 * n));
        p->sort_cap = n;
        size_t bytes = 0;
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, p->sort_buf, p->sort_buf + n, p->sort_buf + 2 * n,
                                                 p->sort_buf + 3 * n, (int)n, 0, 32));
        CUDA_TRY(cudaMalloc(&p->sort_tmp, bytes));
        p->sort_tmp_bytes = bytes;
    }
    return CRP_OK;
}

// Orders the n indices of `list` (all candidates when null) by cell; returns
// the ordered list (inside p->sort_buf).
static crp_status order_by_cell(crp_plan *p, const DevState &s, const uint32_t *list, uint64_t n, int bits,
                                cudaStream_t st, const uint32_t **out) {
    const DevGrid &g = p->dev.fields[0].grid;
    uint32_t *keys_in = p->sort_buf, *keys_out = p->sort_buf + p->sort_cap;
    uint32_t *vals_in = p->sort_buf + 2 * p->sort_cap, *vals_out = p->sort_buf + 3 * p->sort_cap;
    cell_key_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, s.x, s.y, s.z, list, (uint32_t)n,
                                                                (g.ny + 7) / 8, (g.nz + 7) / 8, cell_morton_bits(g),
                                                                keys_in, vals_in);
    CUDA_TRY(cudaGetLastError());
    size_t bytes = p->sort_tmp_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(p->sort_tmp, bytes, keys_in, keys_out, vals_in, vals_out, (int)n, 0,
                                             bits, st));
    *out = vals_out;
    return CRP_OK;
}

// Persistent mode: bounded launches of SMs x ctas_per_sm CTAs that refill
// lanes from the device queue; what a launch leaves (lanes still busy at its
// time budget, queue items not yet taken) is the next launch's queue.
// Bookkeeping between two persistent launches, captured with them: pending
// items no lane took are appended behind the launch's new pending list
// (carry_kernel, all threads), then the queue advances and the launch's
// counters are added to the run totals and cleared (advance_kernel, one
// thread).
__global__ void carry_kernel(const DevQueue *q, const DevCounters *cnt, uint32_t *la, uint32_t *lb) {
    const unsigned long long total = q->n_pending + q->n_main;
    const unsigned long long consumed = cnt->queue_head < total ? cnt->queue_head : total;
    if (consumed >= q->n_pending) return;
    const unsigned long long rest = q->n_pending - consumed, base = cnt->pending_count;
    const uint32_t *pin = q->cur ? lb : la;
    uint32_t *pout = q->cur ? la : lb;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < rest; i += stride)
        pout[base + i] = pin[consumed + i];
}

__global__ void advance_kernel(DevQueue *q, DevCounters *cnt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const unsigned long long total = q->n_pending + q->n_main;
    const unsigned long long consumed = cnt->queue_head < total ? cnt->queue_head : total;
    unsigned long long next_pending = cnt->pending_count;
    if (consumed < q->n_pending) {
        next_pending += q->n_pending - consumed;
    } else {
        q->main_base += consumed - q->n_pending;
        q->n_main -= consumed - q->n_pending;
    }
    q->n_pending = next_pending;
    q->cur ^= 1u;
    q->remaining = q->n_pending + q->n_main;
    q->steps += cnt->steps;
    q->tries += cnt->tries;
    q->field_evals += cnt->field_evals;
    if (total > 0) q->launches++;
    cnt->steps = cnt->tries = cnt->field_evals = 0;
    cnt->queue_head = cnt->pending_count = cnt->active_left = 0;
}

static crp_status ensure_graph_resources(crp_plan *p) {
    if (!p->d_queue) CUDA_TRY(cudaMalloc(&p->d_queue, sizeof(DevQueue)));
    if (!p->h_queue) CUDA_TRY(cudaMallocHost(&p->h_queue, sizeof(DevQueue)));
    if (!p->gstream) CUDA_TRY(cudaStreamCreateWithFlags(&p->gstream, cudaStreamNonBlocking));
    if (!p->ev_in) CUDA_TRY(cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming));
    if (!p->ev_out) CUDA_TRY(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
    return CRP_OK;
}

// Persistent launches of this many rounds (launch, carry, advance) form one
// CUDA graph; the host looks at the queue once per graph.
constexpr int kRoundsPerGraph = 8;

static crp_status run_persistent(crp_plan *p, const crp_candidates *c, uint64_t n,
                                 const crp_run_opts &o, crp_run_stats *stats) {
    cudaStream_t st = (cudaStream_t)o.stream;
    DevState s = to_dev_state(*c);
    DevRecords rec = to_dev_records(o.records);
    const int ctas = o.ctas_per_sm > 0 ? o.ctas_per_sm : (p->tuned_ctas > 0 ? p->tuned_ctas : 2);
    const int refill = o.refill_threshold > 0 ? o.refill_threshold : (p->tuned_refill > 0 ? p->tuned_refill : 8);
    const int burst = o.steps_per_launch > 0 ? o.steps_per_launch : (p->tuned_burst > 0 ? p->tuned_burst : 16);
    if (ctas > 32 || refill > 32) return fail(CRP_ERR_INVALID_ARGUMENT, "ctas_per_sm and refill_threshold must be <= 32");
    crp_status ls = ensure_lists(p, n);
    if (ls) return ls;
    ls = ensure_graph_resources(p);
    if (ls) return ls;
    const int grid = p->num_sms * ctas;
    const unsigned long long budget_ns =
        o.budget_us > 0 ? 1000ull * (unsigned long long)o.budget_us : 25ull * 1000 * 1000;
    cudaStream_t gs = p->gstream;
    // the graph stream follows the caller's stream
    CUDA_TRY(cudaEventRecord(p->ev_in, st));
    CUDA_TRY(cudaStreamWaitEvent(gs, p->ev_in, 0));
    *p->h_queue = DevQueue{};
    p->h_queue->n_main = n;
    p->h_queue->remaining = n;
    CUDA_TRY(cudaMemcpyAsync(p->d_queue, p->h_queue, sizeof(DevQueue), cudaMemcpyHostToDevice, gs));
    CUDA_TRY(cudaMemsetAsync(p->d_cnt, 0, sizeof(DevCounters), gs));
    CUDA_TRY(cudaStreamSynchronize(gs));  // h_queue is rewritten below

    PersistentArgs a{p->d_queue, p->lists, p->lists + p->list_cap, burst, refill, budget_ns,
                     o.max_steps};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int r = 0; r < kRoundsPerGraph && ce == cudaSuccess; r++) {
        ce = (p->precision == CRP_PRECISION_FP64)
            ? launch_fp64_persistent(p->dev, s, a, p->d_cnt, rec, p->fs, grid, gs)
            : launch_mixed_persistent(p->dev, s, a, p->d_cnt, rec, p->fs, grid, gs);
        if (ce == cudaSuccess) {
            carry_kernel<<<p->num_sms * 2, 256, 0, gs>>>(p->d_queue, p->d_cnt, a.list_a, a.list_b);
            advance_kernel<<<1, 32, 0, gs>>>(p->d_queue, p->d_cnt);
            ce = cudaGetLastError();
        }
    }
    cudaError_t ee = cudaStreamEndCapture(gs, &graph);
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(ce != cudaSuccess ? ce : ee, "capture of the persistent launch graph");
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(ce, "instantiation of the persistent launch graph");

    double ms_total = 0;
    crp_status result = CRP_OK;
    for (;;) {
        cudaError_t e = cudaEventRecord(p->ev0, gs);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec, gs);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev1, gs);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p->h_queue, p->d_queue, sizeof(DevQueue), cudaMemcpyDeviceToHost, gs);
        if (e == cudaSuccess) e = cudaStreamSynchronize(gs);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p->ev0, p->ev1);
        if (e != cudaSuccess) { result = cuda_fail(e, "persistent launch graph"); break; }
        ms_total += ms;
        if (p->h_queue->remaining == 0) break;
        if (o.cancel && *o.cancel) { result = fail(CRP_ERR_CANCELLED, "run cancelled by the host flag"); break; }
    }
    cudaGraphExecDestroy(exec);
    if (stats) {
        stats->particle_steps = p->h_queue->steps;
        stats->tries = p->h_queue->tries;
        stats->field_evaluations = p->h_queue->field_evals;
        stats->launches = p->h_queue->launches;
        stats->active_left = p->h_queue->remaining;
        stats->device_ms = ms_total;
    }
    // the caller's stream follows the graph stream
    CUDA_TRY(cudaEventRecord(p->ev_out, gs));
    CUDA_TRY(cudaStreamWaitEvent(st, p->ev_out, 0));
    return result;
}

// The first launch's input chunks of crp_run(): part k covers candidates
// [bounds[k], bounds[k + 1]) and may start once p->ev_chunk[k] has completed.
struct InputChunks {
    uint64_t bounds[kInputChunks + 1];
};

__global__ void iota_kernel(uint32_t *out, uint64_t n) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = (uint32_t)t;
}

// Streams, events and the identity list of crp_run()'s input pipeline.
static crp_status ensure_pipeline(crp_plan *p, uint64_t n, cudaStream_t st) {
    if (!p->copy_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&p->ev_ready, cudaEventDisableTiming));
        for (int k = 0; k < kInputChunks; k++) {
            CUDA_TRY(cudaStreamCreateWithFlags(&p->part_stream[k], cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&p->ev_chunk[k], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&p->ev_part[k], cudaEventDisableTiming));
        }
    }
    if (p->ident_cap < n) {
        if (p->ident) { cudaFree(p->ident); p->ident = nullptr; p->ident_cap = 0; }
        CUDA_TRY(cudaMalloc(&p->ident, sizeof(uint32_t) * n));
        iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p->ident, n);
        CUDA_TRY(cudaGetLastError());
        p->ident_cap = n;
    }
    return CRP_OK;
}

static crp_status run_device(crp_plan *p, const crp_candidates *c, uint64_t n, const crp_run_opts *opts,
                             crp_run_stats *stats, const InputChunks *in);

crp_status crp_run_device(crp_plan *p, const crp_candidates *c, uint64_t n,
                          const crp_run_opts *opts, crp_run_stats *stats) {
    return run_device(p, c, n, opts, stats, nullptr);
}

static crp_status run_device(crp_plan *p, const crp_candidates *c, uint64_t n, const crp_run_opts *opts,
                             crp_run_stats *stats, const InputChunks *in) {
    if (!p || !c) return fail(CRP_ERR_INVALID_ARGUMENT, "plan or candidates is NULL");
    crp_run_opts o{};
    if (opts) o = *opts;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n == 0) return CRP_OK;
    if (!c->id || !c->charge || !c->energy || !c->x || !c->y || !c->z || !c->dx || !c->dy ||
        !c->dz || !c->px || !c->py || !c->pz || !c->trajectory_length || !c->time ||
        !c->current_step || !c->next_step || !c->active || !c->flags)
        return fail(CRP_ERR_INVALID_ARGUMENT, "a candidate array is NULL");
    if (needs_per_candidate(p) && !c->max_length)
        return fail(CRP_ERR_INVALID_ARGUMENT, "per-candidate MaximumTrajectoryLength needs max_length");
    if (needs_step_count(p) && !c->step_count)
        return fail(CRP_ERR_INVALID_ARGUMENT, "DiffusionSDE needs step_count (random stream counter)");
    if (n > 0xffffffffull) return fail(CRP_ERR_CAPACITY, "at most 2^32-1 candidates per run");
    crp_status ps = check_device_arrays(c, o.records);
    if (ps) return ps;
    int mode = o.mode;
    if (mode == CRP_MODE_AUTO) mode = p->tuned_mode ? p->tuned_mode : CRP_MODE_CHUNKED;
    if (mode == CRP_MODE_PERSISTENT) return run_persistent(p, c, n, o, stats);
    cudaStream_t st = (cudaStream_t)o.stream;
    DevState s = to_dev_state(*c);
    DevRecords rec = to_dev_records(o.records);
    int block = o.block_size > 0 ? o.block_size : (p->tuned_block > 0 ? p->tuned_block : 128);
    if (block % 32 || block <= 0 || block > 128)
        return fail(CRP_ERR_INVALID_ARGUMENT, "block size %d: a multiple of 32 up to 128 (the stepping kernels' "
                    "launch bound)", block);
    // grid runs with the default launch length are cell-ordered between launches
    const int key_bits = (p->fs == FS_GRID || p->fs == FS_GRID_PERIODIC) ? cell_key_bits(p->dev.fields[0].grid) : 0;
    const bool cell_order = o.steps_per_launch <= 0 && key_bits > 0 && n >= kSortMinCandidates;
    int spl = o.steps_per_launch > 0 ? o.steps_per_launch : (cell_order ? kSortedStepsPerLaunch : 4096);
    crp_status ls = ensure_lists(p, n);
    if (ls) return ls;
    if (cell_order) {
        ls = ensure_sort(p, n);
        if (ls) return ls;
    }
    double ms_total = 0;
    uint64_t launches = 0;
    // launch 1 covers every candidate; later launches only the ones the
    // previous launch left active (compacted index list)
    uint64_t n_threads = n;
    const uint32_t *list_in = nullptr;
    uint32_t *list_out = p->lists;
    for (;;) {
        CUDA_TRY(cudaMemsetAsync(p->d_cnt, 0, sizeof(DevCounters), st));
        CUDA_TRY(cudaEventRecord(p->ev0, st));
        // candidates start where their source puts them: order from the second launch on
        if (cell_order && list_in && n_threads >= kSortMinCandidates) {
            ls = order_by_cell(p, s, list_in, n_threads, key_bits, st, &list_in);
            if (ls) return ls;
            launches++;  // the key kernel (the radix sort is CUB's)
        }
        auto step = [&](uint64_t nt, const uint32_t *li, cudaStream_t ss) {
            return (p->precision == CRP_PRECISION_FP64)
                ? launch_fp64_chunk(p->dev, s, nt, spl, o.max_steps, p->d_cnt, rec, li, list_out, p->fs, block, ss)
                : launch_mixed_chunk(p->dev, s, nt, spl, o.max_steps, p->d_cnt, rec, li, list_out, p->fs, block, ss);
        };
        cudaError_t e = cudaSuccess;
        if (in && !list_in) {
            // first launch of crp_run(): each input chunk on its own stream once it has arrived
            for (int k = 0; k < kInputChunks && e == cudaSuccess; k++) {
                const uint64_t a = in->bounds[k], b = in->bounds[k + 1];
                cudaStream_t ps = p->part_stream[k];
                CUDA_TRY(cudaStreamWaitEvent(ps, p->ev0, 0));
                CUDA_TRY(cudaStreamWaitEvent(ps, p->ev_chunk[k], 0));
                if (b > a) e = step(b - a, p->ident + a, ps);
                if (e == cudaSuccess) e = cudaEventRecord(p->ev_part[k], ps);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_part[k], 0);
            }
        } else {
            e = step(n_threads, list_in, st);
        }
        if (e != cudaSuccess) return cuda_fail(e, "stepping kernel launch");
        CUDA_TRY(cudaEventRecord(p->ev1, st));
        CUDA_TRY(cudaMemcpyAsync(p->h_cnt, p->d_cnt, sizeof(DevCounters), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, p->ev0, p->ev1));
        ms_total += ms;
        launches++;
        if (stats) {
            stats->particle_steps += p->h_cnt->steps;
            stats->tries += p->h_cnt->tries;
            stats->field_evaluations += p->h_cnt->field_evals;
            stats->active_left = p->h_cnt->active_left;
        }
        if (p->h_cnt->active_left == 0) break;
        n_threads = p->h_cnt->active_left;
        list_in = list_out;
        list_out = (list_out == p->lists) ? p->lists + p->list_cap : p->lists;
        if (o.cancel && *o.cancel) {
            if (stats) { stats->launches = launches; stats->device_ms = ms_total; }
            return fail(CRP_ERR_CANCELLED, "run cancelled by the host flag");
        }
    }
    if (stats) { stats->launches = launches; stats->device_ms = ms_total; }
    return CRP_OK;
}

crp_status crp_run(crp_plan *p, const crp_candidates *h, uint64_t n, const crp_run_opts *opts,
                   crp_run_stats *stats) {
    if (!p || !h) return fail(CRP_ERR_INVALID_ARGUMENT, "plan or candidates is NULL");
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n == 0) return CRP_OK;
    crp_run_opts o{};
    if (opts) o = *opts;
    cudaStream_t st = (cudaStream_t)o.stream;
    const bool per = h->max_length != nullptr, steps = h->step_count != nullptr;
    // 17 doubles (with max_length and step_count) + id + flags + active per candidate
    const size_t per_cand = 17 * 8 + 4 + 4 + 1;
    const size_t slack = 32 * 256;
    if (p->scratch_n < n) {
        if (p->scratch) { cudaFree(p->scratch); p->scratch = nullptr; p->scratch_n = 0; }
        CUDA_TRY(cudaMalloc(&p->scratch, per_cand * n + slack));
        p->scratch_n = n;
    }
    char *base = static_cast<char *>(p->scratch);
    crp_candidates d{};
    size_t off = 0;
    auto take = [&](size_t bytes) { void *r = base + off; off += (bytes + 255) / 256 * 256; return r; };
    // layout: doubles first (aligned), then 4-byte and 1-byte members
    d.charge = (double *)take(8 * n); d.energy = (double *)take(8 * n);
    d.x = (double *)take(8 * n); d.y = (double *)take(8 * n); d.z = (double *)take(8 * n);
    d.dx = (double *)take(8 * n); d.dy = (double *)take(8 * n); d.dz = (double *)take(8 * n);
    d.px = (double *)take(8 * n); d.py = (double *)take(8 * n); d.pz = (double *)take(8 * n);
    d.trajectory_length = (double *)take(8 * n); d.time = (double *)take(8 * n);
    d.current_step = (double *)take(8 * n); d.next_step = (double *)take(8 * n);
    d.max_length = per ? (double *)take(8 * n) : nullptr;
    d.step_count = steps ? (uint64_t *)take(8 * n) : nullptr;
    d.id = (int32_t *)take(4 * n); d.flags = (uint32_t *)take(4 * n);
    d.active = (uint8_t *)take(n);
    if (off > per_cand * n + slack) return fail(CRP_ERR_CUDA, "scratch layout overflow");
#define D2H(m, bytes) CUDA_TRY(cudaMemcpyAsync(h->m, d.m, (bytes), cudaMemcpyDeviceToHost, st))
    // records: device buffer of the same capacity, copied back afterwards
    crp_records drec{};
    crp_records *hrec = o.records;
    if (hrec) {
        uint64_t cap = hrec->capacity;
        size_t rbytes = 8 + cap * (8 + 4 + 10 * 8 + 4) + 16 * 256;
        if (p->rec_cap < cap || !p->rec_scratch) {
            if (p->rec_scratch) cudaFree(p->rec_scratch);
            p->rec_scratch = nullptr;
            CUDA_TRY(cudaMalloc(&p->rec_scratch, rbytes));
            p->rec_cap = cap;
        }
        char *rb = static_cast<char *>(p->rec_scratch);
        size_t ro = 0;
        auto rtake = [&](size_t bytes) { void *r = rb + ro; ro += (bytes + 255) / 256 * 256; return r; };
        drec.capacity = cap;
        drec.count = (uint64_t *)rtake(8);
        drec.index = (uint64_t *)rtake(8 * cap); drec.module = (int32_t *)rtake(4 * cap);
        drec.trajectory_length = (double *)rtake(8 * cap); drec.time = (double *)rtake(8 * cap);
        drec.x = (double *)rtake(8 * cap); drec.y = (double *)rtake(8 * cap); drec.z = (double *)rtake(8 * cap);
        drec.dx = (double *)rtake(8 * cap); drec.dy = (double *)rtake(8 * cap); drec.dz = (double *)rtake(8 * cap);
        drec.energy = (double *)rtake(8 * cap); drec.id = (int32_t *)rtake(4 * cap);
        CUDA_TRY(cudaMemcpyAsync(drec.count, hrec->count, 8, cudaMemcpyHostToDevice, st));
        o.records = &drec;
    }
    // inputs: one chunk (the whole range on st) or kInputChunks chunks on the copy stream, the
    // first launch starting on each as it arrives (chunked mode, large runs)
    const int mode = o.mode == CRP_MODE_AUTO ? (p->tuned_mode ? p->tuned_mode : CRP_MODE_CHUNKED) : o.mode;
    const bool pipe = mode == CRP_MODE_CHUNKED && n >= kPipelineMinCandidates;
    InputChunks chunks{};
    cudaStream_t cs = st;
    if (pipe) {
        crp_status ps = ensure_pipeline(p, n, st);
        if (ps) return ps;
        // the copies overwrite the scratch: after everything st has queued on it
        CUDA_TRY(cudaEventRecord(p->ev_ready, st));
        CUDA_TRY(cudaStreamWaitEvent(p->copy_stream, p->ev_ready, 0));
        cs = p->copy_stream;
    }
    const int nchunks = pipe ? kInputChunks : 1;
    for (int k = 0; k < nchunks; k++) {
        const uint64_t a = n * k / nchunks, b = n * (k + 1) / nchunks, m = b - a;
        chunks.bounds[k] = a;
        chunks.bounds[k + 1] = b;
#define H2D(f, sz) CUDA_TRY(cudaMemcpyAsync(d.f + a, h->f + a, (sz) * m, cudaMemcpyHostToDevice, cs))
        H2D(charge, 8); H2D(energy, 8); H2D(x, 8); H2D(y, 8); H2D(z, 8);
        H2D(dx, 8); H2D(dy, 8); H2D(dz, 8); H2D(px, 8); H2D(py, 8); H2D(pz, 8);
        H2D(trajectory_length, 8); H2D(time, 8); H2D(current_step, 8); H2D(next_step, 8);
        if (per) H2D(max_length, 8);
        if (steps) H2D(step_count, 8);
        H2D(id, 4); H2D(flags, 4); H2D(active, 1);
#undef H2D
        if (pipe) CUDA_TRY(cudaEventRecord(p->ev_chunk[k], cs));
    }
    crp_status rs = run_device(p, &d, n, &o, stats, pipe ? &chunks : nullptr);
    // no copy from the caller's arrays may still be in flight when this returns
    if (pipe) CUDA_TRY(cudaStreamSynchronize(p->copy_stream));
    if (rs != CRP_OK && rs != CRP_ERR_CANCELLED) return rs;
    D2H(x, 8 * n); D2H(y, 8 * n); D2H(z, 8 * n); D2H(dx, 8 * n); D2H(dy, 8 * n); D2H(dz, 8 * n);
    D2H(px, 8 * n); D2H(py, 8 * n); D2H(pz, 8 * n);
    D2H(trajectory_length, 8 * n); D2H(time, 8 * n); D2H(current_step, 8 * n); D2H(next_step, 8 * n);
    if (steps) D2H(step_count, 8 * n);
    D2H(flags, 4 * n); D2H(active, n);
    if (hrec) {
        CUDA_TRY(cudaMemcpyAsync(hrec->count, drec.count, 8, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        uint64_t k = std::min<uint64_t>(*hrec->count, hrec->capacity);
        if (k) {
#define RD2H(m, sz) CUDA_TRY(cudaMemcpyAsync(hrec->m, drec.m, (sz) * k, cudaMemcpyDeviceToHost, st))
            RD2H(index, 8); RD2H(module, 4); RD2H(trajectory_length, 8); RD2H(time, 8);
            RD2H(x, 8); RD2H(y, 8); RD2H(z, 8); RD2H(dx, 8); RD2H(dy, 8); RD2H(dz, 8);
            RD2H(energy, 8); RD2H(id, 4);
#undef RD2H
        }
    }
#undef D2H
    CUDA_TRY(cudaStreamSynchronize(st));
    return rs;
}

crp_status crp_autotune(crp_plan *p, const crp_candidates *c, uint64_t n, uint64_t sample_n,
                        uint64_t steps_per_candidate, void *stream, crp_autotune_result *res) {
    if (!p || !c || !res) return fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    memset(res, 0, sizeof(*res));
    if (n == 0) return CRP_OK;
    const uint64_t m = sample_n == 0 || sample_n > n ? n : sample_n;
    const uint64_t cap = steps_per_candidate ? steps_per_candidate : 256;
    cudaStream_t st = (cudaStream_t)stream;
    // one device block for the trial copy: 17 double / u64 arrays, id, flags, active
    if (p->trial_n < m) {
        if (p->trial) { cudaFree(p->trial); p->trial = nullptr; p->trial_n = 0; }
        CUDA_TRY(cudaMalloc(&p->trial, (17 * 8 + 9) * m + 32 * 256));
        p->trial_n = m;
    }
    char *base = static_cast<char *>(p->trial);
    size_t off = 0;
    auto take = [&](size_t bytes) { void *r = base + off; off += (bytes + 255) / 256 * 256; return r; };
    crp_candidates t{};
    double **dmem[] = {&t.charge, &t.energy, &t.x, &t.y, &t.z, &t.dx, &t.dy, &t.dz, &t.px, &t.py, &t.pz,
                       &t.trajectory_length, &t.time, &t.current_step, &t.next_step, &t.max_length};
    for (double **d : dmem) *d = (double *)take(8 * m);
    t.step_count = (uint64_t *)take(8 * m);
    t.id = (int32_t *)take(4 * m);
    t.flags = (uint32_t *)take(4 * m);
    t.active = (uint8_t *)take(m);
    auto reset = [&]() -> crp_status {
        const double *const src[] = {c->charge, c->energy, c->x, c->y, c->z, c->dx, c->dy, c->dz,
                                     c->px, c->py, c->pz, c->trajectory_length, c->time,
                                     c->current_step, c->next_step, c->max_length};
        for (int k = 0; k < 16; k++) {
            if (src[k]) CUDA_TRY(cudaMemcpyAsync(*dmem[k], src[k], 8 * m, cudaMemcpyDeviceToDevice, st));
            else CUDA_TRY(cudaMemsetAsync(*dmem[k], 0, 8 * m, st));
        }
        CUDA_TRY(cudaMemsetAsync(t.step_count, 0, 8 * m, st));
        CUDA_TRY(cudaMemcpyAsync(t.id, c->id, 4 * m, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(t.flags, c->flags, 4 * m, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(t.active, c->active, m, cudaMemcpyDeviceToDevice, st));
        return CRP_OK;
    };
    struct Cfg { int mode, ctas, refill, burst; };
    std::vector<Cfg> cfgs = {{CRP_MODE_CHUNKED, 0, 0, 0}};
    for (int ctas : {1, 2, 3, 4, 6})
        for (int refill : {1, 8, 16, 32})
            for (int burst : {4, 16, 64}) cfgs.push_back({CRP_MODE_PERSISTENT, ctas, refill, burst});
    double best = -1, chunked = 0;
    Cfg bestc = cfgs[0];
    int trials = 0;
    for (const Cfg &g : cfgs) {
        crp_status rs = reset();
        if (rs) return rs;
        crp_run_opts o{};
        o.mode = g.mode;
        o.ctas_per_sm = g.ctas;
        o.refill_threshold = g.refill;
        o.steps_per_launch = g.mode == CRP_MODE_PERSISTENT ? g.burst : 0;
        o.max_steps = cap;
        o.stream = stream;
        crp_run_stats rstats{};
        rs = crp_run_device(p, &t, m, &o, &rstats);
        if (rs) return rs;
        trials++;
        const double rate = rstats.device_ms > 0 ? rstats.particle_steps / (rstats.device_ms * 1e-3) : 0;
        if (g.mode == CRP_MODE_CHUNKED) chunked = rate;
        if (rate > best) { best = rate; bestc = g; }
    }
    p->tuned_mode = bestc.mode;
    p->tuned_ctas = bestc.ctas;
    p->tuned_refill = bestc.refill;
    p->tuned_burst = bestc.burst;
    res->mode = bestc.mode;
    res->ctas_per_sm = bestc.ctas;
    res->refill_threshold = bestc.refill;
    res->burst = bestc.burst;
    res->trials = trials;
    res->steps_per_second = best;
    res->chunked_steps_per_second = chunked;
    return CRP_OK;
}

crp_status crp_field_eval(crp_plan *p, uint64_t n, const double *pos, double *out, void *stream) {
    if (!p || (n && (!pos || !out))) return fail(CRP_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaError_t e = (p->precision == CRP_PRECISION_FP64)
        ? launch_fp64_field(p->dev, n, pos, out, (cudaStream_t)stream)
        : launch_mixed_field(p->dev, n, pos, out, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "field kernel launch");
    return CRP_OK;
}

}  // extern "C"
