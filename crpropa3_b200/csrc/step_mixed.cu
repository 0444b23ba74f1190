// step_mixed.cu -- the mixed-precision form of the stepping path.
//
// Same modules and module order as the FP64 form (step_fp64.cu), with the
// arithmetic split by what each quantity needs:
//   * FP64: position, trajectory length, time, the step controller's error
//     sum and its pow(), grid coordinates before the cell split, wave phases
//     before range reduction, and the direction vector (accumulated as
//     u <- u + du with du formed in FP32);
//   * FP32: field interpolation and wave sums, the Boris rotation, the
//     Cash-Karp and DiffusionSDE stage derivatives and their weighted sums.
// Rounding errors of FP32 then enter only through increments that are small
// against the FP64 quantities they are added to, which keeps the
// accumulated error of 10^3-10^6 steps at the FP64 level of the increments'
// relative error times their size.
//
// This unit holds the Cash-Karp, DiffusionSDE and generic kernels and
// their launchers; the fixed-step and adaptive Boris kernels are in
// step_mixed_bp.cu.
#include "mixed_device.cuh"

namespace crp {
namespace {


// Chunked launch of a DiffusionSDE chain in coroutine form (the loop of
// chunk_body, every module of the chain in order, each iteration).
#ifndef CRP_SDE_COOP_MIN_BLOCKS
#define CRP_SDE_COOP_MIN_BLOCKS 1
#endif
// pw_field >= 0: index of the plan's plane-wave component, whose mode
// table the block stages in shared memory (dynamic, 48 B per mode) first.
template <int FS>
__global__ void __launch_bounds__(128, CRP_SDE_COOP_MIN_BLOCKS) mixed_sde_coop_kernel(const __grid_constant__ DevPlan P, DevState s, uint64_t n,
                                                               int max_steps, uint64_t step_cap,
                                                               DevCounters *cnt, DevRecords rec,
                                                               const uint32_t *perm, uint32_t *perm_out,
                                                               int pw_field) {
    extern __shared__ __align__(16) unsigned char pw_smem[];
    PwTab tab{nullptr, 0, 0.0};
    if (pw_field >= 0) {
        const DevPlaneWave &w = P.fields[pw_field].pw;
        float4 *t4 = reinterpret_cast<float4 *>(pw_smem);
        for (int q = threadIdx.x; q < 5 * w.npairs; q += blockDim.x) t4[q] = __ldg(w.pairs + q);
        __syncthreads();
        tab = PwTab{t4, w.npairs, w.fast_limit};
    }
    const PwTab *sh = pw_field >= 0 ? &tab : nullptr;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int pi = P.prop_index;
    const DevModule &pm = P.modules[pi];
    StepCount sc;
    Cand c;
    SdeCo co;
    uint64_t i = 0;
    bool loaded = false, live = false, want = false;
    int k = 0;
    if (t < n) {
        i = perm ? perm[t] : t;
        if (s.active[i]) {
            load_cand(s, i, c);
            loaded = live = true;
        }
    }
    for (;;) {
        while (live && !want) {
            if (!(c.active && k < max_steps && (step_cap == 0 || c.steps < step_cap))) {
                live = false;
                break;
            }
            chain_part(P, c, rec, 0, pi);
            if (sde_co_begin<FS>(P, pm, c, co)) {
                want = true;
            } else {
                chain_part(P, c, rec, pi + 1, P.n_modules);
                c.steps++;
                k++;
            }
        }
        if (!__any_sync(0xffffffffu, want)) break;
        if (want) {
            const f3 B = field_at<FS>(P, co.qx, co.qy, co.qz, &c, sh);
            if (!sde_co_consume(P, pm, c, co, B, sc)) {
                want = false;
                chain_part(P, c, rec, pi + 1, P.n_modules);
                c.steps++;
                k++;
            }
        }
    }
    bool still = false;
    if (loaded) {
        still = c.active && (step_cap == 0 || c.steps < step_cap);
        store_cand(s, c);
    }
    flush_counters(cnt, (unsigned long long)k, sc);
    append_active(cnt, perm_out, still, (uint32_t)i);
}


// ------------------------------------------------ block-batched plane waves
// The DiffusionSDE chunked kernel for fields with one PlaneWaveTurbulence
// component.  A field evaluation of one position is a pass over the whole
// mode table (1024 modes: 40 KB); evaluated lane by lane, every lane reads
// the table once per evaluation (shared-memory wavefronts limit that form).
// Here the block batches them: each round, every lane advances its
// coroutine to its next field query and writes the position into shared
// memory (compacted); then warp g sums mode group g (kPwGroups groups, see
// pw_sum_t) for all the block's positions, each lane up to four positions at
// once, so one broadcast read of a mode pair serves up to eight mode
// evaluations; the lanes then add their four group sums in the order
// pw_sum_t uses and the other field components in field_at's order, and
// continue.  Every sum is formed operation for operation as the lane-by-lane
// form does, so the results are the same bits.
#ifndef CRP_SDE_BATCH_MIN_BLOCKS
#define CRP_SDE_BATCH_MIN_BLOCKS 2
#endif
constexpr int kBatchThreads = 128;  // 4 warps: one per mode group

// Group sums of warp `g` for the positions lane + 32 j (j < NP) of the
// block's query list; positions at or past `total` are computed on the first
// query and not written.
template <int NP, bool ALL_FAST>
__device__ __forceinline__ void pw_batch_group(const float4 *tab, int q0, int q1, const double *qpos, int total,
                                               double lim, float *part, int g) {
    const int lane = threadIdx.x & 31;
    double x[NP], y[NP], z[NP];
    bool fast[NP];
    float acc[NP][6];
#pragma unroll
    for (int j = 0; j < NP; j++) {
        const int p = lane + 32 * j < total ? lane + 32 * j : 0;
        x[j] = qpos[p]; y[j] = qpos[kBatchThreads + p]; z[j] = qpos[2 * kBatchThreads + p];
        fast[j] = fmax(fabs(x[j]), fmax(fabs(y[j]), fabs(z[j]))) < lim;
#pragma unroll
        for (int a = 0; a < 6; a++) acc[j][a] = 0.f;
    }
#pragma unroll 2
    for (int q = q0; q < q1; q++) {
        const double2 *kd = reinterpret_cast<const double2 *>(tab + 5 * q);
        const double2 k0 = kd[0], k1 = kd[1], k2 = kd[2];
        const float4 u = tab[5 * q + 3], v = tab[5 * q + 4];
#pragma unroll
        for (int j = 0; j < NP; j++) {
            if (ALL_FAST || fast[j]) pw_pair_add<true>(k0, k1, k2, u, v, x[j], y[j], z[j], acc[j]);
            else pw_pair_add<false>(k0, k1, k2, u, v, x[j], y[j], z[j], acc[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < NP; j++) {
        const int p = lane + 32 * j;
        if (p < total) {
            float *o = part + (size_t)g * 3 * kBatchThreads;
            o[p] = acc[j][0] + acc[j][3];
            o[kBatchThreads + p] = acc[j][1] + acc[j][4];
            o[2 * kBatchThreads + p] = acc[j][2] + acc[j][5];
        }
    }
}

template <bool ALL_FAST>
__device__ __forceinline__ void pw_batch(const float4 *tab, int npairs, const double *qpos, int total, double lim,
                                         float *part) {
    const int g = threadIdx.x >> 5;
    const int q0 = pw_group_begin(npairs, g), q1 = g + 1 < kPwGroups ? pw_group_begin(npairs, g + 1) : npairs;
    const int np = (total + 31) >> 5;  // positions per lane, uniform over the block
    if (np == 1) pw_batch_group<1, ALL_FAST>(tab, q0, q1, qpos, total, lim, part, g);
    else if (np == 2) pw_batch_group<2, ALL_FAST>(tab, q0, q1, qpos, total, lim, part, g);
    else if (np == 3) pw_batch_group<3, ALL_FAST>(tab, q0, q1, qpos, total, lim, part, g);
    else pw_batch_group<4, ALL_FAST>(tab, q0, q1, qpos, total, lim, part, g);
}

template <int FS>
__global__ void __launch_bounds__(kBatchThreads, CRP_SDE_BATCH_MIN_BLOCKS)
mixed_sde_batch_kernel(const __grid_constant__ DevPlan P, DevState s, uint64_t n, int max_steps, uint64_t step_cap, DevCounters *cnt,
                       DevRecords rec, const uint32_t *perm, uint32_t *perm_out, int pw_field) {
    extern __shared__ __align__(16) unsigned char smem[];
    const DevComponent &pwc = P.fields[pw_field];
    const DevPlaneWave &w = pwc.pw;
    float4 *tab = reinterpret_cast<float4 *>(smem);
    double *qpos = reinterpret_cast<double *>(smem + (size_t)w.npairs * 80);  // [3][128]
    float *part = reinterpret_cast<float *>(qpos + 3 * kBatchThreads);       // [4][3][128]
    int *wcount = reinterpret_cast<int *>(part + kPwGroups * 3 * kBatchThreads);  // [4]
    for (int q = threadIdx.x; q < 5 * w.npairs; q += blockDim.x) tab[q] = __ldg(w.pairs + q);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int pi = P.prop_index;
    const DevModule &pm = P.modules[pi];
    StepCount sc;
    Cand c;
    SdeCo co;
    uint64_t i = 0;
    bool loaded = false, live = false, want = false;
    int k = 0;
    if (t < n) {
        i = perm ? perm[t] : t;
        if (s.active[i]) {
            load_cand(s, i, c);
            loaded = live = true;
        }
    }
    __syncthreads();  // the table is staged
    for (;;) {
        // 1. every lane runs its chain to its next field query
        while (live && !want) {
            if (!(c.active && k < max_steps && (step_cap == 0 || c.steps < step_cap))) {
                live = false;
                break;
            }
            chain_part(P, c, rec, 0, pi);
            if (sde_co_begin<FS>(P, pm, c, co)) {
                want = true;
            } else {
                chain_part(P, c, rec, pi + 1, P.n_modules);
                c.steps++;
                k++;
            }
        }
        // 2. the block's queries, compacted: the plane-wave component's position
        const unsigned bal = __ballot_sync(0xffffffffu, want);
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        int base = 0, total = 0;
#pragma unroll
        for (int g = 0; g < kBatchThreads / 32; g++) {
            const int cg = wcount[g];
            base += g < warp ? cg : 0;
            total += cg;
        }
        if (total == 0) break;  // the same for every thread of the block
        const int slot = base + __popc(bal & ((1u << lane) - 1u));
        bool fast = true;
        if (want) {
            double x = co.qx, y = co.qy, z = co.qz;
            component_position(pwc, x, y, z);
            qpos[slot] = x; qpos[kBatchThreads + slot] = y; qpos[2 * kBatchThreads + slot] = z;
            fast = fmax(fabs(x), fmax(fabs(y), fabs(z))) < w.fast_limit;
        }
        const bool all_fast = __syncthreads_and(fast) != 0;
        // 3. warp g sums mode group g for every query
        if (all_fast) pw_batch<true>(tab, w.npairs, qpos, total, w.fast_limit, part);
        else pw_batch<false>(tab, w.npairs, qpos, total, w.fast_limit, part);
        __syncthreads();
        // 4. each querying lane completes its field and takes it
        if (want) {
            const float *o = part;
            const int S = 3 * kBatchThreads;
            const f3 pw = pw_combine(f3mk(o[slot], o[kBatchThreads + slot], o[2 * kBatchThreads + slot]),
                                     f3mk(o[S + slot], o[S + kBatchThreads + slot], o[S + 2 * kBatchThreads + slot]),
                                     f3mk(o[2 * S + slot], o[2 * S + kBatchThreads + slot],
                                          o[2 * S + 2 * kBatchThreads + slot]),
                                     f3mk(o[3 * S + slot], o[3 * S + kBatchThreads + slot],
                                          o[3 * S + 2 * kBatchThreads + slot]));
            f3 B;
            if (FS == FS_PLANE_WAVE || P.n_fields == 1) {
                B = pw;
            } else {  // field_at's sum over the components, in order
                B = f3mk(0.f, 0.f, 0.f);
#pragma unroll 1
                for (int f = 0; f < P.n_fields; f++) {
                    const f3 cf = f == pw_field ? pw : component_field(P.fields[f], co.qx, co.qy, co.qz);
                    B.x += cf.x; B.y += cf.y; B.z += cf.z;
                }
            }
            if (!sde_co_consume(P, pm, c, co, B, sc)) {
                want = false;
                chain_part(P, c, rec, pi + 1, P.n_modules);
                c.steps++;
                k++;
            }
        }
    }
    bool still = false;
    if (loaded) {
        still = c.active && (step_cap == 0 || c.steps < step_cap);
        store_cand(s, c);
    }
    flush_counters(cnt, (unsigned long long)k, sc);
    append_active(cnt, perm_out, still, (uint32_t)i);
}

template <template <int> class Prop, int FS, int CS>
__global__ void __launch_bounds__(128, MinBlocks<Prop<FS>>::value) mixed_persistent_kernel(
    const __grid_constant__ DevPlan P, DevState s, PersistentArgs a, DevCounters *cnt, DevRecords rec) {
    // the queue is written only between launches (advance_kernel)
    const DevQueue q = *a.q;
    const uint32_t *pending_in = q.cur ? a.list_b : a.list_a;
    uint32_t *pending_out = q.cur ? a.list_a : a.list_b;
    persistent_body<Prop<FS>, CS>(P, s, pending_in, q.n_pending, q.main_base, q.n_main, pending_out,
                              a.burst, a.refill, a.budget_ns, a.step_cap, cnt, rec);
}

template <template <int> class Prop>
cudaError_t launch_persistent_prop(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                   DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                   cudaStream_t st) {
#define CRP_PERSIST(FSV, CSV) mixed_persistent_kernel<Prop, FSV, CSV><<<grid, 128, 0, st>>>(P, s, a, cnt, rec)
    if (fs == FS_GRID_PERIODIC) {
        if (P.shape == CS_PM) CRP_PERSIST(FS_GRID_PERIODIC, CS_PM);
        else if (P.shape == CS_PMO) CRP_PERSIST(FS_GRID_PERIODIC, CS_PMO);
        else CRP_PERSIST(FS_GRID_PERIODIC, CS_GENERIC);
    } else if (fs == FS_GRID) {
        CRP_PERSIST(FS_GRID, CS_GENERIC);
    } else if (fs == FS_PLANE_WAVE) {
        if (P.shape == CS_PM) CRP_PERSIST(FS_PLANE_WAVE, CS_PM);
        else if (P.shape == CS_PMO) CRP_PERSIST(FS_PLANE_WAVE, CS_PMO);
        else CRP_PERSIST(FS_PLANE_WAVE, CS_GENERIC);
    } else {
        CRP_PERSIST(FS_GENERIC, CS_GENERIC);
    }
#undef CRP_PERSIST
    return cudaGetLastError();
}

__global__ void mixed_field_kernel(const __grid_constant__ DevPlan P, uint64_t n, const double *pos, double *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    f3 b = field_at<FS_GENERIC>(P, pos[i], pos[n + i], pos[2 * n + i]);
    out[i] = b.x; out[n + i] = b.y; out[2 * n + i] = b.z;
}

}  // namespace

cudaError_t launch_mixed_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                              uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                              const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                              cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    int prop = P.modules[P.prop_index].propagator;
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    if (prop == CRP_PROP_BP)  // step_mixed_bp.cu
        return launch_mixed_bp_chunk(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
    if (prop == CRP_PROP_CK)
        return fixed ? launch_prop<CKFixed>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st)
                     : launch_prop<CKAdaptive>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
    if (block > 128) block = 128;
    const unsigned grid = (unsigned)((n + block - 1) / block);
    // stage the plane-wave table in shared memory when there is exactly one
    // plane-wave component and its table fits in 96 KB (two blocks per SM)
    int pw_field = -1, n_pw = 0;
    for (int f = 0; f < P.n_fields; f++)
        if (P.fields[f].kind == CRP_FIELD_PLANE_WAVE) { pw_field = f; n_pw++; }
    size_t smem = 0;
    if (n_pw == 1 && (size_t)P.fields[pw_field].pw.npairs * 80 <= 96 * 1024)
        smem = (size_t)P.fields[pw_field].pw.npairs * 80;
    else
        pw_field = -1;
    if (pw_field >= 0 && (fs == FS_PLANE_WAVE || fs == FS_GENERIC)) {
        // block-batched plane-wave sums: the table, the block's query positions,
        // the four group sums per query and the warp counts
        const size_t bsmem = smem + 3 * kBatchThreads * sizeof(double) +
                             kPwGroups * 3 * kBatchThreads * sizeof(float) + 4 * sizeof(int);
        const unsigned bgrid = (unsigned)((n + kBatchThreads - 1) / kBatchThreads);
#define CRP_SDE_BATCH(FSV)                                                                               \
    do {                                                                                                 \
        if (bsmem > 48 * 1024)                                                                           \
            cudaFuncSetAttribute(mixed_sde_batch_kernel<FSV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)bsmem);                                                            \
        mixed_sde_batch_kernel<FSV><<<bgrid, kBatchThreads, bsmem, st>>>(P, s, n, max_steps, step_cap, cnt, \
                                                                        rec, perm, perm_out, pw_field);  \
    } while (0)
        if (fs == FS_PLANE_WAVE) CRP_SDE_BATCH(FS_PLANE_WAVE);
        else CRP_SDE_BATCH(FS_GENERIC);
#undef CRP_SDE_BATCH
        return cudaGetLastError();
    }
#define CRP_SDE_COOP(FSV)                                                                              \
    do {                                                                                               \
        if (smem > 48 * 1024)                                                                          \
            cudaFuncSetAttribute(mixed_sde_coop_kernel<FSV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (int)smem);                                                           \
        mixed_sde_coop_kernel<FSV><<<grid, block, smem, st>>>(P, s, n, max_steps, step_cap, cnt, rec,  \
                                                              perm, perm_out, pw_field);               \
    } while (0)
    if (fs == FS_GRID || fs == FS_GRID_PERIODIC) CRP_SDE_COOP(FS_GRID);
    else if (fs == FS_PLANE_WAVE) CRP_SDE_COOP(FS_PLANE_WAVE);
    else CRP_SDE_COOP(FS_GENERIC);
#undef CRP_SDE_COOP
    return cudaGetLastError();
}

cudaError_t launch_mixed_persistent(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                   DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                   cudaStream_t st) {
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    if (pm.propagator == CRP_PROP_BP)
        return fixed ? launch_persistent_prop<BPFixed>(P, s, a, cnt, rec, fs, grid, st)
                     : launch_persistent_prop<BPAdaptive>(P, s, a, cnt, rec, fs, grid, st);
    if (pm.propagator == CRP_PROP_CK)
        return fixed ? launch_persistent_prop<CKFixed>(P, s, a, cnt, rec, fs, grid, st)
                     : launch_persistent_prop<CKAdaptive>(P, s, a, cnt, rec, fs, grid, st);
    return launch_persistent_prop<SDE>(P, s, a, cnt, rec, fs, grid, st);
}

cudaError_t launch_mixed_field(const DevPlan &P, uint64_t n, const double *pos, double *out,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    mixed_field_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(P, n, pos, out);
    return cudaGetLastError();
}


}  // namespace crp
