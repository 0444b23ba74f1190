// step_mixed_bp.cu -- the mixed-precision Boris push (PropagationBP) kernels:
// the chunked kernels of the fixed-step and adaptive forms for every field
// signature, and, for the fixed-step push over a periodic power-of-two
// Grid3f, a chunked kernel that advances two candidates per thread.
//
// Why two per thread: one candidate's step is a chain of dependent FP64 and
// FP32 operations around one gather of the midpoint cell's 8 corners, and
// the warps an SM can hold at the register budget this needs are too few to
// cover the gather and the dependences (the one-candidate kernel issues in
// less than half of its cycles).  Two independent candidates in one thread
// share the plan's constants and loop control, and their two chains
// interleave: both candidates' corner loads are in flight before either is
// used.  Each candidate's arithmetic is the one-candidate kernel's, operation
// for operation (the same inline functions), so the results are the same
// bits; only the schedule differs.
#include "mixed_device.cuh"

#ifndef CRP_BP_PAIR_MIN_BLOCKS
#define CRP_BP_PAIR_MIN_BLOCKS 4
#endif

namespace crp {
namespace {

// PropagationBP::process (PropagationBP.cpp:62) in fixed-step mode for two
// charged candidates over a periodic power-of-two grid: BP<FS_GRID_PERIODIC,
// 1>::process for each, interleaved.  kta, ktb: q c step / (2 E) in FP32.
__device__ __forceinline__ void bp_fixed_pair(const DevGrid &g, double step, Cand &a, Cand &b, float kta,
                                              float ktb) {
    const double hh = 0.5 * step;
    a.px = a.x; a.py = a.y; a.pz = a.z;
    b.px = b.x; b.py = b.y; b.pz = b.z;
    double xa = a.x, ya = a.y, za = a.z, uxa = a.dx, uya = a.dy, uza = a.dz;
    double xb = b.x, yb = b.y, zb = b.z, uxb = b.dx, uyb = b.dy, uzb = b.dz;
    xa = fma(uxa, hh, xa); ya = fma(uya, hh, ya); za = fma(uza, hh, za);
    xb = fma(uxb, hh, xb); yb = fma(uyb, hh, yb); zb = fma(uzb, hh, zb);
    const CellFrac fa = grid_cell_load(g, xa, ya, za, a);
    const CellFrac fb = grid_cell_load(g, xb, yb, zb, b);
    const f3 Ba = grid_cell_interp(fa, a);
    const f3 Bb = grid_cell_interp(fb, b);
    bp_rotate_drift(xa, ya, za, uxa, uya, uza, Ba, kta, hh);
    bp_rotate_drift(xb, yb, zb, uxb, uyb, uzb, Bb, ktb, hh);
    renorm(uxa, uya, uza);
    renorm(uxb, uyb, uzb);
    a.x = xa; a.y = ya; a.z = za; a.dx = uxa; a.dy = uya; a.dz = uza;
    b.x = xb; b.y = yb; b.z = zb; b.dx = uxb; b.dy = uyb; b.dz = uzb;
    set_current_step(a, step);
    set_current_step(b, step);
    a.next = step;
    b.next = step;
}

// Chunked launch, two candidates per thread: thread t takes list entries t
// and t + h (h = ceil(n / 2)), so that each load instruction of a warp
// covers 32 consecutive entries of the (cell-ordered) list.  While both are
// active and within the launch's step budget they advance together; then
// the one left runs on alone through the one-candidate chain.
template <int CS>
__global__ void __launch_bounds__(128, CRP_BP_PAIR_MIN_BLOCKS)
mixed_bp_pair_kernel(DevPlan P, DevState s, uint64_t n, int max_steps, uint64_t step_cap, DevCounters *cnt,
                     DevRecords rec, const uint32_t *perm, uint32_t *perm_out) {
    using Prop = BPFixed<FS_GRID_PERIODIC>;
    const uint64_t h = (n + 1) / 2;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    StepCount sc;
    Cand a, b;
    uint64_t ia = 0, ib = 0;
    bool la = false, lb = false;
    if (t < h) {
        ia = perm ? perm[t] : t;
        if (s.active[ia]) { load_cand(s, ia, a); la = true; }
        if (t + h < n) {
            ib = perm ? perm[t + h] : t + h;
            if (s.active[ib]) { load_cand(s, ib, b); lb = true; }
        }
    }
    if (!la) a.active = false;
    if (!lb) b.active = false;
    auto budget = [&](const Cand &c) {
        int kmax = max_steps;
        if (step_cap) {
            const uint64_t left = step_cap > c.steps ? step_cap - c.steps : 0;
            kmax = left < (uint64_t)kmax ? (int)left : kmax;
        }
        return kmax;
    };
    const int kmax_a = la ? budget(a) : 0, kmax_b = lb ? budget(b) : 0;
    int ka = 0, kb = 0;
    const DevModule &pm = P.modules[0];
    if (la && lb && a.q != 0 && b.q != 0) {
        const double step = pm.max_step;
        // BP::process forms these every step; they do not change along the chain
        const float kta = __fdividef((float)(a.q * (0.5 * kCLight)), (float)a.E) * (float)step;
        const float ktb = __fdividef((float)(b.q * (0.5 * kCLight)), (float)b.E) * (float)step;
        const DevGrid &g = P.fields[0].grid;
        while (a.active && b.active && ka < kmax_a && kb < kmax_b) {
            bp_fixed_pair(g, step, a, b, kta, ktb);
            sc.tries += 2; sc.evals += 2;
            max_trajectory_length(P.modules[1], a, rec, 1);
            max_trajectory_length(P.modules[1], b, rec, 1);
            if (CS == CS_PMO) {
                observer(P, P.modules[2], a, rec, 2);
                observer(P, P.modules[2], b, rec, 2);
            }
            ka++; kb++;
        }
    }
    // the candidate still running, if any, goes on alone
    while (a.active && ka < kmax_a) {
        chain_process<Prop, CS>(P, a, rec, sc);
        ka++;
    }
    while (b.active && kb < kmax_b) {
        chain_process<Prop, CS>(P, b, rec, sc);
        kb++;
    }
    bool still_a = false, still_b = false;
    if (la) {
        a.steps += (uint64_t)ka;
        still_a = a.active && (step_cap == 0 || a.steps < step_cap);
        store_cand(s, a);
    }
    if (lb) {
        b.steps += (uint64_t)kb;
        still_b = b.active && (step_cap == 0 || b.steps < step_cap);
        store_cand(s, b);
    }
    flush_counters(cnt, (unsigned long long)(ka + kb), sc);
    append_active(cnt, perm_out, still_a, (uint32_t)ia);
    append_active(cnt, perm_out, still_b, (uint32_t)ib);
}

}  // namespace

int mixed_chunk_max_per_thread(const DevPlan &P, int fs) {
    const DevModule &pm = P.modules[P.prop_index];
    const bool pair = pm.propagator == CRP_PROP_BP && pm.min_step == pm.max_step && fs == FS_GRID_PERIODIC &&
                      P.prop_index == 0 && (P.shape == CS_PM || P.shape == CS_PMO);
    return pair ? 2 : 1;
}

cudaError_t launch_mixed_bp_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                                  uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                                  const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                                  int per_thread, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    if (per_thread == 2 && mixed_chunk_max_per_thread(P, fs) == 2) {
        if (block > 128) block = 128;  // the kernel's launch bounds
        const uint64_t h = (n + 1) / 2;
        const unsigned grid = (unsigned)((h + block - 1) / block);
        if (P.shape == CS_PM)
            mixed_bp_pair_kernel<CS_PM><<<grid, block, 0, st>>>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out);
        else
            mixed_bp_pair_kernel<CS_PMO><<<grid, block, 0, st>>>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out);
        return cudaGetLastError();
    }
    return fixed ? launch_prop<BPFixed>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st)
                 : launch_prop<BPAdaptive>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
}

}  // namespace crp
