// chain.cuh -- per-candidate register state, the counter-based random
// stream, the break condition and observer modules, output records, and the
// ModuleList loop.  Shared by the FP64 and the mixed-precision translation
// units; the propagation modules come in through the Prop template argument.
#pragma once

#include "device_plan.cuh"
#include "crp_gpu.h"

namespace crp {

// include/crpropa/Units.h:55, :114-115
constexpr double kCLight = 2.99792458e8;
constexpr double kPi = 3.14159265358979323846;
#define CRP_KPC (1e3 * (648000 / 3.14159265358979323846 * 149597870700.0))

// Candidate state while it is being stepped (Candidate.h:27).
struct Cand {
    double x, y, z;     // current position
    double dx, dy, dz;  // current direction
    double px, py, pz;  // previous position
    double E, q;
    double len, time, cur, next, maxlen;
    uint64_t index, steps;
    uint32_t flags;
    int32_t id;
    bool active;
    // The Grid3f cell the last interpolation read: linear indices of its
    // first and last corner and the 8 corner vectors.  A candidate stays in
    // one cell for several steps, so the gathers are skipped while it does;
    // the values are the grid's own, so results do not change.
    long long cell0, cell7;
    float corner[8][3];
};

__device__ __forceinline__ void load_cand(const DevState &s, uint64_t i, Cand &c) {
    c.x = s.x[i]; c.y = s.y[i]; c.z = s.z[i];
    c.dx = s.dx[i]; c.dy = s.dy[i]; c.dz = s.dz[i];
    c.px = s.px[i]; c.py = s.py[i]; c.pz = s.pz[i];
    c.E = s.energy[i]; c.q = s.charge[i];
    c.len = s.len[i]; c.time = s.time[i]; c.cur = s.cur[i]; c.next = s.next[i];
    c.maxlen = s.max_length ? s.max_length[i] : 0.0;
    c.index = i;
    c.steps = s.steps ? s.steps[i] : 0;
    c.flags = s.flags[i];
    c.id = s.id[i];
    c.active = s.active[i] != 0;
    c.cell0 = -1;
    c.cell7 = -1;
}

__device__ __forceinline__ void store_cand(const DevState &s, const Cand &c) {
    uint64_t i = c.index;
    s.x[i] = c.x; s.y[i] = c.y; s.z[i] = c.z;
    s.dx[i] = c.dx; s.dy[i] = c.dy; s.dz[i] = c.dz;
    s.px[i] = c.px; s.py[i] = c.py; s.pz[i] = c.pz;
    s.len[i] = c.len; s.time[i] = c.time; s.cur[i] = c.cur; s.next[i] = c.next;
    if (s.steps) s.steps[i] = c.steps;
    s.flags[i] = c.flags;
    s.active[i] = c.active ? 1 : 0;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint32_t lo0 = 0xD2511F53u * ctr.x, hi0 = __umulhi(0xD2511F53u, ctr.x);
        uint32_t lo1 = 0xCD9E8D57u * ctr.z, hi1 = __umulhi(0xCD9E8D57u, ctr.z);
        ctr = make_uint4(hi1 ^ ctr.y ^ k0, lo1, hi0 ^ ctr.w ^ k1, lo0);
    }
    return ctr;
}

// The per-step stream of one candidate: word w of step s of candidate i is
// word w%4 of Philox(ctr = {lo(4s+w/4), hi(4s+w/4), lo(i), hi(i)}, key = seed).
struct Stream {
    uint64_t seed, cand, step;
    uint4 block;
    int cursor;
    __device__ uint32_t next_u32() {
        int w = cursor++;
        if ((w & 3) == 0) {
            uint64_t c = step * 4 + (uint64_t)(w >> 2);
            block = philox4x32_10(make_uint4((uint32_t)c, (uint32_t)(c >> 32), (uint32_t)cand,
                                             (uint32_t)(cand >> 32)),
                                  (uint32_t)seed, (uint32_t)(seed >> 32));
        }
        switch (w & 3) {
        case 0: return block.x;
        case 1: return block.y;
        case 2: return block.z;
        default: return block.w;
        }
    }
    // continue the stream at word w (as if w words had been drawn)
    __device__ void seek(int w) {
        cursor = w;
        if (w & 3) {
            uint64_t c = step * 4 + (uint64_t)(w >> 2);
            block = philox4x32_10(make_uint4((uint32_t)c, (uint32_t)(c >> 32), (uint32_t)cand,
                                             (uint32_t)(cand >> 32)),
                                  (uint32_t)seed, (uint32_t)(seed >> 32));
        }
    }
};

__device__ __forceinline__ void write_record(const DevRecords &rec, const Cand &c, int module) {
    if (!rec.count) return;
    unsigned long long slot = atomicAdd(rec.count, 1ull);
    if (slot >= rec.capacity) return;
    rec.index[slot] = c.index;
    rec.module[slot] = module;
    rec.len[slot] = c.len;
    rec.time[slot] = c.time;
    rec.x[slot] = c.x; rec.y[slot] = c.y; rec.z[slot] = c.z;
    rec.dx[slot] = c.dx; rec.dy[slot] = c.dy; rec.dz[slot] = c.dz;
    rec.energy[slot] = c.E;
    rec.id[slot] = c.id;
}

// Per-thread counts of one launch (32-bit: a launch is bounded in steps or
// device time), added to the run counters once per warp at its end.
struct StepCount {
    unsigned tries = 0;
    unsigned evals = 0;
};

// MaximumTrajectoryLength::process (BreakCondition.cpp:42) and
// AbstractCondition::reject (Module.cpp:25).
__device__ __forceinline__ void max_trajectory_length(const DevModule &m, Cand &c,
                                                      const DevRecords &rec, int mi) {
    double maxLength = m.per_candidate ? c.maxlen : m.max_length;
    if (c.len >= maxLength) {
        if (m.record) write_record(rec, c, mi);
        c.flags |= CRP_FLAG_REJECTED;
        c.active = false;
    } else {
        double lim = maxLength - c.len;
        c.next = (lim < c.next) ? lim : c.next;  // Candidate::limitNextStep (Candidate.cpp:102)
    }
}

// Arithmetic of the reference's geometry in double precision without
// contraction (this header is also compiled where multiply-adds are fused):
// |v| = sqrt(x*x + y*y + z*z) (Vector3::getR), n.v = x*v.x + y*v.y + z*v.z.
__device__ __forceinline__ double nc_norm(double x, double y, double z) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}
__device__ __forceinline__ double nc_dot(double ax, double ay, double az, double bx, double by, double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}
__device__ __forceinline__ double dmin_std(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax_std(double a, double b) { return (a < b) ? b : a; }  // std::max
// Candidate::limitNextStep (Candidate.cpp:102)
__device__ __forceinline__ void limit_next(Cand &c, double step) { c.next = (step < c.next) ? step : c.next; }

// ParticleID.cpp:37 isNucleus (neutron counted) with HepPID::isNucleus
// (ParticleIDMethods.cc:242): proton, or +/-10LZZZAAAI with A >= Z.
__device__ __forceinline__ bool is_nucleus(int id) {
    if (id == 2112) return true;
    const int a = id < 0 ? -id : id;
    if (a == 2212) return true;
    if ((a / 1000000000) % 10 == 1 && (a / 100000000) % 10 == 0)
        return (a / 10) % 1000 >= (a / 10000) % 1000;
    return false;
}

// Surface::distance of the observer surfaces (Geometry.cpp:19, 41, 64).
__device__ __forceinline__ double surface_distance(const DevFeature &f, double x, double y, double z) {
    if (f.kind == CRP_OBSERVER_SURFACE_SPHERE)
        return __dsub_rn(nc_norm(__dsub_rn(x, f.ax), __dsub_rn(y, f.ay), __dsub_rn(z, f.az)), f.r);
    if (f.kind == CRP_OBSERVER_SURFACE_PLANE)
        return nc_dot(f.bx, f.by, f.bz, __dsub_rn(x, f.ax), __dsub_rn(y, f.ay), __dsub_rn(z, f.az));
    // ParaxialBox: X = point - corner - size / 2
    const double hx = f.bx / 2., hy = f.by / 2., hz = f.bz / 2.;
    const double X = __dsub_rn(__dsub_rn(x, f.ax), hx), Y = __dsub_rn(__dsub_rn(y, f.ay), hy),
                 Z = __dsub_rn(__dsub_rn(z, f.az), hz);
    if ((fabs(X) <= hx) && (fabs(Y) <= hy) && (fabs(Z) <= hz)) {
        const double d = dmin_std(__dsub_rn(hx, fabs(X)), dmin_std(__dsub_rn(hy, fabs(Y)), __dsub_rn(hz, fabs(Z))));
        return -1. * d;
    }
    const double a = dmax_std(0., __dsub_rn(fabs(X), hx)), b = dmax_std(0., __dsub_rn(fabs(Y), hy)),
                 cc = dmax_std(0., __dsub_rn(fabs(Z), hz));
    return nc_norm(a, b, cc);
}

enum { DET_NOTHING = 0, DET_DETECTED = 1, DET_VETO = 2 };

// ObserverFeature::checkDetection of each feature (Observer.cpp:93-394).
__device__ __forceinline__ int check_feature(const DevFeature &f, Cand &c) {
    switch (f.kind) {
    case CRP_OBSERVER_SURFACE_SPHERE:
    case CRP_OBSERVER_SURFACE_PLANE:
    case CRP_OBSERVER_SURFACE_BOX: {  // ObserverSurface (Observer.cpp:394)
        const double cd = surface_distance(f, c.x, c.y, c.z);
        const double pd = surface_distance(f, c.px, c.py, c.pz);
        limit_next(c, fabs(cd));
        if (__dmul_rn(cd, pd) > 0) return DET_NOTHING;
        if (pd == 0) return DET_NOTHING;
        return DET_DETECTED;
    }
    case CRP_OBSERVER_DETECT_ALL: return DET_DETECTED;
    case CRP_OBSERVER_TRACKING: {
        const double d = nc_norm(__dsub_rn(c.x, f.ax), __dsub_rn(c.y, f.ay), __dsub_rn(c.z, f.az));
        if (d > f.r) {
            limit_next(c, fabs(__dsub_rn(d, f.r)));
            return DET_NOTHING;
        }
        limit_next(c, f.step);
        return DET_DETECTED;
    }
    case CRP_OBSERVER_1D:
        if (c.x > 0) {
            limit_next(c, c.x);
            return DET_NOTHING;
        }
        return DET_DETECTED;
    case CRP_OBSERVER_INACTIVE_VETO: return c.active ? DET_NOTHING : DET_VETO;
    case CRP_OBSERVER_NUCLEUS_VETO: return is_nucleus(c.id) ? DET_VETO : DET_NOTHING;
    case CRP_OBSERVER_NEUTRINO_VETO: {
        const int a = c.id < 0 ? -c.id : c.id;
        return (a == 12 || a == 14 || a == 16) ? DET_VETO : DET_NOTHING;
    }
    case CRP_OBSERVER_PHOTON_VETO: return c.id == 22 ? DET_VETO : DET_NOTHING;
    case CRP_OBSERVER_ELECTRON_VETO: return (c.id == 11 || c.id == -11) ? DET_VETO : DET_NOTHING;
    default: return c.id == f.pid ? DET_VETO : DET_NOTHING;  // CRP_OBSERVER_PARTICLE_ID_VETO
    }
}

// Observer::process (Observer.cpp:27): every feature checked in order (each
// may limit the next step); detected when one detects and none vetoes.
__device__ __forceinline__ void observer(const DevPlan &P, const DevModule &m, Cand &c,
                                         const DevRecords &rec, int mi) {
    int state = DET_NOTHING;
#pragma unroll 1
    for (int f = 0; f < m.nfeat; f++) {
        const int st = check_feature(P.feat[m.feat0 + f], c);
        if (st == DET_VETO) state = DET_VETO;
        else if (st == DET_DETECTED && state != DET_VETO) state = DET_DETECTED;
    }
    if (state == DET_DETECTED) {
        if (m.record) write_record(rec, c, mi);
        c.flags |= CRP_FLAG_DETECTED;
        if (m.deactivate) c.active = false;
    }
}

// AbstractCondition::reject (Module.cpp:25) of a boundary.
__device__ __forceinline__ void reject(const DevModule &m, Cand &c, const DevRecords &rec, int mi) {
    if (m.record) write_record(rec, c, mi);
    c.flags |= CRP_FLAG_REJECTED;
    c.active = false;
}

// CubicBoundary, SphericalBoundary, EllipsoidalBoundary, CylindricalBoundary
// ::process (Boundary.cpp:171, 216, 259, 303).
__device__ __forceinline__ void boundary(const DevModule &m, Cand &c, const DevRecords &rec, int mi) {
    if (m.boundary == CRP_BOUNDARY_CUBIC) {
        const double rx = __dsub_rn(c.x, m.cx), ry = __dsub_rn(c.y, m.cy), rz = __dsub_rn(c.z, m.cz);
        const double lo = dmin_std(rx, dmin_std(ry, rz)), hi = dmax_std(rx, dmax_std(ry, rz));
        if ((lo <= 0) || (hi >= m.bsize)) reject(m, c, rec, mi);
        if (m.limit_step) {
            limit_next(c, __dadd_rn(lo, m.margin));
            limit_next(c, __dadd_rn(__dsub_rn(m.bsize, hi), m.margin));
        }
    } else if (m.boundary == CRP_BOUNDARY_SPHERICAL) {
        const double d = nc_norm(__dsub_rn(c.x, m.cx), __dsub_rn(c.y, m.cy), __dsub_rn(c.z, m.cz));
        if (d >= m.bsize) reject(m, c, rec, mi);
        if (m.limit_step) limit_next(c, __dadd_rn(__dsub_rn(m.bsize, d), m.margin));
    } else if (m.boundary == CRP_BOUNDARY_ELLIPSOIDAL) {
        const double d = __dadd_rn(nc_norm(__dsub_rn(c.x, m.cx), __dsub_rn(c.y, m.cy), __dsub_rn(c.z, m.cz)),
                                   nc_norm(__dsub_rn(c.x, m.bx), __dsub_rn(c.y, m.by), __dsub_rn(c.z, m.bz)));
        if (d >= m.bsize) reject(m, c, rec, mi);
        if (m.limit_step) limit_next(c, __dadd_rn(__dsub_rn(m.bsize, d), m.margin));
    } else {  // CRP_BOUNDARY_CYLINDRICAL; pow(v, 2.) and pow(v, 0.5) as v*v and sqrt(v)
        const double dx = __dsub_rn(c.x, m.cx), dy = __dsub_rn(c.y, m.cy), dz = __dsub_rn(c.z, m.cz);
        const double R2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        const double Z = fabs(dz);
        if (R2 < __dmul_rn(m.bradius, m.bradius) && Z < m.bsize / 2.) {
            if (m.limit_step)
                limit_next(c, __dadd_rn(dmin_std(__dsub_rn(m.bradius, __dsqrt_rn(R2)), __dsub_rn(m.bsize / 2., Z)),
                                        m.margin));
            return;
        }
        reject(m, c, rec, mi);
    }
}

// ModuleList::process (ModuleList.cpp.in:54): every module of the chain, in
// order, whether or not an earlier module deactivated the candidate; a
// compiled module sequence for the chain shapes of device_plan.cuh, else the
// module list walked in order.
template <class Prop, int CS = CS_GENERIC>
__device__ __forceinline__ void chain_process(const DevPlan &P, Cand &c, const DevRecords &rec,
                                              StepCount &sc) {
    if (CS == CS_PM || CS == CS_PMO) {
        Prop::process(P, P.modules[0], c, sc);
        max_trajectory_length(P.modules[1], c, rec, 1);
        if (CS == CS_PMO) observer(P, P.modules[2], c, rec, 2);
        return;
    }
#pragma unroll 1
    for (int mi = 0; mi < P.n_modules; mi++) {
        const DevModule &m = P.modules[mi];
        if (m.kind == CRP_MODULE_PROPAGATION) Prop::process(P, m, c, sc);
        else if (m.kind == CRP_MODULE_MAX_TRAJECTORY_LENGTH) max_trajectory_length(m, c, rec, mi);
        else if (m.kind == CRP_MODULE_OBSERVER) observer(P, m, c, rec, mi);
        else boundary(m, c, rec, mi);
    }
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Add this thread's counts to the run counters, one atomic per warp.
__device__ __forceinline__ void flush_counters(DevCounters *cnt, unsigned long long steps,
                                               const StepCount &sc) {
    unsigned long long s = warp_sum(steps), t = warp_sum((unsigned long long)sc.tries),
                       e = warp_sum((unsigned long long)sc.evals);
    if ((threadIdx.x & 31) == 0) {
        if (s) atomicAdd(&cnt->steps, s);
        if (t) atomicAdd(&cnt->tries, t);
        if (e) atomicAdd(&cnt->field_evals, e);
    }
}

// Compaction of the candidates that are still active after a launch: the
// warp's ballot gives each such lane its slot, one atomic per warp reserves
// the warp's slots in `list` (which may be null: count only).  The count is
// cnt->active_left.
__device__ __forceinline__ void append_active(DevCounters *cnt, uint32_t *list, bool still,
                                              uint32_t index) {
    const unsigned mask = __ballot_sync(0xffffffffu, still);
    if (!mask) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&cnt->active_left, (unsigned long long)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (still && list) list[base + __popc(mask & ((1u << lane) - 1u))] = index;
}

// One thread per candidate, at most max_steps chain iterations per launch.
// perm_in (optional) maps thread -> candidate index; the candidates still
// active afterwards are appended to perm_out (optional).
template <class Prop, int CS = CS_GENERIC>
__device__ __forceinline__ void chunk_body(const DevPlan &P, const DevState &s, uint64_t n,
                                           int max_steps, uint64_t step_cap,
                                           DevCounters *cnt, const DevRecords &rec,
                                           const uint32_t *perm_in, uint32_t *perm_out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    StepCount sc;
    unsigned long long steps = 0;
    bool still = false;
    uint64_t i = 0;
    if (t < n) {
        i = perm_in ? perm_in[t] : t;
        if (s.active[i]) {
            Cand c;
            load_cand(s, i, c);
            // iterations this launch may take: max_steps, and what the
            // per-candidate cap leaves; c.steps is kept current inside the
            // loop only for modules that read it (Prop::kReadsStepCount)
            int kmax = max_steps;
            if (step_cap) {
                const uint64_t left = step_cap > c.steps ? step_cap - c.steps : 0;
                kmax = left < (uint64_t)kmax ? (int)left : kmax;
            }
            int k = 0;
            while (c.active && k < kmax) {
                chain_process<Prop, CS>(P, c, rec, sc);
                if (Prop::kReadsStepCount) c.steps++;
                k++;
            }
            if (!Prop::kReadsStepCount) c.steps += (uint64_t)k;
            steps = (unsigned long long)k;
            still = c.active && (step_cap == 0 || c.steps < step_cap);
            store_cand(s, c);
        }
    }
    flush_counters(cnt, steps, sc);
    append_active(cnt, perm_out, still, (uint32_t)i);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Persistent stepping (one launch of SMs x ctas_per_sm CTAs): every lane
// holds one candidate; a lane whose candidate finishes is refilled from the
// work queue.  The queue is the virtual list of n_pending indices in
// pending_in followed by the main index range [main_base, main_base +
// n_main).  A warp refills once at least `refill` of its lanes are free (the
// ballot of free lanes ranks them; one atomic per warp reserves their
// items), runs `burst` chain iterations between refills, and stops after
// budget_ns of device time: lanes that still hold a candidate then store it
// and append its index to pending_out (cnt->pending_count), for the next
// launch.  cnt->queue_head counts the items taken.
template <class Prop, int CS = CS_GENERIC>
__device__ __forceinline__ void persistent_body(const DevPlan &P, const DevState &s,
                                                const uint32_t *pending_in, uint64_t n_pending,
                                                uint64_t main_base, uint64_t n_main,
                                                uint32_t *pending_out, int burst, int refill,
                                                unsigned long long budget_ns, uint64_t step_cap,
                                                DevCounters *cnt, const DevRecords &rec) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint64_t total = n_pending + n_main;
    const unsigned long long t0 = global_ns();
    StepCount sc;
    unsigned long long steps = 0;
    Cand c;
    c.cell0 = -1;
    c.cell7 = -1;
    bool has = false, exhausted = false;
    for (;;) {
        const unsigned freemask = __ballot_sync(full, !has);
        const int nfree = __popc(freemask);
        if (!exhausted && nfree > 0 && (nfree >= refill || nfree == 32)) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(&cnt->queue_head, (unsigned long long)nfree);
            base = __shfl_sync(full, base, 0);
            if (base + nfree >= total) exhausted = true;
            if (!has) {
                const uint64_t t = base + __popc(freemask & ((1u << lane) - 1u));
                if (t < total) {
                    const uint64_t i = t < n_pending ? (uint64_t)pending_in[t] : main_base + (t - n_pending);
                    if (s.active[i] && (step_cap == 0 || (s.steps ? s.steps[i] : 0) < step_cap)) {
                        load_cand(s, i, c);
                        has = true;
                    }
                }
            }
        }
        if (!__ballot_sync(full, has)) {
            if (exhausted) break;
            continue;
        }
        if (has) {
            int kmax = burst;
            if (step_cap) {
                const uint64_t left = step_cap > c.steps ? step_cap - c.steps : 0;
                kmax = left < (uint64_t)kmax ? (int)left : kmax;
            }
            int k = 0;
            while (c.active && k < kmax) {
                chain_process<Prop, CS>(P, c, rec, sc);
                if (Prop::kReadsStepCount) c.steps++;
                k++;
            }
            if (!Prop::kReadsStepCount) c.steps += (uint64_t)k;
            steps += (unsigned long long)k;
            if (!c.active || (step_cap != 0 && c.steps >= step_cap)) {
                store_cand(s, c);
                has = false;
            }
        }
        bool stop = false;
        if (lane == 0) stop = global_ns() - t0 > budget_ns;
        stop = __shfl_sync(full, stop, 0);
        if (stop) {
            if (has) store_cand(s, c);
            const unsigned mask = __ballot_sync(full, has);
            if (mask) {
                unsigned long long pb = 0;
                if (lane == 0) pb = atomicAdd(&cnt->pending_count, (unsigned long long)__popc(mask));
                pb = __shfl_sync(full, pb, 0);
                if (has) pending_out[pb + __popc(mask & ((1u << lane) - 1u))] = (uint32_t)c.index;
            }
            break;
        }
    }
    flush_counters(cnt, steps, sc);
}

}  // namespace crp
