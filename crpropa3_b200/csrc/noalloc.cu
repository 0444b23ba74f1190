// noalloc.cu -- crp_run_device_noalloc: fixed-step Boris push over one
// Grid3f with MaximumTrajectoryLength, for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- a host
// process whose device memory belongs to another allocator (a framework's
// caching allocator that owns the whole device, a real-time loop that must
// not block on the driver's allocator), or a plugin that may only touch the
// buffers its host hands it.  Such a caller owns the grid values and the
// candidate arrays; it cannot create a crp_plan, because plan creation
// uploads the grid and allocates the run's scratch.
//
// The scratch of this entry point -- the run counters and the two
// compaction lists of still-active candidate indices -- is a file-scope
// static __device__ array of fixed size, so at most
// CRP_NOALLOC_MAX_CANDIDATES candidates fit in one call.  Every device that
// loads the library holds that array until the process exits.  Host code
// cannot use the array's name as a device address: the first call on each
// device looks its address up with cudaGetSymbolAddress, with that device
// current, and keeps it; make that first call before any stream capture
// begins.  Every call shares the array: the counters are cleared before each
// launch and the lists are written before they are read, so a call never
// depends on what an earlier call left there, but two calls whose work
// overlaps on the GPU race on it.
//
// Between launches the call reads the counters back to the host and waits
// for the stream, so it returns only when the run is complete.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "crp_gpu.h"
#include "engine_internal.h"

namespace crp {
void set_last_error(const char *msg);                        // crp_engine.cu
crp_status check_device_ptr(const void *ptr, const char *what);  // crp_engine.cu
}

using namespace crp;

namespace {

struct NoAllocScratch {
    DevCounters counters;
    uint32_t lists[2 * (size_t)CRP_NOALLOC_MAX_CANDIDATES];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
NoAllocScratch *g_scratch_addr[kMaxDevices] = {};

crp_status noalloc_fail(crp_status st, const char *msg) {
    set_last_error(msg);
    return st;
}

crp_status cuda_noalloc_fail(cudaError_t e, const char *what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    set_last_error(buf);
    return CRP_ERR_CUDA;
}

// Device address of the static scratch on the current device, looked up once
// per device with that device current.
crp_status scratch_for_current_device(NoAllocScratch **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_noalloc_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(CRP_ERR_UNSUPPORTED, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_noalloc_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_addr[dev] = static_cast<NoAllocScratch *>(ptr);
    }
    *out = g_scratch_addr[dev];
    return CRP_OK;
}

}  // namespace

extern "C" crp_status crp_run_device_noalloc(const crp_noalloc_grid_bp_desc *d,
                                             const crp_candidates *c, uint64_t n, void *stream,
                                             crp_run_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!d || !c) return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "desc or candidates is NULL");
    if (n > CRP_NOALLOC_MAX_CANDIDATES) {
        char buf[256];
        snprintf(buf, sizeof(buf),
                 "crp_run_device_noalloc: %llu candidates exceed the fixed scratch of %u; "
                 "split the batch or use crp_run_device",
                 (unsigned long long)n, (unsigned)CRP_NOALLOC_MAX_CANDIDATES);
        return noalloc_fail(CRP_ERR_CAPACITY, buf);
    }
    if (d->precision != CRP_PRECISION_FP64 && d->precision != CRP_PRECISION_MIXED)
        return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "unknown precision");
    if (!d->grid_values || d->nx == 0 || d->ny == 0 || d->nz == 0)
        return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "Grid3f: empty grid");
    if (d->nx > (1u << 20) || d->ny > (1u << 20) || d->nz > (1u << 20))
        return noalloc_fail(CRP_ERR_CAPACITY, "Grid3f: a dimension beyond 2^20 cells");
    if (!(d->step > 0) || !std::isfinite(d->step))
        return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "PropagationBP: step must be finite and > 0");
    for (int a = 0; a < 3; a++) {
        if (!(d->spacing[a] > 0) || !std::isfinite(d->spacing[a]))
            return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "Grid3f: spacing must be finite and > 0");
        if (!std::isfinite(d->origin[a]))
            return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "Grid3f: origin must be finite");
    }
    // a non-finite maximum length would keep candidates active for ever
    if (!std::isfinite(d->max_length))
        return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "MaximumTrajectoryLength: maximum length must be finite");
    if (n == 0) return CRP_OK;
    const void *const arrays[] = {c->id, c->charge, c->energy, c->x, c->y, c->z, c->dx, c->dy, c->dz,
                                  c->px, c->py, c->pz, c->trajectory_length, c->time,
                                  c->current_step, c->next_step, c->active, c->flags};
    for (const void *q : arrays)
        if (!q) return noalloc_fail(CRP_ERR_INVALID_ARGUMENT, "a candidate array is NULL");
    // host or freed pointers become an error here instead of a fault in the kernel
    for (const void *q : arrays) {
        crp_status st = check_device_ptr(q, "crp_run_device_noalloc: a candidate array");
        if (st != CRP_OK) return st;
    }
    {
        crp_status st = check_device_ptr(c->step_count, "crp_run_device_noalloc: step_count");
        if (st == CRP_OK) st = check_device_ptr(d->grid_values, "crp_run_device_noalloc: grid_values");
        if (st != CRP_OK) return st;
    }

    NoAllocScratch *scratch = nullptr;
    crp_status st = scratch_for_current_device(&scratch);
    if (st != CRP_OK) return st;

    // the chain PropagationBP(grid field, step) -> MaximumTrajectoryLength
    DevPlan P{};
    P.n_fields = 1;
    P.n_modules = 2;
    P.prop_index = 0;
    DevComponent &f = P.fields[0];
    f.kind = CRP_FIELD_GRID;
    DevGrid &g = f.grid;
    g.values = d->grid_values;
    g.values4 = nullptr;
    g.nx = (int)d->nx; g.ny = (int)d->ny; g.nz = (int)d->nz;
    g.reflective = d->reflective;
    g.clip_volume = d->clip_volume;
    auto pow2 = [](uint64_t v) { return v && !(v & (v - 1)); };
    g.pow2 = pow2(d->nx) && pow2(d->ny) && pow2(d->nz);
    g.gox = d->origin[0] + d->spacing[0] / 2;
    g.goy = d->origin[1] + d->spacing[1] / 2;
    g.goz = d->origin[2] + d->spacing[2] / 2;
    g.sx = d->spacing[0]; g.sy = d->spacing[1]; g.sz = d->spacing[2];
    g.inv_sx = 1.0 / d->spacing[0]; g.inv_sy = 1.0 / d->spacing[1]; g.inv_sz = 1.0 / d->spacing[2];
    g.ox = d->origin[0]; g.oy = d->origin[1]; g.oz = d->origin[2];
    g.ex = d->origin[0] + (double)d->nx * d->spacing[0];
    g.ey = d->origin[1] + (double)d->ny * d->spacing[1];
    g.ez = d->origin[2] + (double)d->nz * d->spacing[2];
    DevModule &bp = P.modules[0];
    bp.kind = CRP_MODULE_PROPAGATION;
    bp.propagator = CRP_PROP_BP;
    bp.tolerance = 0.42;
    bp.min_step = d->step;
    bp.max_step = d->step;
    DevModule &mtl = P.modules[1];
    mtl.kind = CRP_MODULE_MAX_TRAJECTORY_LENGTH;
    mtl.max_length = d->max_length;

    DevState s{};
    s.id = c->id; s.charge = c->charge; s.energy = c->energy;
    s.x = c->x; s.y = c->y; s.z = c->z;
    s.dx = c->dx; s.dy = c->dy; s.dz = c->dz;
    s.px = c->px; s.py = c->py; s.pz = c->pz;
    s.len = c->trajectory_length; s.time = c->time; s.cur = c->current_step; s.next = c->next_step;
    s.active = c->active; s.flags = c->flags; s.max_length = nullptr; s.steps = c->step_count;
    DevRecords rec{};

    cudaStream_t stm = (cudaStream_t)stream;
    const int spl = d->steps_per_launch > 0 ? d->steps_per_launch : 4096;
    DevCounters *cnt = &scratch->counters;
    uint32_t *list_a = scratch->lists, *list_b = scratch->lists + CRP_NOALLOC_MAX_CANDIDATES;
    uint64_t n_threads = n;
    const uint32_t *list_in = nullptr;
    uint32_t *list_out = list_a;
    for (;;) {
        cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(DevCounters), stm);
        if (e != cudaSuccess) return cuda_noalloc_fail(e, "clearing the scratch counters");
        e = (d->precision == CRP_PRECISION_FP64)
            ? launch_fp64_chunk(P, s, n_threads, spl, 0, cnt, rec, list_in, list_out, FS_GRID, 128, stm)
            : launch_mixed_chunk(P, s, n_threads, spl, 0, cnt, rec, list_in, list_out, FS_GRID, 128, stm);
        if (e != cudaSuccess) return cuda_noalloc_fail(e, "stepping kernel launch");
        DevCounters h;
        e = cudaMemcpyAsync(&h, cnt, sizeof(DevCounters), cudaMemcpyDeviceToHost, stm);
        if (e != cudaSuccess) return cuda_noalloc_fail(e, "reading the scratch counters");
        e = cudaStreamSynchronize(stm);
        if (e != cudaSuccess) return cuda_noalloc_fail(e, "stepping kernel");
        if (stats) {
            stats->particle_steps += h.steps;
            stats->tries += h.tries;
            stats->field_evaluations += h.field_evals;
            stats->launches += 1;
            stats->active_left = h.active_left;
        }
        if (h.active_left == 0) break;
        n_threads = h.active_left;
        list_in = list_out;
        list_out = (list_out == list_a) ? list_b : list_a;
    }
    return CRP_OK;
}
