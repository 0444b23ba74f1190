// engine_internal.h -- declarations shared between the host engine
// (crp_engine.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_plan.cuh"

namespace crp {

// Field signature the stepping kernels are specialised for.
enum FieldSig {
    FS_GENERIC = 0,    // any sum of (possibly periodic) components
    FS_GRID = 1,       // one MagneticFieldGrid, not wrapped
    FS_PLANE_WAVE = 2, // one PlaneWaveTurbulence, not wrapped
    FS_GRID_PERIODIC = 3  // FS_GRID with a periodic grid of power-of-two dimensions, no
                          // clipVolume (and the padded copy, mixed form): no runtime checks
};

// Persistent stepping launch (chain.cuh persistent_body): `grid` CTAs of 128
// threads take work from the virtual queue described by *q -- its pending
// list (list_a or list_b, by q->cur) followed by its main range -- until it
// is empty or budget_ns of device time have passed; unfinished candidates
// go to the other list.  Kernel parameters are fixed for a whole run, so
// the launches can be captured in a CUDA graph.
struct PersistentArgs {
    const DevQueue *q;
    uint32_t *list_a;
    uint32_t *list_b;
    int burst;
    int refill;
    unsigned long long budget_ns;
    uint64_t step_cap;
};

// step_fp64.cu
// One launch of the chunked stepping kernel: threads t < n advance candidate
// perm[t] (t without perm) by at most max_steps chain iterations; candidates
// still active afterwards are appended to perm_out (may be null) and counted
// in cnt->active_left.
cudaError_t launch_fp64_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                              uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                              const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                              cudaStream_t st);
cudaError_t launch_fp64_field(const DevPlan &P, uint64_t n, const double *pos, double *out,
                              cudaStream_t st);
cudaError_t launch_fp64_persistent(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                   DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                   cudaStream_t st);

// step_mixed.cu
cudaError_t launch_mixed_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                               uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                               const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                               cudaStream_t st);
// step_mixed_bp.cu: the Boris-push part of launch_mixed_chunk
cudaError_t launch_mixed_bp_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                                  uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                                  const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                                  cudaStream_t st);
cudaError_t launch_mixed_persistent(const DevPlan &P, const DevState &s, const PersistentArgs &a,
                                    DevCounters *cnt, const DevRecords &rec, int fs, int grid,
                                    cudaStream_t st);
cudaError_t launch_mixed_field(const DevPlan &P, uint64_t n, const double *pos, double *out,
                               cudaStream_t st);

}  // namespace crp
