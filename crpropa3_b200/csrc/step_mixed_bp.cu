// step_mixed_bp.cu -- the mixed-precision Boris push (PropagationBP) kernels:
// the chunked kernels of the fixed-step and adaptive forms for every field
// signature (the other mixed kernels are in step_mixed.cu; both units share
// mixed_device.cuh).
#include "mixed_device.cuh"

namespace crp {

cudaError_t launch_mixed_bp_chunk(const DevPlan &P, const DevState &s, uint64_t n, int max_steps,
                                  uint64_t step_cap, DevCounters *cnt, const DevRecords &rec,
                                  const uint32_t *perm, uint32_t *perm_out, int fs, int block,
                                  cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const DevModule &pm = P.modules[P.prop_index];
    const bool fixed = pm.min_step == pm.max_step;
    return fixed ? launch_prop<BPFixed>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st)
                 : launch_prop<BPAdaptive>(P, s, n, max_steps, step_cap, cnt, rec, perm, perm_out, fs, block, st);
}

}  // namespace crp
