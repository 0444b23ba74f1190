"""crp_run_device_noalloc: the entry point for callers that cannot allocate.

Callers inside a CUDA-graph capture, under another allocator, or limited to
the buffers their host hands them cannot call cudaMalloc, so they cannot
create a plan.  This entry point runs a fixed-step Boris push over a Grid3f
they already hold on the device, with its scratch in a static device array.

Its results must equal the plan-based entry point's (crp_run_device) bit for
bit -- the tolerance of the FP64 parity tests -- on two calls in a row, the
second of which reuses the scratch the first one left behind.  This file is
collected last so that a run stopping at its first failure has already run
every other test; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, protons, random_grid

pytestmark = pytest.mark.gpu

MEMBERS = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time",
           "current_step", "next_step", "active", "flags")


def _noalloc_desc(d_grid, shape, origin, spacing, step, max_length, precision):
    d = _abi.NoAllocGridBpDesc()
    d.grid_values = d_grid.data_ptr()
    d.nx, d.ny, d.nz = shape
    d.origin[:] = origin
    d.spacing[:] = (spacing,) * 3
    d.step = step
    d.max_length = max_length
    d.precision = precision
    return d


def test_noalloc_matches_plan_run_on_two_calls():
    import torch
    from crpropa3_b200.engine import Plan

    lib = _abi.load()
    rng = np.random.default_rng(77)
    grid = random_grid(rng, 16)
    d_grid = torch.from_numpy(grid).cuda()
    origin, spacing, step, length = (3 * U.kpc, -2 * U.kpc, 0.0), 10 * U.kpc, 1 * U.kpc, 700 * U.kpc
    for call in range(2):
        cands = protons(rng, 3000 + 1000 * call)
        spec = P.ChainSpec([P.GridField(grid, origin, (spacing,) * 3)],
                           [bp_fixed(step), P.MaxTrajectoryLength(length)])
        expected = cands.to_device("cuda")
        Plan(spec).run(expected)

        got = cands.to_device("cuda")
        desc = _noalloc_desc(d_grid, grid.shape[:3], origin, spacing, step, length,
                             _abi.PRECISION_FP64)
        stats = _abi.RunStats()
        s = got.struct()
        _abi.check(lib.crp_run_device_noalloc(C.byref(desc), C.byref(s), cands.n, None,
                                              C.byref(stats)))
        torch.cuda.synchronize()
        a, b = expected.to_host(), got.to_host()
        for name in MEMBERS:
            np.testing.assert_array_equal(getattr(b, name), getattr(a, name),
                                          err_msg=f"call {call}: {name}")
        assert stats.particle_steps > 0
        assert stats.active_left == 0


def test_noalloc_rejects_more_candidates_than_its_scratch_holds():
    lib = _abi.load()
    desc = _abi.NoAllocGridBpDesc()
    desc.grid_values = 1  # never read: the size check comes first
    desc.nx = desc.ny = desc.nz = 4
    desc.step = 1.0
    desc.precision = _abi.PRECISION_FP64
    s = _abi.Candidates()
    st = lib.crp_run_device_noalloc(C.byref(desc), C.byref(s), _abi.NOALLOC_MAX_CANDIDATES + 1,
                                    None, None)
    assert st == _abi.ERR_CAPACITY
    assert "exceed" in _abi.last_error()
