"""crp_run_device_noalloc: the entry point for callers that cannot allocate.

Some callers may not call cudaMalloc: a process whose device memory belongs
to another allocator (a framework's caching allocator that owns the device),
or a plugin limited to the buffers its host hands it.  They cannot create a
plan, so this entry point runs a fixed-step Boris push over a Grid3f they
already hold on the device, with its scratch in a static device array.

Its results must equal the plan-based entry point's (crp_run_device): bit for
bit in the FP64 form (the tolerance of the FP64 parity tests), and within the
mixed form's stated bound (1e-6 relative final position) in the mixed form,
on two calls in a row, the second of which reuses the scratch the first one
left behind.  Periodic, reflective and clipVolume grids are covered.  This
file is collected last so that a run stopping at its first failure has
already run every other test; it passes alone in a fresh process as well.

The argument checks (size limit, host pointers, non-finite spacing or
maximum length) return before any kernel is launched and need no GPU.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, protons, random_grid, rel_pos_err

MEMBERS = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time",
           "current_step", "next_step", "active", "flags")
EXACT_IN_MIXED = ("trajectory_length", "time", "current_step", "next_step", "active", "flags")

# (reflective, clip_volume, origin): the origin puts the start region inside
# the grid for the clipVolume case, so candidates cross its faces
GRID_CASES = {
    "periodic": (False, False, (3 * U.kpc, -2 * U.kpc, 0.0)),
    "reflective": (True, False, (3 * U.kpc, -2 * U.kpc, 0.0)),
    "clip_volume": (False, True, (-80 * U.kpc, -80 * U.kpc, -80 * U.kpc)),
}


def _noalloc_desc(grid_ptr, shape, origin, spacing, step, max_length, precision,
                  reflective=False, clip_volume=False):
    d = _abi.NoAllocGridBpDesc()
    d.grid_values = grid_ptr
    d.nx, d.ny, d.nz = shape
    d.origin[:] = origin
    d.spacing[:] = (spacing,) * 3
    d.step = step
    d.max_length = max_length
    d.precision = precision
    d.reflective = int(reflective)
    d.clip_volume = int(clip_volume)
    return d


@pytest.mark.gpu
@pytest.mark.parametrize("grid_case", list(GRID_CASES))
@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED],
                         ids=["fp64", "mixed"])
def test_noalloc_matches_plan_run_on_two_calls(precision, grid_case):
    import torch
    from crpropa3_b200.engine import Plan

    lib = _abi.load()
    reflective, clip, origin = GRID_CASES[grid_case]
    rng = np.random.default_rng(77)
    grid = random_grid(rng, 16)
    d_grid = torch.from_numpy(grid).cuda()
    spacing, step, length = 10 * U.kpc, 1 * U.kpc, 700 * U.kpc
    for call in range(2):
        cands = protons(rng, 3000 + 1000 * call)
        spec = P.ChainSpec([P.GridField(grid, origin, (spacing,) * 3, reflective=reflective,
                                        clip_volume=clip)],
                           [bp_fixed(step), P.MaxTrajectoryLength(length)], precision=precision)
        expected = cands.to_device("cuda")
        Plan(spec).run(expected)

        got = cands.to_device("cuda")
        desc = _noalloc_desc(d_grid.data_ptr(), grid.shape[:3], origin, spacing, step, length,
                             precision, reflective, clip)
        stats = _abi.RunStats()
        s = got.struct()
        _abi.check(lib.crp_run_device_noalloc(C.byref(desc), C.byref(s), cands.n, None,
                                              C.byref(stats)))
        torch.cuda.synchronize()
        a, b = expected.to_host(), got.to_host()
        if precision == _abi.PRECISION_FP64:
            for name in MEMBERS:
                np.testing.assert_array_equal(getattr(b, name), getattr(a, name),
                                              err_msg=f"call {call}: {name}")
        else:
            for name in EXACT_IN_MIXED:
                np.testing.assert_array_equal(getattr(b, name), getattr(a, name),
                                              err_msg=f"call {call}: {name}")
            err = rel_pos_err(b, a)
            assert err.max() <= 1e-6, (call, err.max())
        assert stats.particle_steps > 0
        assert stats.active_left == 0


def _desc_ok():
    desc = _abi.NoAllocGridBpDesc()
    desc.grid_values = 1  # never read by the checks below
    desc.nx = desc.ny = desc.nz = 4
    desc.spacing[:] = (1.0, 1.0, 1.0)
    desc.step = 1.0
    desc.max_length = 10.0
    desc.precision = _abi.PRECISION_FP64
    return desc


def test_noalloc_rejects_more_candidates_than_its_scratch_holds():
    lib = _abi.load()
    s = _abi.Candidates()
    st = lib.crp_run_device_noalloc(C.byref(_desc_ok()), C.byref(s),
                                    _abi.NOALLOC_MAX_CANDIDATES + 1, None, None)
    assert st == _abi.ERR_CAPACITY
    assert "exceed" in _abi.last_error()


@pytest.mark.parametrize("field,value", [("spacing", 0.0), ("spacing", float("nan")),
                                         ("max_length", float("inf")),
                                         ("max_length", float("nan")), ("step", float("inf"))])
def test_noalloc_rejects_non_finite_or_empty_geometry(field, value):
    lib = _abi.load()
    desc = _desc_ok()
    if field == "spacing":
        desc.spacing[1] = value
    else:
        setattr(desc, field, value)
    s = _abi.Candidates()
    st = lib.crp_run_device_noalloc(C.byref(desc), C.byref(s), 4, None, None)
    assert st == _abi.ERR_INVALID_ARGUMENT, _abi.last_error()


def test_noalloc_rejects_host_arrays():
    """Host (pageable) arrays are refused with an error, never handed to a kernel."""
    lib = _abi.load()
    rng = np.random.default_rng(5)
    cands = protons(rng, 8)
    grid = random_grid(rng, 4)
    desc = _desc_ok()
    desc.grid_values = grid.ctypes.data
    s = cands.struct()
    st = lib.crp_run_device_noalloc(C.byref(desc), C.byref(s), cands.n, None, None)
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert "candidate array" in _abi.last_error() or "CUDA" in _abi.last_error()
