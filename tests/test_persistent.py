"""Persistent batched stepping and its autotuner, on the GPU.

Each candidate's trajectory depends only on its own state, so every launch
shape -- chunked, persistent with any CTAs per SM, refill threshold and
burst, launches cut short by the time budget with their work carried over
to the next launch -- must give bit-identical results."""
import numpy as np
import pytest

from helpers import P, RecordArrays, U, _abi, ck, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step",
         "next_step", "active", "flags", "step_count")


def _nuclei(n, seed):
    """Uneven work: H/He/N/Fe, E^-2 over 0.1-100 EeV, lengths 0.2-2 Mpc."""
    from crpropa3_b200.workloads import IDS, charge_of
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n, per_candidate_length=True)
    ids = np.array([IDS[k] for k in ("H", "He", "N", "Fe")], np.int32)
    c.id[:] = ids[rng.integers(0, 4, n)]
    c.charge[:] = [charge_of(int(i)) for i in c.id]
    u = rng.uniform(0, 1, n)
    emin, emax = 0.1 * U.EeV, 100 * U.EeV
    c.energy[:] = 1 / (1 / emin - u * (1 / emin - 1 / emax))
    c.set_direction(stable_unit_vectors(rng, n))
    c.max_length[:] = rng.uniform(0.2, 2, n) * U.Mpc
    return c


def _spec(grid, precision):
    return P.ChainSpec([P.GridField(grid, (0, 0, 0), (5 * U.kpc,) * 3)],
                       [ck(1e-4, 0.1 * U.kpc, 100 * U.kpc), P.MaxTrajectoryLength(per_candidate=True),
                        P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 0.5 * U.Mpc, True, True)],
                       precision=precision)


def _run(spec, c, **kw):
    from crpropa3_b200.engine import Plan
    d = c.to_device("cuda")
    plan = Plan(spec)
    st = plan.run(d, **kw)
    out = d.to_host()
    return out, st


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_persistent_equals_chunked(precision):
    grid = random_grid(np.random.default_rng(60), 32, brms=1e-12)
    c = _nuclei(6000, 61)
    spec = _spec(grid, precision)
    ref, st0 = _run(spec, c, mode=_abi.MODE_CHUNKED, steps_per_launch=64)
    assert st0.launches > 1
    for kw in (dict(ctas_per_sm=1, refill_threshold=1, steps_per_launch=4),
               dict(ctas_per_sm=3, refill_threshold=16, steps_per_launch=32),
               dict(ctas_per_sm=2, refill_threshold=32, steps_per_launch=8, budget_us=300)):
        got, st = _run(spec, c, mode=_abi.MODE_PERSISTENT, **kw)
        for m in STATE:
            np.testing.assert_array_equal(getattr(got, m), getattr(ref, m), err_msg=f"{kw} {m}")
        assert st.particle_steps == st0.particle_steps
        assert st.active_left == 0
    assert st.launches > 1  # the 300 us budget cut the launches


def test_persistent_records_and_step_cap():
    from crpropa3_b200.engine import Plan
    grid = random_grid(np.random.default_rng(62), 16, brms=1e-12)
    c = _nuclei(3000, 63)
    spec = _spec(grid, _abi.PRECISION_FP64)
    a, b = c.to_device("cuda"), c.to_device("cuda")
    ra, rb = RecordArrays(c.n, device="cuda"), RecordArrays(c.n, device="cuda")
    Plan(spec).run(a, mode=_abi.MODE_CHUNKED, records=ra, max_steps=40)
    Plan(spec).run(b, mode=_abi.MODE_PERSISTENT, records=rb, max_steps=40, budget_us=200)
    ha, hb = a.to_host(), b.to_host()
    ra, rb = ra.to_host(), rb.to_host()
    assert ha.step_count.max() <= 40
    for m in STATE:
        np.testing.assert_array_equal(getattr(hb, m), getattr(ha, m), err_msg=m)
    assert ra.n() == rb.n()
    for k, v in ra.sorted().items():
        np.testing.assert_array_equal(rb.sorted()[k], v, err_msg=k)


def test_device_run_rejects_host_arrays():
    """Host (numpy) arrays handed to crp_run_device are refused with a status,
    not dereferenced on the device."""
    from crpropa3_b200.engine import Plan
    grid = random_grid(np.random.default_rng(66), 8)
    spec = _spec(grid, _abi.PRECISION_FP64)
    c = _nuclei(64, 67)
    d = c.to_device("cuda")
    with pytest.raises(_abi.CrpError) as e:
        Plan(spec).run(d, records=RecordArrays(64))  # host records with device candidates
    assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    import ctypes as C
    lib = _abi.load()
    plan = Plan(spec)
    s = c.struct()  # host candidates through the device entry point
    st = lib.crp_run_device(plan.handle, C.byref(s), c.n, None, None)
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert "host memory" in _abi.last_error()


def test_autotune_then_auto_run():
    from crpropa3_b200.engine import Plan
    grid = random_grid(np.random.default_rng(64), 32, brms=1e-12)
    c = _nuclei(20000, 65)
    spec = _spec(grid, _abi.PRECISION_MIXED)
    plan = Plan(spec)
    d = c.to_device("cuda")
    res = plan.autotune(d, sample_n=8192, steps_per_candidate=64)
    assert res.trials > 10 and res.steps_per_second > 0
    assert res.steps_per_second >= res.chunked_steps_per_second
    np.testing.assert_array_equal(d.to_host().x, c.x)  # the sample was copied, not stepped
    st = plan.run(d)  # MODE_AUTO: the tuned configuration
    ref, _ = _run(spec, c, mode=_abi.MODE_CHUNKED)
    got = d.to_host()
    for m in STATE:
        np.testing.assert_array_equal(getattr(got, m), getattr(ref, m), err_msg=m)


def test_persistent_graph_rounds_and_cancel():
    """Persistent launches run as captured CUDA graphs of several rounds
    (launch, carry-over, queue advance); the host flag is polled between
    graphs: a raised flag ends the run with CRP_ERR_CANCELLED and the
    candidates still to do are reported."""
    import ctypes as C
    from crpropa3_b200.engine import Plan
    grid = random_grid(np.random.default_rng(68), 32, brms=1e-12)
    c = _nuclei(20000, 69)
    spec = _spec(grid, _abi.PRECISION_MIXED)
    # many short rounds: a 50 us budget cuts every launch
    got, st = _run(spec, c, mode=_abi.MODE_PERSISTENT, budget_us=50, ctas_per_sm=1)
    ref, st0 = _run(spec, c, mode=_abi.MODE_CHUNKED)
    for m in STATE:
        np.testing.assert_array_equal(getattr(got, m), getattr(ref, m), err_msg=m)
    assert st.launches > 8  # more than one graph of rounds
    flag = C.c_int32(1)
    plan = Plan(spec)
    d = c.to_device("cuda")
    with pytest.raises(_abi.CrpError) as e:
        plan.run(d, mode=_abi.MODE_PERSISTENT, budget_us=50, ctas_per_sm=1, cancel=C.pointer(flag))
    assert e.value.status == _abi.ERR_CANCELLED
