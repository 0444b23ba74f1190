"""Cell ordering of grid runs (the chunked scheduler orders the still-active
candidates by grid cell between launches once a run has at least 2^16 of
them): a scheduling choice only.  Each candidate's trajectory depends on its
own state alone, so the ordered run must equal the unordered one (an
explicit launch length turns the ordering off) bit for bit, state and
detection records, in both precision forms and for periodic power-of-two,
periodic and reflective grids."""
import numpy as np
import pytest

from helpers import P, RecordArrays, U, _abi, bp_fixed, ck, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

pytestmark = pytest.mark.gpu

N = 1 << 17
STATE = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time", "current_step",
         "next_step", "active", "flags", "step_count")


def _cands(seed=81):
    from crpropa3_b200.workloads import charge_of
    rng = np.random.default_rng(seed)
    c = CandidateArrays(N)
    c.id[:] = 1000010010
    c.charge[:] = charge_of(1000010010)
    c.energy[:] = np.exp(rng.uniform(np.log(1), np.log(100), N)) * U.EeV
    c.set_position(rng.uniform(-100, 100, (N, 3)) * U.kpc)
    c.set_direction(stable_unit_vectors(rng, N))
    c.next_step[:] = 1e30
    return c


CASES = {
    "periodic_pow2_bp": (32, False, lambda: bp_fixed(1 * U.kpc)),
    "periodic_24_bp": (24, False, lambda: bp_fixed(1 * U.kpc)),
    "reflective_ck": (32, True, lambda: ck(1e-4, 0.1 * U.kpc, 1 * U.kpc)),
}


def _spec(case, precision):
    n, reflective, prop = CASES[case]
    grid = random_grid(np.random.default_rng(82), n, brms=1e-12)
    gf = P.GridField(grid, (-80 * U.kpc,) * 3, (10 * U.kpc,) * 3, reflective=reflective)
    return P.ChainSpec([gf], [prop(), P.MaxTrajectoryLength(1.5 * U.Mpc, record=True),
                              P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 600 * U.kpc, True, True)],
                       precision=precision)


def _records(r):
    d = r.sorted()
    k = np.lexsort((np.asarray(d["trajectory_length"]), np.asarray(d["module"]), np.asarray(d["index"])))
    return {name: np.asarray(v)[k] for name, v in d.items()}


@pytest.mark.parametrize("precision", [_abi.PRECISION_MIXED, _abi.PRECISION_FP64])
@pytest.mark.parametrize("case", sorted(CASES))
def test_cell_ordered_run_equals_unordered(case, precision):
    from crpropa3_b200.engine import Plan
    plan = Plan(_spec(case, precision))
    c = _cands()
    a, b = c.to_device("cuda"), c.to_device("cuda")
    ra, rb = RecordArrays(2 * N, device="cuda"), RecordArrays(2 * N, device="cuda")
    sa = plan.run(a, records=ra, mode=_abi.MODE_CHUNKED)                          # ordered, 512-step launches
    sb = plan.run(b, records=rb, mode=_abi.MODE_CHUNKED, steps_per_launch=4096)  # unordered
    assert sa.particle_steps == sb.particle_steps > 0
    assert sa.launches > sb.launches  # the ordered run took more (shorter) launches and key kernels
    ha, hb = a.to_host(), b.to_host()
    for m in STATE:
        np.testing.assert_array_equal(getattr(ha, m), getattr(hb, m), err_msg=m)
    ga, gb = _records(ra.to_host()), _records(rb.to_host())
    assert len(ga["index"]) > 1000
    for k in ga:
        np.testing.assert_array_equal(ga[k], gb[k], err_msg=k)


@pytest.mark.parametrize("precision", [_abi.PRECISION_MIXED, _abi.PRECISION_FP64])
def test_host_run_with_chunked_inputs_equals_device_run(precision):
    """crp_run on host arrays of at least 2^18 candidates copies the inputs
    in chunks and starts the first launch on each chunk as it arrives (one
    stream per chunk): the same candidates, states and records as the device
    run, bit for bit; a count that does not split evenly included."""
    from crpropa3_b200.engine import Plan
    plan = Plan(_spec("periodic_pow2_bp", precision))
    n = (1 << 18) + 5
    rng = np.random.default_rng(83)
    c = CandidateArrays(n)
    from crpropa3_b200.workloads import charge_of
    c.id[:] = 1000010010
    c.charge[:] = charge_of(1000010010)
    c.energy[:] = np.exp(rng.uniform(np.log(1), np.log(100), n)) * U.EeV
    c.set_position(rng.uniform(-100, 100, (n, 3)) * U.kpc)
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    h, d = c.copy(), c.to_device("cuda")
    rh, rd = RecordArrays(2 * n), RecordArrays(2 * n, device="cuda")
    sh = plan.run(h, records=rh, mode=_abi.MODE_CHUNKED)
    sd = plan.run(d, records=rd, mode=_abi.MODE_CHUNKED)
    assert sh.particle_steps == sd.particle_steps > 0
    hd = d.to_host()
    for m in STATE:
        if getattr(h, m) is not None:
            np.testing.assert_array_equal(getattr(h, m), getattr(hd, m), err_msg=m)
    gh, gd = _records(rh), _records(rd.to_host())
    assert len(gh["index"]) > 1000
    for k in gh:
        np.testing.assert_array_equal(gh[k], gd[k], err_msg=k)
