"""The mixed fixed-step Boris kernel that advances two candidates per thread
(over a periodic power-of-two Grid3f) is a schedule, not new arithmetic:
every candidate's trajectory, flags and detection records must equal the
one-candidate kernel's bit for bit.  Covered: the MaximumTrajectoryLength and
the MaximumTrajectoryLength + Observer chain shapes; an odd number of
candidates (the last thread holds one); inactive and neutral candidates;
per-candidate maximum lengths, so that one candidate of a pair ends before
the other and the survivor runs on alone; a per-candidate step cap; cell
ordering between launches (>= 2^16 candidates) and single long launches.
The FP64 form has no pair kernel: the option must not change it."""
import numpy as np
import pytest

from helpers import P, RecordArrays, U, _abi, bp_fixed, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time", "current_step",
         "next_step", "active", "flags", "step_count")


def _cands(n, seed=91, per_candidate=False):
    from crpropa3_b200.workloads import charge_of
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n, per_candidate_length=per_candidate)
    c.id[:] = 1000010010
    c.charge[:] = charge_of(1000010010)
    c.energy[:] = np.exp(rng.uniform(np.log(1), np.log(100), n)) * U.EeV
    c.set_position(rng.uniform(-100, 100, (n, 3)) * U.kpc)
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    c.active[rng.uniform(size=n) < 0.03] = 0
    neutral = rng.uniform(size=n) < 0.02
    c.charge[neutral] = 0.0
    c.id[neutral] = 22
    if per_candidate:
        c.max_length[:] = rng.uniform(0.2, 1.5, n) * U.Mpc
    return c


def _spec(observer, per_candidate, precision=_abi.PRECISION_MIXED):
    grid = random_grid(np.random.default_rng(92), 32, brms=1e-12)
    gf = P.GridField(grid, (-80 * U.kpc,) * 3, (10 * U.kpc,) * 3)
    mods = [bp_fixed(1 * U.kpc),
            P.MaxTrajectoryLength(per_candidate=True, record=True) if per_candidate
            else P.MaxTrajectoryLength(1.2 * U.Mpc, record=True)]
    if observer:
        mods.append(P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 500 * U.kpc, True, True))
    return P.ChainSpec([gf], mods, precision=precision)


def _records(r):
    d = r.sorted()
    k = np.lexsort((np.asarray(d["trajectory_length"]), np.asarray(d["module"]), np.asarray(d["index"])))
    return {name: np.asarray(v)[k] for name, v in d.items()}


def _compare(plan, c, n_rec, **kw):
    a, b = c.to_device("cuda"), c.to_device("cuda")
    ra, rb = RecordArrays(n_rec, device="cuda"), RecordArrays(n_rec, device="cuda")
    sa = plan.run(a, records=ra, mode=_abi.MODE_CHUNKED, candidates_per_thread=1, **kw)
    sb = plan.run(b, records=rb, mode=_abi.MODE_CHUNKED, candidates_per_thread=2, **kw)
    assert sa.particle_steps == sb.particle_steps > 0
    assert sa.tries == sb.tries and sa.field_evaluations == sb.field_evaluations
    ha, hb = a.to_host(), b.to_host()
    for m in STATE:
        np.testing.assert_array_equal(getattr(hb, m), getattr(ha, m), err_msg=m)
    ga, gb = _records(ra.to_host()), _records(rb.to_host())
    assert len(ga["index"]) > 0
    for k in ga:
        np.testing.assert_array_equal(gb[k], ga[k], err_msg=k)
    return sa, sb


@pytest.mark.parametrize("per_candidate", [False, True], ids=["fixed_length", "per_candidate_length"])
@pytest.mark.parametrize("observer", [False, True], ids=["pm", "pmo"])
def test_pair_kernel_equals_single_cell_ordered(observer, per_candidate):
    from crpropa3_b200.engine import Plan
    n = (1 << 17) + 1  # odd: the last thread holds one candidate
    plan = Plan(_spec(observer, per_candidate))
    _compare(plan, _cands(n, per_candidate=per_candidate), 3 * n)


@pytest.mark.parametrize("observer", [False, True], ids=["pm", "pmo"])
def test_pair_kernel_equals_single_small_runs_and_caps(observer):
    from crpropa3_b200.engine import Plan
    plan = Plan(_spec(observer, True))
    for n, kw in ((1, {}), (3, {}), (1001, {}), (4097, {"steps_per_launch": 100}),
                  (5000, {"max_steps": 333})):
        _compare(plan, _cands(n, seed=n, per_candidate=True), 3 * n + 8, **kw)


def test_fp64_form_ignores_candidates_per_thread():
    from crpropa3_b200.engine import Plan
    plan = Plan(_spec(True, False, precision=_abi.PRECISION_FP64))
    _compare(plan, _cands(4099), 3 * 4099)


def test_candidates_per_thread_out_of_range_is_an_error():
    from crpropa3_b200.engine import Plan
    plan = Plan(_spec(False, False))
    c = _cands(64).to_device("cuda")
    with pytest.raises(_abi.CrpError) as e:
        plan.run(c, candidates_per_thread=3)
    assert e.value.status == _abi.ERR_INVALID_ARGUMENT
