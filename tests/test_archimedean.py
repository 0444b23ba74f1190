"""ArchimedeanSpiralField (ArchimedeanSpiralField.cpp:5-46): a radial field
B_0 (R_0 / r)^2 wound into an Archimedean spiral by the rotation (Omega r
sin(theta) / V_w), reversed below z = 0 -- a stellar-wind (Parker) field.

CPU: the oracle's field and stepping against the reference's own
ArchimedeanSpiralField, bit for bit (the origin, where the reference divides
by zero, and the z axis included).  GPU: the device evaluates in FP64 with
CUDA's atan2, sin and cos (within two ulp of glibc's): within 1e-12 of the
largest field value of the oracle's and, for fixed-step Boris trajectories,
within 1e-9 relative final position for 95 % of them (median 1e-12: orbits
near the origin amplify ulp-level differences); the mixed form rounds the FP64 field to
FP32 (bound 1e-6 of the largest field value).
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

AU = U.au
# a solar-wind-like field: 1 nT at 1 au, the Sun's rotation, 400 km/s wind
FIELD = P.ArchimedeanSpiralField(b0=1e-9, r0=AU, omega=2.7e-6, vw=4e5)


def _spec(precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([FIELD], modules or [bp_fixed(0.01 * AU)], precision=precision)


def _positions(n=4000, seed=71, singular=True):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-20, 20, (n, 3)) * AU
    k = n // 8
    pos[:k, 2] = 0.0                                       # z = 0 (not reversed)
    pos[k:2 * k, :2] = 0.0                                 # the z axis: phi = 0
    pos[2 * k:3 * k] *= 1e-3                               # near the origin
    if singular:
        pos[3 * k] = 0.0                                   # the origin: 0 / 0 as in the reference
    return pos


def test_field_oracle_matches_reference(oracle, reference):
    spec = _spec()
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    fin = np.isfinite(a)
    assert not fin.all() and np.abs(a[fin]).max() > 1e-12
    below = pos[:, 2] < 0
    assert below.any() and (~below).any()


def _cands(n=160, seed=72):
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = 1000010010
    c.charge[:] = U.eplus
    c.energy[:] = np.exp(rng.uniform(np.log(10), np.log(1000), n)) * U.GeV
    pos = rng.uniform(-5, 5, (n, 3)) * AU
    c.set_position(pos)
    c.px[:], c.py[:], c.pz[:] = pos[:, 0], pos[:, 1], pos[:, 2]
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


def _chain(prop):
    return [prop, P.MaxTrajectoryLength(50 * AU, record=True),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 30 * AU, True, True)]


STEP_CASES = {"bp": lambda: bp_fixed(0.01 * AU), "ck": lambda: ck(1e-4, 1e-4 * AU, 0.1 * AU)}
STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step",
         "active", "flags")


@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_stepping_oracle_matches_reference(oracle, reference, case):
    spec = _spec(modules=_chain(STEP_CASES[case]()))
    c = _cands()
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    oracle.run(spec, b)
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
    assert (a.flags & _abi.FLAG_DETECTED).any()


@pytest.fixture(scope="module")
def plugin():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    return PluginHarness()


def test_plugin_translates_archimedean(plugin):
    ok, text = plugin.describe(_spec(modules=_chain(bp_fixed(0.01 * AU))))
    assert ok, text
    assert "ArchimedeanSpiralField" in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
def test_device_fp64_field_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    pos = _positions()
    a = oracle.field(_spec(), pos)
    d = Plan(_spec()).field(pos)
    fin = np.isfinite(a)                                   # the origin: inf and NaN, as the reference
    assert not fin.all()
    np.testing.assert_array_equal(np.isfinite(d), fin)
    np.testing.assert_array_equal(d[~fin], a[~fin])
    np.testing.assert_allclose(d[fin], a[fin], rtol=0, atol=1e-12 * np.abs(a[fin]).max())


@pytest.mark.gpu
def test_device_mixed_field_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    pos = _positions(singular=False)
    a = oracle.field(_spec(), pos)
    d = Plan(_spec(_abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-6 * np.abs(a).max())


@pytest.mark.gpu
def test_device_fp64_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    spec = _spec(modules=_chain(STEP_CASES["bp"]()))
    c = _cands()
    a = c.copy()
    oracle.run(spec, a)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    # orbits that pass close to the origin (B ~ 1 / r^2) amplify ulp-level field differences
    assert np.median(rel) <= 1e-12 and np.mean(rel <= 1e-9) >= 0.95, (np.median(rel), rel.max())
