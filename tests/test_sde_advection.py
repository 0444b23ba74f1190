"""DiffusionSDE with an advection field (DiffusionSDE.cpp:47 with driftStep
:255; the fields of AdvectionField.cpp:12-460): UniformAdvectionField,
ConstantSphericalAdvectionField, SphericalAdvectionField, the
one-dimensional Cartesian and spherical shocks, ObliqueAdvectionShock,
SphericalAdvectionShock, the time-dependent OneDimensionalTimeDependentShock
and SedovTaylorBlastWave (TimeDependentAdvectionField.cpp:7-130; the
candidate's time, or 0 inside a list, as AdvectionFieldList passes none) and
their list.

CPU: the oracle's drift against the reference's own DiffusionSDE, bit for
bit, where the step draws no random number into the position: neutral
candidates (position + drift + straight line) and charged candidates in a
field-free region (the field-line trace is NaN and the step is the drift
alone).  Both exercise every advection kind's getField on the reference's
objects, built by their constructors and setters.
GPU: the FP64 form against the oracle, which follows the same Philox stream,
over 50 steps in a uniform field with each advection kind (positions within
1e-12 relative, as the plain DiffusionSDE tests), the mixed form within
1e-6; and the reference's own test_FullTransport set-up (10 TeV protons,
1 nG along z, 1e6 m/s advection along x, epsilon 0.1, 50 kpc): normal
positions (Anderson-Darling below 2.274) with the means and spreads it
expects, within its four-sigma bounds.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC, PC = U.kpc, U.pc

ADVECTION = {
    "uniform": lambda: [P.UniformAdvectionField((1e6, -2e5, 3e5))],
    "constant_spherical": lambda: [P.ConstantSphericalAdvectionField((1 * KPC, 0, 0), 5e5)],
    "spherical": lambda: [P.SphericalAdvectionField((0, 0, 0), 20 * KPC, 8e5, 3 * KPC, 0.9)],
    "cartesian_shock": lambda: [P.OneDimensionalCartesianShock(4.0, 1e7, 100 * PC)],
    "spherical_shock_1d": lambda: [P.OneDimensionalSphericalShock(2 * KPC, 1e7, 4.0, 50 * PC, True)],
    "spherical_shock_1d_warm": lambda: [P.OneDimensionalSphericalShock(2 * KPC, 1e7, 4.0, 50 * PC, False)],
    "oblique_shock": lambda: [P.ObliqueAdvectionShock(3.5, 8e6, 2e6, 200 * PC)],
    "spherical_shock": lambda: [P.SphericalAdvectionShock((0.5 * KPC, 0, 0), 3 * KPC, 2e6, 0.4 * KPC, 2 * KPC, 1e5)],
    "time_shock": lambda: [P.OneDimensionalTimeDependentShock(1e7, 1e7, 2.5e6, 100 * PC, x_sh0=-1 * KPC,
                                                              t_sh0=1e10)],
    "sedov_taylor": lambda: [P.SedovTaylorBlastWave(1e44, 4e-32, 100 * PC)],
    "list_with_time_shock": lambda: [P.UniformAdvectionField((2e5, 0, 0)),
                                     P.OneDimensionalTimeDependentShock(1e7, 1e7, 2.5e6, 100 * PC, x_sh0=1 * KPC)],
    "list": lambda: [P.UniformAdvectionField((2e5, 0, 0)),
                     P.SphericalAdvectionShock((0, 0, 0), 3 * KPC, 2e6, 0.4 * KPC),
                     P.OneDimensionalCartesianShock(4.0, 1e6, 1 * KPC)],
}


def _spec(fields, adv, eps=0.1, min_step=1 * PC, max_step=100 * PC, length=20 * KPC,
          precision=_abi.PRECISION_FP64, seed=7):
    return P.ChainSpec(fields, [P.MaxTrajectoryLength(length),
                                P.Propagation(_abi.PROP_SDE, 1e-4, min_step, max_step, epsilon=eps,
                                              advection=adv)],
                       precision=precision, seed=seed)


def _cands(n, energy, charge=U.eplus, pid=1000010010, seed=0, spread=3 * KPC):
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = pid
    c.charge[:] = charge
    c.energy[:] = energy
    c.set_position(rng.uniform(-spread, spread, (n, 3)))
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step", "active")


# ------------------------------------------------------------------ CPU


@pytest.mark.parametrize("kind", sorted(ADVECTION))
def test_neutral_drift_matches_reference(oracle, reference, kind):
    spec = _spec([P.UniformField((0, 0, 1 * U.nG))], ADVECTION[kind]())
    c = _cands(200, 1 * U.TeV, charge=0.0, pid=22, seed=11)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    oracle.run(spec, b)
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
    assert np.abs(a.position() - c.position()).max() > 1 * KPC


@pytest.mark.parametrize("kind", sorted(ADVECTION))
def test_field_free_drift_matches_reference(oracle, reference, kind):
    """No magnetic field: the field-line trace is NaN and the step is the
    drift alone (DiffusionSDE.cpp:132-146), for a charged candidate."""
    spec = _spec([P.UniformField((0.0, 0.0, 0.0))], ADVECTION[kind](), length=2 * KPC)
    c = _cands(100, 10 * U.TeV, seed=12)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    oracle.run(spec, b)
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
    assert np.abs(a.position() - c.position()).max() > 0


def test_plugin_translates_advection():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    spec = _spec([P.UniformField((0, 0, 1 * U.nG))], ADVECTION["list"]())
    ok, text = PluginHarness().describe(spec)
    assert ok, text
    assert "DiffusionSDE" in text, text


def test_too_many_advection_fields_refused():
    with pytest.raises(ValueError):
        _spec([P.UniformField((0, 0, 1 * U.nG))], ADVECTION["list"]() + ADVECTION["list"]()).desc()


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("kind", sorted(ADVECTION))
def test_device_fp64_follows_oracle_stream(oracle_crpow, kind):
    from crpropa3_b200.engine import Plan
    spec = _spec([P.UniformField((0, 3e-10, 1 * U.nG))], ADVECTION[kind](), min_step=0.1 * PC)
    c = _cands(512, 100 * U.TeV, seed=13)
    a, b = c.copy(), c.copy()
    oracle_crpow.run(spec, a, max_steps=50)
    Plan(spec).run(b, max_steps=50)
    np.testing.assert_array_equal(a.step_count, b.step_count)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-14, np.median(rel)
    assert np.mean(rel <= 1e-12) >= 0.95


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "spherical_shock", "list"])
def test_device_mixed_close_to_oracle(oracle_crpow, kind):
    from crpropa3_b200.engine import Plan
    spec64 = _spec([P.UniformField((0, 3e-10, 1 * U.nG))], ADVECTION[kind](), min_step=0.1 * PC)
    specmx = _spec([P.UniformField((0, 3e-10, 1 * U.nG))], ADVECTION[kind](), min_step=0.1 * PC,
                   precision=_abi.PRECISION_MIXED)
    c = _cands(512, 100 * U.TeV, seed=14)
    a, b = c.copy(), c.copy()
    oracle_crpow.run(spec64, a, max_steps=20)
    Plan(specmx).run(b, max_steps=20)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-6, np.median(rel)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_full_transport_statistics(precision):
    """The reference's test_FullTransport (test/testDiffusionSDE.py:361)."""
    from scipy import stats
    from crpropa3_b200.engine import Plan
    E, L, n, eps, adv = 10 * U.TeV, 50 * KPC, 10_000, 0.1, 1e6
    D = 6.1e24 * (E / (4 * U.GeV)) ** (1.0 / 3.0)
    spec = _spec([P.UniformField((0, 0, 1 * U.nG))], [P.UniformAdvectionField((adv, 0.0, 0.0))], eps=eps,
                 min_step=1 * PC, max_step=10 * KPC, length=L, precision=precision, seed=3)
    c = _cands(n, E, seed=15, spread=0.0)
    Plan(spec).run(c)
    Lt = c.trajectory_length.mean()  # the last step overshoots L (MaximumTrajectoryLength acts first)
    exp_std = {"x": np.sqrt(2 * eps * D * Lt / U.c_light), "y": np.sqrt(2 * eps * D * Lt / U.c_light),
               "z": np.sqrt(2 * D * Lt / U.c_light)}
    exp_mean = {"x": adv * Lt / U.c_light, "y": 0.0, "z": 0.0}
    for axis in ("x", "y", "z"):
        v = getattr(c, axis)
        assert stats.anderson(v).statistic < 2.274, axis
        s_means = exp_std[axis] / np.sqrt(n)
        s_stds = exp_std[axis] / np.sqrt(n) / np.sqrt(2.)
        assert abs((v.mean() - exp_mean[axis]) / 4. / s_means) < 1., (axis, v.mean(), exp_mean[axis])
        assert abs((v.std() - exp_std[axis]) / 4. / s_stds) < 1., (axis, v.std(), exp_std[axis])
