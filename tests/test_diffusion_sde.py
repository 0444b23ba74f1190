"""DiffusionSDE (DiffusionSDE.cpp:47) on the GPU.

* FP64 form against the oracle, which draws from the same counter-based
  Philox stream: on uniform and toroidal fields the positions agree to the
  last bits over 50 steps (they differ only through CUDA's and glibc's log,
  cos, sin, acos in the normal and cone draws, a few ulp).  With plane-wave
  turbulence the phases reach ~1e3 rad, CUDA's and glibc's cos differ in
  the last bit on some of them, and the step-halving loop turns such a bit
  into a different step size: that case is compared in distribution.
* Statistics against the reference's own run (its MT19937 per-thread
  streams), as the reference tests them (test/testDiffusionSDE.py:239-261):
  positions after 50 kpc in a uniform 1 nG field along z with epsilon = 0
  are normal (Anderson-Darling at the 1e-5 level, critical value 2.274),
  with mean 0 and standard deviation sqrt(2 D L / c); and a two-sample
  Kolmogorov-Smirnov test against the reference's sample.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

pytestmark = pytest.mark.gpu


def _sde_chain(fields, tol=1e-4, min_step=1 * U.pc, max_step=10 * U.kpc, eps=0.0, length=50 * U.kpc,
               precision=_abi.PRECISION_FP64, seed=99, observer=None):
    mods = [P.MaxTrajectoryLength(length),
            P.Propagation(_abi.PROP_SDE, tol, min_step, max_step, epsilon=eps)]
    if observer is not None:
        mods.append(observer)
    return P.ChainSpec(fields, mods, precision=precision, seed=seed)


def _cands(n, energy, pos=(0.0, 0.0, 0.0), rng=None):
    c = CandidateArrays(n)
    c.id[:] = 1000010010
    c.charge[:] = U.eplus
    c.energy[:] = energy
    c.set_position(np.tile(np.asarray(pos, float), (n, 1)))
    c.set_direction(stable_unit_vectors(rng or np.random.default_rng(0), n))
    return c


def _anderson_normal(x):
    from scipy import stats
    return stats.anderson(np.asarray(x)).statistic


@pytest.mark.parametrize("field", ["uniform", "toroidal"])
def test_sde_fp64_follows_oracle_stream(oracle_crpow, field):
    from crpropa3_b200.engine import Plan
    fields = {"uniform": [P.UniformField((0, 3e-10, 1 * U.nG))],
              "toroidal": [P.ToroidalField(1 * U.muG)]}[field]
    spec = _sde_chain(fields, min_step=0.1 * U.pc, max_step=100 * U.pc, eps=0.1, length=50 * U.kpc)
    c = _cands(512, 100 * U.TeV, pos=(500 * U.pc, 0, 0), rng=np.random.default_rng(41))
    a, b = c.copy(), c.copy()
    oracle_crpow.run(spec, a, max_steps=50)
    Plan(spec).run(b, max_steps=50)
    np.testing.assert_array_equal(a.step_count, b.step_count)
    assert np.mean(a.trajectory_length == b.trajectory_length) >= 0.95
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-14, np.median(rel)
    assert np.mean(rel <= 1e-12) >= 0.95


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_sde_uniform_field_statistics(precision, reference):
    from scipy import stats
    from crpropa3_b200.engine import Plan
    E, L, n = 10 * U.TeV, 50 * U.kpc, 10_000
    D = 6.1e24 * (E / (4 * U.GeV)) ** (1.0 / 3.0)
    spec = _sde_chain([P.UniformField((0, 0, 1 * U.nG))], precision=precision)
    c = _cands(n, E, rng=np.random.default_rng(42))
    Plan(spec).run(c)
    # MaximumTrajectoryLength acts before the step, so the last step overshoots L:
    # the spread follows the length actually travelled
    std_exp = np.sqrt(2 * D * c.trajectory_length.mean() / U.c_light)
    assert c.trajectory_length.min() >= L
    z = c.z
    assert _anderson_normal(z) < 2.274
    assert abs(z.mean()) < 4 * std_exp / np.sqrt(n)
    assert abs(z.std() - std_exp) < 4 * std_exp / np.sqrt(2 * n)
    np.testing.assert_array_equal(c.x, 0.0)  # epsilon = 0: no perpendicular motion
    ref = _cands(n, E, rng=np.random.default_rng(43))
    reference.run(spec, ref, threads=0, seed=7)
    assert stats.ks_2samp(z, ref.z).pvalue > 1e-4
    assert stats.ks_2samp(c.trajectory_length, ref.trajectory_length).pvalue > 1e-4


def test_sde_exit_distributions_match_reference(oracle, reference):
    """Toroidal field plus plane-wave turbulence, absorption at a sphere of
    300 pc around the origin, sources at 150 pc: exit time and exit
    position against the reference (two-sample KS).  16 modes and 1000
    reference candidates keep the reference's CPU run to seconds."""
    from scipy import stats
    from crpropa3_b200.engine import Plan
    from crpropa3_b200.state import RecordArrays
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0, 16, 11)
    spectrum = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0)
    fields = [P.ToroidalField(1 * U.muG), P.PlaneWaveField(xi, kappa, k, beta, ak, spectrum=spectrum, seed=11)]
    obs = P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 300 * U.pc, True, True)
    spec = _sde_chain(fields, min_step=0.1 * U.pc, max_step=100 * U.pc, eps=0.1, length=1e4 * U.kpc,
                      observer=obs)
    n, n_ref = 4000, 1000
    rng = np.random.default_rng(44)
    E = np.exp(rng.uniform(np.log(100 * U.TeV), np.log(1 * U.PeV), n))
    c = _cands(n, 1.0, pos=(150 * U.pc, 0, 0), rng=rng)
    c.energy[:] = E
    gpu = c.copy()
    rg = RecordArrays(n)
    Plan(spec).run(gpu, records=rg)
    ref = CandidateArrays(n_ref)
    for name in ref.MEMBERS:
        if getattr(ref, name) is not None:
            getattr(ref, name)[:] = getattr(c, name)[:n_ref]
    rr = RecordArrays(n_ref)
    reference.run(spec, ref, rr, threads=0, seed=3)
    assert rg.n() > 0.9 * n and rr.n() > 0.9 * n_ref
    g, r = rg.sorted(), rr.sorted()
    assert stats.ks_2samp(g["time"], r["time"]).pvalue > 1e-4
    gz = g["z"] / np.sqrt(g["x"] ** 2 + g["y"] ** 2 + g["z"] ** 2)
    rz = r["z"] / np.sqrt(r["x"] ** 2 + r["y"] ** 2 + r["z"] ** 2)
    assert stats.ks_2samp(gz, rz).pvalue > 1e-4


@pytest.mark.parametrize("field", ["plane_wave", "toroidal_plus_waves", "grid"])
def test_sde_mixed_coroutine_kernel_equals_per_lane_kernel(oracle, field):
    """The mixed form's chunked launches run DiffusionSDE as a coroutine
    (converged field passes for all waiting lanes); its persistent launches
    run the per-lane step.  Same arithmetic, so bit-identical results."""
    from helpers import random_grid
    from crpropa3_b200.engine import Plan
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0, 64, 11)
    pw = P.PlaneWaveField(xi, kappa, k, beta, ak, spectrum=(0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0),
                          seed=11)
    fields = {"plane_wave": [pw],
              "toroidal_plus_waves": [P.ToroidalField(1 * U.muG), pw],
              "grid": [P.GridField(random_grid(np.random.default_rng(5), 16, brms=1e-10),
                                   (-8 * U.pc,) * 3, (1 * U.pc,) * 3)]}[field]
    obs = P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 300 * U.pc, True, True)
    spec = _sde_chain(fields, min_step=0.1 * U.pc, max_step=100 * U.pc, eps=0.1, length=2 * U.kpc,
                      precision=_abi.PRECISION_MIXED, observer=obs)
    rng = np.random.default_rng(46)
    c = _cands(3000, 1.0, pos=(150 * U.pc, 0, 0), rng=rng)
    c.energy[:] = np.exp(rng.uniform(np.log(10 * U.TeV), np.log(1 * U.PeV), c.n))
    a, b = c.to_device("cuda"), c.to_device("cuda")
    plan = Plan(spec)
    sa = plan.run(a, mode=_abi.MODE_CHUNKED, steps_per_launch=40)
    sb = plan.run(b, mode=_abi.MODE_PERSISTENT, ctas_per_sm=2, steps_per_launch=8)
    ha, hb = a.to_host(), b.to_host()
    for m in ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "next_step", "active",
              "flags", "step_count"):
        np.testing.assert_array_equal(getattr(ha, m), getattr(hb, m), err_msg=m)
    assert sa.particle_steps == sb.particle_steps and sa.tries == sb.tries
    assert sa.launches > 1
