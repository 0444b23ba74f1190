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


@pytest.mark.parametrize("field", ["plane_wave", "toroidal_plus_waves", "toroidal_plus_1024_waves",
                                   "six_waves_periodic", "grid"])
def test_sde_mixed_coroutine_kernel_equals_per_lane_kernel(oracle, field):
    """The mixed form's chunked launches run DiffusionSDE as a coroutine
    whose plane-wave sums the block evaluates together (four warps, one
    mode group each; a grid field: converged passes of the waiting lanes);
    its persistent launches run the per-lane step.  Same arithmetic in the
    same order, so bit-identical results.  Six modes make three pairs, so
    one of the four mode groups is empty."""
    from helpers import random_grid
    from crpropa3_b200.engine import Plan
    spectrum = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0)
    nm = {"toroidal_plus_1024_waves": 1024, "six_waves_periodic": 6}.get(field, 64)
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(*spectrum, nm, 11)
    pw = P.PlaneWaveField(xi, kappa, k, beta, ak, spectrum=spectrum, seed=11)
    if field == "six_waves_periodic":
        pw.periodic = ((-100 * U.pc,) * 3, (250 * U.pc,) * 3, True)
    fields = {"plane_wave": [pw],
              "toroidal_plus_waves": [P.ToroidalField(1 * U.muG), pw],
              "toroidal_plus_1024_waves": [P.ToroidalField(1 * U.muG), pw],
              "six_waves_periodic": [P.ToroidalField(1 * U.muG), pw],
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


def _galactic(n, precision, sphere):
    """The DiffusionSDE workload: 1 muG toroidal field plus 1024-mode
    PlaneWaveTurbulence (0.5 muG, 1-100 pc), epsilon 0.1, 0.1-100 pc steps,
    tolerance 1e-4, protons log-uniform 1 TeV - 1 PeV from (8.5 kpc, 0, 0),
    absorbed by an Observer sphere of radius `sphere` around the origin."""
    from crpropa3_b200 import workloads as W
    spec, cands = W.sde_galactic(n=n, precision=precision)
    spec.modules[1].radius = sphere
    spec.modules[1].record = True
    return spec, cands


def _exit_records(plan_or_ref, spec, cands, n_rec, **kw):
    from crpropa3_b200.engine import Plan
    from crpropa3_b200.state import RecordArrays
    r = RecordArrays(n_rec)
    if isinstance(plan_or_ref, Plan):
        plan_or_ref.run(cands, records=r)
    else:  # the reference
        plan_or_ref.run(spec, cands, r, **kw)
    return r.sorted()


def _exit_stats(r):
    pos = np.stack([r["x"], r["y"], r["z"]], axis=1)
    return r["time"], pos[:, 2] / np.linalg.norm(pos, axis=1)


def test_sde_galactic_exits_match_reference_at_1kpc(reference):
    """The DiffusionSDE workload's field (1024 modes), diffusion and energies
    with the absorbing sphere at 1 kpc and the sources at 0.5 kpc: exit time
    and exit direction, device (mixed form, every candidate run to
    absorption) against the reference's ModuleList::run, two-sample KS.  The
    stated 20 kpc sphere takes the reference's CPU path about 20 core-minutes
    per 100 candidates (~1e5 steps of 12-70 field evaluations each), beyond a
    test; the device runs it in the bench (sde_galactic_full)."""
    from scipy import stats
    from crpropa3_b200.engine import Plan
    from crpropa3_b200.state import RecordArrays
    from oracle import reference_available, run_reference_isolated
    spec, cands = _galactic(8192, _abi.PRECISION_MIXED, 1 * U.kpc)
    cands.set_position(np.tile([0.5 * U.kpc, 0.0, 0.0], (cands.n, 1)))
    gpu = cands.copy()
    g = _exit_records(Plan(spec), spec, gpu, cands.n)
    assert len(g["time"]) == cands.n and not gpu.active.any()
    spec64, _ = _galactic(1, _abi.PRECISION_FP64, 1 * U.kpc)
    n_ref = 200
    rr = RecordArrays(n_ref)
    run_reference_isolated(spec64, cands.head(n_ref), fast=reference_available(fast=True), seed=3,
                           records=rr)
    r = rr.sorted()
    assert len(r["time"]) == n_ref
    gt, gz = _exit_stats(g)
    rt, rz = _exit_stats(r)
    assert stats.ks_2samp(gt, rt).pvalue > 1e-4
    assert stats.ks_2samp(gz, rz).pvalue > 1e-4
