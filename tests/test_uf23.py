"""UF23Field (UF23Field.cpp:59-558): the eight coherent galactic field models
of Unger & Farrar 2023 -- spiral or spur disk field, toroidal + poloidal
(sigmoid or exponential) or twisted halo.

CPU: crp_uf23_defaults against the reference's constructor for every model,
through the field; the oracle's field and stepping against the reference's
own UF23Field, bit for bit.  GPU: the device evaluates in FP64 with CUDA's
exp, log, sin, cos, acos and atan2 (within two ulp of glibc's) and a
correctly rounded pow, so it is compared with the oracle within 1e-12 of
the largest field value and, for fixed-step Boris trajectories, within 1e-9
relative final position; the mixed form evaluates the field in FP32 in the
model's units (kpc, microgauss): within 1e-5 of the largest field value,
fixed-step Boris trajectories within 1e-5 median relative final position.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC = U.kpc
MODELS = {"base": _abi.UF23_BASE, "neCL": _abi.UF23_NECL, "expX": _abi.UF23_EXPX, "spur": _abi.UF23_SPUR,
          "cre10": _abi.UF23_CRE10, "synCG": _abi.UF23_SYNCG, "twistX": _abi.UF23_TWISTX,
          "nebCor": _abi.UF23_NEBCOR}


def _spec(model, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([P.UF23Field(MODELS[model])], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=4000, seed=51):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-32, 32, (n, 3)) * KPC
    k = n // 8
    pos[:k, 2] = 0.0                                       # galactic plane
    pos[k:2 * k, :2] = 0.0                                 # the axis r = 0
    pos[2 * k:3 * k] *= 0.02                               # inner kpc
    r = rng.uniform(7, 9.5, k) * KPC                       # near the spur's reference radius
    a = rng.uniform(-np.pi, np.pi, k)
    pos[3 * k:4 * k, 0], pos[3 * k:4 * k, 1] = r * np.cos(a), r * np.sin(a)
    pos[4 * k] = 0.0
    return pos


@pytest.mark.parametrize("model", sorted(MODELS))
def test_field_oracle_matches_reference(oracle, reference, model):
    spec = _spec(model)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 1e-10
    far = np.linalg.norm(pos, axis=1) > 30 * KPC
    assert far.any() and not np.abs(a[far]).any()          # B = 0 beyond 30 kpc


def test_defaults():
    base = P.UF23Field.defaults(_abi.UF23_BASE)
    # "1 * Gpc" in the constructor resolves to crpropa::Gpc, in metres (Units.h:116)
    assert base.model == 0 and base.poloidal_a == U.Gpc and base.max_radius_squared == 900.0
    assert base.disk_pitch == 1.0106900e+01 * (np.pi / 180.)
    expx = P.UF23Field.defaults(_abi.UF23_EXPX)
    assert expx.poloidal_a == 6.1938701e+00 and expx.poloidal_z == expx.poloidal_a * np.tan(expx.poloidal_xi)
    assert P.UF23Field.defaults(_abi.UF23_TWISTX).twisting_time == 5.4733549e+01
    assert P.UF23Field.defaults(_abi.UF23_SPUR).spur_width == 1.0318114e+01 * (np.pi / 180.)


def _backtrack_cands(n=160, seed=52):
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = -1000010010
    c.charge[:] = -U.eplus
    c.energy[:] = np.exp(rng.uniform(np.log(5), np.log(100), n)) * U.EeV
    pos = np.tile([-8.2 * KPC, 0.0, 0.0], (n, 1))
    c.set_position(pos)
    c.px[:], c.py[:], c.pz[:] = pos[:, 0], pos[:, 1], pos[:, 2]
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


def _chain(prop):
    return [prop, P.MaxTrajectoryLength(100 * KPC, record=True),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 20 * KPC, True, True)]


STEP_CASES = {"base_ck": ("base", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
              "twistX_bp": ("twistX", lambda: bp_fixed(50 * U.pc)),
              "spur_bp": ("spur", lambda: bp_fixed(50 * U.pc)),
              "expX_ck": ("expX", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc))}
STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step",
         "active", "flags")


def _step_spec(case, precision=_abi.PRECISION_FP64):
    model, prop = STEP_CASES[case]
    return _spec(model, precision, _chain(prop()))


@pytest.mark.parametrize("case", sorted(STEP_CASES))
def test_stepping_oracle_matches_reference(oracle, reference, case):
    spec = _step_spec(case)
    c = _backtrack_cands()
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    oracle.run(spec, b)
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
    assert (a.flags & _abi.FLAG_DETECTED).mean() > 0.9


@pytest.fixture(scope="module")
def plugin():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    return PluginHarness()


@pytest.mark.parametrize("model", ["base", "spur", "twistX", "expX"])
def test_plugin_translates_uf23(plugin, model):
    ok, text = plugin.describe(_spec(model, modules=_chain(bp_fixed(KPC))))
    assert ok, text
    assert f"UF23Field model {MODELS[model]}" in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("model", sorted(MODELS))
def test_device_fp64_field_close_to_oracle(oracle, model):
    from crpropa3_b200.engine import Plan
    spec = _spec(model)
    pos = _positions()
    a = oracle.field(spec, pos)
    d = Plan(spec).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-12 * np.abs(a).max())


@pytest.mark.gpu
@pytest.mark.parametrize("model", sorted(MODELS))
def test_device_mixed_field_close_to_oracle(oracle, model):
    from crpropa3_b200.engine import Plan
    pos = _positions()
    a = oracle.field(_spec(model), pos)
    d = Plan(_spec(model, _abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-5 * np.abs(a).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["twistX_bp", "spur_bp"])
def test_device_mixed_bp_trajectories_close_to_oracle(oracle, case):
    from crpropa3_b200.engine import Plan
    c = _backtrack_cands()
    a = c.copy()
    oracle.run(_step_spec(case), a)
    d = c.to_device("cuda")
    Plan(_step_spec(case, _abi.PRECISION_MIXED)).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-5, np.median(rel)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["twistX_bp", "spur_bp"])
def test_device_fp64_bp_trajectories_close_to_oracle(oracle, case):
    from crpropa3_b200.engine import Plan
    spec = _step_spec(case)
    c = _backtrack_cands()
    a = c.copy()
    oracle.run(spec, a)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    np.testing.assert_array_equal(h.flags, a.flags)
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["base_ck", "expX_ck"])
def test_device_fp64_ck_runs_the_same_chains(oracle, case):
    from crpropa3_b200.engine import Plan
    spec = _step_spec(case)
    c = _backtrack_cands()
    a = c.copy()
    oracle.run(spec, a)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-6, np.median(rel)


@pytest.mark.gpu
def test_plugin_uf23_close_to_reference(plugin, reference):
    spec = _step_spec("spur_bp")
    c = _backtrack_cands(seed=53)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.flags, b.flags)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()
