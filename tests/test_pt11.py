"""PT11Field (PT11Field.cpp:8-128): the galactic field of Pshirkov et al.
2011 -- an ASS or BSS logarithmic-spiral disk and an antisymmetric halo.

CPU: crp_pt11_defaults / crp_pt11_use against the reference's constructor
and setters, through the field; the oracle's field and stepping against the
reference's own PT11Field, bit for bit, NaN on the axis r = 0 included.
GPU: the device evaluates in FP64 with CUDA's atan2, cos, log and exp
(within two ulp of glibc's), so it is compared with the oracle within 1e-12
of the largest field value and, for fixed-step Boris trajectories, within
1e-9 relative final position; the mixed form evaluates the field in FP32 in
kpc and muG: within 1e-5 of the largest field value, fixed-step Boris
trajectories within 1e-5 median relative final position.
"""
import math

import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC = U.kpc
MODELS = {"ass_halo": P.PT11Field(), "bss_halo": P.PT11Field(use_ass=False, use_bss=True),
          "ass": P.PT11Field(use_halo=False), "bss": P.PT11Field(False, True, False),
          "halo": P.PT11Field(use_ass=False)}


def _spec(model, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([MODELS[model]], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=4000, seed=61, axis=True):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-25, 25, (n, 3)) * KPC
    k = n // 8
    pos[:k, 2] = 0.0                                       # galactic plane (z > 0 false: southern halo)
    pos[k:2 * k, 2] = rng.uniform(-1.3, 1.3, k) * KPC       # |z| < z0_H
    pos[2 * k:3 * k, :2] *= 0.2                              # r < R_c
    r = rng.uniform(8, 9, k) * KPC                          # around the Sun's radius
    a = rng.uniform(-np.pi, np.pi, k)
    pos[3 * k:4 * k, 0], pos[3 * k:4 * k, 1] = r * np.cos(a), r * np.sin(a)
    if axis:
        pos[4 * k:4 * k + 4, :2] = 0.0                       # r = 0: 0 / 0 as in the reference
    return pos


@pytest.mark.parametrize("model", sorted(MODELS))
def test_field_oracle_matches_reference(oracle, reference, model):
    spec = _spec(model)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.nanmax(np.abs(a)) > 1e-11


def test_defaults_and_switches():
    d = P.PT11Field().desc()
    assert (d.use_ass, d.use_bss, d.use_halo) == (1, 0, 1)
    assert d.pitch == -5.0 * np.pi / 180 and d.b0_hs == 2.0 * U.muG and d.b0_hn == 4.0 * U.muG
    assert d.r_sun == 8.5 * KPC and d.d == -0.6 * KPC
    assert d.phi == d.cos_pitch / d.sin_pitch * math.log1p(d.d / d.r_sun) - math.pi / 2
    b = P.PT11Field(use_ass=False, use_bss=True).desc()
    assert (b.use_ass, b.use_bss) == (0, 1) and b.pitch == -6.0 * np.pi / 180 and b.b0_hs == 4.0 * U.muG
    h = P.PT11Field(use_ass=False).desc()                   # setUseASS(false) changes nothing else
    assert (h.use_ass, h.use_bss, h.use_halo) == (0, 0, 1) and h.pitch == d.pitch and h.b0_hs == d.b0_hs
    with pytest.raises(ValueError):
        P.PT11Field(use_bss=True).desc()


def _backtrack_cands(n=160, seed=62):
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = -1000010010
    c.charge[:] = -U.eplus
    c.energy[:] = np.exp(rng.uniform(np.log(5), np.log(100), n)) * U.EeV
    pos = np.tile([-8.5 * KPC, 0.0, 0.0], (n, 1))
    c.set_position(pos)
    c.px[:], c.py[:], c.pz[:] = pos[:, 0], pos[:, 1], pos[:, 2]
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


def _chain(prop):
    return [prop, P.MaxTrajectoryLength(100 * KPC, record=True),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 20 * KPC, True, True)]


STEP_CASES = {"ass_halo_ck": ("ass_halo", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
              "bss_halo_bp": ("bss_halo", lambda: bp_fixed(50 * U.pc)),
              "ass_halo_bp": ("ass_halo", lambda: bp_fixed(50 * U.pc))}
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


@pytest.mark.parametrize("model", ["ass_halo", "bss", "halo"])
def test_plugin_translates_pt11(plugin, model):
    ok, text = plugin.describe(_spec(model, modules=_chain(bp_fixed(KPC))))
    assert ok, text
    f = MODELS[model]
    assert f"PT11Field ass {int(f.use_ass)} bss {int(f.use_bss)} halo {int(f.use_halo)}" in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("model", sorted(MODELS))
def test_device_fp64_field_close_to_oracle(oracle, model):
    from crpropa3_b200.engine import Plan
    spec = _spec(model)
    pos = _positions()
    a = oracle.field(spec, pos)
    d = Plan(spec).field(pos)
    np.testing.assert_array_equal(np.isnan(d), np.isnan(a))
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-12 * np.nanmax(np.abs(a)))


@pytest.mark.gpu
@pytest.mark.parametrize("model", sorted(MODELS))
def test_device_mixed_field_close_to_oracle(oracle, model):
    from crpropa3_b200.engine import Plan
    pos = _positions(axis=False)
    a = oracle.field(_spec(model), pos)
    d = Plan(_spec(model, _abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-5 * np.abs(a).max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["ass_halo_bp", "bss_halo_bp"])
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
@pytest.mark.parametrize("case", ["ass_halo_bp", "bss_halo_bp"])
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
def test_device_fp64_ck_runs_the_same_chains(oracle):
    from crpropa3_b200.engine import Plan
    spec = _step_spec("ass_halo_ck")
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
def test_plugin_pt11_close_to_reference(plugin, reference):
    spec = _step_spec("bss_halo_bp")
    c = _backtrack_cands(seed=63)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.flags, b.flags)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()
