"""TF17Field (TF17Field.cpp:10-307): the galactic field of Terral & Ferriere
2017 -- disk model Ad1, Bd1 or Dd1 and halo model C0 or C1.

CPU: crp_tf17_defaults against the reference's constructor, through the
field; the oracle's field and stepping against the reference's own
TF17Field, bit for bit, on the axis r = 0, in the plane z = 0 and inside the
inner radius r1 included.
GPU: the device evaluates in FP64 with CUDA's atan2, sin, cos, exp and log
(within two ulp of glibc's), so it is compared with the oracle within 1e-12
of the largest field value and, for fixed-step Boris trajectories, within
1e-9 median and 1e-6 largest relative final position (the disk models' steep
gradients near the plane grow an ulp of field to a few 1e-8 over 100 kpc of
path); the mixed form evaluates the field in FP32 in kpc and muG (bound
1e-5 of the largest field value, as JF12's mixed form; fixed-step Boris
trajectories within 1e-5 median relative final position).
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC = U.kpc
DISKS = {"Ad1": _abi.TF17_AD1, "Bd1": _abi.TF17_BD1, "Dd1": _abi.TF17_DD1}
HALOS = {"C0": _abi.TF17_C0, "C1": _abi.TF17_C1}
MODELS = {f"{d}_{h}": P.TF17Field(DISKS[d], HALOS[h]) for d in DISKS for h in HALOS}
MODELS["Ad1_C1_disk_only"] = P.TF17Field(use_halo=False)
MODELS["Dd1_C0_halo_only"] = P.TF17Field(_abi.TF17_DD1, _abi.TF17_C0, use_disk=False)


def _spec(model, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([MODELS[model]], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=4000, seed=71, axis=True):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-25, 25, (n, 3)) * KPC
    k = n // 8
    pos[:k, 2] = 0.0                                       # galactic plane
    pos[k:2 * k, 2] = rng.uniform(-0.3, 0.3, k) * KPC       # thin disk
    pos[2 * k:3 * k, :2] *= 0.1                              # inside r1 = 3 kpc
    r = rng.uniform(8, 9, k) * KPC                          # around the Sun's radius
    a = rng.uniform(-np.pi, np.pi, k)
    pos[3 * k:4 * k, 0], pos[3 * k:4 * k, 1] = r * np.cos(a), r * np.sin(a)
    if axis:
        pos[4 * k:4 * k + 4, :2] = 0.0                       # r = 0 (the r <= epsilon branches)
        pos[4 * k + 4, :] = 0.0                              # the origin
    return pos


@pytest.mark.parametrize("model", sorted(MODELS))
def test_field_oracle_matches_reference(oracle, reference, model):
    spec = _spec(model)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.nanmax(np.abs(a)) > 1e-12


def test_defaults():
    d = P.TF17Field().desc()
    assert (d.disk_model, d.halo_model, d.use_disk, d.use_halo) == (_abi.TF17_AD1, _abi.TF17_C1, 1, 1)
    assert d.b1_disk == 32.0 * U.muG and d.h_disk == 0.054 * KPC and d.l_p == 50 * KPC
    assert d.p0 == -9.1 * np.pi / 180 and d.epsilon == np.finfo(float).eps
    assert d.cot_p0 == np.cos(d.p0) / np.sin(d.p0)
    b = P.TF17Field(_abi.TF17_BD1, _abi.TF17_C0).desc()
    assert b.a_disk == 0 and b.phi_star_disk == 153 * np.pi / 180 and b.h_p == 9 * KPC
    with pytest.raises(_abi.CrpError):
        P.TF17Field(3, 0).desc()


def _backtrack_cands(n=160, seed=72):
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = -1000010010
    c.charge[:] = -U.eplus
    c.energy[:] = np.exp(rng.uniform(np.log(5), np.log(100), n)) * U.EeV
    pos = np.tile([-8.5 * KPC, 0.0, 0.0], (n, 1))
    c.set_position(pos)
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


def _chain(prop):
    return [prop, P.MaxTrajectoryLength(100 * KPC, record=True),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 20 * KPC, True, True)]


STEP_CASES = {"Ad1_C1_ck": ("Ad1_C1", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
              "Bd1_C0_bp": ("Bd1_C0", lambda: bp_fixed(50 * U.pc)),
              "Dd1_C1_bp": ("Dd1_C1", lambda: bp_fixed(50 * U.pc))}
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
    assert (a.flags & _abi.FLAG_DETECTED).mean() > 0.5


@pytest.fixture(scope="module")
def plugin():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    return PluginHarness()


@pytest.mark.parametrize("model", ["Ad1_C1", "Dd1_C0_halo_only", "Bd1_C1"])
def test_plugin_translates_tf17(plugin, model):
    ok, text = plugin.describe(_spec(model, modules=_chain(bp_fixed(KPC))))
    assert ok, text
    f = MODELS[model]
    disk = {v: k for k, v in DISKS.items()}[f.disk]
    halo = {v: k for k, v in HALOS.items()}[f.halo]
    assert f"TF17Field disk {disk} halo {halo} use disk {int(f.use_disk)} halo {int(f.use_halo)}" in text, text


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
@pytest.mark.parametrize("case", ["Bd1_C0_bp", "Dd1_C1_bp"])
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
@pytest.mark.parametrize("case", ["Bd1_C0_bp", "Dd1_C1_bp"])
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
    assert np.median(rel) <= 1e-9 and rel.max() <= 1e-6, (np.median(rel), rel.max())


@pytest.mark.gpu
def test_plugin_tf17_close_to_reference(plugin, reference):
    spec = _step_spec("Dd1_C1_bp")
    c = _backtrack_cands(seed=73)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.flags, b.flags)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-9 and rel.max() <= 1e-6, (np.median(rel), rel.max())
