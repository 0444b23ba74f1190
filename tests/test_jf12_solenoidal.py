"""JF12FieldSolenoidal (JF12FieldSolenoidal.cpp:8-302): JF12Field with a
divergence-free disk (the spiral's flux redirected in transition regions of
width delta at r1 = 5 kpc and r2 = 20 kpc) and an X field with parabolic field
lines below |z| = zs (Kleimann et al. 2018).

CPU: crp_jf12_solenoidal's derived state (arm crossings, the flux-closing
eighth arm, the azimuth integral's coefficients) against the reference's
constructor through the field; the oracle's field and stepping against the
reference's own JF12FieldSolenoidal, bit for bit, in both transitions, at
|z| = zs and on the axis above it; the setters (transition width, scale
height, deactivateOuterTransition).
GPU: the device evaluates in FP64 with CUDA's log, atan, atan2, sin, cos and
exp (within two ulp of glibc's): field within 1e-12 of the largest field
value, fixed-step Boris trajectories within 1e-9 relative final position;
the mixed form evaluates the field in FP32 in kpc and muG, as for JF12Field
(1e-5 of the largest value; trajectories within 1e-5 median relative final
position).
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC = U.kpc
S = _abi.JF12_VARIANT_SOLENOIDAL


def _turbulent_grid(seed=51, n=32):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    return P.GridField(v, (0.0, 0.0, 0.0), (0.25 * KPC,) * 3)


def _striated_grid(seed=52, n=40):
    rng = np.random.default_rng(seed)
    v = (rng.integers(0, 2, (n, n, n)) * 2 - 1).astype(np.float32)
    return P.ScalarGrid(v, (0.0, 0.0, 0.0), (0.1 * KPC,) * 3, reflective=False)


FIELDS = {
    "default": lambda: P.JF12Field(variant=S),
    "narrow": lambda: P.JF12Field(variant=S, delta=1.0 * KPC, zs=0.2 * KPC),
    "no_outer": lambda: P.JF12Field(variant=S, outer_transition=False),
    "disk_only": lambda: P.JF12Field(variant=S, use_toroidal_halo=False, use_x=False),
    "x_only": lambda: P.JF12Field(variant=S, use_disk=False, use_toroidal_halo=False),
    "wide_x": lambda: P.JF12Field(variant=S, delta=5.0 * KPC, zs=2.0 * KPC, use_disk=False),
    "turbulent_striated": lambda: P.JF12Field(variant=S, striated=_striated_grid(), turbulent=_turbulent_grid()),
}


def _spec(name, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([FIELDS[name]()], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=4000, seed=53):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-21, 21, (n, 3)) * KPC
    k = n // 8
    for j, (lo, hi) in enumerate([(5.0, 8.5), (16.0, 20.0)]):   # the two transitions
        r = rng.uniform(lo, hi, k) * KPC
        a = rng.uniform(-np.pi, np.pi, k)
        sl = slice(j * k, (j + 1) * k)
        pos[sl, 0], pos[sl, 1] = r * np.cos(a), r * np.sin(a)
        pos[sl, 2] = rng.uniform(-1, 1, k) * KPC
    pos[2 * k:3 * k, 2] = rng.uniform(-2.5, 2.5, k) * KPC       # both sides of |z| = zs
    pos[3 * k:3 * k + 10, :2] = 0.0                              # the axis, r = 0
    pos[3 * k:3 * k + 5, 2] = np.array([0.6, -0.7, 3.0, -9.0, 0.1]) * KPC
    pos[3 * k + 5:3 * k + 10, 2] *= 0.01
    pos[3 * k + 10:4 * k, 2] = 0.0                               # the plane
    return pos


# ------------------------------------------------------------------ CPU


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_field_oracle_matches_reference(oracle, reference, name):
    spec = _spec(name)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 1e-10


def test_derived_state():
    d = P.JF12Field(variant=S).parameters()
    assert d.variant == S and d.delta == 3 * KPC and d.z_s == 0.5 * KPC
    assert d.r1 == 5 * KPC and d.r2 == 20 * KPC and d.r1s == d.r1 + 3 * KPC and d.r2s == d.r2 - 3 * KPC
    arms = np.array(d.phi0_arms)
    assert np.all(np.diff(arms[:10]) < 0)                        # clockwise, periodically closed
    assert arms[0] == arms[8] + 2 * np.pi and arms[9] == arms[1] - 2 * np.pi
    b = np.array(d.b_arms)
    assert b[0] == b[8] and b[9] == b[1] and b[10] == b[2]
    flux = sum((arms[i - 1] - arms[i]) * b[i] for i in range(1, 9))
    assert abs(flux) <= 1e-12 * np.abs(b).max() * 2 * np.pi      # the eighth arm closes the flux
    assert P.JF12Field(variant=S, outer_transition=False).parameters().r2s == 20 * KPC
    with pytest.raises(ValueError):
        P.JF12Field(delta=KPC).parameters()


@pytest.mark.parametrize("delta,zs", [(0.0, 0.5), (2.0, 0.0), (7.0, 1.0)])
def test_setters_through_the_field(oracle, reference, delta, zs):
    f = P.JF12Field(variant=S, delta=delta * KPC, zs=zs * KPC)
    spec = P.ChainSpec([f], [bp_fixed(KPC)])
    pos = _positions(1000, seed=54)
    np.testing.assert_array_equal(oracle.field(spec, pos), reference.field(spec, pos))


def _backtrack_cands(n=160, seed=55):
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


STEP_CASES = {"default_ck": ("default", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
              "default_bp": ("default", lambda: bp_fixed(50 * U.pc)),
              "narrow_bp": ("narrow", lambda: bp_fixed(50 * U.pc))}
STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step",
         "active", "flags")


def _step_spec(case, precision=_abi.PRECISION_FP64):
    field, prop = STEP_CASES[case]
    return _spec(field, precision, _chain(prop()))


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


@pytest.mark.parametrize("name", ["default", "no_outer", "turbulent_striated"])
def test_plugin_translates_solenoidal(plugin, name):
    ok, text = plugin.describe(_spec(name, modules=_chain(bp_fixed(KPC))))
    assert ok, text
    assert "JF12FieldSolenoidal regular 1" in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_fp64_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    spec = _spec(name)
    pos = _positions()
    a = oracle.field(spec, pos)
    d = Plan(spec).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-12 * np.nanmax(np.abs(a)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_mixed_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    pos = _positions()
    a = oracle.field(_spec(name), pos)
    d = Plan(_spec(name, _abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-5 * np.nanmax(np.abs(a)))


@pytest.mark.gpu
def test_device_mixed_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    c = _backtrack_cands()
    a = c.copy()
    oracle.run(_step_spec("default_bp"), a)
    d = c.to_device("cuda")
    Plan(_step_spec("default_bp", _abi.PRECISION_MIXED)).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-5, np.median(rel)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["default_bp", "narrow_bp"])
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
def test_plugin_solenoidal_close_to_reference(plugin, reference):
    spec = _step_spec("default_bp")
    c = _backtrack_cands(seed=56)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.flags, b.flags)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()
