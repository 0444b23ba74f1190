"""JF12Field and PlanckJF12bField (JF12Field.cpp:8-376): the Jansson-Farrar
2012 galactic field, regular (disk spiral + molecular ring, toroidal halo,
X field), striated (nearest value of a Grid1f) and turbulent (a Grid3f times
the modelled strength).

CPU: the parameters of crp_jf12_defaults against the reference's
constructors, through the field; the oracle's field and stepping against the
reference's own JF12Field, bit for bit; randomStriated against the
reference's.  GPU: the device FP64 form calls CUDA's exp, sin, cos and atan2,
each within two ulp of glibc's, so it is compared with the oracle within
stated bounds (field: 1e-13 of the largest field value; trajectories of the
fixed-step Boris push: 1e-9 relative final position); the mixed form (FP32
field in kpc and muG units) within 1e-5 of the largest field value and 1e-5
median relative final position.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC = U.kpc
J = P.JF12Field


def _turbulent_grid(seed=41, n=32):
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((n, n, n, 3)).astype(np.float32)
    return P.GridField(v, (0.0, 0.0, 0.0), (0.25 * KPC,) * 3)


def _striated_grid(seed=42, n=40):
    rng = np.random.default_rng(seed)
    v = (rng.integers(0, 2, (n, n, n)) * 2 - 1).astype(np.float32)
    return P.ScalarGrid(v, (0.0, 0.0, 0.0), (0.1 * KPC,) * 3, reflective=False)


FIELDS = {
    "jf12": lambda: J(),
    "planck": lambda: J(variant=_abi.JF12_VARIANT_PLANCK),
    "disk_only": lambda: J(use_toroidal_halo=False, use_x=False),
    "halo_only": lambda: J(use_disk=False, use_x=False),
    "x_only": lambda: J(use_disk=False, use_toroidal_halo=False),
    "striated": lambda: J(striated=_striated_grid()),
    "turbulent": lambda: J(turbulent=_turbulent_grid()),
    "planck_turbulent_striated": lambda: J(variant=_abi.JF12_VARIANT_PLANCK, striated=_striated_grid(),
                                           turbulent=_turbulent_grid()),
    "turbulent_only": lambda: J(use_regular=False, turbulent=_turbulent_grid()),
}


def _spec(name, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([FIELDS[name]()], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=4000, seed=43):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-22, 22, (n, 3)) * KPC
    k = n // 8
    pos[:k, 2] = 0.0                                       # galactic plane (X field at z = 0)
    pos[k:2 * k, :2] = 0.0                                 # the axis (azimuth of r = 0)
    r = rng.uniform(3, 5, k) * KPC                         # molecular ring
    a = rng.uniform(-np.pi, np.pi, k)
    pos[2 * k:3 * k, 0], pos[2 * k:3 * k, 1] = r * np.cos(a), r * np.sin(a)
    pos[3 * k:4 * k] *= 0.05                               # inner kpc
    pos[4 * k] = 0.0
    return pos


# ------------------------------------------------------------------ CPU


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_field_oracle_matches_reference(oracle, reference, name):
    spec = _spec(name)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 1e-10                         # microgauss scale


def test_defaults_distinguish_the_variants():
    a, b = J.defaults(_abi.JF12_VARIANT_JF12), J.defaults(_abi.JF12_VARIANT_PLANCK)
    assert a.variant == 0 and b.variant == 1
    assert a.b_x == 4.6 * U.muG and b.b_x == 1.8 * U.muG
    assert a.b_disk[5] == -4.2 * U.muG and b.b_disk[5] == -3.5 * U.muG
    assert a.r_arms[7] == 15.5 * KPC and a.z0 == 5.3 * KPC
    assert a.use_regular and not a.use_striated and not a.use_turbulent


def test_random_striated_matches_reference(reference):
    g = P.jf12_random_striated(12345)
    np.testing.assert_array_equal(g.values, reference.jf12_random_striated(12345))
    assert set(np.unique(g.values)) == {-1.0, 1.0}


def _backtrack_cands(n=200, seed=44):
    """Antiprotons leaving the Earth's position (-8.5 kpc, 0, 0), 5-100 EeV:
    the backtracking set-up of the reference's galactic-lensing examples."""
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


STEP_CASES = {
    "jf12_ck": ("jf12", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
    "jf12_bp": ("jf12", lambda: bp_fixed(50 * U.pc)),
    "planck_turbulent_striated_ck": ("planck_turbulent_striated", lambda: ck(1e-4, 0.1 * U.pc, 100 * U.pc)),
}
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
    assert (a.flags & _abi.FLAG_DETECTED).mean() > 0.9     # nearly all leave the galaxy


@pytest.fixture(scope="module")
def plugin():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    return PluginHarness()


@pytest.mark.parametrize("name,expect", [
    ("jf12", "JF12Field regular 1 disk 1 halo 1 X 1"),
    ("planck_turbulent_striated", "PlanckJF12bField regular 1"),
    ("planck_turbulent_striated", "turbulent Grid3f 32x32x32"),
    ("striated", "striated Grid1f 40x40x40"),
])
def test_plugin_translates_jf12(plugin, name, expect):
    ok, text = plugin.describe(_spec(name, modules=_chain(bp_fixed(U.kpc))))
    assert ok, text
    assert expect in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_fp64_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    spec = _spec(name)
    pos = _positions()
    a = oracle.field(spec, pos)
    d = Plan(spec).field(pos)
    scale = np.abs(a).max()
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-13 * scale)
    # most points agree to the last bit
    assert np.mean(np.all(d == a, axis=1)) > 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_mixed_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    pos = _positions()
    a = oracle.field(_spec(name), pos)
    d = Plan(_spec(name, _abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-5 * np.abs(a).max())


@pytest.mark.gpu
def test_device_fp64_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    spec = _step_spec("jf12_bp")
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
@pytest.mark.parametrize("case", ["jf12_ck", "planck_turbulent_striated_ck"])
def test_device_fp64_ck_runs_the_same_chains(oracle, case):
    """Adaptive Cash-Karp: an ulp of difference in the field can change a
    step-size decision, after which both runs are within the controller's
    tolerance of the true path, not of each other; the same candidates leave
    through the same sphere and the median position difference is small."""
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
def test_device_mixed_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    c = _backtrack_cands()
    a = c.copy()
    oracle.run(_step_spec("jf12_bp"), a)
    d = c.to_device("cuda")
    Plan(_step_spec("jf12_bp", _abi.PRECISION_MIXED)).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-5, np.median(rel)


@pytest.mark.gpu
def test_device_refuses_jf12_without_parameters():
    from crpropa3_b200.engine import Plan
    spec = _spec("jf12")
    d = spec.desc()
    d.fields[0].jf12.kpc = 0.0
    from crpropa3_b200 import _abi as A
    import ctypes as C
    h = C.c_void_p()
    assert A.load().crp_plan_create(C.byref(d), C.byref(h)) == A.ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_plugin_jf12_close_to_reference(plugin, reference):
    """The reference's own JF12Field through GpuModuleList (FP64 form) against
    ModuleList::run: fixed-step Boris push, same bound as the engine."""
    spec = _step_spec("jf12_bp")
    c = _backtrack_cands(seed=45)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.flags, b.flags)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()
