"""KST24Field (KST24Field.cpp:15-374), the galactic field of Korochkin,
Semikoz & Tinyakov 2024, and CMZField (CMZField.cpp:6-304), the
Galactic-centre field of Guenduez et al.

CPU: crp_kst24_defaults and crp_cmz_defaults against the reference's
constructor and methods, through the field; the oracle's field and stepping
against the reference's own fields, bit for bit: KST24 in both halo layers,
in and around the Local Bubble shell and across the five arms; CMZ with each
of its four parts and all together, at the objects' centres included.
GPU: the device evaluates in FP64 with CUDA's libm (within two ulp of
glibc's): fields within 1e-12 of the largest value (KST24's arms and shell
switch off at a surface, so a point within an ulp of it could differ by the
whole field: none of the seeded points is), fixed-step Boris trajectories
within 1e-9 relative final position; the mixed form evaluates KST24 in FP32
in the model's units (kpc, gauss) and rounds CMZ's FP64 field to FP32: 1e-5
of the largest value, and fixed-step Boris trajectories through KST24 within
1e-5 median relative final position.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

KPC, PC = U.kpc, U.pc

FIELDS = {
    "kst24": lambda: P.KST24Field(),
    "cmz_ic": lambda: P.CMZField(),
    "cmz_mc": lambda: P.CMZField(use_mc=True, use_ic=False),
    "cmz_ntf": lambda: P.CMZField(use_ntf=True, use_ic=False),
    "cmz_radio_arc": lambda: P.CMZField(use_radio_arc=True, use_ic=False),
    "cmz_all": lambda: P.CMZField(use_mc=True, use_ic=True, use_ntf=True, use_radio_arc=True),
}


def _spec(name, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([FIELDS[name]()], modules or [bp_fixed(KPC)], precision=precision)


def _kst24_positions(n=4000, seed=61):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-18, 18, (n, 3))
    k = n // 8
    pos[:k, 2] = rng.uniform(1.0, 2.3, k)                          # northern halo layer and its edges
    pos[k:2 * k, 2] = rng.uniform(-2.7, -1.0, k)                   # southern
    pos[2 * k:3 * k] = [-8.2, 0.095, -0.05] + rng.uniform(-0.3, 0.3, (k, 3))  # Local Bubble and shell
    pos[3 * k:5 * k, 2] = rng.uniform(-1.3, 1.3, 2 * k)            # the arms' layer
    pos[5 * k:5 * k + 4, :2] = 0.0                                  # the axis
    return pos * KPC


def _cmz_positions(n=4000, seed=62):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-200, 200, (n, 3))
    k = n // 8
    pos[:k] = [0.0, -8.3, -6.9] + rng.uniform(-15, 15, (k, 3))     # around Sgr A* and the inner clouds
    pos[k:2 * k] = [0.0, 60.0, 5.0] + rng.uniform(-20, 20, (k, 3))  # the Dust Ridge
    pos[2 * k:3 * k] = [0.0, -40.0, 30.0] + rng.uniform(-60, 60, (k, 3))  # filaments
    mids = np.array([[0, y, z] for y, z in [(-81.59, -16.32), (37.53, -2.37), (97.01, -5.93), (-8.3, -6.9),
                                            (-22.25, 69.73), (26.7, 10.38)]])
    pos[3 * k:3 * k + len(mids)] = mids                             # object centres (r = 0)
    return pos * PC


def _positions(name):
    return _kst24_positions() if name == "kst24" else _cmz_positions()


# ------------------------------------------------------------------ CPU


@pytest.mark.parametrize("name", sorted(FIELDS))
def test_field_oracle_matches_reference(oracle, reference, name):
    spec = _spec(name)
    pos = _positions(name)
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.nanmax(np.abs(a)) > 1e-12


def test_kst24_parameters():
    d = P.KST24Field.desc()
    assert d.north_b == -3.2e-6 and d.south_zmax == -1.22 and d.x_theta_rad == 28.0 * np.pi / 180.
    assert [d.arms[i].phi0_deg for i in range(5)] == [-134.0, -80.0, -2.2, 46.0, 46.0]
    assert abs(np.linalg.norm(np.array(d.lb_dir)) - 1) < 1e-15
    assert d.kpc == KPC and d.gauss == 1e-4


def test_cmz_parameters():
    d = P.CMZField().desc()
    assert (d.use_mc, d.use_ic, d.use_ntf, d.use_radio_arc) == (0, 1, 0, 0)
    assert d.clouds[9].eta == 0.77 and d.clouds[0].eta == 0.01
    assert d.ntf[2].l == 2.72 / 2 * np.log(2)                     # the one a2 given without a unit
    assert d.ntf[6].b == 70.e-6 / 0.48 / 0.48


def _stepping(name):
    rng = np.random.default_rng(63 if name == "kst24" else 64)
    n = 160 if name == "kst24" else 64
    c = CandidateArrays(n)
    if name == "kst24":
        c.id[:] = -1000010010
        c.charge[:] = -U.eplus
        c.energy[:] = np.exp(rng.uniform(np.log(5), np.log(100), n)) * U.EeV
        c.set_position(np.tile([-8.2 * KPC, 0.0, 0.0], (n, 1)))
        chain = [bp_fixed(50 * PC), P.MaxTrajectoryLength(100 * KPC, record=True),
                 P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 20 * KPC, True, True)]
    else:
        c.id[:] = 1000010010
        c.charge[:] = U.eplus
        c.energy[:] = np.exp(rng.uniform(np.log(0.1), np.log(10), n)) * U.EeV
        c.set_position(np.tile([0.0, -8.3 * PC, -6.9 * PC], (n, 1)))
        chain = [ck(1e-4, 1e-2 * PC, 10 * PC), P.MaxTrajectoryLength(2 * KPC, record=True),
                 P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 300 * PC, True, True)]
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return chain, c


STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step",
         "active", "flags")


@pytest.mark.parametrize("name", ["kst24", "cmz_all"])
def test_stepping_oracle_matches_reference(oracle, reference, name):
    chain, c = _stepping(name)
    spec = _spec(name, modules=chain)
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


@pytest.mark.parametrize("name,expect", [("kst24", "KST24Field"),
                                         ("cmz_all", "CMZField MC 1 IC 1 NTF 1 radio arc 1"),
                                         ("cmz_ic", "CMZField MC 0 IC 1 NTF 0 radio arc 0")])
def test_plugin_translates(plugin, name, expect):
    ok, text = plugin.describe(_spec(name))
    assert ok, text
    assert expect in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_fp64_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    spec = _spec(name)
    pos = _positions(name)
    a = oracle.field(spec, pos)
    d = Plan(spec).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-12 * np.nanmax(np.abs(a)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(FIELDS))
def test_device_mixed_field_close_to_oracle(oracle, name):
    from crpropa3_b200.engine import Plan
    pos = _positions(name)
    a = oracle.field(_spec(name), pos)
    d = Plan(_spec(name, _abi.PRECISION_MIXED)).field(pos)
    np.testing.assert_allclose(d, a, rtol=0, atol=1e-5 * np.nanmax(np.abs(a)))


@pytest.mark.gpu
def test_device_mixed_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    chain, c = _stepping("kst24")
    a = c.copy()
    oracle.run(_spec("kst24", modules=chain), a)
    d = c.to_device("cuda")
    Plan(_spec("kst24", _abi.PRECISION_MIXED, modules=chain)).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.98
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel) <= 1e-5, np.median(rel)


@pytest.mark.gpu
def test_device_fp64_bp_trajectories_close_to_oracle(oracle):
    from crpropa3_b200.engine import Plan
    chain, c = _stepping("kst24")
    spec = _spec("kst24", modules=chain)
    a = c.copy()
    oracle.run(spec, a)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    np.testing.assert_array_equal(h.flags, a.flags)
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-9, rel.max()


@pytest.mark.gpu
def test_plugin_cmz_runs_as_the_engine(plugin):
    """The reference's own CMZField (all four parts) translated by
    GpuModuleList runs the same device plan as the engine given the same
    field: bit-identical final states.  (Against ModuleList::run itself the
    runs part: the molecular clouds' mG fields turn 1-10 EeV protons within a
    few steps, and an ulp of field, CUDA's libm against glibc's, grows
    without bound along such paths; the fields themselves are compared with
    the oracle above.)"""
    from crpropa3_b200.engine import Plan
    rng = np.random.default_rng(65)
    n = 256
    c = CandidateArrays(n)
    c.id[:] = 1000010010
    c.charge[:] = U.eplus
    c.energy[:] = np.exp(rng.uniform(np.log(1), np.log(10), n)) * U.EeV
    c.set_position(np.tile([0.0, -8.3 * PC, -6.9 * PC], (n, 1)))
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    chain = [bp_fixed(0.5 * PC), P.MaxTrajectoryLength(1 * KPC, record=True),
             P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 300 * PC, True, True)]
    spec = _spec("cmz_all", modules=chain)
    b = c.copy()
    plugin.run(spec, b)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    for m in STATE:
        np.testing.assert_array_equal(getattr(h, m), getattr(b, m), err_msg=m)
