"""Grid interpolation types and ModulatedMagneticFieldGrid:

* Grid3f tricubic (Grid.h:459, the SIMD form: four-lane float arithmetic
  with the weights rounded to float) and nearest-neighbour (closestValue,
  Grid.h:383), periodic and reflective continuation, with and without
  clipVolume (Grid.h:317-336);
* ModulatedMagneticFieldGrid (MagneticFieldGrid.cpp:51): a Grid3f times a
  Grid1f modulation interpolated trilinear (double products accumulated into
  a float), tricubic (double, Grid.h:498-536) or nearest.

CPU: the oracle's field and stepping against the reference's own Grid and
MagneticFieldGrid objects, bit for bit (the reference built with HAVE_SIMD,
its SIMD_EXTENSIONS option, which the tricubic vector path needs), and the
plugin's translation of such chains.  GPU: the device FP64 form against the
oracle, bit for bit, field and stepping; the mixed form against the oracle
within stated bounds; the plugin against the reference's ModuleList::run.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, protons

KPC = U.kpc
TRI, CUB, NN = (_abi.INTERPOLATION_TRILINEAR, _abi.INTERPOLATION_TRICUBIC,
                _abi.INTERPOLATION_NEAREST_NEIGHBOUR)
INTERP = {"trilinear": TRI, "tricubic": CUB, "nearest": NN}


def _vector_grid(interp, reflective=False, clip=False, n=(16, 12, 10), seed=31):
    rng = np.random.default_rng(seed)
    v = (rng.standard_normal(n + (3,)) * 3e-13).astype(np.float32)
    return P.GridField(v, (-80 * KPC, -60 * KPC, -50 * KPC), (10 * KPC,) * 3, reflective=reflective,
                       clip_volume=clip, interpolation=interp)


def _modulation(interp, reflective=True, clip=False, n=(9, 11, 7), seed=32):
    rng = np.random.default_rng(seed)
    m = rng.uniform(0.2, 2.0, n).astype(np.float32)
    return P.ScalarGrid(m, (-70 * KPC, -75 * KPC, -40 * KPC), (17 * KPC, 13 * KPC, 11 * KPC),
                        reflective=reflective, clip_volume=clip, interpolation=interp)


def _positions(n=3000, seed=33):
    rng = np.random.default_rng(seed)
    # inside, near and well beyond the grids (continuation over several periods)
    pos = rng.uniform(-400, 400, (n, 3)) * KPC
    pos[: n // 3] = rng.uniform(-60, 60, (n // 3, 3)) * KPC
    # grid points and cell faces exactly (ties of the nearest-neighbour round)
    k = rng.integers(-20, 20, (200, 3)).astype(np.float64)
    pos[n // 3: n // 3 + 200] = np.array([-80, -60, -50]) * KPC + (k + 0.5) * 10 * KPC
    pos[n // 3 + 200: n // 3 + 400] = np.array([-80, -60, -50]) * KPC + (k + 1.0) * 10 * KPC
    return pos


VECTOR_CASES = [(i, r, c) for i in ("tricubic", "nearest", "trilinear") for r in (False, True)
                for c in (False, True)]
MOD_CASES = [(gi, mi, mr) for gi in ("trilinear", "tricubic", "nearest")
             for mi in ("trilinear", "tricubic", "nearest") for mr in (True, False)]


def _vector_spec(interp, refl, clip):
    return P.ChainSpec([_vector_grid(INTERP[interp], refl, clip)], [bp_fixed(KPC)])


def _mod_spec(gi, mi, mr, precision=_abi.PRECISION_FP64):
    g = _vector_grid(INTERP[gi])
    return P.ChainSpec([P.ModulatedGridField(g, _modulation(INTERP[mi], reflective=mr))], [bp_fixed(KPC)],
                       precision=precision)


# ------------------------------------------------------------------ CPU


@pytest.mark.parametrize("interp,refl,clip", VECTOR_CASES)
def test_vector_grid_field_oracle_matches_reference(oracle, reference, interp, refl, clip):
    spec = _vector_spec(interp, refl, clip)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 0
    if clip:
        assert (np.abs(a).sum(1) == 0).sum() > 100


@pytest.mark.parametrize("gi,mi,mr", MOD_CASES)
def test_modulated_grid_field_oracle_matches_reference(oracle, reference, gi, mi, mr):
    spec = _mod_spec(gi, mi, mr)
    pos = _positions(seed=34)
    np.testing.assert_array_equal(oracle.field(spec, pos), reference.field(spec, pos))


def test_tricubic_differs_from_trilinear_and_reproduces_grid_points(oracle):
    """Catmull-Rom interpolation passes through the grid values: at a grid
    point the tricubic field is the stored vector, rounded through the float
    lanes; between points it differs from the trilinear field."""
    g = _vector_grid(CUB)
    idx = np.array([[3, 4, 5], [10, 2, 7], [0, 0, 0]])
    pts = np.array(g.origin) + (idx + 0.5) * 10 * KPC
    f = oracle.field(P.ChainSpec([g], [bp_fixed(KPC)]), pts)
    np.testing.assert_allclose(f, g.values[idx[:, 0], idx[:, 1], idx[:, 2]].astype(np.float64),
                               rtol=1e-6, atol=0)
    pos = _positions(1000, seed=35)
    tl = _vector_grid(TRI)
    assert not np.array_equal(oracle.field(P.ChainSpec([g], [bp_fixed(KPC)]), pos),
                              oracle.field(P.ChainSpec([tl], [bp_fixed(KPC)]), pos))


STEP_CASES = ["tricubic_bp", "nearest_bp", "tricubic_reflective_ck", "modulated_bp", "modulated_tricubic_ck"]


def _step_spec(name, precision=_abi.PRECISION_FP64):
    if name == "tricubic_bp":
        fields, prop = [_vector_grid(CUB)], bp_fixed(0.5 * KPC)
    elif name == "nearest_bp":
        fields, prop = [_vector_grid(NN)], bp_fixed(0.5 * KPC)
    elif name == "tricubic_reflective_ck":
        fields, prop = [_vector_grid(CUB, reflective=True)], ck(1e-4, 0.1 * KPC, 5 * KPC)
    elif name == "modulated_bp":
        fields, prop = [P.ModulatedGridField(_vector_grid(TRI), _modulation(TRI))], bp_fixed(0.5 * KPC)
    else:
        fields = [P.ModulatedGridField(_vector_grid(CUB), _modulation(CUB))]
        prop = ck(1e-4, 0.1 * KPC, 5 * KPC)
    mods = [prop, P.MaxTrajectoryLength(150 * KPC, record=True),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 40 * KPC, True, True)]
    return P.ChainSpec(fields, mods, precision=precision)


def _cands(n=300, seed=36):
    c = protons(np.random.default_rng(seed), n, emin=1 * U.EeV, emax=100 * U.EeV, spread=20 * KPC)
    c.next_step[:] = 1e30
    return c


STATE = ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "time", "current_step", "next_step",
         "active", "flags")


@pytest.mark.parametrize("name", STEP_CASES)
def test_stepping_oracle_matches_reference(oracle, reference, name):
    spec = _step_spec(name)
    c = _cands()
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=1)
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


@pytest.mark.parametrize("name,expect", [
    ("tricubic_bp", "Grid3f 16x12x10 spacing 3.08568e+20 reflective 0 clipVolume 0 TRICUBIC"),
    ("nearest_bp", "NEAREST_NEIGHBOUR"),
    ("modulated_tricubic_ck", "ModulatedMagneticFieldGrid Grid3f 16x12x10"),
    ("modulated_bp", "modulation Grid1f 9x11x7"),
])
def test_plugin_translates_interpolation_and_modulated_grid(plugin, name, expect):
    ok, text = plugin.describe(_step_spec(name))
    assert ok, text
    assert expect in text, text


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
@pytest.mark.parametrize("interp,refl,clip", VECTOR_CASES)
def test_device_vector_grid_field_matches_oracle(oracle, interp, refl, clip):
    from crpropa3_b200.engine import Plan
    spec = _vector_spec(interp, refl, clip)
    pos = _positions()
    np.testing.assert_array_equal(Plan(spec).field(pos), oracle.field(spec, pos))


@pytest.mark.gpu
@pytest.mark.parametrize("gi,mi,mr", MOD_CASES)
def test_device_modulated_grid_field_matches_oracle(oracle, gi, mi, mr):
    from crpropa3_b200.engine import Plan
    spec = _mod_spec(gi, mi, mr)
    pos = _positions(seed=34)
    np.testing.assert_array_equal(Plan(spec).field(pos), oracle.field(spec, pos))


@pytest.mark.gpu
@pytest.mark.parametrize("name", STEP_CASES)
def test_device_fp64_stepping_matches_oracle(oracle_crpow, name):
    from crpropa3_b200.engine import Plan
    spec = _step_spec(name)
    c = _cands()
    a = c.copy()
    oracle_crpow.run(spec, a)
    d = c.to_device("cuda")
    Plan(spec).run(d)
    h = d.to_host()
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(h, m), err_msg=m)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tricubic_bp", "modulated_bp", "modulated_tricubic_ck"])
def test_device_mixed_stepping_close_to_oracle(oracle_crpow, name):
    """Mixed form (FP32 field and rotation, FP64 accumulation): the same
    detections for nearly all candidates and final positions close to the
    FP64 path's for the candidates that end the same way."""
    from crpropa3_b200.engine import Plan
    c = _cands()
    a = c.copy()
    oracle_crpow.run(_step_spec(name), a)
    d = c.to_device("cuda")
    Plan(_step_spec(name, _abi.PRECISION_MIXED)).run(d)
    h = d.to_host()
    same = (h.flags == a.flags)
    assert same.mean() >= 0.95
    rel = np.linalg.norm(h.position() - a.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert np.median(rel[same]) <= 1e-5, np.median(rel[same])


@pytest.mark.gpu
def test_device_refuses_unknown_interpolation():
    from crpropa3_b200.engine import Plan
    spec = _vector_spec("trilinear", False, False)
    spec.fields[0].interpolation = 3
    with pytest.raises(Exception, match="interpolation"):
        Plan(spec)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["tricubic_bp", "nearest_bp", "modulated_bp"])
def test_plugin_interpolation_and_modulated_grid_bitwise(plugin, reference, name):
    """The reference's own tricubic / nearest Grid3f and
    ModulatedMagneticFieldGrid objects, run through GpuModuleList (FP64
    form), against ModuleList::run: the same state, bit for bit."""
    spec = _step_spec(name)
    c = _cands()
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=2)
    plugin.run(spec, b)
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
