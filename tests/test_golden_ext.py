"""The oracle (CPU) and the device (GPU) against the second set of golden
fixtures generated from the reference by tests/golden/make_golden.py
(main_ext): tricubic / nearest Grid3f and modulated-grid fields, observer
features and boundaries, JF12Field / PlanckJF12bField, the UF23Field models,
the turbulence draw sequences and the grid file formats.  These pin the
restated functions to the reference without rebuilding it."""
import os

import numpy as np
import pytest

from helpers import RecordArrays, _abi
from crpropa3_b200 import gridtools as G, turbulence as T

import test_grid_interpolation as GI
import test_jf12 as J
import test_observers_boundaries as OB
import test_uf23 as UF

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden_ext.npz")
CHAINS = ("box", "cylindrical", "vetoes", "tracking")


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def test_oracle_interpolation_fields_golden(oracle, golden):
    pos = golden["interp/pos"]
    for interp, refl, clip in GI.VECTOR_CASES:
        np.testing.assert_array_equal(oracle.field(GI._vector_spec(interp, refl, clip), pos),
                                      golden[f"interp/B_{interp}_{int(refl)}_{int(clip)}"])
    for gi, mi, mr in GI.MOD_CASES:
        np.testing.assert_array_equal(oracle.field(GI._mod_spec(gi, mi, mr), pos),
                                      golden[f"modulated/B_{gi}_{mi}_{int(mr)}"])


@pytest.mark.parametrize("name", CHAINS)
def test_oracle_observer_and_boundary_chains_golden(oracle, golden, name):
    c = OB._cands(120, seed=202)
    rec = RecordArrays(20000)
    oracle.run(OB._spec(name), c, rec)
    for m in OB.STATE:
        np.testing.assert_array_equal(getattr(c, m), golden[f"chain_{name}/out_{m}"], err_msg=m)
    for k, v in rec.sorted().items():
        np.testing.assert_array_equal(v, golden[f"chain_{name}/rec_{k}"], err_msg=k)


def test_oracle_galactic_fields_golden(oracle, golden):
    for name in J.FIELDS:
        np.testing.assert_array_equal(oracle.field(J._spec(name), golden["jf12/pos"]), golden[f"jf12/B_{name}"])
    for name in UF.MODELS:
        np.testing.assert_array_equal(oracle.field(UF._spec(name), golden["uf23/pos"]), golden[f"uf23/B_{name}"])


def test_host_tools_golden(golden, tmp_path):
    from crpropa3_b200 import plan as P
    np.testing.assert_array_equal(P.jf12_random_striated(12345).values[:10, :10, :10],
                                  golden["jf12/striated_12345"])
    for kind in (0, 1, 2):
        np.testing.assert_array_equal(T.turbulence_draws(777, kind, 300), golden[f"turbulence/draws_{kind}"])
    v3, v1 = golden["gridfile/v3"], golden["gridfile/v1"]
    props = dict(origin=(1e19, -2e19, 0.5), spacing=(3e19, 3e19, 3e19), reflective=True, clip_volume=False,
                 interpolation=_abi.INTERPOLATION_TRICUBIC)
    for key, v, txt in (("v3_raw", v3, False), ("v1_raw", v1, False), ("v3_txt", v3, True), ("v1_txt", v1, True)):
        path = tmp_path / key
        if txt:
            G.dump_grid_to_txt(v, path, 2.5, True, **props)
        else:
            G.dump_grid(v, path, 2.5)
        assert np.array_equal(np.frombuffer(path.read_bytes(), np.uint8), golden[f"gridfile/{key}"]), key


@pytest.mark.gpu
def test_device_interpolation_fields_golden(golden):
    from crpropa3_b200.engine import Plan
    pos = golden["interp/pos"]
    for interp, refl, clip in GI.VECTOR_CASES:
        np.testing.assert_array_equal(Plan(GI._vector_spec(interp, refl, clip)).field(pos),
                                      golden[f"interp/B_{interp}_{int(refl)}_{int(clip)}"])
    for gi, mi, mr in GI.MOD_CASES:
        np.testing.assert_array_equal(Plan(GI._mod_spec(gi, mi, mr)).field(pos),
                                      golden[f"modulated/B_{gi}_{mi}_{int(mr)}"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CHAINS)
def test_device_fp64_observer_and_boundary_chains_golden(golden, name):
    from crpropa3_b200.engine import Plan
    c = OB._cands(120, seed=202)
    d = c.to_device("cuda")
    rd = RecordArrays(20000, device="cuda")
    Plan(OB._spec(name)).run(d, records=rd)
    h, r = d.to_host(), rd.to_host()
    for m in OB.STATE:
        np.testing.assert_array_equal(getattr(h, m), golden[f"chain_{name}/out_{m}"], err_msg=m)
    for k, v in r.sorted().items():
        np.testing.assert_array_equal(v, golden[f"chain_{name}/rec_{k}"], err_msg=k)


@pytest.mark.gpu
def test_device_galactic_fields_golden(golden):
    """Within the bounds of tests/test_jf12.py and tests/test_uf23.py (CUDA's
    exp, sin, cos, acos, atan2 and log against glibc's)."""
    from crpropa3_b200.engine import Plan
    for name in J.FIELDS:
        g = golden[f"jf12/B_{name}"]
        np.testing.assert_allclose(Plan(J._spec(name)).field(golden["jf12/pos"]), g, rtol=0,
                                   atol=1e-13 * np.abs(g).max())
    for name in UF.MODELS:
        g = golden[f"uf23/B_{name}"]
        np.testing.assert_allclose(Plan(UF._spec(name)).field(golden["uf23/pos"]), g, rtol=0,
                                   atol=1e-12 * np.abs(g).max())
