"""PolarizedSingleModeMagneticField (PolarizedSingleModeMagneticField.cpp:5-64):
one polarised mode B = B_max (u1 cos(k.(x - r0)) + u2 sigma sin(k.(x - r0))).

CPU: crp_single_mode_field's derived state and checks against the
reference's constructor (same messages), the oracle's field and stepping
against the reference's own field, bit for bit.
GPU: the device evaluates in FP64 with CUDA's sin and cos (phases of many
turns: compared within 1e-12 of the amplitude); the mixed form rounds the
FP64 field to FP32 (1e-6 of the amplitude).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, protons

KPC = U.kpc
MODELS = {
    "elliptical": P.SingleModeField(1 * U.muG, 30 * U.pc, 0.5, (1 * KPC, -2 * KPC, 0.3 * KPC), (1.0, 2.0, 0.0),
                                    (-2.0, 1.0, 3.0)),
    "circular_rms": P.SingleModeField(2 * U.nG, 1 * KPC, -1.0, e1=(0.0, 0.0, 2.0), e2=(1.0, 1.0, 0.0),
                                      amplitude_rms="rms", mode="circular"),
    "helicity": P.SingleModeField(0.5 * U.nG, 0.37 * KPC, 1.0, polarization_helicity="helicity",
                                  mode="circular"),
    "linear": P.SingleModeField(3 * U.nG, 2 * KPC, 0.0, e1=(0.0, 3.0, 4.0), e2=(5.0, 0.0, 0.0), mode="linear"),
}


def _spec(model, precision=_abi.PRECISION_FP64, modules=None):
    return P.ChainSpec([MODELS[model]], modules or [bp_fixed(KPC)], precision=precision)


def _positions(n=3000, seed=81):
    return np.random.default_rng(seed).uniform(-300, 300, (n, 3)) * KPC


@pytest.mark.parametrize("model", sorted(MODELS))
def test_field_oracle_matches_reference(oracle, reference, model):
    spec = _spec(model)
    pos = _positions()
    a, b = oracle.field(spec, pos), reference.field(spec, pos)
    np.testing.assert_array_equal(a, b)
    assert np.abs(a).max() > 0


def test_derived_state():
    d = MODELS["linear"].desc()
    np.testing.assert_array_equal(d.u1, [0.0, 0.6, 0.8])
    np.testing.assert_array_equal(d.u2, [1.0, 0.0, 0.0])
    # e_2 x e_1 = (0, -20, 15) / 25, times 2 pi / wavelength
    np.testing.assert_allclose(d.k, np.array([0.0, -0.8, 0.6]) * 2 * np.pi / (2 * KPC), rtol=1e-15)
    r = MODELS["circular_rms"].desc()
    assert r.b_max == np.sqrt(2 / (1 + 1.0)) * 2 * U.nG


@pytest.mark.parametrize("kw,msg", [
    (dict(sigma=1.5), "has to lie in the range [-1;+1]"),
    (dict(sigma=0.5, mode="circular"), "For circular polarization"),
    (dict(sigma=0.5, mode="linear"), "For linear polarization"),
    (dict(e2=(1.0, 0.0, 0.0)), "e_1 and e_2 have to be orthogonal"),
    (dict(wavelength=0.0), "The correlation length cannot be zero."),
    (dict(sigma=0.5, polarization_helicity="helicity"), "In helicity mode only"),
    (dict(mode="spiral"), "Wrong value for flagMode"),
])
def test_constructor_checks(kw, msg):
    args = dict(b0=1e-10, wavelength=1 * KPC, sigma=0.0, e1=(1.0, 0.0, 0.0), e2=(0.0, 1.0, 0.0), mode="elliptical")
    args.update(kw)
    with pytest.raises(_abi.CrpError) as e:
        P.SingleModeField(**args).desc()
    assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    assert msg in str(e.value)


def test_stepping_oracle_matches_reference(oracle, reference):
    spec = _spec("elliptical", modules=[bp_fixed(10 * U.pc), P.MaxTrajectoryLength(20 * KPC)])
    c = protons(np.random.default_rng(82), 200, emin=0.01 * U.EeV, emax=1 * U.EeV)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    oracle.run(spec, b)
    for m in ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "active", "flags"):
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)


def test_plugin_translates_single_mode():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built")
    ok, text = PluginHarness().describe(_spec("helicity"))
    assert ok, text
    assert "PolarizedSingleModeMagneticField sigma 1" in text, text


@pytest.mark.gpu
@pytest.mark.parametrize("model", sorted(MODELS))
def test_device_fields_close_to_oracle(oracle, model):
    from crpropa3_b200.engine import Plan
    pos = _positions()
    a = oracle.field(_spec(model), pos)
    amp = MODELS[model].desc().b_max * max(1.0, abs(MODELS[model].sigma))
    np.testing.assert_allclose(Plan(_spec(model)).field(pos), a, rtol=0, atol=1e-12 * amp)
    np.testing.assert_allclose(Plan(_spec(model, _abi.PRECISION_MIXED)).field(pos), a, rtol=0, atol=1e-6 * amp)
