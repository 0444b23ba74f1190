"""Parity of the CUDA stepping path with the oracle (crp_oracle.c), on the GPU.

Tolerances:
  * FP64 form, Boris push over a Grid3f: bit-identical (the arithmetic is
    + - * / sqrt floor only, compiled without contraction on both sides).
  * FP64 form, fixed-step Cash-Karp: bit-identical.
  * FP64 form, adaptive Cash-Karp / Boris: the step controller calls
    pow(r, -0.2).  The device uses a correctly rounded pow; glibc's pow
    misrounds about 1e-3 of inputs, and one different last bit of a step size
    changes the rest of that trajectory (chaotically, in a turbulent field).
    Bar: bit-identical to the oracle built with the same correctly rounded pow
    (every other operation is then the reference's), and >= 80 % of
    candidates bit-identical to the glibc-pow oracle.
  * mixed form: see test_mixed_precision.py.
  * mixed form: relative final-position error <= 1e-6 against the FP64
    oracle (the stated bound of the mixed-precision form).
"""
import numpy as np
import pytest

from helpers import (P, U, _abi, RecordArrays, bp_fixed, ck, grid_chain, protons, random_grid,
                     rel_pos_err)

pytestmark = pytest.mark.gpu


def _engine():
    from crpropa3_b200.engine import Plan
    return Plan


def _run_both(oracle, spec, cands, cap=4096, **kw):
    Plan = _engine()
    a, b = cands.copy(), cands.copy()
    ra, rb = RecordArrays(cap), RecordArrays(cap)
    oracle.run(spec, a, ra)
    plan = Plan(spec)
    stats = plan.run(b, records=rb, **kw)
    plan.close()
    return a, b, ra, rb, stats


def _assert_same_state(a, b):
    for name in ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time",
                 "current_step", "next_step", "active", "flags"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)


def _assert_same_records(ra, rb):
    assert ra.n() == rb.n()
    sa, sb = ra.sorted(), rb.sorted()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k], err_msg=k)


@pytest.mark.parametrize("reflective", [False, True])
def test_bp_fixed_fp64_bitwise(oracle, reflective):
    rng = np.random.default_rng(11)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, bp_fixed(1 * U.kpc), 2 * U.Mpc, observer_radius=0.5 * U.Mpc,
                      reflective=reflective)
    c = protons(rng, 300)
    a, b, ra, rb, stats = _run_both(oracle, spec, c)
    _assert_same_state(a, b)
    _assert_same_records(ra, rb)
    assert stats.particle_steps > 300 * 100


def test_bp_fixed_fp64_bitwise_non_pow2_grid_and_offset_origin(oracle):
    rng = np.random.default_rng(12)
    grid = (rng.standard_normal((12, 10, 14, 3)) * 1e-13).astype(np.float32)
    spec = P.ChainSpec([P.GridField(grid, (-3 * U.kpc, 7 * U.kpc, 1 * U.kpc), (8 * U.kpc,) * 3)],
                       [bp_fixed(0.7 * U.kpc), P.MaxTrajectoryLength(1 * U.Mpc)])
    c = protons(rng, 200)
    a, b, *_ = _run_both(oracle, spec, c)
    _assert_same_state(a, b)


def test_bp_adaptive_fp64(oracle, oracle_crpow):
    rng = np.random.default_rng(13)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, P.Propagation(_abi.PROP_BP, 1e-3, 0.1 * U.kpc, 10 * U.kpc),
                      2 * U.Mpc, observer_radius=0.7 * U.Mpc)
    c = protons(rng, 300)
    a, b, ra, rb, _ = _run_both(oracle_crpow, spec, c)
    _assert_same_state(a, b)
    _assert_same_records(ra, rb)
    g = c.copy()
    oracle.run(spec, g)
    assert np.mean(rel_pos_err(b, g) == 0) >= 0.8


def test_ck_adaptive_fp64(oracle, oracle_crpow):
    rng = np.random.default_rng(14)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, ck(1e-4, 0.1 * U.kpc, 10 * U.kpc), 2 * U.Mpc,
                      observer_radius=0.7 * U.Mpc)
    c = protons(rng, 300)
    a, b, ra, rb, _ = _run_both(oracle_crpow, spec, c)
    _assert_same_state(a, b)
    _assert_same_records(ra, rb)
    g = c.copy()
    oracle.run(spec, g)
    assert np.mean(rel_pos_err(b, g) == 0) >= 0.8


def test_ck_fixed_fp64_bitwise(oracle):
    rng = np.random.default_rng(15)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, ck(1e-4, 1 * U.kpc, 1 * U.kpc), 1 * U.Mpc)
    c = protons(rng, 200)
    a, b, *_ = _run_both(oracle, spec, c)
    _assert_same_state(a, b)


def test_field_eval_fp64_matches_oracle(oracle):
    rng = np.random.default_rng(18)
    grid = random_grid(rng, 8)
    pos = rng.uniform(-300, 300, (2000, 3)) * U.kpc
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(1e-13, 10 * U.kpc, 300 * U.kpc, 1.0, 5 / 3, 4, 64, 7)
    pw = P.PlaneWaveField(xi, kappa, k, beta, ak)
    cases = [
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3)],
        [P.GridField(grid, (5 * U.kpc, 0, -3 * U.kpc), (10 * U.kpc,) * 3, reflective=True)],
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3, clip_volume=True)],
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3,
                     periodic=((0, 0, 0), (80 * U.kpc,) * 3, True))],
        [pw],
        [P.UniformField((1e-13, -2e-13, 3e-13)), P.ToroidalField(1e-10), pw],
    ]
    Plan = _engine()
    for fields in cases:
        spec = P.ChainSpec(fields, [bp_fixed(U.kpc)])
        ref = oracle.field(spec, pos)
        got = Plan(spec).field(pos)
        if any(isinstance(f, P.PlaneWaveField) for f in fields):
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
        else:
            np.testing.assert_array_equal(got, ref)


def test_field_eval_mixed_close(oracle):
    rng = np.random.default_rng(19)
    grid = random_grid(rng, 8)
    pos = rng.uniform(-300, 300, (2000, 3)) * U.kpc
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(1e-13, 10 * U.kpc, 300 * U.kpc, 1.0, 5 / 3, 4, 256, 9)
    Plan = _engine()
    odd = [xi[:3 * 255], kappa[:3 * 255], k[:255], beta[:255], ak[:255]]  # the mixed table pads to pairs
    for fields in ([P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3)],
                   [P.PlaneWaveField(xi, kappa, k, beta, ak)], [P.PlaneWaveField(*odd)]):
        spec = P.ChainSpec(fields, [bp_fixed(U.kpc)], precision=_abi.PRECISION_MIXED)
        ref = oracle.field(spec, pos)
        got = Plan(spec).field(pos)
        scale = np.sqrt((ref ** 2).sum(1).mean())
        assert np.abs(got - ref).max() <= 2e-5 * scale


def test_empty_and_inactive_inputs(oracle):
    rng = np.random.default_rng(20)
    grid = random_grid(rng, 8)
    spec = grid_chain(grid, 10 * U.kpc, bp_fixed(U.kpc), 100 * U.kpc)
    Plan = _engine()
    plan = Plan(spec)
    from crpropa3_b200.state import CandidateArrays
    stats = plan.run(CandidateArrays(0))
    assert stats.particle_steps == 0
    c = protons(rng, 64)
    c.active[::2] = 0
    a, b, *_ = _run_both(oracle, spec, c)
    _assert_same_state(a, b)
    assert np.all(b.trajectory_length[::2] == 0)
