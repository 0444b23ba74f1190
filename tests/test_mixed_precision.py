"""Error of the mixed-precision form against the FP64 form, on the GPU.

The stated bound: relative final-position error <= 1e-6 against FP64.

In a turbulent field low-rigidity trajectories are chaotic: a perturbation
of one ulp of the starting position (1e-16) grows to O(1) over a few thousand
steps, so no implementation that differs from the FP64 form in any rounding
can stay within 1e-6 of it there.  The tests therefore state the bound where
the FP64 problem is itself well conditioned, measured directly: the
divergence of the FP64 form from the same run started with a direction one
ulp away.  Where
that divergence stays <= 1e-12 (condition number <= 1e4), the mixed form must
be within 1e-6; and the bound must hold for every candidate of a
non-chaotic case (high rigidity, weak field).
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, grid_chain, protons, random_grid, rel_pos_err

pytestmark = pytest.mark.gpu


def _run(spec, cands):
    from crpropa3_b200.engine import Plan
    out = cands.copy()
    Plan(spec).run(out)
    return out


def _one_ulp(c):
    """The same candidates with the x direction component one ulp larger
    (a position at the origin would absorb a one-ulp change)."""
    d = c.copy()
    d.dx[:] = np.nextafter(d.dx, np.inf)
    return d


def _kolmogorov(n, spacing, brms, lmin, lmax):
    from crpropa3_b200.turbulence import grid_turbulence
    return grid_turbulence(n, spacing, brms, lmin, lmax, seed=42)


def test_bp_mixed_bound_weak_deflection(oracle):
    """10-100 EeV protons in 1 nG: every candidate within 1e-6 of FP64."""
    grid = _kolmogorov(64, 10 * U.kpc, 1 * U.nG, 20 * U.kpc, 200 * U.kpc)
    rng = np.random.default_rng(31)
    c = protons(rng, 512, emin=10 * U.EeV, emax=100 * U.EeV, spread=0.0)
    s64 = grid_chain(grid, 10 * U.kpc, bp_fixed(1 * U.kpc), 5 * U.Mpc)
    smx = grid_chain(grid, 10 * U.kpc, bp_fixed(1 * U.kpc), 5 * U.Mpc, precision=_abi.PRECISION_MIXED)
    ref = c.copy()
    oracle.run(s64, ref)
    got = _run(smx, c)
    err = rel_pos_err(got, ref)
    assert err.max() <= 1e-6, err.max()
    np.testing.assert_array_equal(got.trajectory_length, ref.trajectory_length)


@pytest.mark.parametrize("prop", ["bp", "ck"])
def test_mixed_bound_where_fp64_is_well_conditioned(oracle, prop):
    """Chaotic case: the bound holds wherever FP64 itself is stable to 1 ulp."""
    grid = _kolmogorov(64, 10 * U.kpc, 10 * U.nG, 20 * U.kpc, 200 * U.kpc)
    rng = np.random.default_rng(32)
    c = protons(rng, 1024, emin=1 * U.EeV, emax=100 * U.EeV, spread=0.0)
    p = bp_fixed(1 * U.kpc) if prop == "bp" else ck(1e-4, 0.1 * U.kpc, 100 * U.kpc)
    s64 = grid_chain(grid, 10 * U.kpc, p, 3 * U.Mpc)
    smx = grid_chain(grid, 10 * U.kpc, p, 3 * U.Mpc, precision=_abi.PRECISION_MIXED)
    f64 = _run(s64, c)
    f64_ulp = _run(s64, _one_ulp(c))
    mixed = _run(smx, c)
    floor = rel_pos_err(f64_ulp, f64)
    err = rel_pos_err(mixed, f64)
    stable = floor <= 1e-12
    assert stable.mean() >= 0.25, stable.mean()
    assert err[stable].max() <= 1e-6, err[stable].max()
    # and where FP64 diverges from itself, the mixed form diverges no faster
    assert np.median(err) <= max(1e-6, 10 * np.median(floor) * 1e7)
