"""The adjoint's forward model and the oracle's CPU adjoint against the
reference's own PropagationBP (PropagationBP.cpp:62, fixed step) over
MagneticFieldGrid (MagneticFieldGrid.cpp:17), on the CPU.

* Forward model: the adjoint interpolates with double trilinear weights,
  the reference with float weights (Grid.h:559-568); over 200 weakly
  deflecting 1 kpc steps the per-candidate losses agree to 1e-8
  (measured 8e-10).
* Gradients: central differences through the reference's modules, with
  perturbed Grid3f values (relative step 1e-3; the loss is close to linear
  in them), perturbed initial directions (1e-4 rad, tangent plane, since
  the reference normalises directions) and perturbed energies (relative
  1e-4), against the oracle's CPU adjoint.  The float weights of the
  reference put noise of ~1e-5 relative on these differences; the bar is
  2e-3 relative to the largest gradient component.
"""
import numpy as np

from helpers import P, U, bp_fixed, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays

STEP, NSTEPS = 1 * U.kpc, 200
SPACING = 10 * U.kpc
NGRID = 16


def _problem(n=8, seed=90):
    rng = np.random.default_rng(seed)
    grid = random_grid(rng, NGRID, brms=3e-13)
    u0 = stable_unit_vectors(rng, n)
    energy = np.exp(rng.uniform(np.log(5), np.log(50), n)) * U.EeV
    charge = np.full(n, -U.eplus)
    pos = rng.uniform(0, NGRID * 10, (n, 3)) * U.kpc
    target = stable_unit_vectors(rng, n)
    return grid, pos, u0, energy, charge, target


def _reference_losses(reference, grid, pos, u0, energy, charge, target):
    """Per-candidate loss 1 - u_final . target from the reference's own
    PropagationBP + MaximumTrajectoryLength over a MagneticFieldGrid."""
    n = len(energy)
    c = CandidateArrays(n)
    c.id[:] = -1000010010
    c.charge[:] = charge
    c.energy[:] = energy
    c.set_position(pos)
    c.set_direction(u0)
    spec = P.ChainSpec([P.GridField(grid, (0.0, 0.0, 0.0), (SPACING,) * 3)],
                       [bp_fixed(STEP), P.MaxTrajectoryLength(NSTEPS * STEP, record=False)])
    reference.run(spec, c, threads=1)
    return 1.0 - (c.direction() * target).sum(1)


def _adj(oracle, prob):
    grid, pos, u0, energy, charge, target = prob
    return oracle.bp_adjoint(grid, (0.0, 0.0, 0.0), SPACING, STEP, NSTEPS, pos, u0, energy, charge, target)


def test_adjoint_forward_model_tracks_reference(oracle, reference):
    prob = _problem()
    loss_ref = _reference_losses(reference, *prob)
    loss, _, _, _ = _adj(oracle, prob)
    np.testing.assert_allclose(loss, loss_ref, rtol=0, atol=1e-8)


def test_grid_gradient_against_reference_differences(oracle, reference):
    prob = _problem(seed=91)
    grid = prob[0]
    _, _, _, gg = _adj(oracle, prob)
    # the cells with the largest gradient, plus a few at random
    flat = np.argsort(np.abs(gg).ravel())[::-1][:6]
    rng = np.random.default_rng(5)
    flat = np.concatenate([flat, rng.choice(np.flatnonzero(gg.ravel()), 4, replace=False)])
    scale = np.abs(gg).max()
    for f in flat:
        idx = np.unravel_index(f, grid.shape)
        h = np.float32(1e-3 * max(abs(float(grid[idx])), 1e-14))
        gp, gm = grid.copy(), grid.copy()
        gp[idx] += h
        gm[idx] -= h
        hp, hm = float(gp[idx]) - float(grid[idx]), float(grid[idx]) - float(gm[idx])
        lp = _reference_losses(reference, gp, *prob[1:]).sum()
        lm = _reference_losses(reference, gm, *prob[1:]).sum()
        fd = (lp - lm) / (hp + hm)
        assert abs(fd - gg[idx]) <= 2e-3 * scale, (idx, fd, gg[idx], scale)


def test_direction_and_energy_gradients_against_reference_differences(oracle, reference):
    prob = _problem(seed=92)
    grid, pos, u0, energy, charge, target = prob
    _, gu, ge, _ = _adj(oracle, prob)
    n = len(energy)
    rng = np.random.default_rng(6)
    e1 = np.cross(u0, rng.standard_normal((n, 3)))
    e1 /= np.linalg.norm(e1, axis=1)[:, None]
    h = 1e-4
    up = u0 + h * e1
    um = u0 - h * e1
    up /= np.linalg.norm(up, axis=1)[:, None]
    um /= np.linalg.norm(um, axis=1)[:, None]
    lp = _reference_losses(reference, grid, pos, up, energy, charge, target)
    lm = _reference_losses(reference, grid, pos, um, energy, charge, target)
    # up/um lie at angle atan(h) from u0 along e1
    fd_u = (lp - lm) / (2 * np.arctan(h))
    an_u = (gu * e1).sum(1)
    np.testing.assert_allclose(fd_u, an_u, rtol=0, atol=2e-3 * np.abs(an_u).max())
    he = 1e-4 * energy
    lp = _reference_losses(reference, grid, pos, u0, energy + he, charge, target)
    lm = _reference_losses(reference, grid, pos, u0, energy - he, charge, target)
    fd_e = (lp - lm) / (2 * he)
    np.testing.assert_allclose(fd_e, ge, rtol=0, atol=2e-3 * np.abs(ge).max())
