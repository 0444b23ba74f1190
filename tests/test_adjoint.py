"""Adjoint of the fixed-step Boris push (crp_bp_adjoint) on the GPU, checked
against the oracle's CPU reference adjoint, central finite differences of
the FP64 forward model (relative step 1e-6) and the torch.autograd wrapper.
Antiprotons backtracked through a periodic Grid3f (the backtracking
convention of the reference's galactic backtracking examples)."""
import numpy as np
import pytest

from helpers import U, random_grid, stable_unit_vectors

pytestmark = pytest.mark.gpu

STEP, NSTEPS, K = 1 * U.kpc, 300, 16
SPACING = 10 * U.kpc
ORIGIN = (0.0, 0.0, 0.0)


def _problem(n=48, seed=80):
    rng = np.random.default_rng(seed)
    grid = random_grid(rng, 32, brms=3e-13)
    u0 = stable_unit_vectors(rng, n)
    energy = np.exp(rng.uniform(np.log(5), np.log(50), n)) * U.EeV
    charge = np.full(n, -U.eplus)
    pos = rng.uniform(0, 320, (n, 3)) * U.kpc
    target = stable_unit_vectors(rng, n)
    return grid, pos, u0, energy, charge, target


def _gpu(grid, pos, u0, energy, charge, target, k=K, want_grid=True):
    import torch
    from crpropa3_b200.adjoint import bp_loss_and_grads
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    loss, gu, ge, gg = bp_loss_and_grads(t(grid), ORIGIN, SPACING, STEP, NSTEPS, t(pos), t(u0), t(energy),
                                         t(charge), t(target), k, want_grid)
    return (loss.cpu().numpy(), gu.cpu().numpy(), ge.cpu().numpy(),
            gg.cpu().numpy() if gg is not None else None)


def test_adjoint_matches_cpu_reference_adjoint(oracle):
    prob = _problem()
    loss_r, gu_r, ge_r, gg_r = oracle.bp_adjoint(prob[0], ORIGIN, SPACING, STEP, NSTEPS, *prob[1:])
    loss, gu, ge, gg = _gpu(*prob)
    np.testing.assert_allclose(loss, loss_r, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(gu, gu_r, rtol=1e-9, atol=1e-12 * np.abs(gu_r).max())
    np.testing.assert_allclose(ge, ge_r, rtol=1e-9, atol=1e-12 * np.abs(ge_r).max())
    # fixed-point accumulation: unit 2^-36 max|kappa| per contribution
    np.testing.assert_allclose(gg, gg_r, rtol=0, atol=1e-9 * np.abs(gg_r).max())


def test_adjoint_is_deterministic_and_checkpoint_independent():
    prob = _problem(seed=81)
    a = _gpu(*prob)
    b = _gpu(*prob)
    c = _gpu(*prob, k=7)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)  # same bits on every run
    for x, y in zip(a[:3], c[:3]):
        np.testing.assert_array_equal(x, y)  # recomputation from any checkpoint spacing
    np.testing.assert_array_equal(a[3], c[3])


def test_adjoint_matches_central_finite_differences(oracle):
    grid, pos, u0, energy, charge, target = _problem(n=24, seed=82)
    _, gu, ge, gg = _gpu(grid, pos, u0, energy, charge, target)
    L = lambda g=grid, u=u0, e=energy: oracle.bp_loss(g, ORIGIN, SPACING, STEP, NSTEPS, pos, u, e, charge, target)
    # 64 grid values among those with the largest gradients
    flat = np.argsort(-np.abs(gg).ravel())[:64]
    for f in flat:
        g = grid.copy().ravel()
        v = g[f]
        gp, gm = g.copy(), g.copy()
        gp[f] = np.float32(v * (1 + 1e-6))
        gm[f] = np.float32(v * (1 - 1e-6))
        dp, dm = float(gp[f]) - float(v), float(gm[f]) - float(v)
        fd = (L(gp.reshape(grid.shape)) - L(gm.reshape(grid.shape))) / (dp - dm)
        assert abs(fd - gg.ravel()[f]) <= 1e-4 * abs(gg.ravel()[f]) + 1e-6 * np.abs(gg).max(), (f, fd, gg.ravel()[f])
    # initial directions and energies of a few candidates
    for i in range(4):
        for a in range(3):
            up, um = u0.copy(), u0.copy()
            h = 1e-6
            up[i, a] += h
            um[i, a] -= h
            fd = (L(u=up) - L(u=um)) / (2 * h)
            assert abs(fd - gu[i, a]) <= 1e-4 * max(abs(gu[i, a]), 1e-3), (i, a, fd, gu[i, a])
        ep, em = energy.copy(), energy.copy()
        ep[i] *= 1 + 1e-6
        em[i] *= 1 - 1e-6
        fd = (L(e=ep) - L(e=em)) / (ep[i] - em[i])
        assert abs(fd - ge[i]) <= 1e-4 * abs(ge[i]) + 1e-30, (i, fd, ge[i])


def test_autograd_function_gives_momentum_and_grid_gradients():
    import torch
    from crpropa3_b200.adjoint import arrival_loss
    grid, pos, u0, energy, charge, target = _problem(n=32, seed=83)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    p0 = (t(u0) * (t(energy) / U.c_light)[:, None]).clone().requires_grad_(True)
    g = t(grid).clone().requires_grad_(True)
    L = arrival_loss(p0, g, t(pos), t(charge), t(target), ORIGIN, SPACING, STEP, NSTEPS, K)
    L.backward()
    _, gu, ge, gg = _gpu(grid, pos, u0, energy, charge, target)
    un = u0
    pn = energy / U.c_light
    tang = gu - un * (un * gu).sum(1, keepdims=True)
    gp_expected = tang / pn[:, None] + U.c_light * un * ge[:, None]
    np.testing.assert_allclose(p0.grad.cpu().numpy(), gp_expected, rtol=1e-9, atol=1e-12 * np.abs(gp_expected).max())
    np.testing.assert_allclose(g.grad.cpu().numpy(), gg.astype(np.float32), rtol=1e-6, atol=1e-6 * np.abs(gg).max())
    assert abs(L.item() - _gpu(grid, pos, u0, energy, charge, target, want_grid=False)[0].sum()) < 1e-9
