"""Shared inputs for the parity tests: seeded grids, candidates, chains."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

from crpropa3_b200 import _abi, plan as P, units as U  # noqa: E402
from crpropa3_b200.state import CandidateArrays, RecordArrays  # noqa: E402


def normalize(d):
    """ParticleState::setDirection: d / |d| with |d| = sqrt(x*x + y*y + z*z)."""
    d = np.asarray(d, dtype=np.float64)
    n = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    return d / n[:, None]


def stable_unit_vectors(rng, n):
    """Unit vectors that setDirection maps to themselves bit for bit, so that
    the reference's normalisation at Candidate construction changes nothing."""
    out = np.zeros((n, 3))
    filled = 0
    while filled < n:
        d = normalize(rng.standard_normal((2 * (n - filled) + 8, 3)))
        d2 = normalize(d)
        ok = np.all(d2 == d, axis=1)
        take = d[ok][: n - filled]
        out[filled:filled + len(take)] = take
        filled += len(take)
    return out


def random_grid(rng, n, brms=1e-13):
    return (rng.standard_normal((n, n, n, 3)) * brms).astype(np.float32)


def protons(rng, n, emin=1 * U.EeV, emax=100 * U.EeV, spread=50 * U.kpc, origin=(0, 0, 0)):
    c = CandidateArrays(n)
    c.id[:] = 1000010010
    c.charge[:] = U.eplus
    c.energy[:] = emin * np.exp(rng.uniform(0, np.log(emax / emin), n))
    c.set_position(np.asarray(origin) + rng.uniform(-spread, spread, (n, 3)))
    c.set_direction(stable_unit_vectors(rng, n))
    return c


def grid_chain(grid, spacing, prop, max_length, observer_radius=None, precision=_abi.PRECISION_FP64,
               reflective=False, record=True, origin=(0, 0, 0)):
    mods = [prop, P.MaxTrajectoryLength(max_length, record=False)]
    if observer_radius is not None:
        mods.append(P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), observer_radius, True, record))
    return P.ChainSpec([P.GridField(grid, origin, (spacing,) * 3, reflective=reflective)], mods,
                       precision=precision)


def bp_fixed(step):
    return P.Propagation(_abi.PROP_BP, 0.42, step, step)


def ck(tol, min_step, max_step):
    return P.Propagation(_abi.PROP_CK, tol, min_step, max_step)


def rel_pos_err(a: CandidateArrays, b: CandidateArrays):
    pa, pb = a.position(), b.position()
    return np.linalg.norm(pa - pb, axis=1) / np.maximum(np.linalg.norm(pb, axis=1), 1e-300)


def stabilize_directions(c):
    """Replace the candidates' directions by a fixed point of setDirection's
    normalisation (normalised again until it no longer changes), so that the
    reference's Candidate constructor, which normalises, starts from the same
    bits as the device.  Returns the mask of candidates that reached a fixed
    point (the others keep their last iterate)."""
    d = c.direction()
    for _ in range(8):
        d2 = normalize(d)
        if np.array_equal(d2, d):
            break
        d = d2
    c.set_direction(d)
    return np.all(normalize(d) == d, axis=1)
