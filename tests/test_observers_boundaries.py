"""Observer features and boundary conditions beyond the sphere observer:
ObserverSurface over Plane and ParaxialBox, ObserverTracking, Observer1D,
the particle vetoes (inactive, nucleus, neutrino, photon, electron, by id),
observers combining features (Observer.cpp:27-52), and SphericalBoundary,
CubicBoundary, EllipsoidalBoundary, CylindricalBoundary (Boundary.cpp:171-320).

CPU: the oracle against the reference's own modules, bit for bit.  GPU: the
device FP64 form against the oracle built with the correctly rounded pow (the
cylindrical boundary's pow(v, 2) and pow(v, 0.5) are v*v and sqrt(v) on the
device), bit for bit, records included; the mixed form runs the same chains.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays, RecordArrays

F = P.Feature
KPC = U.kpc

# name -> list of non-propagation modules after [BP, MaxTrajectoryLength]
CHAINS = {
    "plane": [P.ObserverSpec(features=[F(_abi.OBSERVER_SURFACE_PLANE, a=(10 * KPC, 0, 0), b=(1, 0, 0))],
                             record=True)],
    "oblique_plane": [P.ObserverSpec(features=[F(_abi.OBSERVER_SURFACE_PLANE, a=(0, 5 * KPC, 0), b=(0.6, 0.8, 0))],
                                     deactivate=False, record=True)],
    "box": [P.ObserverSpec(features=[F(_abi.OBSERVER_SURFACE_BOX, a=(-30 * KPC,) * 3, b=(60 * KPC, 50 * KPC, 40 * KPC))],
                           record=True)],
    "tracking": [P.ObserverSpec(features=[F(_abi.OBSERVER_TRACKING, a=(0, 0, 0), r=25 * KPC, step=2 * KPC)],
                                deactivate=False, record=True)],
    "observer1d": [P.ObserverSpec(features=[F(_abi.OBSERVER_1D)], record=True)],
    "vetoes": [P.ObserverSpec(features=[F(_abi.OBSERVER_SURFACE_SPHERE, a=(0, 0, 0), r=20 * KPC),
                                        F(_abi.OBSERVER_ELECTRON_VETO), F(_abi.OBSERVER_PARTICLE_ID_VETO,
                                                                          particle_id=1000020040),
                                        F(_abi.OBSERVER_NEUTRINO_VETO)], record=True),
               P.ObserverSpec(features=[F(_abi.OBSERVER_DETECT_ALL), F(_abi.OBSERVER_NUCLEUS_VETO),
                                        F(_abi.OBSERVER_PHOTON_VETO), F(_abi.OBSERVER_INACTIVE_VETO)],
                              deactivate=False, record=True)],
    "spherical": [P.BoundarySpec(_abi.BOUNDARY_SPHERICAL, a=(5 * KPC, 0, 0), size=40 * KPC, record=True)],
    "cubic": [P.BoundarySpec(_abi.BOUNDARY_CUBIC, a=(-35 * KPC,) * 3, size=70 * KPC, record=True)],
    "ellipsoidal": [P.BoundarySpec(_abi.BOUNDARY_ELLIPSOIDAL, a=(-20 * KPC, 0, 0), b=(20 * KPC, 0, 0),
                                   size=90 * KPC, record=True)],
    "cylindrical": [P.BoundarySpec(_abi.BOUNDARY_CYLINDRICAL, a=(0, 0, 0), size=60 * KPC, radius=30 * KPC,
                                   margin=0.0, limit_step=True, record=True)],
    "cylindrical_nolimit": [P.BoundarySpec(_abi.BOUNDARY_CYLINDRICAL, a=(0, 0, 0), size=60 * KPC,
                                           radius=30 * KPC, margin=0.0, limit_step=False, record=True)],
    "boundary_and_observer": [P.BoundarySpec(_abi.BOUNDARY_SPHERICAL, a=(0, 0, 0), size=45 * KPC,
                                             margin=0.5 * KPC, record=True),
                              P.ObserverSpec(features=[F(_abi.OBSERVER_SURFACE_PLANE, a=(0, 0, 0), b=(0, 0, 1))],
                                             deactivate=False, record=True)],
}

SPECIES = np.array([1000010010, 1000020040, 11, -11, 22, 12, 1000260560, 2112], np.int32)


def _spec(name, precision=_abi.PRECISION_FP64):
    grid = random_grid(np.random.default_rng(71), 16, brms=3e-13)
    mods = [bp_fixed(0.5 * KPC), P.MaxTrajectoryLength(150 * KPC, record=True)] + CHAINS[name]
    return P.ChainSpec([P.GridField(grid, (-80 * KPC,) * 3, (10 * KPC,) * 3)], mods, precision=precision)


def _cands(n=400, seed=72):
    from crpropa3_b200.workloads import charge_of
    rng = np.random.default_rng(seed)
    c = CandidateArrays(n)
    c.id[:] = SPECIES[rng.integers(0, len(SPECIES), n)]
    c.charge[:] = [charge_of(int(i)) for i in c.id]
    c.energy[:] = np.exp(rng.uniform(np.log(1), np.log(100), n)) * U.EeV
    pos = rng.uniform(-25, 25, (n, 3)) * KPC
    c.set_position(pos)
    c.px[:], c.py[:], c.pz[:] = pos[:, 0], pos[:, 1], pos[:, 2]
    c.set_direction(stable_unit_vectors(rng, n))
    c.next_step[:] = 1e30
    return c


STATE = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time", "next_step",
         "active", "flags")


def _compare(a, b, ra=None, rb=None):
    for m in STATE:
        np.testing.assert_array_equal(getattr(a, m), getattr(b, m), err_msg=m)
    if ra is not None:
        assert ra.n() == rb.n()
        sa, sb = ra.sorted(), rb.sorted()
        # same records; order within a candidate and module is time order
        ka = np.lexsort((sa["trajectory_length"], sa["module"], sa["index"]))
        kb = np.lexsort((sb["trajectory_length"], sb["module"], sb["index"]))
        for k in sa:
            np.testing.assert_array_equal(np.asarray(sa[k])[ka], np.asarray(sb[k])[kb], err_msg=k)


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_oracle_matches_reference(oracle, reference, name):
    spec = _spec(name)
    c = _cands()
    a, b = c.copy(), c.copy()
    ra, rb = RecordArrays(200_000), RecordArrays(200_000)
    reference.run(spec, a, ra, threads=1)
    oracle.run(spec, b, rb)
    _compare(a, b, ra, rb)
    flags = a.flags
    if name == "vetoes":
        assert (flags & _abi.FLAG_DETECTED).any() and not (flags & _abi.FLAG_DETECTED).all()
    elif name.startswith(("spherical", "cubic", "ellipsoidal", "cylindrical")):
        assert ((flags & _abi.FLAG_REJECTED) != 0).sum() > 10
    else:
        assert (flags & _abi.FLAG_DETECTED).any()


def test_more_than_four_features_refused():
    from crpropa3_b200.engine import Plan
    spec = _spec("plane")
    spec.modules[-1] = P.ObserverSpec(features=[F(_abi.OBSERVER_DETECT_ALL)] * 5)
    with pytest.raises(ValueError):
        spec.desc()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CHAINS))
def test_device_fp64_matches_oracle(oracle_crpow, name):
    from crpropa3_b200.engine import Plan
    spec = _spec(name)
    c = _cands()
    a = c.copy()
    ra = RecordArrays(200_000)
    oracle_crpow.run(spec, a, ra)
    d = c.to_device("cuda")
    rd = RecordArrays(200_000, device="cuda")
    Plan(spec).run(d, records=rd)
    _compare(a, d.to_host(), ra, rd.to_host())


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vetoes", "boundary_and_observer", "box"])
def test_device_mixed_runs_the_same_chains(oracle_crpow, name):
    """Mixed form: the same detections and rejections for all but a few
    candidates (FP32 rotation moves trajectories at the 1e-7 level, which can
    move a crossing across a step boundary)."""
    from crpropa3_b200.engine import Plan
    c = _cands()
    a = c.copy()
    oracle_crpow.run(_spec(name), a)
    d = c.to_device("cuda")
    Plan(_spec(name, _abi.PRECISION_MIXED)).run(d)
    h = d.to_host()
    assert np.mean(h.flags == a.flags) >= 0.97
    assert np.mean(h.active == a.active) >= 0.97
