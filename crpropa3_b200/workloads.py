"""The stepping workloads the engine is measured on, with their sizes.

grid_bp_256:  fixed-step PropagationBP (1 kpc) over a Kolmogorov Grid3f of
              256^3 float32 cells (201 MB) at 5 kpc spacing, periodic,
              Brms 10 nG, lMin 10 kpc, lMax 500 kpc, grid seed 42; 10^6
              protons from the origin, isotropic, energies log-uniform
              1-100 EeV; MaximumTrajectoryLength 5 Mpc (5000 steps).
grid_ck_64:   PropagationCK (tolerance 1e-4, 0.1-10 kpc) over a 64^3
              Kolmogorov grid at 10 kpc (Brms 1 nG, lMin 20 kpc, lMax
              200 kpc, seed 42); 10^4 protons; MaximumTrajectoryLength 10 Mpc.
grid_bp_backtrack_128: fixed-step PropagationBP (1 kpc, 2000 steps) of
              antiprotons, log-uniform 5-50 EeV, isotropic, from the origin,
              through a 128^3 Kolmogorov Grid3f at 10 kpc (Brms 3 nG, lMin
              20 kpc, lMax 1280 kpc, seed 42): the forward pass of the
              adjoint workload.
grid_ck_nuclei: PropagationCK (1e-4, 0.1-100 kpc) over the 256^3 grid with
              H, He-4, N-14, Fe-56 in equal parts, E^-2 over 0.1-100 EeV and a
              per-candidate maximum length uniform in 1-50 Mpc.
jf12_backtrack: PropagationCK (1e-4, 0.1 pc-100 pc) in the JF12 regular
              field (JF12Field defaults); antiprotons log-uniform 5-100 EeV
              leaving the Earth's position (-8.5 kpc, 0, 0) isotropically,
              detected by an Observer sphere of 20 kpc around the galactic
              centre, MaximumTrajectoryLength 100 kpc (backtracking).
uf23_backtrack: the same in the UF23Field base model.
pt11_backtrack: the same in PT11Field (ASS disk and halo).
Inputs are synthetic and seeded; sizes are scaled down through `n`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, plan as P, units as U
from .state import CandidateArrays
from .turbulence import grid_turbulence

IDS = {"H": 1000010010, "He": 1000020040, "N": 1000070140, "Fe": 1000260560}


def charge_of(pid: int) -> float:
    lib = _abi.load()
    q = C.c_double()
    _abi.check(lib.crp_particle_charge(int(pid), C.byref(q)))
    return q.value


def source_candidates(n, ids, emin, emax, index, seed, position=(0.0, 0.0, 0.0),
                      abundances=None, per_candidate_length=False,
                      fixed_point=False) -> CandidateArrays:
    """Candidates from a Source(SourcePosition, particle type(s),
    SourcePowerLawSpectrum, SourceIsotropicEmission) via crp_source_sample;
    with fixed_point, directions moved to fixed points of the reference's
    normalisation (fixed_point_directions), as the workloads use them."""
    lib = _abi.load()
    ids = np.asarray(ids, dtype=np.int32)
    ab = np.ones(len(ids)) if abundances is None else np.asarray(abundances, dtype=np.float64)
    d = _abi.SourceDesc()
    d.n_types = len(ids)
    d.spectrum = 1
    d.ids = ids.ctypes.data_as(C.POINTER(C.c_int32))
    d.abundances = ab.ctypes.data_as(C.POINTER(C.c_double))
    d.emin, d.emax, d.index = emin, emax, index
    d.isotropic = 1
    c = CandidateArrays(n, per_candidate_length=per_candidate_length)
    dirs = np.zeros(3 * n)
    _abi.check(lib.crp_source_sample(C.byref(d), seed, n,
                                     c.id.ctypes.data_as(C.POINTER(C.c_int32)),
                                     c.energy.ctypes.data_as(C.POINTER(C.c_double)),
                                     dirs.ctypes.data_as(C.POINTER(C.c_double))))
    d = dirs.reshape(3, n).T
    c.set_direction(fixed_point_directions(d) if fixed_point else d)
    c.set_position(np.tile(np.asarray(position, dtype=np.float64), (n, 1)))
    qs = {int(p): charge_of(int(p)) for p in np.unique(c.id)}
    c.charge[:] = np.vectorize(lambda p: qs[int(p)])(c.id) if n else 0
    return c


def source_candidates_device(n, ids, emin, emax, index, seed, position=(0.0, 0.0, 0.0),
                             abundances=None, first=0, device="cuda") -> CandidateArrays:
    """The candidates of source_candidates drawn on the device
    (crp_source_sample_device): the same features and distributions from a
    counter-based Philox stream, so candidate first + i is the same whichever
    call or rank draws it.  Nothing crosses from the host but the source's
    parameters."""
    import torch
    lib = _abi.load()
    ids = np.asarray(ids, dtype=np.int32)
    ab = np.ones(len(ids)) if abundances is None else np.asarray(abundances, dtype=np.float64)
    d = _abi.SourceDesc()
    d.n_types = len(ids)
    d.spectrum = 1
    d.ids = ids.ctypes.data_as(C.POINTER(C.c_int32))
    d.abundances = ab.ctypes.data_as(C.POINTER(C.c_double))
    d.emin, d.emax, d.index = emin, emax, index
    d.isotropic = 1
    c = CandidateArrays(n, device=device)
    if n == 0:
        return c
    dirs = torch.empty(3 * n, dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(c.id.device).cuda_stream
    _abi.check(lib.crp_source_sample_device(C.byref(d), int(seed), int(first), int(n), c.id.data_ptr(),
                                            c.energy.data_ptr(), dirs.data_ptr(), stream))
    c.dx.copy_(dirs[:n])
    c.dy.copy_(dirs[n:2 * n])
    c.dz.copy_(dirs[2 * n:])
    for k, v in enumerate(np.asarray(position, dtype=np.float64)):
        for name in (("x", "px"), ("y", "py"), ("z", "pz"))[k]:
            getattr(c, name).fill_(float(v))
    for p in np.unique(ids):
        c.charge.masked_fill_(c.id == int(p), charge_of(int(p)))
    c.active.fill_(1)
    return c


def _normalise(d):
    r = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    return d / r[:, None]


def fixed_point_directions(d):
    """Directions that ParticleState::setDirection (ParticleState.cpp:30,
    d / |d|) maps to themselves bit for bit: the reference's Candidate
    constructor normalises the direction it is given, so a Candidate built
    from these arrays holds exactly the bits the device starts from.  d is
    normalised again until it no longer changes; the few that cycle instead
    get their components moved by single ulps until a fixed point is found.
    Every change is a few ulp per component."""
    d = np.array(d, dtype=np.float64)
    for _ in range(8):
        d2 = _normalise(d)
        if np.array_equal(d2, d):
            break
        d = d2
    bad = np.flatnonzero(~np.all(_normalise(d) == d, axis=1))
    for k in range(1, 5):
        if not len(bad):
            break
        for j in range(3):
            for sign in (np.inf, -np.inf):
                if not len(bad):
                    break
                t = d[bad].copy()
                for _ in range(k):
                    t[:, j] = np.nextafter(t[:, j], sign)
                ok = np.all(_normalise(t) == t, axis=1)
                d[bad[ok]] = t[ok]
                bad = bad[~ok]
    return d


def kolmogorov_grid(n, spacing, brms, lmin, lmax, seed=42, device=None):
    """GridTurbulence(TurbulenceSpectrum(brms, lmin, lmax), GridProperties(0, n,
    spacing), seed) with the spectrum's defaults (sIndex 5/3, qIndex 4,
    lBendover 1 m), as the reference builds it from these arguments."""
    return grid_turbulence(n, spacing, brms, lmin, lmax, seed=seed, device=device)


def grid_bp_256(n=1_000_000, grid_n=256, steps=5000, precision=_abi.PRECISION_MIXED, grid=None,
                device=None, seed=1):
    spacing = 5 * U.kpc
    if grid is None:
        grid = kolmogorov_grid(grid_n, spacing, 10 * U.nG, 10 * U.kpc, 500 * U.kpc, 42, device)
    spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (spacing,) * 3)],
                       [P.Propagation(_abi.PROP_BP, 0.42, 1 * U.kpc, 1 * U.kpc),
                        P.MaxTrajectoryLength(steps * U.kpc)], precision=precision)
    cands = source_candidates(n, [IDS["H"]], 1 * U.EeV, 100 * U.EeV, -1.0, seed, fixed_point=True)
    return spec, cands, grid


def grid_bp_backtrack_128(n=100_000, steps=2000, precision=_abi.PRECISION_FP64, grid=None,
                          device=None, seed=4):
    spacing = 10 * U.kpc
    if grid is None:
        grid = kolmogorov_grid(128, spacing, 3 * U.nG, 20 * U.kpc, 1280 * U.kpc, 42, device)
    spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (spacing,) * 3)],
                       [P.Propagation(_abi.PROP_BP, 0.42, 1 * U.kpc, 1 * U.kpc),
                        P.MaxTrajectoryLength(steps * U.kpc)], precision=precision)
    cands = source_candidates(n, [-IDS["H"]], 5 * U.EeV, 50 * U.EeV, -1.0, seed, fixed_point=True)
    return spec, cands, grid


def grid_ck_64(n=10_000, precision=_abi.PRECISION_FP64, grid=None, device=None, seed=1):
    spacing = 10 * U.kpc
    if grid is None:
        grid = kolmogorov_grid(64, spacing, 1 * U.nG, 20 * U.kpc, 200 * U.kpc, 42, device)
    spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (spacing,) * 3)],
                       [P.Propagation(_abi.PROP_CK, 1e-4, 0.1 * U.kpc, 10 * U.kpc),
                        P.MaxTrajectoryLength(10 * U.Mpc)], precision=precision)
    cands = source_candidates(n, [IDS["H"]], 1 * U.EeV, 100 * U.EeV, -1.0, seed, fixed_point=True)
    return spec, cands, grid


def grid_ck_nuclei(n=10_000_000, grid=None, precision=_abi.PRECISION_MIXED, device=None, seed=3,
                   grid_n=256):
    spacing = 5 * U.kpc
    if grid is None:
        grid = kolmogorov_grid(grid_n, spacing, 10 * U.nG, 10 * U.kpc, 500 * U.kpc, 42, device)
    spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (spacing,) * 3)],
                       [P.Propagation(_abi.PROP_CK, 1e-4, 0.1 * U.kpc, 100 * U.kpc),
                        P.MaxTrajectoryLength(per_candidate=True)], precision=precision)
    cands = source_candidates(n, [IDS[k] for k in ("H", "He", "N", "Fe")], 0.1 * U.EeV,
                              100 * U.EeV, -2.0, seed, per_candidate_length=True, fixed_point=True)
    rng = np.random.default_rng(seed)
    cands.max_length[:] = rng.uniform(1, 50, n) * U.Mpc
    return spec, cands, grid


def plane_wave_modes(brms, lmin, lmax, lbendover, sindex, qindex, n_modes, seed):
    """Wave modes of PlaneWaveTurbulence(TurbulenceSpectrum(...), n_modes, seed)
    (PlaneWaveTurbulence.cpp:79) via crp_plane_wave_modes: xi, kappa (n, 3),
    k, beta, Ak (n,)."""
    lib = _abi.load()
    xi, kappa = np.zeros(3 * n_modes), np.zeros(3 * n_modes)
    k, beta, ak = np.zeros(n_modes), np.zeros(n_modes), np.zeros(n_modes)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    _abi.check(lib.crp_plane_wave_modes(brms, lmin, lmax, lbendover, sindex, qindex, n_modes, seed,
                                        dp(xi), dp(kappa), dp(k), dp(beta), dp(ak)))
    return xi.reshape(n_modes, 3), kappa.reshape(n_modes, 3), k, beta, ak


def sde_galactic(n=10_000_000, n_modes=1024, precision=_abi.PRECISION_MIXED, seed=5,
                 source=(8.5 * U.kpc, 0.0, 0.0)):
    """DiffusionSDE (tolerance 1e-4, steps 0.1-100 pc, epsilon 0.1, alpha 1/3,
    scale 1) in B = 1 muG (-y, x, 0)/r plus PlaneWaveTurbulence (n_modes
    modes, Brms 0.5 muG, lMin 1 pc, lMax 100 pc, lBendover 1 pc, Kolmogorov,
    mode seed 11); protons log-uniform 1 TeV - 1 PeV from `source`, absorbed
    by an Observer sphere of 20 kpc around the origin."""
    spectrum = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1 * U.pc, 5.0 / 3.0, 4.0)
    xi, kappa, k, beta, ak = plane_wave_modes(*spectrum, n_modes, 11)
    fields = [P.ToroidalField(1 * U.muG),
              P.PlaneWaveField(xi, kappa, k, beta, ak, spectrum=spectrum, seed=11)]
    spec = P.ChainSpec(fields,
                       [P.Propagation(_abi.PROP_SDE, 1e-4, 0.1 * U.pc, 100 * U.pc, epsilon=0.1,
                                      alpha=1.0 / 3.0, scale=1.0),
                        P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0.0, 0.0, 0.0), 20 * U.kpc,
                                       True, False)],
                       precision=precision, seed=seed)
    cands = source_candidates(n, [IDS["H"]], 1 * U.TeV, 1000 * U.TeV, -1.0, seed, position=source,
                              fixed_point=True)
    return spec, cands


def jf12_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7, variant=_abi.JF12_VARIANT_JF12,
                   field=None):
    """Backtracking through the JF12 regular field (module docstring); `field`
    replaces the JF12Field (uf23_backtrack passes a UF23Field)."""
    spec = P.ChainSpec([field if field is not None else P.JF12Field(variant=variant)],
                       [P.Propagation(_abi.PROP_CK, 1e-4, 0.1 * U.pc, 100 * U.pc),
                        P.MaxTrajectoryLength(100 * U.kpc, record=False),
                        P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0.0, 0.0, 0.0), 20 * U.kpc,
                                       True, False)],
                       precision=precision, seed=seed)
    cands = source_candidates(n, [-IDS["H"]], 5 * U.EeV, 100 * U.EeV, -1.0, seed,
                              position=(-8.5 * U.kpc, 0.0, 0.0), fixed_point=True)
    return spec, cands


def uf23_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7, model=_abi.UF23_BASE):
    """jf12_backtrack with the UF23Field model `model` instead of JF12."""
    return jf12_backtrack(n, precision, seed, field=P.UF23Field(model))


def pt11_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7):
    """jf12_backtrack with PT11Field() (ASS disk and halo) instead of JF12."""
    return jf12_backtrack(n, precision, seed, field=P.PT11Field())


def tf17_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7):
    """jf12_backtrack with TF17Field() (disk Ad1, halo C1) instead of JF12."""
    return jf12_backtrack(n, precision, seed, field=P.TF17Field())


def kst24_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7):
    """jf12_backtrack with KST24Field() instead of JF12."""
    return jf12_backtrack(n, precision, seed, field=P.KST24Field())


def jf12_solenoidal_backtrack(n=1_000_000, precision=_abi.PRECISION_MIXED, seed=7):
    """jf12_backtrack with JF12FieldSolenoidal() (regular field) instead of JF12Field."""
    return jf12_backtrack(n, precision, seed, variant=_abi.JF12_VARIANT_SOLENOIDAL)
