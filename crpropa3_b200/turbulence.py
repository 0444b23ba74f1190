"""Turbulent Grid3f set-up: GridTurbulence (GridTurbulence.cpp:29-123).

The k-space field is drawn exactly as GridTurbulence::initTurbulence does:
loop over ix, iy, iz (iz over n/2+1 values) with the discrete wave numbers
K[i] = i/n - i/(n/2) in float, keep modes with kMin <= |k| <= kMax, and for
each kept mode draw theta then phase from one crpropa::Random(seed) stream
(the engine's MT19937, crp_random_draws); the amplitude is
sqrt(energySpectrum(|k| 2 pi / spacing)) along e1 cos(theta) + e2 sin(theta)
with the (1,1,1) construction of the orthogonal base.  The inverse real FFT
then runs on the device (torch.fft / cuFFT) when one is present, else on the
host, and the grid is rescaled to Brms (scaleGrid / rmsFieldStrength,
GridTools.cpp:16, :59).  FFTW is not part of this image, so the FFT is not
the reference's: grid values are equal to the reference's only in
distribution (zero mean, rms = Brms, the spectrum), not bit for bit.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi


def energy_spectrum(k, brms, lmin, lmax, lbendover=1.0, sindex=5.0 / 3.0, qindex=4.0):
    """TurbulenceSpectrum::energySpectrum (TurbulentField.h:75), not normalised."""
    kh = k * lbendover
    return kh ** qindex / (1.0 + kh * kh) ** ((sindex + qindex) / 2.0 + 1.0)


def check_grid_requirements(n, spacing, lmin, lmax):
    """GridTurbulence::checkGridRequirements (GridTurbulence.cpp:126)."""
    if lmin < 2 * spacing:
        raise RuntimeError("turbulentField: lMin < 2 * spacing")
    if lmax > n * spacing:
        raise RuntimeError("turbulentField: lMax > size")
    if lmax < lmin:
        raise RuntimeError("lMax < lMin")


def _mt_rand(seed: int, count: int) -> np.ndarray:
    lib = _abi.load()
    out = np.zeros(count)
    _abi.check(lib.crp_random_draws(seed, 0, count, 0.0, 0.0, 0.0,
                                    out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def kspace(n, spacing, brms, lmin, lmax, lbendover=1.0, sindex=5.0 / 3.0, qindex=4.0, seed=42,
           draws=None, kind=None, helicity=0.0):
    """The three complex (n, n, n/2+1) arrays B(k) of initTurbulence.
    `draws(seed, count)` returns count Random::rand() values (default: the
    engine's MT19937).  kind TURBULENCE_SIMPLE builds SimpleGridTurbulence's
    instead (SimpleGridTurbulence.cpp:62-95): amplitude randNorm() k^(alpha/2)
    with alpha = -sindex - 2, draws rand, randNorm, rand per mode;
    TURBULENCE_HELICAL HelicalGridTurbulence's (HelicalGridTurbulence.cpp:
    60-116): two helical components of amplitudes mu0 / (4 pi k^3)
    sqrt((1 +- H) / 2) |randNorm() k^(alpha/2)| and phases 2 pi rand."""
    if seed == 0:
        raise ValueError("seed 0 means a random seed in the reference; give a non-zero seed")
    check_grid_requirements(n, spacing, lmin, lmax)
    n2 = n // 2 + 1
    i = np.arange(n)
    K = (i / n - (i // (n // 2))).astype(np.float32)
    ex, ey, ez = np.meshgrid(K, K, K[:n2], indexing="ij")
    k = np.sqrt(ex * ex + ey * ey + ez * ez).astype(np.float32)
    kmin, kmax = spacing / lmax, spacing / lmin
    keep = ~((k.astype(np.float64) < kmin) | (k.astype(np.float64) > kmax))
    m = int(keep.sum())
    simple = kind == _abi.TURBULENCE_SIMPLE
    helical = kind == _abi.TURBULENCE_HELICAL
    if helical:
        d = turbulence_draws(seed, _abi.TURBULENCE_HELICAL, m)
    elif simple:
        d = turbulence_draws(seed, _abi.TURBULENCE_SIMPLE, m)
        theta, norm, phase = 2 * math.pi * d[:, 0], d[:, 1], 2 * math.pi * d[:, 2]
    else:
        u = (draws or _mt_rand)(seed, 2 * m)
        theta = 2 * math.pi * u[0::2]
        phase = 2 * math.pi * u[1::2]
    kx, ky, kz, kk = ex[keep], ey[keep], ez[keep], k[keep]
    one = np.float32(1.0)
    # e1 = n0 x ek, e2 = ek x e1 with n0 = (1, 1, 1), in float (Vector3f)
    e1 = np.stack([one * kz - ky * one, one * kx - kz * one, one * ky - kx * one], 1).astype(np.float32)
    e2 = np.stack([ky * e1[:, 2] - e1[:, 1] * kz, kz * e1[:, 0] - e1[:, 2] * kx,
                   kx * e1[:, 1] - e1[:, 0] * ky], 1).astype(np.float32)
    # ek parallel to (1,1,1) within 1e-3 rad: fixed base (GridTurbulence.cpp:79)
    with np.errstate(invalid="ignore", divide="ignore"):
        cosd = ((kx + ky + kz) / np.sqrt(np.float32(3)) / kk).astype(np.float32)
        ang = np.where(cosd >= 1, 0, np.arccos(np.clip(cosd, -1, 1)))
    par = ang < (1e-3 if helical else np.float32(1e-3))
    e1[par] = np.array([-1, 1, 0], np.float32)
    e2[par] = np.array([1, 1, -2], np.float32)
    e1 /= np.sqrt((e1 * e1).sum(1))[:, None].astype(np.float32)
    e2 /= np.sqrt((e2 * e2).sum(1))[:, None].astype(np.float32)
    if helical:
        k64 = kk.astype(np.float64)
        mu0 = 4 * math.pi * 1e-7
        pre = mu0 / (4 * math.pi * k64 ** 3)
        tot = np.abs(d[:, 0] * np.power(k64, (-sindex - 2) / 2))
        bp = pre * math.sqrt((1 + helicity) / 2) * tot
        bm = pre * math.sqrt((1 - helicity) / 2) * tot
        tp, tm = 2 * math.pi * d[:, 1], 2 * math.pi * d[:, 2]
        ctp, stp, ctm, stm = np.cos(tp), np.sin(tp), np.cos(tm), np.sin(tm)
        re1, re2 = bp * ctp + bm * ctm, -bp * stp + bm * stm
        im1, im2 = bp * stp + bm * stm, bp * ctp - bm * ctm
        s2 = math.sqrt(2.)
        out = []
        for a in range(3):
            arr = np.zeros((n, n, n2), dtype=np.complex64)
            e1a, e2a = e1[:, a].astype(np.float64), e2[:, a].astype(np.float64)
            arr[keep] = (((re1 * e1a + re2 * e2a) / s2).astype(np.float32) +
                         1j * ((im1 * e1a + im2 * e2a) / s2).astype(np.float32))
            out.append(arr)
        return out
    b = (e1 * np.cos(theta).astype(np.float32)[:, None] +
         e2 * np.sin(theta).astype(np.float32)[:, None]).astype(np.float32)
    if simple:
        amp = (norm * np.power(kk.astype(np.float64), (-sindex - 2) / 2)).astype(np.float32)
    else:
        lam = 1 / spacing * 2 * math.pi
        amp = np.sqrt(energy_spectrum(kk.astype(np.float64) * lam, brms, lmin, lmax, lbendover, sindex,
                                      qindex)).astype(np.float32)
    b *= amp[:, None]
    cph, sph = np.cos(phase), np.sin(phase)
    out = []
    for a in range(3):
        arr = np.zeros((n, n, n2), dtype=np.complex64)
        arr[keep] = (b[:, a] * cph).astype(np.float32) + 1j * (b[:, a] * sph).astype(np.float32)
        out.append(arr)
    return out


def grid_turbulence(n, spacing, brms, lmin, lmax, lbendover=1.0, sindex=5.0 / 3.0, qindex=4.0,
                    seed=42, device=None, draws=None, kind=None, helicity=0.0) -> np.ndarray:
    """(n, n, n, 3) float32 Grid3f values of GridTurbulence(spectrum, grid,
    seed), or of SimpleGridTurbulence (kind TURBULENCE_SIMPLE) or
    HelicalGridTurbulence (kind TURBULENCE_HELICAL, helicity H)."""
    bk = kspace(n, spacing, brms, lmin, lmax, lbendover, sindex, qindex, seed, draws, kind, helicity)
    comps = []
    use_torch = False
    if device is not None:
        import torch
        use_torch = torch.cuda.is_available()
    for arr in bk:
        if use_torch:
            import torch
            t = torch.from_numpy(arr).to(device)
            comps.append(torch.fft.irfftn(t, s=(n, n, n), dim=(0, 1, 2)).cpu().numpy().astype(np.float32))
        else:
            comps.append(np.fft.irfftn(arr, s=(n, n, n), axes=(0, 1, 2)).astype(np.float32))
    g = np.stack(comps, axis=-1).astype(np.float32)
    g64 = g.astype(np.float64)
    rms = math.sqrt(float((g64 * g64).sum()) / (n * n * n))
    g *= np.float32(brms / rms)
    return g


def grid_turbulence_with_draws(n, spacing, brms, lmin, lmax, seed, draws):
    """grid_turbulence with the MT19937 draws supplied by the caller (host FFT)."""
    return grid_turbulence(n, spacing, brms, lmin, lmax, seed=seed, draws=draws)


def turbulence_desc(kind, n, spacing, brms, lmin, lmax, lbendover=1.0, sindex=5.0 / 3.0, qindex=4.0,
                    seed=42, helicity=0.0) -> "_abi.TurbulenceDesc":
    d = _abi.TurbulenceDesc()
    d.kind, d.seed, d.n, d.spacing = int(kind), int(seed), int(n), float(spacing)
    d.brms, d.lmin, d.lmax = float(brms), float(lmin), float(lmax)
    d.lbendover, d.sindex, d.qindex, d.helicity = float(lbendover), float(sindex), float(qindex), float(helicity)
    return d


def turbulence_modes(desc) -> int:
    """Number of modes the k-space loop keeps (crp_turbulence_modes)."""
    m = C.c_uint64()
    _abi.check(_abi.load().crp_turbulence_modes(C.byref(desc), C.byref(m)))
    return m.value


def turbulence_draws(seed, kind, n_modes) -> np.ndarray:
    """The k-space loop's Random draws (crp_turbulence_draws), (n_modes, 2 or 3)."""
    per = 2 if kind == _abi.TURBULENCE_GRID else 3
    out = np.zeros(per * n_modes)
    _abi.check(_abi.load().crp_turbulence_draws(int(seed), int(kind), int(n_modes),
                                                out.ctypes.data_as(C.POINTER(C.c_double))))
    return out.reshape(n_modes, per)


def grid_turbulence_device(kind, n, spacing, brms, lmin, lmax, lbendover=1.0, sindex=5.0 / 3.0, qindex=4.0,
                           seed=42, helicity=0.0, device="cuda"):
    """GridTurbulence (kind TURBULENCE_GRID), SimpleGridTurbulence
    (TURBULENCE_SIMPLE) or HelicalGridTurbulence (TURBULENCE_HELICAL)
    generated on the device (crp_turbulence_grid): a (n, n, n, 3) float32
    torch tensor of Grid3f values in device memory, ready for a GridField."""
    import torch
    out = torch.empty((n, n, n, 3), dtype=torch.float32, device=device)
    d = turbulence_desc(kind, n, spacing, brms, lmin, lmax, lbendover, sindex, qindex, seed, helicity)
    stream = torch.cuda.current_stream(out.device).cuda_stream
    _abi.check(_abi.load().crp_turbulence_grid(C.byref(d), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out
