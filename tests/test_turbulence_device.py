"""Turbulent Grid3f generation on the device (crp_turbulence_grid):
GridTurbulence (GridTurbulence.cpp:29-123), SimpleGridTurbulence
(SimpleGridTurbulence.cpp:19-115) and HelicalGridTurbulence
(HelicalGridTurbulence.cpp:19-127).

CPU: the k-space draw sequences against the reference's crpropa::Random
(rand and randNorm interleaved as each loop draws them), bit for bit; the
number of kept modes against the restated k-space mask.  FFTW is absent, so
the reference's grids cannot be produced here; on the GPU the device grid
of GridTurbulence and SimpleGridTurbulence is compared with this package's
host restatement (identical k-space construction and draws, another FFT)
within 1e-4 of Brms, and every kind is checked for rms = Brms, zero mean, a divergence-free
spectrum and, for the helical kind, the sign of the magnetic helicity.
"""
import numpy as np
import pytest

from helpers import _abi
from crpropa3_b200 import turbulence as T

N, SPACING = 32, 1.0
LMIN, LMAX, BRMS = 4.0, 32.0, 1e-10  # kMax = 1/4: no Nyquist-plane modes

KINDS = {"grid": _abi.TURBULENCE_GRID, "simple": _abi.TURBULENCE_SIMPLE, "helical": _abi.TURBULENCE_HELICAL}


@pytest.mark.parametrize("kind", sorted(KINDS))
def test_draw_sequences_match_reference(reference, kind):
    k = KINDS[kind]
    np.testing.assert_array_equal(T.turbulence_draws(1234, k, 5000), reference.turbulence_draws(1234, k, 5000))


def test_randnorm_draws_match_reference(reference):
    import ctypes as C
    out = np.zeros(2000)
    _abi.check(_abi.load().crp_random_draws(77, 4, 2000, 0.0, 0.0, 0.0, out.ctypes.data_as(C.POINTER(C.c_double))))
    np.testing.assert_array_equal(out, reference.random(77, 4, 2000))


def test_mode_count_matches_restated_mask():
    d = T.turbulence_desc(_abi.TURBULENCE_GRID, N, SPACING, BRMS, LMIN, LMAX)
    n2 = N // 2 + 1
    i = np.arange(N)
    K = (i / N - (i // (N // 2))).astype(np.float32)
    ex, ey, ez = np.meshgrid(K, K, K[:n2], indexing="ij")
    k = np.sqrt(ex * ex + ey * ey + ez * ez).astype(np.float32).astype(np.float64)
    keep = ~((k < SPACING / LMAX) | (k > SPACING / LMIN))
    assert T.turbulence_modes(d) == int(keep.sum()) > 1000


def test_bad_descriptors_refused():
    import ctypes as C
    m = C.c_uint64()
    for kw in ({"lmin": 1.0}, {"lmax": 64.0}, {"kind": 7}):
        args = dict(kind=_abi.TURBULENCE_GRID, n=N, spacing=SPACING, brms=BRMS, lmin=LMIN, lmax=LMAX)
        args.update(kw)
        d = T.turbulence_desc(**args)
        assert _abi.load().crp_turbulence_modes(C.byref(d), C.byref(m)) == _abi.ERR_INVALID_ARGUMENT


# ------------------------------------------------------------------ GPU


def _spectral(g):
    """B(k) of a (n, n, n, 3) grid and the wave vectors."""
    bk = np.fft.fftn(g.astype(np.float64), axes=(0, 1, 2))
    f = np.fft.fftfreq(g.shape[0])
    kx, ky, kz = np.meshgrid(f, f, f, indexing="ij")
    return bk, np.stack([kx, ky, kz], -1)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["grid", "simple", "helical"])
def test_device_turbulence_matches_host_restatement(kind):
    g = T.grid_turbulence_device(KINDS[kind], N, SPACING, BRMS, LMIN, LMAX, seed=42, helicity=0.5).cpu().numpy()
    h = T.grid_turbulence(N, SPACING, BRMS, LMIN, LMAX, seed=42, kind=KINDS[kind], helicity=0.5)
    np.testing.assert_allclose(g, h, rtol=0, atol=1e-4 * BRMS)


def test_host_helical_turbulence_helicity_sign():
    """The host restatement of HelicalGridTurbulence: opposite signs of the
    spectral helicity for H = +1 and H = -1, rms = Brms."""
    out = []
    for h in (1.0, -1.0):
        g = T.grid_turbulence(N, SPACING, BRMS, LMIN, LMAX, seed=9, kind=_abi.TURBULENCE_HELICAL, helicity=h)
        assert abs(np.sqrt((g.astype(np.float64) ** 2).sum(-1).mean()) / BRMS - 1) < 1e-6
        bk, kv = _spectral(g)
        out.append(float(np.imag((kv * np.cross(np.conj(bk), bk)).sum(-1)).sum()))
    assert out[0] * out[1] < 0


@pytest.mark.gpu
@pytest.mark.parametrize("kind", sorted(KINDS))
def test_device_turbulence_statistics(kind):
    g = T.grid_turbulence_device(KINDS[kind], N, SPACING, BRMS, LMIN, LMAX, seed=7,
                                 helicity=0.5).cpu().numpy().astype(np.float64)
    rms = np.sqrt((g * g).sum(-1).mean())
    assert abs(rms / BRMS - 1) < 1e-6
    assert np.abs(g.mean(axis=(0, 1, 2))).max() < 1e-3 * BRMS
    bk, kv = _spectral(g)
    div = np.abs((bk * kv).sum(-1))
    assert div.max() < 1e-4 * np.abs(bk).max()


@pytest.mark.gpu
def test_device_helical_turbulence_helicity_sign():
    """k . (B(k)* x B(k)) changes sign with H: maximal helicity of either
    hand gives opposite signs of the summed spectral helicity."""
    out = []
    for h in (1.0, -1.0):
        g = T.grid_turbulence_device(_abi.TURBULENCE_HELICAL, N, SPACING, BRMS, LMIN, LMAX, seed=9,
                                     helicity=h).cpu().numpy()
        bk, kv = _spectral(g)
        out.append(float(np.imag((kv * np.cross(np.conj(bk), bk)).sum(-1)).sum()))
    assert out[0] * out[1] < 0
    assert min(abs(out[0]), abs(out[1])) > 0.1 * max(abs(out[0]), abs(out[1]))


@pytest.mark.gpu
def test_device_turbulence_seeds_differ_and_repeat():
    a = T.grid_turbulence_device(_abi.TURBULENCE_SIMPLE, N, SPACING, BRMS, LMIN, LMAX, seed=3).cpu().numpy()
    b = T.grid_turbulence_device(_abi.TURBULENCE_SIMPLE, N, SPACING, BRMS, LMIN, LMAX, seed=3).cpu().numpy()
    c = T.grid_turbulence_device(_abi.TURBULENCE_SIMPLE, N, SPACING, BRMS, LMIN, LMAX, seed=4).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
