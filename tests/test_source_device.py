"""crp_source_sample_device: Source::getCandidate's features
(SourceMultipleParticleTypes, SourcePowerLawSpectrum, SourceIsotropicEmission
or SourceDirection; Source.cpp:22-150, :742, :808) drawn on the device from a
counter-based Philox4x32-10 stream.

The sequence is not the reference's MT19937 one (crp_source_sample keeps
that), so parity is in two parts:
CPU: the oracle's restatement of the counter-based draws against the
reference's own Source sampler, in distribution (two-sample Kolmogorov-
Smirnov on energies, direction cosines and azimuths; chi-square on the
particle types), and split runs (first > 0) equal to one run.
GPU: the device against that restatement draw for draw: ids exactly,
energies within 5e-16 relative (CUDA's pow and exp against glibc's, within
two ulp, on the same rounded argument), direction components within 5e-16.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import U, _abi

IDS = [1000010010, 1000020040, 1000070140, 1000260560]
AB = [0.5, 0.3, 0.15, 0.05]


def _ks_2samp(a, b):
    """Two-sample Kolmogorov-Smirnov statistic and its asymptotic p-value."""
    a, b = np.sort(a), np.sort(b)
    allv = np.concatenate([a, b])
    d = np.max(np.abs(np.searchsorted(a, allv, side="right") / len(a) -
                      np.searchsorted(b, allv, side="right") / len(b)))
    ne = len(a) * len(b) / (len(a) + len(b))
    lam = (np.sqrt(ne) + 0.12 + 0.11 / np.sqrt(ne)) * d
    k = np.arange(1, 101)
    p = 2 * np.sum((-1) ** (k - 1) * np.exp(-2 * (lam * k) ** 2))
    return d, min(max(p, 0.0), 1.0)


@pytest.mark.parametrize("index", [-1.0, -2.7])
def test_counter_based_draws_match_the_reference_in_distribution(oracle, reference, index):
    n = 100000
    emin, emax = 1 * U.EeV, 100 * U.EeV
    ida, ea, da = oracle.sample_source_philox(20260101, 0, n, IDS, AB, True, emin, emax, index)
    idb, eb, db = reference.sample_source(7, n, (0.0, 0.0, 0.0), IDS, AB, emin, emax, index)
    assert _ks_2samp(np.log(ea), np.log(eb))[1] > 1e-3
    assert _ks_2samp(da[:, 2], db[:, 2])[1] > 1e-3                       # cos(theta) uniform
    assert _ks_2samp(np.arctan2(da[:, 1], da[:, 0]), np.arctan2(db[:, 1], db[:, 0]))[1] > 1e-3
    np.testing.assert_allclose(np.linalg.norm(da, axis=1), 1.0, rtol=0, atol=4e-16)
    ca = np.array([(ida == p).sum() for p in IDS])
    cb = np.array([(idb == p).sum() for p in IDS])
    exp = np.array(AB) / sum(AB) * n
    chi = np.sum((ca - exp) ** 2 / exp)
    assert chi < 16.3, (ca, exp)                                         # 3 dof, p > 0.001
    assert np.sum((cb - exp) ** 2 / exp) < 16.3
    assert ea.min() >= emin and ea.max() <= emax


def test_split_runs_draw_the_same_candidates(oracle):
    a = oracle.sample_source_philox(5, 0, 1000, IDS, AB, True, 1.0, 10.0, -2.0)
    b = oracle.sample_source_philox(5, 600, 400, IDS, AB, True, 1.0, 10.0, -2.0)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x[600:], y)
    c = oracle.sample_source_philox(6, 0, 1000, IDS, AB, True, 1.0, 10.0, -2.0)
    assert not np.array_equal(a[1], c[1])


def test_fixed_energy_and_direction(oracle):
    ids, e, d = oracle.sample_source_philox(9, 0, 50, [2212], None, False, energy=3.0, isotropic=False,
                                            direction=(0.0, 3.0, 4.0))
    assert np.all(ids == 2212) and np.all(e == 3.0)
    np.testing.assert_array_equal(d, np.tile([0.0, 0.6, 0.8], (50, 1)))


def test_rejects_bad_sources_before_any_device_call():
    lib = _abi.load()
    ids = (C.c_int32 * 1)(2212)
    d = _abi.SourceDesc()
    d.n_types = 0
    d.ids = ids
    assert lib.crp_source_sample_device(C.byref(d), 1, 0, 10, None, None, None, None) == _abi.ERR_INVALID_ARGUMENT
    d.n_types, d.spectrum, d.emin, d.emax = 1, 1, 10.0, 1.0
    assert lib.crp_source_sample_device(C.byref(d), 1, 0, 10, None, None, None, None) == _abi.ERR_INVALID_ARGUMENT
    assert "0 <= min <= max" in _abi.last_error()


# ------------------------------------------------------------------ GPU


def _device(seed, first, n, ids, ab, spectrum, emin, emax, index, energy=1.0, isotropic=True,
            direction=(1.0, 0.0, 0.0)):
    import torch
    lib = _abi.load()
    idv = np.asarray(ids, dtype=np.int32)
    abv = None if ab is None else np.asarray(ab, dtype=np.float64)
    d = _abi.SourceDesc()
    d.n_types = len(idv)
    d.ids = idv.ctypes.data_as(C.POINTER(C.c_int32))
    d.abundances = abv.ctypes.data_as(C.POINTER(C.c_double)) if abv is not None else None
    d.spectrum, d.emin, d.emax, d.index, d.energy = int(spectrum), emin, emax, index, energy
    d.isotropic = int(isotropic)
    for k in range(3):
        d.direction[k] = direction[k]
    out_id = torch.empty(n, dtype=torch.int32, device="cuda")
    out_e = torch.empty(n, dtype=torch.float64, device="cuda")
    out_d = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    _abi.check(lib.crp_source_sample_device(C.byref(d), seed, first, n, out_id.data_ptr(), out_e.data_ptr(),
                                            out_d.data_ptr(), torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return out_id.cpu().numpy(), out_e.cpu().numpy(), out_d.cpu().numpy().reshape(3, n).T


CASES = {
    "four_types_power_law": (IDS, AB, True, 1 * U.EeV, 100 * U.EeV, -2.7),
    "equal_types_log_uniform": (IDS, None, True, 1e-3 * U.EeV, 1e3 * U.EeV, -1.0),
    "proton_fixed_energy": ([2212], None, False, 1.0, 1.0, -1.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_device_draws_follow_the_restatement(oracle, case):
    ids, ab, spectrum, emin, emax, index = CASES[case]
    n, first, seed = 300001, 12345, 0x1234_5678_9ABC
    a = oracle.sample_source_philox(seed, first, n, ids, ab, spectrum, emin, emax, index, energy=5.0)
    d = _device(seed, first, n, ids, ab, spectrum, emin, emax, index, energy=5.0)
    np.testing.assert_array_equal(d[0], a[0])
    np.testing.assert_allclose(d[1], a[1], rtol=5e-16, atol=0)
    np.testing.assert_allclose(d[2], a[2], rtol=0, atol=5e-16)


@pytest.mark.gpu
def test_device_fixed_direction_and_split(oracle):
    d = _device(3, 0, 1000, [2212], None, False, 1.0, 1.0, -1.0, energy=2.0, isotropic=False,
                direction=(0.0, 3.0, 4.0))
    np.testing.assert_array_equal(d[2], np.tile([0.0, 0.6, 0.8], (1000, 1)))
    whole = _device(11, 0, 5000, IDS, AB, True, 1.0, 10.0, -2.0)
    tail = _device(11, 3000, 2000, IDS, AB, True, 1.0, 10.0, -2.0)
    for x, y in zip(whole, tail):
        np.testing.assert_array_equal(x[3000:], y)


@pytest.mark.gpu
def test_device_candidates_helper():
    from crpropa3_b200.workloads import source_candidates_device
    c = source_candidates_device(4096, IDS, 1 * U.EeV, 100 * U.EeV, -1.0, seed=8, position=(1.0, 2.0, 3.0))
    h = c.to_host()
    assert set(np.unique(h.id)) <= set(IDS)
    assert np.all(h.active == 1) and np.all(h.x == 1.0) and np.all(h.pz == 3.0)
    q = {p: _abi_charge(p) for p in IDS}
    np.testing.assert_array_equal(h.charge, [q[int(p)] for p in h.id])


def _abi_charge(pid):
    from crpropa3_b200.workloads import charge_of
    return charge_of(pid)
