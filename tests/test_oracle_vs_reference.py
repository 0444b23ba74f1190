"""The oracle against the reference itself (compiled from its sources by
oracle/Makefile into oracle/_ref/), on identical inputs, on the CPU.

Runs wherever the reference library has been built; the golden fixtures in
tests/golden/ carry the same evidence to machines without it."""
import numpy as np
import pytest

from helpers import (P, RecordArrays, U, _abi, bp_fixed, ck, grid_chain, protons, random_grid,
                     stable_unit_vectors)


def _same(a, b, names=("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length",
                       "time", "current_step", "next_step", "active", "flags")):
    for n in names:
        np.testing.assert_array_equal(getattr(a, n), getattr(b, n), err_msg=n)


def _run_both(oracle, reference, spec, c, cap=2048, threads=4):
    a, b = c.copy(), c.copy()
    ra, rb = RecordArrays(cap), RecordArrays(cap)
    sa = oracle.run(spec, a, ra)
    sb = reference.run(spec, b, rb, threads=threads)
    return a, b, ra, rb, sa, sb


@pytest.mark.parametrize("prop", [bp_fixed(1 * U.kpc),
                                  P.Propagation(_abi.PROP_BP, 1e-3, 0.1 * U.kpc, 10 * U.kpc),
                                  ck(1e-4, 1 * U.kpc, 1 * U.kpc),
                                  ck(1e-4, 0.1 * U.kpc, 10 * U.kpc)],
                         ids=["bp_fixed", "bp_adaptive", "ck_fixed", "ck_adaptive"])
@pytest.mark.parametrize("reflective", [False, True])
def test_propagation_bitwise(oracle, reference, prop, reflective):
    rng = np.random.default_rng(101)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, prop, 1 * U.Mpc, observer_radius=0.4 * U.Mpc,
                      reflective=reflective)
    c = protons(rng, 96)
    a, b, ra, rb, sa, sb = _run_both(oracle, reference, spec, c)
    _same(a, b)
    assert sa[0] == sb[0]
    assert ra.n() == rb.n() > 0
    for k, v in ra.sorted().items():
        np.testing.assert_array_equal(v, rb.sorted()[k], err_msg=k)


def test_field_components_bitwise(oracle, reference):
    rng = np.random.default_rng(102)
    grid = random_grid(rng, 8)
    pos = rng.uniform(-200, 200, (500, 3)) * U.kpc
    cases = [
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3)],
        [P.GridField(grid, (1 * U.kpc, 2 * U.kpc, 3 * U.kpc), (9 * U.kpc,) * 3, reflective=True)],
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3, clip_volume=True)],
        [P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3, periodic=((5 * U.kpc, 0, 0), (70 * U.kpc,) * 3, True))],
        [P.UniformField((1e-13, 2e-13, -3e-13)), P.ToroidalField(1e-10)],
    ]
    for fields in cases:
        spec = P.ChainSpec(fields, [bp_fixed(U.kpc)])
        np.testing.assert_array_equal(oracle.field(spec, pos), reference.field(spec, pos))


def test_plane_wave_modes_reproduce_reference_field(oracle, reference):
    """The restated PlaneWaveTurbulence constructor draws the same modes: the
    field from the oracle's modes equals the reference object's field."""
    rng = np.random.default_rng(103)
    pos = rng.uniform(-5, 5, (400, 3)) * U.kpc
    spectrum = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0)
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(*spectrum, 256, 1234)
    spec = P.ChainSpec([P.PlaneWaveField(xi, kappa, k, beta, ak, spectrum=spectrum, seed=1234)],
                       [bp_fixed(U.kpc)])
    np.testing.assert_array_equal(oracle.field(spec, pos), reference.field(spec, pos))


def test_random_and_source_match_reference(oracle, reference):
    for kind, args in ((0, ()), (1, (-2.0, 7.0)), (2, ()), (3, (-1.0, 1.0, 100.0)), (6, ())):
        a = list(args) + [0.0] * (3 - len(args))
        np.testing.assert_array_equal(oracle.random(99, kind, 1000, *a),
                                      reference.random(99, kind, 1000, *a))
    ids = [1000010010, 1000020040, 1000070140, 1000260560]
    o = oracle.sample_source(7, 500, ids, None, 0.1 * U.EeV, 100 * U.EeV, -2.0)
    r = reference.sample_source(7, 500, (0, 0, 0), ids, None, 0.1 * U.EeV, 100 * U.EeV, -2.0)
    for x, y in zip(o, r):
        np.testing.assert_array_equal(x, y)
    for pid in ids + [-1000010010, 2112]:
        from crpropa3_b200.workloads import charge_of
        assert charge_of(pid) == reference.charge(pid)


def test_per_candidate_length_and_neutral(oracle, reference):
    rng = np.random.default_rng(104)
    grid = random_grid(rng, 8)
    from crpropa3_b200.state import CandidateArrays
    c = protons(rng, 64)
    c2 = CandidateArrays(64, per_candidate_length=True)
    for name in c.MEMBERS:
        if getattr(c, name) is not None:
            getattr(c2, name)[:] = getattr(c, name)
    c2.max_length[:] = rng.uniform(50, 500, 64) * U.kpc
    c2.charge[::4] = 0.0  # neutral: rectilinear branch
    c2.id[::4] = 2112
    spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3)],
                       [ck(1e-4, 0.1 * U.kpc, 10 * U.kpc), P.MaxTrajectoryLength(per_candidate=True)])
    a, b, *_ = _run_both(oracle, reference, spec, c2)
    _same(a, b)


@pytest.mark.parametrize("suffix", [".txt", ".txt.gz"])
def test_text_output_matches_reference(reference, tmp_path, suffix):
    """crp_text_output_write against the reference's TextOutput (Event3D);
    a .gz name is gzip on both sides (TextOutput.cpp:41, zstream), compared
    after decompression."""
    import ctypes as C
    rng = np.random.default_rng(105)
    n = 50
    serial = np.arange(1, n + 1, dtype=np.uint64)
    ids = np.full(n, 1000010010, np.int32)
    e = rng.uniform(1, 100, n) * U.EeV
    pos = rng.uniform(-1, 1, (n, 3)) * U.Mpc
    d = stable_unit_vectors(rng, n)
    length = rng.uniform(0, 5, n) * U.Mpc
    src_e = e * 1.0
    src_pos = np.zeros((n, 3))
    src_d = stable_unit_vectors(rng, n)
    ref_path = str(tmp_path / ("ref" + suffix))
    reference.text_output(ref_path, 3, serial, ids, e, pos, d, length, ids, src_e, src_pos, src_d)
    lib = _abi.load()
    desc = _abi.OutputDesc()
    # Event3D columns (Output.cpp:62): D, ID, E, X, P, ID0, E0, X0, P0 (+ serial numbers off)
    for col in (0, 3, 4, 5, 6, 7, 8, 9, 10):
        desc.columns |= 1 << col
    desc.length_scale, desc.time_scale, desc.energy_scale = U.Mpc, U.Myr, U.EeV
    desc.version = b"3.2.1-ref"
    rows = _abi.OutputRows()
    keep = []

    def ptr(a, t=C.c_double):
        a = np.ascontiguousarray(a)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(t))
    rows.serial = ptr(serial, C.c_uint64)
    rows.trajectory_length = ptr(length)
    rows.time = ptr(length / U.c_light)
    rows.id = ptr(ids, C.c_int32)
    rows.energy = ptr(e)
    rows.position = ptr(pos)
    rows.direction = ptr(d)
    rows.source_id = ptr(ids, C.c_int32)
    rows.source_energy = ptr(src_e)
    rows.source_position = ptr(src_pos)
    rows.source_direction = ptr(src_d)
    mine = str(tmp_path / ("mine" + suffix))
    _abi.check(lib.crp_text_output_write(mine.encode(), 0, 1, C.byref(desc), n, C.byref(rows)))
    if suffix.endswith(".gz"):
        import gzip
        with open(mine, "rb") as f:
            assert f.read(2) == b"\x1f\x8b"
        assert gzip.open(mine, "rt").read() == gzip.open(ref_path, "rt").read()
    else:
        assert open(mine).read() == open(ref_path).read()


@pytest.mark.parametrize("prop", [P.Propagation(_abi.PROP_BP, 1e-3, 0.1 * U.kpc, 10 * U.kpc),
                                  ck(1e-4, 0.1 * U.kpc, 10 * U.kpc)], ids=["bp_adaptive", "ck_adaptive"])
def test_reference_with_correctly_rounded_pow_matches_crpow_oracle(oracle_crpow, prop):
    """The reference's sources linked so that pow is the engine's correctly
    rounded pow (libcrp_ref_crpow.so) against the oracle built with the same
    pow: bit for bit, adaptive controllers included.  This pins the build the
    GPU parity tests of the adaptive workloads compare with."""
    from oracle import Reference, reference_available
    if not reference_available(cr_pow=True):
        pytest.skip("reference library not built (make -C oracle ref needs the reference checkout)")
    ref = Reference(cr_pow=True)
    rng = np.random.default_rng(111)
    grid = random_grid(rng, 16, brms=1e-12)
    spec = grid_chain(grid, 10 * U.kpc, prop, 2 * U.Mpc)
    c = protons(rng, 256, emin=0.3 * U.EeV, emax=30 * U.EeV)
    a, b = c.copy(), c.copy()
    oracle_crpow.run(spec, a)
    ref.run(spec, b, threads=4)
    _same(a, b)
