"""The C++ plugin GpuModuleList (crpropa3_b200/plugin): the reference's own
chain objects -- PropagationBP/CK, DiffusionSDE, MagneticFieldGrid over a
Grid3f, PlaneWaveTurbulence, MagneticFieldList, MaximumTrajectoryLength,
Observer with ObserverSurface(Sphere) and a TextOutput or record action --
run through GpuModuleList::run on the device, against the same chain run by
the reference's ModuleList::run (ModuleList.cpp.in:97, :153) on the CPU.

Without a device: the translation of reference chains into the C-ABI plan,
and the refusal (an exception naming the module, never a silent CPU run) of
chains that have no device form.
"""
import numpy as np
import pytest

from helpers import P, U, _abi, bp_fixed, ck, grid_chain, protons, random_grid, stable_unit_vectors
from crpropa3_b200.state import CandidateArrays, RecordArrays


@pytest.fixture(scope="module")
def plugin():
    from oracle import PluginHarness, plugin_harness_available
    if not plugin_harness_available():
        pytest.skip("plugin harness not built (make -C oracle ref-gpu needs the reference checkout)")
    return PluginHarness()


def _grid_spec(prop, n=16, spacing=10 * U.kpc, radius=60 * U.kpc, length=400 * U.kpc,
               precision=_abi.PRECISION_FP64, seed=3, record=True, periodic=False):
    grid = random_grid(np.random.default_rng(seed), n, brms=3e-13)
    gf = P.GridField(grid, (-80 * U.kpc,) * 3, (spacing,) * 3)
    if periodic:
        gf.periodic = ((-80 * U.kpc,) * 3, (n * spacing,) * 3, False)
    mods = [prop, P.MaxTrajectoryLength(length, record=record),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), radius, True, record)]
    return P.ChainSpec([gf], mods, precision=precision)


def _sde_spec(oracle):
    xi, kappa, k, beta, ak = oracle.plane_wave_modes(0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0,
                                                     16, 11)
    fields = [P.ToroidalField(1 * U.muG),
              P.PlaneWaveField(xi, kappa, k, beta, ak,
                               spectrum=(0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0), seed=11)]
    mods = [P.MaxTrajectoryLength(10 * U.kpc),
            P.Propagation(_abi.PROP_SDE, 1e-4, 0.1 * U.pc, 100 * U.pc, epsilon=0.1),
            P.ObserverSpec(_abi.OBSERVER_SURFACE_SPHERE, (0, 0, 0), 300 * U.pc, True, True)]
    return P.ChainSpec(fields, mods, seed=5)


# ------------------------------------------------------------------ CPU


def test_plugin_translates_reference_chains(plugin, oracle):
    ok, text = plugin.describe(_grid_spec(bp_fixed(1 * U.kpc), periodic=True))
    assert ok, text
    assert "PropagationBP" in text and "Grid3f 16x16x16" in text
    assert "PeriodicMagneticField" in text
    assert "MaximumTrajectoryLength" in text and "ObserverSurface(Sphere" in text
    ok, text = plugin.describe(_grid_spec(ck(1e-4, 0.1 * U.kpc, 10 * U.kpc)))
    assert ok and "PropagationCK tolerance 0.0001" in text, text
    ok, text = plugin.describe(_sde_spec(oracle))
    assert ok, text
    assert "DiffusionSDE" in text and "ToroidalMagneticField" in text
    assert "PlaneWaveTurbulence 16 modes" in text


@pytest.mark.parametrize("extra,reason", [
    (1, "SimplePropagation"),
    (2, "MinimumEnergy"),
    (3, "observer positions"),
    (4, "RestrictToRegion"),
    (5, "setMakeRejectedInactive(false)"),
])
def test_plugin_declines_chains_off_the_device_path(plugin, extra, reason):
    ok, text = plugin.describe(_grid_spec(bp_fixed(1 * U.kpc)), extra)
    assert not ok
    assert reason in text, text


def test_plugin_run_of_unsupported_chain_throws(plugin):
    msg = plugin.unsupported_run_message(_grid_spec(bp_fixed(1 * U.kpc)))
    assert msg is not None, "an unsupported chain ran"
    assert "not on the device path" in msg and "SimplePropagation" in msg


# ------------------------------------------------------------------ GPU


def _cands(n, seed=7, spread=20 * U.kpc):
    return protons(np.random.default_rng(seed), n, emin=1 * U.EeV, emax=100 * U.EeV, spread=spread)


def _records_sorted(r: RecordArrays):
    d = r.sorted()
    return {k: np.asarray(v) for k, v in d.items()}


@pytest.mark.gpu
def test_plugin_fixed_bp_bitwise_against_reference(plugin, reference):
    spec = _grid_spec(bp_fixed(1 * U.kpc))
    c = _cands(512)
    a, b = c.copy(), c.copy()
    ra, rb = RecordArrays(2 * c.n), RecordArrays(2 * c.n)
    reference.run(spec, a, ra, threads=4)
    stats, events = plugin.run(spec, b, rb)
    assert stats.launches > 0 and stats.particle_steps > 0
    for name in ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time",
                 "current_step", "next_step", "active", "flags"):
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
    assert events == rb.n() == ra.n()
    ga, gb = _records_sorted(ra), _records_sorted(rb)
    for k in ga:
        np.testing.assert_array_equal(ga[k], gb[k], err_msg=k)


@pytest.mark.gpu
def test_plugin_adaptive_ck_against_reference(plugin, reference):
    spec = _grid_spec(ck(1e-4, 0.1 * U.kpc, 10 * U.kpc))
    c = _cands(256, seed=8)
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=4)
    plugin.run(spec, b)
    # the device's correctly rounded pow differs from glibc's on ~0.1 % of
    # the controller's calls; a differing step size then changes the path
    same = np.all(a.position() == b.position(), axis=1)
    assert same.mean() >= 0.8, same.mean()
    np.testing.assert_array_equal(a.active, b.active)
    np.testing.assert_array_equal(a.flags, b.flags)


@pytest.mark.gpu
def test_plugin_per_candidate_length_bitwise(plugin, reference):
    grid = random_grid(np.random.default_rng(12), 16, brms=3e-13)
    spec = P.ChainSpec([P.GridField(grid, (-80 * U.kpc,) * 3, (10 * U.kpc,) * 3)],
                       [bp_fixed(1 * U.kpc), P.MaxTrajectoryLength(0.0, per_candidate=True, record=True)])
    c = _cands(300, seed=9)
    c.max_length = np.random.default_rng(4).uniform(50, 300, c.n) * U.kpc
    a, b = c.copy(), c.copy()
    reference.run(spec, a, threads=2)
    plugin.run(spec, b)
    np.testing.assert_array_equal(a.position(), b.position())
    np.testing.assert_array_equal(a.trajectory_length, b.trajectory_length)
    np.testing.assert_array_equal(a.flags, b.flags)


def _data_lines(path):
    with open(path) as f:
        lines = f.readlines()
    head = [l for l in lines if l.startswith("#")]
    data = sorted(l for l in lines if not l.startswith("#"))
    return head, data


@pytest.mark.gpu
@pytest.mark.parametrize("output_type", [3, 4])  # Output::Event3D, Output::Everything
def test_plugin_text_output_identical_to_reference(plugin, reference, tmp_path, output_type):
    spec = _grid_spec(bp_fixed(1 * U.kpc), radius=40 * U.kpc, length=300 * U.kpc)
    c = _cands(400, seed=10)
    pr, pg = tmp_path / "ref.txt", tmp_path / "gpu.txt"
    reference.run_textout(spec, c.copy(), pr, output_type, threads=1, serial0=1)
    plugin.run_textout(spec, c.copy(), pg, output_type, serial0=1)
    hr, dr = _data_lines(pr)
    hg, dg = _data_lines(pg)
    assert hr == hg
    assert len(dr) > 100
    assert dr == dg


@pytest.mark.gpu
def test_plugin_particle_collector_identical_to_reference(plugin, reference, tmp_path):
    """A ParticleCollector (clone on) as the observer's detection action
    (ParticleCollector.cpp:23): the plugin replays the detections into the
    user's collector, whose dump (TextOutput Everything) equals the one of
    ModuleList::run, line for line, serial numbers included."""
    spec = _grid_spec(bp_fixed(1 * U.kpc), radius=40 * U.kpc, length=300 * U.kpc)
    c = _cands(400, seed=12)
    pr, pg = tmp_path / "ref.txt", tmp_path / "gpu.txt"
    collector = 100  # the harness's ParticleCollector output type
    reference.run_textout(spec, c.copy(), pr, collector, threads=1, serial0=1)
    plugin.run_textout(spec, c.copy(), pg, collector, serial0=1)
    hr, dr = _data_lines(pr)
    hg, dg = _data_lines(pg)
    assert hr == hg
    assert len(dr) > 100
    assert dr == dg


@pytest.mark.gpu
def test_plugin_run_source_count_identical_to_reference(plugin, tmp_path):
    """ModuleList::run(source, count) with the reference's Source features:
    the plugin draws the candidates on the calling thread in batches (here
    3 batches of 300 and one of 100); the reference runs one thread, so both
    draw the same sequence from crpropa::Random."""
    spec = _grid_spec(bp_fixed(1 * U.kpc), radius=40 * U.kpc, length=300 * U.kpc)
    pr, pg = tmp_path / "ref.txt", tmp_path / "gpu.txt"
    args = ((0.0, 0.0, 0.0), 1000010010, 1 * U.EeV, 100 * U.EeV, -1.0, 1000)
    plugin.run_source_textout(spec, False, *args, pr, 4, seed=21)
    stats = plugin.run_source_textout(spec, True, *args, pg, 4, seed=21, batch=300)
    assert stats.launches >= 4
    hr, dr = _data_lines(pr)
    hg, dg = _data_lines(pg)
    assert hr == hg
    assert len(dr) == 1000
    assert dr == dg


@pytest.mark.gpu
def test_plugin_mixed_precision_within_bound(plugin, reference):
    """Weakly deflected candidates: the mixed form through the plugin stays
    within 1e-6 relative final position of the reference (the bound the
    engine's mixed form is tested to)."""
    spec64 = _grid_spec(bp_fixed(1 * U.kpc), radius=1e3 * U.kpc, length=300 * U.kpc)
    spec_mx = _grid_spec(bp_fixed(1 * U.kpc), radius=1e3 * U.kpc, length=300 * U.kpc,
                         precision=_abi.PRECISION_MIXED)
    c = _cands(256, seed=11)
    c.energy[:] = np.exp(np.random.default_rng(2).uniform(np.log(20), np.log(100), c.n)) * U.EeV
    a, b = c.copy(), c.copy()
    reference.run(spec64, a, threads=2)
    plugin.run(spec_mx, b, precision=_abi.PRECISION_MIXED)
    rel = np.linalg.norm(a.position() - b.position(), axis=1) / np.linalg.norm(a.position(), axis=1)
    assert rel.max() <= 1e-6, rel.max()


def _ob_chains():
    import test_observers_boundaries as T
    return T


@pytest.mark.parametrize("name", ["plane", "box", "tracking", "observer1d", "vetoes", "spherical", "cubic",
                                  "ellipsoidal", "cylindrical", "boundary_and_observer"])
def test_plugin_translates_observer_features_and_boundaries(plugin, name):
    T = _ob_chains()
    ok, text = plugin.describe(T._spec(name))
    assert ok, text
    expect = {"plane": "ObserverSurface(Plane)", "box": "ObserverSurface(ParaxialBox)",
              "tracking": "ObserverTracking", "observer1d": "Observer1D",
              "vetoes": "ObserverParticleIdVeto 1000020040", "spherical": "SphericalBoundary",
              "cubic": "CubicBoundary", "ellipsoidal": "EllipsoidalBoundary",
              "cylindrical": "CylindricalBoundary", "boundary_and_observer": "SphericalBoundary"}[name]
    assert expect in text, text


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["vetoes", "box", "tracking", "cubic", "cylindrical", "boundary_and_observer"])
def test_plugin_observer_features_and_boundaries_bitwise(plugin, reference, name):
    """The reference's Observer features and boundary modules, run through
    GpuModuleList (FP64 form), against ModuleList::run: same state, flags and
    replayed records."""
    T = _ob_chains()
    spec = T._spec(name)
    c = T._cands()
    a, b = c.copy(), c.copy()
    ra, rb = RecordArrays(200_000), RecordArrays(200_000)
    reference.run(spec, a, ra, threads=2)
    plugin.run(spec, b, rb)
    T._compare(a, b, ra, rb)


def _interrupt_chain():
    rng = np.random.default_rng(61)
    grid = random_grid(rng, 16)
    spec = grid_chain(grid, 10 * U.kpc, bp_fixed(1 * U.kpc), 1 * U.Mpc, observer_radius=0.2 * U.Mpc,
                      record=False)
    return spec, protons(rng, 4000, spread=0.0)


def _index_list_text(indices):
    """TextOutput::dumpIndexList (TextOutput.cpp:396): '#', then each index,
    each followed by a tab."""
    return "#\t" + "".join(f"{i}\t" for i in indices)


def test_reference_interrupt_semantics_and_index_list_format(plugin, tmp_path):
    """The reference's own ModuleList::run(candidates), one thread, with SIGINT
    sent by an observer's detection action: the candidates after the one
    being run are not started, their indices go to the interrupt action in
    TextOutput::dumpIndexList's format, and the signal is raised again at
    the end (ModuleList.cpp.in:110-150).  This pins what the plugin test
    below holds the plugin to.  No GPU."""
    spec, c = _interrupt_chain()
    ref = c.copy()
    path = tmp_path / "ref_interrupt.txt"
    assert plugin.run_interrupted(spec, ref, path, gpu=False) == 2  # SIGINT raised again
    first = int(np.flatnonzero(ref.flags & _abi.FLAG_DETECTED)[0])
    assert path.read_text() == _index_list_text(range(first + 1, c.n))
    np.testing.assert_array_equal(ref.trajectory_length[first + 1:], c.trajectory_length[first + 1:])


@pytest.mark.gpu
def test_plugin_interrupted_run_matches_the_reference_semantics(plugin, tmp_path):
    """SIGINT during GpuModuleList::run(candidates), sent at a known point (the
    first detection, replayed during the first batch's write-back): the
    started batch completes exactly as in an uninterrupted run, the later
    batches are left as they were, their indices go to the interrupt action
    in the reference's format, and the signal is raised again at the end."""
    spec, c = _interrupt_chain()
    batch = 1000
    full, got = c.copy(), c.copy()
    plugin.run(spec, full)
    path = tmp_path / "gpu_interrupt.txt"
    assert plugin.run_interrupted(spec, got, path, gpu=True, batch=batch) == 2
    assert path.read_text() == _index_list_text(range(batch, c.n))
    for name in ("x", "y", "z", "dx", "dy", "dz", "trajectory_length", "active", "flags"):
        np.testing.assert_array_equal(getattr(got, name)[:batch], getattr(full, name)[:batch],
                                      err_msg=name)
        np.testing.assert_array_equal(getattr(got, name)[batch:], getattr(c, name)[batch:],
                                      err_msg=name)
