"""Grid files in the reference's formats (GridTools.cpp:134-482): dumpGrid /
loadGrid (raw float32) and dumpGridToTxt / loadGridFromTxt /
loadGrid3fFromTxt / loadGrid1fFromTxt (text with a GridProperties header),
for Grid3f and Grid1f, with conversion factors.  Files written here are
compared byte for byte with the reference's, and each side loads the
other's files to the same values.  CPU only.
"""
import numpy as np
import pytest

from helpers import P, U, _abi
from crpropa3_b200 import gridtools as G

SHAPE = (5, 4, 3)


def _vector(seed=61):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(SHAPE + (3,)) * 3e-10).astype(np.float32)


def _scalar(seed=62):
    rng = np.random.default_rng(seed)
    return rng.uniform(-2, 5, SHAPE).astype(np.float32)


CASES = [("vector", 1.0), ("vector", 1 / U.muG), ("scalar", 1.0), ("scalar", 3.7)]


def _values(kind):
    return _vector() if kind == "vector" else _scalar()


@pytest.mark.parametrize("kind,c", CASES)
def test_binary_dump_identical_to_reference(reference, tmp_path, kind, c):
    v = _values(kind)
    G.dump_grid(v, tmp_path / "mine.raw", c)
    reference.dump_grid(v, tmp_path / "ref.raw", c)
    assert (tmp_path / "mine.raw").read_bytes() == (tmp_path / "ref.raw").read_bytes()


@pytest.mark.parametrize("kind,c", CASES)
def test_binary_load_matches_reference(reference, tmp_path, kind, c):
    v = _values(kind)
    reference.dump_grid(v, tmp_path / "g.raw")
    mine = G.load_grid(SHAPE, tmp_path / "g.raw", c, vector=kind == "vector")
    ref = reference.load_grid(SHAPE, tmp_path / "g.raw", c, vector=kind == "vector")
    np.testing.assert_array_equal(mine, ref)
    with pytest.raises(RuntimeError, match="do not match"):
        G.load_grid((5, 4, 4), tmp_path / "g.raw", vector=kind == "vector")


@pytest.mark.parametrize("kind,c", CASES)
@pytest.mark.parametrize("save_prop", [False, True])
def test_text_dump_identical_to_reference(reference, tmp_path, kind, c, save_prop):
    v = _values(kind)
    props = dict(origin=(-1.5e20, 2.0, 0.25), spacing=(3.0856775807e19, 2e19, 1e19), reflective=True,
                 clip_volume=False, interpolation=_abi.INTERPOLATION_TRICUBIC)
    G.dump_grid_to_txt(v, tmp_path / "mine.txt", c, save_prop, **props)
    reference.dump_grid(v, tmp_path / "ref.txt", c, txt=True, save_prop=save_prop, origin=props["origin"],
                        spacing=props["spacing"], reflective=True, clip=False, interp=_abi.INTERPOLATION_TRICUBIC)
    assert (tmp_path / "mine.txt").read_text() == (tmp_path / "ref.txt").read_text()


@pytest.mark.parametrize("kind", ["vector", "scalar"])
def test_text_load_with_properties_matches_reference(reference, tmp_path, kind):
    v = _values(kind)
    vec = kind == "vector"
    grid = (P.GridField if vec else P.ScalarGrid)(v, (1.0, -2.0, 3.0), (0.5, 0.5, 0.25), reflective=False,
                                                  clip_volume=True, interpolation=_abi.INTERPOLATION_NEAREST_NEIGHBOUR)
    G.dump_grid_to_txt(grid, tmp_path / "g.txt", save_properties=True)
    mine = G.load_grid_with_properties_from_txt(tmp_path / "g.txt", 2.0, vector=vec)
    shape, origin, spacing, flags, values = reference.load_grid_props(tmp_path / "g.txt", 2.0, vector=vec)
    assert mine.values.shape[:3] == shape == SHAPE
    np.testing.assert_array_equal(np.asarray(mine.origin), origin)
    np.testing.assert_array_equal(np.asarray(mine.spacing), spacing)
    assert (mine.reflective, mine.clip_volume, mine.interpolation) == (bool(flags[0]), bool(flags[1]), flags[2])
    np.testing.assert_array_equal(mine.values, values)
    # and the plain loader over the same file (header skipped)
    np.testing.assert_array_equal(G.load_grid_from_txt(SHAPE, tmp_path / "g.txt", vector=vec),
                                  reference.load_grid(SHAPE, tmp_path / "g.txt", vector=vec, txt=True))


def test_round_trip_through_the_reference_and_into_a_plan(reference, oracle, tmp_path):
    """A grid dumped by the reference, loaded here, steps the same as the
    original values."""
    v = _vector()
    reference.dump_grid(v, tmp_path / "g.raw")
    back = G.load_grid(SHAPE, tmp_path / "g.raw")
    np.testing.assert_array_equal(back, v)
    spec_a = P.ChainSpec([P.GridField(v, (0, 0, 0), (U.kpc,) * 3)], [P.Propagation(_abi.PROP_BP, 0.42, U.kpc, U.kpc)])
    spec_b = P.ChainSpec([P.GridField(back, (0, 0, 0), (U.kpc,) * 3)], [P.Propagation(_abi.PROP_BP, 0.42, U.kpc, U.kpc)])
    pos = np.random.default_rng(3).uniform(-10, 10, (100, 3)) * U.kpc
    np.testing.assert_array_equal(oracle.field(spec_a, pos), oracle.field(spec_b, pos))
