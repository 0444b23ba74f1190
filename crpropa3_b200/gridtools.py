"""Grid files in the reference's formats (GridTools.cpp:134-482), so that
grids written by CRPropa load here and grids built here load in CRPropa.

Binary (dumpGrid / loadGrid, GridTools.cpp:134-236): native float32 values
in cell order ix, iy, iz with z fastest (Grid.h:338), three per Grid3f cell
(x, y, z) and one per Grid1f cell, no header; each value scaled by the
conversion factor c.  Text (dumpGridToTxt / loadGridFromTxt,
GridTools.cpp:238-482): one cell per line, components separated by one
space, six significant digits (the default ostream format), optionally
preceded by a '# GridProperties: ...' header line that
loadGrid3fFromTxt / loadGrid1fFromTxt read back.

The scaling rounds as the reference's does: a Grid3f value is a Vector3f,
whose products with the double c happen in float (Vector3.h:305, :363); a
Grid1f value is a float, whose product with c happens in double and is then
rounded to float.
"""
from __future__ import annotations

import os

import numpy as np

from . import _abi
from .plan import GridField, ScalarGrid

_INTERP_NAMES = {_abi.INTERPOLATION_TRILINEAR: "TRILINEAR", _abi.INTERPOLATION_TRICUBIC: "TRICUBIC",
                 _abi.INTERPOLATION_NEAREST_NEIGHBOUR: "NEAREST_NEIGHBOUR"}


def _values(grid):
    v = np.ascontiguousarray(grid.values if hasattr(grid, "values") else grid, dtype=np.float32)
    if v.ndim == 4 and v.shape[3] == 3:
        return v, 3
    if v.ndim == 3:
        return v, 1
    raise ValueError("grid values must have shape (nx, ny, nz, 3) or (nx, ny, nz)")


def _scaled(v, width, c):
    if c == 1:
        return v
    if width == 3:  # Vector3f * double: c rounded to float, float product
        return (v * np.float32(c)).astype(np.float32)
    return (v.astype(np.float64) * float(c)).astype(np.float32)  # float * double, rounded to float


def dump_grid(grid, filename, c=1.0):
    """dumpGrid (GridTools.cpp:194, :213): a GridField / ScalarGrid or a value
    array, scaled by c, as raw float32."""
    v, width = _values(grid)
    with open(filename, "wb") as f:
        f.write(_scaled(v, width, c).astype("=f4").tobytes())


def load_grid(shape, filename, c=1.0, vector=True) -> np.ndarray:
    """loadGrid (GridTools.cpp:134, :165) into a grid of `shape` (nx, ny, nz):
    (nx, ny, nz, 3) float32 for a Grid3f (vector=True), (nx, ny, nz) for a
    Grid1f.  A file whose size is not the grid's raises, as the reference's
    does."""
    nx, ny, nz = (int(s) for s in shape)
    width = 3 if vector else 1
    if not os.path.exists(filename):
        raise RuntimeError(f"load Grid{'3' if vector else '1'}f: {filename} not found")
    if os.path.getsize(filename) // 4 != width * nx * ny * nz:
        raise RuntimeError("loadGrid: file and grid size do not match")
    v = np.fromfile(filename, dtype="=f4").reshape((nx, ny, nz, 3) if vector else (nx, ny, nz))
    return _scaled(v, width, c)


def _fmt(x) -> str:
    """One value as `ostream << x` writes it (precision 6, %g)."""
    return "%g" % x


def _vec(a) -> str:
    return " ".join(_fmt(float(x)) for x in a)


def dump_grid_to_txt(grid, filename, c=1.0, save_properties=False, origin=(0.0, 0.0, 0.0),
                     spacing=(1.0, 1.0, 1.0), reflective=False, clip_volume=False,
                     interpolation=_abi.INTERPOLATION_TRILINEAR):
    """dumpGridToTxt (GridTools.cpp:424, :454).  With a GridField or
    ScalarGrid the header's properties come from it."""
    v, width = _values(grid)
    if isinstance(grid, (GridField, ScalarGrid)):
        origin, spacing = grid.origin, grid.spacing
        reflective, clip_volume, interpolation = grid.reflective, grid.clip_volume, grid.interpolation
    sp = spacing if hasattr(spacing, "__len__") else (spacing,) * 3
    s = _scaled(v, width, c)
    lines = []
    if save_properties:
        nx, ny, nz = v.shape[:3]
        lines.append(f"# GridProperties: Type Grid{width}f\torigin: {_vec(origin)}\tgridsize: {nx} {ny} {nz}"
                     f"\tspacing: {_vec(sp)}\treflective: {int(bool(reflective))}"
                     f"\tclipVolume: {int(bool(clip_volume))}\tinterpolation: {_INTERP_NAMES[int(interpolation)]}\n")
    flat = s.reshape(-1, width)
    lines.extend((_vec(row) if width == 3 else _fmt(float(row[0]))) + "\n" for row in flat)
    with open(filename, "w") as f:
        f.writelines(lines)


def _read_txt(filename, vector):
    if not os.path.exists(filename):
        raise RuntimeError(f"load Grid{'3' if vector else '1'}f: {filename} not found")
    header, values = [], []
    with open(filename) as f:
        for line in f:
            if not values and line.startswith("#"):
                header.append(line.rstrip("\n"))
                continue
            values.extend(line.split())
    return header, values


def load_grid_from_txt(shape, filename, c=1.0, vector=True) -> np.ndarray:
    """loadGridFromTxt (GridTools.cpp:238, :330): values parsed as floats,
    header lines skipped; too few values raise."""
    nx, ny, nz = (int(s) for s in shape)
    width = 3 if vector else 1
    _, vals = _read_txt(filename, vector)
    need = width * nx * ny * nz
    if len(vals) < need:
        raise RuntimeError(f"load Grid{width}f: file too short")
    v = np.array(vals[:need], dtype=np.float32).reshape((nx, ny, nz, 3) if vector else (nx, ny, nz))
    return _scaled(v, width, c)


def load_grid_with_properties_from_txt(filename, c=1.0, vector=True):
    """loadGrid3fFromTxt / loadGrid1fFromTxt (GridTools.cpp:262, :354): the
    grid and its properties from the '# GridProperties:' header, as a
    GridField (vector) or ScalarGrid."""
    header, _ = _read_txt(filename, vector)
    want = "Grid3f" if vector else "Grid1f"
    for line in header:
        if line.find("GridProperties:") != 2:
            continue
        tok = line.split()
        # '#', 'GridProperties:', 'Type', <type>, 'origin:', x, y, z, 'gridsize:', nx, ny, nz,
        # 'spacing:', dx, dy, dz, 'reflective:', r, 'clipVolume:', c, 'interpolation:', name
        if tok[3] != want:
            raise RuntimeError(f"Tried to load {want}, but Gridproperties assume grid type {tok[3]}")
        origin = tuple(float(x) for x in tok[5:8])
        shape = tuple(int(x) for x in tok[9:12])
        spacing = tuple(float(x) for x in tok[13:16])
        reflective, clip = bool(int(tok[17])), bool(int(tok[19]))
        name = tok[21] if len(tok) > 21 else "TRILINEAR"
        interp = {"TRICUBIC": _abi.INTERPOLATION_TRICUBIC,
                  "NEAREST_NEIGHBOUR": _abi.INTERPOLATION_NEAREST_NEIGHBOUR}.get(name, _abi.INTERPOLATION_TRILINEAR)
        v = load_grid_from_txt(shape, filename, c, vector)
        cls = GridField if vector else ScalarGrid
        return cls(v, origin, spacing, reflective=reflective, clip_volume=clip, interpolation=interp)
    raise RuntimeError("could not find GridProperties in file " + filename)
