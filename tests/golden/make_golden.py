"""Generate the golden fixtures of tests/golden/ from the reference itself.

Needs oracle/_ref/libcrp_ref.so (`make -C oracle ref`, which compiles the
reference's stepping path from its sources).  Writes reference_golden.npz
(the stepping chains, fields, draws, sources, charges) and
reference_golden_ext.npz (interpolation types, modulated grids, observer
features and boundaries, the galactic fields, turbulence draws, grid files).  Inputs are seeded; the outputs
are the reference's own ModuleList::run results, field values, random draws
and Source samples.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from helpers import (P, RecordArrays, U, _abi, bp_fixed, ck, grid_chain, protons,  # noqa: E402
                     random_grid)
from oracle import Reference  # noqa: E402

CASES = {
    "bp_fixed": dict(prop=lambda: bp_fixed(1 * U.kpc), reflective=False),
    "bp_fixed_reflective": dict(prop=lambda: bp_fixed(1 * U.kpc), reflective=True),
    "bp_adaptive": dict(prop=lambda: P.Propagation(_abi.PROP_BP, 1e-3, 0.1 * U.kpc, 10 * U.kpc), reflective=False),
    "ck_fixed": dict(prop=lambda: ck(1e-4, 1 * U.kpc, 1 * U.kpc), reflective=False),
    "ck_adaptive": dict(prop=lambda: ck(1e-4, 0.1 * U.kpc, 10 * U.kpc), reflective=False),
}
STATE = ("x", "y", "z", "dx", "dy", "dz", "px", "py", "pz", "trajectory_length", "time",
         "current_step", "next_step", "active", "flags")


def case_inputs(name):
    rng = np.random.default_rng(sum(map(ord, name)))
    grid = random_grid(rng, 16)
    c = protons(rng, 64)
    return grid, c


def main():
    ref = Reference()
    out = {}
    for name, cfg in CASES.items():
        grid, c = case_inputs(name)
        spec = grid_chain(grid, 10 * U.kpc, cfg["prop"](), 1 * U.Mpc, observer_radius=0.4 * U.Mpc,
                          reflective=cfg["reflective"])
        res = c.copy()
        rec = RecordArrays(256)
        steps, _ = ref.run(spec, res, rec, threads=1)
        out[f"{name}/steps"] = np.array([steps])
        for m in STATE:
            out[f"{name}/in_{m}"] = getattr(c, m)
            out[f"{name}/out_{m}"] = getattr(res, m)
        for m in ("id", "charge", "energy"):
            out[f"{name}/in_{m}"] = getattr(c, m)
        srt = rec.sorted()
        for k, v in srt.items():
            out[f"{name}/rec_{k}"] = v
    # fields
    rng = np.random.default_rng(7)
    grid = random_grid(rng, 8)
    pos = rng.uniform(-200, 200, (300, 3)) * U.kpc
    out["field/grid"] = grid
    out["field/pos"] = pos
    for key, f in (("periodic", dict()), ("reflective", dict(reflective=True)), ("clip", dict(clip_volume=True))):
        spec = P.ChainSpec([P.GridField(grid, (0, 0, 0), (10 * U.kpc,) * 3, **f)], [bp_fixed(U.kpc)])
        out[f"field/B_{key}"] = ref.field(spec, pos)
    spectrum = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0)
    pw_pos = rng.uniform(-5, 5, (200, 3)) * U.kpc
    # the reference object is built from (spectrum, Nm = 64, seed); it reads no mode arrays
    spec = P.ChainSpec([P.PlaneWaveField(np.zeros(3 * 64), np.zeros(3 * 64), np.zeros(64), np.zeros(64),
                                         np.zeros(64), spectrum=spectrum, seed=4321)], [bp_fixed(U.kpc)])
    out["planewave/pos"] = pw_pos
    out["planewave/B"] = ref.field(spec, pw_pos)
    out["planewave/spectrum"] = np.array(spectrum)
    # random draws and source
    for kind, args in ((0, ()), (1, (-2.0, 7.0)), (2, ()), (3, (-1.0, 1.0, 100.0)), (3, (-2.0, 0.1, 100.0)), (6, ())):
        a = list(args) + [0.0] * (3 - len(args))
        out[f"random/{kind}_{'_'.join(map(str, args))}"] = ref.random(2024, kind, 500, *a)
    ids = [1000010010, 1000020040, 1000070140, 1000260560]
    sid, se, sd = ref.sample_source(11, 400, (0, 0, 0), ids, None, 0.1 * U.EeV, 100 * U.EeV, -2.0)
    out["source/id"], out["source/energy"], out["source/dir"] = sid, se, sd
    out["charge/ids"] = np.array(ids + [-1000010010, 2112], np.int32)
    out["charge/q"] = np.array([ref.charge(i) for i in out["charge/ids"]])
    np.savez_compressed(os.path.join(HERE, "reference_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_golden.npz"), len(out), "arrays")




def main_ext():
    """reference_golden_ext.npz: the interpolation types, ModulatedMagneticFieldGrid,
    observer features and boundaries, JF12Field / PlanckJF12bField, UF23Field, the
    turbulence draw sequences and the grid file formats, from the reference."""
    import tempfile
    import test_grid_interpolation as GI
    import test_jf12 as J
    import test_observers_boundaries as OB
    import test_uf23 as UF
    ref = Reference()
    out = {}
    pos = GI._positions(600, seed=201)
    out["interp/pos"] = pos
    for interp, refl, clip in GI.VECTOR_CASES:
        out[f"interp/B_{interp}_{int(refl)}_{int(clip)}"] = ref.field(GI._vector_spec(interp, refl, clip), pos)
    for gi, mi, mr in GI.MOD_CASES:
        out[f"modulated/B_{gi}_{mi}_{int(mr)}"] = ref.field(GI._mod_spec(gi, mi, mr), pos)
    for name in ("box", "cylindrical", "vetoes", "tracking"):
        c = OB._cands(120, seed=202)
        res, rec = c.copy(), RecordArrays(20000)
        ref.run(OB._spec(name), res, rec, threads=1)
        for m in OB.STATE:
            out[f"chain_{name}/out_{m}"] = getattr(res, m)
        for k, v in rec.sorted().items():
            out[f"chain_{name}/rec_{k}"] = v
    jpos = J._positions(800, seed=203)
    out["jf12/pos"] = jpos
    for name in J.FIELDS:
        out[f"jf12/B_{name}"] = ref.field(J._spec(name), jpos)
    out["jf12/striated_12345"] = ref.jf12_random_striated(12345)[:10, :10, :10]
    upos = UF._positions(800, seed=204)
    out["uf23/pos"] = upos
    for name in UF.MODELS:
        out[f"uf23/B_{name}"] = ref.field(UF._spec(name), upos)
    for kind in (0, 1, 2):
        out[f"turbulence/draws_{kind}"] = ref.turbulence_draws(777, kind, 300)
    rng = np.random.default_rng(205)
    v3 = (rng.standard_normal((3, 4, 2, 3)) * 1e-10).astype(np.float32)
    v1 = rng.uniform(-1, 3, (3, 4, 2)).astype(np.float32)
    out["gridfile/v3"], out["gridfile/v1"] = v3, v1
    with tempfile.TemporaryDirectory() as d:
        for key, v, txt, prop in (("v3_raw", v3, False, False), ("v1_raw", v1, False, False),
                                  ("v3_txt", v3, True, True), ("v1_txt", v1, True, True)):
            path = os.path.join(d, key)
            ref.dump_grid(v, path, 2.5, txt=txt, save_prop=prop, origin=(1e19, -2e19, 0.5),
                          spacing=(3e19, 3e19, 3e19), reflective=True, clip=False, interp=1)
            with open(path, "rb") as f:
                out[f"gridfile/{key}"] = np.frombuffer(f.read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "reference_golden_ext.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_golden_ext.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
    main_ext()
