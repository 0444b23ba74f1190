"""The C-ABI library: loads, exports every declared symbol, and its host-side
entry points (no device needed) agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helpers import P, ROOT, U, _abi, bp_fixed


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "crp_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:crp_status|uint32_t)\s+(crp_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = _declared_symbols()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name
    from crpropa3_b200 import _signatures
    assert set(names) <= set(_signatures.SIGNATURES), set(names) - set(_signatures.SIGNATURES)


def test_abi_version():
    assert _abi.load().crp_abi_version() == _abi.ABI_VERSION


def test_struct_layouts_match_the_header():
    """Sizes of the ctypes mirrors against a C compile of the header."""
    import subprocess
    import tempfile
    src = ('#include "crp_gpu.h"\n#include <stdio.h>\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
           'sizeof(crp_field_component), sizeof(crp_module_desc), sizeof(crp_plan_desc),'
           'sizeof(crp_candidates), sizeof(crp_records), sizeof(crp_run_opts), sizeof(crp_run_stats),'
           'sizeof(crp_source_desc), sizeof(crp_noalloc_grid_bp_desc));}\n')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    mine = [C.sizeof(t) for t in (_abi.FieldComponent, _abi.ModuleDesc, _abi.PlanDesc, _abi.Candidates,
                                  _abi.Records, _abi.RunOpts, _abi.RunStats, _abi.SourceDesc,
                                  _abi.NoAllocGridBpDesc)]
    assert mine == sizes


def test_particle_charge():
    lib = _abi.load()
    q = C.c_double()
    for pid, z in ((1000010010, 1), (1000260560, 26), (-1000010010, -1), (1000020040, 2), (2112, 0),
                   (22, 0), (11, -1), (-11, 1)):
        assert lib.crp_particle_charge(pid, C.byref(q)) == _abi.OK
        assert q.value == z * U.eplus
    assert lib.crp_particle_charge(211, C.byref(q)) == _abi.ERR_UNSUPPORTED


@pytest.mark.parametrize("kind,args", [(0, ()), (1, (-3.0, 5.0)), (2, ()), (3, (-1.0, 1.0, 100.0)),
                                       (3, (-2.0, 0.1, 100.0)), (6, ())])
def test_random_draws_match_oracle(oracle, kind, args):
    lib = _abi.load()
    n = 2000
    out = np.zeros(n * (3 if kind == 2 else 1))
    a = list(args) + [0.0] * (3 - len(args))
    assert lib.crp_random_draws(1234, kind, n, *a, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
    np.testing.assert_array_equal(out, oracle.random(1234, kind, n, *a))


def test_plane_wave_modes_match_oracle(oracle):
    lib = _abi.load()
    nm = 128
    arrs = [np.zeros(3 * nm), np.zeros(3 * nm), np.zeros(nm), np.zeros(nm), np.zeros(nm)]
    ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
    args = (0.5 * U.muG, 1 * U.pc, 100 * U.pc, 1.0, 5 / 3, 4.0)
    assert lib.crp_plane_wave_modes(*args, nm, 42, *ptrs) == 0
    for got, ref in zip(arrs, oracle.plane_wave_modes(*args, nm, 42)):
        np.testing.assert_array_equal(got, ref)
    assert lib.crp_plane_wave_modes(*args, 1, 42, *ptrs) == _abi.ERR_INVALID_ARGUMENT
    assert "Nm <= 1" in _abi.last_error()


def test_source_sample_matches_oracle(oracle):
    from crpropa3_b200 import workloads as W
    ids = [W.IDS[k] for k in ("H", "He", "N", "Fe")]
    c = W.source_candidates(3000, ids, 0.1 * U.EeV, 100 * U.EeV, -2.0, 5)
    oid, oe, od = oracle.sample_source(5, 3000, ids, None, 0.1 * U.EeV, 100 * U.EeV, -2.0)
    np.testing.assert_array_equal(c.id, oid)
    np.testing.assert_array_equal(c.energy, oe)
    np.testing.assert_array_equal(c.direction(), od)


@pytest.mark.parametrize("bad,msg", [
    (dict(tolerance=2.0), "PropagationBP: target error not in range 0-1"),
    (dict(min_step=-1.0), "PropagationBP: minStep < 0"),
    (dict(min_step=2.0, max_step=1.0), "PropagationBP: minStep > maxStep"),
])
def test_plan_validation_messages(bad, msg):
    kw = dict(tolerance=0.1, min_step=1.0, max_step=1.0)
    kw.update(bad)
    spec = P.ChainSpec([P.UniformField((0, 0, 1e-13))],
                       [P.Propagation(_abi.PROP_BP, kw["tolerance"], kw["min_step"], kw["max_step"])])
    from crpropa3_b200.engine import Plan
    with pytest.raises(_abi.CrpError) as e:
        Plan(spec)
    assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    assert msg in str(e.value)


def test_plan_rejects_chains_off_the_device_path():
    from crpropa3_b200.engine import Plan
    spec = P.ChainSpec([P.UniformField((0, 0, 1e-13))], [P.MaxTrajectoryLength(1.0)])
    with pytest.raises(_abi.CrpError) as e:
        Plan(spec)
    assert e.value.status == _abi.ERR_UNSUPPORTED
    spec = P.ChainSpec([P.UniformField((0, 0, 1e-13))], [bp_fixed(1.0), bp_fixed(1.0)])
    with pytest.raises(_abi.CrpError) as e:
        Plan(spec)
    assert e.value.status == _abi.ERR_UNSUPPORTED


def test_sde_validation_messages():
    from crpropa3_b200.engine import Plan
    for kw, msg in ((dict(epsilon=2.0), "epsilon not in range 0-1"),
                    (dict(alpha=3.0), "alpha not in range 0-2"),
                    (dict(scale=-1.0), "Scale < 0")):
        spec = P.ChainSpec([P.UniformField((0, 0, 1e-13))],
                           [P.Propagation(_abi.PROP_SDE, 1e-4, 1.0, 10.0, **kw)])
        with pytest.raises(_abi.CrpError) as e:
            Plan(spec)
        assert msg in str(e.value)
