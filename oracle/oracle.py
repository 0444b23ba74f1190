"""TEST INFRASTRUCTURE: Python access to the oracle and to the reference.

* `Oracle` wraps oracle/_build/libcrp_oracle.so, the plain-C restatement of
  the stepping path (crp_oracle.c).
* `Reference` wraps oracle/_ref/libcrp_ref.so, the reference itself compiled
  from its sources with the shim ref_shim.cpp (oracle/Makefile), when it has
  been built (it needs the reference checkout at build time only);
  `Reference(cr_pow=True)` the same sources linked so that every pow call is
  the correctly rounded pow of the engine's FP64 form (libcrp_ref_crpow.so).
* `PluginHarness` wraps oracle/_ref/libcrp_ref_gpu.so: the reference's own
  chain objects run through the product's C++ plugin GpuModuleList
  (crpropa3_b200/plugin), the drop-in for ModuleList::run.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this module;
the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from crpropa3_b200 import _abi
from crpropa3_b200.state import CandidateArrays, RecordArrays

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "libcrp_oracle.so")
ORACLE_CRPOW_LIB = os.path.join(HERE, "_build", "libcrp_oracle_crpow.so")
REF_LIB = os.path.join(HERE, "_ref", "libcrp_ref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libcrp_ref_fast.so")
REF_CRPOW_LIB = os.path.join(HERE, "_ref", "libcrp_ref_crpow.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libcrp_ref_gpu.so")

_dp = C.POINTER(C.c_double)


def build_oracle():
    """Compile the oracle (gcc) if its library is missing or stale."""
    src = os.path.join(HERE, "crp_oracle.c")
    if all(os.path.exists(p) and os.path.getmtime(p) >= os.path.getmtime(src)
           for p in (ORACLE_LIB, ORACLE_CRPOW_LIB)):
        return ORACLE_LIB
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
    return ORACLE_LIB


def _dptr(a):
    return a.ctypes.data_as(_dp)


class Oracle:
    """The oracle.  cr_pow=True loads the build whose step controllers use the
    correctly rounded pow of the device's FP64 form instead of glibc's."""

    def __init__(self, cr_pow=False):
        build_oracle()
        lib = C.CDLL(ORACLE_CRPOW_LIB if cr_pow else ORACLE_LIB)
        lib.oracle_run.restype = C.c_int
        lib.oracle_run.argtypes = [C.POINTER(_abi.PlanDesc), C.POINTER(_abi.Candidates), C.c_uint64,
                                   C.POINTER(_abi.Records), C.c_int, C.c_uint64,
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        lib.oracle_field_eval.argtypes = [C.POINTER(_abi.PlanDesc), C.c_uint64, _dp, _dp]
        lib.oracle_random.argtypes = [C.c_uint32, C.c_int, C.c_uint64, C.c_double, C.c_double,
                                      C.c_double, _dp]
        lib.oracle_plane_wave_modes.argtypes = [C.c_double] * 6 + [C.c_int, C.c_uint32] + [_dp] * 5
        lib.oracle_sample_source.argtypes = [C.c_uint32, C.c_uint64, C.c_int,
                                             C.POINTER(C.c_int32), _dp, C.c_double, C.c_double,
                                             C.c_double, C.POINTER(C.c_int32), _dp, _dp]
        lib.oracle_philox_block.argtypes = [C.POINTER(C.c_uint32)] * 3
        lib.oracle_sample_source_philox.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                                    C.POINTER(C.c_int32), _dp, C.c_int, C.c_double, C.c_double,
                                                    C.c_double, C.c_double, C.c_int, _dp, C.POINTER(C.c_int32),
                                                    _dp, _dp]
        adj = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_int,
               C.c_uint64, _dp, _dp, _dp, _dp, _dp]
        lib.oracle_bp_adjoint.argtypes = adj + [_dp, _dp, _dp, _dp]
        lib.oracle_bp_adjoint.restype = C.c_int
        lib.oracle_bp_loss.argtypes = adj
        lib.oracle_bp_loss.restype = C.c_double
        self.lib = lib

    def run(self, spec, cands: CandidateArrays, records: RecordArrays = None, threads=0,
            max_steps=0):
        desc = spec.desc()
        s = cands.struct()
        rs = records.struct() if records is not None else None
        steps, tries = C.c_uint64(), C.c_uint64()
        r = self.lib.oracle_run(C.byref(desc), C.byref(s), cands.n,
                                C.byref(rs) if rs is not None else None, threads, max_steps,
                                C.byref(steps), C.byref(tries))
        assert r == 0
        return steps.value, tries.value

    def run_textout(self, spec, cands: CandidateArrays, path, output_type, threads=1, seed=0,
                    serial0=1):
        """Run with TextOutput(path, output_type) as every observer's action."""
        self._check(self.lib.ref_run_textout(C.byref(spec.desc()), C.byref(cands.struct()),
                                             cands.n, str(path).encode(), output_type, threads,
                                             seed, serial0))

    def field(self, spec, pos):
        pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).T)
        n = pos.shape[1]
        out = np.zeros((3, n))
        self.lib.oracle_field_eval(C.byref(spec.desc()), n, _dptr(pos), _dptr(out))
        return out.T

    def random(self, seed, kind, n, a=0.0, b=0.0, c=0.0):
        out = np.zeros(n * (3 if kind == 2 else 1))
        assert self.lib.oracle_random(seed, kind, n, a, b, c, _dptr(out)) == 0
        return out

    def plane_wave_modes(self, brms, lmin, lmax, lbendover, s, q, nm, seed):
        xi, kappa = np.zeros(3 * nm), np.zeros(3 * nm)
        k, beta, ak = np.zeros(nm), np.zeros(nm), np.zeros(nm)
        assert self.lib.oracle_plane_wave_modes(brms, lmin, lmax, lbendover, s, q, nm, seed,
                                                _dptr(xi), _dptr(kappa), _dptr(k), _dptr(beta),
                                                _dptr(ak)) == 0
        return xi, kappa, k, beta, ak

    def sample_source(self, seed, n, ids, abundances, emin, emax, index):
        ids = np.asarray(ids, dtype=np.int32)
        ab = np.asarray(abundances if abundances is not None else np.ones(len(ids)), dtype=np.float64)
        out_id, e, d = np.zeros(n, np.int32), np.zeros(n), np.zeros(3 * n)
        assert self.lib.oracle_sample_source(seed, n, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                             _dptr(ab), emin, emax, index,
                                             out_id.ctypes.data_as(C.POINTER(C.c_int32)),
                                             _dptr(e), _dptr(d)) == 0
        return out_id, e, d.reshape(n, 3)

    def sample_source_philox(self, seed, first, n, ids, abundances=None, spectrum=True, emin=1.0, emax=10.0,
                             index=-1.0, energy=1.0, isotropic=True, direction=(1.0, 0.0, 0.0)):
        """The counter-based source draws of crp_source_sample_device, restated:
        (ids, energies, directions as an (n, 3) array)."""
        ids = np.asarray(ids, dtype=np.int32)
        ab = None if abundances is None else np.asarray(abundances, dtype=np.float64)
        dirv = np.asarray(direction, dtype=np.float64)
        out_id, e, d = np.zeros(n, np.int32), np.zeros(n), np.zeros(3 * n)
        assert self.lib.oracle_sample_source_philox(
            seed, first, n, len(ids), ids.ctypes.data_as(C.POINTER(C.c_int32)),
            _dptr(ab) if ab is not None else None, int(spectrum), emin, emax, index, energy, int(isotropic),
            _dptr(dirv), out_id.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(e), _dptr(d)) == 0
        return out_id, e, d.reshape(3, n).T.copy()

    def _adj_args(self, grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target):
        g = np.ascontiguousarray(grid, dtype=np.float32)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (origin, (spacing,) * 3, pos, u0, energy, charge, target)]
        self._keep = (g, arrs)
        o, sp, p, u, e, q, t = arrs
        return (g.ctypes.data_as(C.POINTER(C.c_float)), g.shape[0], g.shape[1], g.shape[2], _dptr(o), _dptr(sp),
                float(step), int(n_steps), len(e), _dptr(p), _dptr(u), _dptr(e), _dptr(q), _dptr(t))

    def bp_adjoint(self, grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target):
        """CPU reference adjoint: (loss per candidate, dL/du0, dL/dE, dL/dgrid)."""
        n = len(energy)
        loss, gu, ge = np.zeros(n), np.zeros(3 * n), np.zeros(n)
        gg = np.zeros(np.asarray(grid).shape, dtype=np.float64)
        args = self._adj_args(grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target)
        assert self.lib.oracle_bp_adjoint(*args, _dptr(loss), _dptr(gu), _dptr(ge), _dptr(gg)) == 0
        return loss, gu.reshape(n, 3), ge, gg

    def bp_loss(self, grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target):
        return self.lib.oracle_bp_loss(*self._adj_args(grid, origin, spacing, step, n_steps, pos, u0,
                                                       energy, charge, target))

    def philox(self, ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        self.lib.oracle_philox_block(c, k, o)
        return list(o)


def reference_available(fast=False, cr_pow=False) -> bool:
    return os.path.exists(REF_FAST_LIB if fast else REF_CRPOW_LIB if cr_pow else REF_LIB)


class Reference:
    """The reference's own modules, driven through ref_shim.cpp."""

    def __init__(self, fast=False, cr_pow=False):
        path = REF_FAST_LIB if fast else REF_CRPOW_LIB if cr_pow else REF_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"reference library {path} is not built (make -C oracle ref)")
        lib = C.CDLL(path)
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = [C.POINTER(_abi.PlanDesc), C.POINTER(_abi.Candidates), C.c_uint64,
                                C.POINTER(_abi.Records), C.c_int, C.c_uint32,
                                C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
        lib.ref_field_eval.argtypes = [C.POINTER(_abi.PlanDesc), C.c_uint64, _dp, _dp]
        lib.ref_random.argtypes = [C.c_uint32, C.c_int, C.c_uint64, C.c_double, C.c_double,
                                   C.c_double, _dp]
        lib.ref_sample_source.argtypes = [C.c_uint32, C.c_uint64, _dp, C.c_int,
                                          C.POINTER(C.c_int32), _dp, C.c_double, C.c_double,
                                          C.c_double, C.POINTER(C.c_int32), _dp, _dp]
        lib.ref_charge.restype = C.c_double
        lib.ref_charge.argtypes = [C.c_int32]
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_run_textout.argtypes = [C.POINTER(_abi.PlanDesc), C.POINTER(_abi.Candidates),
                                        C.c_uint64, C.c_char_p, C.c_int, C.c_int, C.c_uint32,
                                        C.c_uint64]
        lib.ref_text_output.argtypes = [C.c_char_p, C.c_int, C.c_uint64, C.POINTER(C.c_uint64),
                                        C.POINTER(C.c_int32), _dp, _dp, _dp, _dp,
                                        C.POINTER(C.c_int32), _dp, _dp, _dp]
        self.lib = lib

    def _check(self, r):
        if r != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def run(self, spec, cands: CandidateArrays, records: RecordArrays = None, threads=0, seed=0):
        desc = spec.desc()
        s = cands.struct()
        rs = records.struct() if records is not None else None
        steps, secs = C.c_uint64(), C.c_double()
        self._check(self.lib.ref_run(C.byref(desc), C.byref(s), cands.n,
                                     C.byref(rs) if rs is not None else None, threads, seed,
                                     C.byref(steps), C.byref(secs)))
        return steps.value, secs.value

    def run_textout(self, spec, cands: CandidateArrays, path, output_type, threads=1, seed=0,
                    serial0=1):
        """Run with TextOutput(path, output_type) as every observer's action."""
        self._check(self.lib.ref_run_textout(C.byref(spec.desc()), C.byref(cands.struct()),
                                             cands.n, str(path).encode(), output_type, threads,
                                             seed, serial0))

    def field(self, spec, pos):
        pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).T)
        n = pos.shape[1]
        out = np.zeros((3, n))
        self._check(self.lib.ref_field_eval(C.byref(spec.desc()), n, _dptr(pos), _dptr(out)))
        return out.T

    def random(self, seed, kind, n, a=0.0, b=0.0, c=0.0):
        out = np.zeros(n * (3 if kind in (2, 5) else 1))
        self._check(self.lib.ref_random(seed, kind, n, a, b, c, _dptr(out)))
        return out

    def dump_grid(self, values, path, c=1.0, txt=False, save_prop=False, origin=(0, 0, 0), spacing=(1, 1, 1),
                  reflective=False, clip=False, interp=0):
        v = np.ascontiguousarray(values, dtype=np.float32)
        width = 3 if v.ndim == 4 else 1
        o, sp = np.asarray(origin, np.float64), np.asarray(spacing, np.float64)
        self.lib.ref_dump_grid.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                           C.c_char_p, C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_int,
                                           C.c_int]
        self._check(self.lib.ref_dump_grid(v.ctypes.data_as(C.POINTER(C.c_float)), width, *v.shape[:3],
                                           str(path).encode(), c, int(txt), int(save_prop), _dptr(o), _dptr(sp),
                                           int(reflective), int(clip), int(interp)))

    def load_grid(self, shape, path, c=1.0, vector=True, txt=False):
        out = np.zeros(tuple(shape) + ((3,) if vector else ()), np.float32)
        self.lib.ref_load_grid.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                           C.c_char_p, C.c_double, C.c_int]
        self._check(self.lib.ref_load_grid(out.ctypes.data_as(C.POINTER(C.c_float)), 3 if vector else 1,
                                           *shape, str(path).encode(), c, int(txt)))
        return out

    def load_grid_props(self, path, c=1.0, vector=True, capacity=1 << 20):
        shape, o, sp = (C.c_uint64 * 3)(), np.zeros(3), np.zeros(3)
        flags = (C.c_int * 3)()
        vals = np.zeros(capacity, np.float32)
        self.lib.ref_load_grid_props.argtypes = [C.c_char_p, C.c_int, C.c_double, C.POINTER(C.c_uint64), _dp,
                                                 _dp, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_uint64]
        self._check(self.lib.ref_load_grid_props(str(path).encode(), 3 if vector else 1, c, shape, _dptr(o),
                                                 _dptr(sp), flags, vals.ctypes.data_as(C.POINTER(C.c_float)),
                                                 capacity))
        shp = tuple(int(x) for x in shape)
        n = int(np.prod(shp)) * (3 if vector else 1)
        return shp, o, sp, tuple(flags), vals[:n].reshape(shp + ((3,) if vector else ()))

    def turbulence_draws(self, seed, kind, n):
        per = 2 if kind == 0 else 3
        out = np.zeros(per * n)
        self.lib.ref_turbulence_draws.argtypes = [C.c_uint32, C.c_int, C.c_uint64, _dp]
        self._check(self.lib.ref_turbulence_draws(seed, kind, n, _dptr(out)))
        return out.reshape(n, per)

    def jf12_random_striated(self, seed):
        out = np.zeros(100 ** 3, np.float32)
        self.lib.ref_jf12_random_striated.argtypes = [C.c_int, C.POINTER(C.c_float)]
        self._check(self.lib.ref_jf12_random_striated(int(seed), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.reshape(100, 100, 100)

    def sample_source(self, seed, n, position, ids, abundances, emin, emax, index):
        ids = np.asarray(ids, dtype=np.int32)
        ab = np.asarray(abundances if abundances is not None else np.ones(len(ids)), dtype=np.float64)
        pos = np.asarray(position, dtype=np.float64)
        out_id, e, d = np.zeros(n, np.int32), np.zeros(n), np.zeros(3 * n)
        self._check(self.lib.ref_sample_source(seed, n, _dptr(pos), len(ids),
                                               ids.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(ab),
                                               emin, emax, index,
                                               out_id.ctypes.data_as(C.POINTER(C.c_int32)),
                                               _dptr(e), _dptr(d)))
        return out_id, e, d.reshape(n, 3)

    def charge(self, pid):
        return self.lib.ref_charge(pid)

    def text_output(self, path, output_type, serial, ids, energy, pos, dirs, length, src_id,
                    src_e, src_pos, src_dir):
        n = len(serial)
        a = lambda x, t=np.float64: np.ascontiguousarray(x, dtype=t)
        serial, ids, src_id = a(serial, np.uint64), a(ids, np.int32), a(src_id, np.int32)
        energy, pos, dirs, length = a(energy), a(pos), a(dirs), a(length)
        src_e, src_pos, src_dir = a(src_e), a(src_pos), a(src_dir)
        self._check(self.lib.ref_text_output(
            path.encode(), output_type, n, serial.ctypes.data_as(C.POINTER(C.c_uint64)),
            ids.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(energy), _dptr(pos), _dptr(dirs),
            _dptr(length), src_id.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(src_e),
            _dptr(src_pos), _dptr(src_dir)))


def _reference_worker(spec, arrays, n, cr_pow, threads, fast=False, seed=0, rec_capacity=0):
    c = CandidateArrays.__new__(CandidateArrays)
    c.n, c.device = n, None
    for name in CandidateArrays.MEMBERS:
        setattr(c, name, arrays.get(name))
    rec = RecordArrays(rec_capacity) if rec_capacity else None
    Reference(fast=fast, cr_pow=cr_pow).run(spec, c, rec, threads=threads, seed=seed)
    out = {name: getattr(c, name) for name in CandidateArrays.MEMBERS if getattr(c, name) is not None}
    if rec is not None:
        out["__records__"] = {name: getattr(rec, name) for name in RecordArrays.MEMBERS}
        out["__records__"]["count"] = rec.count
    return out


def run_reference_isolated(spec, cands: CandidateArrays, cr_pow=False, threads=0, fast=False, seed=0,
                           records: RecordArrays = None) -> CandidateArrays:
    """Reference.run on a copy of the candidates in a freshly spawned process,
    for callers whose own process has run CUDA work: on the GPU box such
    in-process runs of the reference returned differing current_step and
    flags for every candidate of an adaptive Cash-Karp chain (the cause was
    not found), while a clean process reproduced the device bit for bit.
    `records` (host RecordArrays) is filled with the run's records."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    arrays = {name: getattr(cands, name) for name in cands.MEMBERS if getattr(cands, name) is not None}
    cap = records.capacity if records is not None else 0
    # a failed child raises here (BrokenProcessPool) instead of being respawned
    with ProcessPoolExecutor(max_workers=1, mp_context=mp.get_context("spawn")) as ex:
        out = ex.submit(_reference_worker, spec, arrays, cands.n, cr_pow, threads, fast, seed, cap).result()
    if records is not None:
        for name, a in out.pop("__records__").items():
            getattr(records, name)[...] = a
    c = cands.copy()
    for name, a in out.items():
        setattr(c, name, a)
    return c


def plugin_harness_available() -> bool:
    return os.path.exists(REF_GPU_LIB)


class PluginHarness:
    """The reference's chain objects run through the C++ plugin GpuModuleList
    (ref_gpu_shim.cpp).  describe() and unsupported chains need no device."""

    def __init__(self):
        if not os.path.exists(REF_GPU_LIB):
            raise RuntimeError(f"{REF_GPU_LIB} is not built (make -C oracle ref-gpu)")
        lib = C.CDLL(REF_GPU_LIB)
        pd, cd = C.POINTER(_abi.PlanDesc), C.POINTER(_abi.Candidates)
        lib.ref_gpu_last_error.restype = C.c_char_p
        lib.ref_gpu_run.argtypes = [pd, cd, C.c_uint64, C.POINTER(_abi.Records), C.c_int,
                                    C.c_uint64, C.POINTER(_abi.RunStats), C.POINTER(C.c_uint64)]
        lib.ref_gpu_run_textout.argtypes = [pd, cd, C.c_uint64, C.c_char_p, C.c_int, C.c_int,
                                            C.c_uint64, C.c_uint64]
        lib.ref_run_source_textout.argtypes = [pd, C.c_int, C.c_int, _dp, C.c_int32, C.c_double,
                                               C.c_double, C.c_double, C.c_uint64, C.c_uint64,
                                               C.c_char_p, C.c_int, C.c_uint32, C.c_uint64,
                                               C.POINTER(_abi.RunStats)]
        lib.ref_run_interrupted.argtypes = [pd, cd, C.c_uint64, C.c_int, C.c_uint64, C.c_char_p,
                                            C.POINTER(C.c_int)]
        lib.ref_gpu_describe.argtypes = [pd, C.c_int, C.c_char_p, C.c_size_t]
        lib.ref_gpu_unsupported_throws.argtypes = [pd, C.c_char_p, C.c_size_t]
        self.lib = lib

    def _check(self, r):
        if r != 0:
            raise RuntimeError(self.lib.ref_gpu_last_error().decode())

    def run(self, spec, cands: CandidateArrays, records: RecordArrays = None, precision=0, seed=0):
        """GpuModuleList::run(candidate_vector_t*): (run stats, events replayed)."""
        rs = records.struct() if records is not None else None
        stats, events = _abi.RunStats(), C.c_uint64()
        self._check(self.lib.ref_gpu_run(C.byref(spec.desc()), C.byref(cands.struct()), cands.n,
                                         C.byref(rs) if rs is not None else None, precision, seed,
                                         C.byref(stats), C.byref(events)))
        return stats, events.value

    def run_textout(self, spec, cands: CandidateArrays, path, output_type, precision=0, seed=0,
                    serial0=1):
        self._check(self.lib.ref_gpu_run_textout(C.byref(spec.desc()), C.byref(cands.struct()),
                                                 cands.n, str(path).encode(), output_type,
                                                 precision, seed, serial0))

    def run_source_textout(self, spec, gpu, position, pid, emin, emax, index, count, path,
                           output_type, seed=1, serial0=1, batch=0, precision=0):
        """run(source, count) of SourcePosition + SourceParticleType +
        SourcePowerLawSpectrum + SourceIsotropicEmission, on the plugin (gpu)
        or on the reference's ModuleList with one thread."""
        pos = np.ascontiguousarray(position, dtype=np.float64)
        stats = _abi.RunStats()
        self._check(self.lib.ref_run_source_textout(
            C.byref(spec.desc()), 1 if gpu else 0, precision, _dptr(pos), pid, emin, emax, index,
            count, batch, str(path).encode(), output_type, seed, serial0, C.byref(stats)))
        return stats

    def run_interrupted(self, spec, cands: CandidateArrays, path, gpu, batch=0):
        """run(candidates) with SIGINT sent at the first detection and a
        TextOutput(path) interrupt action, on the plugin (gpu, batches of
        `batch`) or on the reference's ModuleList (one thread).  Returns the
        signal the run raised again at its end (0: none)."""
        reraised = C.c_int()
        self._check(self.lib.ref_run_interrupted(C.byref(spec.desc()), C.byref(cands.struct()),
                                                 cands.n, 1 if gpu else 0, batch,
                                                 str(path).encode(), C.byref(reraised)))
        return reraised.value

    def describe(self, spec, extra=0):
        """(on the device path?, plan text or reason) without a device."""
        buf = C.create_string_buffer(1 << 16)
        r = self.lib.ref_gpu_describe(C.byref(spec.desc()), extra, buf, len(buf))
        if r < 0:
            raise RuntimeError(buf.value.decode())
        return r == 1, buf.value.decode()

    def unsupported_run_message(self, spec):
        buf = C.create_string_buffer(4096)
        r = self.lib.ref_gpu_unsupported_throws(C.byref(spec.desc()), buf, len(buf))
        return (buf.value.decode() if r == 1 else None)
