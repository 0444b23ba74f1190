"""Python handle on the C-ABI engine: plans, runs, field evaluation.

Every call goes through include/crp_gpu.h; there is no Python or CPU
implementation of the stepping path behind it.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from .plan import ChainSpec
from .state import CandidateArrays, RecordArrays


def device_count() -> int:
    lib = _abi.load()
    n = C.c_int32(0)
    st = lib.crp_device_count(C.byref(n))
    return n.value if st == _abi.OK else 0


class Plan:
    """A validated, device-resident stepping plan (crp_plan_create)."""

    def __init__(self, spec: ChainSpec):
        self.lib = _abi.load()
        self.spec = spec
        self._desc = spec.desc()
        h = C.c_void_p()
        _abi.check(self.lib.crp_plan_create(C.byref(self._desc), C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.crp_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _opts(mode=_abi.MODE_AUTO, block_size=0, steps_per_launch=0, max_steps=0, stream=None,
              records: Optional[RecordArrays] = None, cancel=None, ctas_per_sm=0,
              refill_threshold=0, budget_us=0):
        o = _abi.RunOpts()
        o.mode, o.block_size, o.steps_per_launch = mode, block_size, steps_per_launch
        o.max_steps, o.ctas_per_sm, o.refill_threshold = max_steps, ctas_per_sm, refill_threshold
        o.budget_us = budget_us
        o.stream = stream
        keep = []
        if records is not None:
            rs = records.struct()
            keep.append(rs)
            o.records = C.pointer(rs)
        if cancel is not None:
            o.cancel = cancel
        return o, keep

    def run(self, cands: CandidateArrays, **kw) -> _abi.RunStats:
        """Run host (numpy) or device (torch) candidate arrays to completion."""
        o, keep = self._opts(**kw)
        s = cands.struct()
        stats = _abi.RunStats()
        fn = self.lib.crp_run if cands.device is None else self.lib.crp_run_device
        _abi.check(fn(self.handle, C.byref(s), cands.n, C.byref(o), C.byref(stats)))
        del keep
        return stats

    def autotune(self, device_cands: CandidateArrays, sample_n=1 << 17, steps_per_candidate=256,
                 stream=None) -> _abi.AutotuneResult:
        """Time launch configurations on a sample of device candidates; the
        best is used by later runs in MODE_AUTO (crp_autotune)."""
        res = _abi.AutotuneResult()
        s = device_cands.struct()
        _abi.check(self.lib.crp_autotune(self.handle, C.byref(s), device_cands.n, sample_n,
                                         steps_per_candidate, stream, C.byref(res)))
        return res

    def field(self, pos) -> np.ndarray:
        """Field of the plan at positions (n, 3) [m] -> (n, 3) [T], on the device."""
        import torch
        pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        n = pos.shape[0]
        dpos = torch.from_numpy(np.ascontiguousarray(pos.T)).cuda()
        out = torch.zeros((3, n), dtype=torch.float64, device="cuda")
        _abi.check(self.lib.crp_field_eval(self.handle, n, C.c_void_p(dpos.data_ptr()),
                                           C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        return out.cpu().numpy().T.copy()
