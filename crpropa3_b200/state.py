"""Structure-of-arrays candidate state and output records.

The device layout is one contiguous array per Candidate member
(include/crpropa/Candidate.h:27, ParticleState.h:22): position, direction,
previous position, energy, charge, trajectory length, time, current and next
step, active flag, condition flags, optional per-candidate maximum length and
the accepted-step counter (the counter of the device random stream).  The
same class holds host (numpy) or device (torch) arrays; `struct()` gives the
crp_candidates view the C-ABI takes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

_NP = {C.c_int32: np.int32, C.c_double: np.float64, C.c_uint8: np.uint8,
       C.c_uint32: np.uint32, C.c_uint64: np.uint64}


def _torch_dtype(ct):
    import torch
    return {C.c_int32: torch.int32, C.c_double: torch.float64, C.c_uint8: torch.uint8,
            C.c_uint32: torch.int32, C.c_uint64: torch.int64}[ct]


def _ptr(arr, ct):
    if arr is None:
        return C.POINTER(ct)()
    if isinstance(arr, np.ndarray):
        return arr.ctypes.data_as(C.POINTER(ct))
    return C.cast(C.c_void_p(arr.data_ptr()), C.POINTER(ct))


class CandidateArrays:
    """n candidates as one array per member (numpy on host, torch on device)."""

    MEMBERS = [name for name, _ in _abi.CANDIDATE_FIELDS]
    OPTIONAL = ("max_length",)

    def __init__(self, n: int, per_candidate_length: bool = False, device=None):
        self.n = int(n)
        self.device = device
        for name, ct in _abi.CANDIDATE_FIELDS:
            if name in self.OPTIONAL and not per_candidate_length:
                setattr(self, name, None)
                continue
            if device is None:
                arr = np.zeros(self.n, dtype=_NP[ct])
            else:
                import torch
                arr = torch.zeros(self.n, dtype=_torch_dtype(ct), device=device)
            setattr(self, name, arr)
        if device is None:
            self.active[:] = 1

    # -- views -------------------------------------------------------------
    def struct(self) -> _abi.Candidates:
        s = _abi.Candidates()
        for name, ct in _abi.CANDIDATE_FIELDS:
            setattr(s, name, _ptr(getattr(self, name), ct))
        return s

    def members(self):
        return {name: getattr(self, name) for name in self.MEMBERS if getattr(self, name) is not None}

    def copy(self) -> "CandidateArrays":
        out = CandidateArrays.__new__(CandidateArrays)
        out.n, out.device = self.n, self.device
        for name in self.MEMBERS:
            a = getattr(self, name)
            setattr(out, name, None if a is None else (a.copy() if isinstance(a, np.ndarray) else a.clone()))
        return out

    def head(self, k: int) -> "CandidateArrays":
        """A copy of the first k candidates (host or device arrays)."""
        k = min(int(k), self.n)
        out = CandidateArrays.__new__(CandidateArrays)
        out.n, out.device = k, self.device
        for name in self.MEMBERS:
            a = getattr(self, name)
            if a is None:
                setattr(out, name, None)
            else:
                setattr(out, name, np.ascontiguousarray(a[:k]) if isinstance(a, np.ndarray)
                        else a[:k].clone())
        return out

    def to_device(self, device="cuda") -> "CandidateArrays":
        import torch
        out = CandidateArrays.__new__(CandidateArrays)
        out.n, out.device = self.n, device
        for name, ct in _abi.CANDIDATE_FIELDS:
            a = getattr(self, name)
            if a is None:
                setattr(out, name, None)
                continue
            t = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else
                                 a.view(np.int64) if a.dtype == np.uint64 else a)
            setattr(out, name, t.to(device))
        return out

    def to_host(self) -> "CandidateArrays":
        if self.device is None:
            return self.copy()
        out = CandidateArrays.__new__(CandidateArrays)
        out.n, out.device = self.n, None
        for name, ct in _abi.CANDIDATE_FIELDS:
            a = getattr(self, name)
            if a is None:
                setattr(out, name, None)
                continue
            h = a.cpu().numpy()
            setattr(out, name, h.view(_NP[ct]))
        return out

    # -- convenience -------------------------------------------------------
    def position(self):
        return np.stack([self.x, self.y, self.z], axis=1)

    def direction(self):
        return np.stack([self.dx, self.dy, self.dz], axis=1)

    def set_position(self, pos):
        pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        self.x[:], self.y[:], self.z[:] = pos[:, 0], pos[:, 1], pos[:, 2]
        self.px[:], self.py[:], self.pz[:] = pos[:, 0], pos[:, 1], pos[:, 2]

    def set_direction(self, d):
        d = np.asarray(d, dtype=np.float64).reshape(-1, 3)
        self.dx[:], self.dy[:], self.dz[:] = d[:, 0], d[:, 1], d[:, 2]

    def nbytes(self) -> int:
        tot = 0
        for name in self.MEMBERS:
            a = getattr(self, name)
            if a is None:
                continue
            tot += a.nbytes if isinstance(a, np.ndarray) else a.numel() * a.element_size()
        return tot


class RecordArrays:
    """Output records (detection / rejection actions), numpy host arrays."""

    MEMBERS = [name for name, _ in _abi.RECORD_FIELDS]

    def __init__(self, capacity: int, device=None):
        self.capacity = int(capacity)
        self.device = device
        for name, ct in _abi.RECORD_FIELDS:
            if device is None:
                setattr(self, name, np.zeros(self.capacity, dtype=_NP[ct]))
            else:
                import torch
                setattr(self, name, torch.zeros(self.capacity, dtype=_torch_dtype(ct), device=device))
        if device is None:
            self.count = np.zeros(1, dtype=np.uint64)
        else:
            import torch
            self.count = torch.zeros(1, dtype=torch.int64, device=device)

    def struct(self) -> _abi.Records:
        s = _abi.Records()
        s.capacity = self.capacity
        s.count = _ptr(self.count, C.c_uint64)
        for name, ct in _abi.RECORD_FIELDS:
            setattr(s, name, _ptr(getattr(self, name), ct))
        return s

    def n(self) -> int:
        c = int(self.count[0])
        return min(c, self.capacity)

    def to_host(self) -> "RecordArrays":
        if self.device is None:
            return self
        out = RecordArrays.__new__(RecordArrays)
        out.capacity, out.device = self.capacity, None
        for name, ct in _abi.RECORD_FIELDS:
            setattr(out, name, getattr(self, name).cpu().numpy().view(_NP[ct]))
        out.count = self.count.cpu().numpy().view(np.uint64)
        return out

    def sorted(self):
        """Records as a dict of arrays sorted by (candidate index, module)."""
        k = self.n()
        order = np.lexsort((self.module[:k], self.index[:k]))
        return {name: getattr(self, name)[:k][order] for name in self.MEMBERS}
