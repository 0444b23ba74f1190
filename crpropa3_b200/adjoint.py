"""Differentiable fixed-step Boris backtracking (crp_bp_adjoint).

`arrival_loss(p0, grid, ...)` returns L = sum_i (1 - u_final,i . target_i)
for candidates with initial momenta p0 (n, 3) [kg m/s] propagated with a
fixed-step Boris push through a periodic Grid3f whose values `grid`
(nx, ny, nz, 3) float32 are differentiated too.  The forward pass calls
crp_bp_forward_loss (no checkpoints kept); backward calls crp_bp_adjoint,
which recomputes the forward pass with FP64 checkpoints every
`checkpoint_every` steps and runs the hand-written adjoint.  PyTorch is only
the autograd wrapper: both passes are the engine's CUDA kernels.

With p0 = (E/c) u0:  dL/dp0 = (I - u0 u0^T) dL/du0 / |p0| + c u0 dL/dE.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi
from . import units as U


def _desc(grid, origin, spacing, step, n_steps, k):
    d = _abi.AdjointDesc()
    d.grid_values = grid.data_ptr()
    d.nx, d.ny, d.nz = grid.shape[:3]
    d.origin[:] = tuple(float(v) for v in origin)
    d.spacing[:] = (float(spacing),) * 3 if not hasattr(spacing, "__len__") else tuple(spacing)
    d.step = float(step)
    d.n_steps = int(n_steps)
    d.checkpoint_every = int(k)
    return d


def _io(n, pos, u0, energy, charge, target, loss, uf=None, gu=None, ge=None, gg=None):
    io = _abi.AdjointIO()
    io.n = n
    p = lambda t: t.data_ptr() if t is not None else None
    io.x, io.y, io.z = p(pos[0]), p(pos[1]), p(pos[2])
    io.dx, io.dy, io.dz = p(u0[0]), p(u0[1]), p(u0[2])
    io.energy, io.charge = p(energy), p(charge)
    io.tx, io.ty, io.tz = p(target[0]), p(target[1]), p(target[2])
    io.loss = p(loss)
    if uf is not None:
        io.ux, io.uy, io.uz = p(uf[0]), p(uf[1]), p(uf[2])
    if gu is not None:
        io.grad_dx, io.grad_dy, io.grad_dz = p(gu[0]), p(gu[1]), p(gu[2])
    io.grad_energy = p(ge)
    io.grad_grid = p(gg)
    return io


def _planar(t):
    t = t.to(torch.float64)
    return [t[:, k].contiguous() for k in range(3)]


def bp_loss_and_grads(grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target,
                      checkpoint_every=100, want_grid=True, stream=None):
    """Direct call of crp_bp_adjoint on device tensors: (loss per candidate,
    dL/du0 (n,3), dL/dE (n,), dL/dgrid or None)."""
    lib = _abi.load()
    grid = grid.contiguous()
    n = u0.shape[0]
    d = _desc(grid, origin, spacing, step, n_steps, checkpoint_every)
    need = C.c_size_t()
    _abi.check(lib.crp_bp_adjoint_workspace(C.byref(d), n, C.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device=grid.device)
    dev = grid.device
    loss = torch.empty(n, dtype=torch.float64, device=dev)
    gu = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(3)]
    ge = torch.empty(n, dtype=torch.float64, device=dev)
    gg = torch.empty(grid.shape, dtype=torch.float64, device=dev) if want_grid else None
    pos_p, u_p, t_p = _planar(pos), _planar(u0), _planar(target)
    io = _io(n, pos_p, u_p, energy.to(torch.float64).contiguous(), charge.to(torch.float64).contiguous(),
             t_p, loss, None, gu, ge, gg)
    _abi.check(lib.crp_bp_adjoint(C.byref(d), C.byref(io), C.c_void_p(ws.data_ptr()), need.value,
                                  stream))
    return loss, torch.stack(gu, 1), ge, gg


class _Tape:
    """Inputs, outputs and workspace of one checkpointed forward pass."""

    def __init__(self, grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target, k):
        lib = _abi.load()
        self.grid = grid.contiguous()
        self.n = u0.shape[0]
        self.desc = _desc(self.grid, origin, spacing, step, n_steps, k)
        need = C.c_size_t()
        _abi.check(lib.crp_bp_adjoint_workspace(C.byref(self.desc), self.n, C.byref(need)))
        dev = self.grid.device
        self.ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
        self.need = need.value
        self.loss = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.gu = [torch.empty(self.n, dtype=torch.float64, device=dev) for _ in range(3)]
        self.ge = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.inputs = (_planar(pos), _planar(u0), energy.to(torch.float64).contiguous(),
                       charge.to(torch.float64).contiguous(), _planar(target))
        self.gg = None

    def io(self):
        p, u, e, q, t = self.inputs
        return _io(self.n, p, u, e, q, t, self.loss, None, self.gu, self.ge, self.gg)


def bp_adjoint_forward(grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target,
                       checkpoint_every=100, stream=None):
    """Checkpointed forward pass (crp_bp_adjoint_forward): returns the tape."""
    tape = _Tape(grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target, checkpoint_every)
    io = tape.io()
    _abi.check(_abi.load().crp_bp_adjoint_forward(C.byref(tape.desc), C.byref(io),
                                                  C.c_void_p(tape.ws.data_ptr()), tape.need, stream))
    return tape


def bp_adjoint_backward(tape, want_grid=True, stream=None):
    """Reverse pass over a tape (crp_bp_adjoint_backward): dL/du0, dL/dE, dL/dgrid."""
    tape.gg = (torch.empty(tape.grid.shape, dtype=torch.float64, device=tape.grid.device)
               if want_grid else None)
    io = tape.io()
    _abi.check(_abi.load().crp_bp_adjoint_backward(C.byref(tape.desc), C.byref(io),
                                                   C.c_void_p(tape.ws.data_ptr()), tape.need, stream))
    return torch.stack(tape.gu, 1), tape.ge, tape.gg


def bp_forward_loss(grid, origin, spacing, step, n_steps, pos, u0, energy, charge, target,
                    stream=None):
    lib = _abi.load()
    grid = grid.contiguous()
    n = u0.shape[0]
    d = _desc(grid, origin, spacing, step, n_steps, 1)
    loss = torch.empty(n, dtype=torch.float64, device=grid.device)
    uf = [torch.empty(n, dtype=torch.float64, device=grid.device) for _ in range(3)]
    io = _io(n, _planar(pos), _planar(u0), energy.to(torch.float64).contiguous(),
             charge.to(torch.float64).contiguous(), _planar(target), loss, uf)
    _abi.check(lib.crp_bp_forward_loss(C.byref(d), C.byref(io), stream))
    return loss, torch.stack(uf, 1)


class BorisArrivalLoss(torch.autograd.Function):
    """L(p0, grid) = sum_i (1 - u_final,i . target_i) through fixed-step Boris."""

    @staticmethod
    def forward(ctx, p0, grid, pos, charge, target, origin, spacing, step, n_steps, checkpoint_every):
        pn = p0.detach().norm(dim=1)
        u0 = p0.detach() / pn[:, None]
        energy = pn * U.c_light
        tape = bp_adjoint_forward(grid.detach(), origin, spacing, step, n_steps, pos, u0, energy,
                                  charge, target, checkpoint_every)
        ctx.tape = tape
        ctx.save_for_backward(p0.detach())
        return tape.loss.sum()

    @staticmethod
    def backward(ctx, gout):
        (p0,) = ctx.saved_tensors
        pn = p0.norm(dim=1)
        u0 = p0 / pn[:, None]
        gu, ge, gg = bp_adjoint_backward(ctx.tape, want_grid=ctx.needs_input_grad[1])
        grid = ctx.tape.grid
        ctx.tape = None
        # dL/dp0 = (I - u u^T) dL/du / |p| + c u dL/dE
        tang = gu - u0 * (u0 * gu).sum(1, keepdim=True)
        gp = tang / pn[:, None] + U.c_light * u0 * ge[:, None]
        gp = (gp * gout).to(p0.dtype)
        ggrid = (gg * gout).to(grid.dtype) if gg is not None else None
        return gp, ggrid, None, None, None, None, None, None, None, None


def arrival_loss(p0, grid, pos, charge, target, origin, spacing, step, n_steps,
                 checkpoint_every=100):
    return BorisArrivalLoss.apply(p0, grid, pos, charge, target, origin, spacing, step, n_steps,
                                  checkpoint_every)
