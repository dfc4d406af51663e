"""K-step MHM evolution of a periodic uniform box and its hand-written adjoint.

``mhm_steps(box, K, solver, params)`` advances a periodic box (torch CUDA tensor
``[5][Z][Y][X]``, x fastest, dimensions multiples of 16) by K solver steps: each step fills the
ghost zones of every patch group from the box (gb_box_gather_device, the single-level, periodic
case of GAMER's Prepare_PatchData), solves all patch groups (gb_fluid_solve_device) and writes the
interiors back (gb_box_scatter_device).  It is a ``torch.autograd.Function``: the forward pass keeps
the box of every step as a checkpoint; the backward pass walks the steps in reverse, re-gathers the
windows of step k from its checkpoint and applies the adjoint of the solver step
(gb_fluid_adjoint_step_device) and of the ghost-zone gather (gb_box_gather_adjoint_device).
Gradients are accumulated in double.
"""
from __future__ import annotations

import ctypes

import torch

from gamer_b200.fluid import FluidSolver, SolverParams, _check, _dptr

PS2 = 16


def _dims(box):
    nc, Z, Y, X = box.shape
    assert X % PS2 == 0 and Y % PS2 == 0 and Z % PS2 == 0, "box dimensions must be multiples of 16"
    return nc, X // PS2, Y // PS2, Z // PS2


def _prec(solver):
    return 2 if solver.precision == "fp64" else 0


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def gather(solver, box):
    nc, npx, npy, npz = _dims(box)
    win = torch.empty((npx * npy * npz, nc, solver.flu_nxt, solver.flu_nxt, solver.flu_nxt), dtype=box.dtype,
                      device=box.device)
    _check(solver.lib.gb_box_gather_device(_dptr(box), _dptr(win), npx, npy, npz, solver.flu_nxt, nc, _prec(solver),
                                           _stream()), "gb_box_gather_device")
    return win


def scatter(solver, out, like):
    nc, npx, npy, npz = _dims(like)
    box = torch.empty_like(like)
    _check(solver.lib.gb_box_scatter_device(_dptr(out), _dptr(box), npx, npy, npz, nc, _prec(solver), _stream()),
           "gb_box_scatter_device")
    return box


def step(solver, box, params: SolverParams):
    win = gather(solver, box)
    out = torch.empty((win.shape[0], box.shape[0], PS2, PS2, PS2), dtype=box.dtype, device=box.device)
    p = SolverParams(**{**params.__dict__, "StoreFlux": False})
    solver.solve_device(win, out, p)
    return scatter(solver, out, box)


def adjoint_step(solver, box, gbox, params: SolverParams, ws_pg=1024):
    """d loss / d box_k from d loss / d box_{k+1} (double), for the step taken from box_k.  The
    adjoint kernels run over at most ``ws_pg`` patch groups at a time (~2.8 MB of workspace each in
    FP32)."""
    nc, npx, npy, npz = _dims(box)
    npg = npx * npy * npz
    win = gather(solver, box)
    gout = torch.empty((npg, nc, PS2, PS2, PS2), dtype=torch.float64, device=box.device)
    _check(solver.lib.gb_box_scatter_adjoint_device(_dptr(gbox), _dptr(gout), npx, npy, npz, nc, _stream()),
           "gb_box_scatter_adjoint_device")
    gin = torch.empty((npg, nc) + (solver.flu_nxt,) * 3, dtype=torch.float64, device=box.device)
    nbytes = ctypes.c_ulonglong()
    _check(solver.lib.gb_fluid_adjoint_workspace_bytes(solver.h, min(npg, ws_pg), ctypes.byref(nbytes)),
           "gb_fluid_adjoint_workspace_bytes")
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=box.device)
    p = params.c()
    _check(solver.lib.gb_fluid_adjoint_step_device(solver.h, _dptr(win), _dptr(gout), _dptr(gin), npg,
                                                   ctypes.byref(p), _dptr(ws), nbytes.value, _stream()),
           "gb_fluid_adjoint_step_device")
    g = torch.empty(box.shape, dtype=torch.float64, device=box.device)
    _check(solver.lib.gb_box_gather_adjoint_device(_dptr(gin), _dptr(g), npx, npy, npz, solver.flu_nxt, nc,
                                                   _stream()), "gb_box_gather_adjoint_device")
    return g


class MHMSteps(torch.autograd.Function):
    """box_K = step^K(box_0); backward by the hand-written adjoint with per-step checkpoints."""

    @staticmethod
    def forward(ctx, box, solver, K, params):
        boxes = [box.detach()]
        cur = boxes[0]
        for _ in range(K):
            cur = step(solver, cur, params)
            boxes.append(cur)
        ctx.solver, ctx.K, ctx.params = solver, K, params
        ctx.save_for_backward(*boxes[:-1])          # checkpoints U_0 .. U_{K-1}
        return cur

    @staticmethod
    def backward(ctx, gK):
        boxes = ctx.saved_tensors
        g = gK.to(torch.float64).contiguous()
        for k in reversed(range(ctx.K)):
            g = adjoint_step(ctx.solver, boxes[k], g, ctx.params)
        return g.to(boxes[0].dtype), None, None, None


def mhm_steps(box, K, solver: FluidSolver, params: SolverParams):
    return MHMSteps.apply(box, solver, K, params)
