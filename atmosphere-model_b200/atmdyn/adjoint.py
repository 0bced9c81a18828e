"""PyTorch binding of the FP64 step and its hand-written adjoint.

:class:`DycoreSegment` is a ``torch.autograd.Function`` that advances the
prognostic interior (dp, pt, ud, vd as float64 CUDA tensors of shape
(nlay, ny, nx)) through a segment of steps with libatmdyn.  Its forward
keeps only the segment's initial state (a checkpoint).  Its backward
restores that state, recomputes the segment once keeping each step's
tape (``atm_step_tape``: its initial state and forward products), and then
runs the adjoint steps in reverse order from the tapes
(``atm_adj_step_tape``: the CUDA adjoint kernels of the sweeps, the remap
and the halo fills, with the limiter branches of the recomputed forward).
:func:`integrate` chains segments of ``checkpoint_every`` steps, so memory
grows with the number of checkpoints plus one segment of states.  The
last segment's forward records its tapes as it goes (the backward starts
there and would recompute it at once), so its backward recomputes
nothing; the peak memory is the same one segment of tapes.

The step is the reference's time loop (src/mod_model.f90:146-177): C-grid
half step, C-grid halo, D-grid step, vertical remap every ``remap_every``
steps, D-grid halo.  The heating term is held at zero.
"""
from __future__ import annotations

import torch

from .dycore import Dycore

FIELD_NAMES = ('dp', 'pt', 'ud', 'vd')


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the handle of the legacy default stream


def _bind_stream(dyn: Dycore):
    """Enqueue the library's work on torch's current stream.  torch reports
    the legacy default stream as handle 0, which atm_set_stream reads as
    'use your own stream', so that case passes cudaStreamLegacy."""
    h = torch.cuda.current_stream().cuda_stream
    dyn.set_stream(h if h else CUDA_STREAM_LEGACY)


def _upload(dyn: Dycore, fields):
    from ._lib import ATM_DP, ATM_PT, ATM_UD, ATM_VD
    for f, t in zip((ATM_DP, ATM_PT, ATM_UD, ATM_VD), fields):
        t = t.detach().contiguous()
        assert t.dtype == torch.float64 and t.is_cuda
        dyn.upload_device(f, t)


def _download(dyn: Dycore, like):
    from ._lib import ATM_DP, ATM_PT, ATM_UD, ATM_VD
    outs = []
    for f in (ATM_DP, ATM_PT, ATM_UD, ATM_VD):
        o = torch.empty_like(like)
        dyn.download_device(f, o)
        outs.append(o)
    return outs


def _record(dyn: Dycore, dt: float, remaps, like, final_state: bool = True):
    """Steps from the context's current state keeping, per step, its tape
    (the initial state and the forward products the adjoint step reads).
    Without ``final_state`` the last step stops before its remap: its tape
    holds the pre-remap state the remap's adjoint needs (the adjoint step
    is told separately that the step remapped), and the remapped state
    itself, the segment's output, is not wanted (a backward's recompute)."""
    tapes = []
    n = len(remaps)
    for i, r in enumerate(remaps):
        tp = torch.empty(dyn.tape_bytes() // 8, dtype=torch.float64, device=like.device)
        remap = bool(r) and (final_state or i + 1 < n)
        dyn.step_tape(dt, remap, tp.data_ptr())
        tapes.append(tp)
    return tapes


class DycoreSegment(torch.autograd.Function):
    """(dp, pt, ud, vd) -> the state after ``len(remaps)`` steps of size dt;
    remaps[i] says whether step i ends with the vertical remap.  With
    ``record`` the forward keeps every step's tape (the segment the
    backward starts with) instead of a checkpoint."""

    @staticmethod
    def forward(ctx, dyn: Dycore, dt: float, remaps, record: bool, dp, pt, ud, vd):
        _bind_stream(dyn)
        _upload(dyn, (dp, pt, ud, vd))
        ctx.dyn, ctx.dt, ctx.remaps = dyn, dt, tuple(bool(r) for r in remaps)
        if record:
            ctx.trajectory = _record(dyn, dt, ctx.remaps, dp)
            ckpt = torch.empty(0, dtype=torch.float64, device=dp.device)
        else:
            ctx.trajectory = None
            ckpt = torch.empty(dyn.state_bytes() // 8, dtype=torch.float64, device=dp.device)
            dyn.state_save(ckpt.data_ptr())
            for r in ctx.remaps:
                dyn.step(dt, remap=r, check_stable=False)
        outs = _download(dyn, dp)
        ctx.save_for_backward(ckpt)
        ctx.mark_non_differentiable()
        return tuple(outs)

    @staticmethod
    def backward(ctx, gdp, gpt, gud, gvd):
        dyn, dt, remaps = ctx.dyn, ctx.dt, ctx.remaps
        (ckpt,) = ctx.saved_tensors
        _bind_stream(dyn)
        if ctx.trajectory is not None:
            tapes = ctx.trajectory
            ctx.trajectory = None
        else:
            # recompute the segment, keeping every step's tape (initial
            # state, C-grid fields, pre-remap state, corner pkap and gz)
            dyn.state_load(ckpt.data_ptr())
            tapes = _record(dyn, dt, remaps, ckpt, final_state=False)
        dyn.adj_zero()
        grads = [g if g is not None else torch.zeros_like(ckpt[:0]) for g in (gdp, gpt, gud, gvd)]
        for name, g in zip(FIELD_NAMES, grads):
            if g.numel():
                dyn.adj_set_device('out', name, g.detach().contiguous().data_ptr())
        for tp, r in zip(reversed(tapes), reversed(remaps)):
            dyn.adj_step_tape(dt, r, tp.data_ptr())
        del tapes
        dyn.adj_halo('out')  # the initial state's halo is the periodic image of its interior
        like = gdp if gdp is not None else (gpt if gpt is not None else (gud if gud is not None else gvd))
        outs = []
        for name in FIELD_NAMES:
            o = torch.empty_like(like)
            dyn.adj_get_device('out', name, o.data_ptr())
            outs.append(o)
        return (None, None, None, None, *outs)


def integrate(dyn: Dycore, fields, nsteps: int, dt: float, remap_every: int, checkpoint_every: int,
              first_step: int = 0):
    """Advance (dp, pt, ud, vd) by nsteps with checkpoints every
    ``checkpoint_every`` steps; differentiable with respect to the inputs."""
    out = tuple(fields)
    grad = torch.is_grad_enabled() and any(f.requires_grad for f in fields)
    s = first_step
    end = first_step + nsteps
    while s < end:
        n = min(checkpoint_every, end - s)
        remaps = [(q + 1) % remap_every == 0 for q in range(s, s + n)]
        out = DycoreSegment.apply(dyn, dt, remaps, grad and s + n >= end, *out)
        s += n
    return out


def gaussian_mask(st, radius: float, device=None):
    """exp(-(r / radius)^2) around the domain centre on the cell centres."""
    x = (torch.arange(st.nx, dtype=torch.float64, device=device) + 0.5) * st.dx
    y = (torch.arange(st.ny, dtype=torch.float64, device=device) + 0.5) * st.dy
    r2 = (x[None, :] - st.nx * st.dx / 2) ** 2 + (y[:, None] - st.ny * st.dy / 2) ** 2
    return torch.exp(-r2 / radius ** 2)
