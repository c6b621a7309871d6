"""Differentiable weighted least-squares unwrapping (the Laplace path's
solve with an adjoint).

The Laplace path (cuphu_laplace.cu:88-247, 385-549) solves, per IRLS pass,

    u = argmin_u  sum_a w_a ((D u)_a - g_a)^2 + eps |u|^2,    eps = 1e-12,

where g are the wrapped phase differences of the arcs, w the per-arc
weights and (D u)_a = u(head) - u(tail).  Its operator L = D^T W D + eps I
is self-adjoint, so the gradient of a loss l(u) costs one more PCG solve:
lambda = L^-1 dl/du, then dl/dg = W D lambda and dl/dw = (D lambda)(g - D u).
Both solves run in the library's persistent solver (cuphu_wls_solve_device),
and the gradients are assembled on the device (cuphu_wls_grad_device).

``WLSSolve`` is the torch.autograd.Function of one solve; ``irls_solve``
composes it with the IRLS reweighting w = w0 / sqrt(e^2 + delta^2),
e = D u - g, so autograd keeps every pass's solution (the checkpointed
IRLS iterates) and differentiates through the reweighting too.  The loss
should act on the continuous solution: the congruence projection
(rint) has zero gradient almost everywhere.

Arc planes are (nrow, ncol) CUDA tensors: "d" planes hold arc
(r, c) -> (r + 1, c) (last row unused), "r" planes arc (r, c) -> (r, c + 1)
(last column unused).  Requires the built library and a CUDA device; there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import CuPhuSolveStats, check, default_solve_options, lib

__all__ = ["wls_solve", "WLSSolve", "irls_solve"]

_PREC = {"mixed": 0, "fp64": 1}


def _vp(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _f32(t):
    return t.detach().to(torch.float32).contiguous()


def wls_solve(gd=None, gr=None, wd=None, wr=None, *, rhs=None, u0=None, precision="fp64",
              max_iter=1000, tol=1e-3, stats=False):
    """One WLS solve without autograd: returns the FP64 solution (and the
    solver statistics with ``stats=True``).  Give (gd, gr) or ``rhs``."""
    if wd is None or wr is None:
        raise ValueError("wd and wr are required")
    nrow, ncol = wd.shape
    dev = wd.device
    if dev.type != "cuda":
        raise ValueError("wls_solve needs CUDA tensors")
    u = torch.empty((nrow, ncol), dtype=torch.float64, device=dev)
    o = default_solve_options(precision=_PREC[precision], max_iter=int(max_iter), tol=float(tol))
    st = CuPhuSolveStats()
    args = [_f32(t) if t is not None else None for t in (gd, gr, rhs, wd, wr)]
    u0c = None if u0 is None else u0.detach().to(torch.float64).contiguous()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        check(lib().cuphu_wls_solve_device(*[_vp(a) for a in args], _vp(u0c), nrow, ncol,
                                           C.byref(o), _vp(u), C.byref(st) if stats else None,
                                           C.c_void_p(stream)))
    return (u, st) if stats else u


class WLSSolve(torch.autograd.Function):
    """u = argmin sum_a w_a ((D u)_a - g_a)^2 + eps |u|^2 with an adjoint
    backward (one extra solve of the self-adjoint operator)."""

    @staticmethod
    def forward(ctx, gd, gr, wd, wr, u0=None, precision="fp64", max_iter=1000, tol=1e-3):
        gd_, gr_, wd_, wr_ = (_f32(t) for t in (gd, gr, wd, wr))
        u = wls_solve(gd_, gr_, wd_, wr_, u0=u0, precision=precision, max_iter=max_iter, tol=tol)
        ctx.save_for_backward(gd_, gr_, wd_, wr_, u)
        ctx.cfg = (precision, max_iter, tol)
        ctx.dtypes = (gd.dtype, gr.dtype, wd.dtype, wr.dtype)
        return u

    @staticmethod
    def backward(ctx, ubar):
        gd, gr, wd, wr, u = ctx.saved_tensors
        precision, max_iter, tol = ctx.cfg
        nrow, ncol = u.shape
        # L 1 = eps 1 and D 1 = 0: the mean of ubar only moves lambda along
        # the constant vector, which D removes, so solve for the rest
        v = ubar.to(torch.float64)
        v = (v - v.mean()).to(torch.float32).contiguous()
        lam = wls_solve(rhs=v, wd=wd, wr=wr, precision=precision, max_iter=max_iter, tol=tol)
        ggd, ggr, gwd, gwr = (torch.empty_like(u) for _ in range(4))
        with torch.cuda.device(u.device):
            stream = torch.cuda.current_stream(u.device).cuda_stream
            check(lib().cuphu_wls_grad_device(_vp(lam), _vp(u), _vp(gd), _vp(gr), _vp(wd), _vp(wr),
                                              nrow, ncol, _vp(ggd), _vp(ggr), _vp(gwd), _vp(gwr),
                                              C.c_void_p(stream)))
        dt = ctx.dtypes
        return (ggd.to(dt[0]), ggr.to(dt[1]), gwd.to(dt[2]), gwr.to(dt[3]), None, None, None, None)


def _arc_diffs(u):
    """(D u) on the two arc planes, zero on the unused last row / column."""
    dd = torch.zeros_like(u)
    dr = torch.zeros_like(u)
    dd[:-1, :] = u[1:, :] - u[:-1, :]
    dr[:, :-1] = u[:, 1:] - u[:, :-1]
    return dd, dr


def irls_solve(gd, gr, w0d, w0r, n_irls=5, delta_max=0.5, delta_min=0.01, precision="fp64",
               max_iter=1000, tol=1e-3):
    """Differentiable IRLS of the Laplace path (cuphu_laplace.cu:214-247,
    385-390, 515-522): solve with w0, then n_irls times reweight
    w = w0 / sqrt(e^2 + delta_k^2), e = D u - g, delta_k = max(delta_min,
    delta_max 0.5^k), and re-solve from the previous solution.  Returns the
    continuous FP64 solution of the last pass (no anchoring)."""
    g64d, g64r = gd.to(torch.float64), gr.to(torch.float64)
    w64d, w64r = w0d.to(torch.float64), w0r.to(torch.float64)
    u = WLSSolve.apply(gd, gr, w0d, w0r, None, precision, max_iter, tol)
    for k in range(n_irls):
        delta = max(delta_min, delta_max * 0.5 ** k)
        dd, dr = _arc_diffs(u)
        ed, er = dd - g64d, dr - g64r
        wd = torch.where(w64d > 0, w64d * torch.rsqrt(ed * ed + delta * delta), torch.zeros_like(ed))
        wr = torch.where(w64r > 0, w64r * torch.rsqrt(er * er + delta * delta), torch.zeros_like(er))
        u = WLSSolve.apply(gd, gr, wd.to(w0d.dtype), wr.to(w0r.dtype), u.detach(), precision,
                           max_iter, tol)
    return u
