"""Differentiable cycle objectives for PyTorch (no counterpart in the reference).

The forward passes are the library's solves; the backward passes are the
library's hand-written adjoint kernel (``pgc_backward_feat_diff``):

* ratio: lambda* = C(C*) / T(C*) over the rescaled costs of the optimal
  cycle C*, so d lambda*/d c_e = 1[e in C*] / T; the rescale factor is held
  fixed and its rounding passed straight through;
* minimum cost: d cost*/d c_e = 1[e in C*];

and the energy's adjoint scatters every cycle edge into the feat_diff
entries its cost reads (plain graph: two; conjugate graph: one, in the
("vanilla", *) and ("feature", *) modes; a ratio whose time column reads
feat_diff, ("*", "feature"), adds its time part with the subgradient of the
matrix maximum on that maximum's entry).  torch carries the gradient on from
feat_diff (e.g. to learnable features).  CUDA feat_diff tensors reach the
library by a device-to-device copy.  ``BlackboxMinCostCycle`` implements blackbox
interpolation (Vlastelica et al., ICLR 2020) over the edge costs: its
backward solves again at w + tau * dL/dy and returns -(y(w) - y(w')) / tau.
"""
from __future__ import annotations

import numpy as np
import torch

from . import backward_feat_diffs, set_feat_diffs_device, solve_batch


def _as_host(fd: torch.Tensor) -> np.ndarray:
    return fd.detach().to(device="cpu", dtype=torch.float64).contiguous().numpy()


def _set_feat_diff(gen, fd: torch.Tensor, synced: bool = False):
    """feat_diff into the handle: a device-to-device copy when it is a CUDA
    tensor (its producer synchronised first, unless the caller did), else
    through host memory."""
    if fd.is_cuda:
        src = fd.detach().to(dtype=torch.float64).contiguous()
        if not synced:
            torch.cuda.current_stream(src.device).synchronize()
        gen.set_feat_diff_device(src.data_ptr(), src.shape[0], src.shape[1])
    else:
        gen.set_feat_diff(_as_host(fd))


def _adjoint(gen, grad_out: torch.Tensor, like: torch.Tensor, synced: bool = False) -> torch.Tensor:
    # the library writes on the handle's own stream and synchronises it before
    # returning; torch's stream must be idle first (grad_out may still be
    # computed on it) unless the caller already synchronised
    grad = torch.empty(like.shape, dtype=torch.float64, device="cuda")
    g = float(grad_out) if synced else None
    if not synced:
        torch.cuda.synchronize()
        g = float(grad_out)
    gen.backward_feat_diff(g, grad.data_ptr())
    return grad.to(device=like.device, dtype=like.dtype)


class RatioCycleObjective(torch.autograd.Function):
    """lambda*(feat_diff) of ``gen`` (a product_graph_generator whose geometry
    and modes are set) by ``solve_with_cost_time_ratio``."""

    @staticmethod
    def forward(ctx, feat_diff, gen, max_depth=None):
        _set_feat_diff(gen, feat_diff)
        _, objective, _ = gen.solve_with_cost_time_ratio("lawlergpu", max_depth)
        ctx.gen = gen
        ctx.save_for_backward(feat_diff)
        return torch.tensor(objective, dtype=feat_diff.dtype, device=feat_diff.device)

    @staticmethod
    def backward(ctx, grad_out):
        (feat_diff,) = ctx.saved_tensors
        return _adjoint(ctx.gen, grad_out, feat_diff), None, None


class MinCostCycleObjective(torch.autograd.Function):
    """Cost of the minimum-cost cycle of ``gen`` as a function of feat_diff."""

    @staticmethod
    def forward(ctx, feat_diff, gen, max_depth=None):
        _set_feat_diff(gen, feat_diff)
        _, objective, _ = gen.solve_with_minimum_cost("dijkstragpu", max_depth)
        ctx.gen = gen
        ctx.save_for_backward(feat_diff)
        return torch.tensor(objective, dtype=feat_diff.dtype, device=feat_diff.device)

    @staticmethod
    def backward(ctx, grad_out):
        (feat_diff,) = ctx.saved_tensors
        return _adjoint(ctx.gen, grad_out, feat_diff), None, None


class _BatchedRatio(torch.autograd.Function):
    @staticmethod
    def forward(ctx, gens, max_depth, *feat_diffs):
        if all(fd.is_cuda for fd in feat_diffs):
            # every producer once, then one batched device-to-device copy
            srcs = [fd.detach().to(dtype=torch.float64).contiguous() for fd in feat_diffs]
            torch.cuda.synchronize()
            set_feat_diffs_device(gens, [s.data_ptr() for s in srcs])
            del srcs
        else:
            for g, fd in zip(gens, feat_diffs):
                _set_feat_diff(g, fd)
        results = solve_batch(gens, "lawlergpu", max_depth)
        ctx.gens = gens
        ctx.save_for_backward(*feat_diffs)
        like = feat_diffs[0]
        return torch.tensor([r[1] for r in results], dtype=like.dtype, device=like.device)

    @staticmethod
    def backward(ctx, grad_out):
        fds = ctx.saved_tensors
        torch.cuda.synchronize()
        go = grad_out.detach().cpu()
        if not all(fd.is_cuda for fd in fds):
            return (None, None) + tuple(_adjoint(g, go[i], fd, synced=True)
                                        for i, (g, fd) in enumerate(zip(ctx.gens, fds)))
        # every adjoint enqueued at once, one wait per graph
        grads = [torch.empty(fd.shape, dtype=torch.float64, device=fd.device) for fd in fds]
        torch.cuda.synchronize()  # the buffers exist before the library's streams write them
        backward_feat_diffs(ctx.gens, [float(x) for x in go], [g.data_ptr() for g in grads])
        return (None, None) + tuple(g.to(dtype=fd.dtype) for g, fd in zip(grads, fds))


def ratio_cycle_objectives(gens, feat_diffs, max_depth=None) -> torch.Tensor:
    """lambda* of many pairs at once (one batched solve), differentiable in every feat_diff."""
    return _BatchedRatio.apply(list(gens), max_depth, *feat_diffs)


def cycle_indicator(gen, rows: int) -> np.ndarray:
    """y[e] = how often product edge e is on the last returned cycle."""
    y = np.zeros(rows, dtype=np.float64)
    np.add.at(y, gen.last_cycle_edges(), 1.0)
    return y


class BlackboxMinCostCycle(torch.autograd.Function):
    """y(w): the edge indicator of the minimum-cost cycle for edge costs w
    ([rows] in edge-id order, set with ``set_cost_vector``).  Backward by
    blackbox interpolation with step ``tau``: w' = w + tau * dL/dy,
    dL/dw = -(y(w) - y(w')) / tau."""

    @staticmethod
    def forward(ctx, w, gen, tau=10.0, max_depth=None):
        wh = _as_host(w)
        gen.set_cost_vector(wh)
        gen.solve_with_minimum_cost("dijkstragpu", max_depth)
        y = cycle_indicator(gen, wh.shape[0])
        ctx.gen, ctx.tau, ctx.max_depth, ctx.w, ctx.y = gen, float(tau), max_depth, wh, y
        return torch.from_numpy(y).to(device=w.device, dtype=w.dtype)

    @staticmethod
    def backward(ctx, grad_y):
        w2 = ctx.w + ctx.tau * _as_host(grad_y)
        ctx.gen.set_cost_vector(w2)
        ctx.gen.solve_with_minimum_cost("dijkstragpu", ctx.max_depth)
        y2 = cycle_indicator(ctx.gen, w2.shape[0])
        g = -(ctx.y - y2) / ctx.tau
        return torch.from_numpy(g).to(device=grad_y.device, dtype=grad_y.dtype), None, None, None
