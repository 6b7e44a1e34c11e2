"""Differentiable halo exchange for PyTorch.

    dx = DifferentiableExchange(ctx, [pattern(fd) for fd in field_descriptors])
    xs = dx(*xs)              # halo exchange in place; differentiable
    ys = stencil7(xs, 0.1)    # the 7-point update of the example program, differentiable

The forward is the exchange itself (a pure copy: every halo element takes its owner's value).
Its adjoint adds every halo gradient into the interior element it was copied from (negated where
the forward negated it, as on cubed-sphere vector components) in a fixed order — the receive
order of the pattern, the order of the CPU explicit transpose — and then zeroes the halo. It runs
in place on the incoming gradient when that has the field's layout (autograd hands each backward
a buffer of its own; a hook that retains the exchange output's gradient would see it modified).

GHEX's Python bindings have no autograd support (bindings/python/src/ghex/structured/regular.py
and unstructured.py wrap the exchange only); this module is the differentiable form of
co.exchange(pattern(field) ...).wait() on the same patterns and field descriptors.

A plan addresses fixed memory. Autograd produces new tensors at every step, so each
DifferentiableExchange keeps a small pool of plans for the forward and for the gradients, keyed by
the data pointers they are bound to (the caching allocator hands out the same few blocks step
after step); a miss rebinds the least recently used plan (ghexb_plan_rebind: a stream-ordered
rewrite of the descriptor tables). Plans hold no references to the tensors they are bound to.
"""
from __future__ import annotations

import ctypes as C
from collections import OrderedDict
from typing import Any, Sequence

import torch

from . import _capi
from ._capi import call
from ._core import BufferInfo, ExchangePlan, _flatten, _layout_of, context

__all__ = ["DifferentiableExchange", "stencil7", "Stencil7", "diffusion_program", "GraphedDiffusion"]


class _PlanPool:
    def __init__(self, ctx: context, bis: Sequence[BufferInfo], size: int):
        self.ctx, self.bis, self.size = ctx, list(bis), size
        self.plans: "OrderedDict[tuple, ExchangePlan]" = OrderedDict()
        self.hits = self.rebinds = self.created = 0

    def get(self, tensors: Sequence[torch.Tensor], stream) -> ExchangePlan:
        key = tuple(t.data_ptr() for t in tensors)
        plan = self.plans.get(key)
        if plan is not None:
            self.plans.move_to_end(key)
            self.hits += 1
            return plan
        if len(self.plans) < self.size:
            plan = ExchangePlan(self.ctx, self.bis)
            self.created += 1
        else:
            _, plan = self.plans.popitem(last=False)
        if plan.bound_pointers() != key:
            plan.rebind(tensors, stream=stream, keep=False)
            self.rebinds += 1
        self.plans[key] = plan
        return plan

    def stats(self) -> dict:
        return {"plans": len(self.plans), "hits": self.hits, "rebinds": self.rebinds, "created": self.created}


class DifferentiableExchange:
    """The halo exchange of a fixed set of buffer_infos as a differentiable function of their
    arrays. Calling it with tensors of the same layouts (shape, strides, dtype, device) as the
    fields the buffer_infos were made from exchanges those tensors in place."""

    def __init__(self, ctx: context, buffer_infos: Sequence[BufferInfo], *, graph: bool = True, pool: int = 8):
        self.context = ctx
        self._bis = _flatten(tuple(buffer_infos))
        templates = [a for bi in self._bis for a in bi.arrays()]
        for t in templates:
            if not isinstance(t, torch.Tensor):
                raise TypeError("the differentiable exchange takes torch tensors")
            if t.dtype not in (torch.float32, torch.float64):
                raise TypeError("the differentiable exchange needs float32 or float64 fields")
        self._layout = [_layout_of(t) for t in templates]
        self._tensor_layout = [(t.shape, t.stride(), t.dtype, t.device) for t in templates]
        self.graph = graph
        self._fwd = _PlanPool(ctx, self._bis, pool)
        self._bwd = _PlanPool(ctx, self._bis, pool)

    def __len__(self) -> int:
        return len(self._layout)

    def pool_stats(self) -> dict:
        """Plan-pool use of the forward exchanges and of the adjoints: lookups that found a plan
        bound to the tensors (hits) and rebinds of a plan to new memory."""
        return {"forward": self._fwd.stats(), "adjoint": self._bwd.stats()}

    def check(self, tensors: Sequence[torch.Tensor]) -> None:
        if len(tensors) != len(self._layout):
            raise ValueError(f"expected {len(self._layout)} tensors, got {len(tensors)}")
        for t, lay in zip(tensors, self._layout):
            if _layout_of(t) != lay:
                raise TypeError("tensor layout differs from the field it stands for")

    def exchange_(self, tensors: Sequence[torch.Tensor]) -> None:
        """Forward exchange in place, outside autograd."""
        self.check(tensors)
        stream = torch.cuda.current_stream(tensors[0].device)
        plan = self._fwd.get(tensors, stream)
        if self.graph:
            plan.graph_launch(stream=stream)
        else:
            plan.launch(stream=stream)

    def adjoint_(self, grads: Sequence[torch.Tensor]) -> None:
        """Adjoint in place on gradient tensors of the fields' layouts, outside autograd."""
        self.check(grads)
        stream = torch.cuda.current_stream(grads[0].device)
        self._bwd.get(grads, stream).adjoint(stream=stream)

    def __call__(self, *tensors: torch.Tensor):
        if len(tensors) == 1 and isinstance(tensors[0], (list, tuple)):
            tensors = tuple(tensors[0])
        out = _ExchangeFunction.apply(self, *tensors)
        return out if isinstance(out, tuple) else (out,)


class _ExchangeFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, dx: DifferentiableExchange, *tensors):
        dx.exchange_(tensors)
        ctx.dx = dx
        ctx.mark_dirty(*tensors)
        return tensors

    @staticmethod
    def backward(ctx, *grads):
        dx: DifferentiableExchange = ctx.dx
        gs = []
        for g, (shape, stride, dtype, dev) in zip(grads, dx._tensor_layout):
            if g is not None and g.shape == shape and g.stride() == stride and g.dtype == dtype:
                gs.append(g)
                continue
            buf = torch.empty_strided(shape, stride, dtype=dtype, device=dev)
            if g is None:
                buf.zero_()
            else:
                buf.copy_(g)
            gs.append(buf)
        dx.adjoint_(gs)
        return (None, *gs)


def _launch_stencil(xs: Sequence[torch.Tensor], outs: Sequence[torch.Tensor], alpha: float, halo: int,
                    adjoint: bool) -> None:
    n = len(xs)
    if n == 0:
        return
    dtype = xs[0].dtype
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("stencil7 computes in float32 or float64")
    ext, st = [], []
    for x, y in zip(xs, outs):
        if x.dim() != 3 or x.dtype != dtype or y.shape != x.shape or y.stride() != x.stride() or not x.is_cuda:
            raise TypeError("stencil7 takes 3-D CUDA tensors of one dtype")
        ext += list(x.shape)
        st += list(x.stride())
    code = _capi.F64 if dtype == torch.float64 else _capi.F32
    stream = torch.cuda.current_stream(xs[0].device).cuda_stream
    call("ghexb_stencil7", code, n, (C.c_void_p * n)(*[x.data_ptr() for x in xs]),
         (C.c_void_p * n)(*[y.data_ptr() for y in outs]), (C.c_int64 * (3 * n))(*ext), (C.c_int64 * (3 * n))(*st),
         halo, float(alpha), int(adjoint), C.c_void_p(stream))


class Stencil7(torch.autograd.Function):
    """y = x + alpha * L(x) on the interior of each domain (7-point Laplacian L), 0 on the halo."""

    @staticmethod
    def forward(ctx, alpha: float, halo: int, *xs):
        outs = [torch.empty_like(x) for x in xs]
        _launch_stencil(xs, outs, alpha, halo, adjoint=False)
        ctx.alpha, ctx.halo = alpha, halo
        ctx.layouts = [(x.shape, x.stride(), x.dtype, x.device) for x in xs]
        return tuple(outs)

    @staticmethod
    def backward(ctx, *gys):
        gin = []
        for g, (shape, stride, dtype, dev) in zip(gys, ctx.layouts):
            if g is None:
                g = torch.zeros(shape, dtype=dtype, device=dev)
            if g.stride() != stride or g.shape != shape:
                buf = torch.empty_strided(shape, stride, dtype=dtype, device=dev)
                buf.copy_(g)
                g = buf
            gin.append(g)
        outs = [torch.empty_strided(shape, stride, dtype=dtype, device=dev) for shape, stride, dtype, dev in ctx.layouts]
        _launch_stencil(gin, outs, ctx.alpha, ctx.halo, adjoint=True)
        return (None, None, *outs)


def stencil7(xs: Sequence[torch.Tensor], alpha: float = 0.1, halo: int = 1):
    out = Stencil7.apply(alpha, halo, *xs)
    return out if isinstance(out, tuple) else (out,)


def diffusion_program(dx: DifferentiableExchange, xs: Sequence[torch.Tensor], steps: int = 10, alpha: float = 0.1,
                      halo: int = 1):
    """steps x (halo exchange, 7-point update); returns the final fields. The first exchange
    writes into xs: pass clones of leaf tensors that require grad."""
    xs = tuple(xs)
    for _ in range(steps):
        xs = dx(*xs)
        xs = stencil7(xs, alpha, halo)
    return xs


def interior_loss(xs: Sequence[torch.Tensor], halo: int = 1) -> torch.Tensor:
    """Sum of squares of the interiors."""
    h = halo
    return sum((x[h:-h, h:-h, h:-h] ** 2).sum() for x in xs)


class GraphedDiffusion:
    """The diffusion program (``steps`` x (halo exchange, 7-point update), loss = sum of squares of
    the final interiors) and its gradient with respect to the input fields, replayed from one CUDA
    graph: the kernels of ``diffusion_program`` and of its backward through torch.autograd, in the
    same order, on buffers of fixed memory, so that the host launches one graph instead of the
    program's kernels one by one.

    The forward alternates two buffer sets; the backward seeds 2 x (final interior) and applies, for
    every step in reverse, the stencil's transpose and then the exchange's adjoint, on two more
    buffer sets. Four exchange plans of its own are bound to the four sets before the capture, so
    the capture holds only kernel launches. ``run(xs)`` copies the inputs in, replays the graph, and returns the loss and
    the gradient (tensors the next run overwrites)."""

    def __init__(self, dx: DifferentiableExchange, templates: Sequence[torch.Tensor], steps: int = 10,
                 alpha: float = 0.1, halo: int = 1):
        templates = list(templates)
        dx.check(templates)
        self.dx, self.steps, self.alpha, self.halo = dx, steps, alpha, halo
        dev = templates[0].device

        def buffers():
            return [torch.zeros_like(t) for t in templates]
        self._inp, self._a, self._b, self._g1, self._g2 = buffers(), buffers(), buffers(), buffers(), buffers()
        stream = torch.cuda.Stream(device=dev)
        stream.wait_stream(torch.cuda.current_stream(dev))

        def plan_for(bufs):
            # a plan of its own, bound to these buffers for the graph's life (a plan of the
            # differentiable exchange's pool may be rebound to other tensors later)
            plan = ExchangePlan(dx.context, dx._bis)
            plan.rebind(bufs, stream=stream)
            return plan
        with torch.cuda.stream(stream):
            self._fwd = [plan_for(bufs) for bufs in (self._a, self._b)]
            self._bwd = [plan_for(bufs) for bufs in (self._g1, self._g2)]
            for plan in self._bwd:
                if plan.info()["adjoint_launches"] != 1:
                    raise ValueError("a graphed program needs an exchange whose adjoint is one kernel")
        torch.cuda.synchronize(dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=stream):
            self.loss, self.grad = self._body()

    def _body(self):
        s = torch.cuda.current_stream()
        h = self.halo
        for x, y in zip(self._a, self._inp):
            x.copy_(y)
        cur, nxt, plans = self._a, self._b, self._fwd
        for k in range(self.steps):
            plans[k % 2].launch(stream=s)
            _launch_stencil(cur, nxt, self.alpha, h, adjoint=False)
            cur, nxt = nxt, cur
        loss = interior_loss(cur, h)
        g, gn, bplans = self._g1, self._g2, self._bwd
        for gt, x in zip(g, cur):
            if self.steps > 0:
                # the last update wrote +0 on every halo cell, so doubling the whole array (exact)
                # gives the seed, 2 x on the interior and +0 elsewhere, in one kernel
                torch.mul(x, 2, out=gt)
            else:
                gt.zero_()
                gt[h:-h, h:-h, h:-h] = 2 * x[h:-h, h:-h, h:-h]
        for k in range(self.steps):
            _launch_stencil(g, gn, self.alpha, h, adjoint=True)
            bplans[(k + 1) % 2].adjoint(stream=s)
            g, gn = gn, g
        return loss, g

    def run(self, xs: Sequence[torch.Tensor]):
        for y, x in zip(self._inp, xs):
            y.copy_(x)
        self.graph.replay()
        return self.loss, self.grad
