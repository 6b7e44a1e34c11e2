"""Oracle of the differentiable-exchange program (test infrastructure only).

GHEX has no stencil; the program is the workload the exchange's adjoint is checked in: per step,
a halo exchange followed by the 7-point update x <- x + alpha * L(x) on the interior (halo of the
result set to 0); loss = sum of squares of the final interiors. Its gradient is computed here by
the explicit transpose: the stencil's transpose, then the exchange's adjoint (oracle.regular's
fixed-order scatter-add, which follows the receive order of GHEX's regular pattern,
structured/regular/halo_generator.hpp:91-146 and structured/pattern.hpp).

Every operation is an elementwise numpy ufunc in the same order as the device kernel, so results
agree bit for bit:

    forward, interior:  s = ((((x[i-1] + x[i+1]) + x[j-1]) + x[j+1]) + x[k-1]) + x[k+1]
                        y = x + alpha * (s - 6 * x)
    adjoint, all cells: G = g on the interior, 0 elsewhere (and outside the array)
                        t = ((((G[i-1] + G[i+1]) + G[j-1]) + G[j+1]) + G[k-1]) + G[k+1]
                        gx = G + alpha * (t - 6 * G)

Arrays are (x, y, z) with any memory order; the halo width h is the same on every side.
"""
from __future__ import annotations

import numpy as np

from . import regular as O


def apply(x: np.ndarray, alpha: float, h: int = 1) -> np.ndarray:
    t = x.dtype.type
    a, six = t(alpha), t(6)
    y = np.zeros_like(x)
    c = x[h:-h, h:-h, h:-h]
    s = x[h - 1:-h - 1, h:-h, h:-h] + x[h + 1:x.shape[0] - h + 1, h:-h, h:-h]
    s = s + x[h:-h, h - 1:-h - 1, h:-h]
    s = s + x[h:-h, h + 1:x.shape[1] - h + 1, h:-h]
    s = s + x[h:-h, h:-h, h - 1:-h - 1]
    s = s + x[h:-h, h:-h, h + 1:x.shape[2] - h + 1]
    y[h:-h, h:-h, h:-h] = c + a * (s - six * c)
    return y


def adjoint(g: np.ndarray, alpha: float, h: int = 1) -> np.ndarray:
    t = g.dtype.type
    a, six = t(alpha), t(6)
    G = np.zeros(tuple(n + 2 for n in g.shape), dtype=g.dtype)      # one cell of zeros around the array
    G[1 + h:-1 - h, 1 + h:-1 - h, 1 + h:-1 - h] = g[h:-h, h:-h, h:-h]
    nx, ny, nz = g.shape
    c = G[1:-1, 1:-1, 1:-1]
    s = G[0:nx, 1:-1, 1:-1] + G[2:, 1:-1, 1:-1]
    s = s + G[1:-1, 0:ny, 1:-1]
    s = s + G[1:-1, 2:, 1:-1]
    s = s + G[1:-1, 1:-1, 0:nz]
    s = s + G[1:-1, 1:-1, 2:]
    out = c + a * (s - six * c)
    return np.asarray(out, order="F") if g.flags["F_CONTIGUOUS"] else out


class Program:
    """steps x (exchange, stencil) over the domains of one regular pattern, one field."""

    def __init__(self, pattern, domains, offsets, steps: int = 10, alpha: float = 0.1, halo: int = 1):
        self.pattern, self.domains, self.offsets = pattern, domains, offsets
        self.steps, self.alpha, self.h = steps, alpha, halo

    def forward(self, xs):
        xs = [x.copy(order="K") for x in xs]
        for _ in range(self.steps):
            O.exchange(self.pattern, self.domains, xs, [self.offsets] * len(xs))
            xs = [apply(x, self.alpha, self.h) for x in xs]
        return xs

    def interior(self, x):
        h = self.h
        return x[h:-h, h:-h, h:-h]

    def loss(self, xs) -> float:
        return float(sum(np.sum(self.interior(x).astype(np.float64) ** 2) for x in xs))

    def gradient(self, xs):
        """d loss / d x0 by the explicit transpose (the forward is linear: no activations kept)."""
        ys = self.forward(xs)
        gs = []
        for y in ys:
            g = np.zeros_like(y)
            self.interior(g)[...] = 2 * self.interior(y)
            gs.append(g)
        for _ in range(self.steps):
            gs = [adjoint(g, self.alpha, self.h) for g in gs]
            O.adjoint(self.pattern, self.domains, gs, [self.offsets] * len(gs))
        return gs
