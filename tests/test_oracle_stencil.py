"""The oracle of the differentiable-exchange program: its explicit-transpose gradient against
central finite differences and dot-product identities, in float64 on the CPU."""
from __future__ import annotations

import numpy as np
import pytest

from ghex_b200 import workloads as W
from oracle import regular as O
from oracle import stencil as S


def small_program(shape=(12, 10, 8), parts=(2, 2, 2), steps=3, dtype=np.float64):
    w = W.config4(shape=shape, dtype=dtype)
    if parts != (2, 2, 2):
        w.domains = W.regular_decomposition(shape, parts)
    spec = w.fields[0]
    doms = [O.Domain(i, f, l) for i, f, l in w.domains]
    pat = O.make_pattern((0, 0, 0), tuple(n - 1 for n in shape), spec.halos, w.periodic, doms)
    prog = S.Program(pat, doms, w.offsets(spec), steps=steps)
    xs = [w.domain_array(d, spec) for d in w.domains]
    return prog, xs


def test_stencil_transpose_identity():
    rng = np.random.default_rng(3)
    for order in ("F", "C"):
        x = np.asarray(rng.standard_normal((9, 7, 6)), order=order)
        g = np.asarray(rng.standard_normal((9, 7, 6)), order=order)
        # <A x, g>_interior == <x, A^T g>
        lhs = np.sum(S.apply(x, 0.1)[1:-1, 1:-1, 1:-1] * g[1:-1, 1:-1, 1:-1])
        rhs = np.sum(x * S.adjoint(g, 0.1))
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


def test_stencil_halo_and_interior():
    x = np.arange(5 * 5 * 5, dtype=np.float64).reshape(5, 5, 5)
    y = S.apply(x, 0.1)
    assert np.all(y[0] == 0) and np.all(y[-1] == 0) and np.all(y[:, 0] == 0) and np.all(y[:, :, -1] == 0)
    # L of a linear function is 0 on the interior
    assert np.array_equal(y[1:-1, 1:-1, 1:-1], x[1:-1, 1:-1, 1:-1])


def test_exchange_adjoint_identity():
    prog, xs = small_program()
    rng = np.random.default_rng(5)
    for x in xs:
        x[np.isnan(x)] = 0
    gs = [rng.standard_normal(x.shape) for x in xs]
    ys = [x.copy() for x in xs]
    O.exchange(prog.pattern, prog.domains, ys, [prog.offsets] * len(ys))
    lhs = sum(np.sum(y * g) for y, g in zip(ys, gs))
    ag = [g.copy() for g in gs]
    O.adjoint(prog.pattern, prog.domains, ag, [prog.offsets] * len(ag))
    rhs = sum(np.sum(x * a) for x, a in zip(xs, ag))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def fd_directional(prog, xs, d, h=1e-6):
    """(L(x + h d) - L(x - h d)) / 2h, evaluated as sum (y+ - y-)(y+ + y-) / 2h over the interiors,
    with the perturbation actually applied (x+ - x-) returned beside it."""
    xp = [x + h * e for x, e in zip(xs, d)]
    xm = [x - h * e for x, e in zip(xs, d)]
    yp, ym = prog.forward(xp), prog.forward(xm)
    fd = sum(np.sum((prog.interior(a) - prog.interior(b)) * (prog.interior(a) + prog.interior(b)))
             for a, b in zip(yp, ym)) / (2 * h)
    deff = [(a - b) / (2 * h) for a, b in zip(xp, xm)]
    return fd, deff


@pytest.mark.parametrize("shape,parts", [((12, 10, 8), (2, 2, 2)), ((14, 9, 7), (3, 1, 2))])
def test_gradient_matches_finite_differences(shape, parts):
    prog, xs = small_program(shape, parts)
    g = prog.gradient(xs)
    rng = np.random.default_rng(11)
    for _ in range(8):
        d = []
        for x in xs:
            e = np.zeros_like(x)
            prog.interior(e)[...] = rng.uniform(-1, 1, prog.interior(e).shape)
            d.append(e)
        fd, deff = fd_directional(prog, xs, d)
        gd = sum(np.sum(prog.interior(a) * prog.interior(b)) for a, b in zip(g, deff))
        assert abs(fd - gd) <= 1e-9 * abs(gd), (fd, gd)


def test_gradient_zero_on_halo():
    prog, xs = small_program()
    for g in prog.gradient(xs):
        m = np.ones(g.shape, dtype=bool)
        m[1:-1, 1:-1, 1:-1] = False
        assert np.all(g[m] == 0)
