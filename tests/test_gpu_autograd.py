"""The differentiable exchange on the device: the 7-point program's forward bit-exact against the
oracle, its autograd gradient bit-exact against the oracle's explicit transpose, and central
finite differences (h = 1e-6, 64 seeded directions) within 1e-9 relative in float64.

Probe directions are d_k = x0 + r_k on the interiors (r_k seeded uniform noise in [-1, 1)), so
that g.d_k is bounded away from zero (g.x0 = 2 |y|^2 for the quadratic loss of a linear program).
For a direction unrelated to the data, g.d is a sum of terms of random sign; some draws land near
zero and their relative error then measures the forward's rounding, not the gradient: the check
on those is made against the scale |g| |d| instead."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from ghex_b200 import autograd as AG
from ghex_b200 import workloads as W
from oracle import regular as O
from oracle import stencil as S

from gpu_helpers import RegularRun, bits_equal, to_device

pytestmark = pytest.mark.gpu

STEPS = 10
ALPHA = 0.1


class Program:
    def __init__(self, w, dev, steps=STEPS):
        self.w = w
        self.run = RegularRun(w, dev)
        self.spec = w.fields[0]
        self.dx = AG.DifferentiableExchange(self.run.ctx, self.run.bis)
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0, 0, 0), tuple(n - 1 for n in w.shape), self.spec.halos, w.periodic, doms)
        self.oracle = S.Program(pat, doms, w.offsets(self.spec), steps=steps, alpha=ALPHA)
        self.steps = steps
        self.host = self.run.host[self.spec.name]
        self.x0 = self.run.dev[self.spec.name]

    def forward(self, xs):
        return AG.diffusion_program(self.dx, [x.clone() for x in xs], self.steps, ALPHA)

    def gradient(self):
        leaves = [x.clone().requires_grad_(True) for x in self.x0]
        ys = AG.diffusion_program(self.dx, [x.clone() for x in leaves], self.steps, ALPHA)
        AG.interior_loss(ys).backward()
        return [l.grad for l in leaves]


def interior(a):
    return a[1:-1, 1:-1, 1:-1]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("order", ["F", "C"])
def test_stencil_kernels_bit_exact(cuda, dtype, order):
    rng = np.random.default_rng(7)
    xs = [np.asarray(rng.standard_normal(s), dtype=dtype, order=order) for s in ((9, 7, 6), (34, 20, 5), (3, 3, 3))]
    dev = [to_device(x, cuda) for x in xs]
    ys = AG.stencil7(dev, ALPHA)
    for x, y in zip(xs, ys):
        assert bits_equal(y.cpu().numpy(), S.apply(x, ALPHA)) == 0
    outs = [torch.empty_like(d) for d in dev]
    AG._launch_stencil(dev, outs, ALPHA, 1, adjoint=True)
    for x, o in zip(xs, outs):
        assert bits_equal(o.cpu().numpy(), S.adjoint(x, ALPHA)) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("halo", [1, 2])
def test_stencil_kernels_edges_bit_exact(cuda, dtype, halo):
    """Halo 2; 35 domains in one call (two launches of at most 32); extents that leave partial
    32 x 8 patches and several slabs of planes (z extent 53 and 70); a strided view whose rows are
    not contiguous: forward and transpose bit-exact against the oracle."""
    rng = np.random.default_rng(11 + halo)
    shapes = [(5 + (d % 7), 6 + (d % 5), 5 + (d % 3)) for d in range(33)] + [(40, 19, 53), (33, 9, 70)]
    xs = [np.asarray(rng.standard_normal(s), dtype=dtype, order="F") for s in shapes]
    dev = [to_device(x, cuda) for x in xs]
    big = torch.zeros((2 * 38, 17, 25), dtype=dev[0].dtype, device=cuda)
    view = big[::2, :, 1:-2]                     # strides (2, .., ..) over a C-ordered base
    view.copy_(torch.from_numpy(np.asarray(rng.standard_normal(view.shape), dtype=dtype)).to(cuda))
    xs.append(view.cpu().numpy())
    dev.append(view)
    for adjoint in (False, True):
        outs = [torch.empty_strided(d.shape, d.stride(), dtype=d.dtype, device=cuda) for d in dev]
        AG._launch_stencil(dev, outs, ALPHA, halo, adjoint=adjoint)
        ref = S.adjoint if adjoint else S.apply
        for x, o in zip(xs, outs):
            assert bits_equal(o.cpu().numpy(), ref(x, ALPHA, halo)) == 0


def test_stencil_rejects_bad_arguments(cuda):
    x = torch.zeros((2, 5, 5), dtype=torch.float64, device=cuda)
    with pytest.raises(Exception, match="twice the halo"):
        AG.stencil7([x])
    y = torch.zeros((5, 5, 5), dtype=torch.float64, device=cuda)
    with pytest.raises(Exception, match="overlap"):
        AG._launch_stencil([y], [y], ALPHA, 1, adjoint=False)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_program_small_bit_exact(cuda, dtype):
    p = Program(W.config4(shape=(32, 24, 16), dtype=dtype), cuda)
    ys = p.forward(p.x0)
    ref = p.oracle.forward(p.host)
    assert sum(bits_equal(y.detach().cpu().numpy(), r) for y, r in zip(ys, ref)) == 0
    g = p.gradient()
    gref = p.oracle.gradient(p.host)
    assert sum(bits_equal(a.cpu().numpy(), b) for a, b in zip(g, gref)) == 0


def fd_check(p, g, ndir, h=1e-6, seed=1234, along_data=True):
    """Worst relative error of the central difference against g.d over ndir directions
    (against |g| |d| when along_data is False)."""
    gen = torch.Generator(device=p.x0[0].device).manual_seed(seed)
    worst = 0.0
    with torch.no_grad():
        gnorm = float(sum(torch.sum(interior(a) ** 2) for a in g)) ** 0.5
        for _ in range(ndir):
            d = []
            for x in p.x0:
                e = torch.zeros_like(x)
                interior(e).uniform_(-1, 1, generator=gen)
                if along_data:
                    interior(e).add_(interior(x))
                d.append(e)
            xp = [x + h * e for x, e in zip(p.x0, d)]
            xm = [x - h * e for x, e in zip(p.x0, d)]
            yp, ym = p.forward(xp), p.forward(xm)
            fd = sum(torch.sum((interior(a) - interior(b)) * (interior(a) + interior(b))) for a, b in zip(yp, ym))
            fd = float(fd) / (2 * h)
            deff = [(interior(a) - interior(b)) / (2 * h) for a, b in zip(xp, xm)]
            gd = float(sum(torch.sum(interior(gg) * e) for gg, e in zip(g, deff)))
            scale = abs(gd) if along_data else gnorm * float(sum(torch.sum(e ** 2) for e in deff)) ** 0.5
            worst = max(worst, abs(fd - gd) / scale)
    return worst


def test_program_small_finite_differences(cuda):
    p = Program(W.config4(shape=(32, 24, 16)), cuda)
    g = p.gradient()
    assert fd_check(p, g, 64) <= 1e-9
    assert fd_check(p, g, 16, seed=99, along_data=False) <= 1e-9


def test_program_full_size(cuda):
    """256x256x128 float64 split 2x2x2, halo 1, periodic; 10 steps."""
    p = Program(W.config4(), cuda)
    g = p.gradient()
    gref = p.oracle.gradient(p.host)
    assert sum(bits_equal(a.cpu().numpy(), b) for a, b in zip(g, gref)) == 0
    assert fd_check(p, g, 64) <= 1e-9


def test_program_float32_full_size_bit_exact(cuda):
    p = Program(W.config4(dtype=np.float32), cuda)
    ys = p.forward(p.x0)
    ref = p.oracle.forward(p.host)
    assert sum(bits_equal(y.detach().cpu().numpy(), r) for y, r in zip(ys, ref)) == 0
    g = p.gradient()
    gref = p.oracle.gradient(p.host)
    assert sum(bits_equal(a.cpu().numpy(), b) for a, b in zip(g, gref)) == 0


def test_layout_mismatch_rejected(cuda):
    p = Program(W.config4(shape=(16, 16, 8)), cuda)
    bad = [x.clone().contiguous() for x in p.x0]  # C order instead of x fastest
    with pytest.raises(TypeError):
        p.dx(*bad)


def test_plan_pool_rebinds(cuda):
    """More distinct tensor sets than plans in the pool: every call still exchanges its own."""
    p = Program(W.config4(shape=(16, 16, 8)), cuda, steps=1)
    p.dx._fwd.size = 2
    sets = [[x.clone() for x in p.x0] for _ in range(5)]
    ref = [x.copy(order="K") for x in p.host]
    O.exchange(p.oracle.pattern, p.oracle.domains, ref, [p.oracle.offsets] * len(ref))
    for s in sets + sets[:2]:
        with torch.no_grad():
            p.dx.exchange_(s)
    torch.cuda.synchronize()
    for s in sets:
        assert sum(bits_equal(t.cpu().numpy(), r) for t, r in zip(s, ref)) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_graphed_program_same_bits(cuda, dtype):
    """The program and its gradient replayed from one CUDA graph (GraphedDiffusion) give the
    autograd program's loss and gradient bit for bit, and the oracle's gradient, on two different
    inputs through the same graph."""
    p = Program(W.config4(shape=(32, 24, 16), dtype=dtype), cuda)
    graphed = AG.GraphedDiffusion(p.dx, p.x0, STEPS, ALPHA)
    for scale in (1.0, -0.5):
        xs = [x * scale for x in p.x0]
        leaves = [x.clone().requires_grad_(True) for x in xs]
        ys = AG.diffusion_program(p.dx, [x.clone() for x in leaves], STEPS, ALPHA)
        loss = AG.interior_loss(ys)
        loss.backward()
        loss_g, grad_g = graphed.run(xs)
        torch.cuda.synchronize()
        assert bits_equal(loss_g.cpu().numpy(), loss.detach().cpu().numpy()) == 0
        assert sum(bits_equal(g.cpu().numpy(), l.grad.cpu().numpy()) for g, l in zip(grad_g, leaves)) == 0
    g_ref = p.oracle.gradient([h * -0.5 for h in p.host])
    assert sum(bits_equal(g.cpu().numpy(), r) for g, r in zip(grad_g, g_ref)) == 0
