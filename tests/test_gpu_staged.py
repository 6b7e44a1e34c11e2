"""The staged form of the batched exchange (tensor-map loads into shared memory, writes from
there, beside the element kernel), bit-exact against the oracle: every element size, memory order
and component count of the layout test, the cubed sphere's transposed and reversed edges with
negated vector components, and the full-size workloads; at several stage sizes and pipeline
shapes, with the kernel's status word clear (every bounded wait ended in time)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from ghex_b200 import workloads as W
from ghex_b200.structured import cubed_sphere as C
from ghex_b200.structured import regular as R
from gpu_helpers import RegularRun, bits_equal, to_device
from oracle import cubed_sphere as OC
from oracle import regular as O
from test_gpu_layouts import HALOS, PERIODIC, SHAPE, _values

pytestmark = pytest.mark.gpu

SHAPES = [(1, 8, 16384, 4, 1), (2, 8, 16384, 4, 1), (2, 4, 4096, 8, 2), (2, 16, 2048, 2, 1)]


def staged_launch_ok(plan, tens, host, expected, mode, stages, stage_bytes, consumers, ctas, require=True):
    plan.set_staged(mode, stages, stage_bytes, consumers, ctas)
    info = plan.info()
    assert info["staged_mode"] == mode
    assert info["staged_boxes"] > 0 or not require
    for t, a in zip(tens, host):
        t.copy_(torch.from_numpy(a))
    plan.launch(plan.BATCHED)
    assert plan.staged_status() == 0
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
    # the graph of the batched form, replayed twice
    for t, a in zip(tens, host):
        t.copy_(torch.from_numpy(a))
    plan.graph_launch()
    plan.graph_launch()
    assert plan.staged_status() == 0
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int64, np.uint16, np.uint8])
@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("ncomp", [1, 3])
def test_staged_dtypes_orders_components(cuda, dtype, order, ncomp):
    doms_spec = W.regular_decomposition(SHAPE, (2, 2, 1), 3)
    ctx = R.make_context()
    hg = R.HaloGenerator(((0, 0, 0), tuple(n - 1 for n in SHAPE)),
                         [(HALOS[2 * k], HALOS[2 * k + 1]) for k in range(3)], PERIODIC)
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in doms_spec]
    pat = R.make_pattern(ctx, hg, doms)
    rng = np.random.default_rng(23)
    offsets = (HALOS[0], HALOS[2], HALOS[4])
    host, tens, bis = [], [], []
    for dm, (_, f, l) in zip(doms, doms_spec):
        ext = tuple(l[k] - f[k] + 1 + HALOS[2 * k] + HALOS[2 * k + 1] for k in range(3))
        a = np.asarray(_values(rng, ext + ((ncomp,) if ncomp > 1 else ()), dtype), order=order)
        host.append(a)
        t = torch.from_numpy(a).to(cuda)
        tens.append(t)
        bis.append(pat(R.make_field_descriptor(dm, t, offsets, ext)))
    plan = R.make_exchange_plan(ctx, bis)
    odoms = [O.Domain(i, f, l) for i, f, l in doms_spec]
    opat = O.make_pattern((0, 0, 0), tuple(n - 1 for n in SHAPE), HALOS, PERIODIC, odoms)
    expected = [a.copy(order="K") for a in host]
    O.exchange(opat, odoms, expected, [offsets] * len(odoms))
    # components stored fastest leave no contiguous source rows: nothing is staged then
    require = not (order == "C" and ncomp > 1)
    for mode in (1, 2):
        for shape in SHAPES[:2]:
            staged_launch_ok(plan, tens, host, expected, mode, shape[1], shape[2], shape[3], shape[4],
                             require=require and mode == 2)


@pytest.mark.parametrize("shape", SHAPES, ids=["8x16K", "8x16K-2", "4x4K-8w-2cta", "16x2K-2w"])
def test_staged_cfg1_small(cuda, shape):
    run = RegularRun(W.config1(shape=(60, 45, 15)), cuda)
    plan = R.make_exchange_plan(run.ctx, run.bis)
    exp = run.oracle()
    names = list(run.dev)
    tens = [t for n in names for t in run.dev[n]]
    host = [a for n in names for a in run.host[n]]
    expected = [a for n in names for a in exp[n]]
    staged_launch_ok(plan, tens, host, expected, shape[0], shape[1], shape[2], shape[3], shape[4])


def test_staged_cfg1_full_size(cuda):
    run = RegularRun(W.config1(), cuda)
    plan = R.make_exchange_plan(run.ctx, run.bis)
    exp = run.oracle()
    names = list(run.dev)
    tens = [t for n in names for t in run.dev[n]]
    host = [a for n in names for a in run.host[n]]
    expected = [a for n in names for a in exp[n]]
    for mode in (1, 2):
        staged_launch_ok(plan, tens, host, expected, mode, 8, 16384, 4, 1)


@pytest.mark.parametrize("shape", [(48, 8, 2), (384, 90, 2)], ids=["small", "cfg3"])
@pytest.mark.parametrize("mode", [1, 2])
def test_staged_cubed_sphere(cuda, shape, mode):
    edge, levels, split = shape
    w = W.config3(edge=edge, levels=levels, split=split)
    ctx = C.make_context()
    cube = C.cube(w.edge, w.levels)
    doms = [C.DomainDescriptor(cube, *b) for b in w.domains]
    pat = C.make_pattern(ctx, C.HaloGenerator(w.halo), doms)
    s_host = [w.domain_array(d, 1, 1) for d in w.domains]
    v_host = [w.domain_array(d, 2, 2) for d in w.domains]
    tens, bis = [], []
    for arrays, nc, vec in ((s_host, 1, False), (v_host, 2, True)):
        ts = [to_device(a, cuda) for a in arrays]
        tens += ts
        bis += [pat(C.make_field_descriptor(d, t, w.offsets(), a.shape[:3], nc, vec)) for d, t, a in zip(doms, ts, arrays)]
    plan = C.make_exchange_plan(ctx, bis)
    odoms = [OC.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    opat = OC.make_pattern(w.edge, (w.halo,) * 4, odoms)
    expected = []
    for arrays, vec in ((s_host, False), (v_host, True)):
        ex = [a.copy(order="K") for a in arrays]
        OC.exchange(opat, odoms, ex, [w.offsets()] * len(odoms), w.edge, vec)
        expected += ex
    staged_launch_ok(plan, tens, s_host + v_host, expected, mode, 8, 16384, 4, 1)
    if shape[0] == 48:
        staged_launch_ok(plan, tens, s_host + v_host, expected, mode, 4, 2048, 2, 2)


def test_staged_then_element_kernel_again(cuda):
    """Switching the staged form off restores the element kernel's tables."""
    run = RegularRun(W.config1(shape=(60, 45, 15)), cuda)
    plan = R.make_exchange_plan(run.ctx, run.bis)
    exp = run.oracle()
    plan.set_staged(2)
    plan.set_staged(0)
    assert plan.info()["staged_boxes"] == 0
    plan.launch(plan.BATCHED)
    assert run.mismatches(exp) == {}


def test_staged_rejects_bad_shapes(cuda):
    run = RegularRun(W.config0(), cuda)
    plan = R.make_exchange_plan(run.ctx, run.bis)
    for bad in [dict(mode=3), dict(stages=1), dict(stages=17), dict(stage_bytes=100), dict(consumers=9),
                dict(stages=16, stage_bytes=65536)]:
        with pytest.raises(RuntimeError):
            plan.set_staged(**bad)
