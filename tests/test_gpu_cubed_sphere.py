"""GPU parity of the cubed-sphere exchange: the reference test's known answers, and bit-exact
agreement with the oracle (and with GHEX's own code where it is built) on the benchmark shape."""
import numpy as np
import pytest
import torch

from cs_cases import EDGE, HALO, LEVELS, MEM_HALO, N, NCOMP, domains, fields
from ghex_b200 import workloads as W
from ghex_b200.structured import cubed_sphere as C
from gpu_helpers import bits_equal, to_device
from oracle import cubed_sphere as O
from oracle import reflib

pytestmark = pytest.mark.gpu


def device_exchange(ctx, edge, levels, halo, boxes, arrays_per_field, offsets, ncomps, vectors, form="co"):
    cube = C.cube(edge, levels)
    doms = [C.DomainDescriptor(cube, *b) for b in boxes]
    pat = C.make_pattern(ctx, C.HaloGenerator(halo), doms)
    tens, bis = [], []
    for arrays, nc, isv in zip(arrays_per_field, ncomps, vectors):
        ts = [to_device(a, torch.device("cuda", 0)) for a in arrays]
        tens.append(ts)
        bis += [pat(C.make_field_descriptor(d, t, offsets, a.shape[:3], nc, isv)) for d, t, a in zip(doms, ts, arrays)]
    if form == "co":
        C.make_communication_object(ctx).exchange(bis).wait()
    else:
        plan = C.make_exchange_plan(ctx, bis)
        plan.launch({"per_field": plan.PER_FIELD, "per_box": plan.PER_BOX, "batched": plan.BATCHED}[form])
    torch.cuda.synchronize()
    return [[t.cpu().numpy() for t in ts] for ts in tens]


@pytest.mark.parametrize("is_vector", [False, True])
@pytest.mark.parametrize("form", ["co", "per_field", "per_box"])
def test_reference_test_known_answers(cuda, is_vector, form):
    ctx = C.make_context()
    got = device_exchange(ctx, EDGE, LEVELS, HALO, domains(), [fields()], (MEM_HALO, MEM_HALO, 0), [NCOMP],
                          [is_vector], form)[0]
    odoms = [O.Domain(t, (x0, x1), (y0, y1), LEVELS) for t, x0, x1, y0, y1 in domains()]
    exp = fields()
    O.exchange(O.make_pattern(EDGE, (HALO,) * 4, odoms), odoms, exp, [(MEM_HALO, MEM_HALO, 0)] * 24, EDGE, is_vector)
    for (t, x0, _, y0, _), a, e in zip(domains(), got, exp):
        assert bits_equal(a, e) == 0
        if reflib.available():
            assert reflib.cs_check_field(np.asfortranarray(a), t, x0, y0, MEM_HALO, N, LEVELS, NCOMP, is_vector, HALO) == 0


@pytest.mark.parametrize("shape", [(48, 8, 2), (384, 90, 2)], ids=["small", "cfg3"])
def test_cfg3_scalar_and_vector_bitexact(cuda, shape):
    edge, levels, split = shape
    w = W.config3(edge=edge, levels=levels, split=split)
    s_host = [w.domain_array(d, 1, 1) for d in w.domains]
    v_host = [w.domain_array(d, 2, 2) for d in w.domains]
    ctx = C.make_context()
    got_s, got_v = device_exchange(ctx, w.edge, w.levels, w.halo, w.domains, [s_host, v_host], w.offsets(), [1, 2],
                                   [False, True])
    odoms = [O.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    pat = O.make_pattern(w.edge, (w.halo,) * 4, odoms)
    O.exchange(pat, odoms, s_host, [w.offsets()] * len(odoms), w.edge, False)
    O.exchange(pat, odoms, v_host, [w.offsets()] * len(odoms), w.edge, True)
    assert sum(bits_equal(a, e) for a, e in zip(got_s, s_host)) == 0
    assert sum(bits_equal(a, e) for a, e in zip(got_v, v_host)) == 0
    # cube-corner cells are never received: NaN stays, everything else is a number
    nan_cells = sum(int(np.isnan(a[..., 0]).sum()) for a in got_s)
    h = w.halo
    assert nan_cells == 24 * h * h * w.levels


def test_cubed_adjoint_bitexact(cuda):
    w = W.config3(edge=24, levels=4, split=2)
    rng = np.random.default_rng(3)
    grads = [np.asfortranarray(rng.standard_normal(w.extents(d) + (2,))) for d in w.domains]
    ctx = C.make_context()
    cube = C.cube(w.edge, w.levels)
    doms = [C.DomainDescriptor(cube, *b) for b in w.domains]
    pat = C.make_pattern(ctx, C.HaloGenerator(w.halo), doms)
    ts = [to_device(g, cuda) for g in grads]
    bis = [pat(C.make_field_descriptor(d, t, w.offsets(), g.shape[:3], 2, True)) for d, t, g in zip(doms, ts, grads)]
    plan = C.make_exchange_plan(ctx, bis)
    plan.adjoint()
    torch.cuda.synchronize()
    odoms = [O.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    O.adjoint(O.make_pattern(w.edge, (w.halo,) * 4, odoms), odoms, grads, [w.offsets()] * len(odoms), w.edge, True)
    assert sum(bits_equal(t.cpu().numpy(), g) for t, g in zip(ts, grads)) == 0


@pytest.mark.parametrize("tuning", [(4, 128), (8, 256), (16, 512)])
def test_every_form_and_tuning(cuda, tuning):
    """Every launch form at several tunings (including the edges whose transform swaps x and y)
    bit-exact against the oracle."""
    w = W.config3(edge=48, levels=8, split=2)
    s_host = [w.domain_array(d, 1, 1) for d in w.domains]
    v_host = [w.domain_array(d, 2, 2) for d in w.domains]
    ctx = C.make_context()
    cube = C.cube(w.edge, w.levels)
    doms = [C.DomainDescriptor(cube, *b) for b in w.domains]
    pat = C.make_pattern(ctx, C.HaloGenerator(w.halo), doms)
    ts = [to_device(a, cuda) for a in s_host]
    tv = [to_device(a, cuda) for a in v_host]
    bis = [pat(C.make_field_descriptor(d, t, w.offsets(), a.shape[:3], 1, False)) for d, t, a in zip(doms, ts, s_host)]
    bis += [pat(C.make_field_descriptor(d, t, w.offsets(), a.shape[:3], 2, True)) for d, t, a in zip(doms, tv, v_host)]
    plan = C.make_exchange_plan(ctx, bis)
    plan.set_tuning(*tuning)
    odoms = [O.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    opat = O.make_pattern(w.edge, (w.halo,) * 4, odoms)
    es = [a.copy(order="K") for a in s_host]
    ev = [a.copy(order="K") for a in v_host]
    O.exchange(opat, odoms, es, [w.offsets()] * len(odoms), w.edge, False)
    O.exchange(opat, odoms, ev, [w.offsets()] * len(odoms), w.edge, True)
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        for t, a in zip(ts + tv, s_host + v_host):
            t.copy_(torch.from_numpy(a))
        plan.launch(form)
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(ts + tv, es + ev)) == 0
