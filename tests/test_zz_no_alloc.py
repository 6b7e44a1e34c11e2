"""ghexb_exchange_noalloc, the exchange entry point that allocates no device memory, gives the same
halos as the oracle and as the plan-based entry point, bit for bit, on consecutive calls.

It serves callers that cannot allocate device memory when they exchange (an application whose
memory manager owns the device memory, or code that must not call cudaMalloc/cudaFree because those
may synchronize the device). Its work tables live in one fixed device array shared by all calls,
so consecutive calls must each rewrite it completely; every case below calls it twice in a row
(halos reset to NaN in between) and then on another field set, so that no state of an earlier call
leaks into a later one. The unstructured case places index lists in the array (list tiles address
them there), the cubed-sphere case runs the negated vector components. This file is collected last
on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import golden_cases as G
from ghex_b200 import _capi
from ghex_b200 import unstructured as U
from ghex_b200 import workloads as W
from ghex_b200.structured import cubed_sphere as CS
from ghex_b200.structured import regular as R
from gpu_helpers import RegularRun, bits_equal, to_device
from oracle import cubed_sphere as OC
from oracle import unstructured as OU

pytestmark = pytest.mark.gpu


def noalloc_exchange(ctx, bis, stream=None):
    handles = [bi.handle() for bi in bis]
    arr = (C.c_void_p * len(handles))(*handles)
    s = stream if stream is not None else torch.cuda.current_stream()
    _capi.call("ghexb_exchange_noalloc", ctx._h, arr, len(handles), C.c_void_p(s.cuda_stream))
    torch.cuda.synchronize()


def plan_result(w, cuda, ctx):
    ref = RegularRun(w, cuda, ctx=ctx)
    plan = R.make_exchange_plan(ref.ctx, ref.bis)
    plan.launch(plan.BATCHED)
    torch.cuda.synchronize()
    return {name: [t.cpu().numpy() for t in tens] for name, tens in ref.dev.items()}


def test_noalloc_regular_matches_oracle_and_plan(cuda):
    ctx = R.make_context()
    w1 = W.config1(shape=(60, 45, 15))
    run = RegularRun(w1, cuda, ctx=ctx)
    oracle1 = run.oracle()
    assert run.mismatches(oracle1) != {}  # halos start as NaN
    planned = plan_result(w1, cuda, ctx)
    for name in oracle1:
        assert sum(bits_equal(a, b) for a, b in zip(planned[name], oracle1[name])) == 0

    noalloc_exchange(ctx, run.bis)  # first call: also looks up the scratch array on this device
    assert run.mismatches(oracle1) == {}
    run.reset()  # halos back to NaN
    noalloc_exchange(ctx, run.bis)  # second call in a row, same tables rewritten
    assert run.mismatches(oracle1) == {}

    # a different field set through the same scratch array
    w2 = W.config0()
    run2 = RegularRun(w2, cuda, ctx=ctx)
    noalloc_exchange(ctx, run2.bis)
    assert run2.mismatches(run2.oracle()) == {}
    assert run2.mismatches(plan_result(w2, cuda, ctx)) == {}


def test_noalloc_unstructured_index_lists(cuda):
    g = G.unstructured_domains()
    arrs = G.unstructured_arrays()
    spec = [(r, g[r]["all"], g[r]["outer_lids"]) for r in sorted(g)]
    ctx = U.make_context()
    doms = [U.DomainDescriptor(*d) for d in spec]
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    f64 = [np.array(arrs[f"in_C_{r}"]) for r in sorted(g)]
    f32 = [x.astype(np.float32) for x in f64]
    host = [f64, f32]
    tens = [[torch.from_numpy(a).to(cuda) for a in field] for field in host]
    bis = [pat(U.make_field_descriptor(d, t)) for ts in tens for d, t in zip(doms, ts)]

    odoms = [OU.Domain(*d) for d in spec]
    recv, send, _ = OU.make_pattern(odoms)
    expected = []
    for field in host:
        ex = [a.copy() for a in field]
        OU.exchange(recv, send, ex)
        expected.append(ex)
    # the reference's own outputs pin the oracle on this case
    for r, e in zip(sorted(g), expected[0]):
        assert bits_equal(e, arrs[f"out_C_{r}"]) == 0

    for call in range(2):
        for ts, field in zip(tens, host):
            for t, a in zip(ts, field):
                t.copy_(torch.from_numpy(a))
        noalloc_exchange(ctx, bis)
        for ts, ex in zip(tens, expected):
            for t, e in zip(ts, ex):
                assert bits_equal(t.cpu().numpy(), e) == 0, f"call {call}"


def test_noalloc_cubed_sphere_vector_signs(cuda):
    w = W.config3(edge=48, levels=8, split=2)
    ctx = CS.make_context()
    cube = CS.cube(w.edge, w.levels)
    doms = [CS.DomainDescriptor(cube, *b) for b in w.domains]
    pat = CS.make_pattern(ctx, CS.HaloGenerator(w.halo), doms)
    host = {"s": [w.domain_array(d, 1, 1) for d in w.domains], "v": [w.domain_array(d, 2, 2) for d in w.domains]}
    tens = {k: [to_device(a, cuda) for a in v] for k, v in host.items()}
    bis = []
    for k, nc, vec in (("s", 1, False), ("v", 2, True)):
        bis += [pat(CS.make_field_descriptor(d, t, w.offsets(), a.shape[:3], nc, vec))
                for d, t, a in zip(doms, tens[k], host[k])]
    odoms = [OC.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    opat = OC.make_pattern(w.edge, (w.halo,) * 4, odoms)
    expected = {}
    for k, vec in (("s", False), ("v", True)):
        ex = [a.copy(order="K") for a in host[k]]
        OC.exchange(opat, odoms, ex, [w.offsets()] * len(odoms), w.edge, vec)
        expected[k] = ex
    for call in range(2):
        for k in tens:
            for t, a in zip(tens[k], host[k]):
                t.copy_(torch.from_numpy(a))
        noalloc_exchange(ctx, bis)
        for k in tens:
            for t, e in zip(tens[k], expected[k]):
                assert bits_equal(t.cpu().numpy(), e) == 0, f"call {call}, field {k}"


def test_noalloc_refuses_oversized_tables_and_capture(cuda):
    # 2048 domains of 4^3 cells, halo 1: more than 53,000 halo boxes, whose tiles need more than
    # the 4 MiB of the scratch array; refused before any copy or launch
    ctx = R.make_context()
    shape, parts = (64, 64, 32), (16, 16, 8)
    domains = W.regular_decomposition(shape, parts)
    hg = R.HaloGenerator(((0, 0, 0), tuple(n - 1 for n in shape)), (1, 1, 1), (True, True, True))
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in domains]
    pat = R.make_pattern(ctx, hg, doms)
    tens = [torch.zeros((6, 6, 6), dtype=torch.float64, device=cuda).permute(2, 1, 0) for _ in domains]
    bis = [pat(R.make_field_descriptor(d, t, (1, 1, 1), (6, 6, 6))) for d, t in zip(doms, tens)]
    with pytest.raises(RuntimeError, match="no-alloc scratch"):
        noalloc_exchange(ctx, bis)

    # a stream under capture is refused (the tables are copied from a buffer of the call)
    w = W.config0()
    run = RegularRun(w, cuda, ctx=ctx)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with pytest.raises(RuntimeError, match="captured"):
        with torch.cuda.graph(g, stream=s):
            handles = [bi.handle() for bi in run.bis]
            arr = (C.c_void_p * len(handles))(*handles)
            _capi.call("ghexb_exchange_noalloc", ctx._h, arr, len(handles), C.c_void_p(s.cuda_stream))
    torch.cuda.synchronize()
    # the entry point still works afterwards
    noalloc_exchange(ctx, run.bis)
    assert run.mismatches(run.oracle()) == {}
