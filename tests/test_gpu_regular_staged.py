"""GPU parity of the staged regular pattern (structured/regular/make_pattern.hpp:47-256): the
stages exchanged one after the other on the device give GHEX's own staged outputs (golden
fixtures), the known answers of test_simple_regular_domain.cpp, and the oracle's staged exchange
for other element sizes and memory orders; every stage's plan in every form."""
import numpy as np
import pytest
import torch

import golden_cases as G
import regular_cases as RC
from ghex_b200.structured import regular as R
from gpu_helpers import bits_equal, to_device
from oracle import regular as O

pytestmark = pytest.mark.gpu


def _device_stages(case, tensors, ctx=None):
    ctx = ctx or R.make_context()
    dim = len(case["shape"])
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in case["domains"]]
    pats = R.make_staged_pattern(ctx, doms, case["lookup"], (0,) * dim, tuple(n - 1 for n in case["shape"]),
                                 case["halos"], case["periodic"])
    ext = lambda t: tuple(t.shape[:dim])
    fds = [R.make_field_descriptor(d, t, case["offsets"], ext(t)) for d, t in zip(doms, tensors)]
    return ctx, pats, fds


@pytest.mark.parametrize("name", ["simple_2d_1x1", "simple_2d_2x2"])
def test_simple_2d_staged(cuda, name):
    case = RC.staged_cases()[name]
    gold = G.staged_arrays()
    n = len(case["domains"])
    tens = [to_device(RC.pairs_view(gold[f"{name}_in_{i}"]), cuda) for i in range(n)]
    ctx, pats, fds = _device_stages(case, tens)
    co = R.make_communication_object(ctx)
    for p in pats:
        co.exchange([p(f) for f in fds]).wait()
    for i, ((_, f, l), t) in enumerate(zip(case["domains"], tens)):
        got = t.cpu().numpy()
        assert bits_equal(got, RC.pairs_view(gold[f"{name}_out_{i}"])) == 0
        assert RC.simple_2d_check(got, f, l, (True, True), case["dims"]) == []


def test_uneven_3d_staged_golden(cuda):
    case = RC.staged_cases()["uneven_3d"]
    gold = G.staged_arrays()
    n = len(case["domains"])
    host = [gold[f"uneven_3d_in_{i}"] for i in range(n)]
    tens = [to_device(np.asfortranarray(a), cuda) for a in host]
    ctx, pats, fds = _device_stages(case, tens)
    co = R.make_communication_object(ctx)
    for p in pats:
        co.exchange([p(f) for f in fds]).wait()
    assert sum(bits_equal(t.cpu().numpy(), gold[f"uneven_3d_out_{i}"]) for i, t in enumerate(tens)) == 0
    # every stage's plan, in every form, gives the same result
    plans = [R.make_exchange_plan(ctx, [p(f) for f in fds]) for p in pats]
    for form in (plans[0].BATCHED, plans[0].PER_FIELD, plans[0].PER_BOX):
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        for pl in plans:
            pl.launch(form)
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), gold[f"uneven_3d_out_{i}"]) for i, t in enumerate(tens)) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.int64, np.uint16, np.uint8])
@pytest.mark.parametrize("order", ["F", "C"])
def test_staged_dtypes_orders(cuda, dtype, order):
    case = RC.staged_cases()["uneven_3d"]
    rng = np.random.default_rng(31)
    host = []
    for _, f, l in case["domains"]:
        ext = tuple(l[k] - f[k] + 1 + case["halos"][2 * k] + case["halos"][2 * k + 1] for k in range(3))
        host.append(np.asarray(rng.integers(0, 200, size=ext).astype(dtype), order=order))
    tens = [to_device(a, cuda) for a in host]
    ctx, pats, fds = _device_stages(case, tens)
    co = R.make_communication_object(ctx)
    for p in pats:
        co.exchange([p(f) for f in fds]).wait()
    doms = [O.Domain(i, f, l) for i, f, l in case["domains"]]
    st = O.make_staged_pattern((0, 0, 0), tuple(n - 1 for n in case["shape"]), case["halos"], case["periodic"],
                               doms, case["lookup"])
    expected = [a.copy(order="K") for a in host]
    O.exchange_staged(st, doms, expected, [case["offsets"]] * len(doms))
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
