"""Element sizes, memory orders, components and padded strides through the device exchange:
every box and list element class of the kernels in every form, and the adjoint for float fields,
bit-exact against the oracle."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from ghex_b200 import unstructured as U
from ghex_b200 import workloads as W
from ghex_b200.structured import regular as R
from gpu_helpers import bits_equal
from oracle import regular as O
from oracle import unstructured as OU

pytestmark = pytest.mark.gpu

SHAPE = (20, 16, 12)
HALOS = (2, 1, 1, 2, 1, 0)
PERIODIC = (True, False, True)


def _values(rng, shape, dtype):
    if np.dtype(dtype).kind == "f":
        return rng.standard_normal(shape).astype(dtype)
    info = np.iinfo(dtype)
    return rng.integers(info.min // 2, info.max // 2, size=shape, dtype=dtype)


def _run_forms(plan, tens, host, expected, adjoint_expected):
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        plan.launch(form)
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0, form
    if adjoint_expected is not None:
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        plan.adjoint()
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, adjoint_expected)) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int64, np.int32, np.uint16, np.uint8])
@pytest.mark.parametrize("order", ["F", "C"])
@pytest.mark.parametrize("ncomp", [1, 3])
def test_regular_dtypes_orders_components(cuda, dtype, order, ncomp):
    """Uneven 2x2x1 split, asymmetric halos, periodic in x and z."""
    doms_spec = W.regular_decomposition(SHAPE, (2, 2, 1), 3)
    ctx = R.make_context()
    hg = R.HaloGenerator(((0, 0, 0), tuple(n - 1 for n in SHAPE)),
                         [(HALOS[2 * k], HALOS[2 * k + 1]) for k in range(3)], PERIODIC)
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in doms_spec]
    pat = R.make_pattern(ctx, hg, doms)
    rng = np.random.default_rng(17)
    offsets = (HALOS[0], HALOS[2], HALOS[4])
    host, tens, bis = [], [], []
    for dm, (_, f, l) in zip(doms, doms_spec):
        ext = tuple(l[k] - f[k] + 1 + HALOS[2 * k] + HALOS[2 * k + 1] for k in range(3))
        shape = ext + ((ncomp,) if ncomp > 1 else ())
        a = np.asarray(_values(rng, shape, dtype), order=order)
        host.append(a)
        t = torch.from_numpy(a).to(cuda)
        assert t.stride() == torch.from_numpy(a).stride()
        tens.append(t)
        bis.append(pat(R.make_field_descriptor(dm, t, offsets, ext)))
    plan = R.make_exchange_plan(ctx, bis)
    odoms = [O.Domain(i, f, l) for i, f, l in doms_spec]
    opat = O.make_pattern((0, 0, 0), tuple(n - 1 for n in SHAPE), HALOS, PERIODIC, odoms)
    expected = [a.copy(order="K") for a in host]
    O.exchange(opat, odoms, expected, [offsets] * len(odoms))
    adj = None
    if np.dtype(dtype).kind == "f":
        adj = [a.copy(order="K") for a in host]
        O.adjoint(opat, odoms, adj, [offsets] * len(odoms))
    _run_forms(plan, tens, host, expected, adj)


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int32, np.uint16, np.uint8])
@pytest.mark.parametrize("levels", [1, 3, 7])
@pytest.mark.parametrize("layout", ["levels_first", "levels_last", "padded_first", "padded_last"])
def test_unstructured_units_and_strides(cuda, dtype, levels, layout):
    """Columns of 1 to 7 levels (16-byte units only where every column is 16-byte aligned, else
    element units); levels first or last, dense or with an outer stride beyond the levels or the
    vertices. Padding outside the field is left as it was."""
    w = W.config2(ni=32, nj=48, parts=4, levels=levels)
    rng = np.random.default_rng(5)
    host, tens, bases = [], [], []
    for d in w.domains:
        n = d[1].size
        if layout == "levels_first":
            base = torch.from_numpy(np.ascontiguousarray(_values(rng, (n, levels), dtype))).to(cuda)
            t = base
        elif layout == "levels_last":
            base = torch.from_numpy(np.asfortranarray(_values(rng, (n, levels), dtype))).to(cuda)
            t = base
        elif layout == "padded_first":
            base = torch.from_numpy(np.ascontiguousarray(_values(rng, (n, levels + 3), dtype))).to(cuda)
            t = base[:, :levels]
        else:
            base = torch.from_numpy(np.asfortranarray(_values(rng, (n + 5, levels), dtype))).to(cuda)
            t = base[:n]
        host.append(t.cpu().numpy().copy())
        tens.append(t)
        bases.append((base, base.cpu().numpy().copy()))
    ctx = U.make_context()
    doms = [U.DomainDescriptor(*d) for d in w.domains]
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    fds = [U.make_field_descriptor(d, t) for d, t in zip(doms, tens)]
    assert all(f.levels == levels for f in fds)
    bis = [pat(f) for f in fds]
    plan = U.make_exchange_plan(ctx, bis)
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    expected = [a.copy() for a in host]
    OU.exchange(recv, send, expected)
    adj = None
    if np.dtype(dtype).kind == "f":
        adj = [a.copy() for a in host]
        OU.adjoint(recv, send, adj)
    _run_forms(plan, tens, host, expected, adj)
    for (base, before), t in zip(bases, tens):
        after = base.cpu().numpy()
        mask = np.ones(after.shape, dtype=bool)
        mask[:t.shape[0], :t.shape[1]] = False
        assert bits_equal(after[mask], before[mask]) == 0
