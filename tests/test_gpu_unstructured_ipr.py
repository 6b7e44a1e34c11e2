"""GPU parity of the in-place receive (unstructured/communication_object_ipr.hpp): GHEX's own
outputs on its in-place receive test case, including a receive list out of storage order, one
communication object per domain as in GHEX's test, from one thread and from two; the
owner-grouped lattice against the ordinary exchange; the layouts it rejects."""
import threading

import numpy as np
import pytest
import torch

import golden_cases as G
from ghex_b200 import unstructured as U
from ghex_b200 import workloads as W
from gpu_helpers import bits_equal
from oracle import unstructured as OU

pytestmark = pytest.mark.gpu


def _fixture(cuda, levels, case):
    doms, perm = G.ipr_case()
    arrs = G.ipr_arrays()
    ctx = U.make_context()
    ud = [U.DomainDescriptor(d, doms[d]["gids"], doms[d]["halo_lids"]) for d in sorted(doms)]
    hg = U.HaloGenerator(perm) if case else U.HaloGenerator()
    pat = U.make_pattern(ctx, hg, ud)
    tens = [torch.from_numpy(arrs[f"{case}in_{levels}_{d}"]).to(cuda) for d in sorted(doms)]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, tens)]
    expected = [arrs[f"{case}out_{levels}_{d}"] for d in sorted(doms)]
    return ctx, bis, tens, expected


@pytest.mark.parametrize("levels", [1, 2])
@pytest.mark.parametrize("case", ["", "perm_"])
def test_one_object_per_domain(cuda, levels, case):
    ctx, bis, tens, expected = _fixture(cuda, levels, case)
    cos = [U.make_communication_object_ipr(ctx, bi) for bi in bis]
    for _ in range(2):  # the second exchange reuses the plan
        hs = [co.exchange() for co in cos]
        for h in hs:
            h.wait()
            assert h.is_ready()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0


def test_two_threads(cuda):
    """GHEX's test_in_place_receive_threads: each thread owns two domains' objects, exchanges
    and waits; the exchange launches when the second thread has posted."""
    ctx, bis, tens, expected = _fixture(cuda, 2, "perm_")
    errors = []

    def run(pair):
        try:
            co = U.make_communication_object_ipr(ctx, pair)
            co.exchange().wait(timeout=60)
        except BaseException as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=run, args=(bis[2 * i:2 * i + 2],)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    torch.cuda.synchronize()
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_owner_grouped_lattice(cuda, dtype):
    """Halos grouped by owner: the in-place receive equals the ordinary exchange, through the
    communication object and through an explicit plan in every form."""
    w = W.config2(ni=64, nj=96, parts=8, levels=16, halo_by_owner=True)
    host = [w.domain_array(d, dtype, 3) for d in w.domains]
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    expected = [a.copy() for a in host]
    OU.exchange_in_place(recv, send, expected, odoms)
    plain = [a.copy() for a in host]
    OU.exchange(recv, send, plain)
    assert sum(bits_equal(a, b) for a, b in zip(expected, plain)) == 0
    ctx = U.make_context()
    ud = [U.DomainDescriptor(*d) for d in w.domains]
    pat = U.make_pattern(ctx, U.HaloGenerator(), ud)
    tens = [torch.from_numpy(a).to(cuda) for a in host]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, tens)]
    U.make_communication_object_ipr(ctx, bis).exchange().wait()
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
    plan = U.make_exchange_plan(ctx, bis, in_place_receive=True)
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        plan.launch(form)
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0


def test_rejected_layouts(cuda):
    """Halos interleaved across owners (GHEX's Python 4-domain case) and levels-last storage."""
    doms = G.unstructured_domains()
    ctx = U.make_context()
    ud = [U.DomainDescriptor(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    pat = U.make_pattern(ctx, U.HaloGenerator(), ud)
    tens = [torch.zeros((d.size(), 2), dtype=torch.float64, device=cuda) for d in ud]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, tens)]
    with pytest.raises(RuntimeError, match="consecutive halo rows"):
        U.make_communication_object_ipr(ctx, bis).exchange()
    idoms, _ = G.ipr_case()
    ctx = U.make_context()
    ud = [U.DomainDescriptor(d, idoms[d]["gids"], idoms[d]["halo_lids"]) for d in sorted(idoms)]
    pat = U.make_pattern(ctx, U.HaloGenerator(), ud)
    tens = [torch.zeros((2, d.size()), dtype=torch.float64, device=cuda).t() for d in ud]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, tens)]
    with pytest.raises(RuntimeError, match="levels of a halo element stored contiguously"):
        U.make_exchange_plan(ctx, bis, in_place_receive=True)
