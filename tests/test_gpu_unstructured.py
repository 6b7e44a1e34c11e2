"""GPU parity of the unstructured exchange: the reference's 4-domain test case (known answers and
GHEX's own outputs) and the benchmark's lattice, bit-exact against the oracle."""
import numpy as np
import pytest
import torch

import golden_cases as G
from ghex_b200 import unstructured as U
from ghex_b200 import workloads as W
from gpu_helpers import bits_equal
from oracle import unstructured as OU

pytestmark = pytest.mark.gpu


def run_device(ctx, doms_spec, arrays_per_field, form="co", halo_gen=None):
    doms = [U.DomainDescriptor(*d) for d in doms_spec]
    pat = U.make_pattern(ctx, halo_gen or U.HaloGenerator(), doms)
    tens, bis = [], []
    for arrays in arrays_per_field:
        ts = []
        for a in arrays:
            t = torch.from_numpy(a).to("cuda")
            assert t.stride() == torch.from_numpy(a).stride()
            ts.append(t)
        tens.append(ts)
        bis += [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, ts)]
    if form == "co":
        U.make_communication_object(ctx).exchange(bis).wait()
    elif form == "adjoint":
        U.make_exchange_plan(ctx, bis).adjoint()
    else:
        plan = U.make_exchange_plan(ctx, bis)
        plan.launch({"per_field": plan.PER_FIELD, "per_box": plan.PER_BOX, "batched": plan.BATCHED}[form])
    torch.cuda.synchronize()
    return [[t.cpu().numpy() for t in ts] for ts in tens]


@pytest.mark.parametrize("order", ["C", "F"])
@pytest.mark.parametrize("form", ["co", "per_box"])
def test_reference_fixture(cuda, order, form):
    g = G.unstructured_domains()
    arrs = G.unstructured_arrays()
    spec = [(r, g[r]["all"], g[r]["outer_lids"]) for r in sorted(g)]
    f64 = [np.array(arrs[f"in_{order}_{r}"], order=order) for r in sorted(g)]
    f32 = [x.astype(np.float32, order=order) for x in f64]
    one = [np.ascontiguousarray(x[:, 0]) for x in f64]  # a single level
    got64, got32, got1 = run_device(U.make_context(), spec, [f64, f32, one], form)
    for r, a, b, c in zip(sorted(g), got64, got32, got1):
        ref = arrs[f"out_{order}_{r}"]
        assert bits_equal(a, ref) == 0
        assert bits_equal(b, ref.astype(np.float32)) == 0
        assert bits_equal(c, np.ascontiguousarray(ref[:, 0])) == 0
        assert G.unstructured_check(a, g[r], r, 2) == 0


def test_explicit_halo_gids(cuda):
    g = G.unstructured_domains()
    arrs = G.unstructured_arrays()
    spec = [(r, g[r]["all"], g[r]["outer_lids"]) for r in sorted(g)]
    gens = [U.HaloGenerator.from_gids(g[r]["outer"]) for r in sorted(g)]
    f = [arrs[f"in_C_{r}"].copy() for r in sorted(g)]
    got = run_device(U.make_context(), spec, [f], halo_gen=gens)[0]
    for r, a in zip(sorted(g), got):
        assert bits_equal(a, arrs[f"out_C_{r}"]) == 0


def test_adjoint_with_repeated_gids(cuda):
    """The fixture's halos hold repeated gids (periodic images): one owner feeds several halo slots
    of one message, which the device adjoint must add in order."""
    g = G.unstructured_domains()
    spec = [(r, g[r]["all"], g[r]["outer_lids"]) for r in sorted(g)]
    rng = np.random.default_rng(9)
    grads = [rng.standard_normal((len(g[r]["all"]), 3)) for r in sorted(g)]
    got = run_device(U.make_context(), spec, [[x.copy() for x in grads]], form="adjoint")[0]
    odoms = [OU.Domain(*d) for d in spec]
    recv, send, _ = OU.make_pattern(odoms)
    OU.adjoint(recv, send, grads)
    for a, e in zip(got, grads):
        assert bits_equal(a, e) == 0


@pytest.mark.parametrize("levels_first", [True, False])
def test_cfg2_bitexact(cuda, levels_first):
    w = W.config2() if levels_first else W.config2(ni=128, nj=256, levels=8)
    f64 = [w.domain_array(d, np.float64, 1, levels_first) for d in w.domains]
    f32 = [w.domain_array(d, np.float32, 2, levels_first) for d in w.domains]
    got64, got32 = run_device(U.make_context(), w.domains, [f64, f32], "batched")
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    OU.exchange(recv, send, f64)
    OU.exchange(recv, send, f32)
    assert sum(bits_equal(a, e) for a, e in zip(got64, f64)) == 0
    assert sum(bits_equal(a, e) for a, e in zip(got32, f32)) == 0
    assert not any(np.isnan(a).any() for a in got64)  # every halo vertex has an owner


@pytest.mark.parametrize("share", [0, 1, 2, 4])
def test_bulk_kernel_shares_bitexact(cuda, share):
    """The bulk column kernel (cp.async.bulk through shared memory) taking none, a quarter, half
    (beside the element kernel on a second stream) and all of the lists, in the batched form and
    its graph: bit-exact against the oracle, and the staged/bulk status word stays 0."""
    w = W.config2(ni=256, nj=512, levels=64)
    f64 = [w.domain_array(d, np.float64, 1, True) for d in w.domains]
    f32 = [w.domain_array(d, np.float32, 2, True) for d in w.domains]
    doms = [U.DomainDescriptor(*d) for d in w.domains]
    ctx = U.make_context()
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    tens, bis = [], []
    for arrays in (f64, f32):
        ts = [torch.from_numpy(a).to("cuda") for a in arrays]
        tens.append(ts)
        bis += [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, ts)]
    plan = U.make_exchange_plan(ctx, bis)
    plan.set_bulk(share)
    info = plan.info()
    assert info["bulk_share"] == share and (info["bulk_tiles"] > 0) == (share > 0)
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    exp64, exp32 = [a.copy() for a in f64], [a.copy() for a in f32]
    OU.exchange(recv, send, exp64)
    OU.exchange(recv, send, exp32)
    for launch in (lambda: plan.launch(plan.BATCHED), lambda: plan.graph_launch()):
        for ts, arrays in zip(tens, (f64, f32)):
            for t, a in zip(ts, arrays):
                t.copy_(torch.from_numpy(a))
        launch()
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens[0], exp64)) == 0
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens[1], exp32)) == 0
    assert plan.staged_status() == 0


@pytest.mark.parametrize("levels_first", [True, False])
def test_cfg2_adjoint_one_launch_bitexact(cuda, levels_first):
    """The unstructured adjoint in gather form: one launch, every owner column adds its halo
    images in receive order (bit-exact against the explicit transpose), halos zeroed."""
    w = W.config2() if levels_first else W.config2(ni=128, nj=256, levels=8)
    rng = np.random.default_rng(21)
    order = "C" if levels_first else "F"
    g64 = [np.asarray(rng.standard_normal((d[1].size, w.levels)), order=order) for d in w.domains]
    g32 = [np.asarray(rng.standard_normal((d[1].size, w.levels)), dtype=np.float32, order=order) for d in w.domains]
    ctx = U.make_context()
    doms = [U.DomainDescriptor(*d) for d in w.domains]
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    t64 = [torch.from_numpy(a).to("cuda") for a in g64]
    t32 = [torch.from_numpy(a).to("cuda") for a in g32]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, t64)] + \
          [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, t32)]
    plan = U.make_exchange_plan(ctx, bis)
    assert plan.info()["adjoint_launches"] == 1
    plan.adjoint()
    torch.cuda.synchronize()
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    OU.adjoint(recv, send, g64)
    OU.adjoint(recv, send, g32)
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(t64, g64)) == 0
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(t32, g32)) == 0


def test_bulk_plan_rebind_bitexact(cuda):
    """A plan whose lists move through tensor maps (four-column bulk tiles) rebound to other
    memory: its maps are made again for the new fields, and the exchange there is bit-exact."""
    w = W.config2(ni=256, nj=512, levels=64)
    f64 = [w.domain_array(d, np.float64, 1, True) for d in w.domains]
    doms = [U.DomainDescriptor(*d) for d in w.domains]
    ctx = U.make_context()
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    first = [torch.from_numpy(a).to("cuda") for a in f64]
    plan = U.make_exchange_plan(ctx, [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, first)])
    plan.set_bulk(4)
    assert plan.info()["bulk_tiles"] > 0
    second = [torch.from_numpy(a).to("cuda") for a in f64]
    plan.rebind(second)
    plan.graph_launch()
    torch.cuda.synchronize()
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    exp = [a.copy() for a in f64]
    OU.exchange(recv, send, exp)
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(second, exp)) == 0
    assert sum(bits_equal(t.cpu().numpy(), a) for t, a in zip(first, f64)) == 0  # the old memory untouched
    assert plan.staged_status() == 0


@pytest.mark.parametrize("share", [2, 4])
def test_adjoint_bulk_gather_shares_bitexact(cuda, share):
    """The bulk gather kernel (columns by cp.async.bulk through shared memory, sums in shared
    memory in receive order) taking half or all of the owners, beside the element gather kernel:
    bit-exact against the explicit transpose, status word 0."""
    w = W.config2(ni=256, nj=512, levels=64)
    rng = np.random.default_rng(23)
    g64 = [np.asarray(rng.standard_normal((d[1].size, w.levels)), order="C") for d in w.domains]
    g32 = [np.asarray(rng.standard_normal((d[1].size, w.levels)), dtype=np.float32, order="C") for d in w.domains]
    ctx = U.make_context()
    doms = [U.DomainDescriptor(*d) for d in w.domains]
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    t64 = [torch.from_numpy(a).to("cuda") for a in g64]
    t32 = [torch.from_numpy(a).to("cuda") for a in g32]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, t64)] + \
          [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, t32)]
    plan = U.make_exchange_plan(ctx, bis)
    plan.set_adjoint_bulk(share)
    info = plan.info()
    assert info["gather_bulk"] == share and info["gather_bulk_tiles"] > 0
    assert info["adjoint_launches"] == (2 if share < 4 else 1)
    plan.adjoint()
    torch.cuda.synchronize()
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    OU.adjoint(recv, send, g64)
    OU.adjoint(recv, send, g32)
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(t64, g64)) == 0
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(t32, g32)) == 0
    assert plan.staged_status() == 0


@pytest.mark.parametrize("levels", [1, 2])
def test_receive_domain_ids_generator(levels):
    """make_pattern(ctx, hg, recv_domain_ids_gen, domains) of GHEX's C++ test case: GHEX's own
    outputs, through the communication object and an explicit plan in every form; the adjoint
    (float64) against the oracle's transpose."""
    hc = G.hinted_case()
    arrs = G.hinted_arrays()
    ids = sorted(hc["domains"])
    ctx = U.make_context()
    ud = [U.DomainDescriptor(d, hc["domains"][d]["gids"], hc["domains"][d]["halo_lids"]) for d in ids]
    pat = U.make_pattern(ctx, U.HaloGenerator(hc["halo_gids"]), lambda dom: hc["hints"][dom.domain_id()], ud)
    host = [arrs[f"in_{levels}_{d}"] for d in ids]
    tens = [torch.from_numpy(a).to("cuda") for a in host]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, tens)]
    U.make_communication_object(ctx).exchange(bis).wait()
    expected = [arrs[f"out_{levels}_{d}"] for d in ids]
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
    plan = U.make_exchange_plan(ctx, bis)
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        plan.launch(form)
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
    if host[0].dtype == np.float64:
        odoms = [OU.Domain(d, hc["domains"][d]["gids"], hc["domains"][d]["halo_lids"]) for d in ids]
        recv, send, _ = OU.make_pattern_hinted(odoms, [hc["hints"][d] for d in ids], [hc["halo_gids"]] * len(ids))
        adj = [a.copy() for a in host]
        OU.adjoint(recv, send, adj)
        for t, a in zip(tens, host):
            t.copy_(torch.from_numpy(a))
        plan.adjoint()
        torch.cuda.synchronize()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, adj)) == 0
