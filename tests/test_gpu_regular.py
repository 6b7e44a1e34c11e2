"""GPU parity of the regular structured exchange: bit-exact against the oracle, through the C ABI."""
import numpy as np
import pytest
import torch

from ghex_b200 import _capi
from ghex_b200 import workloads as W
from ghex_b200.structured import regular as R
from gpu_helpers import RegularRun, bits_equal, to_device
from regular_cases import DIM, HALO, simple_2d_check, simple_2d_domains, simple_2d_fields

pytestmark = pytest.mark.gpu


def test_cfg0_exchange_bitexact(cuda):
    run = RegularRun(W.config0(), cuda)
    expected = run.oracle()
    co = R.make_communication_object(run.ctx)
    co.exchange(run.bis).wait()
    assert run.mismatches(expected) == {}


@pytest.mark.parametrize("form", ["batched", "per_field", "per_box", "graph"])
def test_cfg1_small_all_forms_bitexact(cuda, form):
    run = RegularRun(W.config1(shape=(60, 45, 15)), cuda)
    expected = run.oracle()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    if form == "graph":
        plan.graph_launch()
    else:
        plan.launch({"batched": plan.BATCHED, "per_field": plan.PER_FIELD, "per_box": plan.PER_BOX}[form])
    assert run.mismatches(expected) == {}
    info = plan.info()
    assert info["num_fields"] == 5 * 27


def test_cfg1_full_size_bitexact(cuda):
    w = W.config1()
    run = RegularRun(w, cuda)
    expected = run.oracle()
    co = R.make_communication_object(run.ctx)
    for _ in range(2):  # second exchange reuses the cached plan and graph
        co.exchange(run.bis).wait()
    assert run.mismatches(expected) == {}
    plan = R.make_exchange_plan(run.ctx, run.bis)
    info = plan.info()
    # algorithmic bytes = sum over written halo cells of sizeof(T) * 2
    n64 = sum(int(np.count_nonzero(~np.isnan(e) & np.isnan(h))) for e, h in zip(expected["f64_0"], run.host["f64_0"]))
    n32 = sum(int(np.count_nonzero(~np.isnan(e) & np.isnan(h))) for e, h in zip(expected["f32_0"], run.host["f32_0"]))
    assert info["algorithmic_bytes"] == 3 * n64 * 16 + 2 * n32 * 8


@pytest.mark.parametrize("per_thread,block", [(4, 32), (8, 128), (16, 512), (16, 96)])
def test_tunings_bitexact(cuda, per_thread, block):
    run = RegularRun(W.config1(shape=(50, 40, 12)), cuda)
    expected = run.oracle()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    plan.set_tuning(per_thread, block, 1)
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        run.reset()
        plan.launch(form)
        assert run.mismatches(expected) == {}


def test_bad_tuning_rejected(cuda):
    run = RegularRun(W.config1(shape=(50, 40, 12)), cuda)
    plan = R.make_exchange_plan(run.ctx, run.bis)
    with pytest.raises(Exception, match="4, 8 or 16"):
        plan.set_tuning(5, 128)
    with pytest.raises(Exception, match="multiple of 32"):
        plan.set_tuning(8, 100)


def test_autotune_then_bitexact(cuda):
    run = RegularRun(W.config1(shape=(80, 60, 24)), cuda)
    expected = run.oracle()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    info = plan.autotune(repeats=2)
    assert info["elems_per_thread"] in (4, 8, 16) and info["block"] in (128, 256, 512)
    run.reset()
    plan.graph_launch()
    assert run.mismatches(expected) == {}


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_autotune_keeps_fields(cuda, dtype):
    """The autotuner times exchanges and adjoints on the plan's own fields: after it, every cell
    (interiors and halos) holds what one exchange of the original values leaves."""
    shape = (40, 30, 12)
    w = W.RegularWorkload("tune", shape, (True, True, False), W.regular_decomposition(shape, (2, 2, 1), 3))
    w.fields = [W.FieldSpec("f", dtype, (2, 2, 1, 1, 1, 1), 4), W.FieldSpec("g", dtype, (1, 1, 1, 1, 0, 0), 9)]
    run = RegularRun(w, cuda)
    expected = run.oracle()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    info = plan.autotune(repeats=2)
    assert info["gather_scale"] in (-1, 0, 1, 2)
    assert run.mismatches(expected) == {}


@pytest.mark.parametrize("periodic", [(True, True), (False, True)])
def test_simple_2d_known_answer(cuda, periodic):
    """test_simple_regular_domain.cpp's check on the device: (x, y) int32 pairs, x fastest."""
    doms = simple_2d_domains()
    host = simple_2d_fields(doms)
    ctx = R.make_context()
    hg = R.HaloGenerator(((0, 0), (2 * DIM - 1, 4 * (DIM // 2) - 1)), (HALO, HALO), periodic)
    dds = [R.DomainDescriptor(i, (f, l)) for i, f, l in doms]
    pat = R.make_pattern(ctx, hg, dds)
    tens, bis = [], []
    for dd, a in zip(dds, host):
        # memory order [y][x][pair] as the reference's layout_map<1,0> field of array<int,2>
        buf = np.ascontiguousarray(a.transpose(1, 0, 2)).transpose(1, 0, 2)
        t = to_device(buf, cuda)
        tens.append(t)
        fd = R.make_field_descriptor(dd, t, (HALO, HALO), (DIM + 2 * HALO, DIM // 2 + 2 * HALO))
        bis.append(pat(fd))
    co = R.make_communication_object(ctx)
    co.exchange(bis).wait()
    for (i, f, l), t in zip(doms, tens):
        assert simple_2d_check(t.cpu().numpy(), f, l, periodic) == [], f"domain {i}"


def test_busy_guard_and_errors(cuda):
    run = RegularRun(W.config0(), cuda)
    co = R.make_communication_object(run.ctx)
    h = co.exchange(run.bis)
    with pytest.raises(_capi.GhexError) as e:
        co.exchange(run.bis)
    assert e.value.code == _capi.ERR_BUSY and "not finished" in str(e.value)
    h.wait()
    co.exchange(run.bis).wait()
    # a neighbour without a field in the exchange
    with pytest.raises(_capi.GhexError) as e:
        co.exchange(run.bis[:3]).wait()
    assert e.value.code == _capi.ERR_INCOMPATIBLE


def test_out_of_range_box_is_rejected(cuda):
    w = W.config0()
    ctx = R.make_context()
    hg = R.HaloGenerator(((0, 0, 0), (63, 63, 63)), (2, 2, 2), (True, True, True))
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
    pat = R.make_pattern(ctx, hg, doms)
    # memory padded for halo 1 only: the halo-2 boxes do not fit
    tens = [torch.zeros((34, 34, 34), dtype=torch.float64, device=cuda) for _ in doms]
    bis = [pat(R.make_field_descriptor(d, t, (1, 1, 1), (34, 34, 34))) for d, t in zip(doms, tens)]
    with pytest.raises(_capi.GhexError) as e:
        R.make_exchange_plan(ctx, bis)
    assert e.value.code == _capi.ERR_RANGE


@pytest.mark.parametrize("gather_scale", [0, -1, 1, 2])
@pytest.mark.parametrize("cfg", ["cfg0", "cfg1_small", "cfg4_small"])
def test_adjoint_bitexact(cuda, cfg, gather_scale):
    """The device adjoint equals the oracle's fixed-order explicit transpose bit for bit, on random
    data in every cell (halos included), at every gather-tile size."""
    from oracle import regular as O
    w = {"cfg0": W.config0(), "cfg1_small": W.config1(shape=(50, 40, 12)),
         "cfg4_small": W.config4(shape=(32, 32, 16))}[cfg]
    run = RegularRun(w, cuda)
    rng = np.random.default_rng(5)
    grads = {}
    for name, tens in run.dev.items():
        grads[name] = []
        for t in tens:
            g = rng.standard_normal(t.shape).astype(t.cpu().numpy().dtype)
            g = np.asfortranarray(g)
            t.copy_(torch.from_numpy(g))
            grads[name].append(g)
    torch.cuda.synchronize()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    plan.set_adjoint_tuning(gather_scale)
    info = plan.info()
    assert info["adjoint_launches"] == 1 and info["adjoint_cells"] > 0 and info["gather_scale"] == gather_scale
    plan.adjoint()
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for spec in specs:
            O.adjoint(pat, doms, grads[spec.name], [w.offsets(spec)] * len(doms))
    assert run.mismatches(grads) == {}


@pytest.mark.parametrize("halos", [(2, 1, 1, 1, 0, 0), (3, 3, 1, 2, 1, 1), (1, 1, 1, 1, 1, 1)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_paired_x_faces_bitexact(cuda, halos, dtype):
    """x-face boxes of both sides of a row boundary move as one contiguous segment (equal and
    unequal halo widths): every form bit-exact against the oracle."""
    shape = (24, 20, 10)
    w = W.RegularWorkload("pairs", shape, (True, True, False), W.regular_decomposition(shape, (3, 2, 1), 7))
    w.fields = [W.FieldSpec("f", dtype, halos, 5), W.FieldSpec("g", dtype, halos, 6)]
    run = RegularRun(w, cuda)
    expected = run.oracle()
    plan = R.make_exchange_plan(run.ctx, run.bis)
    assert plan.info()["pairs"] >= 2 * len(w.domains)
    for pairs in (1, 0):
        plan.set_tuning(0, 0, pairs)
        assert plan.info()["use_pairs"] == pairs
        for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
            run.reset()
            plan.launch(form)
            assert run.mismatches(expected) == {}
    run.reset()
    plan.graph_launch()
    assert run.mismatches(expected) == {}


@pytest.mark.parametrize("ranks", [1, 2, 4])
def test_mixed_3d_known_answers(cuda, ranks):
    """test_regular_domain.cpp on the device: fields of array<double, 3>, array<float, 3> and
    array<int, 3> cells (components innermost, x fastest) on two patterns with different halos,
    all exchanged by one communication object call; bit-exact against the oracle and passing the
    test's check_values."""
    import regular_cases as RC
    from oracle import regular as O
    doms, g_last = RC.mixed_3d_domains(ranks)
    ctx = R.make_context()
    dds = [R.DomainDescriptor(i, (f, l)) for i, f, l in doms]
    pats = {h: R.make_pattern(ctx, R.HaloGenerator(((0, 0, 0), g_last), [(h[2 * k], h[2 * k + 1]) for k in range(3)],
                                                   (True, True, True)), dds)
            for h in (RC.MIXED_HALOS_1, RC.MIXED_HALOS_2)}
    odoms = [O.Domain(i, f, l) for i, f, l in doms]
    bis, runs = [], []
    ext = tuple(RC.MIXED_EXT[k] + 2 * RC.MIXED_OFFSET[k] for k in range(3))
    for dtype, halos in ((np.float64, RC.MIXED_HALOS_1), (np.float32, RC.MIXED_HALOS_2), (np.int32, RC.MIXED_HALOS_1)):
        host = [RC.mixed_3d_field(d, dtype) for d in doms]
        tens = [to_device(a, cuda) for a in host]
        bis += [pats[halos](R.make_field_descriptor(dd, t, RC.MIXED_OFFSET, ext)) for dd, t in zip(dds, tens)]
        expected = [a.copy() for a in host]
        O.exchange(O.make_pattern((0, 0, 0), g_last, halos, (True, True, True), odoms), odoms, expected,
                   [RC.MIXED_OFFSET] * len(doms))
        runs.append((halos, tens, expected))
    R.make_communication_object(ctx).exchange(bis).wait()
    for halos, tens, expected in runs:
        got = [t.cpu().numpy() for t in tens]
        assert sum(bits_equal(g, e) for g, e in zip(got, expected)) == 0
        assert sum(RC.mixed_3d_check(g, d, halos, ranks, g_last) for g, d in zip(got, doms)) == 0
