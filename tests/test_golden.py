"""The oracle restatements reproduce GHEX's own outputs (golden fixtures made by running the
reference's exchange) bit for bit, and the fixtures pass the known answers of the reference's
tests (CPU)."""
import numpy as np
import pytest

import cs_cases as cs
import golden_cases as G
from ghex_b200 import workloads as W
from oracle import cubed_sphere as OC
from oracle import regular as OR
from oracle import unstructured as OU


def bits(a):
    return np.ascontiguousarray(a).view(f"u{a.itemsize}")


@pytest.mark.parametrize("order", ["C", "F"])
def test_unstructured_fixture_known_answers_and_oracle(order):
    doms = G.unstructured_domains()
    arrs = G.unstructured_arrays()
    for r in sorted(doms):
        assert G.unstructured_check(arrs[f"out_{order}_{r}"], doms[r], r, 2) == 0
        assert G.unstructured_check(arrs[f"in_{order}_{r}"], doms[r], r, 2) > 0  # halos start at -1
    odoms = [OU.Domain(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    recv, send, _ = OU.make_pattern(odoms)
    fields = [np.array(arrs[f"in_{order}_{r}"], order=order) for r in sorted(doms)]
    OU.exchange(recv, send, fields)
    for r, f in zip(sorted(doms), fields):
        assert np.array_equal(bits(f), bits(arrs[f"out_{order}_{r}"]))


def test_unstructured_fixture_with_explicit_halo_gids():
    """halo_generator(gids) with each domain's outer gid list gives the same exchange."""
    doms = G.unstructured_domains()
    arrs = G.unstructured_arrays()
    odoms = [OU.Domain(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    recv, send, _ = OU.make_pattern(odoms, [doms[r]["outer"] for r in sorted(doms)])
    fields = [arrs[f"in_C_{r}"].copy() for r in sorted(doms)]
    OU.exchange(recv, send, fields)
    for r, f in zip(sorted(doms), fields):
        assert np.array_equal(bits(f), bits(arrs[f"out_C_{r}"]))


def test_unstructured_cpp_pattern_matches_oracle():
    from ghex_b200 import unstructured as U
    doms = G.unstructured_domains()
    ctx = U.make_context(device=0)
    ud = [U.DomainDescriptor(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    for r, d in zip(sorted(doms), ud):
        assert d.domain_id() == r and d.size() == len(doms[r]["all"]) and d.inner_size() == len(doms[r]["inner"])
    p = U.make_pattern(ctx, U.HaloGenerator(), ud)
    odoms = [OU.Domain(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    recv, send, max_tag = OU.make_pattern(odoms)
    for i in range(len(ud)):
        assert p.index_lists(i) == [(e.neighbor, e.lids) for e in recv[i]]
        assert p.index_lists(i, send=True) == [(e.neighbor, e.lids) for e in send[i]]
    assert p.max_tag() == max_tag


@pytest.mark.parametrize("kind", ["scalar", "vector"])
def test_cubed_sphere_golden(kind):
    arrs = G.cubed_arrays()
    odoms = [OC.Domain(t, (x0, x1), (y0, y1), cs.LEVELS) for t, x0, x1, y0, y1 in cs.domains()]
    fields = cs.fields()
    OC.exchange(OC.make_pattern(cs.EDGE, (cs.HALO,) * 4, odoms), odoms, fields,
                [(cs.MEM_HALO, cs.MEM_HALO, 0)] * len(odoms), cs.EDGE, kind == "vector")
    for i, f in enumerate(fields):
        assert np.array_equal(bits(f), bits(arrs[f"{kind}_{i}"]))


@pytest.mark.parametrize("case", ["periodic", "batched"])
def test_regular_golden(case):
    arrs = G.regular_arrays()
    w = (W.RegularWorkload("16^3", (16, 16, 16), (True, True, True), W.regular_decomposition((16, 16, 16), (2, 2, 2)),
                           [W.FieldSpec("f64", np.float64, (1,) * 6, 7)]) if case == "periodic"
         else W.config1(shape=(40, 30, 12)))
    for halos, specs in w.halo_groups().items():
        doms = [OR.Domain(i, f, l) for i, f, l in w.domains]
        pat = OR.make_pattern((0,) * 3, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for s in specs:
            fields = [w.domain_array(d, s) for d in w.domains]
            OR.exchange(pat, doms, fields, [w.offsets(s)] * len(doms))
            for i, f in enumerate(fields):
                assert np.array_equal(bits(f), bits(arrs[f"{case}_{s.name}_{i}"])), (s.name, i)
