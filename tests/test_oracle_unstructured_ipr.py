"""The in-place receive (unstructured/communication_object_ipr.hpp) restated in the oracle:
GHEX's own outputs on its in-place receive test case (golden fixtures), the known answers of
that test (check_exchanged_data, test/unstructured/unstructured_test_case.hpp), the placement of
a receive list that is out of storage order, and the layouts it rejects (CPU)."""
import numpy as np
import pytest

import golden_cases as G
from ghex_b200 import workloads as W
from oracle import reflib
from oracle import unstructured as OU


def _domains():
    doms, perm = G.ipr_case()
    return doms, perm, [OU.Domain(d, doms[d]["gids"], doms[d]["halo_lids"]) for d in sorted(doms)]


@pytest.mark.parametrize("levels", [1, 2])
@pytest.mark.parametrize("case", ["", "perm_"])
def test_oracle_matches_reference_outputs(levels, case):
    doms, perm, odoms = _domains()
    arrs = G.ipr_arrays()
    recv, send, _ = OU.make_pattern(odoms, None if not case else [perm] * len(odoms))
    fields = [arrs[f"{case}in_{levels}_{d}"].copy() for d in sorted(doms)]
    OU.exchange_in_place(recv, send, fields, odoms)
    for d, f in zip(sorted(doms), fields):
        assert f.dtype == arrs[f"{case}out_{levels}_{d}"].dtype
        assert np.array_equal(f, arrs[f"{case}out_{levels}_{d}"])


@pytest.mark.parametrize("levels", [1, 2])
def test_reference_outputs_pass_known_answers(levels):
    """Every halo row of a domain received from domain `did` holds did*10000 + gid*100 + level;
    the inner rows keep id*10000 + gid*100 + level."""
    doms, _, odoms = _domains()
    arrs = G.ipr_arrays()
    recv, _, _ = OU.make_pattern(odoms)
    for d in sorted(doms):
        out = arrs[f"out_{levels}_{d}"].reshape(len(doms[d]["gids"]), levels)
        owner = {lid: sorted(doms)[en.neighbor] for en in recv[d] for lid in en.lids}
        for x, g in enumerate(doms[d]["gids"]):
            src = owner.get(x, d)
            assert list(out[x]) == [src * 10000 + g * 100 + l for l in range(levels)]


def test_out_of_order_receive_lands_on_consecutive_rows():
    """With the permuted halo generator a receive list is out of storage order; GHEX puts its
    k-th value on row first + k, so the result differs from the ordinary exchange there."""
    doms, perm, odoms = _domains()
    arrs = G.ipr_arrays()
    recv, send, _ = OU.make_pattern(odoms, [perm] * len(odoms))
    assert any(en.lids != sorted(en.lids) for es in recv for en in es)
    ipr = [arrs[f"perm_in_2_{d}"].copy() for d in sorted(doms)]
    plain = [a.copy() for a in ipr]
    OU.exchange_in_place(recv, send, ipr, odoms)
    OU.exchange(recv, send, plain)
    assert any(not np.array_equal(a, b) for a, b in zip(ipr, plain))
    for d, es in enumerate(recv):
        for en in es:
            rows = np.arange(en.lids[0], en.lids[0] + len(en.lids))
            assert np.array_equal(np.sort(ipr[d][rows], axis=0), np.sort(plain[d][np.asarray(en.lids)], axis=0))


def test_rows_outside_the_halo_are_rejected():
    """The 4-domain case of GHEX's Python test stores halos interleaved across owners: an
    in-place receive would overwrite rows of other receives."""
    doms = G.unstructured_domains()
    odoms = [OU.Domain(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    recv, _, _ = OU.make_pattern(odoms)
    with pytest.raises(ValueError, match="consecutive halo rows"):
        OU.in_place_rows(recv, odoms)


def test_owner_grouped_lattice_places_like_the_exchange():
    w = W.config2(ni=32, nj=48, parts=4, levels=3, halo_by_owner=True)
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    rows = OU.in_place_rows(recv, odoms)
    assert all(list(en.lids) == r for es, rs in zip(recv, rows) for en, r in zip(es, rs))
    plain = W.config2(ni=32, nj=48, parts=4, levels=3)
    assert any(not np.array_equal(a[1], b[1]) for a, b in zip(w.domains, plain.domains))


@pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int32])
def test_oracle_matches_reference_on_lattice(dtype):
    """GHEX's communication_object_ipr run live on the owner-grouped lattice, 5 levels."""
    w = W.config2(ni=24, nj=40, parts=4, levels=5, halo_by_owner=True)
    rng = np.random.default_rng(9)
    arrays = [np.ascontiguousarray((rng.standard_normal((d[1].size, 5)) * 1000).astype(dtype)) for d in w.domains]
    ref = [a.copy() for a in arrays]
    reflib.unstructured_exchange_ipr([(d[0], d[1], d[2]) for d in w.domains], 5, ref)
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    OU.exchange_in_place(recv, send, arrays, odoms)
    for a, b in zip(arrays, ref):
        assert np.array_equal(a, b)
