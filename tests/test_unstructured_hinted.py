"""make_pattern with a receive domain ids generator (unstructured/pattern.hpp:371-588): the
send and receive maps of GHEX's check_send_halos_indices / check_recv_halos_indices, GHEX's own
exchange outputs (golden fixtures) and the known answers of check_exchanged_data, through the
oracle and through the library's pattern (CPU; the device exchange is in the gpu tests)."""
import numpy as np
import pytest

import golden_cases as G
from ghex_b200 import _capi
from ghex_b200 import unstructured as U
from oracle import reflib
from oracle import unstructured as OU


def _oracle():
    hc = G.hinted_case()
    ids = sorted(hc["domains"])
    doms = [OU.Domain(d, hc["domains"][d]["gids"], hc["domains"][d]["halo_lids"]) for d in ids]
    recv, send, max_tag = OU.make_pattern_hinted(doms, [hc["hints"][d] for d in ids], [hc["halo_gids"]] * len(ids))
    return hc, ids, doms, recv, send, max_tag


def test_oracle_maps_are_the_reference_test_maps():
    hc, ids, doms, recv, send, max_tag = _oracle()
    for i, d in enumerate(ids):
        assert {ids[e.neighbor]: e.lids for e in recv[i]} == hc["recv"][d]
        assert {ids[e.neighbor]: e.lids for e in send[i]} == hc["send"][d]
        for e in recv[i]:
            assert e.tag == (ids[e.neighbor] << 7) + d
    assert max_tag == (3 << 7) + 3


def test_library_pattern_matches_the_reference_test_maps():
    hc, ids, _, recv, send, max_tag = _oracle()
    ctx = U.make_context(device=0)
    ud = [U.DomainDescriptor(d, hc["domains"][d]["gids"], hc["domains"][d]["halo_lids"]) for d in ids]
    p = U.make_pattern(ctx, U.HaloGenerator(hc["halo_gids"]), lambda dom: hc["hints"][dom.domain_id()], ud)
    for i, d in enumerate(ids):
        assert {ids[nb]: lids for nb, lids in p.index_lists(i)} == hc["recv"][d]
        assert {ids[nb]: lids for nb, lids in p.index_lists(i, send=True)} == hc["send"][d]
    assert p.max_tag() == max_tag


class _RdigHalo:
    """The reference's recv_domain_ids_gen::halo shape: accessor methods."""

    def __init__(self, ids, rem):
        self._ids, self._rem = ids, rem

    def domain_ids(self):
        return self._ids

    def remote_indices(self):
        return self._rem

    def ranks(self):
        return [0] * len(self._ids)


def test_generator_objects_and_errors():
    hc, ids, *_ = _oracle()
    ctx = U.make_context(device=0)
    ud = [U.DomainDescriptor(d, hc["domains"][d]["gids"], hc["domains"][d]["halo_lids"]) for d in ids]
    hg = U.HaloGenerator(hc["halo_gids"])
    p = U.make_pattern(ctx, hg, lambda dom: _RdigHalo(*hc["hints"][dom.domain_id()]), ud)
    assert [lids for _, lids in p.index_lists(0)] == [hc["recv"][0][k] for k in sorted(hc["recv"][0])]
    bad_owner = lambda dom: ([7] * len(hc["hints"][dom.domain_id()][0]), hc["hints"][dom.domain_id()][1])
    with pytest.raises(_capi.GhexError, match="unknown domain 7"):
        U.make_pattern(ctx, hg, bad_owner, ud)
    # domain 0's halo element gid 1 named as local index 7 of domain 1 (an outer element there)
    outer_ref = lambda dom: (hc["hints"][dom.domain_id()][0],
                             [7] + hc["hints"][dom.domain_id()][1][1:] if dom.domain_id() == 0
                             else hc["hints"][dom.domain_id()][1])
    with pytest.raises(_capi.GhexError, match="not an inner element"):
        U.make_pattern(ctx, hg, outer_ref, ud)
    short = lambda dom: (hc["hints"][dom.domain_id()][0][:-1], hc["hints"][dom.domain_id()][1][:-1])
    with pytest.raises(_capi.GhexError, match="entries for the"):
        U.make_pattern(ctx, hg, short, ud)


@pytest.mark.parametrize("levels", [1, 2])
def test_oracle_matches_reference_outputs_and_known_answers(levels):
    hc, ids, doms, recv, send, _ = _oracle()
    arrs = G.hinted_arrays()
    fields = [arrs[f"in_{levels}_{d}"].copy() for d in ids]
    OU.exchange(recv, send, fields)
    for d, f in zip(ids, fields):
        assert np.array_equal(f, arrs[f"out_{levels}_{d}"])
    # check_exchanged_data: halo row from owner o holds o*10000 + gid*100 + level
    for i, d in enumerate(ids):
        out = arrs[f"out_{levels}_{d}"].reshape(len(hc["domains"][d]["gids"]), levels)
        owner = {lid: ids[e.neighbor] for e in recv[i] for lid in e.lids}
        for x, g in enumerate(hc["domains"][d]["gids"]):
            src = owner.get(x, d)
            assert list(out[x]) == [src * 10000 + g * 100 + l for l in range(levels)]


@pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built")
def test_reference_live_with_permuted_remote_order():
    """Hints that list a halo's owners out of gid order still pair each halo element with the
    named remote index: GHEX's own code and the oracle agree."""
    hc, ids, doms, *_ = _oracle()
    rng = np.random.default_rng(8)
    halo = [int(g) for g in rng.permutation(hc["halo_gids"])]
    hints = []
    for d in doms:
        lids = d.make_outer_lids(halo)
        owners, rem = [], []
        for lid in lids:
            g = d.gids[lid]
            o = next(x for x in doms if g in x.inner)
            owners.append(o.id)
            rem.append(o.inner[g])
        hints.append((owners, rem))
    arrays = [np.ascontiguousarray(rng.standard_normal((len(d.gids), 3))) for d in doms]
    ref = [a.copy() for a in arrays]
    reflib.unstructured_exchange_hinted([(d.id, d.gids, d.outer_lids) for d in doms], halo, hints, 3, ref)
    recv, send, _ = OU.make_pattern_hinted(doms, hints, [halo] * len(doms))
    OU.exchange(recv, send, arrays)
    assert all(np.array_equal(a, b) for a, b in zip(arrays, ref))
