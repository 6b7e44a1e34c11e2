"""The staged regular pattern (structured/regular/make_pattern.hpp:47-256) on the CPU: the
oracle's restatement against GHEX's own staged exchange (golden fixtures), the known answers of
test_simple_regular_domain.cpp after the staged exchange, staged == full exchange on consistent
decompositions, the C++ pattern's spaces and tags against the oracle's, and the refused
zero-width case."""
import numpy as np
import pytest

import golden_cases as G
import regular_cases as RC
from ghex_b200 import _capi
from ghex_b200 import workloads as W
from ghex_b200.structured import regular as R
from oracle import reflib
from oracle import regular as O


def _stages(case):
    doms = [O.Domain(i, f, l) for i, f, l in case["domains"]]
    dim = len(case["shape"])
    st = O.make_staged_pattern((0,) * dim, tuple(n - 1 for n in case["shape"]), case["halos"], case["periodic"],
                               doms, case["lookup"])
    return doms, st


@pytest.mark.parametrize("name", ["simple_2d_1x1", "simple_2d_2x2", "uneven_3d"])
def test_oracle_matches_reference_outputs(name):
    case = RC.staged_cases()[name]
    gold = G.staged_arrays()
    doms, st = _stages(case)
    arrays = [gold[f"{name}_in_{i}"] for i in range(len(doms))]
    O.exchange_staged(st, doms, arrays, [case["offsets"]] * len(doms))
    for i, a in enumerate(arrays):
        assert np.array_equal(a, gold[f"{name}_out_{i}"])


@pytest.mark.parametrize("name", ["simple_2d_1x1", "simple_2d_2x2"])
def test_reference_outputs_pass_known_answers(name):
    case = RC.staged_cases()[name]
    gold = G.staged_arrays()
    for i, (_, f, l) in enumerate(case["domains"]):
        assert RC.simple_2d_check(RC.pairs_view(gold[f"{name}_out_{i}"]), f, l, (True, True), case["dims"]) == []
        assert RC.simple_2d_check(RC.pairs_view(gold[f"{name}_in_{i}"]), f, l, (True, True), case["dims"]) != []


@pytest.mark.parametrize("shape,parts,halos,periodic", [
    ((16, 12, 10), (2, 2, 2), (1, 1, 1, 1, 1, 1), (True, True, True)),
    ((20, 16, 12), (3, 2, 3), (2, 1, 1, 2, 1, 2), (False, False, False)),
    ((9, 7, 5), (1, 1, 1), (2, 2, 1, 1, 1, 1), (True, True, False)),
    ((16, 12, 10), (2, 3, 1), (3, 3, 3, 3, 0, 0), (False, True, False))])
def test_staged_equals_full_exchange(shape, parts, halos, periodic):
    spec = W.regular_decomposition(shape, parts, 3)
    doms = [O.Domain(i, f, l) for i, f, l in spec]
    st = O.make_staged_pattern((0, 0, 0), tuple(n - 1 for n in shape), halos, periodic, doms,
                               W.cartesian_lookup(parts))
    full = O.make_pattern((0, 0, 0), tuple(n - 1 for n in shape), halos, periodic, doms)
    rng = np.random.default_rng(1)
    offs = (halos[0], halos[2], halos[4])
    arrs = [rng.standard_normal(tuple(d.last[k] - d.first[k] + 1 + halos[2 * k] + halos[2 * k + 1] for k in range(3)))
            for d in doms]
    a, b = [x.copy() for x in arrs], [x.copy() for x in arrs]
    O.exchange_staged(st, doms, a, [offs] * len(doms))
    O.exchange(full, doms, b, [offs] * len(doms))
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def _cpp_stages(case):
    ctx = R.make_context(device=0)
    dim = len(case["shape"])
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in case["domains"]]
    return ctx, R.make_staged_pattern(ctx, doms, case["lookup"], (0,) * dim, tuple(n - 1 for n in case["shape"]),
                                      case["halos"], case["periodic"])


@pytest.mark.parametrize("name", ["simple_2d_1x1", "simple_2d_2x2", "uneven_3d"])
def test_cpp_pattern_matches_oracle(name):
    case = RC.staged_cases()[name]
    _, st = _stages(case)
    ctx, pats = _cpp_stages(case)
    dim = len(case["shape"])
    assert len(pats) == dim
    pad = lambda t: tuple(t) + (0,) * (4 - len(t))
    for (recv, send), p in zip(st, pats):
        tags = [e.tag for es in recv for e in es]
        assert p.max_tag() == max(tags + [0])
        for d in range(len(case["domains"])):
            for side, entries in ((False, recv[d]), (True, send[d])):
                want = [(e.neighbor, pad(s.lfirst), pad(s.llast), pad(s.gfirst), pad(s.glast))
                        for e in entries for s in e.spaces]
                assert p.spaces(d, send=side) == want


def test_zero_halo_on_one_side_is_refused():
    """A zero halo width on one side only: the reference's staged messages do not match (a
    receive expects data the sender never packs); both the oracle and the library refuse it."""
    shape, parts, halos, periodic = (20, 16, 12), (3, 2, 2), (2, 1, 1, 2, 1, 0), (True, False, True)
    spec = W.regular_decomposition(shape, parts, 3)
    with pytest.raises(ValueError, match="does not match"):
        O.make_staged_pattern((0, 0, 0), tuple(n - 1 for n in shape), halos, periodic,
                              [O.Domain(i, f, l) for i, f, l in spec], W.cartesian_lookup(parts))
    ctx = R.make_context(device=0)
    with pytest.raises(_capi.GhexError, match="staged pattern"):
        R.make_staged_pattern(ctx, [R.DomainDescriptor(i, (f, l)) for i, f, l in spec], W.cartesian_lookup(parts),
                              (0, 0, 0), tuple(n - 1 for n in shape), halos, periodic)


def test_lookup_results_are_checked():
    case = RC.staged_cases()["uneven_3d"]
    ctx = R.make_context(device=0)
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in case["domains"]]
    with pytest.raises(_capi.GhexError, match="unknown domain"):
        R.make_staged_pattern(ctx, doms, lambda i, off: 999, (0, 0, 0), (19, 15, 11), case["halos"], case["periodic"])


@pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_live():
    """GHEX's make_staged_pattern run from the reference sources on a float32 3-D case."""
    shape, parts, halos, periodic = (18, 14, 10), (2, 2, 3), (1, 2, 2, 1, 1, 1), (False, True, True)
    spec = W.regular_decomposition(shape, parts, 5)
    rng = np.random.default_rng(4)
    arrs = [np.asfortranarray(rng.standard_normal(
        tuple(l[k] - f[k] + 1 + halos[2 * k] + halos[2 * k + 1] for k in range(3))).astype(np.float32))
        for _, f, l in spec]
    offs = (halos[0], halos[2], halos[4])
    ref = [a.copy(order="F") for a in arrs]
    reflib.regular_staged_exchange(shape, halos, periodic, spec, W.cartesian_lookup(parts), ref, offs)
    doms = [O.Domain(i, f, l) for i, f, l in spec]
    st = O.make_staged_pattern((0, 0, 0), tuple(n - 1 for n in shape), halos, periodic, doms, W.cartesian_lookup(parts))
    O.exchange_staged(st, doms, arrs, [offs] * len(doms))
    assert all(np.array_equal(a, b) for a, b in zip(arrs, ref))
