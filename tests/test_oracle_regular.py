"""The oracle's regular exchange reproduces the known answers of the reference's tests (CPU)."""
import numpy as np
import pytest

from ghex_b200 import workloads as W
from oracle import regular as O
from regular_cases import DIM, HALO, owner_check, simple_2d_check, simple_2d_domains, simple_2d_fields


@pytest.mark.parametrize("periodic", [(True, True), (True, False), (False, True), (False, False)])
def test_simple_2d_known_answer(periodic):
    doms = simple_2d_domains()
    fields = simple_2d_fields(doms)
    pat = O.make_pattern((0, 0), (2 * DIM - 1, 4 * (DIM // 2) - 1), (HALO,) * 4, periodic,
                         [O.Domain(i, f, l) for i, f, l in doms])
    O.exchange(pat, [O.Domain(i, f, l) for i, f, l in doms], fields, [(HALO, HALO)] * len(doms))
    for (i, f, l), a in zip(doms, fields):
        assert simple_2d_check(a, f, l, periodic) == [], f"domain {i}"


def test_simple_2d_check_detects_errors():
    """Plant a wrong halo value in the oracle's output: the ported check must flag it."""
    doms = simple_2d_domains()
    fields = simple_2d_fields(doms)
    pat = O.make_pattern((0, 0), (15, 15), (HALO,) * 4, (True, True), [O.Domain(i, f, l) for i, f, l in doms])
    O.exchange(pat, [O.Domain(i, f, l) for i, f, l in doms], fields, [(HALO, HALO)] * len(doms))
    fields[3][0, 0] = (99, 99)
    assert len(simple_2d_check(fields[3], doms[3][1], doms[3][2], (True, True))) == 1


def run_oracle(w):
    out = {}
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for spec in specs:
            arrays = [w.domain_array(d, spec) for d in w.domains]
            O.exchange(pat, doms, arrays, [w.offsets(spec)] * len(doms))
            out[spec.name] = arrays
    return out


def test_cfg0_owner_values():
    w = W.config0()
    res = run_oracle(w)
    spec = w.fields[0]
    assert owner_check(w, res[spec.name], spec) == 0
    # 8 x (34^3 - 32^3) halo cells, all owned (periodic in x, y, z)
    assert sum(int(np.isnan(a).sum()) for a in res[spec.name]) == 0


def test_cfg1_small_owner_values():
    w = W.config1(shape=(40, 30, 12))
    res = run_oracle(w)
    for spec in w.fields:
        assert owner_check(w, res[spec.name], spec) == 0, spec.name
    # non-periodic x and z: boundary halos stay NaN
    a = res["f64_0"][0]
    assert np.isnan(a[0, 5, 0])


def test_owner_check_detects_errors():
    w = W.config0()
    res = run_oracle(w)
    spec = w.fields[0]
    res[spec.name][2][0, 4, 4] = 0.125
    assert owner_check(w, res[spec.name], spec) == 1


def test_adjoint_is_transpose():
    """<E x, y> == <x, E^T y> for the linear map 'x -> exchanged x' on random inputs."""
    w = W.config1(shape=(20, 15, 9))
    halos, specs = next(iter(w.halo_groups().items()))
    doms = [O.Domain(i, f, l) for i, f, l in w.domains]
    pat = O.make_pattern((0,) * 3, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
    rng = np.random.default_rng(0)
    ext = [w.extents(d, specs[0]) for d in w.domains]
    x = [rng.standard_normal(e) for e in ext]
    y = [rng.standard_normal(e) for e in ext]
    Ex = [a.copy() for a in x]
    O.exchange(pat, doms, Ex, [w.offsets(specs[0])] * len(doms))
    ETy = [a.copy() for a in y]
    O.adjoint(pat, doms, ETy, [w.offsets(specs[0])] * len(doms))
    lhs = sum(float((a * b).sum()) for a, b in zip(Ex, y))
    rhs = sum(float((a * b).sum()) for a, b in zip(x, ETy))
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs))


@pytest.mark.parametrize("ranks", [1, 2, 4])
def test_mixed_3d_known_answers(ranks):
    """test_regular_domain.cpp: three fields of array<double|float|int, 3> cells, two patterns with
    different halos, every cell of the grown domains holding its wrapped global coordinate."""
    import regular_cases as RC
    doms, g_last = RC.mixed_3d_domains(ranks)
    odoms = [O.Domain(i, f, l) for i, f, l in doms]
    for dtype, halos in ((np.float64, RC.MIXED_HALOS_1), (np.float32, RC.MIXED_HALOS_2), (np.int32, RC.MIXED_HALOS_1)):
        pat = O.make_pattern((0, 0, 0), g_last, halos, (True, True, True), odoms)
        arrs = [RC.mixed_3d_field(d, dtype) for d in doms]
        O.exchange(pat, odoms, arrs, [RC.MIXED_OFFSET] * len(doms))
        assert sum(RC.mixed_3d_check(a, d, halos, ranks, g_last) for a, d in zip(arrs, doms)) == 0
