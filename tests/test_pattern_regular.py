"""Regular patterns built by the C++ host side equal the oracle's restatement of GHEX's
make_pattern (no GPU needed)."""
import numpy as np
import pytest

from ghex_b200 import workloads as W
from ghex_b200.structured import regular as R
from oracle import regular as O


def product_pattern(ctx, shape, halos, periodic, doms):
    dim = len(shape)
    hg = R.HaloGenerator(((0,) * dim, tuple(n - 1 for n in shape)),
                         [(halos[2 * k], halos[2 * k + 1]) for k in range(dim)], periodic)
    return R.make_pattern(ctx, hg, [R.DomainDescriptor(i, (f, l)) for i, f, l in doms])


def oracle_pattern(shape, halos, periodic, doms):
    dim = len(shape)
    return O.make_pattern((0,) * dim, tuple(n - 1 for n in shape), halos, periodic,
                          [O.Domain(i, f, l) for i, f, l in doms])


def flatten(opat, dim):
    out = []
    for entries in opat:
        lst = []
        for en in entries:
            for s in en.spaces:
                pad = lambda t: tuple(t) + (0,) * (4 - dim)
                lst.append((en.neighbor, pad(s.lfirst), pad(s.llast), pad(s.gfirst), pad(s.glast)))
        out.append(lst)
    return out


CASES = [
    ("cfg0", (64, 64, 64), (1, 1, 1, 1, 1, 1), (True, True, True), W.regular_decomposition((64, 64, 64), (2, 2, 2))),
    ("cfg1-f64", (400, 300, 96), (3, 3, 3, 3, 0, 0), (False, True, False), W.config1().domains),
    ("cfg1-f32", (400, 300, 96), (2, 2, 2, 2, 1, 1), (False, True, False), W.config1().domains),
    ("2d-simple", (16, 16), (3, 3, 3, 3), (True, True), W.regular_decomposition((16, 16), (2, 4))),
    ("2d-nonperiodic", (16, 16), (3, 3, 3, 3), (False, False), W.regular_decomposition((16, 16), (2, 4))),
    ("1d-halo-wider-than-domain", (10,), (3, 2), (True,), W.regular_decomposition((10,), (5,))),
    ("3d-asym", (20, 12, 9), (2, 0, 1, 3, 0, 2), (True, False, True), W.regular_decomposition((20, 12, 9), (3, 2, 1), seed=3)),
    ("3d-single-domain-periodic", (8, 8, 8), (1, 2, 1, 2, 1, 2), (True, True, True), [(0, (0, 0, 0), (7, 7, 7))]),
]


@pytest.mark.parametrize("name,shape,halos,periodic,doms", CASES, ids=[c[0] for c in CASES])
def test_recv_spaces_match_oracle(name, shape, halos, periodic, doms):
    ctx = R.make_context(device=0)
    p = product_pattern(ctx, shape, halos, periodic, doms)
    op = oracle_pattern(shape, halos, periodic, doms)
    expect = flatten(op, len(shape))
    for i in range(len(doms)):
        assert p.spaces(i) == expect[i], f"domain {i}"
    n_entries = sum(len(e) for e in op)
    assert p.max_tag() == max(0, n_entries - 1)


@pytest.mark.parametrize("name,shape,halos,periodic,doms", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_send_spaces_mirror_recv(name, shape, halos, periodic, doms):
    """Every receive space appears once as a send space of its source, in the source's frame."""
    ctx = R.make_context(device=0)
    p = product_pattern(ctx, shape, halos, periodic, doms)
    dim = len(shape)
    firsts = [d[1] for d in doms]
    recv = sorted((i, nb, s[2], s[3]) for i in range(len(doms)) for (nb, *s) in
                  [(sp[0], sp[1], sp[2], sp[3], sp[4]) for sp in p.spaces(i)])
    send = []
    for j in range(len(doms)):
        for nb, lf, ll, gf, gl in p.spaces(j, send=True):
            for k in range(dim):
                assert lf[k] == gf[k] - firsts[j][k] and ll[k] == gl[k] - firsts[j][k]
            send.append((nb, j, gf, gl))
    assert sorted(send) == sorted((i, nb, gf, gl) for (i, nb, gf, gl) in recv)


def test_halo_generator_python_matches_oracle():
    dom = R.DomainDescriptor(0, ((0, 10, 4), (9, 19, 7)))
    hg = R.HaloGenerator(((0, 0, 0), (29, 19, 7)), ((2, 1), 3, (0, 1)), (True, False, True))
    got = hg(dom)
    exp = O.halo_boxes(O.Domain(0, (0, 10, 4), (9, 19, 7)), (0, 0, 0), (29, 19, 7), (2, 1, 3, 3, 0, 1),
                       (True, False, True))
    assert got == [(s.lfirst, s.llast, s.gfirst, s.glast) for s in exp]
    # C++ '%' semantics in the periodic wrap
    assert O._cmod(-7, 5) == -2 and R._cmod(-7, 5) == -2
