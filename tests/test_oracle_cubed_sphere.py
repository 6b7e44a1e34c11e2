"""Cubed sphere on the CPU: the oracle restatement and the C++ host patterns against GHEX's own
code and the known answers of its cubed-sphere test."""
import numpy as np
import pytest

from cs_cases import EDGE, HALO, LEVELS, MEM_HALO, N, NCOMP, domains, fields
from oracle import cubed_sphere as O
from oracle import reflib

needs_ref = pytest.mark.skipif(not reflib.available(), reason="oracle/_ref (the reference build) is not built")


def oracle_run(is_vector):
    doms = [O.Domain(t, (x0, x1), (y0, y1), LEVELS) for t, x0, x1, y0, y1 in domains()]
    pat = O.make_pattern(EDGE, (HALO,) * 4, doms)
    arrs = fields()
    O.exchange(pat, doms, arrs, [(MEM_HALO, MEM_HALO, 0)] * len(doms), EDGE, is_vector)
    return arrs


def ref_run(is_vector):
    arrs = fields()
    reflib.cubed_exchange(EDGE, LEVELS, (HALO,) * 4, domains(), [(NCOMP, is_vector, (MEM_HALO, MEM_HALO, 0), arrs)])
    return arrs


@needs_ref
@pytest.mark.parametrize("is_vector", [False, True])
def test_reference_code_passes_its_own_checks(is_vector):
    """The reference's exchange, run here, satisfies the reference test's expectations: pins the
    transport stand-ins and the check harness."""
    for (t, x0, _, y0, _), a in zip(domains(), ref_run(is_vector)):
        assert reflib.cs_check_field(a, t, x0, y0, MEM_HALO, N, LEVELS, NCOMP, is_vector, HALO) == 0


@needs_ref
@pytest.mark.parametrize("is_vector", [False, True])
def test_oracle_passes_reference_checks_and_matches_reference(is_vector):
    got = oracle_run(is_vector)
    ref = ref_run(is_vector)
    for (t, x0, _, y0, _), a, r in zip(domains(), got, ref):
        assert reflib.cs_check_field(a, t, x0, y0, MEM_HALO, N, LEVELS, NCOMP, is_vector, HALO) == 0
        assert np.array_equal(a.view(np.uint32), r.view(np.uint32))


@needs_ref
def test_reference_checks_detect_errors():
    """A wrong value planted in the oracle's output fails the reference checks."""
    got = oracle_run(True)
    t, x0, _, y0, _ = domains()[5]
    got[5][MEM_HALO - 1, MEM_HALO + 2, 1, 1] += 1  # one left-halo cell
    assert reflib.cs_check_field(got[5], t, x0, y0, MEM_HALO, N, LEVELS, NCOMP, True, HALO) == 1


def test_cube_corners_stay_empty():
    """Cube-corner diagonal halo regions intersect no tile and keep their initial value."""
    got = oracle_run(False)
    a = got[0]  # tile 0, domain (0, 0): its bottom-left corner is a cube corner
    assert np.all(a[MEM_HALO - HALO:MEM_HALO, MEM_HALO - HALO:MEM_HALO] == -1)


def test_cpp_pattern_matches_oracle():
    from ghex_b200.structured import cubed_sphere as C
    ctx = C.make_context(device=0)
    cube = C.cube(EDGE, LEVELS)
    doms = [C.DomainDescriptor(cube, t, x0, x1, y0, y1) for t, x0, x1, y0, y1 in domains()]
    p = C.make_pattern(ctx, C.HaloGenerator(HALO), doms)
    odoms = [O.Domain(t, (x0, x1), (y0, y1), LEVELS) for t, x0, x1, y0, y1 in domains()]
    opat = O.make_pattern(EDGE, (HALO,) * 4, odoms)
    for i, entries in enumerate(opat):
        exp = [(en.neighbor, s.lfirst, s.llast, s.gfirst, s.glast) for en in entries for s in en.spaces]
        assert p.spaces(i) == exp, f"domain {i}"
    assert p.max_tag() == sum(len(e) for e in opat) - 1


@pytest.mark.parametrize("halos", [(3, 3, 3, 3), (1, 2, 0, 3), (2, 0, 2, 1)])
@pytest.mark.parametrize("split", [1, 2, 3])
def test_cpp_pattern_matches_oracle_other_shapes(halos, split):
    from ghex_b200.structured import cubed_sphere as C
    edge, levels = 12, 3
    step = edge // split
    boxes = [(t, i * step, (i + 1) * step - 1, j * step, (j + 1) * step - 1)
             for t in range(6) for j in range(split) for i in range(split)]
    ctx = C.make_context(device=0)
    cube = C.cube(edge, levels)
    p = C.make_pattern(ctx, C.HaloGenerator(halos), [C.DomainDescriptor(cube, *b) for b in boxes])
    opat = O.make_pattern(edge, halos, [O.Domain(t, (x0, x1), (y0, y1), levels) for t, x0, x1, y0, y1 in boxes])
    for i, entries in enumerate(opat):
        exp = [(en.neighbor, s.lfirst, s.llast, s.gfirst, s.glast) for en in entries for s in en.spaces]
        assert p.spaces(i) == exp, f"domain {i}"


def test_transform_tables_round_trip():
    """Every tile transform composed with its inverse is the identity on tile coordinates, as the
    reference's test_cubed_sphere_transform.cpp checks."""
    c = 7
    for t in range(6):
        for n in range(4):
            fw, inv = O.forward(t, n), O.inverse(t, n)
            for x in range(-3, c + 3):
                for y in range(-3, c + 3):
                    X, Y = O.apply(fw, x, y, c)
                    assert O.apply(inv, X, Y, c) == (x, y)
