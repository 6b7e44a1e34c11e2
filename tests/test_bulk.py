"""bulk_communication_object (bulk_communication_object.hpp): fields registered ahead, exchanged
repeatedly; the bulk parts of test_simple_regular_domain.cpp (the full pattern, and the staged
pattern with one bulk object per stage) on the device, and the registration rules on the CPU."""
import numpy as np
import pytest
import torch

import golden_cases as G
import regular_cases as RC
from ghex_b200 import GenericBulkCommunicationObject
from ghex_b200.structured import regular as R
from gpu_helpers import bits_equal, to_device


class FakeDeviceArray:
    def __init__(self, shape, address):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (address, False),
                                         "version": 3, "strides": None}


def test_registration_closes_at_init():
    ctx = R.make_context(device=0)
    hg = R.HaloGenerator(((0, 0, 0), (7, 7, 7)), [1, 1, 1], [True] * 3)
    pat = R.make_pattern(ctx, hg, [R.DomainDescriptor(0, ((0, 0, 0), (7, 7, 7)))])
    bi = pat(R.make_field_descriptor(pat.domains[0], FakeDeviceArray((10, 10, 10), 1 << 40), (1, 1, 1), (10, 10, 10)))
    bco = R.make_bulk_communication_object(ctx)
    with pytest.raises(RuntimeError, match="at least one field"):
        bco.init()
    bco.add_fields(bi)
    bco.init()
    with pytest.raises(RuntimeError, match="initialized already"):
        bco.add_field(bi)


def _fields(case, cuda):
    gold = G.staged_arrays()
    name = "simple_2d_2x2"
    n = len(case["domains"])
    return [to_device(RC.pairs_view(gold[f"{name}_in_{i}"]), cuda) for i in range(n)], \
           [RC.pairs_view(gold[f"{name}_out_{i}"]) for i in range(n)]


@pytest.mark.gpu
def test_simple_2d_bulk_full_and_staged(cuda):
    case = RC.staged_cases()["simple_2d_2x2"]
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in case["domains"]]
    ctx = R.make_context()
    gl = tuple(n - 1 for n in case["shape"])
    ext = lambda t: tuple(t.shape[:2])
    # full pattern, one bulk object for every domain's field
    tens, expected = _fields(case, cuda)
    hg = R.HaloGenerator(((0, 0), gl), [(RC.HALO, RC.HALO)] * 2, (True, True))
    pat = R.make_pattern(ctx, hg, doms)
    bco = R.make_bulk_communication_object(ctx)
    for d, t in zip(doms, tens):
        bco.add_field(pat(R.make_field_descriptor(d, t, case["offsets"], ext(t))))
    bco.init()
    gbco = GenericBulkCommunicationObject(bco)
    for _ in range(2):
        gbco.exchange().wait()
        assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
    for (_, f, l), t in zip(case["domains"], tens):
        assert RC.simple_2d_check(t.cpu().numpy(), f, l, (True, True), case["dims"]) == []
    # staged pattern, one bulk object per stage, exchanged in turn
    tens, expected = _fields(case, cuda)
    stages = R.make_staged_pattern(ctx, doms, case["lookup"], (0, 0), gl, case["halos"], case["periodic"])
    fds = [R.make_field_descriptor(d, t, case["offsets"], ext(t)) for d, t in zip(doms, tens)]
    bulks = []
    for sp in stages:
        b = R.make_bulk_communication_object(ctx)
        b.add_fields([sp(f) for f in fds])
        b.init()
        bulks.append(GenericBulkCommunicationObject(b))
    for b in bulks:
        h = b.exchange()
        h.wait()
        assert h.is_ready()
    assert sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected)) == 0
