"""Host logic of the in-place receive communication objects, without a GPU: one object per
domain posts its exchange; the exchange of the pattern launches only once every domain with a
halo has posted, a wait() before that reports the missing domains, and a second exchange()
before the launch is refused. Fields sit at fake device addresses that are never dereferenced
(nothing is launched here)."""
import pytest

import golden_cases as G
from ghex_b200 import unstructured as U
from ghex_b200.structured import regular as R


class FakeDeviceArray:
    def __init__(self, shape, address):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (address, False),
                                         "version": 3, "strides": None}


def _setup():
    doms, _ = G.ipr_case()
    ctx = U.make_context(device=0)
    ud = [U.DomainDescriptor(d, doms[d]["gids"], doms[d]["halo_lids"]) for d in sorted(doms)]
    pat = U.make_pattern(ctx, U.HaloGenerator(), ud)
    bis = [pat(U.make_field_descriptor(d, FakeDeviceArray((d.size(), 2), (1 << 40) + (i << 20))))
           for i, d in enumerate(ud)]
    return ctx, pat, bis


def test_wait_reports_domains_that_did_not_post():
    ctx, pat, bis = _setup()
    cos = [U.make_communication_object_ipr(ctx, bi) for bi in bis[:3]]
    hs = [co.exchange() for co in cos]
    assert not any(h.is_ready() for h in hs)
    with pytest.raises(RuntimeError, match=r"domain\(s\) \[3\] have not posted"):
        hs[0].wait(timeout=0.2)
    with pytest.raises(RuntimeError, match="earlier exchange operation was not finished"):
        cos[1].exchange()


def test_arguments_are_checked():
    ctx, pat, bis = _setup()
    with pytest.raises(ValueError, match="one field per domain"):
        U.make_communication_object_ipr(ctx, [bis[0], bis[0]])
    rctx = R.make_context(device=0)
    hg = R.HaloGenerator(((0, 0, 0), (7, 7, 7)), [1, 1, 1], [True] * 3)
    rpat = R.make_pattern(rctx, hg, [R.DomainDescriptor(0, ((0, 0, 0), (7, 7, 7)))])
    rbi = rpat(R.make_field_descriptor(rpat.domains[0], FakeDeviceArray((10, 10, 10), 1 << 40), (1, 1, 1),
                                       (10, 10, 10)))
    with pytest.raises(TypeError, match="unstructured pattern"):
        U.make_communication_object_ipr(rctx, rbi)
    with pytest.raises(TypeError, match="unstructured pattern"):
        U.make_communication_object_ipr(ctx, [bis[0], rbi])


def test_objects_of_one_pattern_share_one_group():
    ctx, pat, bis = _setup()
    a = U.make_communication_object_ipr(ctx, bis[0])
    b = U.make_communication_object_ipr(ctx, bis[1:3])
    assert a._group is b._group
    assert a._group.required == {0, 1, 2, 3}
