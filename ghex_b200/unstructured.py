"""Unstructured grids: the drop-in for ghex.unstructured (bindings/python/src/ghex/unstructured.py).

    dom = DomainDescriptor(id, gids_in_storage_order, outer_local_ids)
    pattern = make_pattern(ctx, HaloGenerator(), [dom, ...])
    f = make_field_descriptor(dom, tensor)            # tensor of shape (n,) or (n, levels)
    co.exchange([pattern(f), ...]).wait()

The halo generator may be one generator for every domain or a list with one per domain.

In-place receive (unstructured/communication_object_ipr.hpp): one communication object per
domain's field, ``co = make_communication_object_ipr(ctx, pattern(f)); co.exchange().wait()``.
"""
from __future__ import annotations

import ctypes as C
import threading
import weakref
from typing import Any, Optional, Sequence, Union

from ._capi import call, int64_array
from ._core import (Architecture, BufferInfo, CommunicationObject, FieldDescriptorBase, PatternContainer, check_arch,
                    _flatten, array_info, context, make_bulk_communication_object, make_communication_object, make_context,
                    make_exchange_plan)

__all__ = ["DomainDescriptor", "HaloGenerator", "make_pattern", "make_field_descriptor", "wrap_field",
           "make_communication_object", "make_bulk_communication_object", "make_communication_object_ipr", "make_context", "make_exchange_plan"]


class DomainDescriptor:
    """unstructured::domain_descriptor(id, gids, outer_lids) (user_concepts.hpp:145-174):
    ``indices`` are the global ids in storage order, ``halo_indices`` the local ids of the outer
    (halo) elements."""

    def __init__(self, index: int, indices: Sequence[int], halo_indices: Sequence[int]):
        import numpy as np
        self._id = int(index)
        self.gids = np.asarray(indices, dtype=np.int64).ravel()
        self.outer_lids = np.asarray(halo_indices, dtype=np.int64).ravel()
        if np.unique(self.outer_lids).size != self.outer_lids.size:
            raise ValueError("repeated outer (local) index")
        if self.outer_lids.size and (self.outer_lids.min() < 0 or self.outer_lids.max() >= self.gids.size):
            raise ValueError("outer local index out of range")
        inner = np.ones(self.gids.size, dtype=bool)
        inner[self.outer_lids] = False
        if np.unique(self.gids[inner]).size != int(inner.sum()):
            raise ValueError("repeated inner (global) index")
        self._inner = int(inner.sum())

    def domain_id(self) -> int:
        return self._id

    def size(self) -> int:
        return int(self.gids.size)

    def inner_size(self) -> int:
        return self._inner


class HaloGenerator:
    """unstructured::halo_generator (user_concepts.hpp:180-256): all outer gids of a domain, or
    the gids of an explicit list that are outer in the domain, in list order."""

    def __init__(self, gids: Optional[Sequence[int]] = None):
        self.gids = None if gids is None else [int(g) for g in gids]

    @classmethod
    def from_gids(cls, gids: Sequence[int]) -> "HaloGenerator":
        return cls(gids)


class Pattern(PatternContainer):
    grid_type = "unstructured"
    domain_id_type = "int"

    def __init__(self, ctx: context, handle, domains: Sequence[DomainDescriptor]):
        super().__init__(ctx, handle, [d.domain_id() for d in domains])
        self.domains = list(domains)


def _hints_of(found) -> tuple:
    """(owner ids, remote indices) from what a receive domain ids generator returned: an object
    with domain_ids() and remote_indices() (attributes or methods, as the reference's halo type),
    or a tuple (domain_ids, remote_indices[, ranks])."""
    if isinstance(found, (tuple, list)):
        return list(found[0]), list(found[1])
    get = lambda name: (lambda v: v() if callable(v) else v)(getattr(found, name))
    return list(get("domain_ids")), list(get("remote_indices"))


def make_pattern(context: context, halo_gen: Union[HaloGenerator, Sequence[HaloGenerator]], *args) -> Pattern:
    """make_pattern<unstructured::grid>(ctx, halo_gen, domains), or with a receive domain ids
    generator make_pattern(ctx, halo_gen, recv_domain_ids_gen, domains) (pattern_container.hpp:
    112-146): ``recv_domain_ids_gen(domain)`` returns, for each halo element in the halo
    generator's order, its owner domain id and its local index in the owner."""
    if len(args) == 1:
        rdig, domain_range = None, args[0]
    elif len(args) == 2:
        rdig, domain_range = args
    else:
        raise TypeError("make_pattern(ctx, halo_gen, [recv_domain_ids_gen,] domains)")
    domains = list(domain_range)
    if not domains:
        raise ValueError("make_pattern needs at least one domain")
    gens = list(halo_gen) if isinstance(halo_gen, (list, tuple)) else [halo_gen] * len(domains)
    if len(gens) != len(domains):
        raise ValueError("one halo generator per domain is needed")
    import numpy as np
    gid_off = np.cumsum([0] + [d.gids.size for d in domains])
    outer_off = np.cumsum([0] + [d.outer_lids.size for d in domains])
    gids = np.concatenate([d.gids for d in domains])
    outer = np.concatenate([d.outer_lids for d in domains])
    halo_off_arr = halo_arr = None
    if any(g.gids is not None for g in gens):
        halo_lists = [d.gids[np.sort(d.outer_lids)] if g.gids is None else np.asarray(g.gids, dtype=np.int64)
                      for d, g in zip(domains, gens)]
        halo_off_arr = int64_array(np.cumsum([0] + [h.size for h in halo_lists]))
        halo_arr = int64_array(np.concatenate(halo_lists) if halo_lists else np.zeros(0, dtype=np.int64))
    h = C.c_void_p()
    common = (context._h, len(domains), int64_array([d.domain_id() for d in domains]), int64_array(gid_off),
              int64_array(gids), int64_array(outer_off), int64_array(outer), halo_off_arr, halo_arr)
    if rdig is None:
        call("ghexb_pattern_create_unstructured", *common, C.byref(h))
    else:
        hints = [_hints_of(rdig(d)) for d in domains]
        for ids_, rem in hints:
            if len(ids_) != len(rem):
                raise ValueError("the receive domain ids generator gives domain ids and remote indices of different lengths")
        hoff = np.cumsum([0] + [len(a) for a, _ in hints])
        call("ghexb_pattern_create_unstructured_hinted", *common, int64_array(hoff),
             int64_array([v for a, _ in hints for v in a]), int64_array([v for _, b in hints for v in b]), C.byref(h))
    return Pattern(context, h, domains)


class FieldDescriptor(FieldDescriptorBase):
    """unstructured::data_descriptor<gpu>(dom, field, levels, levels_first, outer_stride)
    (user_concepts.hpp:524-535); levels and their order follow the array's shape and strides as
    in the reference's binding (_pyghex/unstructured/field_descriptor.cpp:141-180)."""

    def __init__(self, domain_desc: DomainDescriptor, field: Any):
        super().__init__(field)
        info = array_info(field)
        shape, strides, es = info["shape"], info["strides"], info["itemsize"]
        if len(shape) > 2:
            raise TypeError("field has too many dimensions")
        if shape[0] != domain_desc.size():
            raise TypeError("field's first dimension must match the size of the domain")
        levels_first, outer = True, 0
        if len(shape) == 2 and strides[1] != es:
            levels_first = False
            if strides[0] != es or strides[1] % es:
                raise TypeError("field's strides are not compatible with GHEX")
            outer = strides[1] // es
        elif len(shape) == 2:
            if strides[0] % es:
                raise TypeError("field's strides are not compatible with GHEX")
            outer = strides[0] // es
        elif strides[0] != es:
            raise TypeError("field's strides are not compatible with GHEX")
        self.domain_desc = domain_desc
        self.info = info
        self.levels = 1 if len(shape) == 1 else int(shape[1])
        self.levels_first = levels_first
        self.outer_stride = int(outer)

    def domain_key(self) -> int:
        return self.domain_desc.domain_id()

    def domain_id(self) -> int:
        return self.domain_desc.domain_id()

    def _spec(self) -> dict:
        return {"kind": "list", "domain": self.domain_desc.domain_id(), "dtype": self.info["dtype"],
                "levels": self.levels, "levels_first": bool(self.levels_first), "outer_stride": self.outer_stride}


def make_field_descriptor(domain_desc: DomainDescriptor, field: Any, *,
                          arch: Optional[Architecture] = Architecture.GPU) -> FieldDescriptor:
    check_arch(field, arch)
    return FieldDescriptor(domain_desc, field)


def wrap_field(*args, **kwargs) -> FieldDescriptor:
    return make_field_descriptor(*args, **kwargs)


# --------------------------------------------------------------------------------------------
# in-place receive
# --------------------------------------------------------------------------------------------
#: seconds a wait() of an in-place receive exchange waits for the other domains to post theirs
IPR_WAIT_TIMEOUT = 30.0

_groups_lock = threading.Lock()


class _InPlaceRound:
    __slots__ = ("handle", "error", "lock")

    def __init__(self):
        self.handle = None
        self.error: Optional[BaseException] = None
        self.lock = threading.Lock()


class _InPlaceGroup:
    """The in-place receive communication objects of one pattern container. Every domain lives
    in this process, so the messages between the domains are the copies of one exchange: it is
    launched when every domain with a halo or a send has posted its exchange()."""

    def __init__(self, ctx: context, pattern: "Pattern"):
        self.cond = threading.Condition()
        self.co = CommunicationObject(ctx, in_place_receive=True)
        self.required = {pattern._ids[i] for i in range(len(pattern))
                         if pattern.num_spaces(i) or pattern.num_spaces(i, True)}
        self.posted: dict = {}
        self.round = _InPlaceRound()

    @staticmethod
    def of(ctx: context, pattern: "Pattern") -> "_InPlaceGroup":
        """The group of `pattern` in `ctx`, made on first use and dropped with the pattern."""
        with _groups_lock:
            groups = ctx.__dict__.setdefault("_in_place_groups", weakref.WeakKeyDictionary())
            group = groups.get(pattern)
            if group is None:
                group = _InPlaceGroup(ctx, pattern)
                groups[pattern] = group
            return group

    def post(self, bis: list) -> _InPlaceRound:
        with self.cond:
            ids = [bi.field.domain_id() for bi in bis]
            if any(i in self.posted for i in ids):
                raise RuntimeError("earlier exchange operation was not finished")
            for i, bi in zip(ids, bis):
                self.posted[i] = bi
            rnd = self.round
            if self.required <= set(self.posted):
                fields = [self.posted[i] for i in sorted(self.posted)]
                self.posted = {}
                self.round = _InPlaceRound()
                try:
                    rnd.handle = self.co.exchange(fields)
                except BaseException as e:
                    rnd.error = e
                    raise
                finally:
                    self.cond.notify_all()
            return rnd

    def missing(self) -> list:
        return sorted(self.required - set(self.posted))

    def wait(self, rnd: _InPlaceRound, timeout: Optional[float]) -> None:
        with self.cond:
            done = self.cond.wait_for(lambda: rnd.handle is not None or rnd.error is not None,
                                      IPR_WAIT_TIMEOUT if timeout is None else timeout)
            if not done:
                raise RuntimeError(
                    f"in-place receive: domain(s) {self.missing()} have not posted their exchange; every "
                    "domain lives in this process, so each one's exchange() must be called before a wait() "
                    "can complete")
        if rnd.error is not None:
            raise RuntimeError(f"in-place receive exchange failed: {rnd.error}") from rnd.error
        with rnd.lock:
            rnd.handle.wait()


class InPlaceHandle:
    """communication_object_ipr::handle (communication_object_ipr.hpp:65-99)."""

    def __init__(self, group: _InPlaceGroup, rnd: _InPlaceRound):
        self._group, self._round = group, rnd

    def wait(self, timeout: Optional[float] = None) -> None:
        self._group.wait(self._round, timeout)

    def is_ready(self) -> bool:
        r = self._round
        if r.error is not None:
            return True
        if r.handle is None:
            return False
        with r.lock:
            return r.handle.is_ready()

    def progress(self) -> None:
        self.is_ready()


class CommunicationObjectIPR:
    """unstructured::communication_object_ipr (communication_object_ipr.hpp:30-186): the exchange
    of one field whose halo, per neighbour, is stored on consecutive rows, so that GHEX receives
    each message straight into it. The k-th value of a neighbour's message lands on row
    first + k, first being the first local index of that neighbour's receive list (:127-141).

    One process holds every domain here: the exchange of all domains of the pattern runs as one
    stream-ordered kernel, launched once every domain with a halo has called exchange(); wait()
    returns when it has completed (and raises if a domain never posts its exchange). Fields whose
    received rows are not halo rows received once, or whose levels are not contiguous rows, raise
    when the exchange is launched. ``buffer_info`` may also be a list of buffer_infos of distinct
    domains of one pattern."""

    def __init__(self, ctx: context, buffer_info):
        bis = _flatten((buffer_info,))
        if not bis:
            raise ValueError("an in-place receive needs a buffer_info")
        pattern = bis[0].pattern
        if not isinstance(pattern, Pattern) or any(bi.pattern is not pattern for bi in bis):
            raise TypeError("an in-place receive needs buffer_infos of one unstructured pattern")
        ids = [bi.field.domain_id() for bi in bis]
        if len(set(ids)) != len(ids):
            raise ValueError("one field per domain")
        self.context = ctx
        self._bis = bis
        self._group = _InPlaceGroup.of(ctx, pattern)

    def exchange(self) -> InPlaceHandle:
        return InPlaceHandle(self._group, self._group.post(self._bis))


def make_communication_object_ipr(ctx: context, buffer_info) -> CommunicationObjectIPR:
    """make_communication_object_ipr(ctx, buffer_info) (communication_object_ipr.hpp:188-196)."""
    return CommunicationObjectIPR(ctx, buffer_info)
