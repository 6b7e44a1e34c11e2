"""Unstructured grids: the drop-in for ghex.unstructured (bindings/python/src/ghex/unstructured.py).

    dom = DomainDescriptor(id, gids_in_storage_order, outer_local_ids)
    pattern = make_pattern(ctx, HaloGenerator(), [dom, ...])
    f = make_field_descriptor(dom, tensor)            # tensor of shape (n,) or (n, levels)
    co.exchange([pattern(f), ...]).wait()

The halo generator may be one generator for every domain or a list with one per domain.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Optional, Sequence, Union

from ._capi import call, int64_array
from ._core import (Architecture, FieldDescriptorBase, PatternContainer, array_info, context,
                    make_communication_object, make_context, make_exchange_plan)

__all__ = ["DomainDescriptor", "HaloGenerator", "make_pattern", "make_field_descriptor", "wrap_field",
           "make_communication_object", "make_context", "make_exchange_plan"]


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


def make_pattern(context: context, halo_gen: Union[HaloGenerator, Sequence[HaloGenerator]],
                 domain_range: Sequence[DomainDescriptor]) -> Pattern:
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
    call("ghexb_pattern_create_unstructured", context._h, len(domains), int64_array([d.domain_id() for d in domains]),
         int64_array(gid_off), int64_array(gids), int64_array(outer_off), int64_array(outer), halo_off_arr, halo_arr,
         C.byref(h))
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

    def _wrap(self, pattern: PatternContainer):
        h = C.c_void_p()
        call("ghexb_field_wrap_unstructured", pattern._h, self.domain_desc.domain_id(), self.info["dtype"],
             C.c_void_p(self.info["ptr"]), self.levels, int(self.levels_first), self.outer_stride, C.byref(h))
        return h


def make_field_descriptor(domain_desc: DomainDescriptor, field: Any, *,
                          arch: Optional[Architecture] = Architecture.GPU) -> FieldDescriptor:
    if arch == Architecture.CPU:
        raise TypeError("ghex_b200 exchanges device memory only (arch=Architecture.GPU)")
    return FieldDescriptor(domain_desc, field)


def wrap_field(*args, **kwargs) -> FieldDescriptor:
    return make_field_descriptor(*args, **kwargs)
