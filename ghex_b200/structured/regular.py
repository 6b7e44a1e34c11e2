"""Regular structured grids: the drop-in for ghex.structured.regular
(bindings/python/src/ghex/structured/regular.py).

    ctx = make_context()
    halo_gen = HaloGenerator(global_indices, halos=((3, 3), (3, 3), (0, 0)), periodicity=(False, True, False))
    pattern = make_pattern(ctx, halo_gen, [DomainDescriptor(i, sub_indices) for ...])
    fields = [make_field_descriptor(dom, tensor, offsets, extents) for ...]
    co = make_communication_object(ctx)
    co.exchange([pattern(f) for f in fields]).wait()

Index sets may be given as anything with ``.dim`` and corner indexing (``s[(0,)*dim]`` is the
first and ``s[(-1,)*dim]`` the last point, as the reference's cartesian_sets.ProductSet) or as
a pair ``(first, last)`` of inclusive coordinate tuples.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Sequence, Union

from .. import _capi
from .._capi import call, int_array, int64_array
from .._core import (Architecture, BufferInfo, CommunicationObject, ExchangePlan, FieldDescriptorBase,
                     PatternContainer, array_info, check_arch, context, make_bulk_communication_object, make_communication_object, make_context,
                     make_exchange_plan)

__all__ = ["Architecture", "DomainDescriptor", "HaloGenerator", "make_pattern", "make_staged_pattern",
           "make_field_descriptor",
           "wrap_field", "make_communication_object", "make_bulk_communication_object", "make_context", "make_exchange_plan", "ExchangePlan",
           "CommunicationObject", "BufferInfo"]


def _corners(indices: Any) -> tuple[tuple[int, ...], tuple[int, ...]]:
    if isinstance(indices, (tuple, list)) and len(indices) == 2 and isinstance(indices[0], (tuple, list)):
        first, last = tuple(int(v) for v in indices[0]), tuple(int(v) for v in indices[1])
    else:
        dim = int(indices.dim)
        first = tuple(int(v) for v in indices[tuple(0 for _ in range(dim))])
        last = tuple(int(v) for v in indices[tuple(-1 for _ in range(dim))])
    if len(first) != len(last):
        raise ValueError("first and last coordinates differ in dimension")
    return first, last


class DomainDescriptor:
    """structured::regular::domain_descriptor(id, first, last) (domain_descriptor.hpp:248-254)."""

    def __init__(self, id_: int, sub_domain_indices: Any) -> None:
        self._id = int(id_)
        self._first, self._last = _corners(sub_domain_indices)

    def domain_id(self) -> int:
        return self._id

    def first(self) -> tuple[int, ...]:
        return self._first

    def last(self) -> tuple[int, ...]:
        return self._last

    @property
    def dim(self) -> int:
        return len(self._first)


class HaloGenerator:
    """structured::regular::halo_generator(g_first, g_last, halos, periodic)
    (halo_generator.hpp:68-78). ``halos`` per dimension is an int or a (minus, plus) pair."""

    def __init__(self, glob_domain_indices: Any, halos: Sequence[Union[int, tuple[int, int]]],
                 periodicity: Sequence[bool]) -> None:
        self.first, self.last = _corners(glob_domain_indices)
        dim = len(self.first)
        if len(halos) != dim or len(periodicity) != dim:
            raise ValueError("halos and periodicity need one entry per dimension")
        pairs = [(h, h) if isinstance(h, int) else tuple(h) for h in halos]
        self.halos = tuple(int(v) for p in pairs for v in p)
        self.periodicity = tuple(bool(p) for p in periodicity)

    @property
    def dim(self) -> int:
        return len(self.first)

    def __call__(self, domain: DomainDescriptor) -> list[tuple[tuple, tuple, tuple, tuple]]:
        """Receive halo boxes of one domain as (local first, local last, global first, global last),
        periodic wrap applied (halo_generator.hpp:91-146)."""
        dim = self.dim
        iv = []
        for k in range(dim):
            f, l = domain.first()[k], domain.last()[k]
            ext = l - f
            hm, hp = self.halos[2 * k], self.halos[2 * k + 1]
            iv.append([(-hm, -1, f - hm, f - 1), (0, ext, f, l), (ext + 1, ext + hp, l + 1, l + hp)])
        boxes = []
        import itertools
        for j, combo in enumerate(itertools.product(range(3), repeat=dim)):
            if j == (3 ** dim) // 2:
                continue
            b = [iv[k][combo[k]] for k in range(dim)]
            if any(t[1] < t[0] for t in b):
                continue
            lf, ll = tuple(t[0] for t in b), tuple(t[1] for t in b)
            gf, gl = [t[2] for t in b], [t[3] for t in b]
            for k in range(dim):
                if not self.periodicity[k]:
                    continue
                ext_h = gl[k] - gf[k]
                ext = self.last[k] + 1 - self.first[k]
                off = gf[k] - self.first[k]
                gf[k] = int(_cmod(off + ext, ext)) + self.first[k]
                gl[k] = gf[k] + ext_h
            boxes.append((lf, ll, tuple(gf), tuple(gl)))
        return boxes


def _cmod(a: int, b: int) -> int:
    """C++ '%' (truncating) for ints."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


class Pattern(PatternContainer):
    grid_type = "structured::regular"
    domain_id_type = "int"

    def __init__(self, ctx: context, handle, domains: Sequence[DomainDescriptor], halo_gen: HaloGenerator):
        super().__init__(ctx, handle, [d.domain_id() for d in domains])
        self.domains = list(domains)
        self.halo_generator = halo_gen
        self.dim = halo_gen.dim


def make_pattern(context: context, halo_gen: HaloGenerator, domain_range: Sequence[DomainDescriptor]) -> Pattern:
    """ghex::make_pattern<structured::grid>(ctx, halo_gen, domains) (pattern_container.hpp:112-120)."""
    domains = list(domain_range)
    if not domains:
        raise ValueError("make_pattern needs at least one domain")
    dim = halo_gen.dim
    for d in domains:
        if d.dim != dim:
            raise ValueError("domain and halo generator differ in dimension")
    h = C.c_void_p()
    call("ghexb_pattern_create_regular", context._h, dim, int_array(halo_gen.first), int_array(halo_gen.last),
         int_array(halo_gen.halos), int_array([int(p) for p in halo_gen.periodicity]), len(domains),
         int64_array([d.domain_id() for d in domains]), int_array([v for d in domains for v in d.first()]),
         int_array([v for d in domains for v in d.last()]), C.byref(h))
    return Pattern(context, h, domains, halo_gen)


def _lookup_id(found: Any) -> int:
    """The domain id in what a domain lookup returned: an int, or an object with an ``id``
    attribute or method (as the reference's neighbor type, which also carries a rank)."""
    if isinstance(found, int):
        return found
    v = getattr(found, "id", None)
    if v is None:
        raise TypeError("a domain lookup must return a domain id or an object with id()")
    return int(v() if callable(v) else v)


def make_staged_pattern(context: context, domain_range: Sequence[DomainDescriptor], domain_lookup,
                        g_first: Sequence[int], g_last: Sequence[int], halos: Sequence,
                        periodic: Sequence[bool]) -> list:
    """structured::regular::make_staged_pattern(ctx, domains, domain_lookup, g_first, g_last,
    halos, periodic) (structured/regular/make_pattern.hpp:47-256): one pattern container per
    dimension; exchanging them one after the other (waiting in between) fills the halos, edges and
    corners included, through the faces. ``domain_lookup(id, offset)`` returns the neighbour of
    domain ``id`` at ``offset`` (a tuple with one entry of -1 or +1) as an id or an object with
    ``id()``; it is called only where the domain has a halo on that side. ``halos`` is the
    reference's flat array (dim0-, dim0+, dim1-, ...) or one (minus, plus) pair per dimension."""
    domains = list(domain_range)
    if not domains:
        raise ValueError("make_staged_pattern needs at least one domain")
    dim = len(g_first)
    flat = [v for h in halos for v in ((h, h) if isinstance(h, int) else h)] if len(halos) == dim else list(halos)
    if len(flat) != 2 * dim or len(periodic) != dim or len(g_last) != dim:
        raise ValueError("halos, periodicity and global corners need one entry per dimension")
    for d in domains:
        if d.dim != dim:
            raise ValueError("domain and global corners differ in dimension")
    nbr = []
    for d in domains:
        for i in range(dim):
            for side, step in ((0, -1), (1, 1)):
                h = flat[2 * i + side]
                edge = d.first()[i] - h >= g_first[i] if step < 0 else d.last()[i] + h <= g_last[i]
                if h > 0 and (periodic[i] or edge):
                    off = [0] * dim
                    off[i] = step
                    nbr.append(_lookup_id(domain_lookup(d.domain_id(), tuple(off))))
                else:
                    nbr.append(-1)
    out = (C.c_void_p * dim)()
    call("ghexb_pattern_create_regular_staged", context._h, dim, int_array(g_first), int_array(g_last),
         int_array(flat), int_array([int(bool(p)) for p in periodic]), len(domains),
         int64_array([d.domain_id() for d in domains]), int_array([v for d in domains for v in d.first()]),
         int_array([v for d in domains for v in d.last()]), int64_array(nbr), out)
    gen = HaloGenerator((tuple(g_first), tuple(g_last)), [(flat[2 * k], flat[2 * k + 1]) for k in range(dim)],
                        periodic)
    return [Pattern(context, C.c_void_p(out[i]), domains, gen) for i in range(dim)]


def _layout_order(strides: Sequence[int]) -> tuple[int, ...]:
    """Layout map from byte strides: the largest stride gets 0, ties broken upwards
    (bindings/python/src/ghex/structured/regular.py:40-62)."""
    ordered = list(reversed(sorted(strides)))
    layout = [ordered.index(s) for s in strides]
    for i, v in enumerate(layout):
        if v in layout[:i]:
            layout[i] = max(layout) + 1
    return tuple(layout)


class FieldDescriptor(FieldDescriptorBase):
    """structured::regular::field_descriptor made by wrap_field<GPU, Layout>(dom, data, offsets,
    extents, strides) (field_descriptor.hpp:187-194); the layout map comes from the array's
    strides as in the reference's Python binding."""

    def __init__(self, domain_desc: DomainDescriptor, field: Any, offsets: Sequence[int], extents: Sequence[int],
                 num_components: int = 1):
        super().__init__(field)
        info = array_info(field)
        ndim = len(info["shape"])
        dim = domain_desc.dim
        if ndim not in (dim, dim + 1):
            raise TypeError("field dimension must equal the domain dimension (+1 for components)")
        if ndim == dim + 1 and num_components == 1:
            num_components = info["shape"][-1]
        self.domain_desc = domain_desc
        self.info = info
        self.offsets = tuple(int(v) for v in offsets) + ((0,) if ndim == dim + 1 and len(offsets) == dim else ())
        self.extents = tuple(int(v) for v in extents) + ((num_components,) if ndim == dim + 1 and len(extents) == dim else ())
        if len(self.offsets) != ndim or len(self.extents) != ndim:
            raise ValueError("offsets and extents need one entry per dimension")
        self.layout = _layout_order(info["strides"])
        self.num_components = int(num_components)
        self.ndim = ndim

    def domain_key(self) -> int:
        return self.domain_desc.domain_id()

    def domain_id(self) -> int:
        return self.domain_desc.domain_id()

    def _spec(self) -> dict:
        return {"kind": "box", "domain": self.domain_desc.domain_id(), "by_index": False, "dtype": self.info["dtype"],
                "ndim": self.ndim, "offsets": tuple(self.offsets), "extents": tuple(self.extents),
                "layout": tuple(self.layout), "strides": tuple(self.info["strides"]), "ncomp": self.num_components,
                "is_vector": False}


def make_field_descriptor(domain_desc: DomainDescriptor, field: Any, offsets: Sequence[int],
                          extents: Sequence[int], *, arch: Architecture = Architecture.GPU,
                          num_components: int = 1) -> FieldDescriptor:
    """(bindings/python/src/ghex/structured/regular.py:65-97). Only GPU arrays are accepted."""
    check_arch(field, arch)
    return FieldDescriptor(domain_desc, field, offsets, extents, num_components)


def wrap_field(*args, **kwargs) -> FieldDescriptor:
    return make_field_descriptor(*args, **kwargs)
