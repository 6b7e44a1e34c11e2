"""Cubed-sphere grids, mirroring GHEX's C++ cubed-sphere API
(structured/cubed_sphere/{domain_descriptor,halo_generator,field_descriptor}.hpp); GHEX's Python
bindings have no cubed-sphere module.

Fields are 4-D arrays indexed (x, y, z, component); the memory layout is taken from the array's
strides, the reference's default being x fastest and the component slowest
(layout_map<3,2,1,0>, field_descriptor.hpp:26).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Sequence, Union

from .._capi import call, int_array
from .._core import (Architecture, FieldDescriptorBase, PatternContainer, array_info, check_arch, context,
                     make_bulk_communication_object, make_communication_object, make_context, make_exchange_plan)
from .regular import _layout_order

__all__ = ["cube", "DomainDescriptor", "HaloGenerator", "make_pattern", "make_field_descriptor", "wrap_field",
           "make_communication_object", "make_bulk_communication_object", "make_context", "make_exchange_plan"]


@dataclass(frozen=True)
class cube:
    """cubed_sphere::cube (domain_descriptor.hpp:26-30)."""

    edge_size: int
    levels: int


class DomainDescriptor:
    """cubed_sphere::domain_descriptor(cube, tile, x_first, x_last, y_first, y_last)."""

    def __init__(self, c: cube, tile: int, x_first: int, x_last: int, y_first: int, y_last: int):
        self.cube = c
        self.tile = int(tile)
        self.x = (int(x_first), int(x_last))
        self.y = (int(y_first), int(y_last))

    def domain_id(self) -> tuple[int, tuple[int, int]]:
        return (self.tile, (self.x[0], self.y[0]))

    def edge_size(self) -> int:
        return self.cube.edge_size

    def first(self) -> tuple[int, int, int, int]:
        return (self.tile, self.x[0], self.y[0], 0)

    def last(self) -> tuple[int, int, int, int]:
        return (self.tile, self.x[1], self.y[1], self.cube.levels - 1)


class HaloGenerator:
    """cubed_sphere::halo_generator(halo) or (halos) with halos in the order of its m_halo array:
    -x, +x, -y, +y (halo_generator.hpp:59-71, used at :113-142)."""

    def __init__(self, halo: Union[int, Sequence[int]]):
        self.halos = (int(halo),) * 4 if isinstance(halo, int) else tuple(int(h) for h in halo)
        if len(self.halos) != 4:
            raise ValueError("a cubed-sphere halo has 4 widths")


class Pattern(PatternContainer):
    grid_type = "structured::cubed_sphere"
    domain_id_type = "cubed_sphere::domain_id_type"

    def __init__(self, ctx: context, handle, domains: Sequence[DomainDescriptor]):
        super().__init__(ctx, handle, [d.domain_id() for d in domains])
        self.domains = list(domains)


def make_pattern(context: context, halo_gen: HaloGenerator, domain_range: Sequence[DomainDescriptor]) -> Pattern:
    domains = list(domain_range)
    if not domains:
        raise ValueError("make_pattern needs at least one domain")
    c = domains[0].cube
    if any(d.cube != c for d in domains):
        raise ValueError("all domains must lie on the same cube")
    h = C.c_void_p()
    call("ghexb_pattern_create_cubed_sphere", context._h, c.edge_size, c.levels, int_array(halo_gen.halos),
         len(domains), int_array([d.tile for d in domains]), int_array([d.x[0] for d in domains]),
         int_array([d.x[1] for d in domains]), int_array([d.y[0] for d in domains]),
         int_array([d.y[1] for d in domains]), C.byref(h))
    return Pattern(context, h, domains)


class FieldDescriptor(FieldDescriptorBase):
    """cubed_sphere::field_descriptor(dom, data, offsets, extents, num_components, is_vector)
    (field_descriptor.hpp:113-121). offsets/extents are given for (x, y, z)."""

    def __init__(self, domain: DomainDescriptor, field: Any, offsets: Sequence[int], extents: Sequence[int],
                 num_components: int = 1, is_vector: bool = False):
        super().__init__(field)
        info = array_info(field)
        if len(info["shape"]) != 4:
            raise TypeError("cubed-sphere fields are 4-dimensional (x, y, z, component)")
        self.domain = domain
        self.info = info
        self.offsets = tuple(int(v) for v in offsets)[:3] + (0,)
        self.extents = tuple(int(v) for v in extents)[:3] + (int(num_components),)
        self.num_components = int(num_components)
        self.is_vector = bool(is_vector)
        self.layout = _layout_order(info["strides"])

    def domain_key(self):
        return self.domain.domain_id()

    def domain_id(self):
        return self.domain.domain_id()

    def _spec(self) -> dict:
        return {"kind": "box", "domain": self.domain_key(), "by_index": True, "dtype": self.info["dtype"], "ndim": 4,
                "offsets": tuple(self.offsets), "extents": tuple(self.extents), "layout": tuple(self.layout),
                "strides": tuple(self.info["strides"]), "ncomp": self.num_components, "is_vector": bool(self.is_vector)}


def make_field_descriptor(domain: DomainDescriptor, field: Any, offsets: Sequence[int], extents: Sequence[int],
                          num_components: int = 1, is_vector: bool = False, *,
                          arch: Architecture = Architecture.GPU) -> FieldDescriptor:
    check_arch(field, arch)
    return FieldDescriptor(domain, field, offsets, extents, num_components, is_vector)


def wrap_field(*args, **kwargs) -> FieldDescriptor:
    return make_field_descriptor(*args, **kwargs)
