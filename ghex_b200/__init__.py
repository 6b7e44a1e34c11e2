"""ghex_b200: B200-native halo exchange for many sub-domains resident on one GPU.

A drop-in for the GPU path of GHEX's make_pattern / make_communication_object /
co.exchange(pattern(field)...).wait(): every halo element moves from the owner's interior to the
neighbour's halo with one read and one write, in a single kernel that walks a work-descriptor
table built once per field set (libghex_b200.so, C ABI in include/ghex_b200.h).

Modules:
    ghex_b200.context                  drop-in for ghex.context (make_context)
    ghex_b200.util                     drop-in for ghex.util (Architecture)
    ghex_b200.structured.regular       drop-in for ghex.structured.regular
    ghex_b200.structured.cubed_sphere  the cubed-sphere grids of GHEX's C++ API
    ghex_b200.unstructured             drop-in for ghex.unstructured
    ghex_b200.autograd                 differentiable exchange (torch.autograd.Function)

The shared library is loaded on first use of the API (not by `python -m ghex_b200.build`).
"""
__version__ = "0.1.0"

_CORE_NAMES = ("Architecture", "make_context", "make_communication_object", "make_exchange_plan",
               "make_bulk_communication_object", "BulkCommunicationObject", "GenericBulkCommunicationObject",
               "host_empty", "dram_floor")


def __getattr__(name):
    if name in _CORE_NAMES:
        from . import _core
        return getattr(_core, name)
    raise AttributeError(name)
