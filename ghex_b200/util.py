"""ghex.util (bindings/python/src/ghex/util.py:22-24): where a field lives."""
from ._core import Architecture

__all__ = ["Architecture"]
