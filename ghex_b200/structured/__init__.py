"""Structured grids: regular (drop-in for ghex.structured.regular) and cubed sphere."""
from . import regular  # noqa: F401
from . import cubed_sphere  # noqa: F401
