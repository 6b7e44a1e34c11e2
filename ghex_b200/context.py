"""ghex.context (bindings/python/src/ghex/context.py): the context object and make_context."""
from ._core import context, make_context

__all__ = ["context", "make_context"]
