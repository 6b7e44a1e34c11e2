"""Objects shared by the structured and unstructured front ends.

Mirrors the object model of GHEX's Python bindings (bindings/python/src/ghex): a context, a
pattern container made by make_pattern, field descriptors bound to a pattern with
``pattern(field)`` (a buffer_info), a communication object whose ``exchange`` returns a handle
with ``wait()``. Everything below the Python objects is the C ABI of libghex_b200.so.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import threading
from typing import Any, Iterable, Sequence

from . import _capi
from ._capi import call


class Architecture(enum.Enum):
    """Where a field lives (bindings/python/src/ghex/util.py:22-24). Both are exchanged by the
    device kernels: GPU fields in device memory, CPU fields in host memory over the host
    interconnect."""

    CPU = "cpu"
    GPU = "gpu"


# --------------------------------------------------------------------------------------------
# device arrays
# --------------------------------------------------------------------------------------------
_TYPESTR = {"<f4": _capi.F32, "<f8": _capi.F64, "<i4": _capi.I32, "<i8": _capi.I64,
            "|u1": _capi.U8, "<u2": _capi.U16}


def _torch():
    try:
        import torch
        return torch
    except ImportError:  # pragma: no cover - torch is part of the environment
        return None


def check_arch(field: Any, arch) -> None:
    """arch=Architecture.CPU names a host field (host memory, read and written in place by the
    device kernels); arch=Architecture.GPU, or None as in GHEX's bindings, accepts either."""
    if arch == Architecture.CPU and array_info(field)["device"] != "host":
        raise TypeError("arch=Architecture.CPU needs a host array")


def array_info(field: Any) -> dict:
    """Pointer, shape, byte strides, dtype code and device of an array.

    Accepts torch tensors on a CUDA device and any object exposing ``__cuda_array_interface__``
    (device memory), and host memory: torch CPU tensors and objects exposing
    ``__array_interface__`` (numpy). Host fields are exchanged in place by the device kernels over
    the host interconnect once a field descriptor has page-locked their pages (``host_pages`` in
    the result); pinned allocations are recognised there page by page (a tensor's is_pinned()
    looks at its first byte only, which may sit on a page locked for a neighbouring array).
    """
    torch = _torch()
    if torch is not None and isinstance(field, torch.Tensor):
        if not field.is_cuda and field.device.type != "cpu":
            raise TypeError(f"unsupported tensor device {field.device}")
        codes = {torch.float32: _capi.F32, torch.float64: _capi.F64, torch.int32: _capi.I32,
                 torch.int64: _capi.I64, torch.uint8: _capi.U8, torch.uint16: _capi.U16}
        if field.dtype not in codes:
            raise TypeError(f"unsupported dtype {field.dtype}")
        es = field.element_size()
        return {"ptr": field.data_ptr(), "shape": tuple(field.shape),
                "strides": tuple(s * es for s in field.stride()), "dtype": codes[field.dtype],
                "itemsize": es, "device": (field.device.index or 0) if field.is_cuda else "host",
                "host_pages": not field.is_cuda}
    cai = getattr(field, "__cuda_array_interface__", None)
    if cai is None:
        hai = getattr(field, "__array_interface__", None)
        if hai is None:
            raise TypeError("expected a CUDA tensor, a host tensor or array, or an object with "
                            "__cuda_array_interface__ / __array_interface__")
        info = _interface_info(hai)
        info.update(device="host", host_pages=True)
        return info
    info = _interface_info(cai)
    info["device"] = None
    return info


def _interface_info(iface: dict) -> dict:
    typestr = iface["typestr"]
    if typestr not in _TYPESTR:
        raise TypeError(f"unsupported dtype {typestr}")
    shape = tuple(iface["shape"])
    itemsize = int(typestr[2:])
    strides = iface.get("strides")
    if strides is None:  # C-contiguous
        strides, s = [], itemsize
        for n in reversed(shape):
            strides.insert(0, s)
            s *= n
    return {"ptr": int(iface["data"][0]), "shape": shape, "strides": tuple(strides),
            "dtype": _TYPESTR[typestr], "itemsize": itemsize}


class _HostPages:
    """Page-locked ranges of ordinary host memory that fields live in, registered with
    ghexb_host_register page-aligned and reference-counted, so that fields sharing pages (views of
    one buffer, small arrays next to each other) share registrations and a range is unregistered
    when its last field is gone."""

    def __init__(self):
        self.lock = threading.Lock()
        self.regs: dict[int, list] = {}       # start -> [end, references, owned]
        self.page_of: dict[int, int] = {}     # page -> start of the registration holding it
        self.page = os.sysconf("SC_PAGE_SIZE")
        self._unregister = _capi.release      # held here: module globals may be gone at exit

    def acquire(self, lo: int, hi: int) -> list[int]:
        P = self.page
        p, end = lo // P * P, -(-hi // P) * P
        held: list[int] = []
        with self.lock:
            try:
                while p < end:
                    start = self.page_of.get(p)
                    if start is not None:
                        self.regs[start][1] += 1
                        held.append(start)
                        p = self.regs[start][0]
                        continue
                    q = p
                    while q < end and q not in self.page_of:
                        q += P
                    owned = C.c_int()
                    call("ghexb_host_register", C.c_void_p(p), q - p, C.byref(owned))
                    self.regs[p] = [q, 1, bool(owned.value)]
                    for page in range(p, q, P):
                        self.page_of[page] = p
                    held.append(p)
                    p = q
            except BaseException:
                self._release(held)
                raise
        return held

    def release(self, held: list[int]) -> None:
        with self.lock:
            self._release(held)

    def _release(self, held: list[int]) -> None:
        for start in held:
            reg = self.regs.get(start)
            if reg is None:
                continue
            reg[1] -= 1
            if reg[1] == 0:
                if reg[2]:
                    self._unregister("ghexb_host_unregister", C.c_void_p(start))
                for page in range(start, reg[0], self.page):
                    self.page_of.pop(page, None)
                del self.regs[start]


_host_pages = _HostPages()


class _HostRegistration:
    """The page-locked ranges one field's host memory is held by, released with the field."""

    def __init__(self, info: dict):
        lo = hi = info["ptr"]
        for n, st in zip(info["shape"], info["strides"]):
            if n == 0:
                self.held = []
                return
            lo += min(0, (n - 1) * st)
            hi += max(0, (n - 1) * st)
        # memory that is page-locked and mapped already (pinned allocations: torch pin_memory,
        # ghex_b200.host_empty, cudaHostAlloc) needs no registration of ours
        mapped = C.c_int()
        call("ghexb_host_is_mapped", C.c_void_p(lo), hi + info["itemsize"] - lo, C.byref(mapped))
        if mapped.value:
            self.held = []
            return
        self.held = _host_pages.acquire(lo, hi + info["itemsize"])

    def __del__(self, _pages=_host_pages):
        _pages.release(getattr(self, "held", []))
        self.held = []


def _layout_of(a: Any) -> tuple:
    i = array_info(a)
    return (i["shape"], i["strides"], i["dtype"], i["device"])


def stream_of(fields: Iterable[Any]):
    """The stream an exchange is ordered on: torch's current stream for torch tensors."""
    torch = _torch()
    for f in fields:
        if torch is not None and isinstance(f, torch.Tensor):
            dev = f.device if f.is_cuda else None  # pinned host tensors: the current device's stream
            return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    return C.c_void_p(0)


# --------------------------------------------------------------------------------------------
# context
# --------------------------------------------------------------------------------------------
class context:
    """Replaces ghex.context (bindings/python/src/ghex/context.py:20-21).

    One process owns every domain of an exchange, so there is no communicator: rank() is 0 and
    size() is 1. ``device`` selects the CUDA device the fields live on.
    """

    def __init__(self, comm: Any = None, thread_safe: bool = False, device: int | None = None):
        if device is None:
            torch = _torch()
            device = torch.cuda.current_device() if torch is not None and torch.cuda.is_available() else 0
        self.device = int(device)
        self.thread_safe = bool(thread_safe)
        h = C.c_void_p()
        call("ghexb_context_create", self.device, C.byref(h))
        self._h = h

    def rank(self) -> int:
        return 0

    def size(self) -> int:
        return 1

    def __del__(self, _release=_capi.release):
        _release("ghexb_context_destroy", getattr(self, "_h", None))
        self._h = None


def make_context(comm: Any = None, thread_safe: bool = False, device: int | None = None) -> context:
    """Replaces ghex.context.make_context(comm, thread_safe)."""
    return context(comm, thread_safe, device)


# --------------------------------------------------------------------------------------------
# patterns and buffer_info
# --------------------------------------------------------------------------------------------
class BufferInfo:
    """A field bound to a pattern (buffer_info.hpp:33-71). Holds references, owns nothing."""

    __slots__ = ("pattern", "field")

    def __init__(self, pattern: "PatternContainer", field: "FieldDescriptorBase"):
        self.pattern = pattern
        self.field = field

    def handle(self) -> C.c_void_p:
        return self.field._bind(self.pattern)

    def arrays(self) -> list:
        return [self.field.array]


class PatternContainer:
    """The result of make_pattern: one pattern per domain (pattern_container.hpp:32-101)."""

    grid_type = "structured"
    domain_id_type = "int"

    def __init__(self, ctx: context, handle: C.c_void_p, domain_ids: Sequence[Any]):
        self.context = ctx
        self._h = handle
        self._ids = list(domain_ids)

    def __call__(self, field: "FieldDescriptorBase") -> BufferInfo:
        if field.domain_key() not in self._ids:
            raise ValueError("field incompatible with available domains!")
        return BufferInfo(self, field)

    def __len__(self) -> int:
        return len(self._ids)

    def size(self) -> int:
        return len(self._ids)

    def max_tag(self) -> int:
        v = C.c_int()
        call("ghexb_pattern_max_tag", self._h, C.byref(v))
        return v.value

    def domain_index(self, key: Any) -> int:
        return self._ids.index(key)

    # -- introspection -------------------------------------------------------------------
    def num_spaces(self, domain_index: int, send: bool = False) -> int:
        n = C.c_int()
        call("ghexb_pattern_num_spaces", self._h, domain_index, int(send), C.byref(n))
        return n.value

    def spaces(self, domain_index: int, send: bool = False) -> list:
        """Iteration spaces as (neighbour index, local first, local last, global first, global last)."""
        out = []
        for k in range(self.num_spaces(domain_index, send)):
            nb = C.c_int()
            arrs = [(C.c_int * 4)() for _ in range(4)]
            call("ghexb_pattern_space", self._h, domain_index, int(send), k, C.byref(nb), *arrs)
            out.append((nb.value, *(tuple(a) for a in arrs)))
        return out

    def index_lists(self, domain_index: int, send: bool = False) -> list:
        """Unstructured entries as (neighbour index, local ids)."""
        out = []
        for k in range(self.num_spaces(domain_index, send)):
            nb, cnt = C.c_int(), C.c_int64()
            call("ghexb_pattern_space_indices", self._h, domain_index, int(send), k, C.byref(nb), None, 0,
                 C.byref(cnt))
            buf = (C.c_int64 * max(1, cnt.value))()
            call("ghexb_pattern_space_indices", self._h, domain_index, int(send), k, C.byref(nb), buf,
                 cnt.value, C.byref(cnt))
            out.append((nb.value, list(buf)[: cnt.value]))
        return out

    def __del__(self, _release=_capi.release):
        _release("ghexb_pattern_destroy", getattr(self, "_h", None))
        self._h = None


class FieldDescriptorBase:
    """A wrapped device array; bound lazily to every pattern it is used with."""

    def __init__(self, array: Any):
        self.array = array
        self._handles: dict[int, C.c_void_p] = {}
        info = array_info(array)
        if info.get("host_pages"):
            # ordinary host memory: page-locked and mapped for the device while this field lives
            self._host = _HostRegistration(info)

    def domain_key(self) -> Any:  # pragma: no cover - abstract
        raise NotImplementedError

    def _spec(self) -> dict:  # pragma: no cover - abstract
        """Everything but the address that wraps this field's memory (wrap_spec): picklable, so
        that another process can wrap the same memory once it has mapped it."""
        raise NotImplementedError

    def _wrap(self, pattern: PatternContainer) -> C.c_void_p:
        return wrap_spec(pattern, self._spec(), self.info["ptr"])

    def _bind(self, pattern: PatternContainer) -> C.c_void_p:
        key = id(pattern)
        h = self._handles.get(key)
        if h is None:
            h = self._wrap(pattern)
            self._handles[key] = h
            self._patterns = getattr(self, "_patterns", []) + [pattern]  # keep patterns alive
        return h

    def __del__(self, _release=_capi.release):
        for h in getattr(self, "_handles", {}).values():
            _release("ghexb_field_destroy", h)
        self._handles = {}


def wrap_spec(pattern: PatternContainer, spec: dict, ptr: int) -> C.c_void_p:
    """A field handle for the memory at `ptr` laid out as `spec` (FieldDescriptorBase._spec) and
    bound to `pattern`."""
    from ._capi import int_array, int64_array
    h = C.c_void_p()
    if spec["kind"] == "list":
        call("ghexb_field_wrap_unstructured", pattern._h, spec["domain"], spec["dtype"], C.c_void_p(ptr),
             spec["levels"], int(spec["levels_first"]), spec["outer_stride"], C.byref(h))
    else:
        dom = pattern.domain_index(spec["domain"]) if spec["by_index"] else spec["domain"]
        call("ghexb_field_wrap", pattern._h, dom, spec["dtype"], C.c_void_p(ptr), spec["ndim"],
             int_array(spec["offsets"]), int_array(spec["extents"]), int_array(spec["layout"]),
             int64_array(spec["strides"]), spec["ncomp"], int(spec["is_vector"]), C.byref(h))
    return h


def _flatten(args: tuple) -> list[BufferInfo]:
    if len(args) == 1 and isinstance(args[0], (list, tuple)):
        args = tuple(args[0])
    out = []
    for a in args:
        if isinstance(a, (list, tuple)):
            out.extend(a)
        else:
            out.append(a)
    for a in out:
        if not isinstance(a, BufferInfo):
            raise TypeError("exchange expects buffer_info objects made by pattern(field)")
    return out


# --------------------------------------------------------------------------------------------
# communication object
# --------------------------------------------------------------------------------------------
class Handle:
    """communication_handle (communication_object.hpp:67-105)."""

    def __init__(self, co: "CommunicationObject", h: C.c_void_p, keep: list):
        self._co = co
        self._h = h
        self._keep = keep

    def wait(self) -> None:
        call("ghexb_handle_wait", self._h)
        self._keep = []

    def is_ready(self) -> bool:
        r = C.c_int()
        call("ghexb_handle_is_ready", self._h, C.byref(r))
        if r.value:
            self._keep = []
        return bool(r.value)

    def progress(self) -> None:
        self.is_ready()

    def __del__(self, _release=_capi.release):
        _release("ghexb_handle_destroy", getattr(self, "_h", None))
        self._h = None


class CommunicationObject:
    """communication_object (communication_object.hpp:111-625).

    ``exchange`` accepts a list of buffer_info objects or buffer_infos as positional arguments
    (_pyghex/structured/regular/communication_object.cpp:60-78). The exchange is ordered on the
    current torch stream of the fields; ``wait()`` blocks the host until it has finished. Calling
    exchange again before wait() raises "earlier exchange operation was not finished".
    """

    def __init__(self, ctx: context, in_place_receive: bool = False):
        self.context = ctx
        h = C.c_void_p()
        call("ghexb_co_create_ipr" if in_place_receive else "ghexb_co_create", ctx._h, C.byref(h))
        self._h = h

    def exchange(self, *buffer_infos) -> Handle:
        bis = _flatten(buffer_infos)
        handles = (C.c_void_p * len(bis))(*[bi.handle() for bi in bis])
        arrays = [a for bi in bis for a in bi.arrays()]
        h = C.c_void_p()
        call("ghexb_co_exchange", self._h, handles, len(bis), stream_of(arrays), C.byref(h))
        return Handle(self, h, [bis, arrays])

    def __del__(self, _release=_capi.release):
        _release("ghexb_co_destroy", getattr(self, "_h", None))
        self._h = None


def make_communication_object(ctx: context) -> CommunicationObject:
    return CommunicationObject(ctx)


class BulkCommunicationObject:
    """bulk_communication_object<rma_range_generator, Pattern, Fields...>
    (bulk_communication_object.hpp:207-687): fields are registered ahead with add_field /
    add_fields, init() closes the registration, exchange() exchanges every registered field and
    returns a handle (wait / is_ready / progress).

    GHEX puts the halos of fields it can address directly (threads and processes of a node,
    rma_put.hpp:200-240) and sends the rest. Here every field lives in one process and the
    exchange kernel already copies each halo cell straight from its owner, so the registered
    fields are exchanged as one work table, built at the first exchange and replayed as one graph
    launch on the fields' stream."""

    def __init__(self, ctx: context):
        self.context = ctx
        self._co = CommunicationObject(ctx)
        self._bis: list[BufferInfo] = []
        self._initialized = False

    def add_field(self, buffer_info: BufferInfo) -> None:
        if self._initialized:
            raise RuntimeError("error: this CO has been initialized already")
        self._bis += _flatten((buffer_info,))

    def add_fields(self, *buffer_infos) -> None:
        for bi in _flatten(buffer_infos):
            self.add_field(bi)

    def init(self) -> None:
        if not self._bis:
            raise RuntimeError("a bulk communication object needs at least one field")
        self._initialized = True

    def exchange(self) -> Handle:
        if not self._initialized:
            self.init()
        return self._co.exchange(self._bis)


class GenericBulkCommunicationObject:
    """generic_bulk_communication_object (bulk_communication_object.hpp:120-171): a type-erased
    holder of a bulk communication object, exchanged through the same exchange()."""

    def __init__(self, bulk: BulkCommunicationObject):
        self._impl = bulk

    def exchange(self) -> Handle:
        return self._impl.exchange()


def make_bulk_communication_object(ctx: context) -> BulkCommunicationObject:
    return BulkCommunicationObject(ctx)


# --------------------------------------------------------------------------------------------
# explicit plans (no reference counterpart): batched / per-field / per-box forms, graph,
# adjoint, autotuning
# --------------------------------------------------------------------------------------------
class ExchangePlan:
    """The work-descriptor table of one set of buffer_infos, built once."""

    BATCHED = _capi.FORM_BATCHED
    PER_FIELD = _capi.FORM_PER_FIELD
    PER_BOX = _capi.FORM_PER_BOX

    def __init__(self, ctx: context, buffer_infos: Sequence[BufferInfo], in_place_receive: bool = False):
        self.context = ctx
        self._bis = _flatten(tuple(buffer_infos))
        self._arrays = [a for bi in self._bis for a in bi.arrays()]
        self._layout = [_layout_of(a) for a in self._arrays]
        self._bound = tuple(array_info(a)["ptr"] for a in self._arrays)
        handles = (C.c_void_p * len(self._bis))(*[bi.handle() for bi in self._bis])
        h = C.c_void_p()
        call("ghexb_plan_create_ipr" if in_place_receive else "ghexb_plan_create", ctx._h, handles,
             len(self._bis), C.byref(h))
        self._h = h

    def info(self) -> dict:
        i = _capi.PlanInfo()
        call("ghexb_plan_get_info", self._h, C.byref(i))
        return i.as_dict()

    def dram_floor(self, sector_bytes: int = 32) -> dict:
        """The least DRAM traffic of one exchange of this plan's fields from a cold cache."""
        return dram_floor(self.context, self._bis, sector_bytes)

    def set_tuning(self, elems_per_thread: int = 0, block: int = 0, use_pairs: int = -1) -> None:
        """Elements per thread (4, 8 or 16) and threads per CTA of the forward kernel (0 keeps), and
        whether x-face pairs move as contiguous segments (1), as separate boxes (0) or as before (-1)."""
        call("ghexb_plan_set_tuning", self._h, elems_per_thread, block, use_pairs)

    def set_staged(self, mode: int = -1, stages: int = 0, stage_bytes: int = 0, consumers: int = 0,
                   ctas_per_sm: int = 0) -> None:
        """Boxes of the batched form moved by the staged (tensor-map) kernel: mode 0 none, 1 short
        rows and transposed edges, 2 every box it can take; and its pipeline shape (0 keeps)."""
        call("ghexb_plan_set_staged", self._h, mode, stages, stage_bytes, consumers, ctas_per_sm)

    def set_bulk(self, share: int = 4) -> None:
        """Quarters (0 to 4) of the contiguous 16-byte-unit index lists moved by the bulk kernel
        (cp.async.bulk through shared memory) in the batched form."""
        call("ghexb_plan_set_bulk", self._h, share)

    def set_adjoint_bulk(self, share: int = 0) -> None:
        """Quarters (0 to 4) of the unstructured owners whose adjoint the bulk gather kernel
        (cp.async.bulk through shared memory) takes, beside the element gather kernel."""
        call("ghexb_plan_set_adjoint_bulk", self._h, share)

    def set_adjoint_tuning(self, gather_scale: int = 0) -> None:
        """Adjoint gather tiles of short rows sized by row length (0), halved (-1), doubled (1) or
        quadrupled (2)."""
        call("ghexb_plan_set_adjoint_tuning", self._h, gather_scale)

    def staged_status(self) -> int:
        """The staged kernel's status word since the last call (0: every wait ended in time)."""
        v = C.c_uint()
        call("ghexb_plan_staged_status", self._h, C.byref(v))
        return v.value

    def _stream(self, stream):
        if stream is None:
            return stream_of(self._arrays)
        if isinstance(stream, C.c_void_p):
            return stream
        if isinstance(stream, int):
            return C.c_void_p(stream)
        return C.c_void_p(getattr(stream, "cuda_stream", stream))

    def launch(self, form: int = _capi.FORM_BATCHED, stream=None) -> None:
        call("ghexb_plan_launch", self._h, form, self._stream(stream))

    def graph_launch(self, stream=None) -> None:
        call("ghexb_plan_graph_launch", self._h, self._stream(stream))

    def adjoint(self, stream=None) -> None:
        call("ghexb_plan_adjoint_launch", self._h, self._stream(stream))

    def bound_pointers(self) -> tuple:
        """Data pointers the plan's tables currently address, one per field."""
        return self._bound

    def rebind(self, arrays: Sequence[Any], stream=None, keep: bool = True) -> None:
        """Points the plan at new memory: arrays[i] takes the place of the i-th field's array and
        must have its shape, strides, dtype and device (checked here). Stream-ordered. With
        keep=False the plan holds no reference to the arrays: the caller keeps them alive while
        the plan's launches run and rebinds before launching on other memory."""
        if len(arrays) != len(self._layout):
            raise ValueError(f"rebind needs {len(self._layout)} arrays")
        ptrs = []
        for new, lay in zip(arrays, self._layout):
            if _layout_of(new) != lay:
                raise TypeError("rebind: array layout differs from the plan's field")
            ptrs.append(array_info(new)["ptr"])
        if stream is None:
            stream = stream_of(arrays)
        call("ghexb_plan_rebind", self._h, (C.c_void_p * len(ptrs))(*ptrs), len(ptrs), self._stream(stream))
        self._bound = tuple(ptrs)
        self._arrays = list(arrays) if keep else []

    def autotune(self, repeats: int = 10, stream=None) -> dict:
        i = _capi.PlanInfo()
        call("ghexb_plan_autotune", self._h, self._stream(stream), repeats, C.byref(i))
        return i.as_dict()

    def __del__(self, _release=_capi.release):
        _release("ghexb_plan_destroy", getattr(self, "_h", None))
        self._h = None


class _HostBlock:
    """Page-locked host memory from ghexb_host_alloc, freed with the last array that uses it."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        call("ghexb_host_alloc", max(1, int(nbytes)), C.byref(p))
        self.ptr, self.nbytes = p.value, int(nbytes)

    def __del__(self, _release=_capi.release):
        _release("ghexb_host_free", getattr(self, "ptr", None))


def host_empty(shape, dtype, order: str = "F"):
    """A numpy array in page-locked host memory mapped for the device (cudaHostAlloc, mapped and
    portable): a host field the exchange kernels read and write in place over the host
    interconnect. The memory lives as long as the array (or any view of it)."""
    import numpy as np
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) if len(shape) else 1
    block = _HostBlock(n * dt.itemsize)
    buf = (C.c_char * max(1, n * dt.itemsize)).from_address(block.ptr)
    buf._owner = block
    return np.frombuffer(buf, dtype=dt, count=n).reshape(shape, order=order)


def dram_floor(ctx: context, buffer_infos: Sequence[BufferInfo], sector_bytes: int = 32) -> dict:
    """The least DRAM traffic of one exchange of these fields from a cold cache, with
    `sector_bytes` as the DRAM access granularity: sectors holding halo sources are read, sectors
    holding halo elements are written back, sectors written in part without a source element are
    read first (host-only replay of every element's addresses; no device needed)."""
    bis = _flatten(tuple(buffer_infos))
    handles = [bi.handle() for bi in bis]
    arr = (C.c_void_p * len(handles))(*handles)
    r, w = C.c_int64(), C.c_int64()
    call("ghexb_plan_dram_floor", ctx._h, arr, len(handles), int(sector_bytes), C.byref(r), C.byref(w))
    return {"sector_bytes": int(sector_bytes), "read": r.value, "write": w.value, "total": r.value + w.value}


def make_exchange_plan(ctx: context, buffer_infos: Sequence[BufferInfo], in_place_receive: bool = False) -> ExchangePlan:
    return ExchangePlan(ctx, buffer_infos, in_place_receive)
