"""Sharded exchange across processes, one per GPU.

GHEX exchanges between ranks by packing send buffers, posting them through oomph and unpacking
what arrives (communication_object.hpp:433-512, packer.hpp:32-59). Here every process maps the
field memory of the other processes' domains into its own address space (CUDA IPC) and one
exchange kernel per process moves its part of the halos directly between the GPUs' memories:

* pull (the default): a process fills its own halos, reading the peers' interiors;
* push: a process writes its interior values into the peers' halos; the adjoint of this form
  gathers, for every local owner element, all its images wherever they lie.

No descriptor is in two processes' plans and together they hold every descriptor of the exchange,
so the result is the single-process exchange's, bit for bit. An exchange is ordered by a barrier
on each side: every process's fields are final before any kernel starts, and none changes its
fields before every kernel is done. With an NCCL process group the barriers are all-reduces on the
exchange's stream (stream-ordered, the host does not wait); otherwise the host synchronises the
device and meets the others at a gloo barrier.

The API mirrors GHEX's for domains spread over ranks: ``make_context(group)``
(context.hpp:20-35), ``make_pattern(ctx, halo_gen, local_domains)`` (pattern_container.hpp:112-146,
whose set-up gathers every rank's domains: structured/pattern.hpp:214-568),
``make_communication_object(ctx)`` and ``co.exchange(...).wait()``.
"""
from __future__ import annotations

import ctypes as C
import importlib
from typing import Any, Sequence

from . import _capi
from . import _core
from ._capi import call

PULL = 1
PUSH = 2
_MODES = {"pull": PULL, "push": PUSH, PULL: PULL, PUSH: PUSH}


def _dist():
    import torch.distributed as dist
    return dist


def _torch_stream(stream: C.c_void_p, device: int):
    """The torch stream of a raw CUDA stream handle (the device's default stream for a null one)."""
    import torch
    dev = torch.device("cuda", device)
    if not stream.value:
        return torch.cuda.default_stream(dev)
    return torch.cuda.ExternalStream(stream.value, device=dev)


class context(_core.context):
    """ghex::context(MPI_Comm) over a torch.distributed process group (the default group when
    ``group`` is None). Host collectives run on a gloo group (the group itself when it is gloo, else
    a gloo group over the same ranks, made collectively here)."""

    def __init__(self, group: Any = None, device: int | None = None):
        # every process of the default group makes its context at the same point: with an NCCL
        # group the gloo group of the host collectives is made here, collectively
        super().__init__(None, False, device)
        dist = _dist()
        if not dist.is_initialized():
            raise RuntimeError("a distributed context needs torch.distributed to be initialised")
        self.group = group
        self._rank = dist.get_rank(group)
        self._size = dist.get_world_size(group)
        backend = dist.get_backend(group)
        self.device_barriers = backend == "nccl"
        if backend == "gloo":
            self.host_group = group
        else:
            ranks = dist.get_process_group_ranks(group) if group is not None else list(range(dist.get_world_size()))
            self.host_group = dist.new_group(ranks, backend="gloo")
        self._patterns: dict[int, _core.PatternContainer] = {}

    def rank(self) -> int:
        return self._rank

    def size(self) -> int:
        return self._size

    def all_gather(self, obj: Any) -> list:
        out = [None] * self._size
        _dist().all_gather_object(out, obj, group=self.host_group)
        return out

    def host_barrier(self) -> None:
        _dist().barrier(group=self.host_group)

    def agree(self, error: BaseException | None) -> None:
        """Collective: raises on every process when any process passes an error, so that a
        failure on one process never leaves the others waiting in a later collective."""
        errors = self.all_gather(None if error is None else f"{type(error).__name__}: {error}")
        bad = [(r, e) for r, e in enumerate(errors) if e is not None]
        if bad:
            if error is not None:
                raise error
            r, e = bad[0]
            raise RuntimeError(f"rank {r} failed: {e}")


def make_context(group: Any = None, device: int | None = None) -> context:
    return context(group, device)


class Pattern:
    """The pattern of every process's domains (the same on every process, domains in id order);
    binds this process's fields."""

    def __init__(self, ctx: context, pattern: _core.PatternContainer, owner: dict, seq: int):
        self.context = ctx
        self.pattern = pattern
        self.owner = owner  # domain key -> rank
        self.seq = seq
        pattern._shard_seq = seq
        ctx._patterns[seq] = pattern

    def __call__(self, field: _core.FieldDescriptorBase) -> _core.BufferInfo:
        key = field.domain_key()
        r = self.owner.get(key)
        if r != self.context.rank():
            where = "no process" if r is None else f"rank {r}"
            raise ValueError(f"field incompatible with available domains! (domain {key!r} belongs to {where})")
        return self.pattern(field)

    def local_domains(self) -> list:
        return [k for k, r in self.owner.items() if r == self.context.rank()]

    def __len__(self) -> int:
        return len(self.owner)


def make_pattern(ctx: context, halo_gen: Any, *args) -> Pattern:
    """make_pattern(ctx, halo_gen, [recv_domain_ids_gen,] local_domains), collective: every process
    passes its own domains (and, for unstructured grids, a halo generator per domain or one for
    all); the grid kind follows the domain descriptors' module."""
    if not args:
        raise TypeError("make_pattern(ctx, halo_gen, [recv_domain_ids_gen,] local_domains)")
    local, extra = list(args[-1]), args[:-1]
    parts = ctx.all_gather(local)
    domains = [d for part in parts for d in part]
    if not domains:
        raise ValueError("make_pattern needs at least one domain")
    # domains in the order of their ids, whichever rank holds them: the order of descriptors, and
    # so of the adjoint's additions into an owner, is then that of a single process given the
    # domains in id order
    order = sorted(range(len(domains)), key=lambda k: domains[k].domain_id())
    if isinstance(halo_gen, (list, tuple)):
        if len(halo_gen) != len(local):
            raise ValueError("one halo generator per local domain is needed")
        gens = [h for part in ctx.all_gather(list(halo_gen)) for h in part]
        halo_gen = [gens[k] for k in order]
    domains = [domains[k] for k in order]
    module = importlib.import_module(type(domains[0]).__module__)
    pattern = module.make_pattern(ctx, halo_gen, *extra, domains)
    owner = {}
    for r, part in enumerate(parts):
        for d in part:
            key = d.domain_id()
            if key in owner:
                raise ValueError(f"domain {key!r} is given by ranks {owner[key]} and {r}")
            owner[key] = r
    seq = len(ctx._patterns)
    return Pattern(ctx, pattern, owner, seq)


def ipc_export(ptr: int) -> tuple[bytes, int]:
    """(handle, offset) of the device allocation holding `ptr`."""
    h = C.create_string_buffer(_capi.IPC_HANDLE_BYTES)
    off = C.c_int64()
    call("ghexb_ipc_export", C.c_void_p(ptr), h, C.byref(off))
    return h.raw, off.value


def ipc_open(handle: bytes, offset: int) -> int:
    p = C.c_void_p()
    call("ghexb_ipc_open", handle, offset, C.byref(p))
    return p.value


def ipc_close(handle: bytes) -> None:
    call("ghexb_ipc_close", handle)


def _local_meta(ctx: context, bis: list, share: bool) -> list:
    meta = []
    for bi in bis:
        seq = getattr(bi.pattern, "_shard_seq", None)
        if seq is None or ctx._patterns.get(seq) is not bi.pattern:
            raise ValueError("a sharded exchange needs fields bound to patterns of distributed.make_pattern")
        ptr = bi.field.info["ptr"]
        meta.append({"pattern": seq, "spec": bi.field._spec(), "ptr": ptr, "ipc": ipc_export(ptr) if share else None})
    return meta


class _FieldSet:
    """Every process's fields of one exchange as field handles of this process: its own, and the
    others' wrapped around their memory mapped here (or around their bare addresses, for host-only
    checks that dereference nothing)."""

    def __init__(self, ctx: context, bis: list, share: bool):
        self.context = ctx
        self._remote: list[C.c_void_p] = []
        self._opened: list[bytes] = []
        meta, err = None, None
        try:
            meta = _local_meta(ctx, bis, share)
        except Exception as e:  # reported to every process below
            err = e
        everyone = ctx.all_gather(meta)
        ctx.agree(err)
        handles, local = [], []
        try:
            for r, part in enumerate(everyone):
                if r == ctx.rank():
                    handles += [bi.handle() for bi in bis]
                    local += [1] * len(bis)
                    continue
                for m in part:
                    ptr = m["ptr"]
                    if share:
                        handle, off = m["ipc"]
                        ptr = ipc_open(handle, off)
                        self._opened.append(handle)
                    h = _core.wrap_spec(ctx._patterns[m["pattern"]], m["spec"], ptr)
                    self._remote.append(h)
                    handles.append(h)
                    local.append(0)
        except Exception as e:
            err = e
        if err is not None:
            self.release()
        ctx.agree(err)
        self.n = len(handles)
        self.handles = (C.c_void_p * self.n)(*handles)
        self.local = bytes(local)

    def release(self, _release=_capi.release) -> None:
        for h in self._remote:
            _release("ghexb_field_destroy", h)
        self._remote = []
        for handle in self._opened:
            try:
                ipc_close(handle)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
        self._opened = []

    def __del__(self):
        self.release()


def check_sharded(ctx: context, buffer_infos: Sequence[_core.BufferInfo], mode: Any = "pull") -> int:
    """Host-only replay of this process's part of a sharded exchange (ghexb_plan_check_sharded),
    collective: the elements it moves, every address inside its field. Needs no device."""
    bis = _core._flatten(tuple(buffer_infos))
    fs = _FieldSet(ctx, bis, share=False)
    n = C.c_int64()
    try:
        call("ghexb_plan_check_sharded", ctx._h, fs.handles, fs.n, fs.local, _MODES[mode], C.byref(n))
    finally:
        fs.release()
    return n.value


class ShardedPlan:
    """This process's part of a sharded exchange, collective to build: its plan holds the
    descriptors that write (pull) or read (push) its fields. ``exchange()`` runs it between two
    barriers; ``autotune()`` tunes it (collective; every process times real exchanges, which
    write disjoint halo elements and read no halo)."""

    def __init__(self, ctx: context, buffer_infos: Sequence[_core.BufferInfo], mode: Any = "pull"):
        import torch
        self.context = ctx
        self.mode = _MODES[mode]
        self._bis = _core._flatten(tuple(buffer_infos))
        self._arrays = [a for bi in self._bis for a in bi.arrays()]
        self._fields = _FieldSet(ctx, self._bis, share=True)
        h = C.c_void_p()
        err = None
        try:
            call("ghexb_plan_create_sharded", ctx._h, self._fields.handles, self._fields.n, self._fields.local,
                 self.mode, C.byref(h))
        except Exception as e:  # every process learns of it, then raises
            err = e
        if err is not None:
            self._fields.release()
        else:
            self._h = h
        try:
            ctx.agree(err)
        except Exception:
            if err is None:
                self.release()
            raise
        self._token = torch.zeros(1, device=torch.device("cuda", ctx.device)) if ctx.device_barriers else None
        # no process leaves the collective build (and changes its fields) while another still
        # builds: a plan build uploads tables and may autotune
        torch.cuda.synchronize(ctx.device)
        ctx.host_barrier()

    def info(self) -> dict:
        i = _capi.PlanInfo()
        call("ghexb_plan_get_info", self._h, C.byref(i))
        return i.as_dict()

    def _stream(self, stream):
        if stream is None:
            return _core.stream_of(self._arrays)
        return stream if isinstance(stream, C.c_void_p) else C.c_void_p(int(stream))

    def barrier(self, stream=None) -> None:
        """Every process's work on its exchange stream before this point is done before any work
        after it: an all-reduce on the stream (NCCL), or the host's (device synchronised, then a
        gloo barrier)."""
        import torch
        ctx = self.context
        if ctx.device_barriers:
            with torch.cuda.stream(_torch_stream(self._stream(stream), ctx.device)):
                _dist().all_reduce(self._token, group=ctx.group)
        else:
            torch.cuda.synchronize(ctx.device)
            ctx.host_barrier()

    def exchange(self, stream=None) -> None:
        s = self._stream(stream)
        self.barrier(s)
        call("ghexb_plan_graph_launch", self._h, s)
        self.barrier(s)

    def adjoint(self, stream=None) -> None:
        """Adjoint of the exchange (push plans): every halo value, in whichever process, is added
        into its local owner in the single-process order, and the halo is zeroed."""
        if self.mode != PUSH:
            raise ValueError("the adjoint of a sharded exchange runs on its push plan")
        s = self._stream(stream)
        self.barrier(s)
        call("ghexb_plan_adjoint_launch", self._h, s)
        self.barrier(s)

    def autotune(self, repeats: int = 10, stream=None) -> dict:
        s = self._stream(stream)
        i = _capi.PlanInfo()
        self.barrier(s)
        call("ghexb_plan_autotune", self._h, s, repeats, C.byref(i))
        self.barrier(s)
        return i.as_dict()

    def release(self, _release=_capi.release) -> None:
        _release("ghexb_plan_destroy", getattr(self, "_h", None))
        self._h = None
        fields = getattr(self, "_fields", None)
        if fields is not None:
            fields.release()

    def __del__(self):
        self.release()


def make_sharded_plan(ctx: context, buffer_infos: Sequence[_core.BufferInfo], mode: Any = "pull") -> ShardedPlan:
    return ShardedPlan(ctx, buffer_infos, mode)


class Handle:
    """communication_handle (communication_object.hpp:627-648): the exchange is done on every
    process once the stream reaches this point."""

    def __init__(self, stream: C.c_void_p, device: int):
        self._stream, self._device = stream, device

    def wait(self) -> None:
        _torch_stream(self._stream, self._device).synchronize()

    def is_ready(self) -> bool:
        return _torch_stream(self._stream, self._device).query()

    def progress(self) -> None:
        pass


class CommunicationObject:
    """make_communication_object(ctx) for domains spread over processes (communication_object.hpp:
    653-660). ``exchange(...)`` is collective: every process passes its own fields, in the same
    order of patterns and fields per domain. The plans are cached by every process's fields (the
    processes agree on a hit on the host, so that a build is always collective)."""

    def __init__(self, ctx: context, mode: Any = "pull", max_plans: int = 8):
        self.context = ctx
        self.mode = _MODES[mode]
        self.max_plans = max_plans
        self._plans: dict = {}

    def exchange(self, *buffer_infos) -> Handle:
        bis = _core._flatten(buffer_infos)
        mine = tuple((getattr(bi.pattern, "_shard_seq", None), bi.field.info["ptr"], repr(sorted(bi.field._spec().items())))
                     for bi in bis)
        key = tuple(self.context.all_gather(mine))
        plan = self._plans.get(key)
        if plan is None:
            if len(self._plans) >= self.max_plans:
                self._plans.pop(next(iter(self._plans))).release()
            plan = self._plans[key] = ShardedPlan(self.context, bis, self.mode)
        s = plan._stream(None)
        plan.exchange(s)
        return Handle(s, self.context.device)

    def release(self) -> None:
        for p in self._plans.values():
            p.release()
        self._plans = {}


def make_communication_object(ctx: context, mode: Any = "pull") -> CommunicationObject:
    return CommunicationObject(ctx, mode)
