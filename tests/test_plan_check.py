"""Host replay of every kernel address (ghexb_plan_check): all accesses of the forward and adjoint
kernels stay inside the wrapped field memory, for the benchmark configurations (no GPU needed).
Fields are wrapped at fake, aligned device addresses: nothing is dereferenced."""
import ctypes as C

import pytest

from ghex_b200 import _capi
from ghex_b200 import workloads as W
from ghex_b200.structured import regular as R


class FakeField(R.FieldDescriptor):
    """A field descriptor for an address that is never dereferenced (host-only checks)."""

    def __init__(self, dom, ptr, dtype, itemsize, offsets, extents):
        self.array = None
        self._handles = {}
        strides, s = [], itemsize
        for e in extents:
            strides.append(s)
            s *= e
        self.info = {"ptr": ptr, "shape": tuple(extents), "strides": tuple(strides), "dtype": dtype,
                     "itemsize": itemsize, "device": 0}
        self.domain_desc = dom
        self.offsets, self.extents = tuple(offsets), tuple(extents)
        self.layout = R._layout_order(self.info["strides"])
        self.num_components, self.ndim = 1, len(extents)


def regular_handles(w):
    ctx = R.make_context(device=0)
    keep, handles = [ctx], []
    base = 1 << 40
    for halos, specs in w.halo_groups().items():
        hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                             [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
        doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
        pat = R.make_pattern(ctx, hg, doms)
        keep.append(pat)
        for spec in specs:
            es = 8 if spec.dtype.__name__ == "float64" else 4
            code = _capi.F64 if es == 8 else _capi.F32
            for dm, d in zip(doms, w.domains):
                ext = w.extents(d, spec)
                f = FakeField(dm, base, code, es, w.offsets(spec), ext)
                n = 1
                for e in ext:
                    n *= e
                base += ((n * es + 255) // 256) * 256
                keep.append(f)
                handles.append(pat(f).handle())
    return ctx, keep, handles


@pytest.mark.parametrize("cfg", ["cfg0", "cfg1", "cfg4"])
def test_regular_plan_accesses_in_bounds(cfg):
    w = {"cfg0": W.config0, "cfg1": W.config1, "cfg4": W.config4}[cfg]()
    ctx, keep, handles = regular_handles(w)
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    _capi.call("ghexb_plan_check", ctx._h, arr, len(handles), C.byref(n))
    assert n.value > 0


def test_check_rejects_too_small_memory():
    """Extents smaller than the halo: the plan is refused before any kernel could run."""
    w = W.config0()
    ctx = R.make_context(device=0)
    hg = R.HaloGenerator(((0, 0, 0), (63, 63, 63)), (2, 2, 2), (True, True, True))
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
    pat = R.make_pattern(ctx, hg, doms)
    fs = [FakeField(d, (1 << 40) + i * (1 << 30), _capi.F64, 8, (1, 1, 1), (34, 34, 34)) for i, d in enumerate(doms)]
    handles = [pat(f).handle() for f in fs]
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    rc = _capi.lib.ghexb_plan_check(ctx._h, arr, len(handles), C.byref(n))
    assert rc == _capi.ERR_RANGE
