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
    """The replay covers every forward element once and, in the gather-form adjoint, every halo
    image once (owners pairwise distinct, images equal to the forward destinations)."""
    from oracle import regular as O
    w = {"cfg0": W.config0, "cfg1": W.config1, "cfg4": W.config4}[cfg]()
    ctx, keep, handles = regular_handles(w)
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    _capi.call("ghexb_plan_check", ctx._h, arr, len(handles), C.byref(n))
    halo = 0
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(k - 1 for k in w.shape), halos, w.periodic, doms)
        halo += O.halo_cells(pat) * len(specs)
    assert n.value == 2 * halo


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


def cubed_handles(w_edge, w_levels, halo, boxes, ncomps, vectors, mem_halo=None, dtype_size=8):
    from ghex_b200.structured import cubed_sphere as CS
    mem_halo = halo if mem_halo is None else mem_halo
    ctx = CS.make_context(device=0)
    cube = CS.cube(w_edge, w_levels)
    doms = [CS.DomainDescriptor(cube, *b) for b in boxes]
    pat = CS.make_pattern(ctx, CS.HaloGenerator(halo), doms)
    keep, handles, base = [ctx, pat], [], 1 << 40
    code = _capi.F64 if dtype_size == 8 else _capi.F32
    for nc, isv in zip(ncomps, vectors):
        for d, b in zip(doms, boxes):
            nx, ny = b[2] - b[1] + 1 + 2 * mem_halo, b[4] - b[3] + 1 + 2 * mem_halo
            ext = (nx, ny, w_levels, nc)
            strides = (dtype_size, dtype_size * nx, dtype_size * nx * ny, dtype_size * nx * ny * w_levels)
            f = CS.FieldDescriptor.__new__(CS.FieldDescriptor)
            f.array, f._handles, f.domain = None, {}, d
            f.info = {"ptr": base, "shape": ext, "strides": strides, "dtype": code, "itemsize": dtype_size, "device": 0}
            f.offsets, f.extents = (mem_halo, mem_halo, 0, 0), ext
            f.num_components, f.is_vector, f.layout = nc, isv, R._layout_order(strides)
            base += ((nx * ny * w_levels * nc * dtype_size + 255) // 256) * 256
            keep.append(f)
            handles.append(pat(f).handle())
    return ctx, keep, handles


@pytest.mark.parametrize("case", ["cfg3", "reference-test"])
def test_cubed_plan_accesses_in_bounds(case):
    from ghex_b200 import workloads as W
    if case == "cfg3":
        w = W.config3()
        ctx, keep, handles = cubed_handles(w.edge, w.levels, w.halo, w.domains, [1, 2], [False, True])
    else:
        boxes = [(t, x0, x0 + 4, y0, y0 + 4) for t in range(6) for (x0, y0) in ((0, 0), (5, 0), (0, 5), (5, 5))]
        ctx, keep, handles = cubed_handles(10, 6, 2, boxes, [8, 8], [False, True], mem_halo=3, dtype_size=4)
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    _capi.call("ghexb_plan_check", ctx._h, arr, len(handles), C.byref(n))
    assert n.value > 0


def unstructured_handles(doms_spec, levels, levels_first, dtype_size=8):
    from ghex_b200 import unstructured as U
    ctx = U.make_context(device=0)
    doms = [U.DomainDescriptor(*d) for d in doms_spec]
    pat = U.make_pattern(ctx, U.HaloGenerator(), doms)
    keep, handles, base = [ctx, pat], [], 1 << 40
    code = _capi.F64 if dtype_size == 8 else _capi.F32
    for d in doms:
        n = d.size()
        f = U.FieldDescriptor.__new__(U.FieldDescriptor)
        f.array, f._handles, f.domain_desc = None, {}, d
        f.info = {"ptr": base, "shape": (n, levels), "dtype": code, "itemsize": dtype_size, "device": 0}
        f.levels, f.levels_first, f.outer_stride = levels, levels_first, 0
        base += ((n * levels * dtype_size + 255) // 256) * 256
        keep.append(f)
        handles.append(pat(f).handle())
    return ctx, keep, handles


@pytest.mark.parametrize("case", ["cfg2-f64", "cfg2-f32", "fixture-levels-last"])
def test_unstructured_plan_accesses_in_bounds(case):
    import golden_cases as G
    from ghex_b200 import workloads as W
    if case.startswith("cfg2"):
        doms = W.config2().domains
        ctx, keep, handles = unstructured_handles(doms, 64, True, 8 if case.endswith("64") else 4)
    else:
        g = G.unstructured_domains()
        doms = [(r, g[r]["all"], g[r]["outer_lids"]) for r in sorted(g)]
        ctx, keep, handles = unstructured_handles(doms, 2, False)
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    _capi.call("ghexb_plan_check", ctx._h, arr, len(handles), C.byref(n))
    assert n.value > 0


@pytest.mark.parametrize("name", ["simple_2d_2x2", "uneven_3d"])
def test_staged_plan_accesses_in_bounds(name):
    """Every stage of a staged pattern: accesses stay inside the fields, and the forward writes
    each receive cell of the stage once."""
    import regular_cases as RC
    case = RC.staged_cases()[name]
    dim = len(case["shape"])
    ctx = R.make_context(device=0)
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in case["domains"]]
    pats = R.make_staged_pattern(ctx, doms, case["lookup"], (0,) * dim, tuple(n - 1 for n in case["shape"]),
                                 case["halos"], case["periodic"])
    keep, base = [], 1 << 40
    fields = []
    for d, (_, f, l) in zip(doms, case["domains"]):
        ext = tuple(l[k] - f[k] + 1 + case["halos"][2 * k] + case["halos"][2 * k + 1] for k in range(dim))
        fields.append(FakeField(d, base, _capi.F64, 8, case["offsets"], ext))
        n = 1
        for e in ext:
            n *= e
        base += ((n * 8 + 255) // 256) * 256
    for p in pats:
        handles = [p(f).handle() for f in fields]
        arr = (C.c_void_p * len(handles))(*handles)
        n = C.c_int64()
        _capi.call("ghexb_plan_check", ctx._h, arr, len(handles), C.byref(n))
        cells = 0
        for i in range(len(doms)):
            for _, lf, ll, _, _ in p.spaces(i):
                c = 1
                for k in range(dim):
                    c *= ll[k] - lf[k] + 1
                cells += c
        assert n.value == 2 * cells
