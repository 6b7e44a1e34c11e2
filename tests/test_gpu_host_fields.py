"""Fields in host memory: the device kernels read the source cells from host memory and write
the halo cells into it, bit-exact against the oracle, for the three grids, through the
communication object and explicit plans; pinned tensors as they are, ordinary numpy arrays and
torch CPU tensors page-locked by their field descriptors (the reference's own Python test runs on
numpy arrays this way)."""
import numpy as np
import pytest
import torch

from ghex_b200 import Architecture
from ghex_b200 import unstructured as U
from ghex_b200 import workloads as W
from ghex_b200.structured import cubed_sphere as C
from ghex_b200.structured import regular as R
from gpu_helpers import RegularRun, bits_equal
from oracle import cubed_sphere as OC
from oracle import unstructured as OU

pytestmark = pytest.mark.gpu


def pinned(a: np.ndarray) -> torch.Tensor:
    src = torch.from_numpy(a)
    t = torch.empty_strided(tuple(src.shape), tuple(src.stride()), dtype=src.dtype, pin_memory=True)
    t.copy_(src)
    assert t.is_pinned() and t.stride() == src.stride()
    return t


def test_regular_pinned_host_fields(cuda):
    w = W.config1(shape=(40, 30, 12))
    run = RegularRun(w, cuda)
    expected = run.oracle()
    host = {name: [pinned(a) for a in arrays] for name, arrays in run.host.items()}
    bis = []
    for halos, specs in w.halo_groups().items():
        pat = run.patterns[halos]
        for spec in specs:
            for dm, d, t in zip(pat.domains, w.domains, host[spec.name]):
                bis.append(pat(R.make_field_descriptor(dm, t, w.offsets(spec), w.extents(d, spec),
                                                       arch=Architecture.CPU)))
    co = R.make_communication_object(run.ctx)
    co.exchange(bis).wait()
    for name, ts in host.items():
        assert sum(bits_equal(t.numpy(), e) for t, e in zip(ts, expected[name])) == 0
    plan = R.make_exchange_plan(run.ctx, bis)
    for form in (plan.BATCHED, plan.PER_FIELD, plan.PER_BOX):
        for name, ts in host.items():
            for t, a in zip(ts, run.host[name]):
                t.copy_(torch.from_numpy(a))
        plan.launch(form)
        torch.cuda.synchronize()
        for name, ts in host.items():
            assert sum(bits_equal(t.numpy(), e) for t, e in zip(ts, expected[name])) == 0


def test_unstructured_pinned_host_fields(cuda):
    w = W.config2(ni=48, nj=64, parts=6, levels=8)
    host = [w.domain_array(d, np.float64, 1) for d in w.domains]
    odoms = [OU.Domain(*d) for d in w.domains]
    recv, send, _ = OU.make_pattern(odoms)
    expected = [a.copy() for a in host]
    OU.exchange(recv, send, expected)
    ctx = U.make_context()
    ud = [U.DomainDescriptor(*d) for d in w.domains]
    pat = U.make_pattern(ctx, U.HaloGenerator(), ud)
    ts = [pinned(a) for a in host]
    bis = [pat(U.make_field_descriptor(d, t)) for d, t in zip(ud, ts)]
    U.make_communication_object(ctx).exchange(bis).wait()
    assert sum(bits_equal(t.numpy(), e) for t, e in zip(ts, expected)) == 0


def test_cubed_sphere_pinned_host_vector_field(cuda):
    w = W.config3(edge=48, levels=4, split=2)
    host = [w.domain_array(d, 2, 2) for d in w.domains]
    odoms = [OC.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
    expected = [a.copy(order="K") for a in host]
    OC.exchange(OC.make_pattern(w.edge, (w.halo,) * 4, odoms), odoms, expected, [w.offsets()] * len(odoms), w.edge,
                True)
    ctx = C.make_context()
    cube = C.cube(w.edge, w.levels)
    doms = [C.DomainDescriptor(cube, *b) for b in w.domains]
    pat = C.make_pattern(ctx, C.HaloGenerator(w.halo), doms)
    ts = [pinned(a) for a in host]
    bis = [pat(C.make_field_descriptor(d, t, w.offsets(), a.shape[:3], 2, True)) for d, t, a in zip(doms, ts, host)]
    C.make_communication_object(ctx).exchange(bis).wait()
    assert sum(bits_equal(t.numpy(), e) for t, e in zip(ts, expected)) == 0


def test_pageable_host_fields(cuda):
    """Ordinary numpy arrays and torch CPU tensors: the field descriptor page-locks their memory
    (shared pages reference-counted) and the exchange runs on it in place."""
    w = W.config1(shape=(40, 30, 12))
    run = RegularRun(w, cuda)
    expected = run.oracle()
    host = {name: [np.array(a, order="K") if i % 2 else torch.from_numpy(np.array(a, order="K"))
                   for i, a in enumerate(arrays)] for name, arrays in run.host.items()}
    bis = []
    for halos, specs in w.halo_groups().items():
        pat = run.patterns[halos]
        for spec in specs:
            for dm, d, t in zip(pat.domains, w.domains, host[spec.name]):
                bis.append(pat(R.make_field_descriptor(dm, t, w.offsets(spec), w.extents(d, spec),
                                                       arch=Architecture.CPU)))
    for _ in range(2):
        R.make_communication_object(run.ctx).exchange(bis).wait()
    for name, ts in host.items():
        got = [t.numpy() if isinstance(t, torch.Tensor) else t for t in ts]
        assert sum(bits_equal(g, e) for g, e in zip(got, expected[name])) == 0


def test_numpy_fields_as_in_the_reference_python_test(cuda):
    """test/bindings/python/test_structured_pattern.py with every process's domain in this one:
    2x2x1 domains of a (2*26) x 26 x 1 grid, halos ((2, 1), (1, 1), (0, 0)), periodic in x and y,
    three float64 numpy fields (x fastest) holding their domain's grid coordinate along one
    dimension each, and a field holding the domain's id; after one exchange every halo cell inside
    the global grid holds the coordinates and id of the domain that owns it."""
    nx, ny, nz = 2 * 26, 26, 1
    dims = (2, 2, 1)
    halos = ((2, 1), (1, 1), (0, 0))
    periodic = (True, True, False)
    spec = W.regular_decomposition((nx, ny, nz), dims)
    coords = {i: (f[0] // (nx // dims[0]), f[1] // (ny // dims[1]), 0) for i, f, _ in spec}
    ctx = R.make_context()
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in spec]
    pat = R.make_pattern(ctx, R.HaloGenerator(((0, 0, 0), (nx - 1, ny - 1, nz - 1)), halos, periodic), doms)
    fields, bis = {}, []
    for d, (i, f, l) in zip(doms, spec):
        ext = tuple(l[k] - f[k] + 1 + halos[k][0] + halos[k][1] for k in range(3))
        off = tuple(h[0] for h in halos)
        arrs = [np.zeros(ext, dtype=np.float64, order="F") for _ in range(4)]
        inner = tuple(slice(off[k], off[k] + l[k] - f[k] + 1) for k in range(3))
        for k in range(3):
            arrs[k][inner] = coords[i][k]
        arrs[3][inner] = i
        fields[i] = (f, arrs, off)
        bis += [pat(R.make_field_descriptor(d, a, off, ext)) for a in arrs]
    R.make_communication_object(ctx).exchange(bis).wait()
    owner_of = {c: i for i, c in coords.items()}
    box = {i: (f, l) for i, f, l in spec}
    for i, (f, arrs, off) in fields.items():
        for m in np.ndindex(*arrs[0].shape):
            g = tuple(m[k] - off[k] + f[k] for k in range(3))
            if not all(0 <= g[k] < (nx, ny, nz)[k] for k in range(3)):
                continue
            c = tuple(int(arrs[k][m]) for k in range(3))
            owner = owner_of[c]
            lo, hi = box[owner]
            assert all(lo[k] <= g[k] <= hi[k] for k in range(3)), (i, m, c)
            assert int(arrs[3][m]) == owner


def test_device_array_with_cpu_arch_refused(cuda):
    w = W.config0()
    run = RegularRun(w, cuda)
    halos, specs = next(iter(w.halo_groups().items()))
    pat = run.patterns[halos]
    dm, d = pat.domains[0], w.domains[0]
    with pytest.raises(TypeError, match="host array"):
        R.make_field_descriptor(dm, run.dev[specs[0].name][0], w.offsets(specs[0]), w.extents(d, specs[0]),
                                arch=Architecture.CPU)


def test_library_host_memory_fields(cuda):
    """Fields in page-locked host memory from ghex_b200.host_empty (cudaHostAlloc, mapped): the
    exchange runs on them in place, bit-exact, and the memory is released with the arrays."""
    from ghex_b200 import host_empty
    w = W.config1(shape=(40, 30, 12))
    run = RegularRun(w, cuda)
    expected = run.oracle()
    host = {}
    for name, arrays in run.host.items():
        hs = []
        for a in arrays:
            h = host_empty(a.shape, a.dtype, order="F")
            h[...] = a
            hs.append(h)
        host[name] = hs
    bis = []
    for halos, specs in w.halo_groups().items():
        pat = run.patterns[halos]
        for spec in specs:
            for dm, d, h in zip(pat.domains, w.domains, host[spec.name]):
                bis.append(pat(R.make_field_descriptor(dm, h, w.offsets(spec), w.extents(d, spec),
                                                       arch=Architecture.CPU)))
    co = R.make_communication_object(run.ctx)
    for _ in range(2):
        co.exchange(bis).wait()
        for name, hs in host.items():
            assert sum(bits_equal(h, e) for h, e in zip(hs, expected[name])) == 0
