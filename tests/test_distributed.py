"""Sharded exchange across processes (ghex_b200.distributed), host side, as two gloo ranks on the
CPU: every rank builds the same patterns from the domains all ranks pass, wraps the other ranks'
fields at their (never dereferenced) addresses, and replays its part of the exchange
(ghexb_plan_check_sharded). The parts are disjoint and together are the single-process exchange:
in the pull form a rank writes exactly its domains' halos, in the push form it reads exactly its
domains' interiors."""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _fake_regular(R, dom, base, spec, w):
    """A regular field descriptor at a fake address (host-only checks)."""
    import numpy as np
    ext = w.extents(dom, spec)
    es = np.dtype(spec.dtype).itemsize
    f = R.FieldDescriptor.__new__(R.FieldDescriptor)
    strides, s = [], es
    for e in ext:
        strides.append(s)
        s *= e
    from ghex_b200 import _capi
    f.array, f._handles = None, {}
    f.info = {"ptr": base, "shape": tuple(ext), "strides": tuple(strides), "dtype": _capi.F64 if es == 8 else _capi.F32,
              "itemsize": es, "device": 0}
    f.domain_desc = R.DomainDescriptor(dom[0], (dom[1], dom[2]))
    f.offsets, f.extents = tuple(w.offsets(spec)), tuple(ext)
    f.layout = R._layout_order(f.info["strides"])
    f.num_components, f.ndim = 1, len(ext)
    return f, ((s + 255) // 256) * 256


def regular_case(ctx, rank, world):
    """cfg1 at a small size, domains dealt round-robin to the ranks; expected halo elements per rank
    for the pull and push forms from the oracle's pattern."""
    from ghex_b200 import distributed as D
    from ghex_b200 import workloads as W
    from ghex_b200.structured import regular as R
    from oracle import regular as O
    w = W.config1(shape=(60, 45, 15))
    mine = [i for i in range(len(w.domains)) if i % world == rank]
    bis, keep = [], []
    base = (1 << 40) + rank * (1 << 36)
    pull = push = 0
    for halos, specs in w.halo_groups().items():
        hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                             [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
        pat = D.make_pattern(ctx, hg, [R.DomainDescriptor(i, (f, l)) for i, f, l in (w.domains[j] for j in mine)])
        keep.append(pat)
        for spec in specs:
            for j in mine:
                f, size = _fake_regular(R, w.domains[j], base, spec, w)
                base += size
                keep.append(f)
                bis.append(pat(f))
        opat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic,
                              [O.Domain(i, f, l) for i, f, l in w.domains])
        for i, entries in enumerate(opat):
            for en in entries:
                cells = O.halo_cells([[en]]) * len(specs)
                pull += cells if i in mine else 0
                push += cells if en.neighbor in mine else 0
    return bis, keep, pull, push


def cubed_case(ctx, rank, world):
    from ghex_b200 import _capi
    from ghex_b200 import distributed as D
    from ghex_b200.structured import cubed_sphere as CS
    from ghex_b200.structured import regular as R
    edge, levels, halo = 12, 4, 2
    cube = CS.cube(edge, levels)
    boxes = [(t, x0, x0 + 5, y0, y0 + 5) for t in range(6) for (x0, y0) in ((0, 0), (6, 0), (0, 6), (6, 6))]
    mine = [b for i, b in enumerate(boxes) if i % world == rank]
    pat = D.make_pattern(ctx, CS.HaloGenerator(halo), [CS.DomainDescriptor(cube, *b) for b in mine])
    bis, keep, base = [], [pat], (1 << 40) + rank * (1 << 36)
    for nc, isv in ((1, False), (2, True)):
        for b in mine:
            nx, ny = b[2] - b[1] + 1 + 2 * halo, b[4] - b[3] + 1 + 2 * halo
            ext = (nx, ny, levels, nc)
            strides = (8, 8 * nx, 8 * nx * ny, 8 * nx * ny * levels)
            f = CS.FieldDescriptor.__new__(CS.FieldDescriptor)
            f.array, f._handles, f.domain = None, {}, CS.DomainDescriptor(cube, *b)
            f.info = {"ptr": base, "shape": ext, "strides": strides, "dtype": _capi.F64, "itemsize": 8, "device": 0}
            f.offsets, f.extents = (halo, halo, 0, 0), ext
            f.num_components, f.is_vector, f.layout = nc, isv, R._layout_order(strides)
            base += ((nx * ny * levels * nc * 8 + 255) // 256) * 256
            keep.append(f)
            bis.append(pat(f))
    return bis, keep, None, None


def unstructured_case(ctx, rank, world):
    import golden_cases as G
    from ghex_b200 import _capi
    from ghex_b200 import distributed as D
    from ghex_b200 import unstructured as U
    g = G.unstructured_domains()
    mine = [r for r in sorted(g) if r % world == rank]
    doms = [U.DomainDescriptor(r, g[r]["all"], g[r]["outer_lids"]) for r in mine]
    pat = D.make_pattern(ctx, U.HaloGenerator(), doms)
    bis, keep, base = [], [pat], (1 << 40) + rank * (1 << 36)
    for d in doms:
        n = d.size()
        f = U.FieldDescriptor.__new__(U.FieldDescriptor)
        f.array, f._handles, f.domain_desc = None, {}, d
        f.info = {"ptr": base, "shape": (n, 2), "dtype": _capi.F64, "itemsize": 8, "device": 0}
        f.levels, f.levels_first, f.outer_stride = 2, True, 0
        base += ((n * 2 * 8 + 255) // 256) * 256
        keep.append(f)
        bis.append(pat(f))
    return bis, keep, None, None


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from ghex_b200 import _capi
        from ghex_b200 import distributed as D
        ctx = D.make_context(device=0)
        res = {}
        for name, case in (("regular", regular_case), ("cubed", cubed_case), ("unstructured", unstructured_case)):
            bis, keep, want_pull, want_push = case(ctx, rank, world)
            got_pull = D.check_sharded(ctx, bis, "pull")
            got_push = D.check_sharded(ctx, bis, "push")
            # the whole exchange: every field marked local, as one process holding all domains
            fs = D._FieldSet(ctx, bis, share=False)
            n = C.c_int64()
            _capi.call("ghexb_plan_check_sharded", ctx._h, fs.handles, fs.n, bytes([1] * fs.n), 1, C.byref(n))
            fs.release()
            res[name] = (got_pull, got_push, want_pull, want_push, n.value)
        # a field of another rank's domain is refused
        from ghex_b200.structured import regular as R
        from ghex_b200 import workloads as W
        w = W.config1(shape=(60, 45, 15))
        hg = R.HaloGenerator(((0, 0, 0), (59, 44, 14)), [(1, 1)] * 3, (False, True, False))
        pat = D.make_pattern(ctx, hg, [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains if i % world == rank])
        other = [d for d in w.domains if d[0] % world != rank][0]
        spec = W.FieldSpec("x", __import__("numpy").float64, (1, 1, 1, 1, 1, 1), 1)
        f, _ = _fake_regular(R, other, 1 << 40, spec, w)
        try:
            pat(f)
            refused = False
        except ValueError as e:
            refused = "belongs to rank" in str(e)
        # a failure on one rank reaches every rank: rank 1 passes a field of a pattern that is not
        # distributed, and both ranks raise instead of waiting on each other
        bis, keep, _, _ = regular_case(ctx, rank, world)
        if rank == 1:
            plain = R.make_pattern(ctx, hg, [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains])
            g, _ = _fake_regular(R, w.domains[1], 1 << 41, spec, w)
            keep += [plain, g]
            bis = bis + [plain(g)]
        try:
            D.check_sharded(ctx, bis, "pull")
            failure = None
        except ValueError as e:
            failure = ("ValueError", "distributed.make_pattern" in str(e))
        except RuntimeError as e:
            failure = ("RuntimeError", "rank 1 failed" in str(e))
        out.put((rank, res, refused and failure is not None and failure[1], ))
    finally:
        dist.destroy_process_group()


def test_sharded_parts_partition_the_exchange():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (v, refused)) for r, v, refused in (q.get(timeout=300) for _ in ps))
    # (refused also holds: a failure on rank 1 raised on both ranks)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r][1], "a field of another rank's domain was accepted"
    for name in ("regular", "cubed", "unstructured"):
        (p0, s0, wp0, ws0, full0), (p1, s1, wp1, ws1, full1) = res[0][0][name], res[1][0][name]
        assert full0 == full1 > 0
        assert p0 + p1 == full0, name        # pull parts: every halo element written by one rank
        assert s0 + s1 == full0, name        # push parts: every halo element read by one rank
        assert min(p0, p1, s0, s1) > 0, name
        if wp0 is not None:
            assert (p0, p1, s0, s1) == (wp0, wp1, ws0, ws1), name
