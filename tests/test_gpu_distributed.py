"""Sharded exchange on the device: two processes share one GPU, each owning half the domains, its
fields mapped into the other through CUDA IPC. The processes meet at host barriers (gloo) around
every exchange, so no kernel waits on another process's kernel. Pull and push forms, the push
form's adjoint, an autotuned plan and the communication object are bit-exact against the oracle's
single-process exchange, on a regular grid and on the cubed sphere (vector components negated
across rotated edges, some of them between the processes)."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def _regular(ctx, rank, world, dev):
    import numpy as np
    from ghex_b200 import distributed as D
    from ghex_b200 import workloads as W
    from ghex_b200.structured import regular as R
    from gpu_helpers import to_device
    w = W.config1(shape=(50, 40, 12))
    mine = [i for i in range(len(w.domains)) if i % world == rank]
    host, tens, bis, keep = [], [], [], []
    for halos, specs in w.halo_groups().items():
        hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                             [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
        doms = {i: R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains}
        pat = D.make_pattern(ctx, hg, [doms[i] for i in mine])
        keep.append(pat)
        for spec in specs:
            for i in mine:
                d = w.domains[i]
                a = w.domain_array(d, spec)
                t = to_device(a, dev)
                fd = R.make_field_descriptor(doms[i], t, w.offsets(spec), w.extents(d, spec))
                keep.append(fd)
                host.append((spec.name, i, a))
                tens.append(t)
                bis.append(pat(fd))
    return w, mine, host, tens, bis, keep


def _oracle_regular(w, grads=None):
    """The single-process oracle exchange (or, given grads, adjoint) of every field."""
    from oracle import regular as O
    out = {}
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for spec in specs:
            if grads is None:
                arrays = [w.domain_array(d, spec) for d in w.domains]
                O.exchange(pat, doms, arrays, [w.offsets(spec)] * len(doms))
            else:
                arrays = [g.copy(order="K") for g in grads[spec.name]]
                O.adjoint(pat, doms, arrays, [w.offsets(spec)] * len(doms))
            for i, a in enumerate(arrays):
                out[(spec.name, i)] = a
    return out


def _cubed(ctx, rank, world, dev):
    """The cubed sphere at 48 x 48 x 8 per tile, 2 x 2 domains per tile dealt round-robin: a scalar
    and a vector field (components negated across rotated edges)."""
    from ghex_b200 import distributed as D
    from ghex_b200 import workloads as W
    from ghex_b200.structured import cubed_sphere as CS
    from gpu_helpers import to_device
    w = W.config3(edge=48, levels=8, split=2)
    mine = [i for i in range(len(w.domains)) if i % world == rank]
    cube = CS.cube(w.edge, w.levels)
    pat = D.make_pattern(ctx, CS.HaloGenerator(w.halo), [CS.DomainDescriptor(cube, *w.domains[i]) for i in mine])
    host, tens, bis, keep = [], [], [], [pat]
    for name, nc, isv, seed in (("s", 1, False, 1), ("v", 2, True, 2)):
        for i in mine:
            a = w.domain_array(w.domains[i], nc, seed)
            t = to_device(a, dev)
            fd = CS.make_field_descriptor(CS.DomainDescriptor(cube, *w.domains[i]), t, w.offsets(), a.shape[:3], nc, isv)
            keep.append(fd)
            host.append((name, i, a))
            tens.append(t)
            bis.append(pat(fd))
    return w, host, tens, bis, keep


def _oracle_cubed(w, grads=None):
    """Single-process oracle over the domains in id order (the order of a distributed pattern)."""
    from oracle import cubed_sphere as O
    order = sorted(range(len(w.domains)), key=lambda i: (w.domains[i][0], (w.domains[i][1], w.domains[i][3])))
    odoms = [O.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in (w.domains[i] for i in order)]
    pat = O.make_pattern(w.edge, (w.halo,) * 4, odoms)
    out = {}
    for name, nc, isv, seed in (("s", 1, False, 1), ("v", 2, True, 2)):
        if grads is None:
            arrays = [w.domain_array(w.domains[i], nc, seed) for i in order]
            O.exchange(pat, odoms, arrays, [w.offsets()] * len(odoms), w.edge, isv)
        else:
            arrays = [grads[(name, i)].copy(order="K") for i in order]
            O.adjoint(pat, odoms, arrays, [w.offsets()] * len(odoms), w.edge, isv)
        for i, a in zip(order, arrays):
            out[(name, i)] = a
    return out


def _mismatches(host, tens, expected):
    import torch
    from gpu_helpers import bits_equal
    torch.cuda.synchronize()
    return sum(bits_equal(t.cpu().numpy(), expected[(name, i)]) for (name, i, _), t in zip(host, tens))


def _reset(host, tens, arrays=None):
    import torch
    for k, ((name, i, a), t) in enumerate(zip(host, tens)):
        t.copy_(torch.from_numpy(a if arrays is None else arrays[(name, i)]))
    torch.cuda.synchronize()


def _rank(rank: int, world: int, port: int, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    res = {}
    try:
        import numpy as np
        from ghex_b200 import distributed as D
        ctx = D.make_context(device=0)
        assert not ctx.device_barriers
        w, mine, host, tens, bis, keep = _regular(ctx, rank, world, dev)
        expected = _oracle_regular(w)

        pull = D.make_sharded_plan(ctx, bis, "pull")
        info = pull.info()
        res["pull_halo_elements"] = info["halo_elements"]
        pull.exchange()
        res["pull"] = _mismatches(host, tens, expected)

        _reset(host, tens)
        pull.autotune(repeats=2)
        _reset(host, tens)
        pull.exchange()
        res["pull_autotuned"] = _mismatches(host, tens, expected)
        pull.release()

        _reset(host, tens)
        push = D.make_sharded_plan(ctx, bis, "push")
        push.exchange()
        res["push"] = _mismatches(host, tens, expected)

        # adjoint: seeded random values in every cell of every field (all ranks draw the same)
        rng = np.random.default_rng(11)
        grads = {}
        for halos, specs in w.halo_groups().items():
            for spec in specs:
                grads[spec.name] = [np.asfortranarray(rng.standard_normal(w.domain_array(d, spec).shape)
                                                      .astype(w.domain_array(d, spec).dtype)) for d in w.domains]
        seeded = {(name, i): g for name, gs in grads.items() for i, g in enumerate(gs)}
        _reset(host, tens, seeded)
        push.adjoint()
        res["adjoint"] = _mismatches(host, tens, _oracle_regular(w, grads))
        try:
            pull_again = D.make_sharded_plan(ctx, bis, "pull")
            pull_again.adjoint()
            res["pull_adjoint_refused"] = False
        except ValueError:
            res["pull_adjoint_refused"] = True
        pull_again.release()
        push.release()

        # the cubed sphere: pull and push forms, and the push form's adjoint
        cw, chost, ctens, cbis, ckeep = _cubed(ctx, rank, world, dev)
        cexp = _oracle_cubed(cw)
        for mode in ("pull", "push"):
            _reset(chost, ctens)
            plan = D.make_sharded_plan(ctx, cbis, mode)
            plan.exchange()
            res[f"cubed_{mode}"] = _mismatches(chost, ctens, cexp)
            if mode == "push":
                crng = np.random.default_rng(5)
                # every rank draws every domain's gradient in the same order
                allg = {}
                for name, nc, seed in (("s", 1, 1), ("v", 2, 2)):
                    for i, d in enumerate(cw.domains):
                        shape = cw.domain_array(d, nc, seed).shape
                        allg[(name, i)] = np.asfortranarray(crng.standard_normal(shape))
                _reset(chost, ctens, allg)
                plan.adjoint()
                res["cubed_adjoint"] = _mismatches(chost, ctens, _oracle_cubed(cw, allg))
            plan.release()

        _reset(host, tens)
        co = D.make_communication_object(ctx)
        co.exchange(bis).wait()
        res["co"] = _mismatches(host, tens, expected)
        _reset(host, tens)
        co.exchange(bis).wait()  # the cached plan
        res["co_cached"] = _mismatches(host, tens, expected)
        res["co_plans"] = len(co._plans)
        co.release()
        ctx.host_barrier()
        out.put((rank, res, None))
    except Exception as e:  # reported to the test, which fails with it
        import traceback
        out.put((rank, res, traceback.format_exc()))
        raise
    finally:
        dist.destroy_process_group()


def test_sharded_exchange_two_processes_one_gpu(cuda):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = {}
    for _ in ps:
        r, res, err = q.get(timeout=600)
        assert err is None, f"rank {r}:\n{err}"
        got[r] = res
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in (0, 1):
        res = got[r]
        assert res["pull_halo_elements"] > 0
        for k in ("pull", "pull_autotuned", "push", "adjoint", "co", "co_cached", "cubed_pull", "cubed_push",
                  "cubed_adjoint"):
            assert res[k] == 0, (r, k, res[k])
        assert res["pull_adjoint_refused"]
        assert res["co_plans"] == 1
