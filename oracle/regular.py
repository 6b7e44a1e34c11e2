"""Oracle for regular structured grids (test infrastructure only).

Restates, in plain Python and numpy:
  * structured::regular::halo_generator::operator()  structured/regular/halo_generator.hpp:91-146
  * halo_generator::intersect                        structured/regular/halo_generator.hpp:148-158
  * make_pattern_impl<structured grid>::apply         structured/pattern.hpp:214-365
  * the exchange: pack (structured/regular/field_descriptor.hpp:72-83, pack_kernels.hpp:66-101)
    followed by unpack (field_descriptor.hpp:85-96, pack_kernels.hpp:103-138) with the buffer
    removed — the value that lands in a halo cell is the value of the cell it was packed from.
  * make_staged_pattern (structured/regular/make_pattern.hpp:47-256) and the exchange of its
    stages one after the other, each as GHEX's message passing: all send spaces packed, then
    the k-th receive space of an entry filled from the k-th send space of the sender's entry;
  * the adjoint: the explicit transpose of that copy, visited in receive-map order
    (pattern order, then neighbour id, then iteration space, then for_loop order of
    util/for_each.hpp:84-112): owner += halo; halo = 0.

Fields are numpy arrays indexed by coordinate (x, y, z[, component]) whose index 0 is the first
cell of the wrapped memory; `offsets` locate the domain's first cell in it.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np


def _cmod(a: int, b: int) -> int:
    """C++ '%' on ints (truncates toward zero)."""
    r = abs(a) % abs(b)
    return -r if a < 0 else r


@dataclass
class Domain:
    id: int
    first: tuple
    last: tuple


@dataclass
class Space:
    lfirst: tuple
    llast: tuple
    gfirst: tuple
    glast: tuple


@dataclass
class Entry:
    neighbor: int             # index of the source domain
    tag: int
    spaces: list = field(default_factory=list)


def halo_boxes(dom: Domain, g_first, g_last, halos, periodic) -> list[Space]:
    """halo_generator::operator() (halo_generator.hpp:91-146)."""
    dim = len(dom.first)
    iv = []
    for k in range(dim):
        f, l = dom.first[k], dom.last[k]
        ext = l - f
        hm, hp = halos[2 * k], halos[2 * k + 1]
        iv.append([(-hm, -1, f - hm, f - 1), (0, ext, f, l), (ext + 1, ext + hp, l + 1, l + hp)])
    out = []
    # compute_spaces (:161-195): dimension 0 varies slowest
    for j, combo in enumerate(itertools.product(range(3), repeat=dim)):
        if j == 3 ** dim // 2:
            continue
        b = [iv[k][combo[k]] for k in range(dim)]
        if any(t[1] < t[0] for t in b):
            continue
        gf, gl = [t[2] for t in b], [t[3] for t in b]
        for k in range(dim):
            if not periodic[k]:
                continue
            ext_h = gl[k] - gf[k]
            ext = g_last[k] + 1 - g_first[k]
            off = gf[k] - g_first[k]
            gf[k] = _cmod(off + ext, ext) + g_first[k]
            gl[k] = gf[k] + ext_h
        out.append(Space(tuple(t[0] for t in b), tuple(t[1] for t in b), tuple(gf), tuple(gl)))
    return out


def make_pattern(g_first, g_last, halos, periodic, domains: Sequence[Domain]) -> list[list[Entry]]:
    """Receive entries per domain (structured/pattern.hpp:240-365), single process."""
    dim = len(g_first)
    recv = []
    for d in domains:
        by_src: dict[int, list[Space]] = {}
        for h in halo_boxes(d, g_first, g_last, halos, periodic):
            for e in domains:
                gf = tuple(max(h.gfirst[k], e.first[k]) for k in range(dim))
                gl = tuple(min(h.glast[k], e.last[k]) for k in range(dim))
                if all(gf[k] <= gl[k] for k in range(dim)):
                    lf = tuple(h.lfirst[k] + gf[k] - h.gfirst[k] for k in range(dim))
                    ll = tuple(h.lfirst[k] + gl[k] - h.gfirst[k] for k in range(dim))
                    by_src.setdefault(e.id, []).append(Space(lf, ll, gf, gl))
        recv.append(by_src)
    idx = {d.id: i for i, d in enumerate(domains)}
    tag = -1
    out = []
    for by_src in recv:
        entries = []
        for sid in sorted(by_src):
            tag += 1
            entries.append(Entry(idx[sid], tag, by_src[sid]))
        out.append(entries)
    return out


def make_staged_pattern(g_first, g_last, halos, periodic, domains: Sequence[Domain], lookup) -> list:
    """One (receive entries, send entries) pair per dimension (make_pattern.hpp:47-256), single
    process: per domain the entries in neighbour-id order, tags a running counter over the
    stage's receive entries, a send entry tagged as the receive entry it feeds. lookup(id,
    offset) -> neighbour id, called only where the domain has a halo on that side."""
    dim = len(g_first)
    idx = {d.id: i for i, d in enumerate(domains)}
    recv = [[{} for _ in domains] for _ in range(dim)]
    send = [[{} for _ in domains] for _ in range(dim)]
    for di, d in enumerate(domains):
        lf, ll = [0] * dim, [d.last[k] - d.first[k] for k in range(dim)]
        gf, gl = list(d.first), list(d.last)
        for i in range(dim):
            hm, hp = halos[2 * i], halos[2 * i + 1]
            has_left = hm > 0 and (periodic[i] or gf[i] - hm >= g_first[i])
            has_right = hp > 0 and (periodic[i] or gl[i] + hp <= g_last[i])

            def space(lo, hi):
                a_lf, a_ll, a_gf, a_gl = list(lf), list(ll), list(gf), list(gl)
                a_lf[i], a_ll[i] = lo, hi
                a_gf[i], a_gl[i] = gf[i] + lo - lf[i], gf[i] + hi - lf[i]
                return Space(tuple(a_lf), tuple(a_ll), tuple(a_gf), tuple(a_gl))

            def neighbour(step):
                off = [0] * dim
                off[i] = step
                return lookup(d.id, tuple(off))

            if has_left:
                recv[i][di].setdefault(neighbour(-1), []).append(space(lf[i] - hm, lf[i] - 1))
            if has_right:
                send[i][di].setdefault(neighbour(1), []).append(space(ll[i] + 1 - hm, ll[i]))
                recv[i][di].setdefault(neighbour(1), []).append(space(ll[i] + 1, ll[i] + hp))
            if has_left:
                send[i][di].setdefault(neighbour(-1), []).append(space(lf[i], lf[i] - 1 + hp))
                lf[i] -= hm
                gf[i] -= hm
            if has_right:
                ll[i] += hp
                gl[i] += hp
    stages = []
    for i in range(dim):
        tag = -1
        r_out = []
        for di in range(len(domains)):
            entries = []
            for nid in sorted(recv[i][di]):
                tag += 1
                entries.append(Entry(idx[nid], tag, recv[i][di][nid]))
            r_out.append(entries)
        s_out = []
        for di in range(len(domains)):
            entries = []
            for nid in sorted(send[i][di]):
                # an entry holding only empty spaces (zero halo width on that side) may feed no
                # receive entry; it carries nothing and keeps tag 0
                rtag = next((e.tag for e in r_out[idx[nid]] if e.neighbor == di), 0)
                entries.append(Entry(idx[nid], rtag, send[i][di][nid]))
            s_out.append(entries)
        # every receive space needs a non-empty send space of the same shape feeding it; with a
        # zero halo width on one side only, the reference's messages do not match (the receive
        # expects data the sender never packs), which is refused here
        for d, entries in enumerate(r_out):
            for en in entries:
                sent = [x for x in s_out[en.neighbor] if x.neighbor == d]
                full = [sp for x in sent for sp in x.spaces if _nonempty(sp)]
                if len(full) != len(en.spaces) or any(
                        tuple(a - b for a, b in zip(r.llast, r.lfirst)) != tuple(a - b for a, b in zip(f.llast, f.lfirst))
                        for r, f in zip(en.spaces, full)):
                    raise ValueError(f"staged pattern: what domain {domains[d].id} receives from domain "
                                     f"{domains[en.neighbor].id} does not match what that domain sends")
        stages.append((r_out, s_out))
    return stages


def _nonempty(sp: Space) -> bool:
    return all(b >= a for a, b in zip(sp.lfirst, sp.llast))


def exchange_staged(stages, domains: Sequence[Domain], fields: Sequence[np.ndarray], offsets: Sequence[tuple]) -> None:
    """The stages in order; within one, every send space is read before any receive space is
    written (pack, then unpack)."""
    dim = len(domains[0].first)
    for recv, send in stages:
        moves = []
        for d, entries in enumerate(recv):
            for en in entries:
                e = en.neighbor
                sent = next(x for x in send[e] if x.neighbor == d and x.tag == en.tag)
                # a side with a zero halo width sends an empty space, which carries nothing
                spaces = [x for x in sent.spaces if _nonempty(x)]
                for rs, ss in zip(en.spaces, spaces):
                    dlo = tuple(rs.lfirst[k] + offsets[d][k] for k in range(dim))
                    dhi = tuple(rs.llast[k] + offsets[d][k] for k in range(dim))
                    slo = tuple(ss.lfirst[k] + offsets[e][k] for k in range(dim))
                    shi = tuple(ss.llast[k] + offsets[e][k] for k in range(dim))
                    moves.append((d, _slices(dlo, dhi), fields[e][_slices(slo, shi)].copy()))
        for d, dst, vals in moves:
            fields[d][dst] = vals


def _slices(lo, hi):
    return tuple(slice(a, b + 1) for a, b in zip(lo, hi))


def exchange(pattern, domains: Sequence[Domain], fields: Sequence[np.ndarray], offsets: Sequence[tuple]) -> None:
    """Fills every halo cell of every field in place with the value of its owner."""
    for d, entries in enumerate(pattern):
        dim = len(domains[d].first)
        for en in entries:
            e = en.neighbor
            for s in en.spaces:
                dlo = tuple(s.lfirst[k] + offsets[d][k] for k in range(dim))
                dhi = tuple(s.llast[k] + offsets[d][k] for k in range(dim))
                slo = tuple(s.gfirst[k] - domains[e].first[k] + offsets[e][k] for k in range(dim))
                shi = tuple(s.glast[k] - domains[e].first[k] + offsets[e][k] for k in range(dim))
                fields[d][_slices(dlo, dhi)] = fields[e][_slices(slo, shi)]


def adjoint(pattern, domains: Sequence[Domain], grads: Sequence[np.ndarray], offsets: Sequence[tuple]) -> None:
    """Explicit transpose of exchange(): owner += halo, then halo = 0, in receive-map order.

    Within one iteration space the owner cells are distinct, so the vectorised update of a space
    is the same sequence of additions as the cell-by-cell for_loop."""
    for d, entries in enumerate(pattern):
        dim = len(domains[d].first)
        for en in entries:
            e = en.neighbor
            for s in en.spaces:
                dlo = tuple(s.lfirst[k] + offsets[d][k] for k in range(dim))
                dhi = tuple(s.llast[k] + offsets[d][k] for k in range(dim))
                slo = tuple(s.gfirst[k] - domains[e].first[k] + offsets[e][k] for k in range(dim))
                shi = tuple(s.glast[k] - domains[e].first[k] + offsets[e][k] for k in range(dim))
                ds, ss = _slices(dlo, dhi), _slices(slo, shi)
                grads[e][ss] = grads[e][ss] + grads[d][ds]
                grads[d][ds] = 0


def halo_cells(pattern) -> int:
    n = 0
    for entries in pattern:
        for en in entries:
            for s in en.spaces:
                n += int(np.prod([b - a + 1 for a, b in zip(s.lfirst, s.llast)]))
    return n
