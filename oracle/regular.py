"""Oracle for regular structured grids (test infrastructure only).

Restates, in plain Python and numpy:
  * structured::regular::halo_generator::operator()  structured/regular/halo_generator.hpp:91-146
  * halo_generator::intersect                        structured/regular/halo_generator.hpp:148-158
  * make_pattern_impl<structured grid>::apply         structured/pattern.hpp:214-365
  * the exchange: pack (structured/regular/field_descriptor.hpp:72-83, pack_kernels.hpp:66-101)
    followed by unpack (field_descriptor.hpp:85-96, pack_kernels.hpp:103-138) with the buffer
    removed — the value that lands in a halo cell is the value of the cell it was packed from.
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
