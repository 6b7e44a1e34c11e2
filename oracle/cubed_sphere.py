"""Oracle for cubed-sphere grids (test infrastructure only).

Restates, in plain Python and numpy:
  * the tile neighbour table and the affine tile transforms
    (structured/cubed_sphere/transform.hpp:41-128) — data of the cube's coordinate system;
  * cubed_sphere::halo_generator::operator() (structured/cubed_sphere/halo_generator.hpp:75-196);
  * halo_generator::intersect with the inverse transform (:225-284) inside the generic structured
    make_pattern (structured/pattern.hpp:240-365);
  * the exchange with the unpack transform: a halo cell (x, y) of a domain on tile t that lies on
    neighbour tile n receives the value at T(x, y) of that tile, component 0 negated when
    rotation[2] == -1 and component 1 when rotation[1] == -1 for vector fields, no swap
    (structured/cubed_sphere/field_descriptor.hpp:80-108,142-167);
  * the adjoint: owner += (negated) halo, halo = 0, in receive-map order.

Fields are numpy arrays indexed (x, y, z, component) of the padded memory; `offsets` are the (x, y, z)
memory coordinates of the domain's first cell.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TILE_NB = ((4, 1, 5, 2), (0, 3, 5, 2), (0, 3, 1, 4), (2, 5, 1, 4), (2, 5, 3, 0), (4, 1, 3, 0))
# (rotation, translation, offset) per direction -x, +x, -y, +y for even and odd tiles
_EVEN = (((0, -1, 1, 0), (1, 1), (-1, 0)), ((1, 0, 0, 1), (-1, 0), (0, 0)),
         ((1, 0, 0, 1), (0, 1), (0, 0)), ((0, 1, -1, 0), (-1, 1), (0, -1)))
_ODD = (((1, 0, 0, 1), (1, 0), (0, 0)), ((0, -1, 1, 0), (1, -1), (-1, 0)),
        ((0, 1, -1, 0), (1, 1), (0, -1)), ((1, 0, 0, 1), (0, -1), (0, 0)))
IDENTITY = ((1, 0, 0, 1), (0, 0), (0, 0))


def forward(tile: int, n: int):
    return (_EVEN if tile % 2 == 0 else _ODD)[n]


def inverse(tile: int, n: int):
    """The transform of the neighbour tile back towards `tile` (transform.hpp:116-128)."""
    nb = TILE_NB[tile][n]
    m = TILE_NB[nb].index(tile)
    return forward(nb, m)


def apply(tr, x, y, c):
    r, t, o = tr
    return r[0] * x + r[1] * y + t[0] * c + o[0], r[2] * x + r[3] * y + t[1] * c + o[1]


def switched(tr):
    return tr[0][0] == 0


def reversed_x(tr):
    return tr[0][1] == -1 if switched(tr) else tr[0][0] == -1


def reversed_y(tr):
    return tr[0][2] == -1 if switched(tr) else tr[0][3] == -1


@dataclass
class Domain:
    tile: int
    x: tuple  # (first, last)
    y: tuple
    levels: int

    @property
    def first(self):
        return (self.tile, self.x[0], self.y[0], 0)

    @property
    def last(self):
        return (self.tile, self.x[1], self.y[1], self.levels - 1)

    def key(self):
        """domain_id_type ordering: tile, then y_first, then x_first (domain_descriptor.hpp:52-61)."""
        return (self.tile, self.y[0], self.x[0])


@dataclass
class Space:
    lfirst: tuple
    llast: tuple
    gfirst: tuple
    glast: tuple


@dataclass
class Entry:
    neighbor: int
    tag: int
    spaces: list = field(default_factory=list)


def _isect(a, b):
    return tuple(max(p, q) for p, q in zip(a[0], b[0])), tuple(min(p, q) for p, q in zip(a[1], b[1]))


def _le(a, b):
    return all(p <= q for p, q in zip(a, b))


def halo_boxes(d: Domain, c: int, h):
    """(local box, global box) pairs of one domain (halo_generator.hpp:75-196)."""
    t = d.tile
    dom = (d.first, d.last)
    loc0 = (0, 0, 0, 0)
    loc1 = (0, d.x[1] - d.x[0], d.y[1] - d.y[0], d.levels - 1)
    tile_box = ((t, 0, 0, 0), (t, c - 1, c - 1, d.levels - 1))
    nb = []
    for axis, sign in ((1, -1), (1, 1), (2, -1), (2, 1)):
        f, l = list(tile_box[0]), list(tile_box[1])
        f[axis] += sign * c
        l[axis] += sign * c
        nb.append((tuple(f), tuple(l)))

    def mk(gf, gl):
        lf = tuple(loc0[i] + gf[i] - dom[0][i] for i in range(4))
        ll = tuple(loc1[i] + gl[i] - dom[1][i] for i in range(4))
        return (lf, ll), (gf, gl)

    f0, l0 = dom
    regions = [
        mk((t, f0[1] - h[0], f0[2] - h[2], 0), (t, l0[1] + h[1], f0[2] - 1, l0[3])),  # bottom with corners
        mk((t, f0[1] - h[0], f0[2], 0), (t, f0[1] - 1, l0[2], l0[3])),               # left
        mk((t, l0[1] + 1, f0[2], 0), (t, l0[1] + h[1], l0[2], l0[3])),               # right
        mk((t, f0[1] - h[0], l0[2] + 1, 0), (t, l0[1] + h[1], l0[2] + h[3], l0[3])),  # top with corners
    ]

    def isect2(box2, b):
        (lf, ll), (gf, gl) = box2
        g = _isect((gf, gl), b)
        nlf = tuple(lf[i] + g[0][i] - gf[i] for i in range(4))
        nll = tuple(ll[i] + g[1][i] - gl[i] for i in range(4))
        return (nlf, nll), g

    out = []
    for r in regions:
        own = isect2(r, tile_box)
        if own[1][0][1] <= own[1][1][1] and own[1][0][2] <= own[1][1][2]:
            out.append(own)
        for n in range(4):
            (lf, ll), (gf, gl) = isect2(r, nb[n])
            if not (gf[1] <= gl[1] and gf[2] <= gl[2]):
                continue
            tr = forward(t, n)
            fx, fy = apply(tr, gf[1], gf[2], c)
            lx, ly = apply(tr, gl[1], gl[2], c)
            x0, x1 = (lx, fx) if reversed_x(tr) else (fx, lx)
            y0, y1 = (ly, fy) if reversed_y(tr) else (fy, ly)
            out.append(((lf, ll), ((TILE_NB[t][n], x0, y0, gf[3]), (TILE_NB[t][n], x1, y1, gl[3]))))
    return out


def _intersect_domain(d: Domain, a, b: Domain, c: int):
    """halo_generator::intersect(d, a_local, a_global, b_global) (halo_generator.hpp:225-284); None
    when empty or on another tile."""
    (alf, all_), (agf, agl) = a
    tile = agf[0]
    if tile != b.tile:
        return None
    bg = (b.first, b.last)
    if tile != d.tile:
        g = _isect((agf, agl), bg)
        if not _le(g[0], g[1]):
            return None
        n = TILE_NB[d.tile].index(tile)
        tr = inverse(d.tile, n)
        fx, fy = apply(tr, g[0][1], g[0][2], c)
        lx, ly = apply(tr, g[1][1], g[1][2], c)
        fx, fy, lx, ly = fx - d.x[0], fy - d.y[0], lx - d.x[0], ly - d.y[0]
        lf, ll = list(alf), list(all_)
        lf[3] += g[0][3] - agf[3]
        ll[3] += g[1][3] - agl[3]
        lf[1], ll[1] = (lx, fx) if reversed_x(tr) else (fx, lx)
        lf[2], ll[2] = (ly, fy) if reversed_y(tr) else (fy, ly)
        return Space(tuple(lf), tuple(ll), g[0], g[1])
    g = _isect((agf, agl), bg)
    if not _le(g[0], g[1]):
        return None
    lf = tuple(alf[i] + g[0][i] - agf[i] for i in range(4))
    ll = tuple(all_[i] + g[1][i] - agl[i] for i in range(4))
    return Space(lf, ll, g[0], g[1])


def make_pattern(edge: int, halos, domains: list[Domain]) -> list[list[Entry]]:
    recv = []
    for d in domains:
        by = {}
        for box in halo_boxes(d, edge, halos):
            if not _le(box[0][0], box[0][1]):
                continue
            for ei, e in enumerate(domains):
                s = _intersect_domain(d, box, e, edge)
                if s is not None:
                    by.setdefault(e.key(), (ei, []))[1].append(s)
        recv.append(by)
    tag = -1
    out = []
    for by in recv:
        entries = []
        for k in sorted(by):
            tag += 1
            entries.append(Entry(by[k][0], tag, by[k][1]))
        out.append(entries)
    return out


def _space_maps(d: Domain, e: Domain, s: Space, edge: int):
    """Destination and source memory coordinates of every cell of a receive space."""
    xs = np.arange(s.lfirst[1], s.llast[1] + 1)
    ys = np.arange(s.lfirst[2], s.llast[2] + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    tr = IDENTITY
    if s.gfirst[0] != d.tile:
        tr = forward(d.tile, TILE_NB[d.tile].index(s.gfirst[0]))
    GX, GY = apply(tr, X + d.x[0], Y + d.y[0], edge)
    return X, Y, GX - e.x[0], GY - e.y[0], tr


def exchange(pattern, domains, fields, offsets, edge, is_vector=False) -> None:
    for di, entries in enumerate(pattern):
        d = domains[di]
        od = offsets[di]
        for en in entries:
            e = domains[en.neighbor]
            oe = offsets[en.neighbor]
            for s in en.spaces:
                X, Y, SX, SY, tr = _space_maps(d, e, s, edge)
                z0, z1 = s.lfirst[3], s.llast[3] + 1
                vals = fields[en.neighbor][SX + oe[0], SY + oe[1], z0 + oe[2]:z1 + oe[2], :].copy()
                if is_vector:
                    if tr[0][2] == -1:
                        vals[..., 0] = -vals[..., 0]
                    if vals.shape[-1] > 1 and tr[0][1] == -1:
                        vals[..., 1] = -vals[..., 1]
                fields[di][X + od[0], Y + od[1], z0 + od[2]:z1 + od[2], :] = vals


def adjoint(pattern, domains, grads, offsets, edge, is_vector=False) -> None:
    for di, entries in enumerate(pattern):
        d = domains[di]
        od = offsets[di]
        for en in entries:
            e = domains[en.neighbor]
            oe = offsets[en.neighbor]
            for s in en.spaces:
                X, Y, SX, SY, tr = _space_maps(d, e, s, edge)
                z0, z1 = s.lfirst[3], s.llast[3] + 1
                h = grads[di][X + od[0], Y + od[1], z0 + od[2]:z1 + od[2], :].copy()
                if is_vector:
                    if tr[0][2] == -1:
                        h[..., 0] = -h[..., 0]
                    if h.shape[-1] > 1 and tr[0][1] == -1:
                        h[..., 1] = -h[..., 1]
                idx = (SX + oe[0], SY + oe[1], slice(z0 + oe[2], z1 + oe[2]), slice(None))
                grads[en.neighbor][idx] = grads[en.neighbor][idx] + h
                grads[di][X + od[0], Y + od[1], z0 + od[2]:z1 + od[2], :] = 0
