"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every input is generated here from a seed.
  * values: splitmix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number generators",
    OOPSLA 2014; the finaliser constants of Vigna's public-domain splitmix64) of the seed and a
    global linear index, mapped to [-1, 1); halos start as NaN;
  * regular grids: a global box split into a tensor product of (optionally uneven, seeded)
    intervals, one domain per cell of the product, fields padded by their halo widths and stored
    x fastest.

Arrays are numpy arrays indexed by coordinate (x, y, z[, c]) with x the fastest dimension in
memory (Fortran order), index 0 being the first cell of the padded memory.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, index: np.ndarray) -> np.ndarray:
    """The splitmix64 output for state seed + (index + 1) * golden gamma (uint64 arithmetic)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + (np.asarray(index, dtype=np.uint64) + np.uint64(1)) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def unit_values(seed: int, index: np.ndarray) -> np.ndarray:
    """splitmix64 mapped to [-1, 1): the top 53 bits as a fraction, times 2, minus 1."""
    z = splitmix64(seed, index)
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def uneven_splits(n: int, parts: int, rng: np.random.Generator, lo: float = 0.5, hi: float = 1.5) -> list[tuple[int, int]]:
    """Split [0, n) into `parts` intervals whose lengths lie within [lo, hi] x the mean."""
    mean = n / parts
    for _ in range(10000):
        w = rng.uniform(lo, hi, size=parts)
        lengths = np.floor(w / w.sum() * n).astype(int)
        lengths[-1] = n - lengths[:-1].sum()
        if np.all(lengths >= int(np.ceil(lo * mean))) and np.all(lengths <= int(np.floor(hi * mean))):
            break
    else:  # pragma: no cover - the bounds above always admit a solution for parts >= 1
        raise RuntimeError("could not draw an uneven split")
    out, s = [], 0
    for L in lengths:
        out.append((s, s + int(L) - 1))
        s += int(L)
    return out


def even_splits(n: int, parts: int) -> list[tuple[int, int]]:
    base, rem = divmod(n, parts)
    out, s = [], 0
    for p in range(parts):
        L = base + (1 if p < rem else 0)
        out.append((s, s + L - 1))
        s += L
    return out


@dataclass
class FieldSpec:
    name: str
    dtype: type
    halos: tuple          # (x-, x+, y-, y+, z-, z+)
    seed: int


@dataclass
class RegularWorkload:
    name: str
    shape: tuple                       # global cells per dimension
    periodic: tuple
    domains: list                      # (id, first, last) with inclusive global coordinates
    fields: list = field(default_factory=list)

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def parts(self) -> tuple:
        """Blocks per dimension of the tensor-product split."""
        return tuple(len({d[1][k] for d in self.domains}) for k in range(self.dim))

    def halo_groups(self) -> dict:
        """Fields grouped by halo widths (one pattern per group)."""
        groups: dict = {}
        for f in self.fields:
            groups.setdefault(f.halos, []).append(f)
        return groups

    def extents(self, dom, spec: FieldSpec) -> tuple:
        _, first, last = dom
        return tuple(last[k] - first[k] + 1 + spec.halos[2 * k] + spec.halos[2 * k + 1] for k in range(self.dim))

    def offsets(self, spec: FieldSpec) -> tuple:
        return tuple(spec.halos[2 * k] for k in range(self.dim))

    def domain_array(self, dom, spec: FieldSpec) -> np.ndarray:
        """Interior = splitmix64(seed, global linear index) in [-1, 1), halo = NaN; x fastest."""
        _, first, last = dom
        ext = self.extents(dom, spec)
        off = self.offsets(spec)
        a = np.full(ext, np.nan, dtype=spec.dtype, order="F")
        grids = np.meshgrid(*[np.arange(first[k], last[k] + 1, dtype=np.int64) for k in range(self.dim)], indexing="ij")
        lin = np.zeros(grids[0].shape, dtype=np.int64)
        stride = 1
        for k in range(self.dim):
            lin += grids[k] * stride
            stride *= self.shape[k]
        vals = unit_values(spec.seed, lin).astype(spec.dtype)
        a[tuple(slice(off[k], off[k] + last[k] - first[k] + 1) for k in range(self.dim))] = vals
        return a


def regular_decomposition(shape: Sequence[int], parts: Sequence[int], seed: int | None = None) -> list:
    """Domains of a tensor-product split, ids in x-fastest order."""
    rng = np.random.default_rng(seed) if seed is not None else None
    splits = [uneven_splits(n, p, rng) if rng is not None else even_splits(n, p) for n, p in zip(shape, parts)]
    doms = []
    for idx, combo in enumerate(np.ndindex(*reversed(parts))):
        c = tuple(reversed(combo))
        first = tuple(splits[k][c[k]][0] for k in range(len(shape)))
        last = tuple(splits[k][c[k]][1] for k in range(len(shape)))
        doms.append((idx, first, last))
    return doms


def cartesian_lookup(parts: Sequence[int]):
    """Domain lookup of a regular_decomposition (ids in x-fastest order), periodic in every
    dimension: lookup(id, offset) is the id of the domain `offset` blocks away."""
    dim = len(parts)

    def lookup(i: int, offset) -> int:
        c, r = [], i
        for k in range(dim):
            c.append(r % parts[k])
            r //= parts[k]
        n, stride = 0, 1
        for k in range(dim):
            n += ((c[k] + offset[k]) % parts[k]) * stride
            stride *= parts[k]
        return n

    return lookup


def config0(seed: int = 42) -> RegularWorkload:
    """64^3 float64 split 2x2x2, halo 1 on all sides, periodic in x, y and z."""
    w = RegularWorkload("cfg0: 64^3 f64, 2x2x2, halo 1, periodic xyz", (64, 64, 64), (True, True, True),
                        regular_decomposition((64, 64, 64), (2, 2, 2)))
    w.fields = [FieldSpec("f64", np.float64, (1, 1, 1, 1, 1, 1), seed)]
    return w


def config1(seed: int = 42, shape=(400, 300, 96)) -> RegularWorkload:
    """400x300x96 split 3x3x3 at seeded uneven points; 3 float64 fields with halo (3,3,3,3,0,0)
    and 2 float32 fields with halo (2,2,2,2,1,1); periodic in y only."""
    w = RegularWorkload(f"cfg1: {shape[0]}x{shape[1]}x{shape[2]} uneven 3x3x3, 3 f64 (3,3,3,3,0,0) + 2 f32 (2,2,2,2,1,1), periodic y",
                        tuple(shape), (False, True, False), regular_decomposition(shape, (3, 3, 3), seed))
    w.fields = [FieldSpec(f"f64_{i}", np.float64, (3, 3, 3, 3, 0, 0), seed + 1 + i) for i in range(3)] + \
               [FieldSpec(f"f32_{i}", np.float32, (2, 2, 2, 2, 1, 1), seed + 11 + i) for i in range(2)]
    return w


def config4(seed: int = 42, dtype=np.float64, shape=(256, 256, 128)) -> RegularWorkload:
    """256x256x128 split 2x2x2, halo 1, periodic (the differentiable stencil program)."""
    w = RegularWorkload(f"cfg4: {shape[0]}x{shape[1]}x{shape[2]} 2x2x2 halo 1 periodic", tuple(shape), (True, True, True),
                        regular_decomposition(shape, (2, 2, 2)))
    w.fields = [FieldSpec("x", dtype, (1, 1, 1, 1, 1, 1), seed)]
    return w


# ---------------------------------------------------------------------------------------------
# cubed sphere
# ---------------------------------------------------------------------------------------------
# Face orientation of the cube: the outward normal and the directions of increasing x and y of
# each tile, chosen so that neighbouring tiles share edges as in the tile table of the
# cubed-sphere transforms. Only the smoothness of the synthetic values depends on it.
_FACES = (((1, 0, 0), (0, 1, 0), (0, 0, 1)), ((0, 1, 0), (-1, 0, 0), (0, 0, 1)), ((0, 0, 1), (0, 1, 0), (-1, 0, 0)),
          ((-1, 0, 0), (0, 0, 1), (0, 1, 0)), ((0, -1, 0), (0, 0, 1), (1, 0, 0)), ((0, 0, -1), (1, 0, 0), (0, 1, 0)))


@dataclass
class CubedSphereWorkload:
    name: str
    edge: int
    levels: int
    halo: int
    domains: list      # (tile, x_first, x_last, y_first, y_last)
    seed: int

    def extents(self, dom) -> tuple:
        _, x0, x1, y0, y1 = dom
        return (x1 - x0 + 1 + 2 * self.halo, y1 - y0 + 1 + 2 * self.halo, self.levels)

    def offsets(self) -> tuple:
        return (self.halo, self.halo, 0)

    def cell_centres(self, dom):
        """Unit-sphere points of the domain's cell centres, shape (nx, ny, 3)."""
        t, x0, x1, y0, y1 = dom
        n, ex, ey = (np.array(v, dtype=np.float64) for v in _FACES[t])
        a = -1.0 + (np.arange(x0, x1 + 1) + 0.5) * 2.0 / self.edge
        b = -1.0 + (np.arange(y0, y1 + 1) + 0.5) * 2.0 / self.edge
        A, B = np.meshgrid(a, b, indexing="ij")
        p = n[None, None, :] + A[..., None] * ex[None, None, :] + B[..., None] * ey[None, None, :]
        return p / np.linalg.norm(p, axis=-1, keepdims=True)

    def domain_array(self, dom, ncomp: int, field_seed: int) -> np.ndarray:
        """(x, y, z, c) memory, x fastest: interior = low-order spherical harmonics of the cell
        centres (different per component and level) + 1e-3 seeded uniform noise; halos NaN."""
        t, x0, x1, y0, y1 = dom
        nx, ny = x1 - x0 + 1, y1 - y0 + 1
        h = self.halo
        a = np.full(self.extents(dom) + (ncomp,), np.nan, dtype=np.float64, order="F")
        p = self.cell_centres(dom)
        X, Y, Z = p[..., 0], p[..., 1], p[..., 2]
        rng = np.random.default_rng([self.seed, field_seed, t, x0, y0])
        lev = np.arange(self.levels, dtype=np.float64)[None, None, :]
        for c in range(ncomp):
            base = [1.0 + 0.5 * Z + 0.3 * X * Y + 0.2 * (3 * Z * Z - 1),   # s / u
                    0.4 * X - 0.6 * Y + 0.25 * X * Z,                       # v
                    0.7 * Y * Z - 0.1 * (X * X - Y * Y)][c % 3]
            vals = base[..., None] * (1.0 + 0.01 * lev) + 1e-3 * rng.uniform(-1.0, 1.0, size=(nx, ny, self.levels))
            a[h:h + nx, h:h + ny, :, c] = vals
        return a


def config3(seed: int = 42, edge: int = 384, levels: int = 90, split: int = 2, halo: int = 3) -> CubedSphereWorkload:
    """6 tiles of edge x edge cells, `levels` levels, every tile split split x split, halo 3."""
    step = edge // split
    doms = [(t, i * step, (i + 1) * step - 1, j * step, (j + 1) * step - 1)
            for t in range(6) for j in range(split) for i in range(split)]
    return CubedSphereWorkload(f"cfg3: cubed sphere 6x{edge}^2x{levels}, {split}x{split} per tile, halo {halo}, "
                               f"f64 scalar + f64 vector (u,v)", edge, levels, halo, doms, seed)


# ---------------------------------------------------------------------------------------------
# unstructured: periodic triangulated lattice partitioned by recursive coordinate bisection
# ---------------------------------------------------------------------------------------------
# the six neighbours of a vertex of a triangulated lattice (each quad split along (i,j)-(i+1,j+1))
LATTICE_NEIGHBOURS = ((1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1))


def rcb(x: np.ndarray, y: np.ndarray, parts: int) -> np.ndarray:
    """Recursive coordinate bisection: the part of every point; each level halves every part at
    the median of its longer coordinate extent (parts must be a power of two)."""
    part = np.zeros(x.size, dtype=np.int32)
    groups = [np.arange(x.size)]
    while len(groups) < parts:
        nxt = []
        for g in groups:
            gx, gy = x[g], y[g]
            c = gx if (gx.max() - gx.min()) >= (gy.max() - gy.min()) else gy
            order = np.argsort(c, kind="stable")
            half = g.size // 2
            nxt += [g[order[:half]], g[order[half:]]]
        groups = nxt
    for p, g in enumerate(groups):
        part[g] = p
    return part


@dataclass
class UnstructuredWorkload:
    name: str
    levels: int
    domains: list  # (id, gids (int64), outer_lids (int64))
    seed: int

    def domain_array(self, dom, dtype, field_seed: int, levels_first: bool = True) -> np.ndarray:
        """(n, levels): inner vertex rows = splitmix64(seed, gid*levels + level) in [-1, 1), halo
        rows NaN; levels contiguous (C order) when levels_first, else vertices contiguous."""
        _, gids, outer = dom
        n = gids.size
        a = np.full((n, self.levels), np.nan, dtype=dtype, order="C" if levels_first else "F")
        inner = np.ones(n, dtype=bool)
        inner[outer] = False
        idx = gids[inner][:, None].astype(np.int64) * self.levels + np.arange(self.levels)[None, :]
        a[inner] = unit_values(self.seed * 1000003 + field_seed, idx).astype(dtype)
        return a


def config2(seed: int = 42, ni: int = 1024, nj: int = 2048, parts: int = 16, levels: int = 64,
            halo_by_owner: bool = False) -> UnstructuredWorkload:
    """A periodic ni x nj triangulated lattice, vertex ids permuted by the seed, coordinates
    jittered by uniform +-0.3 cell, partitioned into `parts` domains by recursive coordinate
    bisection; every domain stores its inner vertices (ascending lattice index) followed by its
    1-ring halo (ascending gid; with halo_by_owner, grouped by owning domain first, as an
    in-place receive needs)."""
    rng = np.random.default_rng(seed)
    n = ni * nj
    perm = rng.permutation(n).astype(np.int64)
    i = np.repeat(np.arange(ni), nj)
    j = np.tile(np.arange(nj), ni)
    x = i + rng.uniform(-0.3, 0.3, size=n)
    y = j + rng.uniform(-0.3, 0.3, size=n)
    part = rcb(x, y, parts)
    halo_of = [[] for _ in range(parts)]
    for di, dj in LATTICE_NEIGHBOURS:
        nb = ((i + di) % ni) * nj + (j + dj) % nj
        cut = part[nb] != part
        src_part, nbv = part[cut], nb[cut]
        order = np.argsort(src_part, kind="stable")
        src_part, nbv = src_part[order], nbv[order]
        bounds = np.searchsorted(src_part, np.arange(parts + 1))
        for p in range(parts):
            halo_of[p].append(nbv[bounds[p]:bounds[p + 1]])
    doms = []
    for p in range(parts):
        inner = np.nonzero(part == p)[0]
        halo = np.unique(np.concatenate(halo_of[p]))
        hg = perm[halo]
        if halo_by_owner:
            hg = hg[np.lexsort((hg, part[halo]))]
        else:
            hg = np.sort(hg)
        gids = np.concatenate([perm[inner], hg])
        outer = np.arange(inner.size, gids.size, dtype=np.int64)
        doms.append((p, gids, outer))
    order = ", halos grouped by owner" if halo_by_owner else ""
    return UnstructuredWorkload(f"cfg2: periodic triangulated lattice {ni}x{nj} ({n} vertices), RCB into {parts} "
                                f"domains, 1-ring halos{order}, {levels} levels", levels, doms, seed)
