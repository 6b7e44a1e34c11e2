"""Known-answer cases of the reference's regular-grid tests, shared by the oracle tests (CPU) and the
GPU parity tests.

* simple_2d: test/structured/regular/test_simple_regular_domain.cpp:38-140 — 2-D, 8 domains of
  DIM x DIM/2 cells (DIM = 8) laid out as in make_domain (:162-168) for a 2x2 process grid with
  two domains per process, halo HALO = 3, element = the global (x, y) pair of the cell; after the
  exchange every halo cell holds the coordinate of its periodic owner, or (-1, -1) outside a
  non-periodic boundary (expected/compare/check, :97-140).
* owner check (cfg0-style): every halo cell equals the value of the cell it wraps to, NaN beyond a
  non-periodic boundary.
"""
from __future__ import annotations

import numpy as np

DIM, HALO = 8, 3


def simple_2d_domains(dims=(2, 2)):
    """(id, first, last) of the domains: ranks on a dims grid with x fastest (sim(), :470-474),
    2 domains each (make_domain, :162-168)."""
    doms = []
    for rank in range(dims[0] * dims[1]):
        cy, cx = divmod(rank, dims[0])
        for i in range(2):
            x = cx * DIM
            y = (cy * 2 + i) * (DIM // 2)
            doms.append((rank * 2 + i, (x, y), (x + DIM - 1, y + DIM // 2 - 1)))
    return doms


def simple_2d_fields(doms):
    """Fields of (x, y) int32 pairs, -1 outside the interior; shape (DIM+2H, DIM/2+2H, 2)."""
    out = []
    for _, first, _ in doms:
        a = np.full((DIM + 2 * HALO, DIM // 2 + 2 * HALO, 2), -1, dtype=np.int32)
        xs = np.arange(DIM) + first[0]
        ys = np.arange(DIM // 2) + first[1]
        a[HALO:HALO + DIM, HALO:HALO + DIM // 2, 0] = xs[:, None]
        a[HALO:HALO + DIM, HALO:HALO + DIM // 2, 1] = ys[None, :]
        out.append(a)
    return out


def _expected(coord, dim, first, last, periodic):
    """expected() of the reference test (:97-105)."""
    ext = last + 1 - first
    res = first + coord
    if first == 0 and coord < 0:
        res = dim * DIM + coord if periodic else -1
    if last == dim * DIM - 1 and coord >= ext:
        res = coord - ext if periodic else -1
    return res


def simple_2d_check(a, first, last, periodic, dims=(2, 2)):
    """check() of the reference test (:118-134): returns the list of mismatching cells."""
    bad = []
    for j in range(-HALO, DIM // 2 + HALO):
        y = _expected(j, dims[1], first[1], last[1], periodic[1])
        for i in range(-HALO, DIM + HALO):
            x = _expected(i, dims[0], first[0], last[0], periodic[0])
            ex, ey = (-1, -1) if (x == -1 or y == -1) else (x, y)
            v = a[i + HALO, j + HALO]
            if (int(v[0]), int(v[1])) != (ex, ey):
                bad.append(((i, j), (int(v[0]), int(v[1])), (ex, ey)))
    return bad


def owner_check(w, arrays, spec):
    """Every halo cell of every domain equals the value at its (periodically wrapped) owner
    coordinate, or NaN where no owner exists. Returns the number of mismatching cells."""
    dim = w.dim
    glob = {}
    off = w.offsets(spec)
    for (i, first, last), a in zip(w.domains, arrays):
        glob[i] = (first, last, a)
    bad = 0
    for (i, first, last), a in zip(w.domains, arrays):
        ext = a.shape[:dim]
        grids = np.meshgrid(*[np.arange(ext[k]) - off[k] + first[k] for k in range(dim)], indexing="ij")
        owner_vals = np.full(ext, np.nan, dtype=a.dtype)
        valid = np.ones(ext, dtype=bool)
        g = []
        for k in range(dim):
            c = grids[k]
            if w.periodic[k]:
                c = np.mod(c, w.shape[k])
            else:
                valid &= (c >= 0) & (c < w.shape[k])
            g.append(c)
        for j, (f2, l2, b) in glob.items():
            inside = valid.copy()
            for k in range(dim):
                inside &= (g[k] >= f2[k]) & (g[k] <= l2[k])
            if not inside.any():
                continue
            idx = tuple(g[k][inside] - f2[k] + off[k] for k in range(dim))
            owner_vals[inside] = b[idx]
        # compare bit patterns (NaN-aware)
        u = np.dtype(f"u{a.itemsize}")
        bad += int(np.count_nonzero(owner_vals.view(u) != np.ascontiguousarray(a).view(u)))
    return bad


# ---- staged pattern (make_staged_pattern, structured/regular/make_pattern.hpp) ------------------
def simple_2d_lookup(dims):
    """domain_lu of the reference test (:170-191): the neighbour of domain `id` at `offset`."""
    def lookup(id_, offset):
        rank = id_ // 2
        y_ = id_ - 2 * rank
        y = rank // dims[0]
        x = rank - y * dims[0]
        y = ((2 * y + y_ + offset[1]) + dims[1] * 2) % (dims[1] * 2)
        x = (x + offset[0] + dims[0]) % dims[0]
        n_rank = (y // 2) * dims[0] + x
        return 2 * n_rank + (y % 2)
    return lookup


def simple_2d_packed(doms):
    """The (x, y) int32 pairs of simple_2d_fields as one int64 per cell (x in the low half), in
    the test's layout: x fastest (layout_map<1, 0>)."""
    out = []
    for a in simple_2d_fields(doms):
        p = (a[..., 1].astype(np.int64) << 32) | (a[..., 0].astype(np.int64) & 0xFFFFFFFF)
        out.append(np.asfortranarray(p))
    return out


def pairs_view(packed: np.ndarray) -> np.ndarray:
    """The int64 cells of simple_2d_packed as an (x, y, 2) int32 array over the same memory:
    component innermost, then x, then y."""
    nx, ny = packed.shape
    buf = np.asfortranarray(packed).ravel(order="F").view(np.int32)
    return np.lib.stride_tricks.as_strided(buf, shape=(nx, ny, 2), strides=(8, 8 * nx, 4))


def staged_cases() -> dict:
    """Workloads of the staged pattern: the 2-D test case for one process (dims 1x1) and for a
    2x2 process grid, and an uneven 3-D split with asymmetric halos."""
    from ghex_b200 import workloads as W
    out = {}
    for dims in ((1, 1), (2, 2)):
        doms = simple_2d_domains(dims)
        out[f"simple_2d_{dims[0]}x{dims[1]}"] = {
            "shape": (dims[0] * DIM, dims[1] * DIM), "halos": (HALO,) * 4, "periodic": (True, True),
            "domains": doms, "lookup": simple_2d_lookup(dims), "offsets": (HALO, HALO), "dims": dims,
            "arrays": (lambda doms=doms: simple_2d_packed(doms))}
    shape, parts, halos = (20, 16, 12), (3, 2, 3), (2, 1, 1, 2, 1, 2)
    doms3 = W.regular_decomposition(shape, parts, 3)

    def arrays3():
        rng = np.random.default_rng(23)
        return [np.asfortranarray(rng.standard_normal(
            tuple(l[k] - f[k] + 1 + halos[2 * k] + halos[2 * k + 1] for k in range(3)))) for _, f, l in doms3]
    out["uneven_3d"] = {"shape": shape, "halos": halos, "periodic": (True, False, True), "domains": doms3,
                        "lookup": W.cartesian_lookup(parts), "offsets": (halos[0], halos[2], halos[4]),
                        "arrays": arrays3}
    return out



# ---- 3-D mixed element types (test/structured/regular/test_regular_domain.cpp) ---------------
MIXED_EXT = (4, 3, 2)                 # local_ext
MIXED_OFFSET = (3, 3, 3)              # offset (the largest halo)
MIXED_HALOS_1 = (0, 0, 1, 0, 1, 2)    # pattern 1: fields 1 and 3
MIXED_HALOS_2 = (2, 2, 2, 2, 2, 2)    # pattern 2: field 2


def mixed_3d_domains(ranks: int):
    """(id, first, last) of the 2 x ranks domains of parameters::parameters (:559-590): rank r
    owns domains 2r and 2r+1, x blocks 2(r%2) and 2(r%2)+1 of 4, y block r/2, one z block; the
    global box is 4 x-blocks wide whatever the number of ranks."""
    ex, ey, ez = MIXED_EXT
    doms = []
    for r in range(ranks):
        for k in range(2):
            xb = (r % 2) * 2 + k
            yb = r // 2
            doms.append((2 * r + k, (xb * ex, yb * ey, 0), ((xb + 1) * ex - 1, (yb + 1) * ey - 1, ez - 1)))
    g_last = (ex * 4 - 1, ((ranks - 1) // 2 + 1) * ey - 1, ez - 1)
    return doms, g_last


def mixed_3d_field(dom, dtype):
    """fill_values (:606-620): interior cells hold their global (x, y, z) as 3 components of the
    element type, every other cell zero; memory x fastest with the 3 components innermost (an
    array<T, 3> per cell), extents local_ext + 2 * offset."""
    _, first, _ = dom
    ext = tuple(MIXED_EXT[k] + 2 * MIXED_OFFSET[k] for k in range(3))
    buf = np.zeros((ext[2], ext[1], ext[0], 3), dtype=dtype)  # C order: z, y, x, component
    a = buf.transpose(2, 1, 0, 3)                                # indexed (x, y, z, component)
    o = MIXED_OFFSET
    for k in range(3):
        g = np.arange(MIXED_EXT[k]) + first[k]
        shape = [1, 1, 1]
        shape[k] = MIXED_EXT[k]
        a[o[0]:o[0] + MIXED_EXT[0], o[1]:o[1] + MIXED_EXT[1], o[2]:o[2] + MIXED_EXT[2], k] = g.reshape(shape)
    return a


def mixed_3d_check(a, dom, halos, ranks: int, g_last) -> int:
    """check_values (:633-690) with all dimensions periodic: every cell of the domain grown by its
    halos holds its wrapped global coordinate. With one rank the global box is not covered, and
    the reference skips the low-x halo of the even domain and the high-x halo of the odd one.
    Returns the number of mismatching cells."""
    d_id, first, last = dom
    i = d_id % 2
    hxl, hxr = halos[0], halos[1]
    if ranks == 1 and i == 0:
        hxl = 0
    if ranks == 1 and i == 1:
        hxr = 0
    bad = 0
    o = MIXED_OFFSET
    for x in range(first[0] - hxl, last[0] + hxr + 1):
        for y in range(first[1] - halos[2], last[1] + halos[3] + 1):
            for z in range(first[2] - halos[4], last[2] + halos[5] + 1):
                want = [(c % (g_last[k] + 1)) for k, c in enumerate((x, y, z))]
                v = a[x - first[0] + o[0], y - first[1] + o[1], z - first[2] + o[2]]
                if [int(t) for t in v] != want:
                    bad += 1
    return bad
