"""The configuration of the reference's cubed-sphere exchange test
(test/structured/cubed_sphere/test_cubed_sphere_exchange.cpp:846-990): cube edge 10, 6 levels,
every tile split into 2x2 domains of 5x5, halo 2, memory padded for 3, 8 float components,
interior value 100000*(tile+1) + 10000*id + 1000*c + 100*x + 10*y + z, everything else -1."""
from __future__ import annotations

import numpy as np

EDGE, LEVELS, HALO, MEM_HALO, N, NCOMP = 10, 6, 2, 3, 5, 8
EXT = N + 2 * MEM_HALO


def id_to_int(x_first, y_first):
    """id_to_int of the reference test (:102-108)."""
    if x_first == 0 and y_first == 0:
        return 0
    if y_first == 0:
        return 1
    if x_first == 0:
        return 2
    return 3


def domains():
    """(tile, x_first, x_last, y_first, y_last) in the test's order per tile."""
    out = []
    for t in range(6):
        for (x0, y0) in ((0, 0), (5, 0), (0, 5), (5, 5)):
            out.append((t, x0, x0 + 4, y0, y0 + 4))
    return out


def fields(ncomp=NCOMP):
    """Field memory (x, y, z, c), x fastest, float32."""
    out = []
    for (t, x0, _, y0, _) in domains():
        a = np.full((EXT, EXT, LEVELS, ncomp), -1, dtype=np.float32, order="F")
        x = np.arange(N)[:, None, None, None]
        y = np.arange(N)[None, :, None, None]
        z = np.arange(LEVELS)[None, None, :, None]
        c = np.arange(ncomp)[None, None, None, :]
        a[MEM_HALO:MEM_HALO + N, MEM_HALO:MEM_HALO + N, :, :] = (
            100000 * (t + 1) + 10000 * id_to_int(x0, y0) + 1000 * c + 100 * x + 10 * y + z)
        out.append(a)
    return out
