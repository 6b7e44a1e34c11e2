"""The DRAM floor of an exchange (ghexb_plan_dram_floor): the sectors a cold-cache exchange cannot
avoid reading and writing, computed by the library from its own tables, equal those computed
independently here from the oracle's exchange of address-valued arrays (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

from ghex_b200 import _capi
from ghex_b200 import workloads as W
from oracle import regular as O
from test_plan_check import regular_handles


def oracle_floor(w, sector):
    """Every field holds the byte address of each of its cells (fields laid out as regular_handles
    lays them out); after the oracle's exchange a halo cell holds its source's address."""
    base = 1 << 40
    reads, writes = [], []
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for spec in specs:
            es = np.dtype(spec.dtype).itemsize
            arrays = []
            for d in w.domains:
                ext = w.extents(d, spec)
                n = int(np.prod(ext))
                arrays.append((base + np.arange(n, dtype=np.int64) * es).reshape(ext, order="F"))
                base += ((n * es + 255) // 256) * 256
            before = [a.copy() for a in arrays]
            O.exchange(pat, doms, arrays, [w.offsets(spec)] * len(doms))
            for a, b in zip(arrays, before):
                m = a != b
                reads.append(np.stack([a[m], np.full(m.sum(), es)], 1))
                writes.append(np.stack([b[m], np.full(m.sum(), es)], 1))
    rd, wr = np.concatenate(reads), np.concatenate(writes)
    rs = np.unique(rd[:, 0] // sector)
    ws, inv = np.unique(wr[:, 0] // sector, return_inverse=True)
    wbytes = np.bincount(inv, weights=wr[:, 1])
    fill = np.setdiff1d(ws[wbytes < sector], rs)
    return (len(rs) + len(fill)) * sector, len(ws) * sector


@pytest.mark.parametrize("cfg", ["cfg0", "cfg1-small", "cfg4-small"])
@pytest.mark.parametrize("sector", [32, 64, 128])
def test_floor_matches_oracle(cfg, sector):
    w = {"cfg0": W.config0, "cfg1-small": lambda: W.config1(shape=(60, 45, 15)),
         "cfg4-small": lambda: W.config4(shape=(32, 24, 16))}[cfg]()
    ctx, keep, handles = regular_handles(w)
    arr = (C.c_void_p * len(handles))(*handles)
    r, wb = C.c_int64(), C.c_int64()
    _capi.call("ghexb_plan_dram_floor", ctx._h, arr, len(handles), sector, C.byref(r), C.byref(wb))
    assert (r.value, wb.value) == oracle_floor(w, sector)
    # the floor never falls below the algorithmic bytes' own sectors, nor above one sector per element
    halo = sum(O.halo_cells(O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), h, w.periodic,
                                           [O.Domain(i, f, l) for i, f, l in w.domains])) * len(s)
               for h, s in w.halo_groups().items())
    assert wb.value <= halo * sector


def test_floor_rejects_bad_sector():
    w = W.config0()
    ctx, keep, handles = regular_handles(w)
    arr = (C.c_void_p * len(handles))(*handles)
    r, wb = C.c_int64(), C.c_int64()
    assert _capi.lib.ghexb_plan_dram_floor(ctx._h, arr, len(handles), 48, C.byref(r), C.byref(wb)) == _capi.ERR_INVALID
    assert _capi.lib.ghexb_plan_dram_floor(ctx._h, arr, len(handles), 8, C.byref(r), C.byref(wb)) == _capi.ERR_INVALID
