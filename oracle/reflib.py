"""ctypes access to oracle/_ref/libghex_ref.so — GHEX 0.4.0's own CPU exchange and test checks
(built by oracle/ref/build.py) — test infrastructure only.

`available()` is False when the library has not been built (it is built from the reference
sources, which exist only where the reference tree is mounted; the built library travels with the
working tree).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libghex_ref.so"
_lib = None

F32, F64, I32, I64 = 0, 1, 2, 3
_CODES = {np.dtype(np.float32): F32, np.dtype(np.float64): F64, np.dtype(np.int32): I32, np.dtype(np.int64): I64}


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} has not been built (python oracle/ref/build.py)")
        _lib = C.CDLL(str(LIB))
    return _lib


def _ints(v):
    v = [int(x) for x in v]
    return (C.c_int * max(1, len(v)))(*v)


def _i64(v):
    v = [int(x) for x in v]
    return (C.c_int64 * max(1, len(v)))(*v)


def _ptrs(arrays):
    for a in arrays:
        assert a.flags["F_CONTIGUOUS"] or a.ndim == 1 or (a.ndim == 2 and a.flags["C_CONTIGUOUS"]), \
            "the reference driver expects x-fastest (Fortran-ordered) memory"
    return (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


def _check(rc):
    if rc != 0:
        buf = C.create_string_buffer(4096)
        lib().ghexref_last_error(buf, len(buf))
        raise RuntimeError(buf.value.decode())


def regular_exchange(shape, periodic_groups, domains, fields, iterations: int = 0) -> float:
    """Runs the reference's regular exchange in place.

    periodic_groups: list of (halos (2*dim), periodic (dim)) — one pattern each;
    fields: list of (group index, offsets, [array per domain]) with x-fastest arrays.
    Returns seconds per exchange over `iterations` timed exchanges (after one untimed)."""
    dim = len(shape)
    arrays, offs, exts, groups, dts = [], [], [], [], []
    for g, off, arrs in fields:
        groups.append(g)
        dts.append(_CODES[arrs[0].dtype])
        offs += list(off)
        for a in arrs:
            exts += list(a.shape[:dim])
            arrays.append(a)
    sec = C.c_double()
    _check(lib().ghexref_regular_exchange(
        dim, _ints([0] * dim), _ints([n - 1 for n in shape]), len(domains), _ints([d[0] for d in domains]),
        _ints([v for d in domains for v in d[1]]), _ints([v for d in domains for v in d[2]]), len(periodic_groups),
        _ints([h for hs, _ in periodic_groups for h in hs]), _ints([int(p) for _, ps in periodic_groups for p in ps]),
        len(fields), _ints(groups), _ints(dts), _ptrs(arrays), _ints(offs), _ints(exts), iterations, C.byref(sec)))
    return sec.value


def regular_staged_exchange(shape, halos, periodic, domains, lookup, arrays, offsets, iterations: int = 0) -> float:
    """The reference's staged pattern (make_staged_pattern) with one field, x-fastest arrays of
    one dtype, exchanged stage after stage by one communication object. lookup(id, offset) is the
    domain lookup; it is tabulated for offsets -1 and +1 along every dimension."""
    dim = len(shape)
    nbr = []
    for i_d, first, last in domains:
        for i in range(dim):
            for step in (-1, 1):
                off = [0] * dim
                off[i] = step
                h = halos[2 * i + (0 if step < 0 else 1)]
                nbr.append(int(lookup(i_d, tuple(off))) if h > 0 else -1)
    exts = [v for a in arrays for v in a.shape[:dim]]
    sec = C.c_double()
    _check(lib().ghexref_regular_staged_exchange(
        dim, _ints([0] * dim), _ints([n - 1 for n in shape]), len(domains), _ints([d[0] for d in domains]),
        _ints([v for d in domains for v in d[1]]), _ints([v for d in domains for v in d[2]]), _ints(halos),
        _ints([int(p) for p in periodic]), _i64(nbr), _CODES[arrays[0].dtype], _ptrs(arrays), _ints(offsets),
        _ints(exts), iterations, C.byref(sec)))
    return sec.value


def cubed_exchange(edge, levels, halos, domains, fields, iterations: int = 0) -> float:
    """domains: (tile, x_first, x_last, y_first, y_last); fields: list of
    (ncomp, is_vector, offsets (x, y, z), [array (x, y, z, c) per domain]), one dtype for all."""
    arrays, ncomp, vec, offs, exts = [], [], [], [], []
    for nc, isv, off, arrs in fields:
        ncomp.append(nc)
        vec.append(int(isv))
        offs += list(off)
        for a in arrs:
            exts += list(a.shape[:3])
            arrays.append(a)
    sec = C.c_double()
    _check(lib().ghexref_cubed_exchange(
        _CODES[arrays[0].dtype], edge, levels, _ints(halos), len(domains), _ints([d[0] for d in domains]),
        _ints([d[1] for d in domains]), _ints([d[2] for d in domains]), _ints([d[3] for d in domains]),
        _ints([d[4] for d in domains]), len(fields), _ints(ncomp), _ints(vec), _ptrs(arrays), _ints(offs),
        _ints(exts), iterations, C.byref(sec)))
    return sec.value


def unstructured_exchange(domains, fields, iterations: int = 0) -> float:
    """domains: (id, gids, outer_lids); fields: list of (levels, levels_first, [array per domain])
    where an array is (n,) or (n, levels) in C order (levels_first) or F order."""
    gid_off, gids, outer_off, outer = [0], [], [0], []
    for _, g, o in domains:
        gids += list(g)
        gid_off.append(len(gids))
        outer += list(o)
        outer_off.append(len(outer))
    arrays, dts, lev, lf = [], [], [], []
    for L, first, arrs in fields:
        lev.append(L)
        lf.append(int(first))
        dts.append(_CODES[arrs[0].dtype])
        arrays += arrs
    sec = C.c_double()
    ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    _check(lib().ghexref_unstructured_exchange(
        len(domains), _ints([d[0] for d in domains]), _i64(gid_off), _ints(gids), _i64(outer_off), _i64(outer),
        len(fields), _ints(dts), _ints(lev), _ints(lf), ptrs, iterations, C.byref(sec)))
    return sec.value


def unstructured_exchange_hinted(domains, halo_gids, hints, levels: int, arrays, iterations: int = 0) -> float:
    """The reference's make_pattern with a receive domain ids generator (one communication object,
    all domains): hints[k] = (owner ids, remote indices) of domain k's halo elements in the halo
    generator's order; halo_gids: the halo generator's gid list (None: all outer gids); arrays
    one (n,) or C-ordered (n, levels) array per domain, float64 or int32."""
    gid_off, gids, outer_off, outer = [0], [], [0], []
    for _, g, o in domains:
        gids += list(g)
        gid_off.append(len(gids))
        outer += list(o)
        outer_off.append(len(outer))
    hoff, hid, hrem = [0], [], []
    for ids_, rem in hints:
        hid += list(ids_)
        hrem += list(rem)
        hoff.append(len(hid))
    sec = C.c_double()
    ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    _check(lib().ghexref_unstructured_exchange_hinted(
        len(domains), _ints([d[0] for d in domains]), _i64(gid_off), _ints(gids), _i64(outer_off), _i64(outer),
        _ints(halo_gids or []), -1 if halo_gids is None else len(halo_gids), _i64(hoff), _ints(hid), _ints(hrem),
        _CODES[arrays[0].dtype], int(levels), ptrs, iterations, C.byref(sec)))
    return sec.value


def unstructured_exchange_ipr(domains, levels: int, arrays, iterations: int = 0, halo_gids=None) -> float:
    """The reference's in-place receive: one communication_object_ipr per domain, every exchange
    posted, then every handle waited on. arrays: one (n,) or C-ordered (n, levels) array per
    domain, one dtype (float32, float64 or int32); halo_gids: the halo generator's gid list
    (None: all outer gids)."""
    gid_off, gids, outer_off, outer = [0], [], [0], []
    for _, g, o in domains:
        gids += list(g)
        gid_off.append(len(gids))
        outer += list(o)
        outer_off.append(len(outer))
    for a in arrays:
        assert a.flags["C_CONTIGUOUS"], "levels-first arrays expected"
    sec = C.c_double()
    ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    _check(lib().ghexref_unstructured_exchange_ipr(
        len(domains), _ints([d[0] for d in domains]), _i64(gid_off), _ints(gids), _i64(outer_off), _i64(outer),
        _ints(halo_gids or []), -1 if halo_gids is None else len(halo_gids), _CODES[arrays[0].dtype], int(levels), ptrs,
        iterations, C.byref(sec)))
    return sec.value


def cs_check_field(data: np.ndarray, tile: int, x_first: int, y_first: int, mem_halo: int, n: int, levels: int,
                   ncomp: int, is_vector: bool, halo: int) -> int:
    """check_field of the reference's cubed-sphere test on a float32 field (x, y, z, c), x fastest:
    returns the number of failed expectations."""
    assert data.dtype == np.float32 and data.flags["F_CONTIGUOUS"]
    f = lib().ghexref_cs_check_field
    f.argtypes = [C.c_void_p] + [C.c_int] * 9
    return f(data.ctypes.data, tile, x_first, y_first, mem_halo, n, levels, ncomp, int(is_vector), halo)
