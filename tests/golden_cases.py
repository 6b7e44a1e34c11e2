"""Loaders of the golden fixtures in tests/golden/ (made by tests/golden/make_golden.py from GHEX's
own code)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def unstructured_domains() -> dict:
    d = json.loads((GOLDEN / "unstructured_4domain.json").read_text())
    return {int(k): v for k, v in d.items()}


def unstructured_arrays() -> dict:
    with np.load(GOLDEN / "unstructured_4domain.npz") as z:
        return {k: z[k] for k in z.files}


def cubed_arrays() -> dict:
    with np.load(GOLDEN / "cubed_sphere_test.npz") as z:
        return {k: z[k] for k in z.files}


def regular_arrays() -> dict:
    with np.load(GOLDEN / "regular_small.npz") as z:
        return {k: z[k] for k in z.files}


def unstructured_check(data: np.ndarray, dom: dict, rank: int, levels: int) -> int:
    """check_field of test_unstructured_domain_descriptor.py: inner values keep
    rank*1000 + 10*gid + l, halo values equal 10*gid + l modulo 1000. Returns the mismatches."""
    inner = set(dom["inner"])
    bad = 0
    for x, gid in enumerate(dom["all"]):
        for l in range(levels):
            v = data[x, l]
            if gid in inner:
                bad += v != rank * 1000 + 10 * gid + l
            else:
                bad += (v - 1000 * int(v / 1000)) != 10 * gid + l
    return int(bad)


def ipr_case() -> tuple[dict, list]:
    """The domains of GHEX's in-place receive test ({id: {"gids", "halo_lids"}}) and the permuted
    halo generator gid list of the second case."""
    d = json.loads((GOLDEN / "unstructured_ipr.json").read_text())
    perm = d.pop("permuted_halo_gids")
    return {int(k): v for k, v in d.items()}, perm


def ipr_arrays() -> dict:
    with np.load(GOLDEN / "unstructured_ipr.npz") as z:
        return {k: z[k] for k in z.files}


def staged_arrays() -> dict:
    with np.load(GOLDEN / "regular_staged.npz") as z:
        return {k: z[k] for k in z.files}


def hinted_case() -> dict:
    """The C++ unstructured test case with its receive domain ids generator: domains, hints
    (owner ids, remote indices), the halo generator's gid list and the expected send / receive
    maps, all keyed by domain id."""
    d = json.loads((GOLDEN / "unstructured_hinted.json").read_text())
    conv = lambda m: {int(k): v for k, v in m.items()}
    return {"domains": conv(d["domains"]), "hints": conv(d["hints"]), "halo_gids": d["halo_gids"],
            "send": {int(k): conv(v) for k, v in d["send"].items()},
            "recv": {int(k): conv(v) for k, v in d["recv"].items()}}


def hinted_arrays() -> dict:
    with np.load(GOLDEN / "unstructured_hinted.npz") as z:
        return {k: z[k] for k in z.files}
