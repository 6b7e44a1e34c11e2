"""Generates the golden fixtures of tests/golden/ from the reference.

    python tests/golden/make_golden.py --reference <GHEX source tree>   (or GHEX_REFERENCE=<tree>)

* unstructured_4domain.json — the hand-built 4-domain unstructured test case of GHEX's Python
  test (test/bindings/python/test_unstructured_domain_descriptor.py: the `domains` literal, read
  as text with ast, never imported);
* unstructured_4domain.npz — its fields (2 levels, value rank*1000 + 10*gid + level on inner
  vertices, -1 elsewhere, both storage orders) exchanged by GHEX's own code (oracle/_ref);
* cubed_sphere_test.npz — the cubed-sphere test configuration of
  test/structured/cubed_sphere/test_cubed_sphere_exchange.cpp, scalar and vector, exchanged by
  GHEX's own code;
* unstructured_ipr.json / unstructured_ipr.npz — the 4-domain case of GHEX's in-place receive
  test (make_domain_ipr, test/unstructured/unstructured_test_case.hpp, its vector literals read
  as text), initialised as its initialize_data (domain_id*10000 + gid*100 + level on inner
  vertices, 0 elsewhere) with 1 level (int32) and 2 levels (float64), exchanged by GHEX's own
  communication_object_ipr (oracle/_ref); and the same with a halo generator whose gid list
  (seeded permutation, kept in the json under "permuted_halo_gids") orders some receive lists
  against the storage order, so that the received values land on rows first + k, not on the
  receive list's rows;
* unstructured_hinted.json / unstructured_hinted.npz — the 4-domain case of GHEX's C++
  unstructured tests with its receive domain ids generator (make_domain, make_halo_gen,
  recv_domain_ids_gen and the send / receive maps of check_send_halos_indices and
  check_recv_halos_indices in test/unstructured/unstructured_test_case.hpp and
  test_user_concepts.cpp, read as text), its fields initialised as initialize_data with 1 level
  (int32) and 2 levels (float64), exchanged through make_pattern(ctx, hg, rdig, domains) by
  GHEX's own code;
* regular_staged.npz — the staged pattern (make_staged_pattern): the 2-D case of
  test/structured/regular/test_simple_regular_domain.cpp (one process: two 8x4 domains stacked
  in y, halo 3, periodic, cells holding their (x, y) coordinates, the test's domain lookup) and a
  3-D uneven 3x2x3 split with asymmetric halos, exchanged stage by stage by GHEX's own code;
* regular_small.npz — small regular cases (periodic 2x2x2 halo 1; uneven 3x3x3 with the five
  fields of the benchmark's batched case) exchanged by GHEX's own code.

Every input is seeded or analytic; the script needs the reference tree and oracle/_ref.
"""
from __future__ import annotations

import argparse
import os
import ast
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def read_domains_literal(reference: Path) -> dict:
    src = (reference / "test" / "bindings" / "python" / "test_unstructured_domain_descriptor.py").read_text()
    for node in ast.parse(src).body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == "domains" for t in node.targets):
            return ast.literal_eval(node.value)
    raise RuntimeError("no `domains` literal found")


def read_ipr_domains(reference: Path) -> dict:
    """{id: {"gids": [...], "halo_lids": [...]}} from make_domain_ipr's switch cases."""
    import re
    src = (reference / "test" / "unstructured" / "unstructured_test_case.hpp").read_text()
    body = src[src.index("make_domain_ipr(domain_id_type id)"):]
    body = body[:body.index("default:")]
    out = {}
    for m in re.finditer(r"case\s+(\d+):.*?gids\s*=\s*\{([^}]*)\}.*?halo_lids\s*=\s*\{([^}]*)\}", body, re.S):
        out[int(m.group(1))] = {"gids": [int(v) for v in m.group(2).split(",")],
                                "halo_lids": [int(v) for v in m.group(3).split(",")]}
    if len(out) != 4:
        raise RuntimeError("make_domain_ipr: expected 4 domains")
    return out


def permuted_ipr_halo(doms: dict) -> list:
    """A seeded permutation of all gids as a halo generator's list, for which every receive list
    of the in-place receive still starts at the first row of a block of halo rows received once,
    and a receive list is out of storage order."""
    from oracle import unstructured as OU
    odoms = [OU.Domain(d, doms[d]["gids"], doms[d]["halo_lids"]) for d in sorted(doms)]
    allg = sorted({g for d in doms.values() for g in d["gids"]})
    rng = np.random.default_rng(2024)
    for _ in range(10000):
        gl = [int(g) for g in rng.permutation(allg)]
        recv, _, _ = OU.make_pattern(odoms, [gl] * len(odoms))
        try:
            OU.in_place_rows(recv, odoms)
        except ValueError:
            continue
        if any(e.lids != sorted(e.lids) for entries in recv for e in entries):
            return gl
    raise RuntimeError("no permuted halo order found")


def read_hinted_case(reference: Path) -> dict:
    """Domains, receive domain ids generator tables and expected send / receive maps of the C++
    unstructured test case."""
    import re
    src = (reference / "test" / "unstructured" / "unstructured_test_case.hpp").read_text()

    def block(start, end):
        b = src[src.index(start):]
        return b[:b.index(end)]

    md = block("make_domain(domain_id_type id)", "default:")
    doms = {int(m.group(1)): {"gids": [int(v) for v in m.group(2).split(",")],
                              "halo_lids": [int(v) for v in m.group(3).split(",")]}
            for m in re.finditer(r"case\s+(\d+):.*?gids\s*=\s*\{([^}]*)\}.*?halo_lids\s*=\s*\{([^}]*)\}", md, re.S)}
    rd = block("halo operator()(const domain_descriptor_type& domain) const", "std::vector<int> ranks")
    hints = {int(m.group(1)): [[int(v) for v in m.group(2).split(",")], [int(v) for v in m.group(3).split(",")]]
             for m in re.finditer(r"case\s+(\d+):.*?domain_ids\.insert\(domain_ids\.end\(\),\s*\{([^}]*)\}\)"
                                  r".*?remote_indices\.insert\(remote_indices\.end\(\),\s*\{([^}]*)\}\)", rd, re.S)}

    def ref_maps(fn):
        b = block(f"void\n{fn}(const pattern_type& p)", "EXPECT")
        return {int(m.group(1)): {int(a): [int(v) for v in c.split(",")] for a, c in
                                  re.findall(r"domain_id_type\{(\d+)\},\s*local_indices_type\{([^}]*)\}", m.group(2))}
                for m in re.finditer(r"case\s+(\d+):(.*?)break;", b, re.S)}
    if len(doms) != 4 or len(hints) != 4:
        raise RuntimeError("unexpected test case layout")
    halo = sorted({v["gids"][l] for v in doms.values() for l in v["halo_lids"]})  # make_halo_gen
    return {"domains": doms, "hints": hints, "halo_gids": halo, "send": ref_maps("check_send_halos_indices"),
            "recv": ref_maps("check_recv_halos_indices")}


def ipr_fields(doms: dict, levels: int, dtype) -> list:
    """initialize_data of the reference's unstructured test case, levels first."""
    arrays = []
    for d in sorted(doms):
        gids, halo = doms[d]["gids"], set(doms[d]["halo_lids"])
        a = np.zeros((len(gids), levels), dtype=dtype)
        for x, g in enumerate(gids):
            if x not in halo:
                a[x] = [d * 10000 + g * 100 + l for l in range(levels)]
        arrays.append(a if levels > 1 else np.ascontiguousarray(a[:, 0]))
    return arrays


def unstructured_fields(dom: dict, rank: int, levels: int, order: str) -> np.ndarray:
    inner = set(dom["inner"])
    a = np.full((len(dom["all"]), levels), -1.0, dtype=np.float64, order=order)
    for x, gid in enumerate(dom["all"]):
        if gid in inner:
            for l in range(levels):
                a[x, l] = rank * 1000 + 10 * gid + l
    return a


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("GHEX_REFERENCE"),
                    help="GHEX source tree (default: $GHEX_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        raise SystemExit("give the GHEX source tree with --reference or GHEX_REFERENCE")
    reference = Path(a.reference)
    from oracle import reflib
    from oracle.ref import build as refbuild
    refbuild.build(str(reference))
    if not reflib.available():
        raise SystemExit("oracle/_ref is not built")

    # ---- unstructured 4-domain case
    doms = read_domains_literal(reference)
    (HERE / "unstructured_4domain.json").write_text(json.dumps({str(k): v for k, v in doms.items()}, indent=1))
    out = {}
    rdoms = [(r, doms[r]["all"], doms[r]["outer_lids"]) for r in sorted(doms)]
    for order, first in (("C", True), ("F", False)):
        fields = [unstructured_fields(doms[r], r, 2, order) for r in sorted(doms)]
        for r, f in zip(sorted(doms), fields):
            out[f"in_{order}_{r}"] = f.copy()
        reflib.unstructured_exchange(rdoms, [(2, first, fields)])
        for r, f in zip(sorted(doms), fields):
            out[f"out_{order}_{r}"] = f
    np.savez_compressed(HERE / "unstructured_4domain.npz", **out)

    # ---- in-place receive case
    idoms = read_ipr_domains(reference)
    rdoms = [(d, idoms[d]["gids"], idoms[d]["halo_lids"]) for d in sorted(idoms)]
    perm = permuted_ipr_halo(idoms)
    (HERE / "unstructured_ipr.json").write_text(json.dumps(
        {**{str(k): v for k, v in idoms.items()}, "permuted_halo_gids": perm}, indent=1))
    out = {}
    for levels, dtype in ((1, np.int32), (2, np.float64)):
        for tag, gl in (("", None), ("perm_", perm)):
            arrays = ipr_fields(idoms, levels, dtype)
            for d, x in zip(sorted(idoms), arrays):
                out[f"{tag}in_{levels}_{d}"] = x.copy()
            reflib.unstructured_exchange_ipr(rdoms, levels, arrays, halo_gids=gl)
            for d, x in zip(sorted(idoms), arrays):
                out[f"{tag}out_{levels}_{d}"] = x
    np.savez_compressed(HERE / "unstructured_ipr.npz", **out)

    # ---- receive domain ids generator
    hc = read_hinted_case(reference)
    (HERE / "unstructured_hinted.json").write_text(json.dumps(
        {k: ({str(a): b for a, b in v.items()} if isinstance(v, dict) else v) for k, v in hc.items()}, indent=1))
    hdoms = hc["domains"]
    rdoms = [(d, hdoms[d]["gids"], hdoms[d]["halo_lids"]) for d in sorted(hdoms)]
    out = {}
    for levels, dtype in ((1, np.int32), (2, np.float64)):
        arrays = ipr_fields(hdoms, levels, dtype)
        for d, x in zip(sorted(hdoms), arrays):
            out[f"in_{levels}_{d}"] = x.copy()
        reflib.unstructured_exchange_hinted(rdoms, hc["halo_gids"], [hc["hints"][d] for d in sorted(hdoms)], levels,
                                            arrays)
        for d, x in zip(sorted(hdoms), arrays):
            out[f"out_{levels}_{d}"] = x
    np.savez_compressed(HERE / "unstructured_hinted.npz", **out)

    # ---- staged regular pattern
    import regular_cases as rc
    out = {}
    for name, case in rc.staged_cases().items():
        arrays = case["arrays"]()
        for i, x in enumerate(arrays):
            out[f"{name}_in_{i}"] = x.copy(order="K")
        reflib.regular_staged_exchange(case["shape"], case["halos"], case["periodic"], case["domains"],
                                       case["lookup"], arrays, case["offsets"])
        for i, x in enumerate(arrays):
            out[f"{name}_out_{i}"] = x
    np.savez_compressed(HERE / "regular_staged.npz", **out)

    # ---- cubed sphere test configuration
    import cs_cases as cs
    out = {}
    for vec in (False, True):
        arrs = cs.fields()
        reflib.cubed_exchange(cs.EDGE, cs.LEVELS, (cs.HALO,) * 4, cs.domains(),
                              [(cs.NCOMP, vec, (cs.MEM_HALO, cs.MEM_HALO, 0), arrs)])
        for i, x in enumerate(arrs):
            out[f"{'vector' if vec else 'scalar'}_{i}"] = x
    np.savez_compressed(HERE / "cubed_sphere_test.npz", **out)

    # ---- small regular cases
    from ghex_b200 import workloads as W
    out = {}
    for name, w in (("periodic", W.RegularWorkload("16^3 2x2x2 halo 1 periodic", (16, 16, 16), (True, True, True),
                                                      W.regular_decomposition((16, 16, 16), (2, 2, 2)),
                                                      [W.FieldSpec("f64", np.float64, (1,) * 6, 7)])),
                    ("batched", W.config1(shape=(40, 30, 12)))):
        groups = list(w.halo_groups().items())
        fields = []
        for gi, (halos, specs) in enumerate(groups):
            for s in specs:
                arrs = [w.domain_array(d, s) for d in w.domains]
                fields.append((gi, w.offsets(s), arrs, s.name))
        reflib.regular_exchange(w.shape, [(h, w.periodic) for h, _ in groups], w.domains,
                                [(g, off, arrs) for g, off, arrs, _ in fields])
        for g, off, arrs, fname in fields:
            for i, x in enumerate(arrs):
                out[f"{name}_{fname}_{i}"] = x
    np.savez_compressed(HERE / "regular_small.npz", **out)
    for p in sorted(HERE.glob("*.np*")) + sorted(HERE.glob("*.json")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
