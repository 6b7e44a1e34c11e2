#!/usr/bin/env python
"""Benchmark of the batched halo exchange on B200.

Workload of the headline line: the batched structured exchange of uneven domains — global grid
400x300x96 split 3x3x3 at seeded uneven points into 27 domains, three float64 fields with halo
(3,3,3,3,0,0) and two float32 fields with halo (2,2,2,2,1,1), x fastest, periodic in y only,
splitmix64 interiors, NaN halos. One step = one exchange of all five fields of all 27 domains.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config cfg1|...]

value        effective GB/s of the batched, graph-captured exchange (algorithmic bytes = halo
             elements x sizeof(T) x (1 read + 1 write)) summed over all ranks; every timed exchange
             starts with a cold L2 (a read of an unrelated buffer of twice the L2 size runs before
             it, outside its events)
e2e          the same metric through the public API (co.exchange(...).wait()) with the fields in
             pinned host memory: every step exchanges them in place, the kernel reading the owner
             cells from host memory and writing the halo cells into it over the host interconnect
             (only the touched cells cross it); `e2e.full_copy` is the other form, every field
             copied to the device, exchanged there and copied back each step
roofline     achieved GB/s of the exchange kernel (the only kernel of the batched form) against the
             measured HBM copy bandwidth; traffic = DRAM bytes per launch from an ncu capture
cpu_baseline GHEX's own CPU exchange (single rank holding every domain, built from the reference
             sources against single-process stand-ins), timed on one host core; it also checks the
             device result bit for bit
configs      the unstructured, cubed-sphere and differentiable workloads measured the same way
             (batched and per-field forms, adjoint for the differentiable one)

--impl reference times GHEX's CPU exchange alone on all host cores (one process per core, each
exchanging its own copy of the workload) and prints the same metric.

With --gpus N > 1 (torchrun, one process per GPU) every rank runs an independent replica: the path
moves no data between GPUs.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "halo GB/s vs HBM peak & exchanges/s: batched vs per-field kernels, bit-exact"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["cfg0", "cfg1", "cfg1_staged", "cfg2", "cfg2_ipr", "cfg3", "cfg4", "cfg4_f32"],
                    default="cfg1")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the other workloads")
    ap.add_argument("--baseline-seconds", type=float, default=10.0)
    ap.add_argument("--calibrate", action="store_true",
                    help="time a plain row-copy kernel on the exchange's access pattern (rows of n elements at a row "
                         "stride) and contiguous copies, cold L2, and print one JSON line")
    ap.add_argument("--sharded", choices=["pull", "push"], default=None,
                    help="cfg1 sharded over the ranks (one per GPU, domains dealt round-robin): each rank's "
                         "kernel moves its part of the exchange through the other GPUs' memory, between two "
                         "NCCL barriers on the exchange's stream (ghex_b200.distributed); total work fixed")
    ap.add_argument("--bulk-ab", action="store_true",
                    help="time the bulk column kernel's shares of the lists against the element kernel on cfg2")
    ap.add_argument("--staged-ab", action="store_true",
                    help="time the staged (tensor-map) form against the element kernel on cfg1, cfg3 and cfg4")
    ap.add_argument("--calibrate-host", action="store_true",
                    help="the same row pattern in pinned host memory (the e2e form's access over the host "
                         "interconnect) and host<->device copies")
    ap.add_argument("--profile", choices=["batched", "per_field", "adjoint", "program"], default=None,
                    help="only run `--steps` launches of one form after `--warmup` (for ncu captures); "
                         "`program` replays the graphed differentiable program of cfg4 or cfg4_f32")
    ap.add_argument("--tuning", default=None,
                    help="the tuning of the headline workload's plan, as printed in the bench line's "
                         "roofline.traffic_tuning (e.g. k8.b128.p0.s1.st8x16384.c4.g1; a trailing .a<-1..2> sets the adjoint's "
                         "gather-tile scale), instead of the autotuner's "
                         "choice (for --profile runs and ncu launch lists, whose serialised timing would mislead the "
                         "autotuner)")
    return ap.parse_args()


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


TUNING_KEYS = ("elems_per_thread", "block", "grid", "pairs", "use_pairs", "staged_mode", "staged_boxes", "staged_items",
               "stages", "stage_bytes", "stage_consumers", "stage_ctas_per_sm", "bulk_share", "bulk_tiles")


def tuning_key(info: dict) -> str:
    """The tuning that decides a launch's kernels and their shapes, as a short string (the key of
    profiles/traffic.json)."""
    k = f"k{info['elems_per_thread']}.b{info['block']}.p{info['use_pairs']}.s{info['staged_mode']}"
    if info["staged_mode"]:
        k += f".st{info['stages']}x{info['stage_bytes']}.c{info['stage_consumers']}.g{info['stage_ctas_per_sm']}"
    if info["bulk_tiles"]:
        k += f".u{info['bulk_share']}"
    return k


def apply_tuning(plan, key: str) -> None:
    """Sets a plan to the tuning named by tuning_key(), optionally followed by `.a<scale>`, the
    adjoint's gather-tile scale (-1 to 2)."""
    parts = {}
    forward = []
    for tok in key.split("."):
        if tok.startswith("st"):
            a, b = tok[2:].split("x")
            parts["stages"], parts["stage_bytes"] = int(a), int(b)
        else:
            parts[tok[0]] = int(tok[1:])
        if not tok.startswith("a"):
            forward.append(tok)
    plan.set_tuning(parts["k"], parts["b"], parts["p"])
    plan.set_staged(parts["s"], parts.get("stages", 0), parts.get("stage_bytes", 0), parts.get("c", 0), parts.get("g", 0))
    plan.set_bulk(parts.get("u", 0))
    if "a" in parts:
        plan.set_adjoint_tuning(parts["a"])
    if tuning_key(plan.info()) != ".".join(forward):
        raise ValueError(f"tuning {key} not applied: {tuning_key(plan.info())}")


def ncu_traffic(cfg: str, key: str):
    """DRAM bytes per launch of the batched form (all its kernels) from the committed ncu summary,
    captured at this tuning; None when no capture of this tuning is committed."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            entry = json.loads(p.read_text()).get(cfg, {}).get(key)
            return entry if isinstance(entry, dict) else None
        except Exception:
            return None
    return None


def roofline_block(alg: float, ms: float, peak: float, peak_kind: str, plan, cfg: str, info: dict) -> dict:
    """Achieved algorithmic GB/s against the measured HBM copy bandwidth; beside it the DRAM floor
    of the exchange (the sectors it cannot avoid, 32-byte granularity) and, where an ncu capture of
    this tuning is committed, the measured DRAM traffic per launch."""
    achieved = alg / (ms * 1e-3) / 1e9
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "peak_source": peak_kind}
    fl = plan.dram_floor(32)
    out["floor"] = {"sector_bytes": 32, "bytes": fl["total"], "read": fl["read"], "write": fl["write"],
                    "alg_over_floor": alg / fl["total"],
                    "frac_on_floor": fl["total"] / (ms * 1e-3) / 1e9 / peak}
    # B200 fetches 128-byte lines from DRAM for these scattered reads whatever the L2 fetch
    # granularity limit says (ncu dram__bytes_read matches a 128-byte line model), and writes
    # back 32-byte sectors: the floor the hardware imposes
    fl128 = plan.dram_floor(128)
    hw = fl128["read"] + fl["write"]
    out["floor_hw"] = {"read_line_bytes": 128, "write_sector_bytes": 32, "bytes": hw, "read": fl128["read"],
                       "write": fl["write"], "alg_over_floor": alg / hw,
                       "frac_on_floor": hw / (ms * 1e-3) / 1e9 / peak}
    key = tuning_key(info)
    tr = ncu_traffic(cfg, key)
    out["traffic"] = tr["dram_bytes"] if tr else None
    out["traffic_tuning"] = key
    if tr:
        out["dram_frac"] = tr["dram_bytes"] / (ms * 1e-3) / 1e9 / peak
        out["traffic_capture"] = tr.get("capture")
    return out


# ------------------------------------------------------------------------------------------
# clocks during the timed region (NVML, read-only)
# ------------------------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index: int, period_s: float = 0.002):
        self.samples, self.reasons = [], 0
        self.period = period_s
        self._stop = threading.Event()
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.nv is not None:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv is not None:
            self.t.join()

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        reasons = [n for bit, n in self.REASONS.items() if self.reasons & bit and n != "gpu_idle"]
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------------------------------
# workloads on the host (numpy) and on the device (the drop-in API)
# ------------------------------------------------------------------------------------------
def workload(cfg: str):
    from ghex_b200 import workloads as W
    if cfg == "cfg2_ipr":
        return W.config2(halo_by_owner=True)
    if cfg == "cfg1_staged":
        return W.config1()
    if cfg == "cfg4_f32":
        return W.config4(dtype=np.float32)
    return {"cfg0": W.config0, "cfg1": W.config1, "cfg2": W.config2, "cfg3": W.config3, "cfg4": W.config4}[cfg]()


class Case:
    """One workload: host arrays, their device copies, buffer_infos and an exchange plan.
    fields: (name, host arrays, device tensors, extra) with extra = (ncomp, is_vector) for the
    cubed sphere."""

    def __init__(self, cfg: str, dev, device_index: int = 0):
        import torch
        self.cfg = cfg
        self.w = w = workload(cfg)
        self.kind = {"cfg2": "unstructured", "cfg2_ipr": "unstructured", "cfg3": "cubed_sphere"}.get(cfg, "regular")
        self.in_place = cfg == "cfg2_ipr"  # unstructured in-place receive
        self.staged = cfg == "cfg1_staged"  # one pattern per dimension, exchanged in turn
        self.stage_bis = []
        self.fields = []
        self.bis = []
        self.wrappers = []  # per field: device tensors of every domain -> their buffer_infos
        if self.kind == "regular":
            from ghex_b200 import workloads as W
            from ghex_b200.structured import regular as R
            self.api = R
            self.ctx = R.make_context(device=device_index)
            self.stage_bis = [[] for _ in range(w.dim)] if self.staged else []
            for halos, specs in w.halo_groups().items():
                hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                                     [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
                doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
                pat = R.make_pattern(self.ctx, hg, doms)
                stages = (R.make_staged_pattern(self.ctx, doms, W.cartesian_lookup(w.parts), (0,) * w.dim,
                                                tuple(n - 1 for n in w.shape), halos, w.periodic)
                          if self.staged else [])
                for s in specs:
                    host = [w.domain_array(d, s) for d in w.domains]
                    tens = [torch.from_numpy(a).to(dev) for a in host]
                    self.fields.append((s.name, host, tens, None))
                    wrap = (lambda ts, pat=pat, doms=doms, s=s: [
                        pat(R.make_field_descriptor(dm, t, w.offsets(s), w.extents(d, s)))
                        for dm, d, t in zip(doms, w.domains, ts)])
                    self.wrappers.append(wrap)
                    self.bis += wrap(tens)
                    for i, sp in enumerate(stages):
                        self.stage_bis[i] += [sp(bi.field) for bi in self.bis[-len(tens):]]
            names = sorted({np.dtype(s.dtype).name for s in w.fields}, reverse=True)
            self.dtype = "+".join(n.replace("float", "f") for n in names)
        elif self.kind == "cubed_sphere":
            from ghex_b200.structured import cubed_sphere as C
            self.api = C
            self.ctx = C.make_context(device=device_index)
            cube = C.cube(w.edge, w.levels)
            doms = [C.DomainDescriptor(cube, *b) for b in w.domains]
            pat = C.make_pattern(self.ctx, C.HaloGenerator(w.halo), doms)
            for name, nc, vec, seed in (("scalar", 1, False, 1), ("vector", 2, True, 2)):
                host = [w.domain_array(d, nc, seed) for d in w.domains]
                tens = [torch.from_numpy(a).to(dev) for a in host]
                self.fields.append((name, host, tens, (nc, vec)))
                wrap = (lambda ts, host=host, nc=nc, vec=vec: [
                    pat(C.make_field_descriptor(d, t, w.offsets(), a.shape[:3], nc, vec))
                    for d, t, a in zip(doms, ts, host)])
                self.wrappers.append(wrap)
                self.bis += wrap(tens)
            self.dtype = "f64"
        else:
            from ghex_b200 import unstructured as U
            self.api = U
            self.ctx = U.make_context(device=device_index)
            doms = [U.DomainDescriptor(*d) for d in w.domains]
            pat = U.make_pattern(self.ctx, U.HaloGenerator(), doms)
            for name, dt, seed in (("f64", np.float64, 1), ("f32", np.float32, 2)):
                host = [w.domain_array(d, dt, seed) for d in w.domains]
                tens = [torch.from_numpy(a).to(dev) for a in host]
                self.fields.append((name, host, tens, None))
                wrap = lambda ts: [pat(U.make_field_descriptor(d, t)) for d, t in zip(doms, ts)]
                self.wrappers.append(wrap)
                self.bis += wrap(tens)
            self.dtype = "f64+f32"
        for _, host, tens, _ in self.fields:
            for a, t in zip(host, tens):
                assert t.stride() == torch.from_numpy(a).stride()
        self.plan = self.api.make_exchange_plan(self.ctx, self.bis, in_place_receive=self.in_place)
        self.alg = self.plan.info()["algorithmic_bytes"]
        self.stage_plans = [self.api.make_exchange_plan(self.ctx, b) for b in self.stage_bis]

    def reset(self):
        import torch
        for _, host, tens, _ in self.fields:
            for t, a in zip(tens, host):
                t.copy_(torch.from_numpy(a))
        torch.cuda.synchronize()

    # ---- the CPU side: GHEX's own exchange where built, else the numpy restatement ---------
    def reference(self, iterations: int):
        """Exchanges copies of the host arrays on the CPU; returns (seconds per exchange over
        `iterations` timed exchanges after one untimed, the exchanged arrays, kind)."""
        from oracle import reflib
        w = self.w
        arrays = [[a.copy(order="K") for a in f[1]] for f in self.fields]
        if reflib.available():
            if self.kind == "regular":
                groups = list(w.halo_groups().items())
                gi = {h: i for i, (h, _) in enumerate(groups)}
                spec_of = {s.name: s for s in w.fields}
                fl = [(gi[spec_of[f[0]].halos], w.offsets(spec_of[f[0]]), arrs) for f, arrs in zip(self.fields, arrays)]
                sec = reflib.regular_exchange(w.shape, [(h, w.periodic) for h, _ in groups], w.domains, fl, iterations)
            elif self.kind == "cubed_sphere":
                fl = [(f[3][0], f[3][1], w.offsets(), arrs) for f, arrs in zip(self.fields, arrays)]
                sec = reflib.cubed_exchange(w.edge, w.levels, (w.halo,) * 4, w.domains, fl, iterations)
            elif self.in_place:  # one communication_object_ipr per domain and field
                sec = sum(reflib.unstructured_exchange_ipr(w.domains, w.levels, arrs, iterations) for arrs in arrays)
            else:
                sec = reflib.unstructured_exchange(w.domains, [(w.levels, True, arrs) for arrs in arrays], iterations)
            return sec, arrays, "reference"
        t0 = time.perf_counter()
        for it in range(iterations + 1):
            if it == 1:
                t0 = time.perf_counter()
            self._port_exchange(arrays)
        return (time.perf_counter() - t0) / max(1, iterations), arrays, "port"

    def _port_exchange(self, arrays):
        w = self.w
        if self.kind == "regular":
            from oracle import regular as O
            spec_of = {s.name: s for s in w.fields}
            for f, arrs in zip(self.fields, arrays):
                s = spec_of[f[0]]
                doms = [O.Domain(i, a, b) for i, a, b in w.domains]
                pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), s.halos, w.periodic, doms)
                O.exchange(pat, doms, arrs, [w.offsets(s)] * len(doms))
        elif self.kind == "cubed_sphere":
            from oracle import cubed_sphere as O
            doms = [O.Domain(t, (x0, x1), (y0, y1), w.levels) for t, x0, x1, y0, y1 in w.domains]
            pat = O.make_pattern(w.edge, (w.halo,) * 4, doms)
            for f, arrs in zip(self.fields, arrays):
                O.exchange(pat, doms, arrs, [w.offsets()] * len(doms), w.edge, f[3][1])
        else:
            from oracle import unstructured as O
            doms = [O.Domain(*d) for d in w.domains]
            recv, send, _ = O.make_pattern(doms)
            for arrs in arrays:
                if self.in_place:
                    O.exchange_in_place(recv, send, arrs, doms)
                else:
                    O.exchange(recv, send, arrs)

    def mismatches(self, expected) -> int:
        bad = 0
        for f, exp in zip(self.fields, expected):
            for t, e in zip(f[2], exp):
                got = t.cpu().numpy()
                u = np.dtype(f"u{e.itemsize}")
                bad += int(np.count_nonzero(np.ascontiguousarray(got).view(u) != np.ascontiguousarray(e).view(u)))
        return bad


# ------------------------------------------------------------------------------------------
# reference arm: GHEX's CPU exchange on all host cores
# ------------------------------------------------------------------------------------------
def _reference_worker(cfg: str, seconds: float, barrier, queue):
    """One process of the reference arm: builds its own copy of the workload, sizes its timed run
    to about `seconds` from one measured exchange, waits for every other process at `barrier` and
    then times its exchanges, so that the timed windows of all processes overlap. Puts
    (seconds per exchange, kind, exchanges, window start, window end) with wall-clock window ends."""
    try:
        from oracle import reflib
        w = workload(cfg)
        groups = list(w.halo_groups().items())
        fields = []
        for gi, (h, specs) in enumerate(groups):
            for s in specs:
                fields.append((gi, w.offsets(s), [w.domain_array(d, s) for d in w.domains]))
        if reflib.available():
            pg = [(h, w.periodic) for h, _ in groups]
            est = reflib.regular_exchange(w.shape, pg, w.domains, fields, 1)
            iters = max(2, int(np.ceil(seconds / max(est, 1e-6))))
            barrier.wait(timeout=900)
            sec = reflib.regular_exchange(w.shape, pg, w.domains, fields, iters)
            kind = "reference"
        else:
            from oracle import regular as O
            pats = []
            for h, _ in groups:
                doms = [O.Domain(i, f, l) for i, f, l in w.domains]
                pats.append((O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), h, w.periodic, doms), doms))

            def once():
                for gi, off, arrs in fields:
                    pat, doms = pats[gi]
                    O.exchange(pat, doms, arrs, [off] * len(doms))
            t0 = time.perf_counter()
            once()
            iters = max(2, int(np.ceil(seconds / max(time.perf_counter() - t0, 1e-6))))
            barrier.wait(timeout=900)
            t0 = time.perf_counter()
            for _ in range(iters):
                once()
            sec = (time.perf_counter() - t0) / iters
            kind = "port"
        end = time.time()
        queue.put((sec, kind, iters, end - sec * iters, end))
    except Exception as e:  # reported by the parent
        try:
            barrier.abort()
        except Exception:
            pass
        queue.put((None, repr(e), 0, 0.0, 0.0))


def alg_bytes_host(cfg: str) -> int:
    """Algorithmic bytes of a regular workload, from the restated pattern (no device needed)."""
    from oracle import regular as O
    w = workload(cfg)
    alg = 0
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for s in specs:
            alg += O.halo_cells(pat) * np.dtype(s.dtype).itemsize * 2
    return alg


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import multiprocessing as mp
    cfg = args.config if args.config in ("cfg0", "cfg1", "cfg4") else "cfg1"
    # one process per host core, each holding its own copy of the workload (about 0.5 GB for the
    # 400x300x96 case), as many as the free host memory allows
    procs = max(1, os.cpu_count() or 1)
    try:
        import psutil
        procs = max(1, min(procs, int(psutil.virtual_memory().available / (1.5 * 2**30))))
    except Exception:
        pass
    # every process times about `seconds` of exchanges of its own copy, all windows overlapping
    seconds = float(os.environ.get("GHEXB_REFERENCE_SECONDS", "2.0"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    barrier = ctx.Barrier(procs)
    ps = [ctx.Process(target=_reference_worker, args=(cfg, seconds, barrier, q)) for _ in range(procs)]
    for p in ps:
        p.start()
    res = [q.get() for _ in ps]
    for p in ps:
        p.join()
    good = [r for r in res if r[0]]
    if not good or len(good) < len(res):
        bad = [r for r in res if not r[0]]
        print(json.dumps({"impl": "reference", "unavailable": f"the CPU exchange failed: {bad[0][1]}"}), flush=True)
        return
    alg = alg_bytes_host(cfg)
    rates = sorted(1.0 / r[0] for r in good)  # exchanges per second of each process
    rate = sum(rates)  # all processes, their timed windows overlapping
    start, end = max(r[3] for r in good), min(r[4] for r in good)
    durations = [r[4] - r[3] for r in good]
    overlap = max(0.0, end - start) / max(durations)
    value = rate * alg / 1e9
    kind = good[0][1]
    iters = sorted(r[2] for r in good)
    sample = (f"{len(good)} processes, each timing {iters[0]}-{iters[-1]} exchanges (about {seconds:g} s, after 1 "
              f"untimed) of {cfg} on its own copy of the workload, started together at a barrier; GHEX's CPU "
              "exchange " + ("built from the reference sources (g++ -O3 -march=x86-64-v2)" if kind == "reference"
                             else "restated in numpy"))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / rate, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (seeded splitmix64)",
            "config": {"workload": workload(cfg).name},
            "exchanges_per_s": rate,
            "processes": {"count": len(good), "window_overlap": overlap,
                          "exchanges_per_s_each": {"min": rates[0], "median": float(np.median(rates)), "max": rates[-1]},
                          "seconds_each": {"min": min(durations), "max": max(durations)}},
            "cpu_baseline": {"value": value, "unit": "GB/s", "cores": len(good), "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def max_over_ranks(value: float, world: int, device) -> float:
    """The largest value over all ranks (every rank calls it at the same point)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Timer:
    """Device time of `launch` per step with CUDA events on `stream`, max over ranks.

    mode "cold" (the headline protocol): every timed step starts with a cold L2 (a read of
    `flush`, twice the L2 size, outside the events); the launch's dirty lines are written back
    during the next step's flush, outside the events.
    mode "warm": steps back to back with no flush (the steady state of repeated exchanges whose
    working set stays in L2).
    mode "writeback": as "cold", but the events also span the flush that follows the launch, and
    the time of a flush that follows a flush is subtracted: the exchange plus the write-back of
    the lines it dirtied."""

    def __init__(self, stream, flush, world, dev):
        self.stream, self.flush, self.world, self.dev = stream, flush, world, dev

    def _run(self, launch, steps, warmup, mode):
        import torch
        import torch.distributed as dist
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        flush = self.flush if mode != "warm" else None
        with torch.cuda.stream(self.stream):
            for _ in range(warmup):
                launch()
            self.stream.synchronize()
            if self.world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            for k in range(steps):
                if flush is not None:
                    flush.sum()
                ev[k][0].record(self.stream)
                launch()
                if mode == "writeback":
                    flush.sum()
                ev[k][1].record(self.stream)
            torch.cuda.synchronize()
            if self.world > 1:
                dist.barrier()
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    def __call__(self, launch, steps, warmup, mode="cold"):
        ms = self._run(launch, steps, warmup, mode)
        if mode == "writeback":
            ms -= self._run(lambda: None, steps, warmup, mode)
        return max_over_ranks(ms, self.world, self.dev)


def e2e_ms(case, stream, steps, world, dev):
    """Public API end to end, every step: pinned host fields -> device, co.exchange(...).wait(),
    device -> host. Consecutive steps alternate between two device copies of the fields (and two
    communication objects) on two streams, so that a step's device -> host copy runs on one copy
    engine while the next step's host -> device copy runs on the other."""
    import torch
    pinned = [[torch.from_numpy(a).pin_memory() for a in f[1]] for f in case.fields]
    outs = [[torch.empty_like(p).pin_memory() for p in ps] for ps in pinned]
    h2d = sum(p.numel() * p.element_size() for ps in pinned for p in ps)
    sets = []
    for k in range(2):
        tens = [f[2] for f in case.fields] if k == 0 else [[torch.empty_like(t) for t in f[2]] for f in case.fields]
        bis = [bi for wrap, ts in zip(case.wrappers, tens) for bi in wrap(ts)]
        sets.append((tens, bis, case.api.make_communication_object(case.ctx),
                     stream if k == 0 else torch.cuda.Stream(device=dev)))

    def step(it):
        tens, bis, co, s = sets[it % 2]
        with torch.cuda.stream(s):
            for ts, ps in zip(tens, pinned):
                for t, p in zip(ts, ps):
                    t.copy_(p, non_blocking=True)
            co.exchange(bis).wait()
            for ts, os_ in zip(tens, outs):
                for t, o in zip(ts, os_):
                    o.copy_(t, non_blocking=True)

    for it in range(2):
        step(it)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(sets[0][3])
    sets[1][3].wait_event(e0)
    for it in range(steps):
        step(it)
    last, other = sets[(steps - 1) % 2][3], sets[steps % 2][3]
    done = torch.cuda.Event()
    done.record(other)
    last.wait_event(done)  # e1 follows the work of both streams
    e1.record(last)
    torch.cuda.synchronize()
    return max_over_ranks(e0.elapsed_time(e1) / steps, world, dev), h2d


def e2e_host_ms(case, steps, warmup, world, dev, alloc="library"):
    """Public API end to end on host fields: the fields live in pinned host memory and every step
    is `co.exchange(...).wait()` on them; the exchange kernel reads the source cells from host
    memory and writes the halo cells into it over the host interconnect, and wait() returns when
    the halos are in host memory. Returns (ms per step, bytes read from host, bytes written to
    host, bit-exact against the device-resident exchange)."""
    import torch
    from ghex_b200 import host_empty
    host = []
    for f in case.fields:
        ts = []
        for a in f[1]:
            src = torch.from_numpy(a)
            if alloc == "library":
                # page-locked, mapped host memory from the library (cudaHostAlloc)
                t = torch.from_numpy(host_empty(a.shape, a.dtype, order="F" if a.flags["F_CONTIGUOUS"] else "C"))
            else:
                t = torch.empty_strided(tuple(src.shape), tuple(src.stride()), dtype=src.dtype, pin_memory=True)
            assert t.stride() == src.stride()
            t.copy_(src)
            ts.append(t)
        host.append(ts)
    bis = [bi for wrap, ts in zip(case.wrappers, host) for bi in wrap(ts)]
    co = case.api.make_communication_object(case.ctx)
    for _ in range(warmup):
        co.exchange(bis).wait()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        co.exchange(bis).wait()
    e1.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3 / steps
    ms = max(e0.elapsed_time(e1) / steps, wall)
    case.reset()
    case.plan.launch(case.plan.BATCHED)
    torch.cuda.synchronize()
    ok = True
    for f, hs in zip(case.fields, host):
        for h, d in zip(hs, f[2]):
            a, b = h.numpy(), d.cpu().numpy()
            u = np.dtype(f"u{a.itemsize}")
            ok = ok and np.array_equal(a.view(u), b.view(u))
    return max_over_ranks(ms, world, dev), case.alg // 2, case.alg // 2, ok


def measure_config(cfg, dev, timer, peak, steps, warmup, autotune=True, baseline=True) -> dict:
    """Batched and per-field exchange of one workload (plus the adjoint of the differentiable one)."""
    case = Case(cfg, dev, dev.index)
    plan = case.plan
    s = timer.stream.cuda_stream
    tuning = plan.autotune(repeats=20, stream=s) if autotune else plan.info()
    ms_b = timer(lambda: plan.graph_launch(s), steps, warmup)
    ms_warm = timer(lambda: plan.graph_launch(s), steps, warmup, mode="warm")
    ms_wb = timer(lambda: plan.graph_launch(s), steps, warmup, mode="writeback")
    ms_f = timer(lambda: plan.launch(plan.PER_FIELD, s), max(10, steps // 2), warmup)
    out = {"workload": case.w.name, "algorithmic_bytes": case.alg, "dtype": case.dtype,
           "batched": {"ms": ms_b, "GB/s": case.alg / ms_b / 1e6, "exchanges_per_s": 1e3 / ms_b,
                       "roofline_frac": case.alg / ms_b / 1e6 / peak},
           "l2": {"cold_ms": ms_b, "warm_ms": ms_warm, "cold_with_writeback_ms": ms_wb},
           "roofline": roofline_block(case.alg, ms_b, peak, "measured", plan, cfg, plan.info()),
           "per_field": {"ms": ms_f, "GB/s": case.alg / ms_f / 1e6, "exchanges_per_s": 1e3 / ms_f},
           "batched_vs_per_field": ms_f / ms_b,
           "tuning": {k: tuning[k] for k in TUNING_KEYS}}
    if plan.info()["staged_mode"]:
        out["staged_status"] = plan.staged_status()
    if cfg in ("cfg2", "cfg3", "cfg4", "cfg4_f32"):
        ms_a = timer(lambda: plan.adjoint(s), steps, warmup)
        out["adjoint"] = {"ms": ms_a, "vs_forward": ms_a / ms_b, "launches": plan.info()["adjoint_launches"],
                          "gather_scale": plan.info()["gather_scale"], "gather_bulk": plan.info()["gather_bulk"]}
    if baseline:
        case.reset()
        plan.launch(plan.BATCHED, s)
        sec, expected, kind = case.reference(1 if cfg in ("cfg2", "cfg2_ipr", "cfg3") else 3)
        out["bitexact"] = case.mismatches(expected) == 0
        out["cpu_baseline"] = {"value": case.alg / sec / 1e9, "unit": "GB/s", "cores": 1, "kind": kind, "ms": sec * 1e3}
    return out


def program_case(dev, dtype):
    """The 256x256x128 workload (2x2x2 domains, halo 1, periodic) as a differentiable exchange:
    (workload, DifferentiableExchange, host arrays, device fields)."""
    import torch
    from ghex_b200 import autograd as AG
    from ghex_b200 import workloads as W
    from ghex_b200.structured import regular as R
    w = W.config4(dtype=dtype)
    spec = w.fields[0]
    ctx = R.make_context(device=dev.index)
    hg = R.HaloGenerator(((0,) * 3, tuple(n - 1 for n in w.shape)), [(1, 1)] * 3, w.periodic)
    doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
    pat = R.make_pattern(ctx, hg, doms)
    host = [w.domain_array(d, spec) for d in w.domains]
    x0 = [torch.from_numpy(a).to(dev) for a in host]
    bis = [pat(R.make_field_descriptor(dm, t, w.offsets(spec), w.extents(d, spec))) for dm, d, t in zip(doms, w.domains, x0)]
    return w, AG.DifferentiableExchange(ctx, bis), host, x0


def profile_program(args, dev) -> None:
    """`--profile program`: the graphed differentiable program (10 x (exchange, 7-point update),
    forward and backward) of cfg4 (float64) or cfg4_f32, replayed `--warmup + --steps` times."""
    import torch
    from ghex_b200 import autograd as AG
    dtype = np.float32 if args.config == "cfg4_f32" else np.float64
    w, dx, _, x0 = program_case(dev, dtype)
    graphed = AG.GraphedDiffusion(dx, x0, 10, 0.1)
    for _ in range(args.warmup + args.steps):
        graphed.run(x0)
    torch.cuda.synchronize()
    print(json.dumps({"profile": "program", "config": w.name, "dtype": np.dtype(dtype).name,
                      "replays": args.warmup + args.steps}), flush=True)


def measure_program(dev, timer, dtype, steps, warmup, baseline=True) -> dict:
    """The differentiable program of the 256x256x128 workload (2x2x2 domains, halo 1, periodic): 10
    x (halo exchange, 7-point update x <- x + 0.1 L(x)), loss = sum of squares of the final
    interiors, forward and backward through torch.autograd. One timed step = the whole program,
    forward and backward (the backward runs the exchange's adjoint kernel and the stencil's
    transpose); also timed: the forward alone."""
    import torch
    from ghex_b200 import autograd as AG
    w, dx, host, x0 = program_case(dev, dtype)
    spec = w.fields[0]
    nsteps, alpha = 10, 0.1
    out = {}

    def fwd_bwd():
        leaves = [x.clone().requires_grad_(True) for x in x0]
        ys = AG.diffusion_program(dx, [l.clone() for l in leaves], nsteps, alpha)
        AG.interior_loss(ys).backward()
        out["grad"] = [l.grad for l in leaves]
        out["ys"] = ys

    def fwd():
        with torch.no_grad():
            AG.diffusion_program(dx, [x.clone() for x in x0], nsteps, alpha)

    with torch.cuda.stream(timer.stream):
        ms_fb = timer(fwd_bwd, steps, warmup)
        ms_f = timer(fwd, steps, warmup)
        fwd_bwd()
    torch.cuda.synchronize()
    # the same program and gradient replayed from one CUDA graph
    graphed = AG.GraphedDiffusion(dx, x0, nsteps, alpha)
    with torch.cuda.stream(timer.stream):
        ms_graph = timer(lambda: graphed.run(x0), steps, warmup)
        loss_g, grad_g = graphed.run(x0)
    torch.cuda.synchronize()
    loss_a = AG.interior_loss(out["ys"]).detach()

    def bits(a, b):
        return torch.equal(a.contiguous().view(torch.int64 if a.dtype == torch.float64 else torch.int32),
                           b.contiguous().view(torch.int64 if b.dtype == torch.float64 else torch.int32))
    res = {"workload": w.name + f", {nsteps} x (exchange, 7-point update), loss = sum of squares, forward + backward",
           "dtype": np.dtype(dtype).name.replace("float", "f"),
           "forward_backward_ms": ms_fb, "forward_ms": ms_f, "inner_steps": nsteps,
           "forward_backward_ms_per_inner_step": ms_fb / nsteps, "plan_pool": dx.pool_stats(),
           "graphed": {"forward_backward_ms": ms_graph, "forward_backward_ms_per_inner_step": ms_graph / nsteps,
                       "form": "GraphedDiffusion: the same kernels in one CUDA graph on fixed buffers",
                       "same_bits_as_autograd": bool(bits(loss_g, loss_a) and all(bits(g, a) for g, a in zip(grad_g, out["grad"])))}}
    if baseline:
        from oracle import regular as O
        from oracle import stencil as S
        odoms = [O.Domain(i, f, l) for i, f, l in w.domains]
        opat = O.make_pattern((0,) * 3, tuple(n - 1 for n in w.shape), spec.halos, w.periodic, odoms)
        prog = S.Program(opat, odoms, w.offsets(spec), steps=nsteps, alpha=alpha)
        ys_ref = prog.forward(host)
        g_ref = prog.gradient(host)

        def same(a, b):
            u = np.dtype(f"u{b.itemsize}")
            return np.array_equal(np.ascontiguousarray(a).view(u), np.ascontiguousarray(b).view(u))
        res["bitexact"] = all(same(y.detach().cpu().numpy(), r) for y, r in zip(out["ys"], ys_ref)) and \
            all(same(g.cpu().numpy(), r) for g, r in zip(out["grad"], g_ref))
        res["checked"] = "final fields and the gradient against the oracle's program and explicit transpose"
    return res


def measure_staged(dev, timer, peak, steps, warmup, autotune=True, baseline=True) -> dict:
    """The batched workload through staged patterns (one pattern per dimension, exchanged in
    turn: three dependent launches, no edge or corner boxes) beside the one-launch exchange."""
    case = Case("cfg1_staged", dev, dev.index)
    s = timer.stream.cuda_stream
    if autotune:
        case.plan.autotune(repeats=20, stream=s)
        for pl in case.stage_plans:
            pl.autotune(repeats=20, stream=s)
    ms_staged = timer(lambda: [pl.graph_launch(s) for pl in case.stage_plans], steps, warmup)
    ms_full = timer(lambda: case.plan.graph_launch(s), steps, warmup)
    out = {"workload": case.w.name + ", staged pattern", "algorithmic_bytes": case.alg, "dtype": case.dtype,
           "staged": {"ms": ms_staged, "GB/s": case.alg / ms_staged / 1e6, "launches": len(case.stage_plans),
                      "roofline_frac": case.alg / ms_staged / 1e6 / peak},
           "full": {"ms": ms_full, "GB/s": case.alg / ms_full / 1e6},
           "staged_vs_full": ms_staged / ms_full,
           "descriptors": {"staged": sum(pl.info()["num_descriptors"] for pl in case.stage_plans),
                           "full": case.plan.info()["num_descriptors"]}}
    if baseline:
        import torch
        case.reset()
        for pl in case.stage_plans:
            pl.launch(pl.BATCHED, s)
        torch.cuda.synchronize()
        _, expected, _ = case.reference(1)  # the full pattern's exchange: staged must equal it
        out["bitexact"] = case.mismatches(expected) == 0
    return out


def calibrate(args):
    """Access-pattern calibration: how fast a plain kernel (ghexb_calibrate_rows: the exchange
    kernel's lane mapping without its work records) moves rows of n float64 elements spaced one
    x-row of a halo field apart (stride 139 elements, 96 x 3000 rows, as the x faces of the
    400x300x96 workload), cold L2 (device) or from pinned host memory over the host interconnect
    (--calibrate-host), beside contiguous copies of the same bytes. Prints one JSON line."""
    import ctypes as C
    import torch
    from ghex_b200 import _capi
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)
    timer = Timer(stream, flush, 1, dev)
    host = args.calibrate_host
    where = ("host memory from ghex_b200.host_empty (cudaHostAlloc, mapped; torch pin_memory beside it)" if host
             else "device memory, cold L2")
    out = {"calibration": f"ghexb_calibrate_rows, rows of n float64 spaced 139 elements apart, {where}; CUDA events, "
                          "mean of the timed launches", "rows": {}}
    shape = (96, 3000, 139)
    if host:
        from ghex_b200 import host_empty
        a = torch.from_numpy(host_empty(shape, np.float64, order="C"))
        b = torch.from_numpy(host_empty(shape, np.float64, order="C"))
        a.zero_()
        b.zero_()
        ta = torch.zeros(shape, dtype=torch.float64, pin_memory=True)
        tb = torch.zeros(shape, dtype=torch.float64, pin_memory=True)
    else:
        a = torch.zeros(shape, dtype=torch.float64, device=dev)
        b = torch.zeros_like(a)
    rows = shape[0] * shape[1]
    for n in ((1, 3, 6, 12) if host else (1, 3, 8, 32, 128)):
        def launch(n=n, mode=0, x=a, y=b):
            _capi.call("ghexb_calibrate_rows", C.c_void_p(x.data_ptr() + 3 * 8), C.c_void_p(y.data_ptr()), rows, n,
                       shape[2], shape[2], 8, mode, C.c_void_p(stream.cuda_stream))
        ms = timer(launch, 5 if host else 20, 2 if host else 3)
        r = out["rows"][f"n={n}"] = {"rows": rows, "us": ms * 1e3, "rows_per_ns": rows / (ms * 1e6),
                                     "useful_GB/s": 2 * rows * n * 8 / (ms * 1e-3) / 1e9}
        if host:
            ms = timer(lambda: launch(n, 0, ta, tb), 3, 1)
            r["torch_pinned_rows_per_ns"] = rows / (ms * 1e6)
        else:
            # the halves of a copy, and the copy with the write-back of its rows inside the timing
            r["read_only_rows_per_ns"] = rows / (timer(lambda: launch(n, 1), 20, 3) * 1e6)
            r["write_only_rows_per_ns"] = rows / (timer(lambda: launch(n, 2), 20, 3) * 1e6)
            r["write_only_with_writeback_rows_per_ns"] = rows / (timer(lambda: launch(n, 2), 20, 3, mode="writeback") * 1e6)
            r["copy_with_writeback_rows_per_ns"] = rows / (timer(launch, 20, 3, mode="writeback") * 1e6)
    if host:
        x = torch.ones(64 << 20 >> 3, dtype=torch.float64, pin_memory=True)
        y = torch.empty(64 << 20 >> 3, dtype=torch.float64, device=dev)
        ms = timer(lambda: y.copy_(x, non_blocking=True), 5, 2)
        out["h2d_64MB"] = {"us": ms * 1e3, "GB/s": x.numel() * 8 / (ms * 1e-3) / 1e9}
        ms = timer(lambda: x.copy_(y, non_blocking=True), 5, 2)
        out["d2h_64MB"] = {"us": ms * 1e3, "GB/s": x.numel() * 8 / (ms * 1e-3) / 1e9}
    else:
        for mb in (8, 35, 70):
            x = torch.ones(mb * (1 << 20) // 8, dtype=torch.float64, device=dev)
            y = torch.empty_like(x)
            ms = timer(lambda: y.copy_(x), 20, 3)
            out[f"contiguous_{mb}MB"] = {"us": ms * 1e3, "GB/s (read+write)": 2 * x.numel() * 8 / (ms * 1e-3) / 1e9}
    print(json.dumps(out), flush=True)


def staged_ab(args):
    """The staged form (tensor-map loads into shared memory) against the element kernel, per
    workload: cold-L2 time of the batched graph at the element kernel's autotuned shape, then with
    the staged kernel beside it in modes 1 and 2 at several pipeline shapes. One JSON line."""
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)
    timer = Timer(stream, flush, 1, dev)
    s = stream.cuda_stream
    out = {"staged_ab": "cold-L2 CUDA-event time of the batched graph, mean of 40 launches", "configs": {}}
    for cfg in ("cfg1", "cfg3", "cfg4"):
        case = Case(cfg, dev, 0)
        plan = case.plan
        plan.autotune(repeats=20, stream=s)
        plan.set_staged(0)
        rows = []
        for mode, shape in ((0, (8, 16384, 4, 1)), (1, (8, 16384, 4, 1)), (1, (4, 16384, 4, 2)), (2, (8, 16384, 4, 1)),
                            (2, (6, 16384, 8, 1)), (2, (4, 16384, 4, 2))):
            plan.set_staged(mode, *shape)
            ms = timer(lambda: plan.graph_launch(s), 40, 5)
            info = plan.info()
            rows.append({"tuning": tuning_key(info), "us": ms * 1e3, "staged_boxes": info["staged_boxes"],
                         "staged_items": info["staged_items"], "element_tiles": info["num_tiles"],
                         "status": plan.staged_status()})
        out["configs"][cfg] = rows
        del case, plan
    print(json.dumps(out), flush=True)


def bulk_ab(args):
    """The bulk column kernel (cp.async.bulk through shared memory) against the element kernel on
    the unstructured workloads: cold-L2 time of the batched graph at the autotuned element shape
    with the bulk kernel taking 0 to 4 quarters of the lists (beside the element kernel on a second
    stream when both have work), two runs of 40 launches each. One JSON line."""
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)
    timer = Timer(stream, flush, 1, dev)
    s = stream.cuda_stream
    out = {"bulk_ab": "cold-L2 CUDA-event time of the batched graph, us, two runs of 40 launches", "configs": {}}
    for cfg in ("cfg2", "cfg2_ipr"):
        case = Case(cfg, dev, 0)
        plan = case.plan
        info = plan.autotune(repeats=20, stream=s)
        row = {"autotuned": tuning_key(info)}
        for share in (0, 1, 2, 3, 4):
            plan.set_bulk(share)
            row[f"share{share}"] = {"us": [timer(lambda: plan.graph_launch(s), 40, 5) * 1e3 for _ in range(2)],
                                    "bulk_tiles": plan.info()["bulk_tiles"], "element_tiles": plan.info()["num_tiles"]}
        row["status"] = plan.staged_status()
        out["configs"][cfg] = row
        del case, plan
    print(json.dumps(out), flush=True)


def run_sharded(args) -> None:
    """cfg1 sharded over the ranks: every rank holds the fields of its domains only; one step is a
    sharded exchange (NCCL barrier, this rank's kernel, NCCL barrier), timed with CUDA events on the
    exchange's stream after a cold-L2 read, max over ranks. Without torchrun it runs as one rank
    (every domain local, the barriers trivial)."""
    import datetime
    import socket
    import torch
    import torch.distributed as dist
    from ghex_b200 import distributed as D
    from ghex_b200.structured import regular as R
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world == 1 and "MASTER_PORT" not in os.environ:
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]), RANK="0", WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    w = workload(args.config if args.config in ("cfg0", "cfg1", "cfg4") else "cfg1")
    mine = [i for i in range(len(w.domains)) if i % world == rank]
    ctx = D.make_context(device=local)
    bis, keep, local_fields = [], [], []
    for halos, specs in w.halo_groups().items():
        hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                             [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
        doms = {i: R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains}
        pat = D.make_pattern(ctx, hg, [doms[i] for i in mine])
        keep.append(pat)
        for spec in specs:
            for i in mine:
                a = w.domain_array(w.domains[i], spec)
                t = torch.from_numpy(a).to(dev)
                fd = R.make_field_descriptor(doms[i], t, w.offsets(spec), w.extents(w.domains[i], spec))
                keep.append(fd)
                local_fields.append((spec.name, i, a, t))
                bis.append(pat(fd))
    stream = torch.cuda.Stream(device=dev)
    s = stream.cuda_stream
    plan = D.make_sharded_plan(ctx, bis, args.sharded)
    tuning = plan.info() if args.no_autotune else plan.autotune(repeats=10, stream=s)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)
    timer = Timer(stream, flush, world, dev)
    sampler = ClockSampler(dev.index)
    with sampler:
        ms = timer(lambda: plan.exchange(s), args.steps, max(3, args.warmup))
    clocks = sampler.summary()
    # the whole exchange's bytes: every rank's part
    part = torch.tensor([plan.info()["algorithmic_bytes"]], dtype=torch.float64, device=dev)
    dist.all_reduce(part)
    alg = int(part.item())
    # bit-exact against GHEX's CPU exchange (or the numpy restatement) of every domain
    for name, i, a, t in local_fields:
        t.copy_(torch.from_numpy(a))
    torch.cuda.synchronize()
    plan.exchange(s)
    torch.cuda.synchronize()
    from oracle import regular as O
    bad = 0
    for halos, specs in w.halo_groups().items():
        odoms = [O.Domain(i, f, l) for i, f, l in w.domains]
        opat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, odoms)
        for spec in specs:
            arrays = [w.domain_array(d, spec) for d in w.domains]
            O.exchange(opat, odoms, arrays, [w.offsets(spec)] * len(odoms))
            for name, i, a, t in local_fields:
                if name == spec.name:
                    e = arrays[i]
                    u = np.dtype(f"u{e.itemsize}")
                    bad += int(np.count_nonzero(np.ascontiguousarray(t.cpu().numpy()).view(u) != np.ascontiguousarray(e).view(u)))
    bad_t = torch.tensor([bad], dtype=torch.float64, device=dev)
    dist.all_reduce(bad_t)
    peak, peak_kind = peaks()
    line = {"metric": METRIC, "value": alg / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (seeded splitmix64 interiors, NaN halos)",
            "config": {"workload": w.name, "form": f"sharded exchange, {args.sharded} form: NCCL barrier, one kernel "
                       "per rank through mapped peer memory, NCCL barrier",
                       "domains": len(w.domains), "algorithmic_bytes_per_exchange": alg,
                       "l2": "cold: a read of twice the L2 size before every timed exchange, outside its events",
                       "parallelism": f"sharded x{world}", "tuning": {k: tuning[k] for k in TUNING_KEYS}},
            "exchanges_per_s": 1e3 / ms, "bitexact": int(bad_t.item()) == 0, "clocks": clocks,
            "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9 / world, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms * 1e-3) / 1e9 / world / peak, "peak_source": peak_kind,
                         "per": "GPU (the whole exchange's bytes over the GPUs)"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.release()
    del keep
    dist.barrier()
    dist.destroy_process_group()


def main():
    args = parse()
    if args.sharded:
        run_sharded(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if args.calibrate or args.calibrate_host:
        calibrate(args)
        return
    if args.staged_ab:
        staged_ab(args)
        return
    if args.bulk_ab:
        bulk_ab(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    if args.profile == "program":
        profile_program(args, dev)
        return
    case = Case(args.config, dev, local)
    plan = case.plan
    if args.profile:
        if args.tuning:
            apply_tuning(plan, args.tuning)
        else:
            plan.autotune(repeats=20)
        launch = {"batched": lambda: plan.launch(plan.BATCHED), "per_field": lambda: plan.launch(plan.PER_FIELD),
                  "adjoint": lambda: plan.adjoint()}[args.profile]
        for _ in range(args.warmup + args.steps):
            launch()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "config": case.w.name, "launches": args.warmup + args.steps,
                          "tuning": tuning_key(plan.info()), "plan": plan.info()}), flush=True)
        return
    alg = case.alg
    stream = torch.cuda.Stream(device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)
    timer = Timer(stream, flush, world, dev)
    peak, peak_kind = peaks()
    s = stream.cuda_stream
    if args.tuning:
        apply_tuning(plan, args.tuning)
        tuning = plan.info()
    else:
        tuning = plan.info() if args.no_autotune else plan.autotune(repeats=20, stream=s)

    sampler = ClockSampler(dev.index)
    with sampler:
        ms_batched = timer(lambda: plan.graph_launch(s), args.steps, max(3, args.warmup))
    clocks = sampler.summary()
    info = plan.info()
    # kernels per graph launch: the element kernel, and the staged kernel beside it when it has items
    kernels = (1 if info["num_tiles"] > 0 else 0) + (1 if info["staged_items"] > 0 else 0)
    launches = args.steps * kernels
    staged_status = plan.staged_status() if info["staged_mode"] else 0
    ms_warm = timer(lambda: plan.graph_launch(s), args.steps, max(3, args.warmup), mode="warm")
    ms_wb = timer(lambda: plan.graph_launch(s), args.steps, max(3, args.warmup), mode="writeback")
    k_small = max(10, min(args.steps, 200))
    ms_field = timer(lambda: plan.launch(plan.PER_FIELD, s), k_small, max(3, args.warmup))
    ms_box = timer(lambda: plan.launch(plan.PER_BOX, s), max(5, k_small // 4), 3)
    e2e_copy, copy_bytes = e2e_ms(case, stream, max(3, min(args.steps, 20)), world, dev)
    e2e, h2d, d2h, e2e_ok = e2e_host_ms(case, max(10, min(args.steps, 200)), max(3, args.warmup), world, dev)
    e2e_torch, _, _, e2e_torch_ok = e2e_host_ms(case, max(10, min(args.steps, 200)), max(3, args.warmup), world, dev,
                                                alloc="torch")

    achieved = alg / (ms_batched * 1e-3) / 1e9
    n_logical = len({f[0] for f in case.fields})
    line = {
        "metric": METRIC, "value": world * achieved, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": case.dtype, "data": "synthetic (seeded splitmix64 interiors, NaN halos)",
        "config": {"workload": case.w.name, "form": "batched kernel, CUDA graph", "domains": len(case.w.domains),
                   "algorithmic_bytes_per_exchange": alg,
                   "l2": "cold: a read of an unrelated buffer of twice the L2 size before every timed exchange, "
                         "outside its events",
                   "parallelism": f"replicas x{world}",
                   "tuning": {k: tuning[k] for k in TUNING_KEYS}},
        "exchanges_per_s": world * 1e3 / ms_batched,
        "per_field": {"ms_per_step": ms_field, "GB/s": world * alg / (ms_field * 1e-3) / 1e9,
                      "exchanges_per_s": world * 1e3 / ms_field, "launches_per_exchange": n_logical},
        "per_box": {"ms_per_step": ms_box, "GB/s": world * alg / (ms_box * 1e-3) / 1e9,
                    "exchanges_per_s": world * 1e3 / ms_box, "launches_per_exchange": info["num_descriptors"]},
        "batched_vs_per_field": ms_field / ms_batched,
        "roofline": roofline_block(alg, ms_batched, peak, peak_kind, plan, args.config, info),
        "l2": {"cold_ms": ms_batched, "warm_ms": ms_warm, "cold_with_writeback_ms": ms_wb,
               "warm": "steps back to back, no flush", "cold_with_writeback": "the events also span the flush after "
               "the exchange, minus a flush after a flush: the exchange plus the write-back of what it dirtied"},
        "e2e": {"value": world * alg / (e2e * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e, "bitexact": e2e_ok,
                "form": "fields in page-locked host memory from ghex_b200.host_empty (cudaHostAlloc, mapped), "
                        "co.exchange(...).wait() per step: the exchange kernel reads the source cells from host memory "
                        "and writes the halo cells into it",
                "torch_pinned": {"value": world * alg / (e2e_torch * 1e-3) / 1e9, "ms_per_step": e2e_torch,
                                 "bitexact": e2e_torch_ok, "form": "the same, fields in torch pin_memory tensors"},
                "full_copy": {"value": world * alg / (e2e_copy * 1e-3) / 1e9, "ms_per_step": e2e_copy,
                              "h2d_bytes_per_step": copy_bytes, "d2h_bytes_per_step": copy_bytes,
                              "form": "every field copied to the device, exchanged there and copied back"}},
        "gpu_launches": launches,
        "kernels_per_exchange": kernels,
        "clocks": clocks,
    }
    if info["staged_mode"]:
        line["staged_status"] = staged_status
    if rank == 0 and world == 1 and not args.no_baseline:
        case.reset()
        plan.launch(plan.BATCHED, s)
        torch.cuda.synchronize()
        est, _, _ = case.reference(1)
        iters = max(1, int(args.baseline_seconds / max(est, 1e-6)))
        sec, expected, kind = case.reference(iters)
        line["bitexact"] = case.mismatches(expected) == 0
        line["cpu_baseline"] = {
            "value": alg / sec / 1e9, "unit": "GB/s", "cores": 1, "kind": kind,
            "sample": f"{iters} timed exchanges (after 1 untimed) of the full workload by GHEX's CPU exchange "
                      + ("built from the reference sources" if kind == "reference" else "restated in numpy")
                      + ", one process, one core"}
    if rank == 0 and world == 1 and not args.no_configs:
        del case
        line["configs"] = {}
        for cfg in ("cfg2", "cfg2_ipr", "cfg3", "cfg4", "cfg4_f32"):
            if cfg != args.config:
                line["configs"][cfg] = measure_config(cfg, dev, timer, peak, min(args.steps, 200), max(3, args.warmup),
                                                      not args.no_autotune, not args.no_baseline)
        for name, dt in (("cfg4_program", np.float64), ("cfg4_f32_program", np.float32)):
            line["configs"][name] = measure_program(dev, timer, dt, min(args.steps, 50), max(3, args.warmup),
                                                    not args.no_baseline)
        line["configs"]["cfg1_staged"] = measure_staged(dev, timer, peak, min(args.steps, 200), max(3, args.warmup),
                                                        not args.no_autotune, not args.no_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
