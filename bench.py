#!/usr/bin/env python
"""Benchmark of the batched halo exchange on B200.

Workload (N = 1 line): the batched structured exchange of uneven domains — global grid
400x300x96 split 3x3x3 at seeded uneven points into 27 domains, three float64 fields with halo
(3,3,3,3,0,0) and two float32 fields with halo (2,2,2,2,1,1), x fastest, periodic in y only,
splitmix64 interiors, NaN halos. One step = one exchange of all five fields of all 27 domains.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config cfg1|cfg0|cfg4]

value      effective GB/s of the batched, graph-captured exchange (algorithmic bytes = halo cells x
           sizeof(T) x (1 read + 1 write)) summed over all ranks; every timed exchange starts with a
           cold L2 (a 2 x L2 read of an unrelated buffer runs before it, outside its events)
e2e        the same metric through the public API with the fields in pinned host memory:
           host->device copy of every field, co.exchange(...).wait(), device->host copy back
roofline   achieved GB/s of the exchange kernel (the only kernel of the batched form) against the
           measured HBM copy bandwidth
With --gpus N > 1 (torchrun, one process per GPU) every rank runs an independent replica of the
workload: the path moves no data between GPUs.
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
    ap.add_argument("--config", choices=["cfg0", "cfg1", "cfg4"], default="cfg1")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--baseline-seconds", type=float, default=10.0)
    ap.add_argument("--profile", choices=["batched", "per_field", "adjoint"], default=None,
                    help="only run `--steps` launches of one form after `--warmup` (for ncu captures)")
    return ap.parse_args()


def workload(cfg: str):
    from ghex_b200 import workloads as W
    return {"cfg0": W.config0, "cfg1": W.config1, "cfg4": W.config4}[cfg]()


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(cfg: str):
    """DRAM bytes per launch of the exchange kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get(cfg)
        except Exception:
            return None
    return None


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
# CPU baseline: the oracle restatement of the reference's exchange, timed on the host
# ------------------------------------------------------------------------------------------
def _oracle_worker(cfg: str, seconds: float, queue):
    from oracle import regular as O
    w = workload(cfg)
    groups = []
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        groups.append((pat, doms, [([w.domain_array(d, s) for d in w.domains], w.offsets(s)) for s in specs]))
    n = 0
    t0 = time.perf_counter()
    while True:
        for pat, doms, fields in groups:
            for arrays, off in fields:
                O.exchange(pat, doms, arrays, [off] * len(doms))
        n += 1
        if time.perf_counter() - t0 >= seconds:
            break
    queue.put((n, time.perf_counter() - t0))


def cpu_baseline(cfg: str, alg_bytes: int, seconds: float, processes: int = 1) -> dict:
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_oracle_worker, args=(cfg, seconds, q)) for _ in range(processes)]
    for p in procs:
        p.start()
    res = [q.get() for _ in procs]
    for p in procs:
        p.join()
    rate = sum(n / t for n, t in res)  # exchanges per second, all processes
    return {"value": rate * alg_bytes / 1e9, "unit": "GB/s", "cores": processes, "kind": "port",
            "sample": f"{sum(n for n, _ in res)} exchanges of {cfg} by the numpy oracle "
                      f"({processes} process(es), {seconds:.0f} s each)",
            "exchanges_per_s": rate}


# ------------------------------------------------------------------------------------------
# reference arm
# ------------------------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args.config)
    from oracle import regular as O
    alg = 0
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for s in specs:
            alg += O.halo_cells(pat) * np.dtype(s.dtype).itemsize * 2
    procs = min(os.cpu_count() or 1, 16)
    per_step = max(1.0, 30.0 / max(1, args.steps + args.warmup))
    b = cpu_baseline(args.config, alg, seconds=per_step * args.steps, processes=procs)
    line = {"impl": "reference", "metric": METRIC, "value": b["value"], "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / b["exchanges_per_s"] * procs,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
            "data": "synthetic (seeded splitmix64)", "config": {"workload": w.name},
            "cpu_baseline": {k: b[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": b["value"], "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
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

    from ghex_b200.structured import regular as R
    sys.path.insert(0, str(ROOT / "tests"))

    w = workload(args.config)
    ctx = R.make_context(device=local)
    host, tens, bis = {}, {}, []
    for halos, specs in w.halo_groups().items():
        hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                             [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
        doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
        pat = R.make_pattern(ctx, hg, doms)
        for s in specs:
            host[s.name] = [w.domain_array(d, s) for d in w.domains]
            tens[s.name] = [torch.from_numpy(a).to(dev) for a in host[s.name]]
            bis += [pat(R.make_field_descriptor(dm, t, w.offsets(s), w.extents(d, s)))
                    for dm, d, t in zip(doms, w.domains, tens[s.name])]
    plan = R.make_exchange_plan(ctx, bis)
    if args.profile:
        launch = {"batched": lambda: plan.launch(plan.BATCHED), "per_field": lambda: plan.launch(plan.PER_FIELD),
                  "adjoint": lambda: plan.adjoint()}[args.profile]
        for _ in range(args.warmup + args.steps):
            launch()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "config": w.name, "launches": args.warmup + args.steps,
                          "plan": plan.info()}), flush=True)
        return
    tuning = plan.info() if args.no_autotune else plan.autotune(repeats=5)
    info = plan.info()
    alg = info["algorithmic_bytes"]
    stream = torch.cuda.Stream(device=dev)
    l2 = torch.cuda.get_device_properties(dev).L2_cache_size
    flush = torch.ones(max(2 * l2, 64 << 20) // 4, dtype=torch.float32, device=dev)

    def timed(launch, steps, kernels_per_step):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                launch()
            stream.synchronize()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            for k in range(steps):
                flush.sum()
                ev[k][0].record(stream)
                launch()
                ev[k][1].record(stream)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps, steps * kernels_per_step

    sampler = ClockSampler(dev.index)
    with sampler:
        ms_batched, launches = timed(lambda: plan.graph_launch(stream.cuda_stream), args.steps, 1)
    clocks = sampler.summary()
    k_small = max(10, min(args.steps, 200))
    ms_field, _ = timed(lambda: plan.launch(plan.PER_FIELD, stream.cuda_stream), k_small, 0)
    ms_box, _ = timed(lambda: plan.launch(plan.PER_BOX, stream.cuda_stream), max(5, k_small // 4), 0)

    # bit-exact check of the exchanged halos against the oracle on this rank's data
    import oracle.regular as O
    bad = 0
    for halos, specs in w.halo_groups().items():
        doms = [O.Domain(i, f, l) for i, f, l in w.domains]
        pat = O.make_pattern((0,) * w.dim, tuple(n - 1 for n in w.shape), halos, w.periodic, doms)
        for s in specs:
            exp = [a.copy(order="K") for a in host[s.name]]
            O.exchange(pat, doms, exp, [w.offsets(s)] * len(doms))
            for t, e in zip(tens[s.name], exp):
                got = t.cpu().numpy()
                u = np.dtype(f"u{e.itemsize}")
                bad += int(np.count_nonzero(np.ascontiguousarray(got).view(u) != np.ascontiguousarray(e).view(u)))

    # end to end through the public API with host buffers
    co = R.make_communication_object(ctx)
    pinned = {k: [torch.from_numpy(a).pin_memory() for a in v] for k, v in host.items()}
    outs = {k: [torch.empty_like(p).pin_memory() for p in v] for k, v in pinned.items()}
    h2d = sum(p.numel() * p.element_size() for v in pinned.values() for p in v)
    e2e_steps = max(3, min(args.steps, 20))
    with torch.cuda.stream(stream):
        for it in range(e2e_steps + 2):
            if it == 2:
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            for k in tens:
                for t, p in zip(tens[k], pinned[k]):
                    t.copy_(p, non_blocking=True)
            co.exchange(bis).wait()
            for k in tens:
                for t, o in zip(tens[k], outs[k]):
                    o.copy_(t, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())

    peak, peak_kind = peaks()
    achieved = alg / (ms_batched * 1e-3) / 1e9
    value = world * alg / (ms_batched * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic (seeded splitmix64 interiors, NaN halos)",
        "config": {"workload": w.name, "form": "batched persistent kernel, CUDA graph", "domains": len(w.domains),
                   "fields": len(w.fields), "algorithmic_bytes_per_exchange": alg,
                   "l2": "cold: a 2 x L2 read of an unrelated buffer before every timed exchange, outside its events",
                   "parallelism": f"replicas x{world}", "tuning": {k: tuning[k] for k in ("elems_per_thread", "block", "grid")}},
        "exchanges_per_s": world * 1e3 / ms_batched,
        "per_field": {"ms_per_step": ms_field, "GB/s": world * alg / (ms_field * 1e-3) / 1e9,
                      "exchanges_per_s": world * 1e3 / ms_field, "launches_per_exchange": len(w.fields)},
        "per_box": {"ms_per_step": ms_box, "GB/s": world * alg / (ms_box * 1e-3) / 1e9,
                    "exchanges_per_s": world * 1e3 / ms_box, "launches_per_exchange": info["num_descriptors"]},
        "batched_vs_per_field": ms_field / ms_batched,
        "bitexact": bad == 0, "mismatched_elements": bad,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": ncu_traffic(args.config)},
        "e2e": {"value": world * alg / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d, "ms_per_step": e2e_ms},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_baseline:
        line["cpu_baseline"] = cpu_baseline(args.config, alg, args.baseline_seconds, 1)
        line["cpu_baseline"].pop("exchanges_per_s", None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
