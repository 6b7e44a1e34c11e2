"""Helpers for GPU tests: run the product on a regular workload and the oracle on the same inputs."""
from __future__ import annotations

import numpy as np
import torch

from ghex_b200.structured import regular as R
from oracle import regular as O


def to_device(a: np.ndarray, dev) -> torch.Tensor:
    """Copies a numpy array to the device keeping its strides (x-fastest arrays stay x-fastest)."""
    t = torch.from_numpy(a)
    out = t.to(dev)
    assert out.stride() == t.stride()
    return out


def bits_equal(a: np.ndarray, b: np.ndarray) -> int:
    """Number of elements whose bit patterns differ (NaN-aware bit-exact comparison)."""
    u = np.dtype(f"u{a.itemsize}")
    return int(np.count_nonzero(np.ascontiguousarray(a).view(u) != np.ascontiguousarray(b).view(u)))


class RegularRun:
    """A regular workload on the device through the drop-in API: one pattern per halo group,
    one field descriptor per (field, domain)."""

    def __init__(self, w, dev, ctx=None):
        self.w = w
        self.ctx = ctx or R.make_context()
        self.host = {}
        self.dev = {}
        self.patterns = {}
        self.fds = {}
        self.bis = []
        for halos, specs in w.halo_groups().items():
            hg = R.HaloGenerator(((0,) * w.dim, tuple(n - 1 for n in w.shape)),
                                 [(halos[2 * k], halos[2 * k + 1]) for k in range(w.dim)], w.periodic)
            doms = [R.DomainDescriptor(i, (f, l)) for i, f, l in w.domains]
            pat = R.make_pattern(self.ctx, hg, doms)
            self.patterns[halos] = pat
            for spec in specs:
                arrays = [w.domain_array(d, spec) for d in w.domains]
                self.host[spec.name] = arrays
                tens = [to_device(a, dev) for a in arrays]
                self.dev[spec.name] = tens
                fds = [R.make_field_descriptor(dm, t, w.offsets(spec), w.extents(d, spec))
                       for dm, d, t in zip(doms, w.domains, tens)]
                self.fds[spec.name] = fds
                self.bis += [pat(f) for f in fds]

    def oracle(self):
        out = {}
        for halos, specs in self.w.halo_groups().items():
            doms = [O.Domain(i, f, l) for i, f, l in self.w.domains]
            pat = O.make_pattern((0,) * self.w.dim, tuple(n - 1 for n in self.w.shape), halos, self.w.periodic, doms)
            for spec in specs:
                arrays = [a.copy(order="K") for a in self.host[spec.name]]
                O.exchange(pat, doms, arrays, [self.w.offsets(spec)] * len(doms))
                out[spec.name] = arrays
        return out

    def mismatches(self, expected) -> dict:
        torch.cuda.synchronize()
        bad = {}
        for name, tens in self.dev.items():
            n = sum(bits_equal(t.cpu().numpy(), e) for t, e in zip(tens, expected[name]))
            if n:
                bad[name] = n
        return bad

    def reset(self):
        for name, tens in self.dev.items():
            for t, a in zip(tens, self.host[name]):
                t.copy_(torch.from_numpy(a))
        torch.cuda.synchronize()
