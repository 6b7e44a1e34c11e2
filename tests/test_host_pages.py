"""The registry of page-locked host ranges behind host-memory fields (no GPU): against a stand-in
for ghexb_host_register that refuses overlapping registrations, random acquisitions and releases
keep every held page inside a live registration, never overlap two registrations, and unregister
a range with its last holder."""
import ctypes as C
import random

import pytest

from ghex_b200 import _core


@pytest.fixture
def fake_pages(monkeypatch):
    live = {}

    def fake_call(name, *args):
        assert name == "ghexb_host_register"
        p, n, owned = args[0].value, args[1], args[2]
        for s, e in live.items():
            assert not (p < e and s < p + n), "overlapping registration"
        live[p] = p + n
        owned._obj.value = 1

    def fake_release(name, handle):
        assert name == "ghexb_host_unregister" and handle.value in live
        del live[handle.value]

    monkeypatch.setattr(_core, "call", fake_call)
    pages = _core._HostPages()
    pages._unregister = fake_release
    return pages, live


def test_random_acquire_release(fake_pages):
    pages, live = fake_pages
    P = pages.page
    rng = random.Random(1)
    held = []
    for _ in range(5000):
        if held and rng.random() < 0.45:
            pages.release(held.pop(rng.randrange(len(held)))[2])
        else:
            lo = P + rng.randrange(0, 64 * P)
            hi = lo + rng.randrange(1, 6 * P)
            held.append((lo, hi, pages.acquire(lo, hi)))
        for lo, hi, _ in held:
            for p in range(lo // P * P, hi, P):
                assert any(s <= p < e for s, e in live.items())
    for _, _, h in held:
        pages.release(h)
    assert not live and not pages.regs and not pages.page_of


def test_neighbours_share_pages(fake_pages):
    pages, live = fake_pages
    P = pages.page
    a = pages.acquire(10 * P + 100, 10 * P + 900)      # one page
    b = pages.acquire(10 * P + 1000, 12 * P + 50)      # shares page 10, adds pages 11-12
    assert len(live) == 2 and pages.regs[10 * P][1] == 2
    pages.release(a)
    assert 10 * P in live                              # still held by b
    pages.release(b)
    assert not live
