"""Batched and served instances: admission and backfill (CPU, with a fake
executor), and on the GPU that every result is the same alone and in the
mix, through the native batch scheduler and through the server."""
import threading
import time

import numpy as np
import pytest

from spiffe_b200 import abi, serve


def fake_requests(sizes):
    return [serve.ScanRequest(i, "pillbox", 40, 30, 256, 0.0, 80e6, 1e-9, 0.0, 1, i) for i in range(len(sizes))]


class FakeWork:
    """execute() sleeps for the request's duration and records the memory in
    use while it runs."""

    def __init__(self, sizes, durations):
        self.sizes, self.durations = sizes, durations
        self.lock = threading.Lock()
        self.in_use, self.peak, self.order = 0, 0, []

    def footprint(self, r):
        return self.sizes[r.index]

    def execute(self, r):
        with self.lock:
            self.in_use += self.sizes[r.index]
            self.peak = max(self.peak, self.in_use)
            self.order.append(r.index)
        time.sleep(self.durations[r.index])
        with self.lock:
            self.in_use -= self.sizes[r.index]
        return r.index


def test_budget_is_never_exceeded():
    rng = np.random.default_rng(0)
    sizes = list(rng.integers(1, 10, 40))
    work = FakeWork(sizes, [0.01] * 40)
    s = serve.Server(12, workers=8, execute=work.execute, footprint=work.footprint)
    rows = s.serve(fake_requests(sizes), rate=400.0)
    assert work.peak <= 12
    assert all(r["error"] is None and r["result"] == r["index"] for r in rows)
    assert all(r["start"] >= r["arrival"] - 1e-9 and r["end"] >= r["start"] for r in rows)


def test_fifo_without_backfill():
    sizes = [8, 8, 1, 1, 8, 1]
    work = FakeWork(sizes, [0.03] * 6)
    s = serve.Server(10, workers=4, backfill=False, execute=work.execute, footprint=work.footprint)
    s.serve(fake_requests(sizes), rate=1e6)
    assert work.order == list(range(6))


def test_backfill_passes_a_blocked_head():
    # request 0 holds 8 of 10; request 1 (8) must wait, 2 and 3 (1 each) fit beside 0
    sizes = [8, 8, 1, 1]
    work = FakeWork(sizes, [0.2, 0.01, 0.01, 0.01])
    s = serve.Server(10, workers=4, backfill=True, execute=work.execute, footprint=work.footprint)
    s.serve(fake_requests(sizes), rate=1e6)
    assert work.order.index(2) < work.order.index(1) and work.order.index(3) < work.order.index(1)


def test_bypass_limit_starts_the_head():
    # a stream of small requests would pass the big head forever without the limit
    sizes = [6, 6] + [1] * 30
    work = FakeWork(sizes, [0.05, 0.05] + [0.02] * 30)
    s = serve.Server(8, workers=8, backfill=True, max_bypass=3, execute=work.execute, footprint=work.footprint)
    s.serve(fake_requests(sizes), rate=1e6)
    assert work.order.index(1) <= 2 + 3


def test_percentile_and_draws():
    assert serve.percentile([3, 1, 2, 4], 50) == 2 and serve.percentile([3, 1, 2, 4], 99) == 4
    a, b = serve.draw_requests(50), serve.draw_requests(50)
    assert a == b
    for r in a:
        assert 120 * 0.99 <= r.nz <= 1500 and 80 * 0.99 <= r.nr <= 400
        assert 1e4 * 0.99 <= r.n_macro <= 5e5 and 0 <= r.phase_deg <= 90
        assert 60e6 <= r.peak_field <= 120e6 and 0.05e-9 * 0.99 <= r.charge <= 2e-9 * 1.01
    assert {r.kind for r in a} == {"pillbox", "gun"}


def snapshot(g, r):
    from spiffe_b200 import gpu  # noqa: F401

    f = abi.Fields(r.nz, r.nr, 0.0, 1.0, 1.0)
    out = g.fields(f)
    b = g.download_beam(abi.Beam(r.capacity))
    k = np.argsort(b["particleID"][: b.np])
    return {**{n: out[n].copy() for n in ("Ez", "Er", "Bphi", "Jz", "Jr", "Psi")},
            **{n: b[n][: b.np][k].copy() for n in ("z", "r", "pz", "pr")}}


def same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in a)


@pytest.mark.gpu
def test_batch_result_is_the_same_alone_and_in_the_mix():
    from spiffe_b200 import gpu

    reqs = serve.draw_requests(6, steps=150, size_scale=0.25, particle_scale=0.02)
    alone = []
    for r in reqs:
        g, _ = serve.build(r)
        g.run_steps(r.steps)
        alone.append(snapshot(g, r))
        g.close()
    insts = [serve.build(r)[0] for r in reqs]
    done = gpu.batch_run(insts, [r.steps for r in reqs], workers=4, chunk=7)
    assert all(t > 0 for t in done)
    for g, r, a in zip(insts, reqs, alone):
        assert same(snapshot(g, r), a), r
        g.close()


@pytest.mark.gpu
def test_served_result_is_the_same_alone_and_in_the_mix():
    reqs = serve.draw_requests(8, steps=100, size_scale=0.25, particle_scale=0.02)
    alone = {}
    for r in reqs:
        g, _ = serve.build(r)
        g.run_steps(r.steps)
        alone[r.index] = serve.collect(g, r)
        g.close()
    s = serve.Server(budget_bytes=sum(serve.footprint_bytes(r) for r in reqs) / 3, workers=4)
    rows = s.serve(reqs, rate=200.0)
    assert all(o["error"] is None for o in rows), [o["error"] for o in rows]
    assert max(o["peak_in_use"] for o in rows) <= s.budget
    for o in rows:
        a, b = alone[o["index"]], o["result"]
        assert a["np"] == b["np"] and a["records"] == b["records"]
        assert a["moments"] == b["moments"]


@pytest.mark.gpu
def test_footprint_bounds_the_device_memory():
    import torch

    reqs = serve.draw_requests(4, steps=1, size_scale=1.0, particle_scale=0.2)
    torch.cuda.init()
    for r in reqs:
        free0, _ = torch.cuda.mem_get_info()
        g, _ = serve.build(r)
        g.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        used = free0 - free1
        g.close()
        assert used <= serve.footprint_bytes(r), (r, used, serve.footprint_bytes(r))
