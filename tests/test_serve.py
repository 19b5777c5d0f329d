"""Serving scheduler (serve.py) on a host-only executor with a virtual clock.

The GPU part (results identical alone and in the mix) is in
tests/test_gpu_serve.py; here the scheduling rules are checked: every
request completes or is superseded by a camera move, each completed
request receives exactly its target samples in order after its last
reset, admission keeps the device footprint within the budget, arrivals
during a tick join at the next one, and the batched loop beats the serial
baseline on a loaded stream.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _serve():
    spec = importlib.util.spec_from_file_location("oxpt_serve_sched", ROOT / "oxideav-render-vulkan_b200" / "serve.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["oxpt_serve_sched"] = mod
    spec.loader.exec_module(mod)
    return mod


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 0.0)


class FakeExecutor:
    """Device time = paths / rate + a fixed cost per launch group, like a
    GPU whose small launches leave it idle."""

    def __init__(self, clock, rate=1e8, launch_cost=2e-3):
        self.clock, self.rate, self.launch_cost = clock, rate, launch_cost
        self.log = {}       # session id -> list of (first, count)
        self.cur = {}       # session id -> samples since the last reset
        self.next_id = 0
        self.open_sessions = set()
        self.busy_until = 0.0

    def resident_bytes(self):
        return 1000

    def footprint(self, r):
        return r.pixels * 16

    def open(self, r):
        h = self.next_id
        self.next_id += 1
        self.log[h] = []
        self.cur[h] = 0
        self.open_sessions.add(h)
        return h

    def move(self, h, camera, spp):
        self.log[h].append(("reset",))
        self.cur[h] = 0

    def _trace(self, h, n, px):
        self.log[h].append((self.cur[h], n))
        self.cur[h] += n
        return n * px

    def refine(self, work):
        # the device runs ticks back to back: a queued tick starts when the
        # previous one ends, or now if the device is idle
        paths = sum(self._trace(h, n, self.px[h]) for h, n in work)
        start = max(self.busy_until, self.clock.t)
        self.busy_until = start + paths / self.rate + self.launch_cost
        return self.busy_until

    def wait(self, mark):
        self.clock.t = max(self.clock.t, mark)

    def refine_alone(self, h, n):
        self.clock.t += self._trace(h, n, self.px[h]) / self.rate + self.launch_cost * max(1, n // 4)

    def sync(self):
        pass

    def finished(self, h, o):
        pass

    def close(self, h):
        self.open_sessions.discard(h)


def _stream(mod, rng, n=120, lam=40.0, moves=0.3):
    reqs, t, opened = [], 0.0, []
    for rid in range(n):
        t += rng.exponential(1.0 / lam)
        if opened and rng.random() < moves:
            base = reqs[opened[int(rng.integers(len(opened)))]]
            key = base.session if base.session is not None else base.rid
            reqs.append(mod.Request(rid, t, base.scene, base.width, base.height, int(rng.choice([4, 16, 64])),
                                    ((rng.random(), 1.0, 3.0), (0.0, 0.0, 0.0)), key))
        else:
            side = int(rng.choice([64, 128, 256]))
            reqs.append(mod.Request(rid, t, int(rng.integers(8)), side, side, int(rng.choice([4, 16, 64, 256]))))
            opened.append(rid)
    return reqs


def _patch_px(ex, server_or_none, reqs):
    # the fake needs each handle's pixel count: wrap open
    orig = ex.open
    ex.px = {}

    def open_(r):
        h = orig(r)
        ex.px[h] = r.pixels
        return h

    ex.open = open_


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_every_request_completes_with_its_samples_in_order(seed):
    mod = _serve()
    rng = np.random.default_rng(seed)
    reqs = _stream(mod, rng)
    clock = Clock()
    ex = FakeExecutor(clock)
    _patch_px(ex, None, reqs)
    budget = 1000 + 40 * 256 * 256 * 16
    st = mod.Server(ex, budget, tick_paths=1 << 20, clock=clock, sleep=clock.sleep).run(reqs)
    assert len(st.outcomes) == len(reqs)
    done = st.completed()
    sup = [o for o in st.outcomes if o.superseded]
    assert len(done) + len(sup) == len(reqs) and len(done) > len(reqs) // 2
    assert all(o.latency > 0 and o.admitted >= o.arrival for o in done)
    assert st.peak_bytes <= budget
    assert not ex.open_sessions
    # per session: after its last reset, samples 0..spp-1 in order, contiguous
    by_rid = {r.rid: r for r in reqs}
    for h, log in ex.log.items():
        seg = log[max((i for i, e in enumerate(log) if e == ("reset",)), default=-1) + 1:]
        nxt = 0
        for first, n in seg:
            assert first == nxt
            nxt += n
        assert nxt in {r.spp for r in reqs}  # ends exactly at a target
    assert {o.rid for o in done} <= set(by_rid)


def test_admission_waits_for_memory_and_serves_first_come_first():
    mod = _serve()
    clock = Clock()
    ex = FakeExecutor(clock, rate=1e7)
    reqs = [mod.Request(i, 0.001 * i, 0, 256, 256, 64) for i in range(6)]
    _patch_px(ex, None, reqs)
    budget = 1000 + 2 * 256 * 256 * 16  # two sessions at a time
    st = mod.Server(ex, budget, tick_paths=1 << 18, clock=clock, sleep=clock.sleep).run(reqs)
    adm = [o.admitted for o in sorted(st.outcomes, key=lambda o: o.rid)]
    assert adm == sorted(adm)
    assert st.peak_bytes <= budget
    assert adm[2] >= min(o.finished for o in st.outcomes[:2])


def test_batched_loop_beats_serial_plain_on_a_loaded_stream():
    mod = _serve()
    rng = np.random.default_rng(7)
    reqs = _stream(mod, rng, n=150, moves=0.0)
    ca, cb = Clock(), Clock()
    ea, eb = FakeExecutor(ca), FakeExecutor(cb)
    _patch_px(ea, None, reqs)
    _patch_px(eb, None, reqs)
    served = mod.Server(ea, 1 << 40, tick_paths=1 << 22, clock=ca, sleep=ca.sleep).run(reqs)
    serial = mod.run_serial(eb, reqs, clock=cb, sleep=cb.sleep)
    assert served.msamples_per_s() > serial.msamples_per_s()
    assert served.percentile(99) < serial.percentile(99)


class _View:
    """Stands in for a tracer view: records what the executor asks of it."""
    made = 0

    def __init__(self, owner):
        _View.made += 1
        self.owner, self.calls = owner, []

    def sync_view(self, opts):
        self.calls.append(("sync", opts))

    def set_camera(self, eye=None, target=None):
        self.calls.append(("camera", eye))

    def reset(self):
        self.calls.append(("reset",))

    def refine(self, n):
        self.calls.append(("refine", n))

    def finish(self):
        self.calls.append(("finish",))


class _Owner:
    def view(self):
        return _View(self)


def test_gpu_executor_keeps_closed_views_per_scene():
    """Closed sessions' views wait for the next request on their scene: a
    reused view is reset and its camera override cleared, at most
    `idle_views` wait per scene, and views that traced on their own (the
    serial baseline's) are not kept."""
    mod = _serve()
    _View.made = 0
    owners = [_Owner(), _Owner()]
    ex = mod.GpuExecutor(pkg=None, owners=owners, options=lambda r: (r.width, r.height), executor=object(),
                         idle_views=1)
    r0 = mod.Request(0, 0.0, 0, 64, 64, 4, camera=((1.0, 2.0, 3.0), (0.0, 0.0, 0.0)))
    v0 = ex.open(r0)
    ex.close(v0)
    v1 = ex.open(mod.Request(1, 0.0, 0, 32, 32, 4))          # same scene: the kept view
    assert v1 is v0 and _View.made == 1
    assert ("reset",) in v1.calls and ("camera", None) in v1.calls
    v2 = ex.open(mod.Request(2, 0.0, 1, 32, 32, 4))          # another scene: a new view
    assert v2 is not v0 and _View.made == 2
    v3 = ex.open(mod.Request(3, 0.0, 0, 32, 32, 4))          # scene 0's kept view is in use
    assert _View.made == 3
    ex.close(v1)
    ex.close(v3)                                             # one kept per scene
    assert len(ex.pool[0]) == 1
    ex.refine_alone(v2, 4)
    ex.close(v2)                                             # traced alone: not kept
    assert not ex.pool.get(1)
