"""Serving loop: progressive render requests over resident scenes, with
continuous batching and memory-footprint admission.

The reference renders one scene per `GpuPathTracer`; a service in front of
it would run requests one after another. Here scenes (prepared buffers,
BVHs, four-wide trees, tables) stay resident in HBM, every request is a
session (a view of its scene with its own camera, resolution, sample
target and accumulator), and a scheduler advances all admitted sessions
together: each tick gives every session a share of a path budget and
traces all of them as one batched wavefront (oxpt_batch.h), so requests
that arrive while others are on the GPU start at the next tick and their
work overlaps on the device. Admission is by measured device footprint
against a budget, first come first served. A camera move on a session
resets its accumulation, as `sync` does for a camera change; a request
superseded by a later move on the same session before it completed is
reported as such, not as a latency sample.

Results do not depend on the mix: a session's samples are traced with
their own sample indices and added in sample order whatever the tick
split, so its accumulator equals the one a render of that request alone
gives, bit for bit (tests/test_gpu_serve.py).

The scheduler is independent of the GPU: it drives an executor (`open`,
`move`, `refine`, `close`, `footprint`, `sync`); `GpuExecutor` is the CUDA
one, tests also drive it with a host-only fake.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

Camera = Tuple[Tuple[float, float, float], Tuple[float, float, float]]  # eye, target


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds after the stream starts
    scene: int                     # resident scene index
    width: int
    height: int
    spp: int                       # target samples per pixel
    camera: Optional[Camera] = None
    session: Optional[int] = None  # a camera move on the session opened by this request id

    @property
    def pixels(self) -> int:
        return self.width * self.height


@dataclass
class Outcome:
    rid: int
    arrival: float
    admitted: float = -1.0
    finished: float = -1.0
    paths: int = 0
    superseded: bool = False

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Session:
    key: int                       # request id that opened it
    handle: object
    req: Request
    samples: int = 0
    bytes: int = 0


@dataclass
class Stats:
    outcomes: List[Outcome] = field(default_factory=list)
    wall: float = 0.0
    ticks: int = 0
    peak_bytes: int = 0

    def completed(self) -> List[Outcome]:
        return [o for o in self.outcomes if o.finished >= 0 and not o.superseded]

    def percentile(self, q: float) -> float:
        lat = sorted(o.latency for o in self.completed())
        if not lat:
            return float("nan")
        k = min(len(lat) - 1, max(0, int(round(q / 100.0 * (len(lat) - 1)))))
        return lat[k]

    def msamples_per_s(self) -> float:
        return sum(o.paths for o in self.outcomes) / max(self.wall, 1e-9) / 1e6


class Server:
    """Continuous-batching scheduler over an executor.

    tick_paths: paths traced per tick across all sessions (each active
    session gets an equal share, at least one sample, at most what it has
    left); budget: device bytes for scenes, executor state and sessions;
    max_sessions: sessions admitted at once."""

    def __init__(self, executor, budget: int, tick_paths: int = 1 << 24, max_sessions: int = 256,
                 clock: Callable[[], float] = time.perf_counter, sleep: Callable[[float], None] = time.sleep):
        self.ex = executor
        self.budget = budget
        self.tick_paths = tick_paths
        self.max_sessions = max_sessions
        self.clock = clock
        self.sleep = sleep

    def run(self, requests: Sequence[Request]) -> Stats:
        stats = Stats()
        out: Dict[int, Outcome] = {}
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting: collections.deque = collections.deque()
        active: Dict[int, _Session] = {}     # session key -> session (samples counted as queued)
        current: Dict[int, int] = {}         # session key -> request id it is rendering
        closed: Dict[int, Request] = {}      # finished sessions, for later moves
        inflight = None                      # (mark, [(session, request id, n)]) of the queued tick
        used = self.ex.resident_bytes()
        t0 = self.clock()

        def retire(tick):
            mark, work = tick
            self.ex.wait(mark)
            now = self.clock() - t0
            for sess, rid, n in work:
                o = out[rid]
                if o.superseded:
                    continue
                o.paths += n * sess.req.pixels
                if current.get(sess.key) == rid and sess.samples >= sess.req.spp and sess.key in active:
                    o.finished = now
                    self.ex.finished(sess.handle, o)
                    self.ex.close(sess.handle)
                    closed[sess.key] = sess.req
                    del active[sess.key]
                    del current[sess.key]
                    nonlocal used
                    used -= sess.bytes

        while pending or waiting or active or inflight:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                out[r.rid] = Outcome(r.rid, r.arrival)
                stats.outcomes.append(out[r.rid])
                key = r.session if r.session is not None else r.rid
                if r.session is not None and key in active:
                    # camera move on an open session: reset it in place (the
                    # reset is ordered after any queued tick on the device)
                    sess = active[key]
                    out[current[key]].superseded = True
                    self.ex.move(sess.handle, r.camera, r.spp)
                    sess.req = Request(r.rid, r.arrival, sess.req.scene, sess.req.width, sess.req.height, r.spp,
                                       r.camera, key)
                    sess.samples = 0
                    current[key] = r.rid
                    out[r.rid].admitted = now
                    continue
                if r.session is not None:
                    for w in waiting:  # a move on a session still waiting replaces its request
                        wkey = w.session if w.session is not None else w.rid
                        if wkey == key:
                            out[w.rid].superseded = True
                    waiting = collections.deque(w for w in waiting if not out[w.rid].superseded)
                    if key in closed:
                        prev = closed[key]
                        r = Request(r.rid, r.arrival, prev.scene, prev.width, prev.height, r.spp, r.camera, key)
                waiting.append(r)
            # admission, first come first served
            while waiting and len(active) < self.max_sessions:
                r = waiting[0]
                need = self.ex.footprint(r)
                if used + need > self.budget and (active or inflight):
                    break
                waiting.popleft()
                key = r.session if r.session is not None else r.rid
                h = self.ex.open(r)
                active[key] = _Session(key, h, r, 0, need)
                current[key] = r.rid
                used += need
                out[r.rid].admitted = self.clock() - t0
            stats.peak_bytes = max(stats.peak_bytes, used)
            # queue the next tick: an equal share of the path budget for every
            # session with samples left
            todo = [sess for sess in active.values() if sess.samples < sess.req.spp]
            tick = None
            if todo:
                share = max(1, self.tick_paths // len(todo))
                work = []
                for sess in todo:
                    n = max(1, min(sess.req.spp - sess.samples, share // max(1, sess.req.pixels)))
                    sess.samples += n
                    work.append((sess, current[sess.key], n))
                mark = self.ex.refine([(sess.handle, n) for sess, _, n in work])
                tick = (mark, work)
                stats.ticks += 1
            if inflight is not None:
                retire(inflight)
            inflight = tick
            if inflight is None and not active and not waiting and pending:
                wait = pending[0].arrival - (self.clock() - t0)
                if wait > 0:
                    self.sleep(wait)
        stats.wall = self.clock() - t0
        return stats


def run_serial(executor, requests: Sequence[Request], clock: Callable[[], float] = time.perf_counter,
               sleep: Callable[[float], None] = time.sleep) -> Stats:
    """The plain baseline: requests in arrival order, one at a time, each
    rendered to its target by one plain refine. A request whose session
    has a later move that arrived before it started is skipped as
    superseded."""
    stats = Stats()
    reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
    closed: Dict[int, Request] = {}
    t0 = clock()
    for i, r in enumerate(reqs):
        o = Outcome(r.rid, r.arrival)
        stats.outcomes.append(o)
        now = clock() - t0
        if r.arrival > now:
            sleep(r.arrival - now)
            now = clock() - t0
        key = r.session if r.session is not None else r.rid
        if any(q.session == key and q.arrival <= now for q in reqs[i + 1:]):
            o.superseded = True
            continue
        if r.session is not None and r.session in closed:
            prev = closed[r.session]
            r = Request(r.rid, r.arrival, prev.scene, prev.width, prev.height, r.spp, r.camera, r.session)
        o.admitted = now
        h = executor.open(r)
        executor.refine_alone(h, r.spp)
        executor.sync()
        o.finished = clock() - t0
        o.paths = r.spp * r.pixels
        executor.finished(h, o)
        executor.close(h)
        closed[key] = r
    stats.wall = clock() - t0
    return stats


class GpuExecutor:
    """Sessions are views of resident owner tracers; ticks are batched
    refines on one executor context."""

    def __init__(self, pkg, owners: List[object], options: Callable[[Request], object], executor=None,
                 keep: Optional[Callable[[Outcome], bool]] = None, idle_views: int = 2):
        self.pkg = pkg
        self.owners = owners
        self.options = options
        # Closed sessions' views wait here for the next request on their
        # scene: freeing a view's device buffers (and allocating a new
        # one's) would synchronise the device between queued ticks.
        # Only views that batched ticks traced are kept: a view that traced
        # on its own (refine_alone) holds its own wavefront state, gigabytes
        # that would pile up in the pool.
        self.idle_views = idle_views
        self.pool: Dict[int, List[object]] = {}
        self.scene_of: Dict[int, int] = {}
        self.alone: set = set()
        if executor is None:
            executor = pkg.GpuPathTracer(0)
            # Job-major NEE for mixed batches: a warp's lanes may hold
            # vertices of scenes with different numbers of lights, and the
            # vertex-major kernel's per-vertex job loops then diverge
            # (served stream: 142 against 121 Msamples/s).
            executor.set_tuning(nee_variant=1)
        self.exe = executor
        self.keep = keep
        self.kept: Dict[int, object] = {}

    def resident_bytes(self) -> int:
        total = 0
        for o in self.owners:
            m = o.memory()
            total += m["scene"] + m["tables"] + m["images"] + m["working"]
        m = self.exe.memory()
        return total + m["working"] + (1 << 30)  # + the executor's wavefront state, grown on first use

    def footprint(self, r: Request) -> int:
        return r.pixels * 16  # the session's accumulator; scene and tables are the owner's

    def open(self, r: Request):
        idle = self.pool.get(r.scene)
        reused = bool(idle)
        v = idle.pop() if reused else self.owners[r.scene].view()
        v.sync_view(self.options(r))
        if r.camera is not None:
            v.set_camera(eye=r.camera[0], target=r.camera[1])
        elif reused:
            v.set_camera(None)
        if reused:
            v.reset()  # same options as the view's last request would keep its samples
        self.scene_of[id(v)] = r.scene
        return v  # tables and params bind on the first refine

    def move(self, v, camera: Optional[Camera], spp: int):
        if camera is not None:
            v.set_camera(eye=camera[0], target=camera[1])
        else:
            v.set_camera(None)

    def refine(self, work):
        """Queues one batched tick; returns a mark to wait for."""
        import ctypes as C
        self.pkg.refine_batch([v for v, _ in work], [n for _, n in work], executor=self.exe)
        m = C.c_uint64()
        self.pkg._native.lib().oxpt_mark(self.exe.ctx, C.byref(m))
        return m.value

    def wait(self, mark):
        self.pkg._native.lib().oxpt_wait_mark(self.exe.ctx, mark)

    def refine_alone(self, v, n: int):
        self.alone.add(id(v))
        v.refine(n)

    def sync(self):
        self.exe.finish()

    def finished(self, v, o: Outcome):
        if self.keep is not None and self.keep(o):
            self.kept[o.rid] = v.read_accum()

    def close(self, v):
        v.finish()
        scene = self.scene_of.pop(id(v), None)
        if id(v) in self.alone:
            self.alone.discard(id(v))
            return
        idle = self.pool.setdefault(scene, [])
        if scene is not None and len(idle) < self.idle_views:
            idle.append(v)
