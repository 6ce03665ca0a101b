"""Serving loop: continuous batching of mixed 2D / 3D / 3D-stitch solves on one GPU.

The reference has no serving layer (it runs one CLI solve at a time; its only
related piece is the one-off VRAM estimate of run_3d_stitched,
fdtd3d_core.py:1405-1450).  This loop takes a stream of timed requests and:

  * admits a request when its device footprint fits the HBM budget (first fit
    in arrival order, with the oldest waiting request's footprint held back so
    a large job is not starved by a run of small ones);
  * keeps every admitted solve resident (fields, CPML psi, coefficients, DFT
    sums stay on the device until the result is read);
  * advances all resident solves concurrently (CUDA stream priorities put the
    short 2D work ahead of 3D jobs and those ahead of stitch jobs): the 2D requests of one time step
    and wavelength share ONE batched launch per half step (lens_batch2d_step
    over every tile of every member; a request joins the running batch at the
    next quantum boundary with its own step origin, n_start) and each 3D or
    stitch job runs on a CUDA stream of its own, in quanta of steps, so their
    kernels overlap on the GPU;
  * hands stitch-window phasors from window to window on the device
    (stitch3d.StitchSolve) and builds the next window's geometry on a host
    thread while the current window runs;
  * records arrival, admission, first launch and completion of each request,
    so p50 / p99 latency and the aggregate cell-update rate can be reported.

Each request's result does not depend on what else runs: batch members are
updated tile by tile from their own arrays only, and every 3D / stitch job owns
its grid, so a request alone and in the mix gives the same numbers.
"""
import concurrent.futures as cf
import time
from collections import deque
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np
import torch

from . import batch2d as B
from . import engine as E
from .geometry import build_2d, build_3d
from .solver3d import Solve3D
from .stitch3d import StitchSolve


@dataclass
class Request:
    """kind '2d': spec = geometry.Spec2D; '3d': geometry.Spec3D; 'stitch':
    stitch3d.StitchPlan (steps is then the per-window count of the plan).

    status: 'waiting', 'running', 'done', or the request's end without a result:
    'rejected' (its footprint exceeds the whole budget), 'cancelled'
    (Server.cancel, or cancel_at seconds after the stream's start), 'failed'
    (its host-side setup raised; error holds the message).  A request that ends
    without a result frees its memory and slot; the others carry on."""
    rid: int
    kind: str
    spec: Any
    steps: int
    arrival: float = 0.0
    t_admit: Optional[float] = None
    t_start: Optional[float] = None
    t_done: Optional[float] = None
    footprint: int = 0
    result: Any = None
    status: str = 'waiting'
    error: Optional[str] = None
    cancel_at: Optional[float] = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival

    def cell_updates(self):
        s = self.spec
        if self.kind == '2d':
            return s.nx * s.ny * self.steps
        if self.kind == '3d':
            return s.nx * s.ny * s.nz * self.steps
        return s.cell_updates()


def _pitch(n):
    return -(-n // 32) * 32


def footprint(req, storage='f32'):
    """Device bytes a request holds while resident."""
    s = req.spec
    if req.kind == '2d':
        es = 4 if storage == 'f32' else 2
        P = _pitch(s.ny)
        psi = 4 * (2 * s.nx * 2 * s.npml + 2 * P * 2 * s.npml)
        return s.nx * P * (3 * es + 4 * 4 + 8) + psi + 64 * 1024
    if req.kind == '3d':
        cells = s.nx * s.ny * _pitch(s.nz)
        lossy = s.stack.lossy or any(np.iscomplexobj(b.n) for b in s.beads)
        return cells * 4 * (2 * (6 + 12) + 3 + (3 if lossy else 0) + 2 + 1) + (1 << 20)
    return s.window_bytes()


def admission(queue, used, budget, n2d, n3d, slots2d, slots3d):
    """Which waiting requests to admit, in arrival order (`queue`): first fit
    under the memory budget and the slot limits of their kind, except that the
    oldest request that does not fit keeps its claim on the memory (later ones
    are admitted only in what is left beside it), so a large job is not starved
    by a run of small ones.  A request larger than the whole budget can never
    run and is rejected.  Returns (admitted, rejected); changes nothing."""
    admitted, rejected = [], []
    held = 0
    for r in queue:
        if r.footprint > budget:
            rejected.append(r)
            continue
        is2d = r.kind == '2d'
        if not (n2d < slots2d if is2d else n3d < slots3d):
            continue
        if used + held + r.footprint > budget:
            if held == 0:
                held = r.footprint
            continue
        admitted.append(r)
        used += r.footprint
        if is2d:
            n2d += 1
        else:
            n3d += 1
    return admitted, rejected


class _Batch2D:
    """The running batch of 2D requests sharing one time step and wavelength."""

    def __init__(self, server, key):
        self.srv, self.key = server, key
        self.members = []            # (request, Instance)
        self.building = []           # (request, future of its geometry)
        self.joining = []
        self.group = None
        self.n = 0                   # batch step counter
        self.table = None
        self.stream = torch.cuda.Stream(device=server.dev, priority=server.prio['2d'])
        self.event = None

    def busy(self):
        return self.event is not None and not self.event.query()

    def idle(self):
        return not self.members and not self.joining and not self.building

    def size(self):
        return len(self.members) + len(self.joining) + len(self.building)

    def _table(self, steps):
        """Step table over the members' own steps [0, steps) (the sweep's table)."""
        if self.table is None or self.table.n < steps:
            q = self.members[0][1]
            sp = q.spec
            self.table = E.StepTable(0, max(steps, 1), sp.dt, q.omega, 2 * np.pi * sp.f0,
                                     E.cw_envelope(sp.f0, sp.ramp_periods), device=self.srv.dev)

    def pump(self, now):
        """Retire finished members, take in the joining ones, launch the next quantum."""
        if self.busy() or (not self.members and not self.joining and
                           not any(f.done() for _, f in self.building)):
            return False
        self.event = None
        done = [(r, q) for r, q in self.members if self.n - q.s.n_start >= q.steps]
        if done:
            for r, q in done:
                ph = q.phasor()
                r.result = dict(phasor=ph.cpu(), K=q.overlap(ph))
                r.t_done = time.perf_counter() - self.srv.t0
                r.status = 'done'
                self.srv.release(r)
            self.members = [m for m in self.members if m not in done]
        changed = bool(done)
        gone = [(r, q) for r, q in self.members if r.status == 'cancelled']
        for r, q in gone:
            self.srv.release(r)
        if gone:
            self.members = [m for m in self.members if m not in gone]
            changed = True
        ready = [(r, f) for r, f in self.building if f.done()]
        for r, f in ready:
            self.building.remove((r, f))
            if r.status == 'cancelled':
                self.srv.release(r)
                continue
            if f.exception() is not None:
                self.srv.fail(r, f.exception())
                continue
            self.joining.append((r, B.Instance(r.spec, r.steps, self.srv.dtype, self.srv.dev, f.result())))
        if self.joining:
            for r, q in self.joining:
                q.s.n_start = self.n
            self.members += self.joining
            self.joining = []
            changed = True
        if not self.members:
            self.group = None
            return bool(done)
        if changed or self.group is None:
            self._table(max(q.steps for _, q in self.members))
            self.group = B.Group([q for _, q in self.members], self.srv.storage_code, self.srv.by, self.srv.dev)
            self.stream.wait_stream(torch.cuda.current_stream())
        left = min(q.steps - (self.n - q.s.n_start) for _, q in self.members)
        k = min(self.srv.quantum2d, left)
        self.group.step(self.table, self.n, k, stream=self.stream)
        for r, _ in self.members:
            if r.t_start is None:
                r.t_start = now
                r.status = 'running'
        self.n += k
        self.event = torch.cuda.Event()
        self.event.record(self.stream)
        self.srv.launched += k * 2
        return True


class _Job:
    """A resident 3D or stitch solve on its own stream; geo_future builds its
    (first window's) geometry on a host thread."""

    def __init__(self, server, req, geo_future):
        self.srv, self.req, self.geo = server, req, geo_future
        self.stream = torch.cuda.Stream(device=server.dev, priority=server.prio[req.kind])
        self.event = None
        self.solve = None

    def busy(self):
        return self.event is not None and not self.event.query()

    def _start(self):
        r, srv = self.req, self.srv
        if r.kind == '3d':
            self.solve = Solve3D(r.spec, r.steps, device=srv.dev, geo=self.geo.result())
        else:
            p = r.spec
            self.Efull = np.zeros((p.Nx_full, p.Nj, p.Nk), np.complex64)
            self.Iavg = np.zeros((p.Nx_full, p.Nj, p.Nk), np.float32)

            def sink(w, g_lo, g_hi, Ew, Ia):
                self.Efull[g_lo:g_hi] = Ew
                self.Iavg[g_lo:g_hi] = Ia
            self.solve = StitchSolve(p, E, sink, device=srv.dev, stream=self.stream, pool=srv.pool,
                                     geo0=self.geo.result())
        self.stream.wait_stream(torch.cuda.current_stream())

    def pump(self, now):
        if self.busy():
            return False
        self.event = None
        r = self.req
        if r.status == 'cancelled':
            self.solve = None
            self.srv.release(r)
            return True
        if self.solve is None:
            if not self.geo.done():
                return False
            if self.geo.exception() is not None:
                self.srv.fail(r, self.geo.exception())
                return True
            self._start()
        if r.kind == '3d':
            s = self.solve
            if s.n >= s.steps_total:
                res = s.results(stream=self.stream)
                r.result = dict(res, phasor=s.phasor().cpu())
                self._finish()
                return True
            s.run(s.n + self.srv.quantum3d, stream=self.stream)
            self.srv.launched += self.srv.quantum3d
        else:
            s = self.solve
            if s.done:
                r.result = dict(Efull=self.Efull, Iavg=self.Iavg, transmission=s.transmission(), **s.vcsel())
                self._finish()
                return True
            self.srv.launched += s.advance(self.srv.quantum3d)
        if r.t_start is None:
            r.t_start = now
            r.status = 'running'
        self.event = torch.cuda.Event()
        self.event.record(self.stream)
        return True

    def ended(self):
        return self.req.status in ('done', 'cancelled', 'failed')

    def _finish(self):
        self.req.t_done = time.perf_counter() - self.srv.t0
        self.req.status = 'done'
        self.solve = None
        self.srv.release(self.req)


class Server:
    """Continuous-batching request loop on one GPU.

    budget: HBM bytes for resident solves (default 160 GB, capped at 90% of the
    device); quantum2d / quantum3d: steps per launch round of the 2D batch / of
    a 3D or stitch job; storage: 2D field storage ('f32', 'f16', 'bf16');
    slots2d / slots3d: most 2D batch members / 3D and stitch jobs resident at
    once (a request waits for a free slot of its kind and for memory)."""

    def __init__(self, budget=160e9, quantum2d=200, quantum3d=64, storage='f32', by=8, device=None,
                 host_threads=2, slots2d=512, slots3d=4):
        self.dev = E._device(device)
        self.slots2d, self.slots3d = int(slots2d), int(slots3d)
        total = torch.cuda.get_device_properties(self.dev).total_memory
        self.budget = int(min(budget, 0.9 * total))
        self.quantum2d, self.quantum3d = int(quantum2d), int(quantum3d)
        self.storage = storage
        self.storage_code, self.dtype = B.DTYPES[storage]
        self.by = by
        self.pool = cf.ThreadPoolExecutor(max_workers=host_threads)
        # shortest work first on the device: the 2D batch's stream has the highest
        # priority, 3D jobs the middle one, stitch jobs the lowest
        a, b = torch.cuda.Stream.priority_range()
        hi, lo = min(a, b), max(a, b)                    # a lower value runs first
        self.prio = {'2d': hi, '3d': (hi + lo) // 2, 'stitch': lo}
        self.used = 0
        self.t0 = 0.0
        self.launched = 0
        self._cancel = set()
        # host-side geometry builders (run on the pool; an exception fails only its request)
        self.build2d, self.build3d = build_2d, build_3d

    def release(self, req):
        """Give back the memory of an admitted request that ended."""
        if req.t_admit is not None and not getattr(req, '_released', False):
            req._released = True
            self.used -= req.footprint

    def fail(self, req, exc):
        """A request whose host-side setup raised: record it, free its memory."""
        req.status, req.error = 'failed', f'{type(exc).__name__}: {exc}'
        req.t_done = time.perf_counter() - self.t0
        self.release(req)

    def cancel(self, rid):
        """Cancel request `rid`: a waiting request leaves the queue, a running
        one stops at the end of its current quantum (its memory is freed then).
        Safe to call from another thread while run() serves."""
        self._cancel.add(int(rid))

    def _cancels(self, reqs, queue, now):
        for r in reqs:
            if r.status in ('done', 'cancelled', 'failed', 'rejected'):
                continue
            if r.rid in self._cancel or (r.cancel_at is not None and now >= r.cancel_at):
                r.status = 'cancelled'
                r.t_done = now
                if r in queue:
                    queue.remove(r)

    def _admit(self, queue, now, batches, jobs):
        n2d = sum(b.size() for b in batches.values())
        admitted, rejected = admission(queue, self.used, self.budget, n2d, len(jobs), self.slots2d, self.slots3d)
        for r in rejected:
            queue.remove(r)
            r.status, r.t_done = 'rejected', now
            r.error = f'footprint {r.footprint / 1e9:.3f} GB exceeds the budget of {self.budget / 1e9:.3f} GB'
        for r in admitted:
            queue.remove(r)
            self.used += r.footprint
            r.t_admit = now
            if r.kind == '2d':
                sp = r.spec
                key = (round(sp.dt * 1e30), sp.lam_nm)
                b = batches.get(key)
                if b is None:
                    b = batches[key] = _Batch2D(self, key)
                b.building.append((r, self.pool.submit(self.build2d, sp)))
            else:
                spec = r.spec if r.kind == '3d' else r.spec.spec(0)
                jobs.append(_Job(self, r, self.pool.submit(self.build3d, spec)))

    def run(self, requests, realtime=True):
        """Serve `requests` (arrival times in seconds from the start); returns them
        with their timestamps and results filled in.  realtime=False admits each
        request as soon as memory allows, ignoring its arrival time."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            r.footprint = footprint(r, self.storage)
        pending = deque(reqs)
        queue, batches, jobs = [], {}, []
        self.t0 = time.perf_counter()
        self.launched = 0
        while pending or queue or jobs or any(not b.idle() for b in batches.values()):
            now = time.perf_counter() - self.t0
            while pending and (not realtime or pending[0].arrival <= now):
                queue.append(pending.popleft())
            self._cancels(reqs, queue, now)
            if queue:
                self._admit(queue, now, batches, jobs)
            did = False
            for b in batches.values():
                did |= b.pump(now)
            for j in list(jobs):
                did |= j.pump(now)
                if j.ended() and (j.req.status != 'cancelled' or not j.busy()):
                    jobs.remove(j)
            if not did:
                if not jobs and all(b.idle() for b in batches.values()) and pending and not queue:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - self.t0))))
                else:
                    time.sleep(0.0002)
        torch.cuda.synchronize(self.dev)
        return reqs


def summary(reqs):
    """p50 / p99 latency, makespan and aggregate cell-update rate of the
    completed requests of a served stream (with the count of each status)."""
    done = [r for r in reqs if r.status == 'done']
    lat = np.array([r.latency for r in done])
    t_end = max(r.t_done for r in done)
    t_begin = min(r.arrival for r in done)
    cu = sum(r.cell_updates() for r in done)
    by = {}
    for r in done:
        by.setdefault(r.kind, []).append(r.latency)
    statuses = {}
    for r in reqs:
        statuses[r.status] = statuses.get(r.status, 0) + 1
    return dict(requests=len(reqs), statuses=statuses, p50_s=float(np.percentile(lat, 50)),
                p99_s=float(np.percentile(lat, 99)),
                makespan_s=t_end - t_begin, cell_updates=cu, cell_updates_per_s=cu / max(t_end - t_begin, 1e-9),
                by_kind={k: dict(n=len(v), p50_s=float(np.percentile(v, 50)), p99_s=float(np.percentile(v, 99)))
                         for k, v in by.items()})
