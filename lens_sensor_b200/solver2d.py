"""One plain full-domain 2D solve on the GPU with a fixed schedule: the
planar-waveguide run of fdtd2d_core.run_beads(method='full') reduced to its
time-stepping outputs (planar_beads/fdtd2d_core.py:781-890):

  * the CW phasor (2/N) sum F e^{-i w t} of the node field (TE Ez, TM Ey on
    the nodes) over the last `periods` periods of the run (:838-847, :879),
  * snapshots of the driven raw component (TE Ez, TM Ey) every `snap_every`
    steps (the transient frames of the reference's frame writer, :876-890).

schedule_2d() is torch-free so the oracle's FP64 replay of a workload uses the
same windows.
"""
import contextlib
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import engine as E
from ._native import F32 as N_F32
from . import _native as N
from .geometry import Spec2D, build_2d

_HOST_POOL = ThreadPoolExecutor(1, thread_name_prefix='lens-host-stage-2d')


def _touched(shape, dtype):
    """A host array written once, so that its pages are resident before a copy lands in it."""
    a = np.empty(shape, dtype)
    a.view(np.uint8).fill(0)
    return a


def schedule_2d(sp: Spec2D, steps_total, periods=1, snap_every=200):
    """DFT window over the last `periods` periods (steps_per_T = round(T/dt),
    fdtd2d_core.py:757-758) and the snapshot steps (after steps n with
    (n + 1) % snap_every == 0)."""
    n = int(steps_total)
    steps_per_T = max(4, int(round((1.0 / sp.f0) / sp.dt)))
    n_acc = min(n, int(periods) * steps_per_T)
    snaps = list(range(snap_every, n + 1, snap_every)) if snap_every else []
    return dict(omega=2 * np.pi * sp.f0, steps_per_T=steps_per_T, n_acc=n_acc, dft=(n - n_acc, n), snaps=snaps)


class Solve2D:
    """Resident 2D solve of `steps_total` steps.

    engine='resident': the whole schedule in ONE cooperative launch that keeps
    the fields in registers (lens_rs2d_run, bands of x rows exchanging one row
    per half step through L2), the snapshots written by the kernel and the DFT
    accumulated compensated; the grid must fit on the chip (ny <= 576, at most
    20 rows per band);
    engine='persistent': the batched kernels on this one instance in one
    persistent cooperative launch per snapshot period (lens_batch2d_run, the
    grid kept on chip across steps, no launch gaps);
    engine=None (default): 'resident' when the grid fits the chip, else 'batch';
    engine='batch': the batched kernels on this one instance
    (lens_batch2d_step, vector passes over 128 x 2*by tiles; capture() records
    the whole schedule, snapshots included, as one CUDA graph that run()
    replays); engine='tb': the temporally blocked step (lens_tb2d_step,
    LENS_TB_K steps per launch; the schedule and the snapshot period must be
    whole numbers of launch pairs; chunk: rows per warp); engine='step': the
    single-grid engine (lens_te2d_step / lens_tm2d_step), one step per launch
    pair, with the full single-grid epilogue set."""

    def __init__(self, spec: Spec2D, steps_total, periods=1, snap_every=200, device=None, geo=None, engine=None,
                 chunk=16, by=4):
        self.spec = sp = spec
        self.steps_total = int(steps_total)
        t0 = time.perf_counter()
        self.geo = g = geo if geo is not None else build_2d(sp)
        self.t_setup_host = time.perf_counter() - t0
        sc = schedule_2d(sp, steps_total, periods, snap_every)
        self.omega, self.steps_per_T, self.n_acc = sc['omega'], sc['steps_per_T'], sc['n_acc']
        self.dft, self.snap_steps = sc['dft'], sc['snaps']
        coef = {k: g[k] for k in ('ce_e', 'ce_h', 'ca_x', 'ca_y', 'da_x', 'da_y') if g.get(k) is not None}
        self.h2d_bytes = sum(np.asarray(a).nbytes for a in coef.values()) + \
            sum(np.asarray(g['src'][k]).nbytes for k in ('amp', 'ph1', 'ph2'))
        self.table = E.StepTable(0, self.steps_total, sp.dt, g['src']['omega'], self.omega,
                                 E.cw_envelope(sp.f0, sp.ramp_periods), device=device)
        probe = None
        if engine is None:   # the resident launch when the grid fits the chip
            from . import batch2d as B
            probe = B.Instance(sp, self.steps_total, torch.float32, E._device(device), g, kahan=True, window=self.dft)
            engine = 'resident' if B.ResidentGroup.fits([probe]) else 'batch'
        self.engine = engine
        self.graph = None
        if engine == 'resident':
            from . import batch2d as B
            dev = E._device(device)
            self.inst = probe if probe is not None else \
                B.Instance(sp, self.steps_total, torch.float32, dev, g, kahan=True, window=self.dft)
            self.grid = self.epi = None
            shape = (sp.nx, sp.ny) if sp.pol == 's' else (sp.nx, sp.ny - 1)
            self.snaps = torch.zeros((len(self.snap_steps),) + shape, dtype=torch.float32, device=dev)
            frames = [(snap_every, self.snaps)] if self.snap_steps else None
            self.group = B.ResidentGroup([self.inst], dev, frames=frames)
            fld = self.inst.f[0] if sp.pol == 's' else self.inst.f[1]
            self._view = lambda: fld[:shape[0], :shape[1]]
            self.n = 0
            self.launches = 0
            return
        if engine in ('tb', 'batch', 'persistent'):
            from . import batch2d as B
            tb = engine == 'tb'
            span = 2 * N.TB_K
            if tb and (self.steps_total % span or any(m % span for m in self.snap_steps)):
                raise ValueError(f"engine='tb' runs spans of {span} steps: use engine='batch' for this schedule")
            dev = E._device(device)
            self.inst = B.Instance(sp, self.steps_total, torch.float32, dev, g, tb=tb, kahan=tb, window=self.dft)
            self.group = B.Group([self.inst], N_F32, by, dev, tb=tb, chunk=chunk)
            self.grid = self.epi = None
            fld = self.inst.f[0] if sp.pol == 's' else self.inst.f[1]
            shape = (sp.nx, sp.ny) if sp.pol == 's' else (sp.nx, sp.ny - 1)
            self._view = lambda: fld[:shape[0], :shape[1]]
        else:
            self.grid = E.Grid2D(sp.pol, sp.nx, sp.ny, sp.dx, sp.dt, coef, g['cx'], g['cy'], g['src'], device=device)
            self.epi = E.Epi2D(self.grid, dft=self.dft)
            comp = 'ez' if self.grid.pol == 's' else 'ey'
            self._view = lambda: self.grid.view(comp)
        v = self._view()
        self.snaps = torch.zeros((len(self.snap_steps),) + tuple(v.shape), dtype=torch.float32, device=v.device)
        self.n = 0
        self.launches = 0

    def _advance(self, n, m, stream):
        """Steps [n, m)."""
        if self.engine == 'resident':
            self.group.step(self.table, n, m - n, stream)
            self.launches += 1
            return
        if self.engine == 'step':
            self.grid.step(self.table, n, m - n, self.epi, stream)
            self.launches += 2 * (m - n)
            return
        if self.engine == 'persistent':
            self.group.step_persistent(self.table, n, m - n, stream)
            self.launches += 1
            return
        self.group.step(self.table, n, m - n, stream)
        self.launches += self.group.launches(n, m)

    def capture(self):
        """Record the rest of the schedule (steps and snapshot copies) as one CUDA
        graph; the next run() replays it (batched and temporally blocked engines)."""
        if self.engine in ('step', 'persistent', 'resident'):
            raise ValueError(f"engine={self.engine!r} is not captured")
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.snaps.device)
        s.wait_stream(torch.cuda.current_stream())
        n0, l0 = self.n, self.launches
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self._schedule(None)
        torch.cuda.current_stream().wait_stream(s)
        self.n, self._graph_launches, self.launches = n0, self.launches - l0, l0
        self.graph = g
        return self

    def run(self, stream=None):
        """Advance to the end of the schedule, copying the snapshots on the way
        (replaying the captured graph when there is one)."""
        if self.graph is not None:
            with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
                self.graph.replay()
            self.graph = None
            self.n = self.steps_total
            self.launches += self._graph_launches
            return self
        return self._schedule(stream)

    def _schedule(self, stream):
        n = self.n
        if self.engine == 'resident':   # one launch; the kernel writes the snapshot frames
            if self.steps_total > n:
                self._advance(n, self.steps_total, stream)
            self.n = self.steps_total
            return self
        with torch.cuda.stream(stream) if stream is not None else contextlib.nullcontext():
            for q, m in enumerate(self.snap_steps + [self.steps_total]):
                if m > n:
                    self._advance(n, m, stream)
                    n = m
                if q < len(self.snap_steps):
                    self.snaps[q].copy_(self._view())
        self.n = n
        return self

    def check(self):
        """Raise if a resident launch's wait between bands ran out."""
        if self.engine == 'resident':
            self.group.check()

    def phasor(self):
        """(2/N) sum F e^{-i w t} on the nodes (nx, ny), complex128 on the device."""
        if self.engine != 'step':
            return self.inst.phasor()
        return (2.0 / self.n_acc) * self.epi.phasor()

    def stage_host(self):
        """Prepare the host destinations of host_results() on a background thread
        so that it overlaps the stepping (call before run()): a copy into pages
        that are already resident runs at the link's pageable rate instead of
        faulting the pages in (config 0's 30 snapshots, 92 MB: 0.04 s fresh)."""
        shp = (self.spec.nx, self.spec.ny)
        self._staged = _HOST_POOL.submit(lambda: (_touched(shp, np.complex64),
                                                  _touched(tuple(self.snaps.shape), np.float32)))
        return self

    def host_results(self):
        """Phasor (complex64, the reference's CW dtype) and snapshots (float32) on
        the host, into the buffers stage_host() prepared when it was called;
        d2h_bytes counts what crossed."""
        staged, self._staged = getattr(self, '_staged', None), None
        ph_d = self.phasor().to(torch.complex64)
        if staged is not None:
            ph, snaps = staged.result()
            torch.from_numpy(ph).copy_(ph_d)
            torch.from_numpy(snaps).copy_(self.snaps)
        else:
            ph, snaps = ph_d.cpu().numpy(), self.snaps.cpu().numpy()
        self.d2h_bytes = ph.nbytes + snaps.nbytes
        return ph, snaps

