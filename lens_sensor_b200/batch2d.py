"""Batched 2D solves: many uneven TE/TM instances advanced together.

A sweep (tear-film thickness, bead size and position, polarisation) is a list
of geometry.Spec2D.  Instances are packed into groups whose resident state
fits a working-set budget (so a group's fields can stay in the 126 MB L2 across
steps); each group runs its whole schedule as ONE CUDA graph of batched
launches (lens_batch2d_step: one launch per half step for every tile of every
instance in the group).  Field storage is FP32, FP16 or BF16 (arithmetic is
FP32 throughout; coefficients, CPML psi and the DFT stay FP32).

Per instance the output is the CW phasor of the node field (Ez for TE, Ey on
the nodes for TM) over the last 8 periods (fdtd2d_core.py:757-758, 838-847)
and the evanescent overlap K = I_tear / I_guided of the time-averaged
intensity |E|^2/2 at the output window (fdtd_analyzer.py:2842-2935).

The tile shape (rows per block) and the group budget are chosen by a small
autotuner that times candidate configurations on the sweep itself and then
restores the initial state.
"""
import ctypes
import time

import numpy as np
import torch

from . import _native as N
from . import engine as E
from .geometry import build_2d

DTYPES = {'f32': (N.F32, torch.float32), 'f16': (N.F16, torch.float16), 'bf16': (N.BF16, torch.bfloat16)}


MAX_RTYPE = 4


def row_types(arrays, shape, dev, min_rows=8):
    """Row form of an instance's coefficient arrays (LensInst2D.rtype / ctab),
    from the host arrays (no device round trip): each array sits in the leading
    corner of a zero (nx, pitch) block, as on the device; the x rows are grouped
    by their exact bytes over all arrays, and the up to 4 most frequent groups of
    at least min_rows rows become row types (rtype = type, 255 for the other
    rows) whose rows form the table (ntype, ncoef, pitch).  Returns (None, None)
    when no group qualifies."""
    nx, P = shape
    a = np.zeros((nx, len(arrays), P), np.float32)
    for q, v in enumerate(arrays):
        v = np.asarray(v, np.float32)
        a[:v.shape[0], q, :v.shape[1]] = v
    groups = {}
    for i in range(nx):
        groups.setdefault(a[i].tobytes(), []).append(i)
    best = sorted(groups.values(), key=len, reverse=True)[:MAX_RTYPE]
    best = [g for g in best if len(g) >= min_rows]
    if not best:
        return None, None
    rt = np.full(nx, 255, np.uint8)
    tab = np.zeros((len(best), len(arrays), P), np.float32)
    for t, g in enumerate(best):
        rt[g] = t
        tab[t] = a[g[0]]
    return torch.from_numpy(rt).to(dev), torch.from_numpy(tab).to(dev)


class Instance:
    """Device state of one 2D solve in a batch.

    tb: also the second field / psi buffers and the psi level scratch of the
    temporally blocked step (lens_tb2d_step); kahan: a compensated DFT
    accumulator (re, im, c_re, c_im) instead of (re, im); window: the DFT steps
    (default the last 8 periods)."""

    def __init__(self, sp, steps, dtype, dev, geo=None, tb=False, kahan=False, window=None):
        self.spec, self.steps = sp, int(steps)
        geo = build_2d(sp) if geo is None else geo
        self.geo = geo
        nx, ny = sp.nx, sp.ny
        P = self.pitch = E.pitch_of(ny)
        shp = (nx, P)
        self.pol = 0 if sp.pol == 's' else 1
        self.f = [torch.zeros(shp, dtype=dtype, device=dev) for _ in range(3)]
        if self.pol == 0:
            cn = ['ce_e', 'ce_h']
        else:
            cn = ['ca_x', 'ca_y'] + (['da_x', 'da_y'] if geo.get('da_x') is not None else [])
        self.c = [E._pad_upload(geo[k], shp, dev) for k in cn]
        self.rtype, self.ctab = row_types([geo[k] for k in cn], shp, dev)
        self.axx, self.axy = E._Axis(geo['cx'], nx, dev), E._Axis(geo['cy'], ny, dev)
        wxe, wxh, wye, wyh = self.axx.w('e'), self.axx.w('h'), self.axy.w('e'), self.axy.w('h')
        z = lambda a, b: torch.zeros((a, b), dtype=torch.float32, device=dev)
        if self.pol == 0:   # hxy (nx, wyh), hyx (wxh, P), ezx (wxe, P), ezy (nx, wye)
            self.psi = [z(nx, max(1, wyh)), z(max(1, wxh), P), z(max(1, wxe), P), z(nx, max(1, wye))]
        else:               # hzx (wxh, P), hzy (nx, wyh), exy (nx, wye), eyx (wxe, P)
            self.psi = [z(max(1, wxh), P), z(nx, max(1, wyh)), z(nx, max(1, wye)), z(max(1, wxe), P)]
        src = geo['src']
        self.src_t = {k: torch.from_numpy(np.ascontiguousarray(src[k], np.float32)).to(dev)
                      for k in ('amp', 'ph1', 'ph2')}
        self.omega = src['omega']
        f0 = sp.f0
        self.steps_per_T = max(4, int(round((1.0 / f0) / sp.dt)))
        if window is None:
            self.n_acc = min(self.steps, 8 * self.steps_per_T)
            self.window = (self.steps - self.n_acc, self.steps)
        else:
            self.window = (int(window[0]), int(window[1]))
            self.n_acc = self.window[1] - self.window[0]
        self.kahan = bool(kahan)
        self.dft = torch.zeros((nx, P, 4 if self.kahan else 2), dtype=torch.float32, device=dev)
        s = N.Inst2D()
        s.pol, s.nx, s.ny, s.pitch = self.pol, nx, ny, P
        for q in range(3):
            s.f[q] = self.f[q].data_ptr()
        for q, t in enumerate(self.c):
            s.c[q] = t.data_ptr()
        s.ch = float(np.float32(sp.dt / (E.MU0 * sp.dx)))
        s.ax, s.ay = self.axx.ax, self.axy.ax
        for q in range(4):
            s.psi[q] = self.psi[q].data_ptr()
        s.pec = (ctypes.c_int * 4)(1, 1, 1, 1)
        s.src = N.Source(int(src['ix']), E._ptr(self.src_t['amp']), E._ptr(self.src_t['ph1']),
                         E._ptr(self.src_t['ph2']), len(src['amp']), 1, len(src['amp']))
        s.dft_n0, s.dft_n1 = self.window
        s.dft = self.dft.data_ptr()
        if self.rtype is not None:
            s.rtype, s.ctab = self.rtype.data_ptr(), self.ctab.data_ptr()
        self.s = s
        self.tb = None
        if tb:
            self._tb_buffers(dtype, dev)

    def _tb_buffers(self, dtype, dev):
        """Second buffers of the fields and psi, and the scratch of the K - 1
        intermediate psi levels (x strips (w, pitch), y strips (nx, w))."""
        nx, P = self.spec.nx, self.pitch
        self.f1 = [torch.zeros_like(t) for t in self.f]
        self.psi1 = [torch.zeros_like(t) for t in self.psi]
        w = [self.axy.w('h'), self.axx.w('h'), self.axx.w('e'), self.axy.w('e')] if self.pol == 0 else \
            [self.axx.w('h'), self.axy.w('h'), self.axy.w('e'), self.axx.w('e')]
        xs = [False, True, True, False] if self.pol == 0 else [True, False, False, True]
        tot = sum((wq * P if x else nx * wq) for wq, x in zip(w, xs))
        self.psi_lv = torch.zeros(max(1, (N.TB_K - 1) * tot), dtype=torch.float32, device=dev)
        t = N.TB2D()
        t.g = self.s
        for q in range(3):
            t.f1[q] = self.f1[q].data_ptr()
        for q in range(4):
            t.psi1[q] = self.psi1[q].data_ptr()
        t.psi_lv = self.psi_lv.data_ptr()
        t.dft_kahan = 1 if self.kahan else 0
        self.tb = t

    def _state(self):
        extra = (self.f1 + self.psi1 + [self.psi_lv]) if self.tb is not None else []
        return self.f + self.psi + [self.dft] + extra

    def nbytes(self):
        t = self._state() + self.c + ([self.ctab] if self.ctab is not None else [])
        return sum(x.numel() * x.element_size() for x in t)

    def reset(self):
        for t in self._state():
            t.zero_()

    def phasor(self):
        """(2/N) sum F e^{-i w t} on the nodes (nx, ny), complex128 (fdtd2d_core.py:879)."""
        a = self.dft[:, :self.spec.ny].double()
        if self.kahan:
            return (2.0 / self.n_acc) * torch.complex(a[..., 0] - a[..., 2], a[..., 1] - a[..., 3])
        return (2.0 / self.n_acc) * torch.complex(a[..., 0], a[..., 1])

    def overlap(self, ph=None):
        """Evanescent overlap K = I_tear / I_guided at the output window (0.8 of the
        length, 10 % wide) from <E^2> = |E|^2 / 2 (fdtd_analyzer.py:2880-2935)."""
        sp = self.spec
        ph = self.phasor() if ph is None else ph
        I = 0.5 * (ph.real ** 2 + ph.imag ** 2)
        nx, ny = sp.nx, sp.ny
        # the analyzer's display extents (um) and its index rounding (:2737-2747)
        L = nx * sp.dx * 1e6
        y0 = -sp.tear_m * 1e6
        y1 = y0 + ny * sp.dx * 1e6
        xi = lambda v: int(round(v / L * nx))
        vi = lambda v: int(round((v - y0) / (y1 - y0) * ny))
        c, w = 0.8 * L, 0.1 * L
        lo = max(0, xi(c - w / 2))
        hi = max(lo + 1, min(xi(c + w / 2), nx))
        j0, j1 = max(0, vi(0.0)), min(ny, vi(sp.stack.t_wg_um))   # core band; y = 0 is its bottom
        jt = max(0, vi(-sum(t for t, _ in sp.stack.layers)))    # the whole layer stack below
        band = lambda a, b: float(torch.mean(torch.sum(I[lo:hi, a:b], dim=1))) if b > a else 0.0
        g = band(j0, j1)
        return band(jt, j0) / g if g > 0 else 0.0


class Group:
    """Instances advanced by the same batched launches (tb: the temporally
    blocked step, LENS_TB_K steps per launch, warps over `chunk` rows)."""

    def __init__(self, insts, storage, by, dev, tb=False, chunk=64):
        self.insts, self.storage, self.by, self.dev = insts, storage, by, dev
        n = len(insts)
        self.lib = N.load()
        self.tb, self.chunk = bool(tb), int(chunk)
        self.steps = max(q.steps for q in insts)
        self.graph = None
        if self.tb:
            self.host = (N.TB2D * n)(*[q.tb for q in insts])
            first = (ctypes.c_int * (n + 1))()
            nu = self.lib.lens_tb2d_plan(self.host, n, self.chunk, first)
            N.check(min(0, nu))
            self.nunits = nu
            raw = ctypes.string_at(ctypes.addressof(self.host), ctypes.sizeof(self.host))
            self.dev_desc = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
            self.dev_first = torch.tensor(list(first), dtype=torch.int32, device=dev)
            return
        if any(q.kahan for q in insts):
            raise ValueError('the single-step batched kernels accumulate (re, im) DFTs: no compensated instances')
        self.host = (N.Inst2D * n)(*[q.s for q in insts])
        blk = (ctypes.c_int * (n + 1))()
        nblk = self.lib.lens_batch2d_plan(self.host, n, int(by), blk, None)
        N.check(min(0, nblk))
        owner = (ctypes.c_int * max(1, nblk))()
        N.check(min(0, self.lib.lens_batch2d_plan(self.host, n, int(by), blk, owner)))
        self.nblk = nblk
        raw = ctypes.string_at(ctypes.addressof(self.host), ctypes.sizeof(self.host))
        self.dev_desc = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        self.dev_blk = torch.tensor(list(blk), dtype=torch.int32, device=dev)
        self.dev_owner = torch.frombuffer(bytearray(owner), dtype=torch.int32).to(dev)

    def step(self, tab, n0, nsteps, stream=None):
        if self.tb:
            N.check(self.lib.lens_tb2d_step(self.host, ctypes.c_void_p(self.dev_desc.data_ptr()),
                                            ctypes.c_void_p(self.dev_first.data_ptr()), len(self.insts), self.chunk,
                                            self.storage, ctypes.byref(tab.s), int(n0), int(nsteps),
                                            E._stream_ptr(stream)))
            return
        N.check(self.lib.lens_batch2d_step(self.host, ctypes.c_void_p(self.dev_desc.data_ptr()),
                                           ctypes.c_void_p(self.dev_blk.data_ptr()),
                                           ctypes.c_void_p(self.dev_owner.data_ptr()), len(self.insts),
                                           self.storage, int(self.by), ctypes.byref(tab.s), int(n0), int(nsteps),
                                           E._stream_ptr(stream)))

    def step_persistent(self, tab, n0, nsteps, stream=None):
        """Steps [n0, n0 + nsteps) in one persistent cooperative launch
        (lens_batch2d_run); raises if a grid-barrier wait ran out."""
        if self.tb:
            raise ValueError('the persistent launch runs the single-step kernels')
        if not hasattr(self, 'sync'):
            self.sync = torch.zeros(2, dtype=torch.int32, device=self.dev)
            self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        N.check(self.lib.lens_batch2d_run(self.host, ctypes.c_void_p(self.dev_desc.data_ptr()),
                                          ctypes.c_void_p(self.dev_blk.data_ptr()),
                                          ctypes.c_void_p(self.dev_owner.data_ptr()), len(self.insts),
                                          self.storage, int(self.by), ctypes.byref(tab.s), int(n0), int(nsteps),
                                          ctypes.c_void_p(self.sync.data_ptr()), ctypes.c_void_p(self.err.data_ptr()),
                                          E._stream_ptr(stream)))

    def check(self):
        """Raise if the last persistent launch's barrier wait ran out."""
        if hasattr(self, 'err') and int(self.err.item()) != 0:
            raise N.LensError('persistent batched launch: a grid-barrier wait timed out (results invalid)')

    def launches(self, n0, n1):
        """Kernel launches of steps [n0, n1): H and E, plus the TM node DFT on window
        steps; one per LENS_TB_K steps for the temporally blocked step."""
        if self.tb:
            return (n1 - n0) // N.TB_K
        tm = [q.window for q in self.insts if q.pol == 1]
        extra = sum(1 for n in range(n0, n1) if any(a <= n < b for a, b in tm))
        return 2 * (n1 - n0) + extra

    def capture(self, tab):
        """Record the whole schedule [0, steps) as one CUDA graph."""
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.step(tab, 0, self.steps)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g
        return g


# rows per band up to which the resident sweep packs instances into one launch: on
# the 256-instance sweep (B200) 170 G cell-updates/s at 12, 174 G at 16, 156 G at 20
RS_PACK_ROWS = 16


class ResidentGroup:
    """FP32 instances advanced by ONE resident cooperative launch per call
    (lens_rs2d_run): every field value stays in registers from the first step
    to the last, bands of x rows exchanging one row per half step through L2.

    frames: per instance None or (every, tensor (nframes, nx, ny) TE / (nframes,
    nx, ny-1) TM) of snapshot frames written by the kernel; an instance with
    kahan=True accumulates its DFT compensated."""

    def __init__(self, insts, dev, frames=None):
        if any(q.f[0].dtype != torch.float32 for q in insts):
            raise ValueError('the resident launch keeps FP32 state: FP32 instances only')
        n = len(insts)
        self.insts, self.dev = insts, dev
        self.lib = N.load()
        self.steps = max(q.steps for q in insts)
        self.host = (N.Inst2D * n)(*[q.s for q in insts])
        rows, ctas, threads = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        N.check(self.lib.lens_rs2d_plan(self.host, n, ctypes.byref(rows), ctypes.byref(ctas), ctypes.byref(threads)))
        self.rows, self.ctas, self.threads = rows.value, ctas.value, threads.value
        raw = ctypes.string_at(ctypes.addressof(self.host), ctypes.sizeof(self.host))
        self.dev_desc = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
        nb = self.lib.lens_rs2d_scratch_bytes(self.ctas, self.threads)
        self.scratch = torch.empty(max(8, nb), dtype=torch.uint8, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.out = (N.RsOut2D * n)()
        self._frames = []
        for k, q in enumerate(insts):
            self.out[k].kahan = 1 if q.kahan else 0
            fr = frames[k] if frames is not None else None
            if fr is not None:
                every, t = fr
                self.out[k].frames, self.out[k].every, self.out[k].nframes = t.data_ptr(), int(every), int(t.shape[0])
                self._frames.append(t)

    @staticmethod
    def fits(insts, max_rows=None):
        """True when lens_rs2d_plan places these instances on this device (with
        at most max_rows rows per band, when given)."""
        n = len(insts)
        if n < 1 or n > N.RS_MAX_INST:
            return False
        host = (N.Inst2D * n)(*[q.s for q in insts])
        r, c, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ok = N.load().lens_rs2d_plan(host, n, ctypes.byref(r), ctypes.byref(c), ctypes.byref(t)) == 0
        return ok and (max_rows is None or r.value <= max_rows)

    def step(self, tab, n0, nsteps, stream=None):
        N.check(self.lib.lens_rs2d_run(self.host, ctypes.c_void_p(self.dev_desc.data_ptr()), self.out,
                                       len(self.insts), ctypes.byref(tab.s), int(n0), int(nsteps),
                                       ctypes.c_void_p(self.scratch.data_ptr()), self.scratch.numel(),
                                       ctypes.c_void_p(self.err.data_ptr()), E._stream_ptr(stream)))

    def check(self):
        """Raise if the last launch's wait between bands ran out."""
        if int(self.err.item()) != 0:
            raise N.LensError('resident 2D launch: a wait between bands timed out (results invalid)')

    def launches(self, n0, n1):
        return 1 if n1 > n0 else 0


class Sweep:
    """A batched sweep of 2D solves (one shared time step and wavelength).

    storage: 'f32' | 'f16' | 'bf16'.  by: rows per 32-lane tile; budget: bytes of
    resident state per group (None: one group).  autotune() chooses both."""

    def __init__(self, specs, steps, storage='f32', by=8, budget=None, device=None, geos=None, tb=False,
                 chunk=64, resident=False, resident_rows=RS_PACK_ROWS):
        dev = self.dev = E._device(device)
        self.tb, self.chunk = bool(tb), int(chunk)
        self.resident, self.resident_rows = bool(resident), resident_rows
        if self.resident and (self.tb or storage != 'f32'):
            raise ValueError('the resident sweep keeps FP32 state on chip: storage f32, tb False')
        if self.tb and int(steps) % (2 * N.TB_K):
            raise ValueError(f'the temporally blocked sweep runs in spans of {2 * N.TB_K} steps')
        if storage not in DTYPES:
            raise ValueError(f'storage {storage!r}: one of {sorted(DTYPES)}')
        self.storage_name = storage
        self.storage, dtype = DTYPES[storage]
        dts = {round(sp.dt * 1e30) for sp in specs}
        lams = {sp.lam_nm for sp in specs}
        if len(dts) != 1 or len(lams) != 1:
            raise ValueError('a batched sweep shares one time step and one wavelength')
        self.steps = int(steps)
        geos = geos if geos is not None else [None] * len(specs)
        self.insts = [Instance(sp, steps, dtype, dev, geo, tb=self.tb) for sp, geo in zip(specs, geos)]
        sp0 = specs[0]
        self.table = E.StepTable(0, self.steps, sp0.dt, self.insts[0].omega, 2 * np.pi * sp0.f0,
                                 E.cw_envelope(sp0.f0, sp0.ramp_periods), device=dev)
        self.by, self.budget = by, budget
        self.groups = self._groups(by, budget)
        self.tuned = None

    def _groups(self, by, budget):
        if self.resident:
            return self._resident_groups()
        order = sorted(range(len(self.insts)), key=lambda q: -self.insts[q].nbytes())
        groups, cur, size = [], [], 0
        for q in order:
            b = self.insts[q].nbytes()
            if cur and budget is not None and size + b > budget:
                groups.append(cur)
                cur, size = [], 0
            cur.append(self.insts[q])
            size += b
        if cur:
            groups.append(cur)
        return [Group(g, self.storage, by, self.dev, tb=self.tb, chunk=self.chunk) for g in groups]

    def _resident_groups(self):
        """Instances packed into resident launches in order of height (similar
        column counts share a launch's threads): an instance joins the current
        launch while the launch's bands stay within resident_rows rows (longer
        bands cost more per row than they save in waits)."""
        order = sorted(self.insts, key=lambda q: (q.spec.ny, q.spec.nx))
        groups, cur = [], []
        for q in order:
            if cur and not ResidentGroup.fits(cur + [q], self.resident_rows):
                groups.append(cur)
                cur = []
            cur.append(q)
        if cur:
            groups.append(cur)
        for g in groups:
            if not ResidentGroup.fits(g):
                raise ValueError('an instance does not fit the resident launch: use the batched sweep')
        return [ResidentGroup(g, self.dev) for g in groups]

    def cells(self):
        return sum(q.spec.nx * q.spec.ny for q in self.insts)

    def reset(self):
        for q in self.insts:
            q.reset()

    def autotune(self, candidates=((8, None), (4, None), (8, 96 << 20), (4, 96 << 20), (8, 48 << 20), (2, 96 << 20)),
                 probe_steps=24):
        """Time `probe_steps` batched steps of every (rows per tile, group budget)
        candidate on this sweep, keep the fastest, reset the fields.  The
        temporally blocked sweep tunes (rows per chunk, group budget) instead."""
        if self.tb:
            return self._autotune_tb()
        if self.resident:   # one launch per group, its band plan fixed by the device
            self.tuned = [dict(rows=g.rows, ctas=g.ctas, threads=g.threads, instances=len(g.insts))
                          for g in self.groups]
            return self.tuned
        res = []
        for by, budget in candidates:
            groups = self._groups(by, budget)
            for g in groups:              # warm-up
                g.step(self.table, 0, 2)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for g in groups:
                g.step(self.table, 2, probe_steps)
            torch.cuda.synchronize()
            res.append(((time.perf_counter() - t0) / probe_steps, by, budget))
        self.reset()
        best = min(res, key=lambda r: r[0])
        self.by, self.budget = best[1], best[2]
        self.groups = self._groups(self.by, self.budget)
        self.tuned = [dict(by=b, budget=u, s_per_step=t) for t, b, u in res]
        return self.tuned

    def _autotune_tb(self, candidates=((64, None), (32, None), (128, None), (64, 96 << 20), (32, 96 << 20),
                                       (16, None)), probe_steps=24):
        span = 2 * N.TB_K
        probe_steps = max(span, probe_steps // span * span)
        res = []
        for chunk, budget in candidates:
            self.chunk = chunk
            groups = self._groups(self.by, budget)
            for g in groups:              # warm-up
                g.step(self.table, 0, span)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for g in groups:
                g.step(self.table, span, probe_steps)
            torch.cuda.synchronize()
            res.append(((time.perf_counter() - t0) / probe_steps, chunk, budget))
        self.reset()
        best = min(res, key=lambda r: r[0])
        self.chunk, self.budget = best[1], best[2]
        self.groups = self._groups(self.by, self.budget)
        self.tuned = [dict(chunk=c, budget=u, s_per_step=t) for t, c, u in res]
        return self.tuned

    def run(self, graphs=True, persistent=False):
        """Run every group's whole schedule (one CUDA graph per group, or with
        persistent=True one persistent cooperative launch per group); returns
        the number of kernel launches."""
        launches = 0
        if self.resident:
            for g in self.groups:
                g.step(self.table, 0, g.steps)
            torch.cuda.synchronize()
            for g in self.groups:
                g.check()
            return len(self.groups)
        if persistent:
            for g in self.groups:
                g.step_persistent(self.table, 0, g.steps)
            torch.cuda.synchronize()
            for g in self.groups:
                g.check()
            return len(self.groups)
        for g in self.groups:
            if graphs:
                if g.graph is None:
                    g.capture(self.table)
                g.graph.replay()
            else:
                g.step(self.table, 0, g.steps)
            launches += g.launches(0, g.steps)
        return launches

    def results(self):
        out = []
        for q in self.insts:
            ph = q.phasor()
            out.append(dict(pol=q.spec.pol, nx=q.spec.nx, ny=q.spec.ny, phasor=ph, K=q.overlap(ph)))
        return out


def gated_sweep(specs, steps, storage='f16', tol=1e-4, probe_every=16, by=8, budget=None, device=None,
                geos=None, resident=True):
    """A sweep whose FP16 / BF16 field storage is accepted only where it meets
    `tol` (relative L2 phasor error).

    Reduced storage rounds every stored field value to 11 (FP16) or 8 (BF16)
    significant bits, so its error depends on the instance.  The gate probes
    every `probe_every`-th instance of each polarisation in both the reduced
    storage and FP32; a polarisation keeps the reduced storage for its other
    instances only if every one of its probes' phasor error against FP32 is
    within tol / 2 (half the bar, as margin for the instances not probed), and
    runs in FP32 otherwise.  Probes keep their FP32 results.  resident: the FP32
    runs use resident launches (Sweep(resident=True)) where the instances fit.

    Returns (results in the order of specs, each with its 'storage', and a
    report: the probes' errors, the accepted polarisations and the instance
    counts per storage)."""
    if storage not in ('f16', 'bf16'):
        raise ValueError(f'gated storage {storage!r}: f16 or bf16')
    geos = list(geos) if geos is not None else [build_2d(sp) for sp in specs]
    n = len(specs)
    probes = []
    for pol in ('s', 'p'):
        idx = [q for q in range(n) if specs[q].pol == pol]
        probes += idx[::max(1, int(probe_every))]
    probes.sort()
    def sub(ids, st):
        """The sweep of instances ids in storage st; FP32 on resident launches
        when `resident` and they fit the chip, else on the batched launches."""
        kw = dict(by=by, budget=budget, device=device, geos=[geos[q] for q in ids])
        if st == 'f32' and resident:
            try:
                return Sweep([specs[q] for q in ids], steps, st, resident=True, **kw)
            except ValueError:
                pass
        return Sweep([specs[q] for q in ids], steps, st, **kw)
    out = [None] * n
    errs = {}
    if probes:
        ref = sub(probes, 'f32')
        ref.run()
        r32 = ref.results()
        del ref
        red = sub(probes, storage)
        red.run()
        for q, a, b in zip(probes, r32, red.results()):
            errs[q] = float((b['phasor'] - a['phasor']).abs().norm() / max(float(a['phasor'].abs().norm()), 1e-300))
            out[q] = dict(a, storage='f32')
        del red
    ok = {pol: all(errs[q] <= 0.5 * tol for q in probes if specs[q].pol == pol) and
          any(specs[q].pol == pol for q in probes) for pol in ('s', 'p')}
    rest = [q for q in range(n) if out[q] is None]
    for st, ids in ((storage, [q for q in rest if ok[specs[q].pol]]), ('f32', [q for q in rest if not ok[specs[q].pol]])):
        if ids:
            sw = sub(ids, st)
            sw.run()
            for q, r in zip(ids, sw.results()):
                out[q] = dict(r, storage=st)
            del sw
    report = dict(storage=storage, tol=tol, probe_every=int(probe_every),
                  probes=[dict(index=q, pol=specs[q].pol, err=errs[q]) for q in probes],
                  accepted={pol: bool(v) for pol, v in ok.items()},
                  n_reduced=sum(1 for r in out if r['storage'] == storage),
                  n_f32=sum(1 for r in out if r['storage'] == 'f32'))
    return out, report
