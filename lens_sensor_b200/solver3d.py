"""One 3D solve on the GPU: setup, the run_3d time-stepping schedule and its
results.  This is the engine behind fdtd3d_core.run_3d's full-domain CPML path
(planar_3d/fdtd3d_core.py:793-1308):

  * detector boxes of |E|^2 every step (:1139-1142), the input box kept
    downstream of the source and entry facet (flux.py:64-74),
  * time-averaged |E|^2 every steps_per_T//8 steps in the second half (:1144-1148),
  * steady-state DFT over the last 8 periods on the selected components and
    the plane-flux DFT (:1150-1158),
  * the convergence DFT of the driven component on the z mid-plane for the
    window before (:1159-1175).
"""
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import engine as E
from .geometry import Spec3D, build_3d


# one worker that prepares host read-back buffers while the device steps
_HOST_POOL = ThreadPoolExecutor(1, thread_name_prefix='lens-host-stage')


def guard_in_plane(i_in, src_ix, n_max, margin=5):
    """Input detector plane at least `margin` cells downstream of the source
    (common/flux.py:64-74)."""
    lo = int(src_ix) + int(margin)
    return int(i_in) if i_in >= lo else min(lo, int(n_max) - 2)


def schedule_3d(sp: Spec3D, steps_total, x_facet_um):
    """The run_3d schedule of a solve of `steps_total` steps (torch-free, so the
    oracle's FP64 replay of a workload uses the same windows and boxes):
    steady-state DFT over the last 8 periods and the convergence window before
    it (fdtd3d_core.py:757-758, 1150-1175), |E|^2 every steps_per_T // 8 steps
    of the second half (:1144-1148), the input / output detector boxes
    (:1038-1062, the input box kept downstream of the source and facet) and the
    flux planes.  x_facet_um: the entry facet (geometry.build_3d)."""
    Nx = sp.nx
    dx_um = sp.dx_nm / 1000.0
    f0 = sp.f0
    n = int(steps_total)
    steps_per_T = max(4, int(round((1.0 / f0) / sp.dt)))
    n_acc = min(n, 8 * steps_per_T)
    y0_um = -sp.tear_um
    j_wg0 = int(round((0.0 - y0_um) / dx_um))
    j_wg1 = int(round((sp.stack.t_wg_um - y0_um) / dx_um))
    hw = max(2, int(round(1.0 / dx_um)))
    lx = Nx * dx_um

    def xr(xu):
        c = int(round(xu / dx_um))
        return max(0, c - hw), min(Nx, c + hw)
    iin0, iin1 = xr(0.2 * lx)
    iout0, iout1 = xr(0.8 * lx)
    ci = (iin0 + iin1) // 2
    sh = guard_in_plane(ci, max(sp.src_ix, int(round(x_facet_um / dx_um))), Nx) - ci
    iin0, iin1 = iin0 + sh, min(Nx, iin1 + sh)
    nsp = sp.n_sp
    return dict(omega=2 * np.pi * f0, steps_per_T=steps_per_T, n_acc=n_acc, dft=(n - n_acc, n),
                prev=(max(0, n - 2 * n_acc), n - n_acc), n_avg0=n // 2, m_I=max(1, steps_per_T // 8),
                # z range slice(n_sp, -n_sp) of each component (fdtd3d_core.py:1139-1142)
                boxes=[(iin0, iin1, j_wg0, j_wg1, nsp, -nsp), (iout0, iout1, j_wg0, j_wg1, nsp, -nsp)],
                planes={'in': max(1, (iin0 + iin1) // 2), 'out': max(1, (iout0 + iout1) // 2),
                        'src_up': sp.src_ix - 1, 'src_dn': sp.src_ix + 3})


class Solve3D:
    """Resident 3D solve.  comps: components whose phasor is accumulated
    (0 Ex, 1 Ey, 2 Ez; default the driven one).  engine: 'fused' (one step per
    launch, lens_fdtd3d_step), 'tb' (two steps per launch with the epilogues
    fused, lens_fdtd3d_step_tb) or 'twopass' (in place, two passes per step)."""

    def __init__(self, spec: Spec3D, steps_total, comps=None, fused=True, device=None, geo=None, engine=None,
                 tb_chunk=40):
        engine = engine or ('fused' if fused else 'twopass')
        fused = engine != 'twopass'
        self.engine = engine
        self.spec = sp = spec
        self.steps_total = int(steps_total)
        t0 = time.perf_counter()
        self.geo = geo if geo is not None else build_3d(sp)
        self.t_setup_host = time.perf_counter() - t0
        g = self.geo
        Nx, Ny, Nz = sp.nx, sp.ny, sp.nz
        dx_um = sp.dx_nm / 1000.0
        self.grid = E.Grid3D(Nx, Ny, Nz, sp.dx, sp.dt, g['ce'], g['da'], g['cpml'], g['src'],
                             src_comp=sp.src_comp, fused=fused, device=device, tb=engine == 'tb',
                             tb_chunk=tb_chunk)
        self.h2d_bytes = sum(a.nbytes for a in g['ce']) + (0 if g['da'] is None else sum(a.nbytes for a in g['da'])) \
            + sum(np.asarray(g['src'][k]).nbytes for k in ('amp', 'ph1', 'ph2'))
        sc = schedule_3d(sp, self.steps_total, g['x_facet_um'])
        self.omega, self.steps_per_T, self.n_acc = sc['omega'], sc['steps_per_T'], sc['n_acc']
        self.dft, self.prev, self.n_avg0, self.m_I = sc['dft'], sc['prev'], sc['n_avg0'], sc['m_I']
        self.boxes, self.planes = sc['boxes'], sc['planes']
        f0 = sp.f0
        n = self.steps_total
        self.comps = tuple(comps) if comps is not None else (sp.src_comp,)
        src_shape = (Ny - 1, Nz) if sp.src_comp == 1 else (Ny, Nz - 1)
        self.kc = src_shape[1] // 2
        self.table = E.StepTable(0, n, sp.dt, g['src']['omega'], self.omega,
                                 E.cw_envelope(f0, sp.ramp_periods), device=device)
        self.epi = E.Epi3D(self.grid, boxes=self.boxes, dft=self.dft, comps=self.comps,
                           planes=self.planes, conv=(self.kc, self.prev), iavg=True)
        self.n = 0
        self.launches = 0

    def iavg_steps(self, n0, n1):
        """Steps in [n0, n1) after which |E|^2 is accumulated."""
        a = max(n0, self.n_avg0)
        a += (-(a - self.n_avg0)) % self.m_I
        return list(range(a, n1, self.m_I))

    def run(self, n1=None, stream=None):
        """Advance from the current step to n1 (default: the end of the schedule)."""
        n1 = self.steps_total if n1 is None else min(int(n1), self.steps_total)
        n = self.n
        fused = self.grid.s.f[1][0] is not None
        for m in self.iavg_steps(n, n1) + [None]:
            stop = n1 if m is None else m + 1
            if stop > n:
                if self.engine == 'tb':
                    self.launches += self.grid.step_tb(self.table, n, stop - n, self.epi, stream)
                else:
                    self.grid.step(self.table, n, stop - n, self.epi, stream)
                    self.launches += self._launches(n, stop, fused)
                n = stop
            if m is not None:
                self.grid.accum_e2(self.epi.iavg, stream=stream)
                self.launches += 1
        self.n = n
        return self

    def _launches(self, n0, n1, fused):
        """Kernel launches of steps [n0, n1): fused, one step kernel and one box-sum
        kernel (every detector box), plus the window epilogue on DFT /
        convergence-window steps; two passes otherwise."""
        if not fused:
            return 2 * (n1 - n0)
        w0, w1 = self.prev[0], self.dft[1]
        return (n1 - n0) * (1 + (1 if self.boxes else 0)) + max(0, min(n1, w1) - max(n0, w0))

    # ---------------------------------------------------------------- results
    def phasor(self, comp=None):
        """Complex CW amplitude (2/N) sum F e^{-i w t} (fdtd3d_core.py:1271)."""
        comp = self.spec.src_comp if comp is None else comp
        return (2.0 / self.n_acc) * self.epi.phasor(comp)

    def _host_buffers(self, comps, pinned=False):
        """Host complex64 destinations (nx, ny, pitch) of the phasor read-back:
        page-locked torch tensors, or numpy arrays written once so that their
        pages are resident before the copy."""
        out = {}
        for c in comps:
            shape = tuple(self.epi.dft[c].shape[:3])
            if pinned:
                out[c] = torch.empty(shape, dtype=torch.complex64, pin_memory=True)
            else:
                a = np.empty(shape, np.complex64)
                a.view(np.float32).fill(0.0)
                out[c] = a
        return out

    def stage_host(self, comps=None, pinned=False):
        """Prepare the host destinations of phasors_host(comps) on a background
        thread, so that it overlaps the stepping (call before run(); the
        launches run without the GIL).  pinned: page-locked buffers from torch's
        host cache.  The copy back then runs at the link's rate (0.013 s for
        the three 189 MB phasors of a 480 x 192 x 256 grid, against 0.03-0.09 s
        pageable), but a first allocation of that size holds up the kernel
        launches of the concurrent run (0.19 s), so it pays only once the cache
        holds the blocks, for repeated solves in one process."""
        comps = self._accumulated(comps)
        self._staged = (comps, _HOST_POOL.submit(self._host_buffers, comps, pinned))
        return self

    def _accumulated(self, comps):
        comps = self.comps if comps is None else tuple(int(c) for c in comps)
        bad = [c for c in comps if c not in self.comps]
        if bad:
            raise ValueError(f'components {bad} are not accumulated by this solve (comps={self.comps})')
        return comps

    def phasors_host(self, comps=None, stream=None):
        """{comp: (2/N) sum F e^{-i w t}} as host complex64 arrays in each
        component's shape, the dtype of the reference's CW amplitude
        (fdtd3d_core.py:1271, (2/n) times a complex64 accumulator).

        Each component is scaled on the device and copied back in one transfer
        on `stream` (default: the current stream), into the buffers stage_host()
        prepared if it was called for these components, else into new ones.
        Returns once the copies have ended."""
        comps = self._accumulated(comps)
        st = stream if stream is not None else torch.cuda.current_stream()
        staged, self._staged = getattr(self, '_staged', None), None
        host = staged[1].result() if staged is not None and set(comps) <= set(staged[0]) else {}
        host.update(self._host_buffers([c for c in comps if c not in host]))
        scale = 2.0 / self.n_acc
        with torch.cuda.stream(st):
            for c in comps:
                h = host[c]
                pinned = isinstance(h, torch.Tensor)
                (h if pinned else torch.from_numpy(h)).copy_(torch.view_as_complex(self.epi.dft[c]) * scale,
                                                             non_blocking=pinned)
        st.synchronize()
        host = {c: (h.numpy() if isinstance(h, torch.Tensor) else h) for c, h in host.items()}
        self.d2h_bytes = sum(host[c].nbytes for c in comps)
        nx, ny, nz = self.spec.nx, self.spec.ny, self.spec.nz
        shape = {0: (nx - 1, ny, nz), 1: (nx, ny - 1, nz), 2: (nx, ny, nz - 1)}
        return {c: host[c][:shape[c][0], :shape[c][1], :shape[c][2]] for c in comps}

    def results(self, stream=None):
        """Scalars of the finished solve; waits for `stream` (default: the device)."""
        sp, ep = self.spec, self.epi
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.synchronize()
        self.grid.check_flag()
        dx = sp.dx
        box = ep.box_acc.double().cpu().numpy()
        P_in, P_out = float(box[0]) * dx ** 3, float(box[1]) * dx ** 3
        S_in, S_out = ep.flux('in', self.n_acc), ep.flux('out', self.n_acc)
        S_up, S_dn = ep.flux('src_up', self.n_acc), ep.flux('src_dn', self.n_acc)
        a = ep.conv_last.double()
        b = ep.conv_prev.double()
        na, nb = self.n_acc, self.prev[1] - self.prev[0]
        ca = torch.complex(a[..., 0] - a[..., 2], a[..., 1] - a[..., 3]) / max(na, 1)
        cb = torch.complex(b[..., 0] - b[..., 2], b[..., 1] - b[..., 3]) / max(nb, 1)
        rel = float(torch.linalg.norm(ca - cb) / max(float(torch.linalg.norm(ca)), 1e-30)) if nb > 0 else float('nan')
        n_I = len(self.iavg_steps(0, self.steps_total))
        return dict(P_in=P_in, P_out=P_out, transmission=(S_out / S_in if S_in else P_out / max(P_in, 1e-30)),
                    transmission_intensity=P_out / max(P_in, 1e-30), S_in=S_in, S_out=S_out,
                    p_in_si=S_in * dx * dx, p_emit=(S_dn - S_up) * dx * dx, cw_rel_change=rel,
                    n_iavg=n_I, steps_total=self.steps_total)
