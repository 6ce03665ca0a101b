"""3D stitch (domain decomposition along x) on the engine: the window plan and
the resident stepping of one stitch job, shared by the drop-in
fdtd3d_core.run_3d_stitched and the serving loop.

Follows planar_3d/fdtd3d_core.py:1311-1782 (run_3d_stitched):

  * windows of Nx_win cells slide by S cells, overlap O = Nx_win - S; the last
    window ends flush with the domain (:1375-1386);
  * interior windows carry an absorber extension of _EXT = max(n_sp, 10) + 4
    cells behind their end with a CPML, not assembled (:1368-1372, :1558-1560);
  * window 0 carries the VCSEL, CPML + PEC on every face; a window w > 0 is
    open at x-lo and driven on its first O planes by the previous window's
    complex Ex, Ey, Ez amplitudes with a cosine taper (:1515-1517, :1605-1617);
  * every window runs steps_win = int(3 transit / dt) + 400 steps and
    accumulates, over its last 8 periods, the CW amplitude of the driven
    component, the handoff amplitudes of the next window's overlap, the plane
    fluxes of the planes it assembles and <|E|^2> every T/8 (:1638-1650);
  * assembly keeps [0, Nx_win) of window 0 and [O, Nx_win) of later windows
    (the last to the domain end) (:1666-1678).

The handoff amplitudes never leave the device.
"""

import numpy as np
import torch

from .geometry import Sphere, Spec3D, Stack, air_path_um, build_3d
from .physics import C0

N_AIR = 1.0


def guard_in_plane(i_in, src_ix, n_max, margin=5):
    """Input detector plane at least `margin` cells behind the source (flux.py:63-74)."""
    lo = int(src_ix) + int(margin)
    return int(i_in) if i_in >= lo else min(lo, int(n_max) - 2)


class StitchPlan:
    """Window plan and physics of a stitch job (fdtd3d_core.py:1311-1400, 1480-1550).

    stack: geometry.Stack (core index, thickness, layers below, substrate);
    beads: list of geometry.Sphere in global x."""

    def __init__(self, st: Stack, tear_um, lx_um, ly_um, lz_um, dx_nm, window_w_um, slide_um, wg_n,
                 pol='s', lam_nm=850.0, beads=(), n_sponge=None, sponge_um=1.2, input_gap_um=0.0,
                 waist_um=3.0, waist_z_um=3.0, tilt_deg=0.0, offset_y_um=0.0, offset_z_um=0.0,
                 wg_width_um=None, n_clad_side=N_AIR, det_in_um=None, det_out_um=None, n_g_factor=1.10):
        self.st, self.beads = st, list(beads)
        self.tear_um, self.lx_um, self.ly_um, self.lz_um = float(tear_um), lx_um, ly_um, lz_um
        self.dx_nm = dx_nm
        dx = self.dx = dx_nm * 1e-9
        dx_um = self.dx_um = dx_nm / 1000.0
        self.dt = dt = 0.5 * dx / (C0 * np.sqrt(3))
        self.lam_nm = lam_nm
        self.f0 = f0 = C0 / (lam_nm * 1e-9)
        self.omega = 2 * np.pi * f0
        self.y0_um, self.z0_um = -self.tear_um, -lz_um / 2.0
        self.Ny, self.Nz = int(round(ly_um / dx_um)), int(round(lz_um / dx_um))
        self.Nx_full = Nx_full = int(round(lx_um / dx_um))
        self.Nx_win = Nx_win = min(int(round(window_w_um / dx_um)), Nx_full)
        self.S = S = max(1, min(int(round(slide_um / dx_um)), Nx_win))
        self.O = Nx_win - S
        n_sp = int(n_sponge) if n_sponge else int(np.ceil(float(sponge_um) / dx_um))
        self.n_sp = n_sp = min(max(8, n_sp), max(8, min(Nx_win, self.Ny, self.Nz) // 6))
        self.vd = float(input_gap_um or 0.0)
        self.src_ix = n_sp + 6
        self.x_src_um = self.src_ix * dx_um
        self.x_wg_start_um = self.x_src_um + air_path_um(self.vd, dx_um)
        self.EXT = max(n_sp, 10) + 4
        self.x_wg_end_um = lx_um + self.EXT * dx_um
        self.n_win = (int(np.ceil((Nx_full - Nx_win) / S)) + 1) if Nx_full > Nx_win else 1
        transit = window_w_um * 1e-6 * n_g_factor * wg_n / C0
        self.steps_win = int(3.0 * transit / dt) + 400
        steps_per_T = max(4, int(round((1.0 / f0) / dt)))
        self.n_acc = steps_per_T * 8
        self.base = self.steps_win - self.n_acc       # epilogue window start (may be < 0)
        self.n_w0 = max(0, self.base)
        self.acc_n = self.steps_win - self.n_w0
        self.m_I = max(1, int(round((1.0 / f0) / dt)) // 8)
        self.pol = 'p' if str(pol).lower() in ('p', 'tm') else 's'
        self.comp = 1 if self.pol == 'p' else 2
        self.Nj, self.Nk = (self.Ny - 1, self.Nz) if self.pol == 'p' else (self.Ny, self.Nz - 1)
        self.spec_kw = dict(lam_nm=lam_nm, waist_um=waist_um, waist_z_um=waist_z_um, offset_y_um=offset_y_um,
                            offset_z_um=offset_z_um, tilt_deg=tilt_deg, vcsel_distance_um=self.vd,
                            end_facet_um=0.0, wg_width_um=wg_width_um, n_clad_side=n_clad_side)
        # detector planes in global x (fdtd3d_core.py:1521-1550)
        self.det_in_um = 0.2 * lx_um if det_in_um is None else det_in_um
        self.det_out_um = 0.8 * lx_um if det_out_um is None else det_out_um
        self.j_wg0 = int(round((0.0 - self.y0_um) / dx_um))
        self.j_wg1 = int(round((st.t_wg_um - self.y0_um) / dx_um))
        self.gi = guard_in_plane(min(max(int(round(self.det_in_um / dx_um)), 1), Nx_full - 2),
                                 max(self.src_ix, int(round(self.x_wg_start_um / dx_um))), Nx_full)
        self.det_in_um = self.gi * dx_um
        self.go = min(max(int(round(self.det_out_um / dx_um)), 1), Nx_full - 2)
        self.windows = []
        for w in range(self.n_win):
            g0, last = self.gx0(w), w == self.n_win - 1
            glo = 0 if w == 0 else g0 + self.O
            ghi = Nx_full if last else min(g0 + Nx_win, Nx_full)
            fpl = {k: g - g0 for k, g in (('in', self.gi), ('out', self.go)) if glo <= g < ghi and g - g0 >= 1}
            if w == 0:
                fpl.update(src_up=self.src_ix - 1, src_dn=self.src_ix + 3)
            self.windows.append((g0, last, fpl))

    def gx0(self, w):
        """First global plane of window w; the last window ends flush with the domain."""
        return min(w * self.S, max(self.Nx_full - self.Nx_win, 0))

    def nxw(self, w):
        return self.Nx_win + (0 if w == self.n_win - 1 else self.EXT)

    def planes_covered(self):
        return all(any(k in fpl for _, _, fpl in self.windows) for k in ('in', 'out'))

    def spec(self, w):
        """Spec3D of window w in global x."""
        return Spec3D(self.pol, self.nxw(w), self.Ny, self.Nz, self.dx_nm, self.st, self.tear_um, self.beads,
                      npml=10, pec_faces=(('xmin',) if w > 0 else ()), x0_um=self.gx0(w) * self.dx_um,
                      x_wg_end_um=self.x_wg_end_um, n_sp_cells=self.n_sp, **self.spec_kw)

    def taper(self):
        """w_i = (1 + cos(pi i / (O - 1))) / 2 (fdtd3d_core.py:1516-1517)."""
        O = self.O
        return (0.5 * (1.0 + np.cos(np.pi * np.arange(O) / max(O - 1, 1)))).astype(np.float32)

    def window_bytes(self, ncomp=3, lossy=None):
        """Device bytes of the largest window on the engine: two field + psi
        buffers, coefficients (+ damping), DFT sums, Iavg, handoff."""
        lossy = self.st.lossy if lossy is None else lossy
        P = -(-self.Nz // 32) * 32
        cells = self.nxw(0) * self.Ny * P
        hand = 3 * max(self.O, 1) * self.Ny * P * 8
        return cells * 4 * (2 * (6 + 12) + 3 + (3 if lossy else 0) + 2 * ncomp + 1) + 2 * hand

    def cell_updates(self):
        return sum(self.nxw(w) * self.Ny * self.Nz for w in range(self.n_win)) * self.steps_win


class FluxSum:
    """Plane DFTs summed over the windows that carry the plane, with their
    counts (one running PlaneFluxDFT across windows, fdtd3d_core.py:1552, 1644)."""

    def __init__(self, engine):
        self.E = engine
        self.acc, self.n = {}, {}

    def add(self, key, pairs, n):
        if key not in self.acc:
            self.acc[key] = [[sg, aE.clone(), aH.clone()] for sg, aE, aH in pairs]
            self.n[key] = 0
        else:
            for a, (sg, aE, aH) in zip(self.acc[key], pairs):
                a[1] += aE
                a[2] += aH
        self.n[key] += int(n)

    def has(self, key):
        return self.n.get(key, 0) > 0

    def flux(self, key):
        if not self.has(key):
            return float('nan')
        return self.E.plane_flux(self.acc[key], self.n[key])


class StitchSolve:
    """Resident stepping of one stitch job on the engine module `engine`.

    sink(w, g_lo, g_hi, Ew, Ia) receives each window's assembled slab: the CW
    amplitude Ew (complex64 host array, planes [g_lo, g_hi)) and <|E|^2> Ia
    (float32 host array).  advance(n) steps at most n steps and returns the
    steps taken; done is True after the last window."""

    def __init__(self, plan: StitchPlan, engine, sink, device=None, stream=None, pool=None, geo0=None):
        """stream: CUDA stream of the job's kernels (None: the current stream);
        pool: executor that builds the next window's geometry while the current
        window runs (None: built when the window opens); geo0: window 0's
        geometry when already built."""
        self.p, self.E, self.sink = plan, engine, sink
        self.device, self.stream, self.pool = device, stream, pool
        self._next_geo = None
        self._geo0 = geo0
        self.tab = engine.StepTable(0, plan.steps_win, plan.dt, plan.omega, plan.omega,
                                    engine.cw_envelope(plan.f0), device=device)
        self.sc = torch.tensor(2.0 / max(plan.acc_n, 1), dtype=torch.float32)
        self.wtap = plan.taper()
        self.flux = FluxSum(engine)
        self.hand = None
        self.w = 0
        self.geo0 = None
        self.done = False
        self.steps_done = 0
        self._open(0)

    def _open(self, w):
        p, E = self.p, self.E
        if w == 0 and self._geo0 is not None:
            geo, self._geo0 = self._geo0, None
        else:
            geo = self._next_geo.result() if self._next_geo is not None else build_3d(p.spec(w))
        self._next_geo = None
        if self.pool is not None and w + 1 < p.n_win:
            self._next_geo = self.pool.submit(build_3d, p.spec(w + 1))
        if w == 0:
            self.geo0 = geo
        last = w == p.n_win - 1
        self.grid = E.Grid3D(p.nxw(w), p.Ny, p.Nz, p.dx, p.dt, geo['ce'], geo['da'], geo['cpml'],
                             geo['src'] if w == 0 else None, src_comp=p.comp,
                             pec=((1,) if w == 0 else (0,)) + (1,) * 5, fused=True, device=self.device)
        self.fpl = p.windows[w][2]
        self.epi = E.Epi3D(self.grid, dft=(p.n_w0, p.steps_win), comps=(p.comp,) if last else (0, 1, 2),
                           planes=self.fpl, iavg=True)
        self.drive = (E.Drive3D(self.grid, self.hand, self.wtap)
                      if (w > 0 and self.hand is not None and p.O > 0) else None)
        self.n, self.n_I = 0, 0
        if self.stream is not None:      # buffers were zeroed / uploaded on the current stream
            self.stream.wait_stream(torch.cuda.current_stream())

    def advance(self, nmax):
        """Step the current window by at most nmax steps (to the next <|E|^2>
        sample, every m_I steps, or the window end); close the window when it ends."""
        if self.done:
            return 0
        p = self.p
        taken = 0
        while taken < nmax and self.n < p.steps_win:
            n = self.n
            ev = p.n_w0 if n <= p.n_w0 else n + (p.base - n) % p.m_I
            ev = min(ev, p.steps_win - 1, n + (nmax - taken) - 1)
            self.grid.step(self.tab, n, ev - n + 1, self.epi, stream=self.stream, drive=self.drive)
            if ev >= p.base and (ev - p.base) % p.m_I == 0:
                self.grid.accum_e2(self.epi.iavg, stream=self.stream, nx=p.Nx_win)
                self.n_I += 1
            taken += ev - n + 1
            self.n = ev + 1
        self.steps_done += taken
        if self.n >= p.steps_win:
            self._close()
        return taken

    def _close(self):
        p, w, ep = self.p, self.w, self.epi
        g0, last, fpl = p.windows[w]
        if self.stream is not None:
            self.stream.synchronize()
        self.grid.check_flag()
        ph = ep.phasor(p.comp, kind='split')[:p.Nx_win]
        sc = self.sc.to(ph.device)
        Ew = torch.complex(ph.real.float() * sc, ph.imag.float() * sc)
        if not last and p.O > 0:             # handoff of Ex, Ey, Ez over the next overlap
            off = p.gx0(w + 1) - g0
            hand = []
            for c in range(3):
                a = ep.phasor(c, kind='hand')[off:off + p.O]
                hand.append(torch.complex(a.real.float() * sc, a.imag.float() * sc))
            self.hand = hand
        for key in fpl:
            self.flux.add(key, ep.plane_dft(key), p.acc_n)
        l_lo, g_lo = (0, 0) if w == 0 else (p.O, g0 + p.O)
        g_hi = p.Nx_full if last else min(g0 + p.Nx_win, p.Nx_full)
        l_hi = l_lo + (g_hi - g_lo)
        if g_hi > g_lo:
            ia = ep.iavg[l_lo:l_hi, :p.Nj, :p.Nk] * torch.tensor(1.0 / max(self.n_I, 1),
                                                                   dtype=torch.float32).to(ep.iavg.device)
            self.sink(w, g_lo, g_hi, Ew[l_lo:l_hi].cpu().numpy(), ia.cpu().numpy())
        self.grid = self.epi = self.drive = None
        if last:
            self.done = True
            self.hand = None
        else:
            self.w = w + 1
            self._open(self.w)

    def vcsel(self):
        """Emitted and reflected VCSEL power and the input-plane power (fdtd3d_core.py:1755-1760)."""
        p, f = self.p, self.flux
        dx = p.dx
        S_in = f.flux('in') if f.has('in') else None
        ok = f.has('src_up') and f.has('src_dn')
        return dict(p_in=(S_in * dx * dx if S_in is not None else None),
                    p_emit=((f.flux('src_dn') - f.flux('src_up')) * dx * dx) if ok else None,
                    p_refl=(-f.flux('src_up') * dx * dx) if ok else None)

    def transmission(self):
        f = self.flux
        if f.has('in') and f.has('out'):
            S_in, S_out = f.flux('in'), f.flux('out')
            if abs(S_in) > 0:
                return S_out / S_in
        return float('nan')
