"""Stand-in for lens_sensor_b200.engine built on the CPU oracle (TEST INFRASTRUCTURE).

Implements the slice of the engine's 2D interface that the drop-in driver
lens_sensor_b200.fdtd2d_core.run_beads calls (Grid2D, Epi2D, StepTable,
cw_envelope), stepping with oracle.fdtd_oracle.Grid2D in FP32 and accumulating
the epilogue exactly as the reference's loop does (fdtd2d_core.py:781-870).
Tests patch it in to check the driver's schedule (step count, detector
windows, DFT windows, CW convergence extension, snapshots, result keys) on the
CPU against the reference's own known answers.  It is never used by the
product.
"""
import numpy as np
import torch

from oracle import fdtd_oracle as O

F32 = np.float32


def cw_envelope(f0, ramp_periods=None):
    return lambda t: O.cw_envelope(float(t), f0, ramp_periods)


class StepTable:
    def __init__(self, t0, n, dt, omega_src, omega_dft, envelope, device=None):
        self.dt, self.envelope, self.omega = dt, envelope, omega_dft


class Grid2D:
    def __init__(self, pol, nx, ny, dx, dt, coef, cx, cy, src, pec=(1, 1, 1, 1), device=None, full_x=False):
        self.pol = 'p' if str(pol).lower() in ('p', 'tm') else 's'
        self.nx, self.ny, self.dx, self.dt = nx, ny, dx, dt
        if src is None:
            h = _NoSource()
        else:
            h = O.Huygens.__new__(O.Huygens)
            h.ix, h.omega = int(src['ix']), float(src['omega'])
            h.amp, h.ph1, h.ph2 = (np.asarray(src[k], F32) for k in ('amp', 'ph1', 'ph2'))
        self.g = O.Grid2D(self.pol, nx, ny, dx, dt, cx, cy, h, coef, F32, pec)

    def view(self, name):
        return torch.from_numpy(getattr(self.g, name[0].upper() + name[1:]).copy())

    def _state(self):
        names = (('Ez', 'Hx', 'Hy', 'p_hxy', 'p_hyx', 'p_ezx', 'p_ezy') if self.pol == 's' else
                 ('Ex', 'Ey', 'Hz', 'p_hzx', 'p_hzy', 'p_exy', 'p_eyx'))
        return names

    def take_shifted(self, other, n):
        """The reference's roll of the fields and the full-domain psi with the
        trailing rows zeroed (fdtd2d_core.py:1093-1102, boundaries.py:217-221)."""
        for q in self._state():
            a = np.roll(getattr(other.g, q), -n, axis=0)
            a[a.shape[0] - n:, :] = 0
            setattr(self.g, q, a)

    def step(self, table, n0, nsteps, epi=None, stream=None, drive=None):
        if self.g.src.omega is None:
            self.g.src.omega = table.omega
        for n in range(n0, n0 + nsteps):
            t = n * self.dt
            env = float(table.envelope(t))
            hook = (lambda F, t=t, env=env: drive.apply(F, table.omega, t, env)) if drive is not None else None
            self.g.step(n, env, before_pec=hook)
            if epi is not None:
                epi.after(n, t, self.g)


class Drive2D:
    """2D overlap drive exactly as fdtd2d_core.py:1439-1440 / 1462-1463 writes it."""

    def __init__(self, grid, hand, taper, env=None, cos_wt=None, sin_wt=None):
        self.D = np.asarray(torch.as_tensor(hand).numpy(), np.complex64)
        self.O = self.D.shape[0]
        self.w = np.asarray(taper, F32)[:, None]

    def apply(self, F, omega, t, env):
        din = env * np.real(self.D * np.exp(1j * omega * t))
        F[:self.O, :] = self.w * din + (1.0 - self.w) * F[:self.O, :]


class Epi2D:
    def __init__(self, grid, boxes=(), dft=None, dft_ex=False, prev=None, iavg_n0=None, planes=(),
                 dft_raw=False, ex2=False, sx_planes=(), box_split=False):
        nx, ny = grid.nx, grid.ny
        self.grid = grid
        self.boxes = [tuple(b) for b in boxes]
        self.box = np.zeros(len(self.boxes), np.float64)
        self.box_split = box_split
        self.sx_planes = dict(sx_planes)
        self.sx_tot = {k: np.float64(0.0) for k in self.sx_planes}
        self.win = tuple(dft) if dft is not None else (0, 0)
        self.win_prev = tuple(prev) if prev is not None else (0, 0)
        self.acc = np.zeros((nx, ny), np.complex64)
        self.acc_ex = np.zeros((nx, ny), np.complex64) if dft_ex else None
        self.acc_prev = np.zeros((nx, ny), np.complex64)
        self.iavg_n0 = iavg_n0
        self.acc_I = np.zeros((nx, ny), F32)
        self.planes = dict(planes)
        self.flux_acc = None
        self._omega = None
        # run_beads_stitched's own complex64 sums (fdtd2d_core.py:1441-1446, 1471):
        # TE Ez / TM Ey on its grid, TM Ex on the nodes, TM <Ex^2> on the nodes
        self.acc_st = np.zeros((nx, ny) if grid.pol == 's' else (nx, ny - 1), np.complex64)
        self.acc_exa = np.zeros((nx, ny), np.complex64)
        self.acc_ex2 = np.zeros((nx, ny), F32)
        self.ex2 = torch.from_numpy(self.acc_ex2) if ex2 else None

    def after(self, n, t, g):
        if self.flux_acc is None:
            self._omega = float(g.src.omega)
            self.flux_acc = O.PlaneFlux(self._omega, g.dt, F32)
        field = g.field()
        I_E = g.intensity(field)
        for q, (x0, x1, y0, y1) in enumerate(self.boxes):
            if self.box_split:      # fdtd2d_core.py:1148-1150: field^2 and <Ex^2> summed apart
                v = np.sum(field[x0:x1, y0:y1] ** 2, dtype=np.float64)
                if g.pol == 'p':
                    v = v + np.sum(O.tm_ex2_node(g.Ex)[x0:x1, y0:y1], dtype=np.float64)
                self.box[q] += v
            else:
                self.box[q] += np.sum(I_E[x0:x1, y0:y1], dtype=np.float64)
        for k, il in self.sx_planes.items():   # _sx_plane_2d (fdtd2d_core.py:489-497)
            if g.pol == 's':
                hy = 0.5 * (g.Hy[il - 1] + g.Hy[il])
                self.sx_tot[k] += -np.sum(g.Ez[il] * hy, dtype=np.float64)
            else:
                hz = 0.5 * (g.Hz[il - 1] + g.Hz[il])
                self.sx_tot[k] += np.sum(g.Ey[il] * hz, dtype=np.float64)
        if self.win[0] <= n < self.win[1]:
            ph = np.exp(-1j * self._omega * t)
            self.acc += field.astype(np.complex64) * ph
            if self.acc_ex is not None:
                self.acc_ex += g.ex_node().astype(np.complex64) * ph
            p64 = np.complex64(ph)
            if g.pol == 's':
                self.acc_st += g.Ez.astype(np.complex64) * p64
            else:
                self.acc_st += g.Ey.astype(np.complex64) * p64
                self.acc_ex2 += O.tm_ex2_node(g.Ex)
                self.acc_exa += g.ex_node().astype(np.complex64) * p64
            for k, il in self.planes.items():
                self.flux_acc.add(k, t, g.flux_pairs(il))
        elif self.win_prev[0] <= n < self.win_prev[1]:
            self.acc_prev += field.astype(np.complex64) * np.exp(-1j * self._omega * t)
        if self.iavg_n0 is not None and n >= self.iavg_n0:
            self.acc_I += I_E

    @property
    def box_acc(self):
        return torch.from_numpy(self.box.copy())

    def sx(self, name):
        return float(self.sx_tot[name])

    @property
    def iavg(self):
        return torch.from_numpy(self.acc_I.copy())

    def phasor(self, which='dft', kind=None):
        if kind == 'stitch':
            a = self.acc_exa if which == 'dft_ex' else self.acc_st
        else:
            a = dict(dft=self.acc, prev=self.acc_prev, dft_ex=self.acc_ex)[which]
        return torch.from_numpy(a.astype(np.complex128))

    def plane_dft(self, name):
        return [(sg, torch.from_numpy(aE.astype(np.complex128)), torch.from_numpy(aH.astype(np.complex128)))
                for sg, aE, aH in self.flux_acc.acc[name]]

    def restart_dft(self, window):
        self.acc_prev, self.acc = self.acc, np.zeros_like(self.acc)
        if self.acc_ex is not None:
            self.acc_ex[...] = 0
        self.flux_acc = O.PlaneFlux(self._omega, self.grid.dt, F32)
        self.win, self.win_prev = tuple(window), (0, 0)

    def flux(self, name, n_acc):
        return self.flux_acc.flux(name)


# ----------------------------------------------------------------------------- 3D
_COMP = {0: 'Ex', 1: 'Ey', 2: 'Ez'}
_FACES = ('xmin', 'xmax', 'ymin', 'ymax', 'zmin', 'zmax')


class _NoSource:
    """A stitch window without the VCSEL (fdtd3d_core.py:1609-1617)."""
    omega = None

    def inject(self, *a):
        pass


def plane_flux(pairs, n):
    """flux.py:45-57: complex64 products, complex128 sum."""
    s = 0.0
    for sign, aE, aH in pairs:
        e, h = aE.numpy().astype(np.complex64), aH.numpy().astype(np.complex64)
        s += sign * 0.5 * float(np.real(np.sum(e * np.conj(h), dtype=np.complex128)))
    return s * (2.0 / n) ** 2


class Drive3D:
    """Overlap drive of a stitch window, applied as fdtd3d_core.py:1614-1617 does."""

    def __init__(self, grid, hand, taper):
        self.hand = [np.asarray(torch.as_tensor(D).numpy(), np.complex64) for D in hand]
        self.O = len(taper)
        self.w = np.asarray(taper, F32)[:, None, None]

    def apply(self, g, omega, t, env):
        ph = np.complex64(np.exp(1j * omega * t))
        for F, D in zip((g.Ex, g.Ey, g.Ez), self.hand):
            F[:self.O] = self.w * (env * np.real(D * ph)) + (1.0 - self.w) * F[:self.O]


class Grid3D:
    """3D stand-in: oracle FP32 stepping in the reference loop order
    (fdtd3d_core.py:1106-1127; CPML step, PEC, source)."""

    def __init__(self, nx, ny, nz, dx, dt, ce, da, cpml, src, src_comp=1, pec=(1,) * 6, device=None,
                 fused=True):
        self.nx, self.ny, self.nz, self.dx, self.dt = nx, ny, nz, dx, dt
        if src is None:
            h = _NoSource()
        else:
            h = O.Huygens.__new__(O.Huygens)
            h.ix, h.omega = int(src['ix']), float(src['omega'])
            h.amp, h.ph1, h.ph2 = (np.asarray(src[k], F32) for k in ('amp', 'ph1', 'ph2'))
        self.src_comp = src_comp
        faces = tuple(f for f, on in zip(_FACES, pec) if on)
        self.g = O.Grid3D(nx, ny, nz, dx, dt, cpml, ce, da, h, _COMP[src_comp], F32, faces=faces)

    def view(self, name):
        return torch.from_numpy(getattr(self.g, name[0].upper() + name[1:]).copy())

    def _state(self):
        names = (('Ez', 'Hx', 'Hy', 'p_hxy', 'p_hyx', 'p_ezx', 'p_ezy') if self.pol == 's' else
                 ('Ex', 'Ey', 'Hz', 'p_hzx', 'p_hzy', 'p_exy', 'p_eyx'))
        return names

    def take_shifted(self, other, n):
        """The reference's roll of the fields and the full-domain psi with the
        trailing rows zeroed (fdtd2d_core.py:1093-1102, boundaries.py:217-221)."""
        for q in self._state():
            a = np.roll(getattr(other.g, q), -n, axis=0)
            a[a.shape[0] - n:, :] = 0
            setattr(self.g, q, a)

    def step(self, table, n0, nsteps, epi=None, stream=None, drive=None):
        if self.g.src.omega is None:
            self.g.src.omega = table.omega
        for n in range(n0, n0 + nsteps):
            t = n * self.dt
            env = float(table.envelope(t))
            self.g.step(n, env)
            if drive is not None:
                drive.apply(self.g, table.omega, t, env)
            if epi is not None:
                epi.after(n, t, self.g)

    def accum_e2(self, iavg, target=None, stream=None, nx=None):
        nx = self.nx if nx is None else nx
        O.accum_e2(iavg.numpy()[:nx], self.g.Ex[:nx - 1], self.g.Ey[:nx], self.g.Ez[:nx])

    def check_flag(self):
        pass


class Epi3D:
    """3D stand-in: the reference's per-step epilogue (fdtd3d_core.py:1139-1175):
    detector boxes, complex64 DFT of the driven component, plane-flux DFT and the
    convergence planes at z index kc."""

    def __init__(self, grid, boxes=(), dft=None, comps=(1,), planes=(), conv=None, iavg=False):
        self.grid = grid
        cshape = getattr(grid.g, _COMP[grid.src_comp]).shape

        def sl(a, b):
            return slice(a, b if b != 0 else None)
        self.boxes = [(sl(b[0], b[1]), sl(b[2], b[3]), sl(b[4], b[5])) for b in boxes]
        self.box = np.zeros(len(self.boxes), np.float64)
        self.win = tuple(dft)
        self.comps = tuple(comps)
        self.acc = {c: np.zeros(getattr(grid.g, _COMP[c]).shape, np.complex64) for c in comps}
        # run_3d_stitched's own accumulators (fdtd3d_core.py:1640-1649): float32
        # re/im of the volume and complex64 overlap handoff
        self.acc_re = {c: np.zeros(a.shape, F32) for c, a in self.acc.items()}
        self.acc_im = {c: np.zeros(a.shape, F32) for c, a in self.acc.items()}
        self.acc_hand = {c: np.zeros(a.shape, np.complex64) for c, a in self.acc.items()}
        self.planes = dict(planes)
        self.kc, self.prev_win = (conv[0], tuple(conv[1])) if conv is not None else (None, (0, 0))
        self.pl_a = np.zeros(cshape[:2], np.complex64)
        self.pl_b = np.zeros(cshape[:2], np.complex64)
        self._iavg = np.zeros(cshape, F32)
        self.iavg = torch.from_numpy(self._iavg)
        self.flux_acc = None
        self._omega = None

    def after(self, n, t, g):
        if self._omega is None:
            self._omega = float(g.src.omega)
            self.flux_acc = O.PlaneFlux(self._omega, g.dt, F32)
        for q, bx in enumerate(self.boxes):
            self.box[q] += g.box_e2(*bx)
        F = getattr(g, _COMP[self.grid.src_comp])
        if self.win[0] <= n < self.win[1]:
            ph = np.exp(-1j * self._omega * t)
            cs, sn = F32(np.cos(self._omega * t)), F32(np.sin(self._omega * t))
            e64 = np.complex64(np.exp(-1j * self._omega * t))
            for c in self.comps:
                Fc = getattr(g, _COMP[c])
                self.acc[c] += Fc.astype(np.complex64) * ph
                self.acc_re[c] += Fc * cs
                self.acc_im[c] -= Fc * sn
                self.acc_hand[c] += Fc * e64
            for k, il in self.planes.items():
                self.flux_acc.add(k, t, g.flux_pairs(il))
            if self.kc is not None:
                self.pl_b += F[:, :, self.kc].astype(np.complex64) * ph
        elif self.kc is not None and self.prev_win[0] <= n < self.prev_win[1]:
            self.pl_a += F[:, :, self.kc].astype(np.complex64) * np.exp(-1j * self._omega * t)

    @property
    def box_acc(self):
        return torch.from_numpy(self.box.copy())

    def sx(self, name):
        return float(self.sx_tot[name])

    def phasor(self, comp=1, kind=None):
        if kind == 'split':
            return torch.complex(torch.from_numpy(self.acc_re[comp].astype(np.float64)),
                                 torch.from_numpy(self.acc_im[comp].astype(np.float64)))
        a = self.acc_hand[comp] if kind == 'hand' else self.acc[comp]
        return torch.from_numpy(a.astype(np.complex128))

    def plane_dft(self, name):
        return [(sg, torch.from_numpy(aE.astype(np.complex128)), torch.from_numpy(aH.astype(np.complex128)))
                for sg, aE, aH in self.flux_acc.acc[name]]

    def flux(self, name, n_acc):
        return self.flux_acc.flux(name)

    def conv_change(self, n_last, n_prev):
        if n_prev <= 0 or n_last <= 0:
            return float('nan')
        a = self.pl_b / n_last
        b = self.pl_a / n_prev
        return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(a)), 1e-30))

    def restart_dft(self, window):
        self.pl_a, self.pl_b = self.pl_b, np.zeros_like(self.pl_b)
        for c in self.acc:
            self.acc[c][...] = 0
        self.flux_acc = O.PlaneFlux(self._omega, self.grid.dt, F32)
        self.win, self.prev_win = tuple(window), (0, 0)
