"""Device state of one FDTD solve and its stepping through liblens_fdtd.so.

PyTorch provides the device buffers and the stream; every update runs in the
hand-written sm_100a kernels behind the C ABI (include/lens_fdtd.h).  There is
no CPU path: constructing a grid without a CUDA device or without the built
library raises.

Arrays are stored padded (rows of ``pitch`` floats, pitch a multiple of 32);
the ``view`` helpers return the reference-shaped slices
(planar_beads/fdtd2d_core.py:761-768, planar_3d/fdtd3d_core.py:957-962).
"""
import ctypes

import numpy as np
import torch

from . import _native as N
from .physics import MU0

F32 = np.float32


def pitch_of(n):
    return (int(n) + 31) // 32 * 32


def _device(device=None):
    if not torch.cuda.is_available():
        raise N.LensError('lens_sensor_b200 needs a CUDA device (no CPU fallback)')
    return torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())


def _ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream_ptr(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _pad_upload(a, shape, dev):
    """Zero tensor of `shape` with the numpy array `a` in its leading corner."""
    t = torch.zeros(shape, dtype=torch.float32, device=dev)
    a = np.ascontiguousarray(a, dtype=F32)
    t[tuple(slice(0, s) for s in a.shape)] = torch.from_numpy(a).to(dev, non_blocking=False)
    return t


def strip_widths(c):
    """Leading / trailing run of c != 0 (the psi strips, boundaries3d.py:209-221)."""
    c = np.asarray(c)
    n = len(c)
    lo = 0
    while lo < n and c[lo] != 0.0:
        lo += 1
    hi = 0
    while hi < n and c[n - 1 - hi] != 0.0:
        hi += 1
    if lo + hi >= n:
        lo, hi = n, 0
    return lo, hi


class _Axis:
    """Device copy of one CPML axis (b, c, 1/kappa on integer and half nodes).
    full: psi over the whole axis (every node a strip node: b = 1, c = 0 keeps
    psi constant outside the absorber, as the reference's full-domain psi
    arrays do, boundaries.py:172-175)."""

    def __init__(self, prof, n, dev, full=False):
        self.keep = []
        self.ax = N.Axis()
        for tag, length in (('e', n), ('h', n - 1)):
            b = np.asarray(prof['b' + tag], F32)
            c = np.asarray(prof['c' + tag], F32)
            ik = (F32(1.0) / np.asarray(prof['k' + tag], F32)).astype(F32)
            assert len(b) == length, (tag, len(b), length)
            tb, tc, ti = (torch.from_numpy(v.copy()).to(dev) for v in (b, c, ik))
            self.keep += [tb, tc, ti]
            lo, hi = (length, 0) if full else strip_widths(c)
            setattr(self.ax, tag, N.Profile(_ptr(tb), _ptr(tc), _ptr(ti), length, lo, hi))

    def w(self, tag):
        p = getattr(self.ax, tag)
        return p.lo + p.hi


class StepTable:
    """Per-step scalars for steps [t0, t0+n): float32(w_src t), envelope, DFT phases.

    wt follows vcsel.py:153-155 (float32 of the float64 product), the envelope is
    evaluated in float64 (fdtd2d_core.py:784-787) and the DFT phases are
    exp(-i w t) and exp(-i w (t - dt/2)) (flux.py:30-33)."""

    def __init__(self, t0, n, dt, omega_src, omega_dft, envelope, device=None):
        dev = _device(device)
        steps = np.arange(t0, t0 + n, dtype=np.int64)
        t = steps * dt
        self.t0, self.n = int(t0), int(n)
        wt = (omega_src * t).astype(F32)
        env = np.asarray(envelope(t), dtype=np.float64).astype(F32)
        pe = np.exp(-1j * omega_dft * t)
        ph = np.exp(-1j * omega_dft * (t - 0.5 * dt))
        pe2 = np.stack([pe.real, pe.imag], 1).astype(F32)
        ph2 = np.stack([ph.real, ph.imag], 1).astype(F32)
        self.wt, self.env, self.pe, self.ph = (torch.from_numpy(np.ascontiguousarray(v)).to(dev)
                                               for v in (wt, env, pe2, ph2))
        self.s = N.StepTable(_ptr(self.wt), _ptr(self.env), _ptr(self.pe), _ptr(self.ph),
                             self.t0, self.n)


def cw_envelope(f0, ramp_periods=None):
    """Vectorised CW ramp 1 - exp(-(t/(2 sigma_t))^2) (fdtd2d_core.py:784-787);
    sigma_t = 4/(2 pi f0), or ramp_periods/(6 f0) to stretch the 6-sigma start-up."""
    st = 4.0 / (2 * np.pi * f0) if ramp_periods is None else ramp_periods / (6.0 * f0)
    return lambda t: 1 - np.exp(-((np.asarray(t) / (2 * st)) ** 2))


def _kahan_value(buf):
    """Compensated (sum, carry) float32 pairs -> complex128 value sum - carry."""
    b = buf.double()
    return torch.complex(b[..., 0] - b[..., 2], b[..., 1] - b[..., 3])


# ============================================================================ 2D
class Grid2D:
    """One 2D CPML solve (TE: Ez/Hx/Hy, TM: Ex/Ey/Hz) resident on the GPU.

    coef: TE {'ce_e','ce_h'} (nx,ny); TM {'ca_x' (nx-1,ny), 'ca_y' (nx,ny-1),
    optional 'da_x','da_y'} - the arrays of fdtd2d_core._coeffs / _tm_coeffs /
    _tm_loss.  cx, cy: CPML profiles {'ke','be','ce','kh','bh','ch'} along x and y.
    src: dict(ix, amp, ph1, ph2) of the Huygens pair (TM: on the Ey grid).
    full_x: x psi over every row (the co-moving window, whose rolled psi keeps
    its values outside the absorber)."""

    def __init__(self, pol, nx, ny, dx, dt, coef, cx, cy, src, pec=(1, 1, 1, 1), device=None, full_x=False):
        self.lib = N.load()
        dev = self.dev = _device(device)
        self.pol = 'p' if str(pol).lower() in ('p', 'tm') else 's'
        self.nx, self.ny, self.dx, self.dt = int(nx), int(ny), dx, dt
        P = self.pitch = pitch_of(ny)
        shp = (nx, P)
        z = lambda *s: torch.zeros(s if s else shp, dtype=torch.float32, device=dev)
        self.ch = F32(dt / (MU0 * dx))
        self.axx, self.axy = _Axis(cx, nx, dev, full=full_x), _Axis(cy, ny, dev)
        wxe, wxh, wye, wyh = self.axx.w('e'), self.axx.w('h'), self.axy.w('e'), self.axy.w('h')
        if src is None:                # no source (a stitch window driven by its predecessor)
            self.src_t = {}
            s = N.Source(-1, None, None, None, 0, 0, 0)
        else:
            self.src_t = {k: torch.from_numpy(np.ascontiguousarray(src[k], F32)).to(dev)
                          for k in ('amp', 'ph1', 'ph2')}
            s = N.Source(int(src['ix']), _ptr(self.src_t['amp']), _ptr(self.src_t['ph1']),
                         _ptr(self.src_t['ph2']), len(src['amp']), 1, len(src['amp']))
        pec4 = (ctypes.c_int * 4)(*[int(bool(v)) for v in pec])
        if self.pol == 's':
            self.ez, self.hx, self.hy = z(), z(), z()
            self.ce_e = _pad_upload(coef['ce_e'], shp, dev)
            self.ce_h = _pad_upload(coef['ce_h'], shp, dev)
            self.psi = dict(hxy=z(nx, max(1, wyh)), hyx=z(max(1, wxh), P),
                            ezx=z(max(1, wxe), P), ezy=z(nx, max(1, wye)))
            self.s = N.TE2D(nx, ny, P, _ptr(self.ez), _ptr(self.hx), _ptr(self.hy),
                            _ptr(self.ce_e), _ptr(self.ce_h), float(self.ch),
                            self.axx.ax, self.axy.ax, _ptr(self.psi['hxy']), _ptr(self.psi['hyx']),
                            _ptr(self.psi['ezx']), _ptr(self.psi['ezy']), pec4, s)
        else:
            self.ex, self.ey, self.hz = z(), z(), z()
            self.ca_x = _pad_upload(coef['ca_x'], shp, dev)
            self.ca_y = _pad_upload(coef['ca_y'], shp, dev)
            da = coef.get('da_x') is not None
            self.da_x = _pad_upload(coef['da_x'], shp, dev) if da else None
            self.da_y = _pad_upload(coef['da_y'], shp, dev) if da else None
            self.psi = dict(hzx=z(max(1, wxh), P), hzy=z(nx, max(1, wyh)),
                            exy=z(nx, max(1, wye)), eyx=z(max(1, wxe), P))
            self.s = N.TM2D(nx, ny, P, _ptr(self.ex), _ptr(self.ey), _ptr(self.hz),
                            _ptr(self.ca_x), _ptr(self.ca_y), _ptr(self.da_x), _ptr(self.da_y),
                            float(self.ch), self.axx.ax, self.axy.ax,
                            _ptr(self.psi['hzx']), _ptr(self.psi['hzy']), _ptr(self.psi['exy']),
                            _ptr(self.psi['eyx']), pec4, s)

    # reference-shaped views of the resident fields
    def view(self, name):
        nx, ny = self.nx, self.ny
        shapes = dict(ez=(nx, ny), hx=(nx, ny - 1), hy=(nx - 1, ny),
                      ex=(nx - 1, ny), ey=(nx, ny - 1), hz=(nx - 1, ny - 1))
        a, b = shapes[name]
        return getattr(self, name)[:a, :b]

    def state(self):
        """The fields and psi arrays, each with its rows along x."""
        names = ('ez', 'hx', 'hy') if self.pol == 's' else ('ex', 'ey', 'hz')
        return [getattr(self, q) for q in names] + list(self.psi.values())

    def take_shifted(self, other, n):
        """Fields and psi of `other` (same sizes and strips) moved n rows towards
        x = 0, the last n rows zero: the co-moving window's roll
        (fdtd2d_core.py:1093-1102, boundaries.py:217-221)."""
        for a, b in zip(self.state(), other.state()):
            assert a.shape == b.shape, (a.shape, b.shape)
            a.zero_()
            if 0 < n < a.shape[0]:
                a[:a.shape[0] - n].copy_(b[n:])

    def step(self, table, n0, nsteps, epi=None, stream=None, drive=None):
        e = ctypes.byref(epi.s) if epi is not None else None
        if drive is None:
            fn = self.lib.lens_te2d_step if self.pol == 's' else self.lib.lens_tm2d_step
            N.check(fn(ctypes.byref(self.s), ctypes.byref(table.s), e, int(n0), int(nsteps), _stream_ptr(stream)))
        else:
            fn = self.lib.lens_te2d_step_driven if self.pol == 's' else self.lib.lens_tm2d_step_driven
            N.check(fn(ctypes.byref(self.s), ctypes.byref(table.s), e, ctypes.byref(drive.s), int(n0),
                       int(nsteps), _stream_ptr(stream)))


class Drive2D:
    """Overlap drive of a 2D stitch window (fdtd2d_core.py:1439-1440, 1462-1463).

    hand: complex64 amplitudes (O, ny_c) of the driven component (TE Ez, TM Ey);
    taper: the O weights w_i (float32); env, cos_wt, sin_wt: float64 per step
    n - t0 of the step table (the reference's float envelope and complex128
    phase e^{i w t})."""

    def __init__(self, grid, hand, taper, env, cos_wt, sin_wt):
        dev, P = grid.dev, grid.pitch
        D = torch.as_tensor(hand).to(dev)
        O = int(D.shape[0])
        self.taper = torch.from_numpy(np.ascontiguousarray(taper, F32)).to(dev)
        self.hand = torch.zeros((O, P, 2), dtype=torch.float32, device=dev)
        self.hand[:, :D.shape[1], 0] = D.real.float()
        self.hand[:, :D.shape[1], 1] = D.imag.float()
        tab = np.stack([np.asarray(env, np.float64), np.asarray(cos_wt, np.float64),
                        np.asarray(sin_wt, np.float64)], axis=1)
        self.tab = torch.from_numpy(np.ascontiguousarray(tab)).to(dev)
        s = N.Drive2D()
        s.nplanes, s.taper, s.hand, s.tab = O, _ptr(self.taper), _ptr(self.hand), _ptr(self.tab)
        self.s = s


class Epi2D:
    """Epilogue buffers of a 2D solve (detector boxes, DFTs, Iavg, flux planes)."""

    def __init__(self, grid, boxes=(), dft=None, dft_ex=False, prev=None, iavg_n0=None, planes=(),
                 dft_raw=False, ex2=False, sx_planes=(), box_split=False):
        """dft_raw / ex2 (TM): the DFT of Ey on its own grid and the sum of Ex^2 on
        the nodes over the dft window (run_beads_stitched, fdtd2d_core.py:1441-1446).
        sx_planes: {name: il} planes whose time-domain Poynting flux is summed
        over every step (the pulse energies of run_beads_sliding,
        fdtd2d_core.py:1139-1158).  box_split names the reference's separate
        FP64 sums of field^2 and <Ex^2> in a TM box (fdtd2d_core.py:1148-1150);
        the device sums their FP32 sum per cell in FP64 either way."""
        dev, nx, P = grid.dev, grid.nx, grid.pitch
        self.grid = grid
        self.boxes = [tuple(int(v) for v in b) for b in boxes]
        self.box_acc = torch.zeros(max(1, len(boxes)), dtype=torch.float64, device=dev)
        d4 = lambda: torch.zeros((nx, P, 4), dtype=torch.float32, device=dev)
        self.dft = d4() if dft is not None else None
        self.dft_ex = d4() if (dft is not None and dft_ex) else None
        self.prev = d4() if prev is not None else None
        self.dft_raw = d4() if (dft is not None and dft_raw) else None
        self.ex2 = torch.zeros((nx, P), dtype=torch.float32, device=dev) if (dft is not None and ex2) else None
        self.iavg = torch.zeros((nx, P), dtype=torch.float32, device=dev) if iavg_n0 is not None else None
        self.planes = dict(planes)
        self.plane_acc = torch.zeros((max(1, len(self.planes)), 4, P), dtype=torch.float64, device=dev)
        s = N.Epi2D()
        s.nbox = len(self.boxes)
        for q, b in enumerate(self.boxes):
            s.box[q] = (ctypes.c_int * 4)(*b)
        s.box_acc = _ptr(self.box_acc)
        s.dft_n0, s.dft_n1 = dft if dft is not None else (0, 0)
        s.dft, s.dft_ex = _ptr(self.dft), _ptr(self.dft_ex)
        s.prev_n0, s.prev_n1 = prev if prev is not None else (0, 0)
        s.dft_prev = _ptr(self.prev)
        s.iavg_n0 = int(iavg_n0) if iavg_n0 is not None else (1 << 30)
        s.iavg = _ptr(self.iavg)
        s.nplane = len(self.planes)
        for q, il in enumerate(self.planes.values()):
            s.plane[q] = int(il)
        s.plane_acc = _ptr(self.plane_acc)
        s.dft_raw, s.ex2 = _ptr(self.dft_raw), _ptr(self.ex2)
        self.sx_planes = dict(sx_planes)
        self.sx_acc = torch.zeros((max(1, len(self.sx_planes)), P), dtype=torch.float64, device=dev)
        s.nsx = len(self.sx_planes)
        for q, il in enumerate(self.sx_planes.values()):
            s.sx_plane[q] = int(il)
        s.sx_acc = _ptr(self.sx_acc)
        self.s = s

    def sx(self, name):
        """Sum over the steps run of the instantaneous +x flux through plane
        `name`: TE -sum Ez Hy, TM sum Ey Hz, H averaged onto the plane
        (_sx_plane_2d, fdtd2d_core.py:489-497)."""
        q = list(self.sx_planes).index(name)
        tot = float(torch.sum(self.sx_acc[q]))
        return -tot if self.grid.pol == 's' else tot

    def phasor(self, which='dft', kind=None):
        """Accumulated sum(F e^{-i w t}) on the nodes (nx, ny) ('dft_raw': on the
        Ey grid (nx, ny-1)), complex128.  kind='stitch' names the reference's
        complex64 window sums of run_beads_stitched; the device keeps one
        compensated FP32 sum per quantity, which serves both."""
        ny = self.grid.ny - (1 if which == 'dft_raw' else 0)
        return _kahan_value(getattr(self, which))[:, :ny]

    def plane_dft(self, name):
        """[(sign, sum E e^{-iwt}, sum H e^{-iw(t-dt/2)})] of plane `name` (pairs_2d), complex128."""
        q = list(self.planes).index(name)
        a = self.plane_acc[q]
        ny = self.grid.ny if self.grid.pol == 's' else self.grid.ny - 1
        sign = -1.0 if self.grid.pol == 's' else 1.0
        return [(sign, torch.complex(a[0, :ny], a[1, :ny]), torch.complex(a[2, :ny], a[3, :ny]))]

    def restart_dft(self, window):
        """Open a new DFT window [n0, n1) after a failed CW convergence check
        (fdtd2d_core.py:862-869): the finished window becomes the comparison
        window; the DFT, the Ex DFT and the flux planes restart from zero."""
        self.dft, self.prev = self.prev, self.dft
        self.dft.zero_()
        if self.dft_ex is not None:
            self.dft_ex.zero_()
        self.plane_acc.zero_()
        self.s.dft, self.s.dft_prev = _ptr(self.dft), _ptr(self.prev)
        self.s.dft_n0, self.s.dft_n1 = int(window[0]), int(window[1])
        self.s.prev_n0 = self.s.prev_n1 = 0

    def flux(self, name, n_acc):
        """Net +x Poynting flux through plane `name` (flux.py:45-57)."""
        q = list(self.planes).index(name)
        a = self.plane_acc[q]
        ny = self.grid.ny if self.grid.pol == 's' else self.grid.ny - 1
        aE = torch.complex(a[0, :ny], a[1, :ny])
        aH = torch.complex(a[2, :ny], a[3, :ny])
        sign = -1.0 if self.grid.pol == 's' else 1.0
        return float(sign * 0.5 * torch.real(torch.sum(aE * torch.conj(aH)))) * (2.0 / n_acc) ** 2


# ============================================================================ 3D
MAX_CTYPE = 4


def coef_columns(vols, nx, ny, nz, min_count=64):
    """Column form of the coefficient volumes (LensGrid3D.ctype/ctab/cexpl).

    vols: the padded (nx, ny, pitch) float32 device volumes ce_x, ce_y, ce_z
    (+ D_x, D_y, D_z).  The (i, k) columns over y are grouped by an exact
    fingerprint of their bit patterns; the up to 4 most frequent groups (each
    of at least min_count columns) whose members equal their representative bit
    for bit become column types.  Returns (ctype uint8 (nx, pitch), ctab
    float32 (ntype, 6, ny), cexpl uint8 (nx, pitch/32), ntype), or None when no
    group qualifies."""
    dev = vols[0].device
    P = vols[0].shape[2]
    g = torch.Generator(device='cpu').manual_seed(12345)
    w = (torch.randint(1, 2 ** 62, (len(vols), ny), generator=g, dtype=torch.int64) | 1).to(dev)
    h = torch.zeros((nx, P), dtype=torch.int64, device=dev)
    for a, wa in zip(vols, w):   # sum of bit patterns times odd weights (mod 2^64)
        h += (a.view(torch.int32).to(torch.int64) * wa[None, :, None]).sum(dim=1)
    hv = h[:, :nz].reshape(-1)
    uniq, inv, cnt = torch.unique(hv, return_inverse=True, return_counts=True)
    order = torch.argsort(cnt, descending=True)[:MAX_CTYPE].tolist()
    ctype = torch.full((nx, P), 255, dtype=torch.uint8, device=dev)
    ctab = torch.zeros((MAX_CTYPE, 6, ny), dtype=torch.float32, device=dev)
    nt = 0
    for u in order:
        if int(cnt[u]) < min_count:
            break
        pos = torch.nonzero(inv == u).squeeze(1)
        ii, kk = pos // nz, pos % nz
        ok = torch.ones(pos.numel(), dtype=torch.bool, device=dev)
        i0, k0 = int(ii[0]), int(kk[0])
        for c, a in enumerate(vols):
            rep = a[i0, :, k0].view(torch.int32)
            ok &= (a[ii, :, kk].view(torch.int32) == rep[None, :]).all(dim=1)
            ctab[nt, c] = a[i0, :, k0]
        if not bool(ok.any()):
            continue
        ctype[ii[ok], kk[ok]] = nt
        nt += 1
    if nt == 0:
        return None
    ctype[:, nz:] = 0                      # padding columns are never read
    cexpl = (ctype == 255).view(nx, P // 32, 32).any(dim=2).to(torch.uint8).contiguous()
    return ctype.contiguous(), ctab[:nt].contiguous(), cexpl, nt


def plane_flux(pairs, n):
    """sum over pairs of sign * Re(sum aE conj(aH)) / 2, times (2/n)^2 (flux.py:45-57)."""
    tot = 0.0
    for sign, aE, aH in pairs:
        tot += sign * 0.5 * float(torch.real(torch.sum(aE * torch.conj(aH))))
    return tot * (2.0 / n) ** 2


class Grid3D:
    """One 3D CPML solve resident on the GPU (fdtd3d_core.run_3d hot loop state).

    ce: (ce_x, ce_y, ce_z) staggered update factors; da: staggered damping
    (D_x, D_y, D_z) or None; cpml: three profile dicts (x, y, z);
    src: dict(ix, amp (nj,nk), ph1, ph2) on the grid of component src_comp.
    fused=True keeps two field/psi buffers and runs the single-pass TMA kernel;
    fused=False updates one buffer in place with two streaming passes."""

    FIELDS = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')

    def __init__(self, nx, ny, nz, dx, dt, ce, da, cpml, src, src_comp=1, pec=(1,) * 6,
                 device=None, fused=True, tb=False, tb_chunk=40):
        self.lib = N.load()
        dev = self.dev = _device(device)
        self.nx, self.ny, self.nz, self.dx, self.dt = int(nx), int(ny), int(nz), dx, dt
        P = self.pitch = pitch_of(nz)
        shp = (nx, ny, P)
        z = lambda *s: torch.zeros(s if s else shp, dtype=torch.float32, device=dev)
        self.ch = F32(dt / (MU0 * dx))
        self.ax = [_Axis(cpml[a], n, dev) for a, n in enumerate((nx, ny, nz))]
        X, Y, Zp = self.ax
        nbuf = 2 if fused else 1

        self.bufs = [{f: z() for f in self.FIELDS} for _ in range(nbuf)]
        # psi volumes are full-domain (only their CPML strips are touched)
        self.psi = [{q: z() for q in N.PSI_NAMES} for _ in range(nbuf)]
        self.ce = [_pad_upload(a, shp, dev) for a in ce]
        self.da = None if da is None else [_pad_upload(a, shp, dev) for a in da]
        if src is None:                # no source (a stitch window driven by its predecessor)
            self.src_t = {}
            s = N.Source(-1, None, None, None, 0, 0, 0)
        else:
            amp = np.ascontiguousarray(src['amp'], F32)
            self.src_t = {k: torch.from_numpy(np.ascontiguousarray(src[k], F32)).to(dev)
                          for k in ('amp', 'ph1', 'ph2')}
            nj, nk = amp.shape
            s = N.Source(int(src['ix']), _ptr(self.src_t['amp']), _ptr(self.src_t['ph1']),
                         _ptr(self.src_t['ph2']), nj, nk, nk)
        self.src_comp = int(src_comp)
        self.flag = torch.zeros(1, dtype=torch.int32, device=dev)
        g = N.Grid3D()
        g.nx, g.ny, g.nz, g.pitch = nx, ny, nz, P
        for b in range(nbuf):
            for c, f in enumerate(self.FIELDS):
                g.f[b][c] = self.bufs[b][f].data_ptr()
            for q, name in enumerate(N.PSI_NAMES):
                g.psi[b][q] = self.psi[b][name].data_ptr()
        g.cur = 0
        g.ce_x, g.ce_y, g.ce_z = (c.data_ptr() for c in self.ce)
        if self.da is not None:
            g.da_x, g.da_y, g.da_z = (d.data_ptr() for d in self.da)
        g.ch = float(self.ch)
        g.ax, g.ay, g.az = X.ax, Y.ax, Zp.ax
        g.pec = (ctypes.c_int * 6)(*[int(bool(v)) for v in pec])
        g.src = s
        g.src_comp = self.src_comp
        g.flag = self.flag.data_ptr()
        # the fused step reads repeated coefficient columns from a small table
        self.cols = coef_columns(self.ce + (self.da or []), nx, ny, nz) if fused else None
        if self.cols is not None:
            ct, tab, ex, nt = self.cols
            g.ctype, g.ctab, g.cexpl, g.ntype = ct.data_ptr(), tab.data_ptr(), ex.data_ptr(), nt
        self.s = g
        # temporally blocked step: a scratch set of the psi volumes for its intermediate level
        self.tb = None
        if tb:
            if not fused:
                raise ValueError('the temporally blocked 3D step needs both field buffers (fused=True)')
            self.psi_lv = {q: z() for q in N.PSI_NAMES}
            t = N.TB3D()
            for q, name in enumerate(N.PSI_NAMES):
                t.psi_lv[q] = self.psi_lv[name].data_ptr()
            t.chunk = int(tb_chunk)
            self.tb = t

    def __getattr__(self, name):
        if name in Grid3D.FIELDS:
            return self.__dict__['bufs'][self.__dict__['s'].cur][name]
        raise AttributeError(name)

    def view(self, name):
        nx, ny, nz = self.nx, self.ny, self.nz
        shapes = dict(ex=(nx - 1, ny, nz), ey=(nx, ny - 1, nz), ez=(nx, ny, nz - 1),
                      hx=(nx, ny - 1, nz - 1), hy=(nx - 1, ny, nz - 1), hz=(nx - 1, ny - 1, nz))
        a, b, c = shapes[name]
        return getattr(self, name)[:a, :b, :c]

    def step(self, table, n0, nsteps, epi=None, stream=None, drive=None):
        e = ctypes.byref(epi.s) if epi is not None else None
        if drive is None:
            N.check(self.lib.lens_fdtd3d_step(ctypes.byref(self.s), ctypes.byref(table.s), e,
                                              int(n0), int(nsteps), _stream_ptr(stream)))
        else:
            N.check(self.lib.lens_fdtd3d_step_driven(ctypes.byref(self.s), ctypes.byref(table.s), e,
                                                     ctypes.byref(drive.s), int(n0), int(nsteps),
                                                     _stream_ptr(stream)))

    def step_tb(self, table, n0, nsteps, epi=None, stream=None):
        """Steps [n0, n0 + nsteps) on the temporally blocked kernel (LENS_TB3_K steps
        per launch, epilogues fused); an odd leftover step runs on the fused
        single-step kernel.  Returns the number of kernel launches."""
        if self.tb is None:
            raise ValueError('grid built without tb=True')
        e = ctypes.byref(epi.s) if epi is not None else None
        k = N.TB3_K
        m = nsteps // k * k
        launches = 0
        if m:
            N.check(self.lib.lens_fdtd3d_step_tb(ctypes.byref(self.s), ctypes.byref(self.tb), ctypes.byref(table.s), e,
                                                 int(n0), int(m), _stream_ptr(stream)))
            launches += m // k
        if nsteps - m:
            self.step(table, n0 + m, nsteps - m, epi, stream)
            launches += (nsteps - m) * (2 if epi is not None else 1)
        return launches

    def check_flag(self):
        """Raise if a pipeline wait in the fused kernel gave up or a detector box
        saw a NaN / infinity (results invalid)."""
        f = int(self.flag.item())
        if f & 1:
            raise N.LensError('fused 3D kernel: a pipeline wait timed out')
        if f & 2:
            raise N.LensError('3D solve: a detector box sum is not finite (the fields hold NaN or infinity)')

    def accum_e2(self, iavg, target=None, stream=None, nx=None):
        """iavg += |E|^2 on the driven component's grid over x-planes [0, nx)."""
        t = self.src_comp if target is None else target
        N.check(self.lib.lens_fdtd3d_accum_e2(ctypes.byref(self.s), int(t), int(self.nx if nx is None else nx),
                                              _ptr(iavg), _stream_ptr(stream)))


class Drive3D:
    """Overlap drive of a stitch window (fdtd3d_core.py:1611-1617).

    hand: complex amplitudes (complex64) of Ex, Ey, Ez on the first O x-planes,
    shapes (O, ny, nz-ish) of each component's own grid; taper: the O weights
    w_i (float32).  Both are copied into the padded device layout once."""

    def __init__(self, grid, hand, taper):
        dev, ny, P = grid.dev, grid.ny, grid.pitch
        O = int(len(taper))
        w = np.asarray(taper, F32)
        self.taper = torch.from_numpy(np.concatenate([w, (F32(1.0) - w).astype(F32)])).to(dev)
        self.hand = []
        for D in hand:
            t = torch.zeros((O, ny, P, 2), dtype=torch.float32, device=dev)
            D = torch.as_tensor(D).to(dev)
            t[:, :D.shape[1], :D.shape[2], 0] = D.real.float()
            t[:, :D.shape[1], :D.shape[2], 1] = D.imag.float()
            self.hand.append(t)
        s = N.Drive3D()
        s.nplanes = O
        s.taper = _ptr(self.taper)
        for m in range(3):
            s.hand[m] = _ptr(self.hand[m])
        self.s = s


class Epi3D:
    """Epilogue buffers of a 3D solve."""

    def __init__(self, grid, boxes=(), dft=None, comps=(1,), planes=(), conv=None, iavg=False):
        dev, nx, ny, P = grid.dev, grid.nx, grid.ny, grid.pitch
        self.grid = grid
        self.boxes = [tuple(int(v) for v in b) for b in boxes]
        self.box_acc = torch.zeros(max(1, len(boxes)), dtype=torch.float64, device=dev)
        self.dft = [None, None, None]
        if dft is not None:
            for c in comps:
                self.dft[c] = torch.zeros((nx, ny, P, 2), dtype=torch.float32, device=dev)
        self.planes = dict(planes)
        self.plane_acc = torch.zeros((max(1, len(self.planes)), 2, 4, ny, P), dtype=torch.float64,
                                     device=dev)
        nj = grid.s.src.nj
        self.conv_prev = self.conv_last = None
        if conv is not None:
            self.conv_prev = torch.zeros((nx, nj, 4), dtype=torch.float32, device=dev)
            self.conv_last = torch.zeros((nx, nj, 4), dtype=torch.float32, device=dev)
        self.iavg = torch.zeros((nx, ny, P), dtype=torch.float32, device=dev) if iavg else None
        s = N.Epi3D()
        s.nbox = len(self.boxes)
        for q, b in enumerate(self.boxes):
            s.box[q] = (ctypes.c_int * 6)(*b)
        s.box_acc = _ptr(self.box_acc)
        s.dft_n0, s.dft_n1 = dft if dft is not None else (0, 0)
        for c in range(3):
            s.dft[c] = _ptr(self.dft[c])
        if conv is not None:
            s.conv_k, (s.prev_n0, s.prev_n1) = int(conv[0]), conv[1]
        s.conv_prev, s.conv_last = _ptr(self.conv_prev), _ptr(self.conv_last)
        s.nplane = len(self.planes)
        for q, il in enumerate(self.planes.values()):
            s.plane[q] = int(il)
        s.plane_acc = _ptr(self.plane_acc)
        self.s = s

    def phasor(self, comp=1, kind=None):
        """sum F e^{-iwt} of component comp over the DFT window, complex128 in the
        component's shape.  kind ('split', 'hand') names the reference's separate
        accumulators of run_3d_stitched (float32 re/im volume, complex64 overlap);
        the device keeps one FP32 (re, im) sum per component, which serves all."""
        g = self.grid
        nx, ny, nz = g.nx, g.ny, g.nz
        shape = {0: (nx - 1, ny, nz), 1: (nx, ny - 1, nz), 2: (nx, ny, nz - 1)}[comp]
        a = self.dft[comp].double()
        return torch.complex(a[..., 0], a[..., 1])[:shape[0], :shape[1], :shape[2]]

    def plane_dft(self, name):
        """[(sign, sum E e^{-iwt}, sum H e^{-iw(t-dt/2)})] of the two field pairs
        of plane `name` (pairs_3d, flux.py:84-90), complex128."""
        g = self.grid
        q = list(self.planes).index(name)
        out = []
        for pair, (sign, nj, nk) in enumerate(((1.0, g.ny - 1, g.nz), (-1.0, g.ny, g.nz - 1))):
            a = self.plane_acc[q, pair]
            out.append((sign, torch.complex(a[0, :nj, :nk], a[1, :nj, :nk]),
                        torch.complex(a[2, :nj, :nk], a[3, :nj, :nk])))
        return out

    def flux(self, name, n_acc):
        """Net +x Poynting flux (pairs_3d, flux.py:84-90 and :45-57)."""
        return plane_flux(self.plane_dft(name), n_acc)

    def conv_change(self, n_last, n_prev):
        """||a - b|| / ||a|| of the convergence planes a = last / n_last, b = prev / n_prev
        (fdtd3d_core.py:1159-1162); nan without a previous window."""
        if self.conv_last is None or n_prev <= 0 or n_last <= 0:
            return float('nan')
        a = _kahan_value(self.conv_last) / n_last
        b = _kahan_value(self.conv_prev) / n_prev
        return float(torch.linalg.norm(a - b)) / max(float(torch.linalg.norm(a)), 1e-30)

    def restart_dft(self, window):
        """Open a new DFT window [n0, n1) after a failed convergence check
        (fdtd3d_core.py:1162-1170): the last convergence plane becomes the previous
        one; the volume DFTs, the flux planes and the last plane restart from zero."""
        self.conv_prev, self.conv_last = self.conv_last, self.conv_prev
        self.conv_last.zero_()
        for d in self.dft:
            if d is not None:
                d.zero_()
        self.plane_acc.zero_()
        self.s.conv_prev, self.s.conv_last = _ptr(self.conv_prev), _ptr(self.conv_last)
        self.s.dft_n0, self.s.dft_n1 = int(window[0]), int(window[1])
        self.s.prev_n0 = self.s.prev_n1 = 0
