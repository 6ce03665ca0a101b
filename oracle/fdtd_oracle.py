"""NumPy oracle for the lens_sensor FDTD hot path (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module; it is the checker, never the thing measured or shipped.

It restates, with plain NumPy and in the reference's operation order, the setup
and per-step algorithm of s1alknau/lens_sensor's native FDTD path:

* CPML profiles                      planar_beads/boundaries.py:104-151,
                                     planar_3d/boundaries3d.py:150-194
* sub-pixel helpers                  common/subpixel.py:25-94
* Gaussian VCSEL Huygens source      common/vcsel.py:77-170
* 2D materials / coefficients        planar_beads/fdtd2d_core.py:122-349, 445-455
* 2D CPML TE/TM step                 planar_beads/boundaries.py:164-274,
                                     planar_beads/fdtd2d_core.py:781-850
* 3D eps / staggered coefficients    planar_3d/fdtd3d_core.py:119-378, 593-613
* 3D CPML step (psi strips)          planar_3d/boundaries3d.py:201-362
* epilogues (DFT, detectors, Iavg,   planar_beads/fdtd2d_core.py:834-850,
  plane flux)                        planar_3d/fdtd3d_core.py:464-481, 1139-1158,
                                     common/flux.py:19-90

Pinning: ``tests/test_oracle_golden.py`` compares these functions with fixtures
written by running the reference's own code (``tests/golden/make_golden.py``).

Precision: ``dtype=np.float32`` repeats the reference's float32 arithmetic
operation by operation.  ``dtype=np.float64`` is the FP64 oracle: the same
algorithm over the same float32-rounded coefficient and source arrays, with
float64 fields, psi, time phase and accumulators.
"""
import math

import numpy as np

C0 = 2.99792458e8
EPS0 = 8.8541878128e-12
MU0 = 4.0 * np.pi * 1e-7
N_AIR = 1.0
F32 = np.float32


# ---------------------------------------------------------------------------
# CPML profiles (boundaries.py:104-151; boundaries3d.py:150-194 is the same math)
# ---------------------------------------------------------------------------
def cpml_axis(N, n_lo, n_hi, dx, dt, lam_m=850e-9, m=3, R0=1e-6, kappa_max=1.0):
    """Return dict(ke, be, ce) on the N integer nodes and (kh, bh, ch) on the N-1
    half nodes, float32.  Outside the PML: kappa=1, b=1, c=0."""
    if n_lo <= 0 and n_hi <= 0:
        return dict(ke=np.ones(N, F32), be=np.ones(N, F32), ce=np.zeros(N, F32),
                    kh=np.ones(N - 1, F32), bh=np.ones(N - 1, F32), ch=np.zeros(N - 1, F32))
    eta0 = np.sqrt(4e-7 * np.pi / EPS0)
    a_max = 2.0 * np.pi * EPS0 * (C0 / lam_m) / 10.0

    def smax(n):
        return (-(m + 1) * np.log(R0) / (2.0 * eta0 * n * dx)) if n > 0 else 0.0

    def prof(pos):
        depth = np.zeros_like(pos)
        sg = np.zeros_like(pos)
        if n_lo > 0:
            lo = pos < n_lo
            depth[lo] = (n_lo - pos[lo]) / n_lo
            sg[lo] = smax(n_lo)
        if n_hi > 0:
            hi = pos > (N - 1 - n_hi)
            depth[hi] = (pos[hi] - (N - 1 - n_hi)) / n_hi
            sg[hi] = smax(n_hi)
        depth = np.clip(depth, 0.0, 1.0)
        sigma = sg * depth ** m
        kappa = 1.0 + (kappa_max - 1.0) * depth ** m
        a = np.where(depth > 0.0, a_max * (1.0 - depth), 0.0)
        b = np.exp(-(sigma / kappa + a) * dt / EPS0)
        den = sigma * kappa + kappa * kappa * a
        c = np.zeros_like(sigma)
        nz = den > 0.0
        c[nz] = sigma[nz] * (b[nz] - 1.0) / den[nz]
        return kappa.astype(F32), b.astype(F32), c.astype(F32)

    ke, be, ce = prof(np.arange(N, dtype=np.float64))
    kh, bh, ch = prof(np.arange(N - 1, dtype=np.float64) + 0.5)
    return dict(ke=ke, be=be, ce=ce, kh=kh, bh=bh, ch=ch)


# ---------------------------------------------------------------------------
# Sub-pixel smoothing (subpixel.py:25-94)
# ---------------------------------------------------------------------------
def _offs(S, h):
    return ((np.arange(S) + 0.5) / S - 0.5) * h


def circle_fraction(xs, ys, xc, yc, r, h, S=8):
    X = xs[:, None] - xc
    Y = ys[None, :] - yc
    d = np.sqrt(X * X + Y * Y)
    half = h * np.sqrt(2.0) / 2.0
    f = (d <= r - half).astype(np.float64)
    e = np.nonzero((d > r - half) & (d < r + half))
    if len(e[0]):
        o = _offs(S, h)
        px = X[e[0], 0][:, None, None] + o[None, :, None]
        py = Y[0, e[1]][:, None, None] + o[None, None, :]
        f[e] = np.mean((px * px + py * py) <= r * r, axis=(1, 2))
    return f


def sphere_fraction(xs, ys, zs, xc, yc, zc, r, h, S=6):
    X = xs[:, None, None] - xc
    Y = ys[None, :, None] - yc
    Z = zs[None, None, :] - zc
    d = np.sqrt(X * X + Y * Y + Z * Z)
    half = h * np.sqrt(3.0) / 2.0
    f = (d <= r - half).astype(np.float64)
    e = np.nonzero((d > r - half) & (d < r + half))
    if len(e[0]):
        o = _offs(S, h)
        hit = np.zeros(len(e[0]))
        for a in o:
            px = (X[e[0], 0, 0] + a)[:, None, None]
            py = Y[0, e[1], 0][:, None, None] + o[None, :, None]
            pz = Z[0, 0, e[2]][:, None, None] + o[None, None, :]
            hit += np.sum((px * px + py * py + pz * pz) <= r * r, axis=(1, 2))
        f[e] = hit / S ** 3
    return f


def blend(eps, frac, n_incl):
    m = frac > 0
    eps[m] = (1.0 - frac[m]) * eps[m] + frac[m] * (n_incl ** 2)
    return eps


def column_average(ys, dy, eps_of_y, S=16, harmonic=False, shift=0.0):
    off = ((np.arange(S) + 0.5) / S - 0.5) * dy + shift
    Y = np.asarray(ys, dtype=np.float64)[:, None] + off[None, :]
    e = np.asarray(eps_of_y(Y.ravel()))
    cplx = np.iscomplexobj(e)
    e = e.astype(np.complex128 if cplx else np.float64).reshape(Y.shape)
    out = np.complex64 if cplx else np.float32
    if harmonic:
        return (1.0 / np.mean(1.0 / e, axis=1)).astype(out)
    return np.mean(e, axis=1).astype(out)


def loss_sigma(eps_imag, lam_m):
    """common/physics.py:213-215."""
    return 2 * np.pi * C0 / lam_m * EPS0 * np.asarray(eps_imag)


# ---------------------------------------------------------------------------
# Gaussian VCSEL beam and one-way Huygens source (vcsel.py:77-170)
# ---------------------------------------------------------------------------
def beam_params(z_um, waist_um, lambda_nm, n=1.0):
    zr = math.pi * n * waist_um ** 2 / (lambda_nm * 1e-3)
    w = waist_um * math.sqrt(1.0 + (z_um / zr) ** 2)
    R = math.inf if abs(z_um) < 1e-12 else z_um + zr ** 2 / z_um
    return w, R


def _phase(u, R, lambda_nm, n, tilt_deg):
    k = 2 * math.pi * n / (lambda_nm * 1e-3)
    ph = k * math.sin(math.radians(tilt_deg)) * u
    if math.isfinite(R):
        ph = ph - k * u ** 2 / (2.0 * R)
    return ph


def profile_1d(y_um, yc_um, z_um, waist_um, lambda_nm, n=1.0, tilt_deg=0.0):
    y = np.asarray(y_um, dtype=np.float64) - yc_um
    w, R = beam_params(z_um, waist_um, lambda_nm, n)
    return math.sqrt(waist_um / w) * np.exp(-(y / w) ** 2), _phase(y, R, lambda_nm, n, tilt_deg)


def profile_2d(y_um, z_um, yc_um, zc_um, zprop_um, wy0, wz0, lambda_nm, n=1.0, tilt_deg=0.0):
    y = np.asarray(y_um, dtype=np.float64)[:, None] - yc_um
    zz = np.asarray(z_um, dtype=np.float64)[None, :] - zc_um
    wy, Ry = beam_params(zprop_um, wy0, lambda_nm, n)
    wz, Rz = beam_params(zprop_um, wz0, lambda_nm, n)
    amp = math.sqrt((wy0 / wy) * (wz0 / wz)) * np.exp(-(y / wy) ** 2 - (zz / wz) ** 2)
    ph = _phase(y, Ry, lambda_nm, n, tilt_deg) + np.zeros_like(zz)
    if math.isfinite(Rz):
        ph = ph - (2 * math.pi * n / (lambda_nm * 1e-3)) * zz ** 2 / (2.0 * Rz)
    return amp, ph


def kx_dx(lambda_nm, dx_m, c_dt, n=1.0, tilt_deg=0.0):
    w_dt_2 = math.pi * c_dt / (lambda_nm * 1e-9)
    arg = min(1.0, n * dx_m / c_dt * math.sin(w_dt_2))
    return 2.0 * math.asin(arg) * math.cos(math.radians(tilt_deg))


class Huygens:
    """Two soft-source planes ix (+) and ix+1 (-), vcsel.py:136-170."""

    def __init__(self, ix, amp, phase, omega, kdx):
        self.ix = int(ix)
        g = 2.0 * abs(math.sin(kdx)) or 1.0
        self.amp = np.asarray(np.asarray(amp) / g, dtype=F32)
        self.ph1 = np.asarray(np.asarray(phase), dtype=F32)
        self.ph2 = np.asarray(np.asarray(phase) + kdx, dtype=F32)
        self.omega = float(omega)
        self.kdx = float(kdx)

    def on_ey_grid(self):
        s = Huygens.__new__(Huygens)
        s.ix, s.omega, s.kdx = self.ix, self.omega, self.kdx
        s.amp = F32(0.5) * (self.amp[:-1] + self.amp[1:])
        s.ph1 = F32(0.5) * (self.ph1[:-1] + self.ph1[1:])
        s.ph2 = F32(0.5) * (self.ph2[:-1] + self.ph2[1:])
        return s

    def inject(self, F, t, env, fp64=False):
        wt = self.omega * t
        if fp64:
            F[self.ix] += env * np.sin(wt + self.ph1.astype(np.float64)) * self.amp
            F[self.ix + 1] -= env * np.sin(wt + self.ph2.astype(np.float64)) * self.amp
        else:
            F[self.ix] += env * np.sin(F32(wt) + self.ph1) * self.amp
            F[self.ix + 1] -= env * np.sin(F32(wt) + self.ph2) * self.amp


def cw_envelope(t, f0, ramp_periods=None):
    """fdtd2d_core.py:784-787: 1 - exp(-(t/(2 sigma_t))^2), sigma_t = 4/(2 pi f0).
    ramp_periods: sigma_t chosen so that the reference's 6 sigma_t start-up equals
    that many periods."""
    st = 4.0 / (2 * np.pi * f0) if ramp_periods is None else ramp_periods / (6.0 * f0)
    return float(1 - np.exp(-((t / (2 * st)) ** 2)))


# ---------------------------------------------------------------------------
# 2D setup (fdtd2d_core.py:122-349, 445-455)
# ---------------------------------------------------------------------------
def materials_2d(Nx, Ny, dx, y0, wg_n, wg_top, stack, n_sub, bead=None,
                 x_wg=(0.0, None), lam_m=850e-9, tm=False):
    """Flat layer stack (fdtd2d_core.py:122-259, ``stack`` path).

    stack: [(t_um, n), ...] from the core downward (n may be complex);
    n_sub: substrate below the stack (real); bead: dict(xc, yc, r, n) in metres;
    x_wg: (x_start, x_end) of the core in metres (x_end None = open).
    Returns (eps_r f32, sigma f32, tm_patch dict or None)."""
    lossy = any(complex(n).imag > 0 for _, n in stack)
    wg_n_c = complex(wg_n, 0.0) if lossy else wg_n
    edt = np.complex128 if lossy else np.float64
    eps = np.full((Nx, Ny), N_AIR ** 2, dtype=np.complex128 if lossy else np.float32)
    ys = y0 + np.arange(Ny) * dx
    bounds, yt = [], 0.0
    for t_um, n in stack:
        yb = yt - float(t_um) * 1e-6
        nc = complex(n)
        bounds.append((yt, yb, nc if lossy else nc.real))
        yt = yb
    y_sub = yt

    def eps_y(y, core):
        e = np.full(y.shape, N_AIR ** 2, dtype=edt)
        e[y < y_sub] = (float(n_sub) + 0j) ** 2 if lossy else n_sub ** 2
        for a, b, n in bounds:
            e[(y >= b) & (y < a)] = n ** 2
        if core:
            e[(y >= 0.0) & (y < wg_top)] = wg_n_c ** 2
        return e

    col = column_average(ys, dx, lambda y: eps_y(y, False))
    col_core = column_average(ys, dx, lambda y: eps_y(y, True))
    eps[:, :] = col[None, :]
    xs = np.arange(Nx) * dx
    x_end = x_wg[1] if x_wg[1] is not None else np.inf
    in_wg = (xs >= x_wg[0]) & (xs <= x_end)
    if in_wg.any():
        eps[in_wg, :] = col_core[None, :]
    patch = None
    if tm:
        patch = dict(layer=dict(
            in_wg_x=in_wg,
            h_out=column_average(ys[:-1], dx, lambda y: eps_y(y, False).real,
                                 harmonic=True, shift=0.5 * dx),
            h_core=column_average(ys[:-1], dx, lambda y: eps_y(y, True).real,
                                  harmonic=True, shift=0.5 * dx)))
    if bead is not None:
        r, xc, yc, nb = bead['r'], bead['xc'], bead['yc'], bead['n']
        if not (xc + r < xs[0] or xc - r > xs[-1]):
            ix0 = max(0, int((xc - r) / dx) - 2)
            ix1 = min(Nx, int((xc + r) / dx) + 2)
            jy0 = max(0, int((yc - r - ys[0]) / dx) - 2)
            jy1 = min(Ny, int((yc + r - ys[0]) / dx) + 3)
            if ix1 > ix0 and jy1 > jy0:
                if tm:
                    patch.update(eps_bg=eps[ix0:ix1, jy0:jy1].real.astype(np.float64),
                                 ix0=ix0, jy0=jy0, xs=xs[ix0:ix1], ys=ys[jy0:jy1],
                                 xc=xc, yc=yc, r=r, n=nb, dx=dx)
                blend(eps[ix0:ix1, jy0:jy1],
                      circle_fraction(xs[ix0:ix1], ys[jy0:jy1], xc, yc, r, dx),
                      complex(nb, 0.0) if lossy else nb)
    if lossy:
        sig = loss_sigma(eps.imag, lam_m).astype(F32)
        eps = eps.real.astype(F32)
    else:
        sig = np.zeros((Nx, Ny), F32)
    return eps, sig, patch


def te_coeffs(eps, sig, dt, dx):
    """fdtd2d_core.py:262-270."""
    cn = (1 - sig * dt / (2 * EPS0 * eps))
    cd = (1 + sig * dt / (2 * EPS0 * eps))
    return (cn / cd).astype(F32), (dt / (EPS0 * eps * dx) / cd).astype(F32)


def tm_coeffs(eps, sig, dt, dx, patch):
    """fdtd2d_core.py:445-455 + _apply_bead_tm :297-349 + _tm_loss :283-294.
    Returns (Ca_ex, Ca_ey, Da_ex or None, Da_ey or None)."""
    e_ex = 0.5 * (eps[:-1, :] + eps[1:, :])
    e_ey = 0.5 * (eps[:, :-1] + eps[:, 1:])
    ca_x = (dt / (EPS0 * e_ex * dx)).astype(F32)
    ca_y = (dt / (EPS0 * e_ey * dx)).astype(F32)
    c = dt / (EPS0 * dx)
    h = None
    if patch:
        lp = patch.get('layer')
        if lp is not None:
            h = np.where(lp['in_wg_x'][:, None], lp['h_core'][None, :], lp['h_out'][None, :])
            ca_y[...] = (c / h).astype(F32)
        if 'eps_bg' in patch:
            eb_ = patch['eps_bg']
            ix0, jy0 = patch['ix0'], patch['jy0']
            xs, ys, xc, yc, r = patch['xs'], patch['ys'], patch['xc'], patch['yc'], patch['r']
            eb = patch['n'] ** 2

            def tensor(xp_, yp_, ea, eh, comp, h_=None):
                f = circle_fraction(xp_, yp_, xc, yc, r, h_)
                X = xp_[:, None] - xc
                Y = yp_[None, :] - yc
                d = np.maximum(np.sqrt(X * X + Y * Y), 1e-30)
                nc2 = (X / d) ** 2 if comp == 'x' else (Y / d) ** 2
                mean = (1 - f) * ea + f * eb
                hmean = (1 - f) / eh + f / eb
                return f, nc2 * hmean + (1 - nc2) / mean

            dx_ = patch['dx']
            f, inv = tensor(xs[:-1] + 0.5 * dx_, ys, 0.5 * (eb_[:-1] + eb_[1:]),
                            1.0 / (0.5 * (1.0 / eb_[:-1] + 1.0 / eb_[1:])), 'x', dx_)
            sl = (slice(ix0, ix0 + inv.shape[0]), slice(jy0, jy0 + inv.shape[1]))
            blk = ca_x[sl].astype(np.float64)
            m = f > 0
            blk[m] = c * inv[m]
            ca_x[sl] = blk.astype(F32)
            eh = 1.0 / (0.5 * (1.0 / eb_[:, :-1] + 1.0 / eb_[:, 1:]))
            if h is not None:
                hb = h[ix0:ix0 + eh.shape[0], jy0:jy0 + eh.shape[1]]
                eh[:hb.shape[0], :hb.shape[1]] = hb
            f, inv = tensor(xs, ys[:-1] + 0.5 * dx_, 0.5 * (eb_[:, :-1] + eb_[:, 1:]), eh, 'y', dx_)
            sl = (slice(ix0, ix0 + inv.shape[0]), slice(jy0, jy0 + inv.shape[1]))
            blk = ca_y[sl].astype(np.float64)
            m = f > 0
            blk[m] = c * inv[m]
            ca_y[sl] = blk.astype(F32)
    if not bool(np.any(sig > 0)):
        return ca_x, ca_y, None, None
    s_ex = 0.5 * (sig[:-1, :] + sig[1:, :])
    s_ey = 0.5 * (sig[:, :-1] + sig[:, 1:])
    a_ex = s_ex * dt / (2 * EPS0 * e_ex)
    a_ey = s_ey * dt / (2 * EPS0 * e_ey)
    ca_x /= (1 + a_ex).astype(F32)
    ca_y /= (1 + a_ey).astype(F32)
    return ca_x, ca_y, ((1 - a_ex) / (1 + a_ex)).astype(F32), ((1 - a_ey) / (1 + a_ey)).astype(F32)


# ---------------------------------------------------------------------------
# 2D steppers (boundaries.py:164-274; loop order fdtd2d_core.py:781-833)
# ---------------------------------------------------------------------------
class Grid2D:
    """One 2D CPML solve in the reference's array layout (full-domain psi)."""

    def __init__(self, pol, Nx, Ny, dx, dt, cx, cy, src, coef, dtype=F32, pec=(1, 1, 1, 1)):
        self.pol, self.Nx, self.Ny, self.dx, self.dt = pol, Nx, Ny, dx, dt
        self.cx, self.cy, self.src, self.dtype = cx, cy, src, dtype
        self.fp64 = dtype == np.float64
        self.pec = pec
        z = lambda *s: np.zeros(s, dtype)
        up = (lambda a: None if a is None else a.astype(dtype))
        if pol == 's':
            self.ce_e, self.ce_h = up(coef['ce_e']), up(coef['ce_h'])
            self.Ez, self.Hx, self.Hy = z(Nx, Ny), z(Nx, Ny - 1), z(Nx - 1, Ny)
            self.p_hxy, self.p_hyx = z(Nx, Ny - 1), z(Nx - 1, Ny)
            self.p_ezx, self.p_ezy = z(Nx - 2, Ny - 2), z(Nx - 2, Ny - 2)
        else:
            self.ca_x, self.ca_y = up(coef['ca_x']), up(coef['ca_y'])
            self.da_x, self.da_y = up(coef.get('da_x')), up(coef.get('da_y'))
            self.Ex, self.Ey, self.Hz = z(Nx - 1, Ny), z(Nx, Ny - 1), z(Nx - 1, Ny - 1)
            self.p_hzx, self.p_hzy = z(Nx - 1, Ny - 1), z(Nx - 1, Ny - 1)
            self.p_exy, self.p_eyx = z(Nx - 1, Ny - 2), z(Nx - 2, Ny - 1)
        ch = dt / (MU0 * dx)
        self.ch = np.float64(F32(ch)) if self.fp64 else F32(ch)
        P = {k: up(v) for k, v in cx.items()}
        Q = {k: up(v) for k, v in cy.items()}
        self.P, self.Q = P, Q

    def step(self, n, env, before_pec=None):
        """One leapfrog step; before_pec(field) runs after the source and before the
        PEC termination (the stitch drive, fdtd2d_core.py:1439-1441, 1462-1464)."""
        t = n * self.dt
        P, Q, ch = self.P, self.Q, self.ch
        if self.pol == 's':
            Ez, Hx, Hy = self.Ez, self.Hx, self.Hy
            d = Ez[:, 1:] - Ez[:, :-1]
            self.p_hxy = Q['bh'][None, :] * self.p_hxy + Q['ch'][None, :] * d
            Hx -= ch * (d / Q['kh'][None, :] + self.p_hxy)
            d = Ez[1:, :] - Ez[:-1, :]
            self.p_hyx = P['bh'][:, None] * self.p_hyx + P['ch'][:, None] * d
            Hy += ch * (d / P['kh'][:, None] + self.p_hyx)
            dhy = Hy[1:, 1:-1] - Hy[:-1, 1:-1]
            dhx = Hx[1:-1, 1:] - Hx[1:-1, :-1]
            self.p_ezx = P['be'][1:-1, None] * self.p_ezx + P['ce'][1:-1, None] * dhy
            self.p_ezy = Q['be'][None, 1:-1] * self.p_ezy + Q['ce'][None, 1:-1] * dhx
            Ez[1:-1, 1:-1] = (self.ce_e[1:-1, 1:-1] * Ez[1:-1, 1:-1]
                              + self.ce_h[1:-1, 1:-1] * (dhy / P['ke'][1:-1, None] + self.p_ezx
                                                         - dhx / Q['ke'][None, 1:-1] - self.p_ezy))
            self.src.inject(Ez, t, env, self.fp64)
            if before_pec is not None:
                before_pec(Ez)
            xl, xh, yl, yh = self.pec
            if xl: Ez[0, :] = 0.0
            if xh: Ez[-1, :] = 0.0
            if yl: Ez[:, 0] = 0.0
            if yh: Ez[:, -1] = 0.0
        else:
            Ex, Ey, Hz = self.Ex, self.Ey, self.Hz
            dyx = Ey[1:, :] - Ey[:-1, :]
            dxy = Ex[:, 1:] - Ex[:, :-1]
            self.p_hzx = P['bh'][:, None] * self.p_hzx + P['ch'][:, None] * dyx
            self.p_hzy = Q['bh'][None, :] * self.p_hzy + Q['ch'][None, :] * dxy
            Hz -= ch * ((dyx / P['kh'][:, None] + self.p_hzx) - (dxy / Q['kh'][None, :] + self.p_hzy))
            if self.da_x is not None:
                Ex *= self.da_x
                Ey *= self.da_y
            d = Hz[:, 1:] - Hz[:, :-1]
            self.p_exy = Q['be'][None, 1:-1] * self.p_exy + Q['ce'][None, 1:-1] * d
            Ex[:, 1:-1] += self.ca_x[:, 1:-1] * (d / Q['ke'][None, 1:-1] + self.p_exy)
            d = Hz[1:, :] - Hz[:-1, :]
            self.p_eyx = P['be'][1:-1, None] * self.p_eyx + P['ce'][1:-1, None] * d
            Ey[1:-1, :] += -self.ca_y[1:-1, :] * (d / P['ke'][1:-1, None] + self.p_eyx)
            self.src.inject(Ey, t, env, self.fp64)
            if before_pec is not None:
                before_pec(Ey)
            xl, xh, yl, yh = self.pec
            if xl: Ey[0, :] = 0.0
            if xh: Ey[-1, :] = 0.0
            if yl: Ex[:, 0] = 0.0
            if yh: Ex[:, -1] = 0.0

    # -- epilogue fields (fdtd2d_core.py:458-486, 818-834) --
    def field(self):
        if self.pol == 's':
            return self.Ez
        Ey = self.Ey
        out = np.zeros((Ey.shape[0], Ey.shape[1] + 1), self.dtype)
        out[:, 1:-1] = 0.5 * (Ey[:, :-1] + Ey[:, 1:])
        out[:, 0] = Ey[:, 0]
        out[:, -1] = Ey[:, -1]
        return out

    def ex_node(self):
        Ex = self.Ex
        out = np.zeros((Ex.shape[0] + 1, Ex.shape[1]), self.dtype)
        out[1:-1, :] = 0.5 * (Ex[:-1, :] + Ex[1:, :])
        out[0, :] = Ex[0, :]
        out[-1, :] = Ex[-1, :]
        return out

    def intensity(self, field):
        if self.pol == 's':
            return field * field
        s = self.Ex * self.Ex
        out = np.zeros((s.shape[0] + 1, s.shape[1]), self.dtype)
        out[1:-1, :] = 0.5 * (s[:-1, :] + s[1:, :])
        out[0, :] = s[0, :]
        out[-1, :] = s[-1, :]
        return field * field + out

    def flux_pairs(self, il):
        """flux.py:77-81."""
        if self.pol == 's':
            return ((-1.0, self.Ez[il], self.Hy[il - 1], self.Hy[il]),)
        return ((+1.0, self.Ey[il], self.Hz[il - 1], self.Hz[il]),)


def tm_ex2_node(Ex):
    """_tm_ex2_node (fdtd2d_core.py:477-486): Ex^2 squared-averaged onto the nodes."""
    s = Ex * Ex
    out = np.zeros((Ex.shape[0] + 1, Ex.shape[1]), dtype=np.float32)
    out[1:-1, :] = 0.5 * (s[:-1, :] + s[1:, :])
    out[0, :] = s[0, :]
    out[-1, :] = s[-1, :]
    return out


class PlaneFlux:
    """Running DFT of E and of the plane-averaged H on x-planes (flux.py:19-57)."""

    def __init__(self, omega, dt, dtype=F32):
        self.omega, self.dt = float(omega), float(dt)
        self.c = np.complex128 if dtype == np.float64 else np.complex64
        self.acc, self.n = {}, {}

    def add(self, key, t, pairs):
        pe = self.c(np.exp(-1j * self.omega * t))
        ph = self.c(np.exp(-1j * self.omega * (t - 0.5 * self.dt)))
        lst = self.acc.get(key)
        if lst is None:
            lst = [[s, np.zeros(E.shape, self.c), np.zeros(E.shape, self.c)] for s, E, _, _ in pairs]
            self.acc[key] = lst
            self.n[key] = 0
        for a, (s, E, H0, H1) in zip(lst, pairs):
            a[1] += E.astype(self.c) * pe
            a[2] += (0.5 * (H0 + H1)).astype(self.c) * ph
        self.n[key] += 1

    def flux(self, key):
        n = self.n.get(key, 0)
        if not n:
            return float('nan')
        s = 0.0
        for sign, aE, aH in self.acc[key]:
            s += sign * 0.5 * float(np.real(np.sum(aE * np.conj(aH), dtype=np.complex128)))
        return s * (2.0 / n) ** 2


# ---------------------------------------------------------------------------
# 3D setup (fdtd3d_core.py:119-378, 474-494)
# ---------------------------------------------------------------------------
def eps_3d(Nx, Ny, Nz, dx_um, y0_um, z0_um, wg_n, t_wg_um, stack, n_sub, beads=(),
           x_wg_start_um=0.0):
    """build_eps3d (fdtd3d_core.py:119-292) for a slab core with an air zone in
    front of the entry facet (local-x mode), ``stack`` path, tensor data.

    beads: list of dict(x_um, y_um, z_um, d_um, n); each is blended in turn with
    the reference's single-bead procedure (boxes must not overlap).
    Returns (eps (f32 or complex64), tensor dict(layer=..., beads=[...]))."""
    lossy = any(complex(n).imag > 0 for _, n in stack)
    wg_n_c = complex(wg_n, 0.0) if lossy else wg_n
    edt = np.complex128 if lossy else np.float64
    ys = y0_um + np.arange(Ny) * dx_um
    bounds, yt = [], 0.0
    for t_um, n in stack:
        yb = yt - float(t_um)
        nc = complex(n)
        bounds.append((yt, yb, nc if lossy else nc.real))
        yt = yb
    y_sub = yt

    def eps_y(y, core, n_core=None):
        e = np.full(y.shape, N_AIR ** 2, dtype=edt)
        e[y < y_sub] = (float(n_sub) + 0j) ** 2 if lossy else n_sub ** 2
        for a, b, n in bounds:
            e[(y >= b) & (y < a)] = n ** 2
        if core:
            e[(y >= 0.0) & (y < t_wg_um)] = (wg_n_c if n_core is None else n_core) ** 2
        return e

    col = column_average(ys, dx_um, lambda y: eps_y(y, True))
    eps = np.broadcast_to(col[None, :, None], (Nx, Ny, Nz)).copy()
    xs = np.arange(Nx) * dx_um
    if x_wg_start_um and x_wg_start_um > 0:
        eps[xs < x_wg_start_um, :, :] = N_AIR ** 2

    def hcol(core, n_core=None):
        return column_average(ys[:-1], dx_um, lambda y: np.real(eps_y(y, core, n_core)),
                              harmonic=True, shift=0.5 * dx_um).astype(np.float64)
    T = np.full((Nx, Nz), 1, dtype=np.int8)
    if x_wg_start_um and x_wg_start_um > 0:
        T[xs < x_wg_start_um, :] = 3
    cols = np.stack([hcol(False), hcol(True), hcol(True, N_AIR), np.full(Ny - 1, N_AIR ** 2)])
    tp = dict(layer=dict(T=T, cols=cols), beads=[])
    zs_all = z0_um + np.arange(Nz) * dx_um
    for bd in beads:
        r = bd['d_um'] / 2.0
        xc, yc, zc = bd['x_um'], bd.get('y_um', -r), bd.get('z_um', 0.0)
        i0 = max(0, int((xc - r) / dx_um) - 2)
        i1 = min(Nx, int((xc + r) / dx_um) + 3)
        j0 = max(0, int((yc - r - y0_um) / dx_um) - 2)
        j1 = min(Ny, int((yc + r - y0_um) / dx_um) + 3)
        k0 = max(0, int((zc - r - z0_um) / dx_um) - 2)
        k1 = min(Nz, int((zc + r - z0_um) / dx_um) + 3)
        if not (i1 > i0 and j1 > j0 and k1 > k0):
            continue
        sub = eps[i0:i1, j0:j1, k0:k1]
        tp['beads'].append(dict(eps_bg=sub.real.astype(np.float64), i0=i0, j0=j0, k0=k0,
                                xs=xs[i0:i1], ys=ys[j0:j1], zs=zs_all[k0:k1],
                                xc=xc, yc=yc, zc=zc, r=r, n=bd['n']))
        blend(sub, sphere_fraction(xs[i0:i1], ys[j0:j1], zs_all[k0:k1], xc, yc, zc, r, dx_um),
              complex(bd['n'], 0.0) if lossy else bd['n'])
    return eps, tp


def _stag(inv, ax):
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[ax] = slice(None, -1)
    b[ax] = slice(1, None)
    return (F32(0.5) * (inv[tuple(a)] + inv[tuple(b)])).astype(F32)


def coeffs_3d(eps, tp, dt, dx, dx_um, lam_m):
    """_split_eps3 + _inv_loss + _ce_arrays + _stagger_da
    (fdtd3d_core.py:466-494, 305-378).  Returns (ce_x, ce_y, ce_z, (Dx, Dy, Dz) or None)."""
    if np.iscomplexobj(eps):
        e, eim = eps.real.astype(F32), eps.imag.astype(F32)
    else:
        e, eim = eps, None
    inv = F32(dt / (EPS0 * dx)) / e
    da = None
    if eim is not None and np.any(eim > 0):
        a = (F32(np.pi * C0 / lam_m * dt) * eim) / e
        inv /= (1 + a)
        da = ((1 - a) / (1 + a)).astype(F32)
    ces = [_stag(inv, 0), _stag(inv, 1), _stag(inv, 2)]
    lp = tp.get('layer')
    if lp is not None:
        cy = ces[1]
        hinv = (dt / (EPS0 * dx) / lp['cols']).astype(F32)
        T = lp['T'][:, None, :]
        for t in range(hinv.shape[0]):
            np.copyto(cy, hinv[t][None, :, None], where=(T == t))
        if da is not None:
            cy *= _stag(F32(0.5) * (1 + da), 1)
    c = dt / (EPS0 * dx)
    for bp in tp.get('beads', []):
        eb = bp['n'] ** 2
        for ax in range(3):
            ce = ces[ax]
            e0 = bp['eps_bg']
            nb = e0.shape[ax]
            e_nx = np.take(e0, np.minimum(np.arange(nb) + 1, nb - 1), axis=ax)
            e_a = 0.5 * (e0 + e_nx)
            e_h = 1.0 / (0.5 * (1.0 / e0 + 1.0 / e_nx))
            if ax == 1 and lp is not None:
                i0, j0, k0 = bp['i0'], bp['j0'], bp['k0']
                Tb = lp['T'][i0:i0 + e0.shape[0], k0:k0 + e0.shape[2]]
                cols = lp['cols'][:, j0:j0 + e0.shape[1]]
                hb = np.transpose(cols[Tb], (0, 2, 1))
                e_h[:, :hb.shape[1], :] = hb
            fac = _stag(F32(0.5) * (1 + da), ax) if da is not None else None
            o = [0.0, 0.0, 0.0]
            o[ax] = 0.5 * dx_um
            xs, ys, zs = bp['xs'] + o[0], bp['ys'] + o[1], bp['zs'] + o[2]
            a0, b0, c0 = bp['i0'], bp['j0'], bp['k0']
            na = min(len(xs), ce.shape[0] - a0)
            nbb = min(len(ys), ce.shape[1] - b0)
            nc = min(len(zs), ce.shape[2] - c0)
            if na <= 0 or nbb <= 0 or nc <= 0:
                continue
            xs, ys, zs = xs[:na], ys[:nbb], zs[:nc]
            f = sphere_fraction(xs, ys, zs, bp['xc'], bp['yc'], bp['zc'], bp['r'], dx_um)
            m = f > 0
            if m.any():
                X = xs[:, None, None] - bp['xc']
                Y = ys[None, :, None] - bp['yc']
                Z = zs[None, None, :] - bp['zc']
                d = np.maximum(np.sqrt(X * X + Y * Y + Z * Z), 1e-30)
                nc2 = ((X, Y, Z)[ax] / d) ** 2
                ebh = e_h[:na, :nbb, :nc]
                eba = e_a[:na, :nbb, :nc]
                inv_t = nc2 * ((1 - f) / ebh + f / eb) + (1 - nc2) / ((1 - f) * eba + f * eb)
                sl = (slice(a0, a0 + na), slice(b0, b0 + nbb), slice(c0, c0 + nc))
                blk = ce[sl].astype(np.float64)
                val = c * np.broadcast_to(inv_t, f.shape)
                if fac is not None:
                    val = val * fac[sl].astype(np.float64)
                blk[m] = val[m]
                ce[sl] = blk.astype(F32)
    dd = None if da is None else (_stag(da, 0), _stag(da, 1), _stag(da, 2))
    return ces[0], ces[1], ces[2], dd


# ---------------------------------------------------------------------------
# 3D CPML stepper with psi kept only in the PML strips (boundaries3d.py:201-362)
# ---------------------------------------------------------------------------
class _Strip:
    """psi of one stretch direction, stored only where c != 0 (boundaries3d.py:201-251)."""

    def __init__(self, shape, axis, b, c, k, dtype):
        self.parts = []
        N = shape[axis]
        cn = np.abs(np.asarray(c, dtype=np.float64))
        lo = 0
        while lo < N and cn[lo] > 0.0:
            lo += 1
        hi = 0
        while hi < N and cn[N - 1 - hi] > 0.0:
            hi += 1
        if lo + hi >= N:
            lo, hi = N, 0
        bc = lambda v: v.reshape(tuple(-1 if q == axis else 1 for q in range(3)))
        shp = lambda n: tuple(n if q == axis else shape[q] for q in range(3))
        km1 = (1.0 / k - 1.0)
        for a0, a1 in ((0, lo), (N - hi, N)):
            if a1 > a0:
                sl = tuple(slice(a0, a1) if q == axis else slice(None) for q in range(3))
                self.parts.append([sl, bc(b[a0:a1]), bc(c[a0:a1]), np.zeros(shp(a1 - a0), dtype),
                                   bc(km1[a0:a1])])

    def add_into(self, F, dF, coef, sign):
        for sl, b, c, p, km1 in self.parts:
            p *= b
            p += c * dF[sl]
            add = p + km1 * dF[sl]
            if np.ndim(coef) == 0:
                F[sl] += (sign * coef) * add
            else:
                F[sl] += (sign * coef[sl]) * add


class Grid3D:
    """One 3D CPML solve in the reference's array layout."""

    def __init__(self, Nx, Ny, Nz, dx, dt, cpml, ce, da, src, src_comp, dtype=F32,
                 faces=('xmin', 'xmax', 'ymin', 'ymax', 'zmin', 'zmax')):
        self.Nx, self.Ny, self.Nz, self.dx, self.dt = Nx, Ny, Nz, dx, dt
        self.dtype, self.fp64 = dtype, dtype == np.float64
        self.faces = faces
        up = (lambda a: a.astype(dtype))
        self.ce = [up(a) for a in ce]
        self.da = None if da is None else [up(a) for a in da]
        z = lambda *s: np.zeros(s, dtype)
        self.Ex, self.Ey, self.Ez = z(Nx - 1, Ny, Nz), z(Nx, Ny - 1, Nz), z(Nx, Ny, Nz - 1)
        self.Hx, self.Hy, self.Hz = z(Nx, Ny - 1, Nz - 1), z(Nx - 1, Ny, Nz - 1), z(Nx - 1, Ny - 1, Nz)
        ch = dt / (MU0 * dx)
        self.ch = np.float64(F32(ch)) if self.fp64 else F32(ch)
        self.src, self.src_comp = src, src_comp
        X, Y, Zp = ({k: up(v) for k, v in cpml[a].items()} for a in range(3))
        S = lambda shp, ax, P, t, cut=False: _Strip(
            shp, ax, P['b' + t][1:-1] if cut else P['b' + t], P['c' + t][1:-1] if cut else P['c' + t],
            P['k' + t][1:-1] if cut else P['k' + t], dtype)
        sHx, sHy, sHz = (Nx, Ny - 1, Nz - 1), (Nx - 1, Ny, Nz - 1), (Nx - 1, Ny - 1, Nz)
        self.p_hx_z, self.p_hx_y = S(sHx, 2, Zp, 'h'), S(sHx, 1, Y, 'h')
        self.p_hy_x, self.p_hy_z = S(sHy, 0, X, 'h'), S(sHy, 2, Zp, 'h')
        self.p_hz_y, self.p_hz_x = S(sHz, 1, Y, 'h'), S(sHz, 0, X, 'h')
        sEx, sEy, sEz = (Nx - 1, Ny - 2, Nz - 2), (Nx - 2, Ny - 1, Nz - 2), (Nx - 2, Ny - 2, Nz - 1)
        self.p_ex_y, self.p_ex_z = S(sEx, 1, Y, 'e', True), S(sEx, 2, Zp, 'e', True)
        self.p_ey_z, self.p_ey_x = S(sEy, 2, Zp, 'e', True), S(sEy, 0, X, 'e', True)
        self.p_ez_x, self.p_ez_y = S(sEz, 0, X, 'e', True), S(sEz, 1, Y, 'e', True)

    def fields(self):
        return dict(Ex=self.Ex, Ey=self.Ey, Ez=self.Ez, Hx=self.Hx, Hy=self.Hy, Hz=self.Hz)

    def step(self, n, env):
        Ex, Ey, Ez, Hx, Hy, Hz, ch = self.Ex, self.Ey, self.Ez, self.Hx, self.Hy, self.Hz, self.ch
        d1 = Ey[:, :, 1:] - Ey[:, :, :-1]
        d2 = Ez[:, 1:, :] - Ez[:, :-1, :]
        Hx += ch * (d1 - d2)
        self.p_hx_z.add_into(Hx, d1, ch, +1)
        self.p_hx_y.add_into(Hx, d2, ch, -1)
        d1 = Ez[1:, :, :] - Ez[:-1, :, :]
        d2 = Ex[:, :, 1:] - Ex[:, :, :-1]
        Hy += ch * (d1 - d2)
        self.p_hy_x.add_into(Hy, d1, ch, +1)
        self.p_hy_z.add_into(Hy, d2, ch, -1)
        d1 = Ex[:, 1:, :] - Ex[:, :-1, :]
        d2 = Ey[1:, :, :] - Ey[:-1, :, :]
        Hz += ch * (d1 - d2)
        self.p_hz_y.add_into(Hz, d1, ch, +1)
        self.p_hz_x.add_into(Hz, d2, ch, -1)
        if self.da is not None:
            Ex *= self.da[0]
            Ey *= self.da[1]
            Ez *= self.da[2]
        cx, cy, cz = self.ce
        d1 = Hz[:, 1:, 1:-1] - Hz[:, :-1, 1:-1]
        d2 = Hy[:, 1:-1, 1:] - Hy[:, 1:-1, :-1]
        v = Ex[:, 1:-1, 1:-1]
        c = cx[:, 1:-1, 1:-1]
        v += c * (d1 - d2)
        self.p_ex_y.add_into(v, d1, c, +1)
        self.p_ex_z.add_into(v, d2, c, -1)
        d1 = Hx[1:-1, :, 1:] - Hx[1:-1, :, :-1]
        d2 = Hz[1:, :, 1:-1] - Hz[:-1, :, 1:-1]
        v = Ey[1:-1, :, 1:-1]
        c = cy[1:-1, :, 1:-1]
        v += c * (d1 - d2)
        self.p_ey_z.add_into(v, d1, c, +1)
        self.p_ey_x.add_into(v, d2, c, -1)
        d1 = Hy[1:, 1:-1, :] - Hy[:-1, 1:-1, :]
        d2 = Hx[1:-1, 1:, :] - Hx[1:-1, :-1, :]
        v = Ez[1:-1, 1:-1, :]
        c = cz[1:-1, 1:-1, :]
        v += c * (d1 - d2)
        self.p_ez_x.add_into(v, d1, c, +1)
        self.p_ez_y.add_into(v, d2, c, -1)
        f = self.faces
        if 'xmin' in f: Ey[0] = 0; Ez[0] = 0
        if 'xmax' in f: Ey[-1] = 0; Ez[-1] = 0
        if 'ymin' in f: Ex[:, 0] = 0; Ez[:, 0] = 0
        if 'ymax' in f: Ex[:, -1] = 0; Ez[:, -1] = 0
        if 'zmin' in f: Ex[:, :, 0] = 0; Ey[:, :, 0] = 0
        if 'zmax' in f: Ex[:, :, -1] = 0; Ey[:, :, -1] = 0
        self.src.inject(getattr(self, self.src_comp), n * self.dt, env, self.fp64)

    def box_e2(self, xs, ys, zs):
        """_box_E2 (fdtd3d_core.py:477-481)."""
        return sum(np.sum(F[xs, ys, zs] ** 2, dtype=np.float64) for F in (self.Ex, self.Ey, self.Ez))

    def flux_pairs(self, il):
        """flux.py:84-90."""
        return ((+1.0, self.Ey[il], self.Hz[il - 1], self.Hz[il]),
                (-1.0, self.Ez[il], self.Hy[il - 1], self.Hy[il]))


def sq_on_grid(F, tshape, x0, x1):
    """_sq_on_grid (fdtd3d_core.py:438-461)."""
    nF = F.shape[0]
    if nF == tshape[0]:
        S = F[x0:x1] ** 2
    else:
        i = np.arange(x0, x1)
        S = 0.5 * (F[np.clip(i - 1, 0, nF - 1)] ** 2 + F[np.clip(i, 0, nF - 1)] ** 2)
    for ax in (1, 2):
        n, t = S.shape[ax], tshape[ax]
        if n == t:
            continue
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[ax] = slice(None, -1)
        b[ax] = slice(1, None)
        mid = 0.5 * (S[tuple(a)] + S[tuple(b)])
        if n == t + 1:
            S = mid
        else:
            f_ = [slice(None)] * 3
            l_ = [slice(None)] * 3
            f_[ax] = slice(0, 1)
            l_[ax] = slice(-1, None)
            S = np.concatenate([S[tuple(f_)], mid, S[tuple(l_)]], axis=ax)
    return S


def accum_e2(I, Ex, Ey, Ez):
    """_accum_E2 (fdtd3d_core.py:464-474)."""
    Nx = I.shape[0]
    ch = max(32, Nx // 8)
    for x0 in range(0, Nx, ch):
        x1 = min(x0 + ch, Nx)
        I[x0:x1] += (sq_on_grid(Ex, I.shape, x0, x1) + sq_on_grid(Ey, I.shape, x0, x1)
                     + sq_on_grid(Ez, I.shape, x0, x1))
