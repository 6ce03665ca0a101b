"""Host setup of a solve: layer-stack columns, CPML profiles, bead sub-pixel
permittivity, staggered update coefficients and the Gaussian Huygens source.

Setup runs once per solve; the per-step work is in the CUDA engine.  The
arithmetic reproduces the reference's float32 results bit for bit (checked
against the reference-pinned oracle in tests/test_geometry_parity.py):

  CPML profiles          planar_beads/boundaries.py:104-151, planar_3d/boundaries3d.py:150-194
  layer columns          common/subpixel.py:80-94 (16 sub-samples per cell)
  bead area / volume     common/subpixel.py:25-69
  2D coefficients        planar_beads/fdtd2d_core.py:122-349, 445-455
  3D coefficients        planar_3d/fdtd3d_core.py:119-378, 474-494
  source                 common/vcsel.py:77-170

Geometry is organised as COLUMNS: the permittivity depends on y (the layer
stack) and on a small per-(x, z) column type (core column, air in front of the
entry facet, ...); beads are local patches.  Coefficient volumes are expanded
from per-type columns, then the bead boxes are patched.
"""
import itertools
import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .physics import C0, EPS0, N_AIR

F32 = np.float32


# --------------------------------------------------------------------------- CPML
def cpml_axis(N, n_lo, n_hi, dx, dt, lam_m=850e-9, m=3, R0=1e-6, kappa_max=1.0):
    """Graded CFS-CPML profiles of one axis: {'ke','be','ce'} on the N integer
    nodes and {'kh','bh','ch'} on the N-1 half nodes (float32).
    sigma_max = -(m+1) ln R0 / (2 eta0 n dx), a = a_max (1 - depth),
    a_max = 2 pi eps0 f0 / 10, b = exp(-(sigma/kappa + a) dt/eps0),
    c = sigma (b - 1) / (sigma kappa + kappa^2 a)."""
    if n_lo <= 0 and n_hi <= 0:
        one, zero = np.ones, np.zeros
        return dict(ke=one(N, F32), be=one(N, F32), ce=zero(N, F32),
                    kh=one(N - 1, F32), bh=one(N - 1, F32), ch=zero(N - 1, F32))
    eta0 = np.sqrt(4e-7 * np.pi / EPS0)
    a_max = 2.0 * np.pi * EPS0 * (C0 / lam_m) / 10.0
    smax = {n: ((-(m + 1) * np.log(R0) / (2.0 * eta0 * n * dx)) if n > 0 else 0.0) for n in (n_lo, n_hi)}

    def graded(pos):
        depth = np.zeros_like(pos)
        sg = np.zeros_like(pos)
        if n_lo > 0:
            sel = pos < n_lo
            depth[sel] = (n_lo - pos[sel]) / n_lo
            sg[sel] = smax[n_lo]
        if n_hi > 0:
            sel = pos > (N - 1 - n_hi)
            depth[sel] = (pos[sel] - (N - 1 - n_hi)) / n_hi
            sg[sel] = smax[n_hi]
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

    out = {}
    for tag, pos in (('e', np.arange(N, dtype=np.float64)), ('h', np.arange(N - 1, dtype=np.float64) + 0.5)):
        out['k' + tag], out['b' + tag], out['c' + tag] = graded(pos)
    return out


# --------------------------------------------------------------------------- sub-pixel
def _sub(S, h):
    return ((np.arange(S) + 0.5) / S - 0.5) * h


def column_average(ys, dy, eps_of_y, S=16, harmonic=False, shift=0.0):
    """Cell average of eps(y) over [y - dy/2, y + dy/2] + shift with S samples;
    arithmetic (field parallel to the layers) or harmonic (normal to them)."""
    Y = np.asarray(ys, dtype=np.float64)[:, None] + (_sub(S, dy) + shift)[None, :]
    e = np.asarray(eps_of_y(Y.ravel()))
    cplx = np.iscomplexobj(e)
    e = e.astype(np.complex128 if cplx else np.float64).reshape(Y.shape)
    if harmonic:
        return (1.0 / np.mean(1.0 / e, axis=1)).astype(np.complex64 if cplx else F32)
    return np.mean(e, axis=1).astype(np.complex64 if cplx else F32)


def ball_fraction(axes, centre, r, h, S):
    """Share of each grid cell (side h, centred on the nodes axes[0] x axes[1]
    [x axes[2]]) that lies inside the ball |p - centre| <= r: 1 for cells whose
    node is at least half a cell diagonal inside the surface, 0 beyond it, and
    for the cells the surface cuts the share of S samples per axis (at the
    centres of S equal sub-intervals) that fall inside.  The sample squares are
    summed in axis order, so the shares do not depend on how the loop is cut."""
    dim = len(axes)
    rel = [np.asarray(a, np.float64) - c for a, c in zip(axes, centre)]
    grid = np.meshgrid(*rel, indexing='ij', sparse=True)
    dist = np.sqrt(sum(g * g for g in grid))
    half = h * np.sqrt(float(dim)) / 2.0
    share = (dist <= r - half).astype(np.float64)
    cut = np.nonzero((dist > r - half) & (dist < r + half))
    if len(cut[0]):
        off = _sub(S, h)
        lead = [rel[a][cut[a]] for a in range(dim - 1)]
        last = rel[-1][cut[-1]][:, None] + off[None, :]
        last2 = last * last
        inside = np.zeros(len(cut[0]))
        for shift in itertools.product(off, repeat=dim - 1):
            s2 = sum((v + o) * (v + o) for v, o in zip(lead, shift))
            inside += np.count_nonzero(s2[:, None] + last2 <= r * r, axis=1)
        share[cut] = inside / S ** dim
    return share


def circle_fraction(xs, ys, xc, yc, r, h, S=8):
    """Area share of a disc in the cells around the nodes xs x ys (S^2 samples
    on the cells its edge cuts; the material blend of subpixel.py:25-39)."""
    return ball_fraction((xs, ys), (xc, yc), r, h, S)


def sphere_fraction(xs, ys, zs, xc, yc, zc, r, h, S=6):
    """Volume share of a sphere in the cells around xs x ys x zs (S^3 samples on
    the cells its surface cuts; subpixel.py:42-62)."""
    return ball_fraction((xs, ys, zs), (xc, yc, zc), r, h, S)


def _blend(eps, frac, n):
    sel = frac > 0
    eps[sel] = (1.0 - frac[sel]) * eps[sel] + frac[sel] * (n ** 2)


# --------------------------------------------------------------------------- layer stack
@dataclass
class Stack:
    """Planar layer stack: a core of index wg_n and thickness t_wg_um on top of
    `layers` (from the core downward: (thickness_um, n), n complex = absorbing)
    on a substrate n_sub, air above (common/layer_stack.py).

    n_sub may be a float or a depth profile with ``at_depth(d_um)`` (the layered
    cornea).  thick_m, when given, are the layer thicknesses in metres used by
    2D grids (the reference's legacy tear-film path computes them that way);
    k_sub / force_lossy carry the legacy per-layer absorption switch."""
    wg_n: complex
    t_wg_um: float
    layers: List[Tuple[float, complex]]
    n_sub: float
    thick_m: Optional[List[float]] = None
    k_sub: float = 0.0
    force_lossy: bool = False

    @property
    def lossy(self):
        return self.force_lossy or any(complex(n).imag > 0 for _, n in self.layers)

    def eps_of_y(self, unit, core=True, n_core=None):
        """eps(y) in the given length unit (1.0 = metres, 1e-6 = micrometres)."""
        lossy = self.lossy
        bounds, yt = [], 0.0
        for q, (t, n) in enumerate(self.layers):
            if unit == 1.0 and self.thick_m is not None:
                yb = yt - self.thick_m[q]
            else:
                yb = yt - float(t) * (1e-6 / unit)
            nc = complex(n)
            bounds.append((yt, yb, nc if lossy else nc.real))
            yt = yb
        y_sub = yt
        top = self.t_wg_um * (1e-6 / unit)
        wn = complex(self.wg_n) if lossy else complex(self.wg_n).real
        wg = wn if n_core is None else n_core
        dt = np.complex128 if lossy else np.float64
        sub, ks = self.n_sub, self.k_sub
        depth_scale = 1e6 if unit == 1.0 else 1.0

        def f(y):
            e = np.full(y.shape, N_AIR ** 2, dtype=dt)
            mc = y < y_sub
            if hasattr(sub, 'at_depth'):
                nd = sub.at_depth((y_sub - y[mc]) * depth_scale)
                e[mc] = (nd + 1j * ks) ** 2 if lossy else nd ** 2
            else:
                e[mc] = (float(sub) + 1j * ks) ** 2 if lossy else sub ** 2
            for a, b, n in bounds:
                e[(y >= b) & (y < a)] = n ** 2
            if core:
                e[(y >= 0.0) & (y < top)] = wg ** 2
            return e
        return f


# --------------------------------------------------------------------------- source
def beam(z_um, waist_um, lambda_nm, n=1.0):
    """Gaussian beam radius and wavefront radius at z (vcsel.py:84-89)."""
    zr = math.pi * n * waist_um ** 2 / (lambda_nm * 1e-3)
    w = waist_um * math.sqrt(1.0 + (z_um / zr) ** 2)
    return w, (math.inf if abs(z_um) < 1e-12 else z_um + zr ** 2 / z_um)


def _beam_phase(u, R, lambda_nm, n, tilt_deg):
    k = 2 * math.pi * n / (lambda_nm * 1e-3)
    ph = k * math.sin(math.radians(tilt_deg)) * u
    return ph - k * u ** 2 / (2.0 * R) if math.isfinite(R) else ph


def huygens_kdx(lambda_nm, dx_m, c_dt, n=1.0, tilt_deg=0.0):
    """Numerical phase advance per cell of the one-way pair (vcsel.py:126-133)."""
    arg = min(1.0, n * dx_m / c_dt * math.sin(math.pi * c_dt / (lambda_nm * 1e-9)))
    return 2.0 * math.asin(arg) * math.cos(math.radians(tilt_deg))


def huygens_arrays(amp, phase, kdx):
    """(amp, ph1, ph2) float32 of the pair on planes ix, ix+1 (vcsel.py:142-148)."""
    g = 2.0 * abs(math.sin(kdx)) or 1.0
    return (np.asarray(np.asarray(amp) / g, dtype=F32), np.asarray(phase, dtype=F32),
            np.asarray(np.asarray(phase) + kdx, dtype=F32))


def air_path_um(distance_um, dx_um):
    """Air gap between the source plane and the entry facet (vcsel.py:64-70)."""
    return max(float(distance_um or 0.0), max(1.0, 8 * float(dx_um)))


# =========================================================================== 2D
@dataclass
class Bead2D:
    x_um: float
    d_um: float
    n: complex = 1.59
    y_um: Optional[float] = None      # centre; default -r (touching the core)


@dataclass
class Spec2D:
    """A 2D full-domain solve (fdtd2d_core.run_beads, method='full', CPML)."""
    pol: str
    nx: int
    ny: int
    dx: float                          # m
    stack: Stack
    tear_m: float                      # depth below the core bottom (y at j=0 is -tear_m)
    bead: Optional[Bead2D] = None
    npml: int = 10
    lam_nm: float = 850.0
    waist_um: float = 3.0
    ramp_periods: Optional[float] = None
    length_m: Optional[float] = None     # end of the core (default: the whole grid)
    vcsel_distance_um: float = 0.0       # beam waist in front of the entry facet
    vcsel_offset_um: float = 0.0
    vcsel_tilt_deg: float = 0.0
    src_core_only: bool = False
    # stitch window (fdtd2d_core.py:1396-1412): x of node 0 in the whole domain (um)
    # and the CPML cells at the x-lo / x-hi ends (default npml at both)
    x_start_um: Optional[float] = None
    npml_x: Optional[Tuple[int, int]] = None

    @property
    def dt(self):
        return 0.5 * self.dx / (C0 * np.sqrt(2))

    @property
    def src_ix(self):
        return self.npml + 2

    @property
    def f0(self):
        return C0 / (self.lam_nm * 1e-9)


def build_2d(sp: Spec2D):
    """Coefficients, CPML profiles and source of a 2D solve (reference shapes)."""
    Nx, Ny, dx, dt = sp.nx, sp.ny, sp.dx, sp.dt
    lam_m = sp.lam_nm * 1e-9
    air = air_path_um(sp.vcsel_distance_um, dx * 1e6)
    x_facet_um = sp.src_ix * dx * 1e6 + air
    st = sp.stack
    lossy = st.lossy
    ys = -sp.tear_m + np.arange(Ny) * dx
    col = column_average(ys, dx, st.eps_of_y(1.0, core=False))
    col_core = column_average(ys, dx, st.eps_of_y(1.0, core=True))
    x0 = sp.x_start_um * 1e-6 if sp.x_start_um is not None else 0.0
    xs = x0 + np.arange(Nx) * dx
    in_wg = (xs >= x_facet_um * 1e-6) & (xs <= (sp.length_m if sp.length_m is not None else Nx * dx * 1e6 * 1e-6))
    eps = np.empty((Nx, Ny), dtype=np.complex128 if lossy else F32)
    eps[:, :] = col[None, :]
    eps[in_wg, :] = col_core[None, :]
    tm = sp.pol == 'p'
    bead_patch = None
    if sp.bead is not None:
        r = sp.bead.d_um * 1e-6 / 2.0
        xc = sp.bead.x_um * 1e-6
        yc = sp.bead.y_um * 1e-6 if sp.bead.y_um is not None else -r
        if not (xc + r < xs[0] or xc - r > xs[-1]):
            i0, i1 = max(0, int((xc - r - x0) / dx) - 2), min(Nx, int((xc + r - x0) / dx) + 2)
            j0, j1 = max(0, int((yc - r - ys[0]) / dx) - 2), min(Ny, int((yc + r - ys[0]) / dx) + 3)
            if i1 > i0 and j1 > j0:
                bead_patch = dict(bg=eps[i0:i1, j0:j1].real.astype(np.float64), i0=i0, j0=j0,
                                  xs=xs[i0:i1], ys=ys[j0:j1], xc=xc, yc=yc, r=r, n=complex(sp.bead.n).real)
                _blend(eps[i0:i1, j0:j1], circle_fraction(xs[i0:i1], ys[j0:j1], xc, yc, r, dx),
                       complex(sp.bead.n) if lossy else complex(sp.bead.n).real)
    if lossy:
        sig = (2 * np.pi * C0 / lam_m * EPS0 * eps.imag).astype(F32)
        eps = eps.real.astype(F32)
    else:
        sig = np.zeros((Nx, Ny), F32)
    out = dict(eps=eps, sig=sig, x_facet_um=x_facet_um)
    # TE: fdtd2d_core.py:262-270
    cd = (1 + sig * dt / (2 * EPS0 * eps))
    out['ce_e'] = ((1 - sig * dt / (2 * EPS0 * eps)) / cd).astype(F32)
    out['ce_h'] = (dt / (EPS0 * eps * dx) / cd).astype(F32)
    if tm:
        out.update(_tm_coefficients(sp, eps, sig, ys, in_wg, bead_patch))
    # source: Gaussian line source on the Ez nodes (TM: averaged onto Ey), in air
    # in front of the entry facet (fdtd2d_core.py:378-397)
    yc_src = st.t_wg_um * 1e-6 / 2 + sp.vcsel_offset_um * 1e-6
    y_abs = (-sp.tear_m + np.arange(Ny) * dx) * 1e6
    y_um = y_abs - yc_src * 1e6
    w, R = beam(float(sp.vcsel_distance_um or 0.0) - air, sp.waist_um, sp.lam_nm, 1.0)
    amp = math.sqrt(sp.waist_um / w) * np.exp(-(y_um / w) ** 2)
    if sp.src_core_only:
        from .physics import core_source_mask
        amp = amp * core_source_mask(y_abs, st.t_wg_um)
    kdx = huygens_kdx(sp.lam_nm, dx, C0 * dt, 1.0, sp.vcsel_tilt_deg)
    a, p1, p2 = huygens_arrays(amp, _beam_phase(y_um, R, sp.lam_nm, 1.0, sp.vcsel_tilt_deg), kdx)
    if tm:
        h = F32(0.5)
        a, p1, p2 = h * (a[:-1] + a[1:]), h * (p1[:-1] + p1[1:]), h * (p2[:-1] + p2[1:])
    out['src'] = dict(ix=sp.src_ix, amp=a, ph1=p1, ph2=p2, omega=2 * np.pi * sp.f0, air_um=air,
                      iy_src=int(round((yc_src + sp.tear_m) / dx)))
    nlo, nhi = sp.npml_x if sp.npml_x is not None else (sp.npml, sp.npml)
    out['cx'] = cpml_axis(Nx, nlo, nhi, dx, dt, lam_m)
    out['cy'] = cpml_axis(Ny, sp.npml, sp.npml, dx, dt, lam_m)
    return out


def _tm_coefficients(sp, eps, sig, ys, in_wg, bp):
    """Ca_ex / Ca_ey with harmonic layer averages for Ey, the Farjadpour tensor at
    the bead edge and the loss split (fdtd2d_core.py:283-349, 445-455)."""
    dx, dt = sp.dx, sp.dt
    st = sp.stack
    e_ex = 0.5 * (eps[:-1, :] + eps[1:, :])
    e_ey = 0.5 * (eps[:, :-1] + eps[:, 1:])
    ca_x = (dt / (EPS0 * e_ex * dx)).astype(F32)
    c = dt / (EPS0 * dx)
    h_out = column_average(ys[:-1], dx, lambda y: st.eps_of_y(1.0, core=False)(y).real,
                           harmonic=True, shift=0.5 * dx)
    h_core = column_average(ys[:-1], dx, lambda y: st.eps_of_y(1.0, core=True)(y).real,
                            harmonic=True, shift=0.5 * dx)
    h = np.where(in_wg[:, None], h_core[None, :], h_out[None, :])
    ca_y = (c / h).astype(F32)
    if bp is not None:
        bg, i0, j0, xc, yc, r = bp['bg'], bp['i0'], bp['j0'], bp['xc'], bp['yc'], bp['r']
        eb = bp['n'] ** 2

        def tensor(xp, yp, ea, eh, normal_x):
            f = circle_fraction(xp, yp, xc, yc, r, dx)
            X = xp[:, None] - xc
            Y = yp[None, :] - yc
            d = np.maximum(np.sqrt(X * X + Y * Y), 1e-30)
            nc2 = (X / d) ** 2 if normal_x else (Y / d) ** 2
            return f, nc2 * ((1 - f) / eh + f / eb) + (1 - nc2) / ((1 - f) * ea + f * eb)

        for comp in ('x', 'y'):
            if comp == 'x':
                f, inv = tensor(bp['xs'][:-1] + 0.5 * dx, bp['ys'], 0.5 * (bg[:-1] + bg[1:]),
                                1.0 / (0.5 * (1.0 / bg[:-1] + 1.0 / bg[1:])), True)
                tgt = ca_x
            else:
                eh = 1.0 / (0.5 * (1.0 / bg[:, :-1] + 1.0 / bg[:, 1:]))
                hb = h[i0:i0 + eh.shape[0], j0:j0 + eh.shape[1]]
                eh[:hb.shape[0], :hb.shape[1]] = hb
                f, inv = tensor(bp['xs'], bp['ys'][:-1] + 0.5 * dx, 0.5 * (bg[:, :-1] + bg[:, 1:]), eh, False)
                tgt = ca_y
            sl = (slice(i0, i0 + inv.shape[0]), slice(j0, j0 + inv.shape[1]))
            blk = tgt[sl].astype(np.float64)
            sel = f > 0
            blk[sel] = c * inv[sel]
            tgt[sl] = blk.astype(F32)
    out = dict(ca_x=ca_x, ca_y=ca_y)
    if bool(np.any(sig > 0)):
        a_ex = 0.5 * (sig[:-1, :] + sig[1:, :]) * dt / (2 * EPS0 * e_ex)
        a_ey = 0.5 * (sig[:, :-1] + sig[:, 1:]) * dt / (2 * EPS0 * e_ey)
        ca_x /= (1 + a_ex).astype(F32)
        ca_y /= (1 + a_ey).astype(F32)
        out.update(da_x=((1 - a_ex) / (1 + a_ex)).astype(F32), da_y=((1 - a_ey) / (1 + a_ey)).astype(F32))
    return out


# =========================================================================== 3D
@dataclass
class Sphere:
    x_um: float
    d_um: float
    n: complex = 1.59                  # complex: absorbing bead (lossy stacks)
    y_um: Optional[float] = None       # default -r: resting on the core bottom
    z_um: float = 0.0


@dataclass
class Spec3D:
    """A 3D full-domain slab solve (fdtd3d_core.run_3d, CPML on all faces)."""
    pol: str
    nx: int
    ny: int
    nz: int
    dx_nm: float
    stack: Stack
    tear_um: float                     # depth below the core bottom (y at j=0 is -tear_um)
    beads: List[Sphere] = field(default_factory=list)
    npml: int = 10
    lam_nm: float = 850.0
    waist_um: float = 3.0
    ramp_periods: Optional[float] = None
    # run_3d options (fdtd3d_core.py:793-807)
    waist_z_um: Optional[float] = None   # default: waist_um
    offset_y_um: float = 0.0             # source centre offsets from (t_wg/2, 0)
    offset_z_um: float = 0.0
    tilt_deg: float = 0.0                # beam tilt in the x-y plane
    vcsel_distance_um: float = 0.0       # beam waist in front of the entry facet
    n_sponge: Optional[int] = None       # absorber/source offset cells (default from sponge_um)
    sponge_um: float = 1.2
    end_facet_um: float = 0.0            # air over the last end_facet_um of the length
    wg_width_um: Optional[float] = None  # rectangular channel: core only for |z| < width/2
    n_clad_side: float = 1.0             # index beside the channel core
    pec_faces: Tuple[str, ...] = ()      # faces without CPML (PEC mirrors)
    # stitch window (fdtd3d_core.py:119-145, global-x mode): x of node 0 in the
    # whole domain; the core then exists only for x in [entry facet, x_wg_end_um]
    # and the columns outside it keep the layers below an empty core row
    x0_um: Optional[float] = None
    x_wg_end_um: Optional[float] = None
    n_sp_cells: Optional[int] = None     # absorber cells fixed by the caller (window shape)

    @property
    def dx(self):
        return self.dx_nm * 1e-9

    @property
    def dt(self):
        return 0.5 * self.dx / (C0 * np.sqrt(3))

    @property
    def n_sp(self):
        """Sponge thickness in cells (fdtd3d_core.py:381-396), which fixes the source plane."""
        if self.n_sp_cells is not None:
            return int(self.n_sp_cells)
        dx_um = self.dx_nm / 1000.0
        n = int(self.n_sponge) if self.n_sponge else int(np.ceil(float(self.sponge_um) / dx_um))
        n = max(8, n)
        return min(n, max(8, min(self.nx, self.ny, self.nz) // 6))

    @property
    def src_ix(self):
        return self.n_sp + 6

    @property
    def src_comp(self):
        return 1 if self.pol == 'p' else 2

    @property
    def f0(self):
        return C0 / (self.lam_nm * 1e-9)


HOST_THREADS = max(1, min(16, len(os.sched_getaffinity(0))))


def _slabs(n, fn, min_rows=16):
    """fn(i0, i1) over contiguous slabs of [0, n) on up to HOST_THREADS threads
    (the volume builders are NumPy element-wise work, which runs without the GIL)."""
    k = min(HOST_THREADS, n // min_rows)
    if k <= 1:
        fn(0, n)
        return
    b = [n * q // k for q in range(k + 1)]
    with ThreadPoolExecutor(k) as ex:
        for f in [ex.submit(fn, b[q], b[q + 1]) for q in range(k)]:
            f.result()


def _stagger(a, ax):
    """Mean of neighbouring nodes along ax, 0.5 * (a[i] + a[i+1]) in a's precision,
    returned as float32."""
    shp = list(a.shape)
    shp[ax] -= 1
    out = np.empty(shp, dtype=a.dtype)
    half = a.dtype.type(0.5)

    def part(i0, i1):
        if ax == 0:
            lo, hi = a[i0:i1], a[i0 + 1:i1 + 1]
        else:
            s_lo, s_hi = [slice(i0, i1), slice(None), slice(None)], [slice(i0, i1), slice(None), slice(None)]
            s_lo[ax], s_hi[ax] = slice(None, -1), slice(1, None)
            lo, hi = a[tuple(s_lo)], a[tuple(s_hi)]
        o = out[i0:i1]
        np.add(lo, hi, out=o)
        o *= half
    _slabs(shp[0], part)
    return out.astype(F32, copy=False)


def _columns_volume(T, tab):
    """(Nx, Ny, Nz) float32 volume whose (i, :, k) column is tab[T[i, k]]
    (tab: (ntype, Ny) float32, one row per column type)."""
    Nx, Nz = T.shape
    out = np.empty((Nx, tab.shape[1], Nz), F32)

    def part(i0, i1):
        out[i0:i1] = tab[T[i0:i1]].transpose(0, 2, 1)
    _slabs(Nx, part)
    return out


def build_3d(sp: Spec3D):
    """Staggered coefficients (ce_x, ce_y, ce_z), damping (or None), CPML profiles
    and source of a 3D slab solve, in the reference shapes."""
    Nx, Ny, Nz = sp.nx, sp.ny, sp.nz
    dx, dt = sp.dx, sp.dt
    dx_um = sp.dx_nm / 1000.0
    lam_m = sp.lam_nm * 1e-9
    st = sp.stack
    lossy = st.lossy
    y0_um, z0_um = -sp.tear_um, -Nz * dx_um / 2.0
    ys = y0_um + np.arange(Ny) * dx_um
    zs = z0_um + np.arange(Nz) * dx_um
    glob = sp.x0_um is not None
    x0 = float(sp.x0_um) if glob else 0.0
    xs = x0 + np.arange(Nx) * dx_um
    air = air_path_um(sp.vcsel_distance_um, dx_um)
    x_facet_um = sp.src_ix * dx_um + air
    # column types (fdtd3d_core.py:248-261): 0 layers without the core, 1 core
    # stack, 2 channel cladding beside the core, 3 air (in front of the entry
    # facet, over the end facet)
    channel = sp.wg_width_um is not None and 0 < sp.wg_width_um < Nz * dx_um
    if glob:     # stitch window: finite core [facet, x_wg_end], no air columns
        in_wg = xs >= x_facet_um
        if sp.x_wg_end_um is not None:
            in_wg &= xs <= sp.x_wg_end_um
        T = np.zeros((Nx, Nz), dtype=np.int8)
        T[in_wg, :] = 1
        if channel:
            T[np.ix_(in_wg, np.abs(zs) > sp.wg_width_um / 2.0)] = 2
    else:
        T = np.full((Nx, Nz), 1, dtype=np.int8)
        if channel:
            T[:, np.abs(zs) > sp.wg_width_um / 2.0] = 2
        if sp.end_facet_um and sp.end_facet_um > 0:
            T[xs >= (Nx * dx_um - sp.end_facet_um), :] = 3
        T[xs < x_facet_um, :] = 3
    col = column_average(ys, dx_um, st.eps_of_y(1e-6, core=True))
    cols_node = {1: col, 3: np.full(Ny, N_AIR ** 2, dtype=col.dtype)}
    if glob:
        cols_node[0] = column_average(ys, dx_um, st.eps_of_y(1e-6, core=False))
    if channel:   # core rows (0 <= y <= t_wg) set to the cladding index at the nodes
        c2 = col.copy()
        c2[(ys >= 0.0) & (ys <= st.t_wg_um)] = sp.n_clad_side ** 2
        cols_node[2] = c2
    # harmonic Ey columns for the four column types (fdtd3d_core.py:239-261)
    hcol = lambda core, nc=None: column_average(ys[:-1], dx_um, lambda y: np.real(st.eps_of_y(1e-6, core, nc)(y)),
                                                harmonic=True, shift=0.5 * dx_um).astype(np.float64)
    hcols = np.stack([hcol(False), hcol(True), hcol(True, sp.n_clad_side), np.full(Ny - 1, N_AIR ** 2)])
    c0f, c1f = F32(dt / (EPS0 * dx)), F32(np.pi * C0 / lam_m * dt)

    def inv_damp(e_complex_or_real):
        e = np.asarray(e_complex_or_real)
        er = e.real.astype(F32) if np.iscomplexobj(e) else e.astype(F32)
        inv = c0f / er
        if not lossy:
            return inv, None
        a = (c1f * np.asarray(e.imag, F32)) / er
        inv /= (1 + a)
        return inv, ((1 - a) / (1 + a)).astype(F32)

    # volumes from the per-type columns (every column type of T has a column)
    inv_t = {t: inv_damp(c) for t, c in cols_node.items()}
    assert set(np.unique(T).tolist()) <= set(inv_t), (np.unique(T), sorted(inv_t))
    nty = max(inv_t) + 1
    tab_inv = np.zeros((nty, Ny), F32)
    tab_d = np.zeros((nty, Ny), F32)
    for t, (iv, dv) in inv_t.items():
        tab_inv[t] = iv
        if lossy:
            tab_d[t] = dv
    inv = _columns_volume(T, tab_inv)
    D = _columns_volume(T, tab_d) if lossy else None
    # beads: blended eps in their boxes, background kept for the tensor
    patches = []
    for bd in sp.beads:
        r = bd.d_um / 2.0
        xc, yc, zc = bd.x_um, (bd.y_um if bd.y_um is not None else -r), bd.z_um
        i0, i1 = max(0, int((xc - r - x0) / dx_um) - 2), min(Nx, int((xc + r - x0) / dx_um) + 3)
        j0, j1 = max(0, int((yc - r - y0_um) / dx_um) - 2), min(Ny, int((yc + r - y0_um) / dx_um) + 3)
        k0, k1 = max(0, int((zc - r - z0_um) / dx_um) - 2), min(Nz, int((zc + r - z0_um) / dx_um) + 3)
        if not (i1 > i0 and j1 > j0 and k1 > k0):
            continue
        tb = T[i0:i1, k0:k1]
        box = np.empty((i1 - i0, j1 - j0, k1 - k0), dtype=col.dtype)
        for t, cv in cols_node.items():
            box[np.broadcast_to((tb == t)[:, None, :], box.shape)] = np.broadcast_to(
                cv[None, j0:j1, None], box.shape)[np.broadcast_to((tb == t)[:, None, :], box.shape)]
        patches.append(dict(bg=box.real.astype(np.float64), i0=i0, j0=j0, k0=k0, xs=xs[i0:i1],
                            ys=ys[j0:j1], zs=zs[k0:k1], xc=xc, yc=yc, zc=zc, r=r, n=complex(bd.n).real))
        _blend(box, sphere_fraction(xs[i0:i1], ys[j0:j1], zs[k0:k1], xc, yc, zc, r, dx_um),
               complex(bd.n) if lossy else complex(bd.n).real)
        iv, dv = inv_damp(box)
        inv[i0:i1, j0:j1, k0:k1] = iv
        if lossy:
            D[i0:i1, j0:j1, k0:k1] = dv
    ce = [_stagger(inv, 0), None, _stagger(inv, 2)]
    hinv = (dt / (EPS0 * dx) / hcols).astype(F32)
    cy = _columns_volume(T, hinv)                                 # every column type overrides ce_y
    # the loss factor (1 + D) / 2 at the staggered positions of each axis, made once
    half_d = [None, None, None]
    if lossy:
        hD = np.empty_like(D)

        def half_part(i0, i1):
            h = hD[i0:i1]
            np.add(D[i0:i1], F32(1), out=h)
            h *= F32(0.5)
        _slabs(Nx, half_part)
        half_d = [_stagger(hD, ax) for ax in range(3)]
        del hD
        cy *= half_d[1]
    ce[1] = cy
    c = dt / (EPS0 * dx)
    for bp in patches:                                            # Farjadpour tensor at the bead edge
        eb = bp['n'] ** 2
        for ax in range(3):
            e0 = bp['bg']
            nb = e0.shape[ax]
            e_nx = np.take(e0, np.minimum(np.arange(nb) + 1, nb - 1), axis=ax)
            e_a = 0.5 * (e0 + e_nx)
            e_h = 1.0 / (0.5 * (1.0 / e0 + 1.0 / e_nx))
            if ax == 1:
                Tb = T[bp['i0']:bp['i0'] + e0.shape[0], bp['k0']:bp['k0'] + e0.shape[2]]
                hb = np.transpose(hcols[:, bp['j0']:bp['j0'] + e0.shape[1]][Tb], (0, 2, 1))
                e_h[:, :hb.shape[1], :] = hb
            o = [0.0, 0.0, 0.0]
            o[ax] = 0.5 * dx_um
            px, py, pz = bp['xs'] + o[0], bp['ys'] + o[1], bp['zs'] + o[2]
            a0, b0, c0 = bp['i0'], bp['j0'], bp['k0']
            tgt = ce[ax]
            na, nb_, nc = min(len(px), tgt.shape[0] - a0), min(len(py), tgt.shape[1] - b0), min(len(pz), tgt.shape[2] - c0)
            if na <= 0 or nb_ <= 0 or nc <= 0:
                continue
            px, py, pz = px[:na], py[:nb_], pz[:nc]
            f = sphere_fraction(px, py, pz, bp['xc'], bp['yc'], bp['zc'], bp['r'], dx_um)
            sel = f > 0
            if not sel.any():
                continue
            X = px[:, None, None] - bp['xc']
            Y = py[None, :, None] - bp['yc']
            Z = pz[None, None, :] - bp['zc']
            d = np.maximum(np.sqrt(X * X + Y * Y + Z * Z), 1e-30)
            nc2 = ((X, Y, Z)[ax] / d) ** 2
            inv_t3 = nc2 * ((1 - f) / e_h[:na, :nb_, :nc] + f / eb) + (1 - nc2) / ((1 - f) * e_a[:na, :nb_, :nc] + f * eb)
            sl = (slice(a0, a0 + na), slice(b0, b0 + nb_), slice(c0, c0 + nc))
            blk = tgt[sl].astype(np.float64)
            val = c * np.broadcast_to(inv_t3, f.shape)
            if lossy:
                val = val * half_d[ax][sl].astype(np.float64)
            blk[sel] = val[sel]
            tgt[sl] = blk.astype(F32)
    da = None if not lossy else tuple(_stagger(D, ax) for ax in range(3))
    # source on the driven component (fdtd3d_core.py:494-530, vcsel.py:110-123): a
    # Gaussian spot in air (n = 1) in front of the facet, waist vcsel_distance_um
    # before the facet, centred at (t_wg/2 + offset_y, offset_z), tilted in x-y
    pol = sp.pol
    Nj, Nk = (Ny - 1, Nz) if pol == 'p' else (Ny, Nz - 1)
    wy0 = sp.waist_um
    wz0 = sp.waist_um if sp.waist_z_um is None else sp.waist_z_um
    yc = st.t_wg_um / 2 + sp.offset_y_um
    zc = sp.offset_z_um
    yv = y0_um + (np.arange(Nj) + (0.5 if pol == 'p' else 0.0)) * dx_um - yc
    zv = z0_um + (np.arange(Nk) + (0.5 if pol == 's' else 0.0)) * dx_um - zc
    zprop = float(sp.vcsel_distance_um or 0.0) - air
    wy, Ry = beam(zprop, wy0, sp.lam_nm, 1.0)
    wz, Rz = beam(zprop, wz0, sp.lam_nm, 1.0)
    amp = math.sqrt((wy0 / wy) * (wz0 / wz)) * np.exp(-(yv[:, None] / wy) ** 2 - (zv[None, :] / wz) ** 2)
    ph = _beam_phase(yv[:, None], Ry, sp.lam_nm, 1.0, sp.tilt_deg) + np.zeros((1, Nk))
    if math.isfinite(Rz):
        ph = ph - (2 * math.pi / (sp.lam_nm * 1e-3)) * zv[None, :] ** 2 / (2.0 * Rz)
    kdx = huygens_kdx(sp.lam_nm, dx, C0 * dt, 1.0, sp.tilt_deg)
    a, p1, p2 = huygens_arrays(amp, ph, kdx)
    src = dict(ix=sp.src_ix, amp=a, ph1=p1, ph2=p2, omega=2 * np.pi * C0 / lam_m, air_um=air,
               j_src=min(max(int(round((yc - y0_um) / dx_um)), 0), Nj - 1),
               k_src=min(max(int(round((zc - z0_um) / dx_um)), 0), Nk - 1))
    # CPML on the absorbing faces, none on the PEC mirrors (boundaries3d.py:262-302)
    pf = set(sp.pec_faces or ())
    cpml = [cpml_axis(N, 0 if lo in pf else sp.npml, 0 if hi in pf else sp.npml, dx, dt, lam_m)
            for N, lo, hi in ((Nx, 'xmin', 'xmax'), (Ny, 'ymin', 'ymax'), (Nz, 'zmin', 'zmax'))]
    return dict(ce=tuple(ce), da=da, src=src, cpml=cpml, x_facet_um=x_facet_um, T=T)
