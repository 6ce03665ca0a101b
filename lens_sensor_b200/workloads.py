"""The benchmark workloads, built from seeded parameters.

planar2d_te     2D TE planar waveguide 1600 x 480 @ 25 nm, 12-cell CPML, 6000 steps,
                CW ramped over 20 periods, one bead (n 1.59, r 0.4 um) at a seeded x.
waveguide3d_tm  3D TM (Ey) planar waveguide 480 x 192 x 256 @ 30 nm, 10-cell CPML,
                4000 steps, absorbing aqueous 1.333+0.001i, two seeded beads
                (r ~ U(0.3, 0.6) um), phasors of Ex/Ey/Ez.
sweep2d         256 uneven 2D TE/TM solves (tear-film thickness / bead sweep).
stitch3d_plan   3D stitch of a 240 um waveguide: windows of 480 x 192 x 256 @ 30 nm,
                40-cell overlap (19 windows by the reference's window formula).
serving_stream  serving stream: Poisson arrivals of mixed 2D / 3D / stitch requests.

Layer stack (core downward): PMMA core n=1.49 (2 um) / aqueous n=1.333
(1.5 um) / mucin n=1.34 (0.5 um) / cornea n=1.376 substrate; air above.  In 3D
the 192-row cross-section (5.76 um) keeps 1.0 um of cornea and 0.76 um of air.
All inputs are synthetic, generated from numpy default_rng seeds.
"""
import numpy as np

from .geometry import Bead2D, Spec2D, Spec3D, Sphere, Stack
from .stitch3d import StitchPlan

N_PMMA, N_AQ, N_MUCIN, N_CORNEA, N_PS, N_LIPID = 1.49, 1.333, 1.34, 1.376, 1.59, 1.48


def planar2d_te(seed=0):
    rng = np.random.default_rng(seed)
    st = Stack(N_PMMA, 2.0, [(1.5, N_AQ), (0.5, N_MUCIN)], N_CORNEA)
    x = float(rng.uniform(15.0, 30.0))
    return Spec2D('s', 1600, 480, 25e-9, st, 5.0e-6, Bead2D(x, 0.8, N_PS), npml=12,
                  ramp_periods=20.0), 6000


def waveguide3d_tm(seed=1):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 0.6, 2)
    beads = [Sphere(float(rng.uniform(4.5, 7.0)), float(2 * r[0]), N_PS, -float(r[0]), float(rng.uniform(-2, 2))),
             Sphere(float(rng.uniform(8.5, 11.5)), float(2 * r[1]), N_PS, -float(r[1]), float(rng.uniform(-2, 2)))]
    st = Stack(N_PMMA, 2.0, [(1.5, complex(N_AQ, 0.001)), (0.5, N_MUCIN)], N_CORNEA)
    return Spec3D('p', 480, 192, 256, 30.0, st, 3.0, beads, npml=10), 4000


def sweep2d(seed=2, count=256):
    """256 uneven 2D solves: aqueous U(0.5, 5) um, mucin U(0.2, 1), lipid
    U(0, 0.1) (n 1.48), bead r U(0.2, 0.8) um at a random x; widths U{600..2400},
    heights U{300..560} cells at 25 nm; TE and TM alternate; 4000 steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        aq, mu, lip = rng.uniform(0.5, 5.0), rng.uniform(0.2, 1.0), rng.uniform(0.0, 0.1)
        r = rng.uniform(0.2, 0.8)
        nx, ny = int(rng.integers(600, 2401)), int(rng.integers(300, 561))
        layers = ([(lip, N_LIPID)] if lip > 1e-3 else []) + [(aq, N_AQ), (mu, N_MUCIN)]
        st = Stack(N_PMMA, 2.0, layers, N_CORNEA)
        dx = 25e-9
        depth = ny * dx * 1e6 - 2.0 - 1.0            # 1 um of air above the core
        L = nx * dx * 1e6
        x = float(rng.uniform(0.3 * L, 0.8 * L))
        bead = Bead2D(x, float(2 * r), N_PS, -float(lip + r) if lip > 1e-3 else None)
        out.append(Spec2D('s' if q % 2 == 0 else 'p', nx, ny, dx, st, depth * 1e-6, bead, npml=12))
    return out, 4000


def _stack3d(rng, ly_um, air_um=0.5):
    """Core 1.0-1.5 um, absorbing aqueous U(0.5, 1.5) um, mucin 0.3 um, cornea below."""
    t_wg = float(rng.uniform(1.0, 1.5))
    aq = float(rng.uniform(0.5, 1.5))
    st = Stack(N_PMMA, t_wg, [(aq, complex(N_AQ, 0.001)), (0.3, N_MUCIN)], N_CORNEA)
    return st, ly_um - t_wg - air_um


def stitch3d_plan(seed=3, nx_full=8000, nx_win=480, overlap=40, ny=192, nz=256):
    """3D stitch of a 240 um planar waveguide at 30 nm (nx_full = 8000 cells) in
    windows of nx_win x ny x nz cells overlapping by `overlap` cells (slide
    nx_win - overlap), waveguide3d_tm stack (2 um core, absorbing aqueous), two seeded
    beads.  The reference's window count ceil((8000 - 480) / 440) + 1 = 19, the
    last window flush with the domain end (fdtd3d_core.py:1382-1386)."""
    rng = np.random.default_rng(seed)
    dx_nm = 30.0
    dx_um = dx_nm / 1000.0
    S = nx_win - overlap
    st = Stack(N_PMMA, 2.0, [(1.5, complex(N_AQ, 0.001)), (0.5, N_MUCIN)], N_CORNEA)
    lx = nx_full * dx_um
    r = rng.uniform(0.3, 0.6, 2)
    beads = [Sphere(float(rng.uniform(0.2, 0.4) * lx), float(2 * r[0]), N_PS, -float(r[0]), 0.0),
             Sphere(float(rng.uniform(0.6, 0.8) * lx), float(2 * r[1]), N_PS, -float(r[1]), 0.0)]
    return StitchPlan(st, 3.0, lx, ny * dx_um, nz * dx_um, dx_nm, nx_win * dx_um, S * dx_um, N_PMMA, pol='p',
                      beads=beads, waist_um=1.5, waist_z_um=1.5)


def serving_stream(seed=4, count=64, rate=50.0):
    """Serving stream: Poisson arrivals (mean `rate` req/s, seeded) of
    70 % 2D TE/TM solves of the sweep2d size distribution (4000 steps),
    25 % 3D solves of 256-512 x 128-192 x 160-256 cells at 30 nm with 2000-4000
    steps and 5 % 3D stitch jobs of 4-10 windows (windows of 256-384 x 128-160 x
    160-192 cells, 40-cell overlap).  Returns [(kind, spec, steps, arrival)]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    specs2d, steps2d = sweep2d(seed + 100, count)
    out = []
    for q in range(count):
        u = rng.uniform()
        if u < 0.70:
            out.append(('2d', specs2d[q], steps2d, float(t[q])))
            continue
        dx_nm = 30.0
        dx_um = dx_nm / 1000.0
        pol = 'p' if rng.uniform() < 0.5 else 's'
        if u < 0.95:
            nx, ny, nz = int(rng.integers(256, 513)), int(rng.integers(128, 193)), int(rng.integers(160, 257))
            st, tear = _stack3d(rng, ny * dx_um)
            r = float(rng.uniform(0.3, 0.6))
            bead = Sphere(float(rng.uniform(0.35, 0.65) * nx * dx_um), 2 * r, N_PS, -r,
                          float(rng.uniform(-1.0, 1.0)))
            sp = Spec3D(pol, nx, ny, nz, dx_nm, st, tear, [bead], npml=10, waist_um=1.0)
            out.append(('3d', sp, int(rng.integers(2000, 4001)), float(t[q])))
        else:
            nw = int(rng.integers(4, 11))
            nxw, ny, nz = int(rng.integers(256, 385)), int(rng.integers(128, 161)), int(rng.integers(160, 193))
            S = nxw - 40
            st, tear = _stack3d(rng, ny * dx_um)
            lx = (nxw + (nw - 1) * S) * dx_um
            r = float(rng.uniform(0.3, 0.6))
            bead = Sphere(float(rng.uniform(0.3, 0.7) * lx), 2 * r, N_PS, -r, 0.0)
            pl = StitchPlan(st, tear, lx, ny * dx_um, nz * dx_um, dx_nm, nxw * dx_um, S * dx_um, N_PMMA, pol=pol,
                            beads=[bead], waist_um=1.0, waist_z_um=1.0)
            out.append(('stitch', pl, pl.steps_win, float(t[q])))
    return out
