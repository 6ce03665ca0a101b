"""The benchmark workloads, built from seeded parameters.

config 0  2D TE planar waveguide 1600 x 480 @ 25 nm, 12-cell CPML, 6000 steps,
          CW ramped over 20 periods, one bead (n 1.59, r 0.4 um) at a seeded x.
config 1  3D TM (Ey) planar waveguide 480 x 192 x 256 @ 30 nm, 10-cell CPML,
          4000 steps, absorbing aqueous 1.333+0.001i, two seeded beads
          (r ~ U(0.3, 0.6) um), phasors of Ex/Ey/Ez.
config 2  256 uneven 2D TE/TM solves (tear-film thickness / bead sweep).

Layer stack (core downward): PMMA core n=1.49 (2 um) / aqueous n=1.333
(1.5 um) / mucin n=1.34 (0.5 um) / cornea n=1.376 substrate; air above.  In 3D
the 192-row cross-section (5.76 um) keeps 1.0 um of cornea and 0.76 um of air.
All inputs are synthetic, generated from numpy default_rng seeds.
"""
import numpy as np

from .geometry import Bead2D, Spec2D, Spec3D, Sphere, Stack

N_PMMA, N_AQ, N_MUCIN, N_CORNEA, N_PS, N_LIPID = 1.49, 1.333, 1.34, 1.376, 1.59, 1.48


def config0(seed=0):
    rng = np.random.default_rng(seed)
    st = Stack(N_PMMA, 2.0, [(1.5, N_AQ), (0.5, N_MUCIN)], N_CORNEA)
    x = float(rng.uniform(15.0, 30.0))
    return Spec2D('s', 1600, 480, 25e-9, st, 5.0e-6, Bead2D(x, 0.8, N_PS), npml=12,
                  ramp_periods=20.0), 6000


def config1(seed=1):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 0.6, 2)
    beads = [Sphere(float(rng.uniform(4.5, 7.0)), float(2 * r[0]), N_PS, -float(r[0]), float(rng.uniform(-2, 2))),
             Sphere(float(rng.uniform(8.5, 11.5)), float(2 * r[1]), N_PS, -float(r[1]), float(rng.uniform(-2, 2)))]
    st = Stack(N_PMMA, 2.0, [(1.5, complex(N_AQ, 0.001)), (0.5, N_MUCIN)], N_CORNEA)
    return Spec3D('p', 480, 192, 256, 30.0, st, 3.0, beads, npml=10), 4000


def config2(seed=2, count=256):
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
