"""Physical constants and material helpers used by the host setup.

Values match common/physics.py:10-13 of the reference (CODATA constants used
there), so grids, time steps and coefficients agree to the last bit.
"""
import numpy as np

C0 = 2.99792458e8            # m/s
EPS0 = 8.8541878128e-12      # F/m
MU0 = 4.0 * np.pi * 1e-7     # H/m
N_AIR = 1.0


def loss_sigma(eps_imag, lam_m):
    """Conductivity for Im(eps_r) at the operating wavelength: sigma = w0 eps0 eps''
    (common/physics.py:213-215)."""
    return 2 * np.pi * C0 / lam_m * EPS0 * np.asarray(eps_imag)


def dt_2d(dx):
    """Courant 0.5 in 2D (fdtd2d_core.py:626)."""
    return 0.5 * dx / (C0 * np.sqrt(2))


def dt_3d(dx):
    """Courant 0.5 in 3D (fdtd3d_core.py:838)."""
    return 0.5 * dx / (C0 * np.sqrt(3))
