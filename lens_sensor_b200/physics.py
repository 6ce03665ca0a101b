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


# ---------------------------------------------------------------------------
# Material dispersion (common/physics.py:15-120): n(lambda) from published fits.
#   PMMA, polystyrene: one-term Sellmeier (Sultanova et al. 2009)
#   water: four-term Sellmeier (Daimon & Masumura 2007)
#   tear film = water + 0.0035; mucin = tear + 0.0018; cornea, lipid, cornea
#   layers: visible-band value shifted with the water / PMMA dispersion.
# ---------------------------------------------------------------------------
LAM_VIS_UM = 0.5893
_SELL = {
    'pmma': ((1.1819, 0.011313),),
    'polystyrol': ((1.4435, 0.020216),),
    'water': ((5.684027565e-1, 5.101829712e-3), (1.726177391e-1, 1.821153936e-2),
              (2.086189578e-2, 2.620722293e-2), (1.130748688e-1, 1.069792721e1)),
}


def _sellmeier(lam_um, terms):
    l2 = lam_um * lam_um
    return float(np.sqrt(1.0 + sum(B * l2 / (l2 - C) for B, C in terms)))


def _water(l):
    return _sellmeier(l, _SELL['water'])


def _pmma(l):
    return _sellmeier(l, _SELL['pmma'])


def _shift(n_vis, base):
    return lambda l: n_vis + base(l) - base(LAM_VIS_UM)


MATERIALS = {
    'pmma': _pmma,
    'polystyrol': lambda l: _sellmeier(l, _SELL['polystyrol']),
    'water': _water,
    'aqueous': lambda l: _water(l) + 0.0035,
    'cornea': _shift(1.376, _water),
    'mucin': lambda l: _water(l) + 0.0035 + 0.0018,
    'lipid': _shift(1.480, _pmma),
    'epithelium': _shift(1.401, _water),
    'stroma': _shift(1.3765, _water),
    'aqueous_humor': _shift(1.336, _water),
}


def n_at(mat, lam_nm):
    """Refractive index of `mat` at `lam_nm` (common/physics.py:97-106)."""
    return float(MATERIALS[mat](float(lam_nm) / 1000.0))


_CORNEA_UM = dict(epithelium=50.0, bowman=12.0, stroma_end=525.0, endothelium_end=545.0)


class CorneaProfile(float):
    """Layered cornea below the tear film (common/physics.py:124-174): epithelium
    1.401 (0-50 um), Bowman 1.380 (to 62 um), stroma 1.380 -> 1.373 (to 525 um),
    Descemet/endothelium 1.373 (to 545 um), aqueous humour 1.336 below; all shifted
    with the water dispersion.  The float value is the epithelium index."""

    def __new__(cls, lam_nm):
        obj = float.__new__(cls, n_at('epithelium', lam_nm))
        obj.lam_nm = float(lam_nm)
        return obj

    def __reduce__(self):
        return (CorneaProfile, (self.lam_nm,))

    def at_depth(self, d_um):
        d = np.asarray(d_um, dtype=np.float64)
        L = _CORNEA_UM
        b0 = L['epithelium']
        b1 = b0 + L['bowman']
        n = np.full(d.shape, 1.336)
        n = np.where(d < L['endothelium_end'], 1.373, n)
        st = (d >= b1) & (d < L['stroma_end'])
        frac = np.clip((d - b1) / (L['stroma_end'] - b1), 0.0, 1.0)
        n = np.where(st, 1.380 + (1.373 - 1.380) * frac, n)
        n = np.where((d >= b0) & (d < b1), 1.380, n)
        n = np.where(d < b0, 1.401, n)
        lam_um = self.lam_nm / 1000.0
        return n + _water(lam_um) - _water(LAM_VIS_UM)


def cornea_default(lam_nm):
    return CorneaProfile(lam_nm)


def core_source_mask(y_um, t_wg_um, ramp_um=0.2):
    """Source weight when the beam may enter through the core only
    (common/physics.py:227-244): 1 in the core, cos^2 ramp outside."""
    d = np.maximum(-np.asarray(y_um, dtype=np.float64), np.asarray(y_um, dtype=np.float64) - float(t_wg_um))
    return np.where(d <= 0.0, 1.0, np.where(d < ramp_um, np.cos(0.5 * np.pi * d / max(ramp_um, 1e-9)) ** 2, 0.0))
