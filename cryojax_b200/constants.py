"""Physical constants of the image path (float64, host side).

cryojax/constants/_physical_constants.py:10-109.
"""

from __future__ import annotations

import numpy as np

try:  # the reference takes c, m0, e from scipy.constants
    import scipy.constants as _sc

    SPEED_OF_LIGHT, ELECTRON_MASS, ELEMENTARY_CHARGE = _sc.speed_of_light, _sc.electron_mass, _sc.elementary_charge
except Exception:  # pragma: no cover
    SPEED_OF_LIGHT, ELECTRON_MASS, ELEMENTARY_CHARGE = 299792458.0, 9.1093837139e-31, 1.602176634e-19


def wavelength_from_kilovolts(voltage_in_kilovolts):
    """Relativistic electron wavelength in Angstroms (:10-29)."""
    v = 1000.0 * np.asarray(voltage_in_kilovolts, np.float64)
    return 12.2639 / (v + 0.97845e-6 * v**2) ** 0.5


def lorentz_factor_from_kilovolts(voltage_in_kilovolts):
    """(:32-49)"""
    rest_energy = ELECTRON_MASS * SPEED_OF_LIGHT**2
    return 1.0 + ELEMENTARY_CHARGE * (1000.0 * np.asarray(voltage_in_kilovolts, np.float64)) / rest_energy


def interaction_constant_from_kilovolts(voltage_in_kilovolts):
    """lambda * gamma (:52-109)."""
    return wavelength_from_kilovolts(voltage_in_kilovolts) * lorentz_factor_from_kilovolts(voltage_in_kilovolts)


def b_factor_to_variance(b_factor):
    """variance = B / (8 pi^2).  cryojax/constants/_conventions.py:6-27."""
    return np.asarray(b_factor, np.float64) / (8.0 * np.pi**2)


def variance_to_b_factor(variance):
    """B = 8 pi^2 variance.  cryojax/constants/_conventions.py:30-50."""
    return 8.0 * np.pi**2 * np.asarray(variance, np.float64)
