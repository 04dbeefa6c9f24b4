"""Isentropic relations of full-potential flow (pyfp3d/physics/isentropic.py).

Scalar relations are plain host arithmetic with the reference's formulas;
the *_field functions -- the per-element sweeps of the Picard/Newton loops --
run on the B200 through the up3d library.  Arrays in, same kind out.
"""

from __future__ import annotations

import math

import numpy as np

from .. import _lib as L

GAMMA = 1.4
R_GAS = 287.05
M_CRIT_DEFAULT = 0.95
UPWIND_CONST_DEFAULT = 1.5


# ------------------------------------------------------------- scalars (host)

def density_isentropic(q_squared, M_inf, gamma=GAMMA):
    """rho(q^2) with the vacuum guard (physics/isentropic.py:30-58)."""
    exponent = 1.0 / (gamma - 1.0)
    base = 1.0 + 0.5 * (gamma - 1.0) * M_inf ** 2 * (1.0 - q_squared)
    if base < 1e-10:
        base = 1e-10
    return base ** exponent


def speed_of_sound_squared(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:61-76"""
    return 1.0 / (M_inf ** 2) + 0.5 * (gamma - 1.0) * (1.0 - q_squared)


def mach_number_squared(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:80-97"""
    return q_squared * M_inf ** 2 / (1.0 + 0.5 * (gamma - 1.0) * M_inf ** 2 * (1.0 - q_squared))


def critical_speed_squared(M_inf, gamma=GAMMA):
    """physics/isentropic.py:100-118"""
    return (2.0 + (gamma - 1.0) * M_inf ** 2) / ((gamma + 1.0) * M_inf ** 2)


def pressure_coefficient(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:122-143"""
    rho = density_isentropic(q_squared, M_inf, gamma)
    return 2.0 / (gamma * M_inf ** 2) * (rho ** gamma - 1.0)


def pressure_coefficient_incompressible(q_squared):
    """physics/isentropic.py:146-160"""
    return 1.0 - q_squared


def density_derivative_wrt_q_sq(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:164-180"""
    rho = density_isentropic(q_squared, M_inf, gamma)
    return -0.5 * M_inf ** 2 * (rho ** (2.0 - gamma))


def mach_squared_derivative_wrt_q_sq(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:184-206"""
    D = 1.0 + 0.5 * (gamma - 1.0) * M_inf ** 2 * (1.0 - q_squared)
    return M_inf ** 2 * (1.0 + 0.5 * (gamma - 1.0) * M_inf ** 2) / (D * D)


def upwind_factor(q_squared, M_inf, M_crit=M_CRIT_DEFAULT, C=UPWIND_CONST_DEFAULT, gamma=GAMMA):
    """physics/isentropic.py:210-232"""
    M_sq = mach_number_squared(q_squared, M_inf, gamma)
    return C * max(0.0, 1.0 - (M_crit ** 2) / max(M_sq, M_crit ** 2))


def q2_at_mach(mach, M_inf, gamma=GAMMA):
    """physics/isentropic.py:262-289 (+inf at M_inf == 0)."""
    if M_inf == 0.0:
        return math.inf
    m2 = mach * mach
    return m2 * (1.0 + 0.5 * (gamma - 1.0) * M_inf ** 2) / (M_inf ** 2 * (1.0 + 0.5 * (gamma - 1.0) * m2))


# ------------------------------------------------------------- fields (device)

def _field(entry, q_squared, M_inf, gamma):
    t = L.torch()
    d = L.to_device(q_squared, t.float64)
    out = t.empty_like(d)
    L.call(entry, d.data_ptr(), d.numel(), float(M_inf), float(gamma), out.data_ptr(), L.stream_ptr())
    if L.is_torch(q_squared):
        return out
    return out.cpu().numpy().reshape(np.shape(q_squared))


def density_field(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:236-258"""
    return _field("up3d_density", q_squared, M_inf, gamma)


def mach_squared_field(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:318-334"""
    return _field("up3d_mach_squared", q_squared, M_inf, gamma)


def density_derivative_wrt_q_sq_field(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:338-354"""
    return _field("up3d_density_derivative", q_squared, M_inf, gamma)


def mach_squared_derivative_wrt_q_sq_field(q_squared, M_inf, gamma=GAMMA):
    """physics/isentropic.py:358-374"""
    return _field("up3d_mach_squared_derivative", q_squared, M_inf, gamma)


def pressure_coefficient_field(q_squared, M_inf, gamma=GAMMA):
    """Elementwise pressure_coefficient (physics/isentropic.py:122-143)."""
    return _field("up3d_pressure_coefficient", q_squared, M_inf, gamma)


def limit_q2_field(q_squared, M_inf, m_cap, gamma=GAMMA):
    """physics/isentropic.py:293-314"""
    t = L.torch()
    d = L.to_device(q_squared, t.float64)
    out = t.empty_like(d)
    L.call("up3d_limit_q2", d.data_ptr(), d.numel(), float(M_inf), float(m_cap), float(gamma),
           out.data_ptr(), None, L.stream_ptr())
    if L.is_torch(q_squared):
        return out
    return out.cpu().numpy().reshape(np.shape(q_squared))


def validate_physics_bounds(rho, q, M, Cp, M_inf, gamma=GAMMA):
    """Host-side bound check (physics/isentropic.py:377-421)."""
    rho, q, M, Cp = (np.asarray(a.cpu() if L.is_torch(a) else a) for a in (rho, q, M, Cp))
    if np.any(rho <= 0):
        raise ValueError(f"Negative density detected: min={np.min(rho)}")
    if np.any(q < -1e-12):
        raise ValueError(f"Negative speed detected: min={np.min(q)}")
    if np.any(q > 2.0):
        raise ValueError(f"Excessive speed detected: max={np.max(q)} (should be ~1.0-1.4)")
    if np.any(M > 5.0):
        raise ValueError(f"Excessive Mach detected: max={np.max(M)}")
    if np.any(Cp < -5):
        raise ValueError(f"Excessive negative Cp: min={np.min(Cp)}")
    if np.any(Cp > 10):
        raise ValueError(f"Excessive positive Cp: max={np.max(Cp)}")
