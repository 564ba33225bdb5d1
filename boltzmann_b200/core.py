"""The user-facing module, equivalent to ``boltzmann.core`` of djbarker/boltzmann
(python/boltzmann/core.py): the extension's classes plus the collision and parameter helpers.

    from boltzmann_b200.core import Simulation, bgk, trt, CellFlags
"""

from __future__ import annotations

import math
from typing import Literal

import boltzmann_b200.boltzmann as _ext
from boltzmann_b200.boltzmann import Cells, Fluid, Omega, PanicException, Scalar, Simulation

__all__ = [
    "bgk",
    "trt",
    "Device",
    "CellFlags",
    "calc_lbm_params_lu",
    "calc_lbm_params_si",
    "check_lbm_params",
    "Simulation",
    "Fluid",
    "Scalar",
    "Cells",
    "Omega",
    "PanicException",
]

Device = Literal["cpu", "gpu"]  #: accepted device strings; both run on the CUDA device

extension = _ext


def bgk(tau: float) -> Omega:
    """BGK collision with relaxation time ``tau`` (lattice units): omega = 1 / tau
    (python/boltzmann/core.py:40-47)."""
    return Omega.BGK(1.0 / tau)


def trt(tau_pos: float, tau_neg: float | None = None, magic_no: float = 0.25) -> Omega:
    """Two-relaxation-time collision (python/boltzmann/core.py:50-62).

    Without ``tau_neg`` the odd relaxation time follows from the magic parameter
    Lambda = (tau_pos - 1/2)(tau_neg - 1/2), default 1/4.
    """
    if not tau_neg:
        tau_neg = magic_no / (tau_pos - 0.5) + 0.5
    return Omega.TRT(1.0 / tau_pos, 1.0 / tau_neg)


class CellFlags:
    """Per-cell behaviour bits, combinable with ``|`` (src/simulation.rs:79-89).

    The update kernels treat both FIXED_FLUID_* bits alike (the mask ``c & 6``): such a cell
    keeps its initial density and velocity.
    """

    FLUID = 0
    WALL = 1
    FIXED_FLUID_VELOCITY = 2
    FIXED_FLUID_DENSITY = 4
    FIXED_SCALAR_VALUE = 8
    FIXED_FLUID = FIXED_FLUID_VELOCITY | FIXED_FLUID_DENSITY


def check_lbm_params(
    Re: float, L: float, tau: float, M_max: float = 0.1, slack: float = 0.0, bgk: bool = True
) -> None:
    """Asserts the BGK stability bound L >= Re / 24 and the Mach bound on tau
    (python/boltzmann/core.py:84-110)."""
    margin = 1.0 + slack
    tau_limit = math.sqrt(3.0) * M_max * margin * L / Re + 0.5
    min_length = Re / margin / 24.0
    eps = 1e-8
    assert (not bgk) or (L + eps > min_length), (
        f"BGK stability condition violated. {L=} < {min_length}"
    )
    assert tau < tau_limit + eps, f"Mach condition violated. {tau=} > {tau_limit}"


def calc_lbm_params_lu(
    Re: float,
    L: float,
    tau: float | None = None,
    M_max: float = 0.1,
    tau_max: float = 1.0,
    tau_min: float = 0.5,
    slack: float = 0.0,
    bgk: bool = True,
) -> tuple[float, float]:
    """(tau, u) in lattice units for Reynolds number ``Re`` over ``L`` cells
    (python/boltzmann/core.py:113-148). Without ``tau`` the largest tau the Mach bound allows
    is taken, clipped to [tau_min, tau_max]."""
    if tau is None:
        tau = min(max(math.sqrt(3.0) * M_max * L / Re + 0.5, tau_min), tau_max)
    check_lbm_params(Re, L, tau, M_max, slack, bgk)
    nu = (tau - 0.5) / 3.0
    return tau, Re * nu / L


def calc_lbm_params_si(
    dx: float,
    u_si: float,
    L_si: float,
    nu_si: float,
    tau: float | None = None,
    M_max: float = 0.1,
    tau_max: float = 10.0,
    tau_min: float = 0.5,
    slack: float = 0.0,
    bgk: bool = True,
) -> tuple[float, float]:
    """Same as :func:`calc_lbm_params_lu` from SI quantities (python/boltzmann/core.py:151-202)."""
    Re = u_si * L_si / nu_si
    return calc_lbm_params_lu(
        Re, L_si / dx, tau=tau, M_max=M_max, tau_min=tau_min, tau_max=tau_max, slack=slack, bgk=bgk
    )
