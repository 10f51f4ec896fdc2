"""Nondimensional constants of the solver, computed from a case's parameter
set exactly as LunarSolver::calc_physical_constant does
(Z4_Lunar/src/physics/LunarSolver_Tools.cpp:3-45), and the Farfield state of
BuildLunarBackgroundState (Z4_Lunar/include/0_BackgroundState.h:20-66)."""
from __future__ import annotations

import math
from typing import Dict

from . import case as _case


def constants(p: Dict[str, object]) -> Dict[str, float]:
    NA, R_uni, q_e, mu0 = _case.NA, _case.R_UNI, _case.Q_E, _case.MU0
    gamma = _case.GAMMA
    r = p["REF"]
    U_ref = r["U"]
    L_ref = r["L_ref"]
    B_ref = r["B_ref"]
    T_ref = r["T"]
    n_ref = r["n"]
    M_ref = r["Molecular_mass"]
    rho_ref = M_ref * n_ref / NA
    M_H = p["mole_mass1"]
    state_coeff_H = (R_uni * T_ref) / (M_H * U_ref * U_ref)
    hall_coef = B_ref * M_ref / (U_ref * q_e * L_ref * mu0 * rho_ref * NA)
    momentum_hall_coeff = (B_ref * B_ref) / (mu0 * rho_ref * U_ref * U_ref)
    inver_MA2 = B_ref * B_ref / (U_ref * U_ref * mu0 * rho_ref)
    inver_Rem = p["eta_max_lunar"] / (mu0 * U_ref * L_ref)
    return dict(gamma=gamma, cfl=float(p["CFL"]), inver_MA2=inver_MA2, momentum_hall_coeff=momentum_hall_coeff,
                state_coeff=state_coeff_H, M_H=M_H, M_ref=M_ref, ne_hall_floor=0.01, hall_coef=hall_coef,
                inver_Rem=inver_Rem, rho_ref=rho_ref, U_ref=U_ref, L_ref=L_ref, B_ref=B_ref, T_ref=T_ref,
                n_ref=n_ref)


def farfield_state(p: Dict[str, object]):
    """(qinf[5], B_imf[3]) of the Farfield boundary."""
    NA, R_uni = _case.NA, _case.R_UNI
    gamma = _case.GAMMA
    k_B = R_uni / NA
    ini = p["INITIAL"]
    ref = p["REF"]
    B_ref = ref["B_ref"]
    B_imf = [ini["Bx"] / B_ref, ini["By"] / B_ref, ini["Bz"] / B_ref]
    U_ref, n_ref, T_ref, M_ref = ref["U"], ref["n"], ref["T"], ref["Molecular_mass"]
    rho_ref = M_ref / NA * n_ref
    rho0 = (ini["n"] / n_ref) * (ini["Molecular_mass"] / M_ref)
    c_y, c_z = ini["c_y"], ini["c_z"]
    c_x = -math.sqrt(1.0 - c_y * c_y - c_z * c_z)
    u0 = c_x * ini["U"] / U_ref
    v0 = c_y * ini["U"] / U_ref
    w0 = c_z * ini["U"] / U_ref
    p_ini = ini["n"] * k_B * ini["T"]
    p0 = p_ini / (rho_ref * U_ref * U_ref)
    qinf = [rho0, rho0 * u0, rho0 * v0, rho0 * w0,
            0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0) + p0 / (gamma - 1.0)]
    return qinf, B_imf
