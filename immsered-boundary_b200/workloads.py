"""Synthetic workloads for the GPU step, built on the host from scratch.

``vortex_case``: the flux/stage bandwidth workload — an N x N single-level
periodic grid on [0,10]^2 holding an isentropic vortex (strength 5, centred at
(5,5)) advected at Mach 0.5 and 45 degrees, inviscid.  The gas constants are
derived exactly as the reference derives them from its reference scales
(FlowConstants.cpp:5-44) so a run here and a reference run on the same
inputs share every constant bit for bit.
"""
from __future__ import annotations

import math

import numpy as np

from . import ibgpu

# Low-storage multistage coefficients (NS_Solver.H:204-218)
TP = {3: (0.1918, 0.4929, 1.0), 4: (0.1084, 0.2602, 0.5052, 1.0)}


def gas_constants(mach: float, mu_ref: float, u_ref: float = 1.0, roe_ref: float = 1.0,
                  L_ref: float = 1.0) -> dict:
    """FlowConstants.cpp:5-44 with T_ref chosen so the free-stream Mach is
    ``mach`` (T_ref = u_ref^2 / (mach^2 Rg_ref gama), as the reference's case
    file does for Mach 0.1)."""
    gama, Rg_ref, Pr = 1.4, 287.4, 0.72
    T_ref = u_ref * u_ref / (mach * mach * Rg_ref * gama)
    Re = roe_ref * u_ref * L_ref / mu_ref if mu_ref != 0.0 else math.inf
    Ma = u_ref / math.sqrt(gama * Rg_ref * T_ref)
    Rg = 1.0 / (gama * math.pow(Ma, 2))
    Cv = Rg / (gama - 1.0)
    Cp = Cv + Rg
    mu = 1.0
    qk = mu / (Re * Pr * (gama - 1) * math.pow(Ma, 2))
    S_over_T_ref = 110.33333333 / T_ref
    return dict(gama=gama, Rg=Rg, Cv=Cv, Cp=Cp, Ma=Ma, Re=Re, Pr=Pr, qk=qk,
                s_over_t=S_over_T_ref, T_ref=T_ref)


def freestream(g: dict, angle: float) -> list:
    """BCValues::SetInitValues: unit speed at ``angle``, T from the Mach number."""
    u, v, w = math.cos(angle), math.sin(angle), 0.0
    speed = math.pow(math.pow(u, 2) + math.pow(v, 2) + math.pow(w, 2), 0.5)
    T = math.pow(speed / g["Ma"], 2) / (g["gama"] * g["Rg"])
    roe = 1.0
    p = roe * g["Rg"] * T
    e = g["Cv"] * T + 0.5 * (u * u + v * v + w * w)
    return [roe, u, v, w, p, T, e]


def vortex_case(n: int, nstages: int = 4, limiter: int = ibgpu.LIM_VANLEER,
                precision: int = ibgpu.FP64, cfl: float = 0.5, beta: float = 5.0,
                length: float = 10.0) -> tuple[dict, dict, np.ndarray]:
    """Returns (params, cells, prim_rows) for the periodic isentropic vortex."""
    angle = 45.0 / 180.0 * math.pi
    g = gas_constants(0.5, 0.0)
    init = freestream(g, angle)
    h = length / float(n)
    params = dict(g)
    params.update(cfl=cfl, dt_ratio=1.0, dt_var_step=1, nstages=nstages, tp=TP[nstages],
                  limiter=limiter, viscous=0, precision=precision, initvar=init, nlevels=1,
                  dh=[(h, h, 0.1)], march_step=[1], march_left=[0], step_num=[1.0],
                  domain_nx=n, domain_ny=n, periodic_x=1, periodic_y=1, dt0=1.0)
    iy, ix = np.meshgrid(np.arange(n, dtype=np.int32), np.arange(n, dtype=np.int32), indexing="ij")
    ix = ix.ravel()
    iy = iy.ravel()
    flags = np.full(ix.shape, ibgpu.CELL_PRESENT | ibgpu.CELL_NORMAL | ibgpu.CELL_UPDATE |
                    ibgpu.CELL_PRIM | ibgpu.CELL_RESNORM, np.uint8)
    cells = dict(level=np.zeros_like(ix), ix=ix, iy=iy, flags=flags)
    prim = vortex_state(ix, iy, h, g, init, beta)
    return params, cells, prim


def vortex_state(ix, iy, h, g, init, beta, xc=5.0, yc=5.0):
    """Isentropic vortex (Shu): velocity perturbation scaled by c_inf/sqrt(gamma),
    temperature dip -(gamma-1) beta^2/(8 gamma pi^2) exp(1-r^2), isentropic rho."""
    gama, Rg, Cv = g["gama"], g["Rg"], g["Cv"]
    x = (ix.astype(np.float64) + 0.5) * h - xc
    y = (iy.astype(np.float64) + 0.5) * h - yc
    r2 = x * x + y * y
    T_inf = init[5]
    cinf = math.sqrt(gama * Rg * T_inf)
    uscale = cinf / math.sqrt(gama)
    amp = beta / (2.0 * math.pi) * np.exp(0.5 * (1.0 - r2))
    u = init[1] - amp * y * uscale
    v = init[2] + amp * x * uscale
    dT = -(gama - 1.0) * beta * beta / (8.0 * gama * math.pi * math.pi) * np.exp(1.0 - r2)
    T = T_inf * (1.0 + dT)
    roe = init[0] * np.power(T / T_inf, 1.0 / (gama - 1.0))
    p = roe * Rg * T
    e = Cv * T + 0.5 * (u * u + v * v)
    prim = np.stack([roe, u, v, np.zeros_like(u), p, T, e], axis=1)
    return np.ascontiguousarray(prim)


def vortex_exact_density(n: int, t: float, beta: float = 5.0, length: float = 10.0) -> np.ndarray:
    """Exact density of the advected periodic vortex at time t (cell-centre
    samples, nearest periodic image), in the row order of ``vortex_case``."""
    angle = 45.0 / 180.0 * math.pi
    g = gas_constants(0.5, 0.0)
    init = freestream(g, angle)
    h = length / float(n)
    iy, ix = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x = (ix.ravel() + 0.5) * h
    y = (iy.ravel() + 0.5) * h
    xc = (5.0 + init[1] * t) % length
    yc = (5.0 + init[2] * t) % length
    dx = (x - xc + 0.5 * length) % length - 0.5 * length
    dy = (y - yc + 0.5 * length) % length - 0.5 * length
    r2 = dx * dx + dy * dy
    gama = g["gama"]
    dT = -(gama - 1.0) * beta * beta / (8.0 * gama * math.pi * math.pi) * np.exp(1.0 - r2)
    return init[0] * np.power(1.0 + dT, 1.0 / (gama - 1.0))
