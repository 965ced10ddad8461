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
                length: float = 10.0, mach: float = 0.5,
                angle_deg: float = 45.0) -> tuple[dict, dict, np.ndarray]:
    """Returns (params, cells, prim_rows) for the periodic isentropic vortex
    (advection Mach number and direction selectable; 0.5 and 45 degrees are
    the bandwidth workload)."""
    angle = angle_deg / 180.0 * math.pi
    g = gas_constants(mach, 0.0)
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


def naca_params(g: dict, k: int, precision: int) -> dict:
    """Case parameters of a NACA0012 AMR run from a mesh/state record of the
    reference solver (the dict of tests/golden/make_golden.load): gas
    constants, stage coefficients, level sizes and schedules, domain,
    body-force scales, and the dt of snapshot k."""
    s = g["scalars"][k]
    nst = int(s[14])
    dom = g["domain"]
    nlev = int(dom[5])
    sched = g["schedule"].reshape(-1, 6)
    dh = g["dh"].reshape(-1, 3)
    bf = g["body_f"]
    nb = int(dom[4])
    return dict(gama=s[4], Rg=s[5], Cv=s[6], Cp=s[7], Ma=s[8], Re=s[9], Pr=s[10], qk=s[11],
                s_over_t=s[12], cfl=s[13], nstages=nst, tp=list(s[15:15 + nst]),
                dt_var_step=int(s[15 + nst]), dt_ratio=1.0, limiter=1, viscous=1,
                precision=precision, initvar=list(g["initvar"]), nlevels=nlev,
                dh=[tuple(dh[l]) for l in range(nlev)],
                march_step=[int(sched[l, 0]) for l in range(nlev)],
                march_left=[int(sched[l, 3]) for l in range(nlev)],
                step_num=[float(sched[l, 0]) for l in range(nlev)],
                average_step=[int(sched[l, 1]) for l in range(nlev)],
                average_left=[int(sched[l, 4]) for l in range(nlev)],
                prolong_step=[int(sched[l, 2]) for l in range(nlev)],
                prolong_left=[int(sched[l, 5]) for l in range(nlev)],
                domain_nx=int(dom[0]), domain_ny=int(dom[1]), periodic_x=int(dom[2]),
                periodic_y=int(dom[3]), body_level=nlev - 1 if nb > 0 else -1,
                p_ref=bf[3 * nb], area_ref=bf[3 * nb + 1], shear_ref=bf[3 * nb + 2],
                L_ref=bf[3 * nb + 3], mu=bf[3 * nb + 4], dt0=float(s[1]))


def naca_lists(g: dict, k: int) -> dict:
    """The C ABI's lists of a mesh/state record of the reference solver:
    cell list with IBGPU_CELL_* flags, coarse/fine pairs, domain ghosts of
    the x and y faces, immersed-boundary cells and wall patches, and the
    state rows of snapshot k (the arguments of the ibgpu_upload_* calls)."""
    ib = ibgpu
    nlev = int(g["domain"][5])
    nb = int(g["domain"][4])
    body_level = nlev - 1 if nb > 0 else -1
    flags = np.zeros(len(g["level"]), np.uint8)
    for l in range(nlev):
        m = g["level"] == l
        flags[m] = ib.cell_flags_from_boxes(g["kind"][m], g["solid"][m], g["infect"][m],
                                            g["signdis"][m], l == body_level)
    bc = g["bc"].reshape(-1, 9)
    keep = (bc[:, 7] == 0) & (bc[:, 8] == 0)  # x/y faces, z = 0 plane
    return dict(level=g["level"], ix=g["ix"], iy=g["iy"], flags=flags,
                res=g["cf_res"].reshape(-1, 12)[:, [0, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]],
                pro=g["cf_pro"].reshape(-1, 12)[:, [0, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]],
                bc=bc[keep][:, :7], bc_nmv=g["bc_nmv"].reshape(-1, 3)[keep],
                facevar=g["facevar"].reshape(-1, 7), bc_scalars=g["bc_scalars"][:2],
                ib=g["ib"].reshape(-1, 20)[:, :18], ib_f=g["ib_f"].reshape(-1, 16),
                patch=g["patch"].reshape(-1, 17), patch_f=g["patch_f"].reshape(-1, 19),
                body_center=g["body_f"][:3 * nb].reshape(-1, 3), prim=g["prim"][k])


def naca_solver(g: dict, k: int, precision: int):
    """FlowSolver holding the record's mesh (cell list, coarse/fine pairs,
    domain ghosts, immersed-boundary cells and wall patches) and snapshot
    k's state."""
    P = naca_params(g, k, precision)
    L = naca_lists(g, k)
    sol = ibgpu.FlowSolver(P)
    sol.upload_topology(L["level"], L["ix"], L["iy"], L["flags"])
    sol.upload_interfaces(L["res"], L["pro"])
    sol.upload_boundaries(L["bc"], L["bc_nmv"], L["facevar"], L["bc_scalars"][0],
                          L["bc_scalars"][1])
    sol.upload_ib(L["ib"], L["ib_f"], L["patch"], L["patch_f"], L["body_center"])
    sol.init_flow(L["prim"])
    return sol


def naca_tag_rule(nlevels: int, dh, le_x: float = 9.5, le_y: float = 10.0,
                  chord: float = 1.0) -> dict:
    """ibgpu_tag_rule of the NACA0012 case's TagtheBox: rectangles (up 4s,
    down 8s, half-height 4s with s = 0.5^k) around the airfoil on levels
    k < nlevels-2, then the signed-distance band -3 dh_k < signdis <
    max(0.25, 16 dh_finest) inside the airfoil box grown by the band's upper
    limit; coarsening of level l judges against level l-1's region."""
    L = ibgpu.TAG_MAX_LEVELS
    z = lambda: np.zeros(L)  # noqa: E731
    r = dict(body_left_x=le_x, body_right_x=le_x + chord, body_center_y=le_y,
             body_half_height=0.5 * chord, n_rect=nlevels - 2, n_rect_coarsen=nlevels - 2,
             torefine=np.zeros(L, np.int32), toderefine=np.zeros(L, np.int32))
    for pre in ("", "de"):
        for key in ("rect_up", "rect_down", "rect_half", "band_lo", "band_hi", "near_margin"):
            r[pre + key] = z()
    re = max(0.25, 16.0 * float(dh[nlevels - 1]))
    for k in range(nlevels):
        s = 0.5 ** k
        for pre in ("", "de"):
            r[pre + "rect_up"][k] = 4.0 * s
            r[pre + "rect_down"][k] = 8.0 * s
            r[pre + "rect_half"][k] = 4.0 * s
            r[pre + "band_lo"][k] = -3.0 * float(dh[k])
            r[pre + "band_hi"][k] = re
            r[pre + "near_margin"][k] = re
    r["torefine"][:nlevels] = 1
    r["toderefine"][1:nlevels] = 1
    return r


def batch_vortex_cases(ncases: int, seed: int = 0, min_cells: int = 50_000,
                       max_cells: int = 800_000, precision: int = ibgpu.FP64):
    """Independent periodic vortex cases with uneven sizes for the batched
    solver: side n (a multiple of 16) with n^2 log-uniform in [min_cells,
    max_cells], advection Mach uniform in [0.1, 0.8] and direction uniform in
    [-5, 10] degrees from a seeded generator.  Returns a list of
    (params, cells, prim_rows)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ncases):
        cells = math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))
        n = max(16, int(round(math.sqrt(cells) / 16.0)) * 16)
        mach = float(rng.uniform(0.1, 0.8))
        ang = float(rng.uniform(-5.0, 10.0))
        out.append(vortex_case(n, precision=precision, mach=mach, angle_deg=ang))
    return out
