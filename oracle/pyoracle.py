"""ctypes front end of the CPU oracle (test infrastructure only).

Imported by tests/ (to test the GPU path against) and by bench.py's cpu_baseline leg; the
GPU library never imports it.  Provides

* ``read_dump``: reader for the state dumps written by the reference-solver
  oracle driver (oracle/ref_driver.cpp);
* ``OracleLevels``: the dense per-level arrays the C restatement
  (oracle/ib_oracle.c) steps, built from a dump or from cell lists;
* ``step``: one reference time step on those arrays.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libib_oracle.so")

PRESENT, NORMAL, UPDATE, PRIM, RESET, RESNORM = 1, 2, 4, 8, 16, 32
LIM_VANLEER, LIM_MINMOD = 0, 1

# kind codes of a dumped box (oracle/ref_driver.cpp)
K_NORMAL, K_DMGHOST, K_BLOCKGHOST, K_OTHERGHOST = 0, 1, 2, 3


def build_lib() -> str:
    """Compile the C restatement (no contraction, strict IEEE) if needed."""
    src = os.path.join(HERE, "ib_oracle.c")
    hdr = os.path.join(HERE, "ib_oracle.h")
    newest = max(os.path.getmtime(src), os.path.getmtime(hdr))
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
                               "-shared", "-o", LIB_PATH, src, "-lm"])
    return LIB_PATH


class _Params(ctypes.Structure):
    _fields_ = [("gama", ctypes.c_double), ("Rg", ctypes.c_double), ("Cv", ctypes.c_double),
                ("Ma", ctypes.c_double), ("Re", ctypes.c_double), ("qk", ctypes.c_double),
                ("s_over_t", ctypes.c_double), ("cfl", ctypes.c_double),
                ("dt_ratio", ctypes.c_double), ("tp", ctypes.c_double * 4),
                ("initvar", ctypes.c_double * 7), ("nstages", ctypes.c_int),
                ("limiter", ctypes.c_int), ("viscous", ctypes.c_int),
                ("dt_var_step", ctypes.c_int), ("body_level", ctypes.c_int)]


class _Level(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int), ("y0", ctypes.c_int), ("nx", ctypes.c_int),
                ("ny", ctypes.c_int), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double), ("march_step", ctypes.c_int),
                ("march_left", ctypes.c_int), ("step_num", ctypes.c_double),
                ("flags", ctypes.POINTER(ctypes.c_uint8)),
                ("q", ctypes.POINTER(ctypes.c_double) * 7), ("ncopy", ctypes.c_int),
                ("copy_dst", ctypes.POINTER(ctypes.c_int32)),
                ("copy_src", ctypes.POINTER(ctypes.c_int32))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build_lib())
        _lib.ibo_step.restype = ctypes.c_int
        _lib.ibo_step.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(_Level), ctypes.c_int,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double)]
    return _lib


def read_dump(path: str) -> dict:
    """Read a tagged binary dump: [u32 len][name][u32 kind][u64 n][payload]."""
    with open(path, "rb") as f:
        b = f.read()
    out, o = {}, 0
    while o < len(b):
        (n,) = struct.unpack_from("<I", b, o)
        o += 4
        name = b[o:o + n].decode()
        o += n
        kind, cnt = struct.unpack_from("<IQ", b, o)
        o += 12
        dt = np.float64 if kind == 0 else np.int32
        a = np.frombuffer(b, dtype=dt, count=cnt, offset=o).copy()
        o += cnt * a.itemsize
        out[name] = a
    return out


def params_from_dump(d: dict, limiter: int, viscous: bool) -> dict:
    s = d["scalars"]
    nst = int(s[14])
    return dict(gama=s[4], Rg=s[5], Cv=s[6], Cp=s[7], Ma=s[8], Re=s[9], Pr=s[10], qk=s[11],
                s_over_t=s[12], cfl=s[13], nstages=nst, tp=list(s[15:15 + nst]),
                initvar=list(d["initvar"]), limiter=limiter, viscous=int(viscous),
                dt_ratio=1.0, dt_var_step=1)


def cell_flags(kind, solid, infect, signdis, body_level: bool) -> np.ndarray:
    """Per-box flags following UpdateConsVars / ComptNewPrimVar / ResinDomain
    (NS_Solver.cpp:3-194, 844-985; NS_Solver.H:264-378)."""
    kind = np.asarray(kind)
    fl = np.full(kind.shape, PRESENT, np.uint8)
    normal = kind == K_NORMAL
    fl[normal] |= NORMAL
    pos = np.asarray(signdis) > 0.0
    if body_level:
        free = (np.asarray(infect) == -1)
        upd = normal & free & (np.asarray(solid) == 0)
        fl[upd] |= UPDATE
        fl[upd & pos] |= PRIM
        fl[normal & free & ~pos] |= RESET
        fl[normal & free & pos] |= RESNORM
    else:
        fl[normal] |= UPDATE | RESNORM
        fl[normal & pos] |= PRIM
        fl[normal & ~pos] |= RESET
    return fl


class OracleLevels:
    """Dense per-level arrays for the C restatement."""

    def __init__(self, d: dict):
        dom = d["domain"]
        self.nx0, self.ny0 = int(dom[0]), int(dom[1])
        self.periodic = (bool(dom[2]), bool(dom[3]))
        nbody, nlev = int(dom[4]), int(dom[5])
        dh = d["dh"].reshape(-1, 3)
        sched = d["schedule"].reshape(-1, 6)
        self.levels = []
        prim = d["prim"].reshape(-1, 7)
        for l in range(nlev):
            m = d["level"] == l
            ix, iy = d["ix"][m], d["iy"][m]
            x0, y0 = int(ix.min()), int(iy.min())
            nx, ny = int(ix.max()) - x0 + 1, int(iy.max()) - y0 + 1
            slot = (iy - y0) * nx + (ix - x0)
            flags = np.zeros(nx * ny, np.uint8)
            body_level = nbody > 0 and l == nlev - 1
            flags[slot] = cell_flags(d["kind"][m], d["solid"][m], d["infect"][m],
                                     d["signdis"][m], body_level)
            q = np.zeros((7, nx * ny))
            q[:, slot] = prim[m].T
            # periodic/block ghost copies: destination slot <- wrapped source slot
            blk = d["kind"][m] == K_BLOCKGHOST
            ext_x = self.nx0 * (1 << l)
            ext_y = self.ny0 * (1 << l)
            sx = ix[blk] % ext_x if self.periodic[0] else ix[blk]
            sy = iy[blk] % ext_y if self.periodic[1] else iy[blk]
            dst = slot[blk].astype(np.int32)
            src = ((sy - y0) * nx + (sx - x0)).astype(np.int32)
            self.levels.append(dict(
                x0=x0, y0=y0, nx=nx, ny=ny, dx=dh[l, 0], dy=dh[l, 1], dz=dh[l, 2],
                march_step=int(sched[l, 0]), march_left=int(sched[l, 3]),
                step_num=float(sched[l, 0]), flags=flags, q=np.ascontiguousarray(q),
                copy_dst=np.ascontiguousarray(dst), copy_src=np.ascontiguousarray(src),
                slot=slot, mask=m))

    def state_like_dump(self, d: dict) -> np.ndarray:
        """Return the (n, 7) prim array in the row order of dump ``d``."""
        out = np.zeros((len(d["level"]), 7))
        for l, L in enumerate(self.levels):
            m = d["level"] == l
            slot = (d["iy"][m] - L["y0"]) * L["nx"] + (d["ix"][m] - L["x0"])
            out[m] = L["q"][:, slot].T
        return out


def step(P: dict, lv: OracleLevels, ts: int, dt: float):
    """One reference time step in place.  Returns (rc, dt, cfl_dt, res_max)."""
    cp = _Params()
    for k in ("gama", "Rg", "Cv", "Ma", "Re", "qk", "s_over_t", "cfl", "dt_ratio"):
        setattr(cp, k, float(P[k]))
    for i, v in enumerate(P["tp"]):
        cp.tp[i] = v
    for i, v in enumerate(P["initvar"]):
        cp.initvar[i] = v
    cp.nstages = int(P["nstages"])
    cp.limiter = int(P["limiter"])
    cp.viscous = int(P["viscous"])
    cp.dt_var_step = int(P["dt_var_step"])
    cp.body_level = int(P.get("body_level", -1))
    arr = (_Level * len(lv.levels))()
    keep = []
    for i, L in enumerate(lv.levels):
        c = arr[i]
        c.x0, c.y0, c.nx, c.ny = L["x0"], L["y0"], L["nx"], L["ny"]
        c.dx, c.dy, c.dz = L["dx"], L["dy"], L["dz"]
        c.march_step, c.march_left, c.step_num = L["march_step"], L["march_left"], L["step_num"]
        c.flags = L["flags"].ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        for k in range(7):
            c.q[k] = L["q"][k].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        c.ncopy = len(L["copy_dst"])
        c.copy_dst = L["copy_dst"].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        c.copy_src = L["copy_src"].ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        keep.append(L)
    dtv = ctypes.c_double(dt)
    cfl = ctypes.c_double(0.0)
    res = (ctypes.c_double * 5)()
    rc = lib().ibo_step(ctypes.byref(cp), arr, len(lv.levels), int(ts), ctypes.byref(dtv),
                        ctypes.byref(cfl), res)
    return rc, dtv.value, cfl.value, list(res)
