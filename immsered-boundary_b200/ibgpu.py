"""ctypes binding of the ibgpu C ABI (include/ibgpu.h) and a host-side
driver that mirrors the reference solver's step interface.

The reference (C++) drives one time step as
``AMR::InterfaceExchange -> Body::IBConditions_Image -> NS_Solver::TimeMarching``
(main.cpp:87-97); :class:`FlowSolver` offers the same step as
``time_marching()`` over a device-resident state.  All numerics run in the
CUDA library; this module only moves descriptors and host buffers.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libibgpu.so")

ABI_VERSION = 1
MAX_LEVELS = 16

OK, E_ARG, E_CUDA, E_STATE, E_ABORT, E_NOMEM, E_TOPOLOGY, E_TIMEOUT = 0, -1, -2, -3, -4, -5, -6, -7
LIM_VANLEER, LIM_MINMOD = 0, 1
FP64, FP64_EXACT, MIXED = 0, 1, 2
CELL_PRESENT, CELL_NORMAL, CELL_UPDATE, CELL_PRIM, CELL_RESET, CELL_RESNORM, CELL_ALIAS = (
    1, 2, 4, 8, 16, 32, 64)

# every symbol include/ibgpu.h declares
EXPORTS = ("ibgpu_create", "ibgpu_set_stream", "ibgpu_upload_topology", "ibgpu_layout_info",
           "ibgpu_upload_interfaces", "ibgpu_upload_boundaries", "ibgpu_upload_ib",
           "ibgpu_wall_forces", "ibgpu_upload_state", "ibgpu_download_state", "ibgpu_step",
           "ibgpu_set_kernel_timing", "ibgpu_kernel_times", "ibgpu_destroy", "ibgpu_errstr",
           "ibgpu_last_error", "ibgpu_step_periodic_noalloc", "ibgpu_tag_plain",
           "ibgpu_indicator_features", "ibgpu_mlp_forward", "ibgpu_mlp_grad", "ibgpu_mlp_adam",
           "ibgpu_tag_learned", "ibgpu_run", "ibgpu_mlp_train_step", "ibgpu_batch_create",
           "ibgpu_batch_run", "ibgpu_batch_set_timing", "ibgpu_batch_info", "ibgpu_batch_tuning",
           "ibgpu_batch_destroy", "ibgpu_upload_signdis", "ibgpu_tag_mesh",
           "ibgpu_download_state_async", "ibgpu_synchronize", "ibgpu_batch_tag_mesh",
           "ibgpu_batch_table_bytes", "ibgpu_batch_set_grid", "ibgpu_batch_set_block", "ibgpu_upload_state_async",
           "ibgpu_step_async", "ibgpu_step_result", "ibgpu_update_flags", "ibgpu_update_flags_rows",
           "ibgpu_set_state_rows", "ibgpu_build_interfaces", "ibgpu_wall_geometry",
           "ibgpu_wall_distance", "ibgpu_host_register", "ibgpu_host_unregister",
           "ibgpu_wall_distance_near", "ibgpu_wall_fetch")
ROWS_FLOWVARS, ROWS_COMPACT = 7, 4
NOALLOC_MAX_CELLS = 65536
TAG_MAX_LEVELS = 16
TAG_REFINE, TAG_COARSEN = 1, 2
MLP_IN, MLP_STENCIL, MLP_HIDDEN, MLP_CLASSES, MLP_PARAMS = 112, 100, 64, 3, 11587


class Case(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("gama", ctypes.c_double), ("Rg", ctypes.c_double), ("Cv", ctypes.c_double),
        ("Cp", ctypes.c_double), ("Ma", ctypes.c_double), ("Re", ctypes.c_double),
        ("Pr", ctypes.c_double), ("qk", ctypes.c_double), ("s_over_t", ctypes.c_double),
        ("cfl", ctypes.c_double), ("dt_ratio", ctypes.c_double), ("dt_var_step", ctypes.c_int),
        ("nstages", ctypes.c_int), ("tp", ctypes.c_double * 4),
        ("limiter", ctypes.c_int), ("viscous", ctypes.c_int), ("precision", ctypes.c_int),
        ("initvar", ctypes.c_double * 7),
        ("nlevels", ctypes.c_int),
        ("dh", (ctypes.c_double * 3) * MAX_LEVELS),
        ("march_step", ctypes.c_int * MAX_LEVELS), ("march_left", ctypes.c_int * MAX_LEVELS),
        ("step_num", ctypes.c_double * MAX_LEVELS),
        ("domain_nx", ctypes.c_int), ("domain_ny", ctypes.c_int),
        ("periodic_x", ctypes.c_int), ("periodic_y", ctypes.c_int),
        ("average_step", ctypes.c_int * MAX_LEVELS), ("average_left", ctypes.c_int * MAX_LEVELS),
        ("prolong_step", ctypes.c_int * MAX_LEVELS), ("prolong_left", ctypes.c_int * MAX_LEVELS),
        ("body_level", ctypes.c_int),
        ("p_ref", ctypes.c_double), ("area_ref", ctypes.c_double), ("shear_ref", ctypes.c_double),
        ("L_ref", ctypes.c_double), ("mu", ctypes.c_double),
    ]


class CfPairs(ctypes.Structure):
    _fields_ = [("nres", ctypes.c_int64), ("res", ctypes.POINTER(ctypes.c_int32)),
                ("npro", ctypes.c_int64), ("pro", ctypes.POINTER(ctypes.c_int32))]


class Bc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("ghost", ctypes.POINTER(ctypes.c_int32)),
                ("nmv", ctypes.POINTER(ctypes.c_double)), ("nfaces", ctypes.c_int),
                ("facevar", ctypes.POINTER(ctypes.c_double)), ("backpressure", ctypes.c_double),
                ("inlet_flow_angle", ctypes.c_double)]


class Ib(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_int64), ("cell", ctypes.POINTER(ctypes.c_int32)),
                ("cellf", ctypes.POINTER(ctypes.c_double)), ("npatches", ctypes.c_int64),
                ("patch", ctypes.POINTER(ctypes.c_int32)), ("patchf", ctypes.POINTER(ctypes.c_double)),
                ("nbodies", ctypes.c_int), ("body_center", ctypes.POINTER(ctypes.c_double))]


class InterfaceLists(ctypes.Structure):
    _fields_ = [("nres", ctypes.c_int64), ("npro", ctypes.c_int64), ("nghost", ctypes.c_int64),
                ("cap_res", ctypes.c_int64), ("cap_pro", ctypes.c_int64),
                ("cap_ghost", ctypes.c_int64), ("res", ctypes.c_void_p), ("pro", ctypes.c_void_p),
                ("ghost", ctypes.c_void_p)]


# device wall distances of moved bodies (ibgpu_wall_*)
WALL_BOX_OTHER, WALL_BOX_DOMAIN_GHOST, WALL_BOX_BLOCK_GHOST = 0, 1, 2
WALL_MAX_NB = 15
WALL_INTO_BODY, WALL_OUT_OF_BODY = 1, 2
WALL_RESIDENT = 1


class WallLevelGeom(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("center", ctypes.c_void_p), ("neib", ctypes.c_void_p),
                ("kind", ctypes.c_void_p), ("distance_to_dm", ctypes.c_void_p),
                ("nblock", ctypes.c_int64), ("block_in", ctypes.c_void_p),
                ("block_out", ctypes.c_void_p)]


class WallBodies(ctypes.Structure):
    _fields_ = [("nbodies", ctypes.c_int), ("patch_start", ctypes.c_void_p),
                ("pc", ctypes.c_void_p), ("nv", ctypes.c_void_p), ("nb_count", ctypes.c_void_p),
                ("nb", ctypes.c_void_p), ("periodic_y", ctypes.c_int),
                ("critic_ylength", ctypes.c_double), ("dm_length_y", ctypes.c_double)]


class WallPairs(ctypes.Structure):
    _fields_ = [("body", ctypes.c_void_p), ("patch", ctypes.c_void_p),
                ("distance", ctypes.c_void_p), ("signdis", ctypes.c_void_p),
                ("distance_to_body", ctypes.c_void_p), ("solid", ctypes.c_void_p),
                ("moved", ctypes.c_void_p), ("block_moved", ctypes.c_void_p)]


class WallChange(ctypes.Structure):
    _fields_ = [("box", ctypes.c_int32), ("body", ctypes.c_int32), ("patch", ctypes.c_int32),
                ("solid", ctypes.c_uint8), ("moved", ctypes.c_uint8),
                ("pad_", ctypes.c_uint8 * 2), ("distance", ctypes.c_double),
                ("signdis", ctypes.c_double), ("distance_to_body", ctypes.c_double)]


WALL_CHANGE_DTYPE = np.dtype([("box", np.int32), ("body", np.int32), ("patch", np.int32),
                              ("solid", np.uint8), ("moved", np.uint8), ("pad_", np.uint8, 2),
                              ("distance", np.float64), ("signdis", np.float64),
                              ("distance_to_body", np.float64)])


class WallNear(ctypes.Structure):
    _fields_ = [("band", ctypes.c_double), ("capacity", ctypes.c_int64),
                ("changes", ctypes.c_void_p), ("count", ctypes.c_int64),
                ("block_moved", ctypes.c_void_p)]


class Cells(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("level", ctypes.POINTER(ctypes.c_int32)),
                ("ix", ctypes.POINTER(ctypes.c_int32)), ("iy", ctypes.POINTER(ctypes.c_int32)),
                ("flags", ctypes.POINTER(ctypes.c_uint8))]


class Diag(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("cfl_dt", ctypes.c_double),
                ("res_max", ctypes.c_double * 5), ("abort_code", ctypes.c_int),
                ("abort_level", ctypes.c_int), ("abort_ix", ctypes.c_int),
                ("abort_iy", ctypes.c_int), ("abort_step", ctypes.c_int),
                ("cells_marched", ctypes.c_int64)]


_TL = TAG_MAX_LEVELS


class TagRule(ctypes.Structure):
    """ibgpu_tag_rule: the case hook AMR::TagtheBox as data."""
    _fields_ = [("body_left_x", ctypes.c_double), ("body_right_x", ctypes.c_double),
                ("body_center_y", ctypes.c_double), ("body_half_height", ctypes.c_double),
                ("n_rect", ctypes.c_int), ("n_rect_coarsen", ctypes.c_int),
                ("torefine", ctypes.c_int * _TL), ("toderefine", ctypes.c_int * _TL),
                ("rect_up", ctypes.c_double * _TL), ("rect_down", ctypes.c_double * _TL),
                ("rect_half", ctypes.c_double * _TL), ("band_lo", ctypes.c_double * _TL),
                ("band_hi", ctypes.c_double * _TL), ("near_margin", ctypes.c_double * _TL),
                ("derect_up", ctypes.c_double * _TL), ("derect_down", ctypes.c_double * _TL),
                ("derect_half", ctypes.c_double * _TL), ("deband_lo", ctypes.c_double * _TL),
                ("deband_hi", ctypes.c_double * _TL), ("denear_margin", ctypes.c_double * _TL)]


class TagCells(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("level", ctypes.POINTER(ctypes.c_int32)),
                ("ix", ctypes.POINTER(ctypes.c_int32)), ("iy", ctypes.POINTER(ctypes.c_int32)),
                ("xc", ctypes.POINTER(ctypes.c_double)), ("yc", ctypes.POINTER(ctypes.c_double)),
                ("signdis", ctypes.POINTER(ctypes.c_double))]


def make_tag_rule(rule: dict) -> TagRule:
    """ibgpu_tag_rule from a dict with the same keys (arrays of up to 16)."""
    r = TagRule()
    for name, ctype in TagRule._fields_:
        if name not in rule:
            continue
        v = rule[name]
        if hasattr(ctype, "_length_"):
            arr = getattr(r, name)
            vals = np.asarray(v).ravel()
            for k in range(min(len(vals), ctype._length_)):
                arr[k] = vals[k].item()
        else:
            setattr(r, name, v.item() if hasattr(v, "item") else v)
    return r


class _TagCellsHolder:
    """Keeps the numpy arrays of a TagCells alive."""

    def __init__(self, level, ix, iy, xc, yc, signdis):
        self.arrays = [np.ascontiguousarray(level, np.int32), np.ascontiguousarray(ix, np.int32),
                       np.ascontiguousarray(iy, np.int32), np.ascontiguousarray(xc, np.float64),
                       np.ascontiguousarray(yc, np.float64),
                       np.ascontiguousarray(signdis, np.float64)]
        lv, x, y, a, b, s = self.arrays
        i32 = ctypes.POINTER(ctypes.c_int32)
        f64 = ctypes.POINTER(ctypes.c_double)
        self.s = TagCells(len(lv), lv.ctypes.data_as(i32), x.ctypes.data_as(i32),
                          y.ctypes.data_as(i32), a.ctypes.data_as(f64), b.ctypes.data_as(f64),
                          s.ctypes.data_as(f64))
        self.n = len(lv)


class IbgpuError(RuntimeError):
    def __init__(self, code: int, what: str, detail: str = "", diag: Diag | None = None):
        self.code = code
        self.diag = diag
        self.abort_code = diag.abort_code if diag is not None else 0
        msg = f"{what}: {lib().ibgpu_errstr(code).decode()} ({code})"
        if detail:
            msg += f" [{detail}]"
        if diag is not None and diag.abort_code:
            msg += (f" abort code {diag.abort_code} at level {diag.abort_level} "
                    f"cell ({diag.abort_ix},{diag.abort_iy})")
        super().__init__(msg)


_lib = None


def lib(path: str | None = None):
    """Load libibgpu.so (fails loudly when the CUDA library is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"ibgpu CUDA library not built: {p} is missing "
                          "(run immsered-boundary_b200/build_lib.py)")
    L = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    L.ibgpu_create.argtypes = [ctypes.POINTER(Case), ctypes.POINTER(vp)]
    L.ibgpu_set_stream.argtypes = [vp, vp]
    L.ibgpu_upload_topology.argtypes = [vp, ctypes.POINTER(Cells)]
    L.ibgpu_layout_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    L.ibgpu_update_flags.argtypes = [vp, vp]
    L.ibgpu_set_state_rows.argtypes = [vp, ctypes.c_int]
    L.ibgpu_build_interfaces.argtypes = [vp, ctypes.c_int, ctypes.POINTER(Cells),
                                         ctypes.POINTER(InterfaceLists)]
    L.ibgpu_upload_interfaces.argtypes = [vp, ctypes.POINTER(CfPairs)]
    L.ibgpu_upload_boundaries.argtypes = [vp, ctypes.POINTER(Bc)]
    L.ibgpu_upload_ib.argtypes = [vp, ctypes.POINTER(Ib)]
    L.ibgpu_wall_forces.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ibgpu_upload_state.argtypes = [vp, vp]
    L.ibgpu_download_state.argtypes = [vp, vp]
    L.ibgpu_step.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(Diag)]
    L.ibgpu_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(Diag)]
    L.ibgpu_set_kernel_timing.argtypes = [vp, ctypes.c_int]
    L.ibgpu_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    L.ibgpu_step_periodic_noalloc.argtypes = [ctypes.POINTER(Case), ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, vp, vp, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(Diag), vp]
    L.ibgpu_tag_plain.argtypes = [vp, ctypes.POINTER(TagRule), ctypes.POINTER(TagCells), vp]
    L.ibgpu_indicator_features.argtypes = [vp, ctypes.POINTER(TagRule), ctypes.POINTER(TagCells), vp]
    L.ibgpu_mlp_forward.argtypes = [vp, vp, ctypes.c_int64, vp, vp, vp]
    L.ibgpu_mlp_grad.argtypes = [vp, vp, ctypes.c_int64, vp, vp, ctypes.POINTER(ctypes.c_float),
                                 vp, vp]
    L.ibgpu_mlp_adam.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_float]
    L.ibgpu_tag_learned.argtypes = [vp, ctypes.POINTER(TagRule), ctypes.POINTER(TagCells), vp, vp]
    L.ibgpu_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_int64, vp, vp, ctypes.POINTER(ctypes.c_float), vp]
    L.ibgpu_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    L.ibgpu_batch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(Diag)]
    L.ibgpu_batch_set_timing.argtypes = [vp, ctypes.c_int]
    L.ibgpu_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_int64)]
    L.ibgpu_batch_tuning.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]
    L.ibgpu_batch_set_block.argtypes = [vp, ctypes.c_int]
    L.ibgpu_batch_table_bytes.argtypes = [vp]
    L.ibgpu_batch_set_grid.argtypes = [vp, ctypes.c_int]
    L.ibgpu_upload_state_async.argtypes = [vp, vp]
    L.ibgpu_step_async.argtypes = [vp, ctypes.c_int, ctypes.c_double]
    L.ibgpu_step_result.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(Diag)]
    L.ibgpu_upload_signdis.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ibgpu_download_state_async.argtypes = [vp, vp]
    L.ibgpu_batch_tag_mesh.argtypes = [vp, ctypes.POINTER(TagRule), vp, vp]
    L.ibgpu_synchronize.argtypes = [vp]
    L.ibgpu_tag_mesh.argtypes = [vp, ctypes.POINTER(TagRule), vp, vp]
    L.ibgpu_batch_destroy.argtypes = [vp]
    L.ibgpu_batch_destroy.restype = None
    L.ibgpu_destroy.argtypes = [vp]
    L.ibgpu_destroy.restype = None
    L.ibgpu_errstr.argtypes = [ctypes.c_int]
    L.ibgpu_errstr.restype = ctypes.c_char_p
    L.ibgpu_last_error.argtypes = []
    L.ibgpu_last_error.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("ibgpu_destroy", "ibgpu_errstr", "ibgpu_last_error", "ibgpu_batch_destroy"):
            getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _check(rc: int, what: str, diag: Diag | None = None):
    if rc != OK:
        raise IbgpuError(rc, what, lib().ibgpu_last_error().decode(), diag)


def make_case(params: dict) -> Case:
    """Fill an ibgpu_case from a parameter dict (same keys as the fields)."""
    c = Case()
    c.abi_version = ABI_VERSION
    for k in ("gama", "Rg", "Cv", "Cp", "Ma", "Re", "Pr", "qk", "s_over_t", "cfl", "dt_ratio"):
        setattr(c, k, float(params.get(k, 0.0)))
    c.dt_var_step = int(params.get("dt_var_step", 1))
    c.nstages = int(params["nstages"])
    for i, v in enumerate(params["tp"]):
        c.tp[i] = float(v)
    c.limiter = int(params.get("limiter", LIM_VANLEER))
    c.viscous = int(params.get("viscous", 0))
    c.precision = int(params.get("precision", FP64))
    for i, v in enumerate(params["initvar"]):
        c.initvar[i] = float(v)
    nl = int(params["nlevels"])
    c.nlevels = nl
    for l in range(nl):
        for k in range(3):
            c.dh[l][k] = float(params["dh"][l][k])
        c.march_step[l] = int(params["march_step"][l])
        c.march_left[l] = int(params["march_left"][l])
        c.step_num[l] = float(params["step_num"][l])
    c.domain_nx = int(params["domain_nx"])
    c.domain_ny = int(params["domain_ny"])
    c.periodic_x = int(params.get("periodic_x", 0))
    c.periodic_y = int(params.get("periodic_y", 0))
    for l in range(nl):
        c.average_step[l] = int(params.get("average_step", [2] * nl)[l])
        c.average_left[l] = int(params.get("average_left", [1] * nl)[l])
        c.prolong_step[l] = int(params.get("prolong_step", [2] * nl)[l])
        c.prolong_left[l] = int(params.get("prolong_left", [1] * nl)[l])
    c.body_level = int(params.get("body_level", -1))
    for k in ("p_ref", "area_ref", "shear_ref", "L_ref", "mu"):
        setattr(c, k, float(params.get(k, 1.0)))
    return c


def _i32(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _f64(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def step_periodic_noalloc(params: dict, ts: int, nx: int, ny: int, d_rows_in: int,
                          d_rows_out: int, dt: float, stream: int = 0):
    """One step of a periodic single-level grid through the allocation-free
    entry point; d_rows_in/out are device addresses of (nx*ny, 7) float64
    rows in row-major cell order.  Returns (dt, Diag)."""
    case = make_case(params)
    d = Diag()
    dtv = ctypes.c_double(dt)
    rc = lib().ibgpu_step_periodic_noalloc(ctypes.byref(case), int(ts), int(nx), int(ny),
                                           ctypes.c_void_p(d_rows_in), ctypes.c_void_p(d_rows_out),
                                           ctypes.byref(dtv), ctypes.byref(d), ctypes.c_void_p(stream))
    if rc != OK:
        raise IbgpuError(rc, "ibgpu_step_periodic_noalloc", lib().ibgpu_last_error().decode(), d)
    return dtv.value, d


class FlowSolver:
    """GPU time step behind the reference's NS_Solver step interface.

    ``upload_topology`` takes the canonical cell list (level, ix, iy, flags),
    ``init_flow``/``download`` move FlowVariables rows (roe,u,v,w,p,T,e), and
    ``time_marching(ts)`` runs one full step (NS_Solver::TimeMarching plus the
    ghost fills the reference runs before it).
    """

    def __init__(self, params: dict):
        self._case = make_case(params)
        self._ctx = ctypes.c_void_p()
        _check(lib().ibgpu_create(ctypes.byref(self._case), ctypes.byref(self._ctx)), "ibgpu_create")
        self.params = dict(params)
        self.dt = float(params.get("dt0", 1.0))
        self.ncells = 0
        self._keep = []
        self.init_res = None
        self._batches = weakref.WeakSet()  # batches holding this context

    def close(self):
        # a batch runs on its first case's stream and holds the contexts:
        # it goes first
        for b in list(self._batches):
            b.close()
        if self._ctx:
            lib().ibgpu_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        _check(lib().ibgpu_set_stream(self._ctx, ctypes.c_void_p(stream_handle or 0)), "ibgpu_set_stream")

    def upload_topology(self, level, ix, iy, flags):
        lv = np.ascontiguousarray(level, np.int32)
        x = np.ascontiguousarray(ix, np.int32)
        y = np.ascontiguousarray(iy, np.int32)
        f = np.ascontiguousarray(flags, np.uint8)
        cells = Cells(len(lv), lv.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      x.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      y.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                      f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        _check(lib().ibgpu_upload_topology(self._ctx, ctypes.byref(cells)), "ibgpu_upload_topology")
        self.ncells = len(lv)

    def update_flags(self, flags):
        """New IBGPU_CELL_* flags for the rows of the last topology upload
        (a moved body: same mesh, new inside / immersed-boundary cells)."""
        f = np.ascontiguousarray(flags, np.uint8)
        assert len(f) == self.ncells
        _check(lib().ibgpu_update_flags(self._ctx, f.ctypes.data_as(ctypes.c_void_p)),
               "ibgpu_update_flags")

    def update_flags_rows(self, rows, flags):
        """New flags for some rows only (ibgpu_update_flags_rows): rows[k]
        gets flags[k], the other rows keep theirs."""
        r = np.ascontiguousarray(rows, np.int64)
        f = np.ascontiguousarray(flags, np.uint8)
        assert len(r) == len(f)
        _check(lib().ibgpu_update_flags_rows(self._ctx, ctypes.c_int64(len(r)),
                                             r.ctypes.data_as(ctypes.c_void_p),
                                             f.ctypes.data_as(ctypes.c_void_p)),
               "ibgpu_update_flags_rows")

    def build_interfaces(self, nlevels: int, level, ix, iy):
        """Coarse/fine interface lists of the mesh whose leaf cells are
        (level, ix, iy), built on the device: (restriction rows (n, 12),
        prolongation rows (n, 11), interface ghost cells (n, 3))."""
        lv = np.ascontiguousarray(level, np.int32)
        x = np.ascontiguousarray(ix, np.int32)
        y = np.ascontiguousarray(iy, np.int32)
        i32 = ctypes.POINTER(ctypes.c_int32)
        cells = Cells(len(lv), lv.ctypes.data_as(i32), x.ctypes.data_as(i32),
                      y.ctypes.data_as(i32), None)
        out = InterfaceLists()
        rc = lib().ibgpu_build_interfaces(self._ctx, int(nlevels), ctypes.byref(cells),
                                          ctypes.byref(out))
        if rc not in (OK, E_ARG) or (rc == E_ARG and out.nres + out.npro + out.nghost == 0
                                     and len(lv)):
            _check(rc, "ibgpu_build_interfaces")
        res = np.zeros((out.nres, 12), np.int32)
        pro = np.zeros((out.npro, 11), np.int32)
        ghost = np.zeros((out.nghost, 3), np.int32)
        out.cap_res, out.cap_pro, out.cap_ghost = out.nres, out.npro, out.nghost
        out.res, out.pro, out.ghost = (res.ctypes.data, pro.ctypes.data, ghost.ctypes.data)
        _check(lib().ibgpu_build_interfaces(self._ctx, int(nlevels), ctypes.byref(cells),
                                            ctypes.byref(out)), "ibgpu_build_interfaces")
        return res, pro, ghost

    def wall_geometry(self, levels):
        """Boxes of every level for the device wall distances: a list of
        dicts with center (n, 3), neib (n, 9), kind (n), distance_to_dm (n),
        block_in, block_out (ibgpu_wall_geometry)."""
        keep, geoms = [], []
        for g in levels:
            c = np.ascontiguousarray(g["center"], np.float64).reshape(-1, 3)
            nb = np.ascontiguousarray(g["neib"], np.int32).reshape(-1, 9)
            k = np.ascontiguousarray(g["kind"], np.uint8)
            dm = np.ascontiguousarray(g["distance_to_dm"], np.float64)
            bi = np.ascontiguousarray(g.get("block_in", []), np.int32)
            bo = np.ascontiguousarray(g.get("block_out", []), np.int32)
            keep += [c, nb, k, dm, bi, bo]
            geoms.append(WallLevelGeom(len(c), c.ctypes.data, nb.ctypes.data, k.ctypes.data,
                                       dm.ctypes.data, len(bi), bi.ctypes.data, bo.ctypes.data))
        arr = (WallLevelGeom * max(len(geoms), 1))(*geoms)
        _check(lib().ibgpu_wall_geometry(self._ctx, len(geoms), arr), "ibgpu_wall_geometry")

    @staticmethod
    def _wall_bodies(bodies: dict):
        arrs = dict(ps=np.ascontiguousarray(bodies["patch_start"], np.int32),
                    pc=np.ascontiguousarray(bodies["pc"], np.float64),
                    nv=np.ascontiguousarray(bodies["nv"], np.float64),
                    nbc=np.ascontiguousarray(bodies["nb_count"], np.int32),
                    nbl=np.ascontiguousarray(bodies["nb"], np.int32))
        wb = WallBodies(len(arrs["ps"]) - 1, arrs["ps"].ctypes.data, arrs["pc"].ctypes.data,
                        arrs["nv"].ctypes.data, arrs["nbc"].ctypes.data, arrs["nbl"].ctypes.data,
                        int(bodies.get("periodic_y", 0)),
                        float(bodies.get("critic_ylength", 1e300)),
                        float(bodies.get("dm_length_y", 0.0)))
        return wb, arrs

    def wall_distance_near(self, bodies: dict, bands, nboxes, nblocks):
        """ibgpu_wall_distance_near: from the pairs the device holds, per level
        (band, room for nboxes reported boxes, its block-pair count) a
        structured array of the reported boxes (WALL_CHANGE_DTYPE, box order)
        and the block pairs' moved flags."""
        wb, keep = self._wall_bodies(bodies)
        outs = [(np.zeros(max(int(n), 1), WALL_CHANGE_DTYPE), np.zeros(max(int(nbk), 1), np.uint8))
                for n, nbk in zip(nboxes, nblocks)]
        arr = (WallNear * max(len(outs), 1))(*[
            WallNear(float(b), int(n), ch.ctypes.data, 0, bm.ctypes.data)
            for b, n, (ch, bm) in zip(bands, nboxes, outs)])
        _check(lib().ibgpu_wall_distance_near(self._ctx, ctypes.byref(wb), len(outs), arr),
               "ibgpu_wall_distance_near")
        return [(ch[:arr[l].count], bm[:int(nbk)]) for l, ((ch, bm), nbk) in
                enumerate(zip(outs, nblocks))]

    def wall_fetch(self, nboxes):
        """ibgpu_wall_fetch: every level's pairs (dicts of body, patch,
        distance, signdis, distance_to_body, solid) as the device holds them."""
        out, arrs = [], []
        for n in nboxes:
            n = int(n)
            p = dict(body=np.zeros(n, np.int32), patch=np.zeros(n, np.int32),
                     distance=np.zeros(n), signdis=np.zeros(n), distance_to_body=np.zeros(n),
                     solid=np.zeros(n, np.uint8))
            out.append(p)
            arrs.append(WallPairs(*(p[k].ctypes.data for k in (
                "body", "patch", "distance", "signdis", "distance_to_body", "solid")), None, None))
        arr = (WallPairs * max(len(arrs), 1))(*arrs)
        _check(lib().ibgpu_wall_fetch(self._ctx, len(arrs), arr), "ibgpu_wall_fetch")
        return out

    def wall_distance(self, bodies: dict, pairs, resident: bool = False):
        """The bodies' patches (patch_start, pc (n, 3), nv (n, 3), nb_count,
        nb (n, 15); periodic_y, critic_ylength, dm_length_y) and every
        level's pairs (dicts of body, patch, distance, signdis,
        distance_to_body, solid): updated in place, with moved and
        block_moved added (ibgpu_wall_distance).  resident: start from the
        pairs the device kept from the previous call (the dicts' input
        values are not read)."""
        wb, keep = self._wall_bodies(bodies)
        arrs = []
        for p in pairs:
            for key, dt in (("body", np.int32), ("patch", np.int32), ("distance", np.float64),
                            ("signdis", np.float64), ("distance_to_body", np.float64),
                            ("solid", np.uint8)):
                p[key] = np.ascontiguousarray(p[key], dt)
            p["moved"] = np.zeros(len(p["body"]), np.uint8)
            p["block_moved"] = np.zeros(int(p.get("nblock", 0)), np.uint8)
            arrs.append(WallPairs(*(p[k].ctypes.data for k in (
                "body", "patch", "distance", "signdis", "distance_to_body", "solid", "moved",
                "block_moved"))))
        arr = (WallPairs * max(len(arrs), 1))(*arrs)
        _check(lib().ibgpu_wall_distance(self._ctx, ctypes.byref(wb), len(arrs), arr,
                                         WALL_RESIDENT if resident else 0),
               "ibgpu_wall_distance")
        return pairs

    def upload_interfaces(self, res, pro):
        """Coarse/fine pairs as (n, 11) int arrays: level, cx, cy, 4 x (fx, fy)."""
        r, rp = _i32(np.asarray(res, np.int32).reshape(-1, 11))
        p, pp = _i32(np.asarray(pro, np.int32).reshape(-1, 11))
        c = CfPairs(len(r), rp, len(p), pp)
        _check(lib().ibgpu_upload_interfaces(self._ctx, ctypes.byref(c)), "ibgpu_upload_interfaces")

    def upload_boundaries(self, ghost, nmv, facevar, backpressure=0.0, inlet_flow_angle=0.0):
        """Domain ghosts (n, 7): level, x, y, ref_x, ref_y, face, type, in the
        reference's processing order; nmv (n, 3); facevar (nfaces, 7)."""
        g, gp = _i32(np.asarray(ghost, np.int32).reshape(-1, 7))
        n, np_ = _f64(np.asarray(nmv, np.float64).reshape(-1, 3))
        f, fp = _f64(np.asarray(facevar, np.float64).reshape(-1, 7))
        b = Bc(len(g), gp, np_, len(f), fp, float(backpressure), float(inlet_flow_angle))
        _check(lib().ibgpu_upload_boundaries(self._ctx, ctypes.byref(b)), "ibgpu_upload_boundaries")

    def upload_ib(self, cell, cellf, patch, patchf, body_center):
        c, cp = _i32(np.asarray(cell, np.int32).reshape(-1, 18))
        cf, cfp = _f64(np.asarray(cellf, np.float64).reshape(-1, 16))
        p, pp = _i32(np.asarray(patch, np.int32).reshape(-1, 17))
        pf, pfp = _f64(np.asarray(patchf, np.float64).reshape(-1, 19))
        bc, bcp = _f64(np.asarray(body_center, np.float64).reshape(-1, 3))
        ib = Ib(len(c), cp, cfp, len(p), pp, pfp, len(bc), bcp)
        _check(lib().ibgpu_upload_ib(self._ctx, ctypes.byref(ib)), "ibgpu_upload_ib")
        self.nbodies = len(bc)

    # ---- refinement indicator (AMR::TagtheBox and its learned replacement)
    def tag_plain(self, rule: dict, level, xc, yc, signdis, ix=None, iy=None) -> np.ndarray:
        """IBGPU_TAG_REFINE | IBGPU_TAG_COARSEN bits per box, computed on the GPU."""
        z = np.zeros(len(level), np.int32)
        h = _TagCellsHolder(level, z if ix is None else ix, z if iy is None else iy, xc, yc, signdis)
        r = make_tag_rule(rule)
        out = np.zeros(max(h.n, 1), np.uint8)
        _check(lib().ibgpu_tag_plain(self._ctx, ctypes.byref(r), ctypes.byref(h.s),
                                     out.ctypes.data_as(ctypes.c_void_p)), "ibgpu_tag_plain")
        return out[:h.n]

    def indicator_features(self, rule: dict, level, ix, iy, xc, yc, signdis, d_feat: int):
        """Write the boxes' feature rows (BF16 bits, n x 112) to device address d_feat."""
        h = _TagCellsHolder(level, ix, iy, xc, yc, signdis)
        r = make_tag_rule(rule)
        _check(lib().ibgpu_indicator_features(self._ctx, ctypes.byref(r), ctypes.byref(h.s),
                                              ctypes.c_void_p(d_feat)), "ibgpu_indicator_features")

    def tag_learned(self, rule: dict, level, ix, iy, xc, yc, signdis, d_params: int) -> np.ndarray:
        h = _TagCellsHolder(level, ix, iy, xc, yc, signdis)
        r = make_tag_rule(rule)
        out = np.zeros(max(h.n, 1), np.uint8)
        _check(lib().ibgpu_tag_learned(self._ctx, ctypes.byref(r), ctypes.byref(h.s),
                                       ctypes.c_void_p(d_params), out.ctypes.data_as(ctypes.c_void_p)),
               "ibgpu_tag_learned")
        return out[:h.n]

    def upload_signdis(self, signdis):
        s, sp = _f64(signdis)
        _check(lib().ibgpu_upload_signdis(self._ctx, sp), "ibgpu_upload_signdis")

    def tag_mesh(self, rule: dict, d_params: int = 0) -> np.ndarray:
        """Tag bits of every uploaded cell row: learned (d_params) or plain."""
        r = make_tag_rule(rule)
        out = np.zeros(max(self.ncells, 1), np.uint8)
        _check(lib().ibgpu_tag_mesh(self._ctx, ctypes.byref(r), ctypes.c_void_p(d_params or None),
                                    out.ctypes.data_as(ctypes.c_void_p)), "ibgpu_tag_mesh")
        return out[:self.ncells]

    def mlp_forward(self, d_params: int, n: int, d_feat: int, d_class: int, d_logits: int = 0):
        _check(lib().ibgpu_mlp_forward(self._ctx, ctypes.c_void_p(d_params), int(n),
                                       ctypes.c_void_p(d_feat), ctypes.c_void_p(d_class),
                                       ctypes.c_void_p(d_logits or None)), "ibgpu_mlp_forward")

    def mlp_grad(self, d_params: int, n: int, d_feat: int, d_label: int, class_weight,
                 d_grad: int, d_stats: int):
        cw = (ctypes.c_float * 3)(*[float(c) for c in class_weight])
        _check(lib().ibgpu_mlp_grad(self._ctx, ctypes.c_void_p(d_params), int(n),
                                    ctypes.c_void_p(d_feat), ctypes.c_void_p(d_label), cw,
                                    ctypes.c_void_p(d_grad), ctypes.c_void_p(d_stats)),
               "ibgpu_mlp_grad")

    def mlp_train_step(self, d_params: int, d_m: int, d_v: int, d_grad: int, step: int, lr: float,
                       n: int, d_feat: int, d_label: int, class_weight, d_stats: int):
        cw = (ctypes.c_float * 3)(*[float(c) for c in class_weight])
        _check(lib().ibgpu_mlp_train_step(self._ctx, ctypes.c_void_p(d_params), ctypes.c_void_p(d_m),
                                          ctypes.c_void_p(d_v), ctypes.c_void_p(d_grad), int(step),
                                          float(lr), int(n), ctypes.c_void_p(d_feat),
                                          ctypes.c_void_p(d_label), cw, ctypes.c_void_p(d_stats)),
               "ibgpu_mlp_train_step")

    def mlp_adam(self, d_params: int, d_grad: int, d_m: int, d_v: int, step: int, lr: float):
        _check(lib().ibgpu_mlp_adam(self._ctx, ctypes.c_void_p(d_params), ctypes.c_void_p(d_grad),
                                    ctypes.c_void_p(d_m), ctypes.c_void_p(d_v), int(step),
                                    float(lr)), "ibgpu_mlp_adam")

    def wall_forces(self):
        """(nbodies, 6): force(3), moment(3) in the reference's scaling."""
        nb = getattr(self, "nbodies", 0)
        out = np.zeros((max(nb, 1), 6))
        _check(lib().ibgpu_wall_forces(self._ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
               "ibgpu_wall_forces")
        return out[:nb]

    def layout_info(self):
        ns, nt = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().ibgpu_layout_info(self._ctx, ctypes.byref(ns), ctypes.byref(nt)), "ibgpu_layout_info")
        return ns.value, nt.value

    def set_state_rows(self, fields: int):
        """Row format of the state transfers: ROWS_FLOWVARS (7 doubles per cell)
        or ROWS_COMPACT (roe, u, v, p)."""
        _check(lib().ibgpu_set_state_rows(self._ctx, int(fields)), "ibgpu_set_state_rows")
        self.row_fields = int(fields)

    def init_flow(self, prim_rows):
        """Upload state rows (n, 7) or, in the compact format, (n, 4); also
        accepts a host pointer (int)."""
        if isinstance(prim_rows, int):
            _check(lib().ibgpu_upload_state(self._ctx, ctypes.c_void_p(prim_rows)), "ibgpu_upload_state")
            return
        a = np.ascontiguousarray(prim_rows, np.float64)
        assert a.shape == (self.ncells, getattr(self, "row_fields", 7))
        _check(lib().ibgpu_upload_state(self._ctx, a.ctypes.data_as(ctypes.c_void_p)), "ibgpu_upload_state")

    def download(self, out=None):
        if isinstance(out, int):
            _check(lib().ibgpu_download_state(self._ctx, ctypes.c_void_p(out)), "ibgpu_download_state")
            return None
        a = np.empty((self.ncells, getattr(self, "row_fields", 7)), np.float64) if out is None else out
        _check(lib().ibgpu_download_state(self._ctx, a.ctypes.data_as(ctypes.c_void_p)), "ibgpu_download_state")
        return a

    def download_async(self, out_ptr: int):
        """Enqueue a download into host memory at out_ptr (pinned for
        overlap); valid after synchronize()."""
        _check(lib().ibgpu_download_state_async(self._ctx, ctypes.c_void_p(out_ptr)),
               "ibgpu_download_state_async")

    def synchronize(self):
        _check(lib().ibgpu_synchronize(self._ctx), "ibgpu_synchronize")

    def upload_async(self, in_ptr: int):
        """Enqueue an upload of the rows at host address in_ptr (pinned for
        overlap; left unchanged until synchronize() or step_result())."""
        _check(lib().ibgpu_upload_state_async(self._ctx, ctypes.c_void_p(in_ptr)),
               "ibgpu_upload_state_async")

    def step_async(self, ts: int):
        """Enqueue step ts without waiting; the first one after a result
        starts from self.dt, later ones from the dt the device computed."""
        _check(lib().ibgpu_step_async(self._ctx, int(ts), ctypes.c_double(self.dt)),
               "ibgpu_step_async")

    def step_result(self) -> Diag:
        """Wait and report the last asynchronous step (dt into self.dt)."""
        d = Diag()
        dt = ctypes.c_double(self.dt)
        rc = lib().ibgpu_step_result(self._ctx, ctypes.byref(dt), ctypes.byref(d))
        if rc != OK:
            raise IbgpuError(rc, "ibgpu_step_result", lib().ibgpu_last_error().decode(), d)
        self.dt = dt.value
        return d

    def time_marching(self, ts: int) -> Diag:
        d = Diag()
        dt = ctypes.c_double(self.dt)
        rc = lib().ibgpu_step(self._ctx, int(ts), ctypes.byref(dt), ctypes.byref(d))
        if rc != OK:
            raise IbgpuError(rc, "ibgpu_step", lib().ibgpu_last_error().decode(), d)
        self.dt = dt.value
        return d

    def run(self, ts0: int, nsteps: int) -> Diag:
        """nsteps steps back to back, one host synchronisation at the end."""
        d = Diag()
        dt = ctypes.c_double(self.dt)
        rc = lib().ibgpu_run(self._ctx, int(ts0), int(nsteps), ctypes.byref(dt), ctypes.byref(d))
        if rc != OK:
            raise IbgpuError(rc, "ibgpu_run", lib().ibgpu_last_error().decode(), d)
        self.dt = dt.value
        return d

    def set_kernel_timing(self, on: bool):
        _check(lib().ibgpu_set_kernel_timing(self._ctx, int(bool(on))), "ibgpu_set_kernel_timing")

    def kernel_times(self):
        ms = (ctypes.c_double * 3)()
        n = (ctypes.c_int64 * 3)()
        _check(lib().ibgpu_kernel_times(self._ctx, ms, n), "ibgpu_kernel_times")
        return list(ms), list(n)

    def res_normalised(self, diag: Diag, ts: int):
        """ResinDomain's printed residual (NS_Solver.H:331-345): max-norm
        divided by the step-0 value, z component zero in 2-D."""
        r = list(diag.res_max)
        if ts == 0 or self.init_res is None:
            self.init_res = r
        out = [r[i] / self.init_res[i] if self.init_res[i] else float("nan") for i in range(5)]
        out[3] = 0.0
        return out


# box kinds of the reference mesh as the adapters report them
BOX_NORMAL, BOX_DOMAIN_GHOST, BOX_BLOCK_GHOST, BOX_OTHER_GHOST = 0, 1, 2, 3


def cell_flags_from_boxes(kind, solid, infect, signdis, body_level: bool) -> np.ndarray:
    """Per-cell IBGPU_CELL_* flags from the reference's box attributes.

    Encodes which branch of UpdateConsVars / ComptNewPrimVar / ResinDomain
    (NS_Solver.cpp:3-194, 844-985; NS_Solver.H:264-378) a box takes: on the
    finest level of a run with bodies only non-solid, non-immersed-boundary
    boxes are updated, elsewhere every leaf box is; a leaf box inside a body
    (signed distance <= 0) is reset to the free stream instead of recovering
    its primitives.  Block (periodic) ghosts become aliases.
    """
    kind = np.asarray(kind)
    fl = np.full(kind.shape, CELL_PRESENT, np.uint8)
    normal = kind == BOX_NORMAL
    fl[normal] |= CELL_NORMAL
    pos = np.asarray(signdis) > 0.0
    if body_level:
        free = np.asarray(infect) == -1
        upd = normal & free & (np.asarray(solid) == 0)
        fl[upd] |= CELL_UPDATE
        fl[upd & pos] |= CELL_PRIM
        fl[normal & free & ~pos] |= CELL_RESET
        fl[normal & free & pos] |= CELL_RESNORM
    else:
        fl[normal] |= CELL_UPDATE | CELL_RESNORM
        fl[normal & pos] |= CELL_PRIM
        fl[normal & ~pos] |= CELL_RESET
    fl[kind == BOX_BLOCK_GHOST] |= CELL_ALIAS
    return fl


class Batch:
    """Several FlowSolver cases advanced together (ibgpu_batch_*): one
    persistent, graph-replayed launch per stage covers every case's tiles."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s._ctx.value for s in self.solvers])
        self._b = ctypes.c_void_p()
        _check(lib().ibgpu_batch_create(arr, len(self.solvers), ctypes.byref(self._b)),
               "ibgpu_batch_create")
        for s in self.solvers:
            s._batches.add(self)

    def run(self, ts0: int, nsteps: int):
        """nsteps steps of every case; returns the per-case Diag list."""
        n = len(self.solvers)
        dt = (ctypes.c_double * n)(*[s.dt for s in self.solvers])
        diags = (Diag * n)()
        rc = lib().ibgpu_batch_run(self._b, int(ts0), int(nsteps), dt, diags)
        for i, s in enumerate(self.solvers):
            s.dt = dt[i]
        if rc != OK:
            bad = next((d for d in diags if d.abort_code), None)
            raise IbgpuError(rc, "ibgpu_batch_run", lib().ibgpu_last_error().decode(), bad)
        return list(diags)

    def tag_mesh(self, rule: dict, d_params: int = 0, out=None) -> list:
        """Row tags of every case (learned with d_params, else plain); out
        may be a preallocated uint8 array (e.g. pinned) of all cases' rows."""
        r = make_tag_rule(rule)
        n = sum(s.ncells for s in self.solvers)
        if out is None:
            out = np.zeros(max(n, 1), np.uint8)
        _check(lib().ibgpu_batch_tag_mesh(self._b, ctypes.byref(r), ctypes.c_void_p(d_params or None),
                                          out.ctypes.data_as(ctypes.c_void_p)), "ibgpu_batch_tag_mesh")
        res, off = [], 0
        for s in self.solvers:
            res.append(out[off:off + s.ncells])
            off += s.ncells
        return res

    def set_timing(self, on: bool):
        _check(lib().ibgpu_batch_set_timing(self._b, int(bool(on))), "ibgpu_batch_set_timing")

    def set_grid(self, grid: int):
        """CTA count of the merged stage launches: 0 one per work item, > 0
        persistent CTAs, -1 autotuned at the next run (default)."""
        _check(lib().ibgpu_batch_set_grid(self._b, int(grid)), "ibgpu_batch_set_grid")

    def set_block(self, threads: int):
        """Threads per CTA of the merged stage launches: 256 or 288, 0
        autotuned at the next run (default); the same results either way."""
        _check(lib().ibgpu_batch_set_block(self._b, int(threads)), "ibgpu_batch_set_block")

    def info(self) -> dict:
        g, nt, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        ms, nl = ctypes.c_double(), ctypes.c_int64()
        _check(lib().ibgpu_batch_info(self._b, ctypes.byref(g), ctypes.byref(nt), ctypes.byref(p),
                                      ctypes.byref(ms), ctypes.byref(nl)), "ibgpu_batch_info")
        grids, blocks = (ctypes.c_int * 32)(), (ctypes.c_int * 32)()
        tms = (ctypes.c_float * 32)()
        k = lib().ibgpu_batch_tuning(self._b, 32, grids, blocks, tms)
        return dict(grid=g.value, threads=nt.value, period=p.value, stage_ms=ms.value,
                    stage_launches=nl.value,
                    tuning=[(grids[i], blocks[i], tms[i]) for i in range(max(0, min(k, 32)))],
                    table_bytes=lib().ibgpu_batch_table_bytes(self._b))

    def close(self):
        if self._b:
            lib().ibgpu_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
