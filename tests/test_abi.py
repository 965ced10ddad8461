"""The C ABI library (no GPU needed): it loads, it exports every entry point
include/*.h declares, and the ctypes mirrors match the C struct layouts."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ibgpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.ibgpu.lib()
    names = declared_functions()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(lib, n), f"{n} declared but not exported"
    assert set(pkg.ibgpu.EXPORTS) <= set(names)


def test_errstr_without_gpu(pkg):
    lib = pkg.ibgpu.lib()
    assert lib.ibgpu_errstr(0) == b"ok"
    assert b"argument" in lib.ibgpu_errstr(-1)
    assert lib.ibgpu_errstr(-99) == b"unknown error"


def test_null_arguments_are_rejected_without_gpu(pkg):
    lib = pkg.ibgpu.lib()
    assert lib.ibgpu_create(None, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_step(None, 0, None, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_upload_topology(None, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_upload_state_async(None, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_step_async(None, 0, 1.0) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_step_result(None, None, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_batch_set_grid(None, 0) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_batch_table_bytes(None) == 0
    assert lib.ibgpu_wall_geometry(None, 0, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_wall_distance(None, None, 0, None, 0) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_wall_distance_near(None, None, 0, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_wall_fetch(None, 0, None) == pkg.ibgpu.E_ARG
    assert lib.ibgpu_update_flags_rows(None, 0, None, None) == pkg.ibgpu.E_ARG


def test_ctypes_layouts_match_c(pkg, tmp_path):
    ib = pkg.ibgpu
    mirrors = {"ibgpu_case": ib.Case, "ibgpu_cells": ib.Cells, "ibgpu_cf_pairs": ib.CfPairs,
               "ibgpu_bc": ib.Bc, "ibgpu_ib": ib.Ib, "ibgpu_diag": ib.Diag,
               "ibgpu_tag_rule": ib.TagRule, "ibgpu_tag_cells": ib.TagCells,
               "ibgpu_interface_lists": ib.InterfaceLists,
               "ibgpu_wall_level_geom": ib.WallLevelGeom, "ibgpu_wall_bodies": ib.WallBodies,
               "ibgpu_wall_pairs": ib.WallPairs, "ibgpu_wall_change": ib.WallChange,
               "ibgpu_wall_near": ib.WallNear}
    # every field of every mirrored struct
    checks = {c: (cls, [f[0] for f in cls._fields_]) for c, cls in mirrors.items()}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ibgpu.h"', "int main(void){"]
    for cname, (_, fields) in checks.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", INCLUDE, str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split("\n")
    for line in out:
        if not line:
            continue
        cname, what, val = line.split()
        cls = checks[cname][0]
        if what == "size":
            assert ctypes.sizeof(cls) == int(val), f"{cname} size"
        else:
            assert getattr(cls, what).offset == int(val), f"{cname}.{what}"


@pytest.mark.parametrize("compiler,flags", [
    ("gcc", ["-x", "c", "-std=c99", "-pedantic"]),
    ("g++", ["-x", "c++", "-std=c++11", "-pedantic"])])
def test_header_compiles_standalone(tmp_path, compiler, flags):
    """The boundary header stands alone in C (cgo- or FFI-style bindings) and
    in C++ (the reference's own code), with no warning."""
    src = tmp_path / "use.c"
    src.write_text('#include "ibgpu.h"\nint main(void) { ibgpu_ctx *c = 0; '
                   'return ibgpu_create(0, &c) == IBGPU_OK; }\n')
    subprocess.check_call([compiler, *flags, "-Wall", "-Wextra", "-Werror", "-I", INCLUDE,
                           "-c", str(src), "-o", str(tmp_path / "use.o")])


def test_invalid_case_parameters_are_rejected_before_any_device_call(pkg):
    """ibgpu_create validates the case before it touches CUDA, so bad case
    parameters come back as IBGPU_E_ARG with a reason on any machine."""
    ib = pkg.ibgpu
    lib = ib.lib()
    base = dict(nstages=4, tp=[0.1084, 0.2602, 0.5052, 1.0],
                initvar=[1.0, 0.5, 0.0, 0.0, 1 / 1.4, 1.0, 0.0], nlevels=1, dh=[[0.1, 0.1, 0.1]],
                march_step=[1], march_left=[0], step_num=[1.0], domain_nx=32, domain_ny=32)

    def create(case):
        ctx = ctypes.c_void_p()
        rc = lib.ibgpu_create(ctypes.byref(case), ctypes.byref(ctx))
        if ctx:
            lib.ibgpu_destroy(ctx)
        return rc, lib.ibgpu_last_error().decode()

    bad = []
    c = ib.make_case(base)
    c.abi_version += 1
    bad.append((c, "ABI version"))
    for key, val in (("nstages", 0), ("nstages", 5), ("limiter", 2), ("precision", 3),
                     ("dt_var_step", 0)):
        c = ib.make_case(base)
        setattr(c, key, val)
        bad.append((c, "invalid case parameters"))
    for nl in (0, ib.MAX_LEVELS + 1):
        c = ib.make_case(base)
        c.nlevels = nl
        bad.append((c, "invalid case parameters"))
    for field, val in (("march_step", 0), ("dh", 0.0), ("dh", float("nan"))):
        c = ib.make_case(base)
        if field == "march_step":
            c.march_step[0] = val
        else:
            c.dh[0][1] = val
        bad.append((c, "invalid level parameters"))
    for c, why in bad:
        rc, msg = create(c)
        assert rc == ib.E_ARG and why in msg, (why, rc, msg)
    assert lib.ibgpu_create(None, None) == ib.E_ARG


def test_noalloc_entry_point_rejects_unsupported_grids_before_any_device_call(pkg):
    """The allocation-free step checks its case and grid before it touches
    the device: anything but one periodic inviscid level with sides that are
    multiples of 16 and at most IBGPU_NOALLOC_MAX_CELLS cells is IBGPU_E_ARG.
    (The row addresses are never dereferenced on these paths.)"""
    ib = pkg.ibgpu
    base = dict(nstages=4, tp=[0.1084, 0.2602, 0.5052, 1.0],
                initvar=[1.0, 0.5, 0.0, 0.0, 1 / 1.4, 1.0, 0.0], nlevels=1,
                dh=[[0.1, 0.1, 0.1]], march_step=[1], march_left=[0], step_num=[1.0],
                domain_nx=64, domain_ny=64, periodic_x=1, periodic_y=1)
    fake = 1 << 20  # stands for a device address; not read on the rejected paths
    cases = [
        (dict(base, periodic_x=0), 64, 64, "periodic inviscid"),
        (dict(base, viscous=1), 64, 64, "periodic inviscid"),
        (dict(base, domain_nx=48), 64, 64, "periodic inviscid"),
        (dict(base, domain_nx=40, domain_ny=40), 40, 40, "multiple of 16"),
        (dict(base, domain_nx=512, domain_ny=256), 512, 256, "IBGPU_NOALLOC_MAX_CELLS"),
    ]
    for params, nx, ny, why in cases:
        with pytest.raises(ib.IbgpuError) as e:
            ib.step_periodic_noalloc(params, 0, nx, ny, fake, fake, 1.0)
        assert e.value.code == ib.E_ARG and why in str(e.value), (why, str(e.value))
    assert 512 * 256 > ib.NOALLOC_MAX_CELLS
