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


def test_ctypes_layouts_match_c(pkg, tmp_path):
    ib = pkg.ibgpu
    mirrors = {"ibgpu_case": ib.Case, "ibgpu_cells": ib.Cells, "ibgpu_cf_pairs": ib.CfPairs,
               "ibgpu_bc": ib.Bc, "ibgpu_ib": ib.Ib, "ibgpu_diag": ib.Diag,
               "ibgpu_tag_rule": ib.TagRule, "ibgpu_tag_cells": ib.TagCells}
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
