"""The drop-in on the GPU: the reference's own main loop (the oracle driver
mirroring main.cpp:84-116, with the reference's Mesh, AMR, Body and
BCValues built from its own sources) holding a GpuNS_Solver from the C++
binding (immsered-boundary_b200/binding/ibgpu_ns_solver.H), whose
TimeMarching steps through the C ABI on the device, with the wall forces
read back from the device after every step.  Its dt and force history must
equal the reference's own run of the same case (committed histories):
exact build <= 1e-12 in the drag/lift coefficients and relative dt, FP64
build <= 1e-10.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import ORACLE_DIR  # noqa: E402

pytestmark = pytest.mark.gpu

BINARY = os.path.join(ORACLE_DIR, "_ref", "ref_naca_minmod_binding")
F_REF = 0.5 * 1.0 * 0.1
SMALL = {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4", "IB_USER_INIT": "0",
         "IB_NPTS": "120"}
# name of the reference history, its case, steps, binding precision, bound
CASES = [
    ("naca_forces_s400_n64_l3", SMALL, 400, "exact", 1e-12),
    ("naca_forces_s400_n64_l3", SMALL, 400, "fp64", 1e-10),
    ("naca_forces_s1000_n128_l4", make_golden.CONFIG1_ENV, 1000, "fp64", 1e-10),
]


def run_binding(env_case, steps, precision):
    work = tempfile.mkdtemp(prefix="binding_gpu_")
    log = os.path.join(work, "forces.bin")
    prec = {"fp64": 0, "exact": 1, "mixed": 2}[precision]
    env = dict(os.environ)
    env.update(env_case)
    env.update(IB_STEPS=str(steps), IB_FORCES="1", IB_FORCE_LOG=log, IB_BINDING_STEP="1",
               IB_BINDING_PRECISION=str(prec))
    out = subprocess.run([BINARY], cwd=work, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return np.fromfile(log, np.float64).reshape(steps, -1)


@pytest.mark.skipif(not os.path.exists(BINARY), reason="binding oracle not built (make -C oracle)")
@pytest.mark.parametrize("name,env_case,steps,precision,tol", CASES)
def test_reference_loop_steps_through_the_binding(cuda_lib, name, env_case, steps, precision,
                                                  tol):
    ref = make_golden.load(name)["history"]
    got = run_binding(env_case, steps, precision)
    assert got.shape == ref.shape
    assert np.array_equal(got[:, 0], ref[:, 0])  # the same step counter
    dt_err = np.abs(got[:, 2] - ref[:, 2]) / ref[:, 2]
    nb = (ref.shape[1] - 3) // 6
    fg = got[:, 3:].reshape(steps, nb, 6)[:, :, :2]
    fr = ref[:, 3:].reshape(steps, nb, 6)[:, :, :2]
    coef_err = np.abs(fg - fr).max() / F_REF
    total_err = np.abs(fg.sum(axis=1) - fr.sum(axis=1)).max() / F_REF
    print(f"\n{name} {precision}: max rel dt {dt_err.max():.2e}, max |dC| per surface "
          f"{coef_err:.2e}, airfoil {total_err:.2e}")
    assert dt_err.max() <= tol and coef_err <= tol and total_err <= tol
