"""Output from the device state (row f4): the reference's own Tecplot
solution writer (Pltoutput::Output_Soln_Nobody, Pltoutput.cpp:147-170 with
Print_Level_Soln, :417-455: primitive variables, Mach number, wall and
domain distances, box indices and vorticity of every level) fed by
GpuNS_Solver::Download after the binding stepped on the GPU, against the
same writer after the reference's own steps: byte for byte with the exact
build, on the static airfoil and on the pitching one across a regrid (its
wall distances from the device passes)."""
import filecmp
import os
import subprocess
import sys
import tempfile

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402
from conftest import ORACLE_DIR  # noqa: E402

pytestmark = pytest.mark.gpu

REF = os.path.join(ORACLE_DIR, "_ref")
SMALL = {"IB_NX": "64", "IB_LEVELS": "3", "IB_STAGES": "4", "IB_USER_INIT": "0",
         "IB_NPTS": "120", "IB_FORCES": "1"}
CASES = {"naca": ("ref_naca_minmod", SMALL, 30),
         "pitch": ("ref_pitch_minmod", make_golden.PITCH_ENV, 24)}


def solution_file(binary, env_case, steps, gpu):
    work = tempfile.mkdtemp(prefix="plt_")
    env = dict(os.environ)
    env.update(env_case)
    env.update(IB_STEPS=str(steps), IB_PLT="soln")
    if gpu:
        env.update(IB_BINDING_STEP="1", IB_BINDING_PRECISION="1")  # the exact build
        binary += "_binding"
    out = subprocess.run([os.path.join(REF, binary)], cwd=work, env=env, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    path = os.path.join(work, f"soln-{steps}.plt")
    assert os.path.getsize(path) > 100_000
    return path


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_writer_on_the_device_state(cuda_lib, name):
    binary, env_case, steps = CASES[name]
    if not os.path.exists(os.path.join(REF, binary + "_binding")):
        pytest.skip("binding oracle not built (make -C oracle)")
    ref = solution_file(binary, env_case, steps, gpu=False)
    got = solution_file(binary, env_case, steps, gpu=True)
    assert filecmp.cmp(ref, got, shallow=False)
