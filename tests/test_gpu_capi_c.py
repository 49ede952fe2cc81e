"""A C host program (tests/capi_c/newton_step.c, compiled here with gcc against include/dndsb.h and
libdndsb.so) runs the reference's one-Newton-step sequence through the C-ABI alone and reproduces the
goldens of test/cpp/Euler/test_EulerEvaluator.cpp:231-260 and :302-330 (1e-6 relative, the reference's
own tolerance); its residual equals the Python-bound call bit for bit."""
import os
import subprocess

import numpy as np
import pytest
import torch

from tests.newton_case import CASES, initial_state

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _write_mesh(m, path):
    a = m.arrays()
    hdr = np.array([m.dim, m.cell_type, m.face_type, m.n_node, m.n_cell, a["cell2node"].shape[1], m.n_face, a["face2node"].shape[1],
                    a["cell2face"].shape[1], 0], dtype=np.int64)
    with open(path, "wb") as f:
        for x in (hdr, a["coords"], a["cell2node"], a["cell_shift"], a["face2node"], a["face_shift"], a["face2cell"], a["face_zone"],
                  a["face_pshift"], a["cell2face"]):
            f.write(np.ascontiguousarray(x).tobytes())


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("capi") / "newton_step")
    lib = os.path.join(ROOT, "dndsr_b200")
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-Wall", "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "capi_c", "newton_step.c"),
                           "-o", out, f"-L{lib}", "-ldndsb", "-L/usr/local/cuda/lib64", "-lcudart", "-lm", f"-Wl,-rpath,{lib}"])
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_c_program_newton_step(exe, tmp_path, name):
    case = CASES[name]
    m = case["mesh"]()
    mp, rp, up = str(tmp_path / "mesh.bin"), str(tmp_path / "rhs.bin"), str(tmp_path / "u.bin")
    _write_mesh(m, mp)
    from dndsr_b200.solver import RS, EulerEvaluator, VariationalReconstruction
    from tests.newton_case import GAS
    vr = VariationalReconstruction(m, case["vr_py"]).construct()
    ev = EulerEvaluator(vr, dict(nVars=5, riemannSolverType=case["rs"], rsMeanValueEig=case["rsMeanValueEig"], **GAS))
    u = vr.BuildUDof(5)
    vo = case["vr_oracle"]
    if "chi" in case["gold"]:
        init = "2"
        ev.InitializeUDOF(u, 2, case["gold"]["chi"])
    else:
        init = "0"
        u.copy_(torch.tensor(initial_state(case, vr.get("cellBary").reshape(-1, 3)), device="cuda"))
        u.cpu().numpy().tofile(up)
    args = [exe, mp, rp, str(RS[case["rs"]]), str(case["rsMeanValueEig"]), str(case["CFL"]), str(vo["maxOrder"]), str(vo["intOrder"]),
            str(vo["dirWeightScheme"]), str(vo["geomWeightScheme"]), init] + ([up] if init == "0" else [])
    out = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    vals = out.stdout.split()
    rhs_l1, inc_l2 = float(vals[1]), float(vals[3])
    g = case["gold"]
    assert abs(rhs_l1 - g["rhsDensityL1"]) <= g["rel_tol"] * g["rhsDensityL1"]
    assert abs(inc_l2 - g["incL2"]) <= g["rel_tol"] * g["incL2"]
    # the same residual through the Python binding, bit for bit
    dt = torch.zeros(m.n_cell, dtype=torch.float64, device="cuda")
    ev.EvaluateDt(dt, u, case["CFL"])
    rhs = torch.zeros_like(u)
    ev.EvaluateRHS(rhs, u, vr.BuildURec(5))
    got = np.fromfile(rp, dtype=np.float64).reshape(m.n_cell, 5)
    assert np.array_equal(got, rhs.cpu().numpy())
