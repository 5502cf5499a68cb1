"""A plain-C program linked against libedk.so through include/edk.h only."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import workload

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_harness_against_oracle(tmp_path):
    exe = tmp_path / "harness"
    subprocess.check_call(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "edk_abi_harness.c"), "-o", str(exe),
                           "-L", os.path.dirname(edk.LIB_PATH), "-ledk",
                           "-Wl,-rpath," + os.path.dirname(edk.LIB_PATH)])
    m = workload("c1").model
    with open(tmp_path / "model.bin", "wb") as f:
        f.write(np.ascontiguousarray(m.eb).tobytes())
        f.write(np.ascontiguousarray(m.vbc).tobytes())
    x = np.random.default_rng(2).normal(size=4900)
    x.tofile(tmp_path / "x.bin")
    out = subprocess.run([str(exe), "x.bin", "y.bin"], cwd=tmp_path, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    y = np.fromfile(tmp_path / "y.bin")
    assert np.array_equal(y, O.OracleH(m, 4, 4).hmult(x))
    e0 = float(out.stdout.split()[3])
    assert abs(e0 - O.lanczos_e0(O.OracleH(m, 4, 4))["E"][0]) < 1e-10
