"""The reference's own driver (Code/main.cpp and its host sources, unchanged)
built in place against this library's backend shim (oracle/_ref/exec_b200,
see oracle/build_oracle.py): run on the GPU it selects the B200 backend through
gpuAvailable / printGpuInfo / kroupaGPU exactly as it selects its CUDA
backend, and its output file matches the same driver's --cpu (OpenMP) run:
FP64 positions to the print precision (8 decimals), the same atoms in the same
order (prismatic loops add and remove atoms on the host), --fp32 within 1e-4 A.
The driver exists where the reference tree was present at build time; the
test is skipped elsewhere."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXEC = os.path.join(ROOT, "oracle", "_ref", "exec_b200")


def _run(tmp_path, name, yaml, *flags):
    d = tmp_path / name
    d.mkdir()
    r = subprocess.run([EXEC, *flags, os.path.join(ROOT, "tests", "data", yaml)], cwd=d, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = [f for f in os.listdir(d) if f.endswith(".xyz")]
    assert len(out) == 1
    lines = (d / out[0]).read_text().splitlines()
    species = [l.split()[0] for l in lines[2:]]
    pos = np.array([[float(v) for v in l.split()[1:4]] for l in lines[2:]])
    return r.stdout, int(lines[0]), lines[1], species, pos


@pytest.mark.skipif(not os.path.exists(EXEC), reason="reference driver not built (no reference tree at build time)")
@pytest.mark.parametrize("yaml", ["quadrupole_small.yaml", "prismatic_small.yaml"])
def test_reference_driver_on_the_b200_backend(tmp_path, yaml):
    out_cpu, n_cpu, head_cpu, sp_cpu, pos_cpu = _run(tmp_path, "cpu", yaml, "--cpu")
    out_gpu, n_gpu, head_gpu, sp_gpu, pos_gpu = _run(tmp_path, "gpu", yaml)
    assert "--- GPU:" in out_gpu and "--- CPU:" in out_cpu
    assert n_gpu == n_cpu and head_gpu == head_cpu and sp_gpu == sp_cpu
    assert np.abs(pos_gpu - pos_cpu).max() <= 2e-8
    _, n32, _, _, pos32 = _run(tmp_path, "gpu32", yaml, "--fp32")
    assert n32 == n_cpu and np.abs(pos32 - pos_cpu).max() <= 1e-4
