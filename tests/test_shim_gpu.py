"""The C++ shim as the reference driver would use it: a C++ program compiled
against include/backend.hpp and linked with libdisco_backend.so calls
gpuAvailable / printGpuInfo / gpuLineFp64 / kroupaGPU (Code/backend.hpp:57-62)
with std::vector<LoopData> and AtomArrays; its displacements match the oracle
at the reference's fixed nu = 0.35 and images +-1 (FP64 within 1e-9 A, --fp32
within 2e-5 A), and loopSec has one positive entry per loop."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from disco_b200 import _capi as C
from disco_b200 import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _driver(tmp_path):
    cxx = os.environ.get("DISCO_CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "shim_driver"
    subprocess.run([cxx, "-std=c++14", "-O2", "-DWITH_CUDA", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "shim_driver.cpp"), "-L", C.LIB_DIR, "-ldisco_backend",
                    "-ldisco_b200", f"-Wl,-rpath,{C.LIB_DIR}", "-o", str(exe)], check=True)
    return exe


def _write(path, w, fp32):
    with open(path, "wb") as f:
        np.array([w.n, len(w.loops)], dtype=np.int64).tofile(f)
        np.array(w.box, dtype=np.float64).tofile(f)
        np.array([1 if fp32 else 0, 0], dtype=np.int32).tofile(f)
        for a in (w.x, w.y, w.z):
            np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        for lp in w.loops:
            pts = (lp.vx, lp.vy, lp.vz) if lp.line else (lp.x, lp.y, lp.z)
            np.array([1 if lp.line else 0, len(pts[0])], dtype=np.int32).tofile(f)
            p = lp.phys
            np.array([p.bx, p.by, p.bz, p.mx, p.my, p.mz, p.nx, p.ny, p.nz, p.dS, lp.cx, lp.cy, lp.cz],
                     dtype=np.float64).tofile(f)
            for a in pts:
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)


@pytest.mark.parametrize("kind,fp32,tol", [("line", False, 1e-9), ("line", True, 2e-5),
                                           ("loopons", False, 1e-9)])
def test_reference_driver_through_the_shim(tmp_path, kind, fp32, tol):
    if kind == "line":
        w = W.quadrupole(cells=10)
    else:
        w = W.bcc_prismatic(cells=14, rmin=6.0, rmax=12.0, n_inter=2, n_vac=2)
    exe = _driver(tmp_path)
    _write(tmp_path / "in.bin", w, fp32)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    assert "--- GPU:" in r.stdout
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    n, nl = w.n, len(w.loops)
    u = out[:3 * n].reshape(3, n)
    ref = np.stack(O.displace(w.x, w.y, w.z, w.loops, w.box, images=1, nu=0.35))
    assert np.abs(u - ref).max() <= tol
    assert out[3 * n] > 0.0
    assert (out[3 * n + 1:3 * n + 1 + nl] > 0.0).all()
