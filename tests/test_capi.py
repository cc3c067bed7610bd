"""The C-ABI boundary without a GPU: the libraries load, export every symbol
their headers declare, and reject bad arguments with the documented codes."""
import ctypes
import os
import re

import numpy as np
import pytest

from disco_b200 import _capi as C
from disco_b200 import backend as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(disco_(?:b200|geom)_[a-z0-9_]+)\s*\(", src)))


@pytest.mark.parametrize("header,path", [("disco_b200.h", C.CUDA_LIB_PATH),
                                         ("disco_geometry.h", C.GEOM_LIB_PATH)])
def test_library_exports_every_declared_symbol(header, path):
    names = _declared(header)
    assert len(names) >= 10
    lib = ctypes.CDLL(path)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_shim_exports_reference_backend_interface():
    """libdisco_backend.so defines the four GPU functions of Code/backend.hpp:57-62."""
    out = os.popen(f"nm -D --defined-only {C.SHIM_LIB_PATH}").read()
    for sym in ("_Z12gpuAvailablev", "_Z12printGpuInfov", "_Z11gpuLineFp64v",
                "_Z9kroupaGPURK10AtomArraysRKSt6vectorI8LoopDataSaIS3_EEdddRK10GpuOptionsR13BackendTiming"):
        assert sym in out, sym


def test_options_default_are_the_references_fixed_values():
    o = B.options()
    assert o.images == 1 and o.nu == 0.35 and o.precision == C.DISCO_FP64
    lib = C.cuda_lib()
    d = C.DiscoOptions()
    lib.disco_b200_options_default(ctypes.byref(d))
    assert d.chunk_pairs == -1.0 and d.image_split == 0


def test_strerror_covers_every_code():
    lib = C.cuda_lib()
    for code in range(8):
        assert lib.disco_b200_strerror(code).decode() != "unknown status"
    assert lib.disco_b200_line_fp64() == 1


def test_bad_arguments_are_rejected():
    lib = C.cuda_lib()
    box = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    h = ctypes.c_void_p()
    # null plan out-pointer
    assert lib.disco_b200_plan_create(None, 0, box, None, 0, None) == C.DISCO_EINVAL
    # negative box
    bad = (ctypes.c_double * 3)(1.0, -1.0, 1.0)
    assert lib.disco_b200_plan_create(None, 0, bad, None, 0, ctypes.byref(h)) == C.DISCO_EINVAL
    # image range and nu out of range
    o = B.options(images=9)
    assert lib.disco_b200_plan_create(None, 0, box, ctypes.byref(o), 0, ctypes.byref(h)) == C.DISCO_EINVAL
    o = B.options(nu=0.5)
    assert lib.disco_b200_plan_create(None, 0, box, ctypes.byref(o), 0, ctypes.byref(h)) == C.DISCO_EINVAL
    o = B.options(image_split=3)
    assert lib.disco_b200_plan_create(None, 0, box, ctypes.byref(o), 0, ctypes.byref(h)) == C.DISCO_EINVAL
    assert b"image_split" in lib.disco_b200_last_error()
    # null atoms
    assert lib.disco_b200_displace(None, None, 0, box, None, None) == C.DISCO_EINVAL


@pytest.mark.skipif(B.gpu_available(), reason="a GPU is present")
def test_no_device_reports_enodev():
    """Without a GPU the product path fails loudly: no CPU fallback."""
    assert not B.gpu_available()
    a = B.AtomArrays.zeros_like_positions(np.zeros(3), np.zeros(3), np.zeros(3))
    with pytest.raises(C.DiscoError) as e:
        B.kroupa_gpu(a, [], 10.0, 10.0, 10.0)
    assert e.value.status == C.DISCO_ENODEV
    buf = ctypes.create_string_buffer(64)
    assert C.cuda_lib().disco_b200_device_info(buf, 64) == C.DISCO_ENODEV


def test_ctypes_structures_match_the_header(tmp_path):
    """Every structure of include/disco_b200.h has the size and field offsets of
    its ctypes mirror (a C program compiled against the header prints them)."""
    import ctypes
    import shutil
    import subprocess
    from disco_b200 import _capi as C
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    pairs = {"disco_atoms": C.DiscoAtoms, "disco_loop_phys": C.DiscoLoopPhys, "disco_loop": C.DiscoLoop,
             "disco_options": C.DiscoOptions, "disco_sample": C.DiscoSample, "disco_timing": C.DiscoTiming,
             "disco_plan_stats": C.DiscoPlanStats, "disco_slab_loop": C.DiscoSlabLoop,
             "disco_slab_info": C.DiscoSlabInfo, "disco_copy": C.DiscoCopy, "disco_far_norm": C.DiscoFarNorm,
             "disco_learned_options": C.DiscoLearnedOptions, "disco_learned_report": C.DiscoLearnedReport}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "disco_b200.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
