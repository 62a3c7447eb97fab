"""The C ABI library: it loads, exports every entry point include/lbmgpu.h declares, and
rejects bad descriptors before touching CUDA.  No kernel runs here (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import lbmgpu
from oracle import cases, refsc, sc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lbmgpu.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(lbmgpu_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = lbmgpu.lib()
    names = declared_functions()
    assert len(names) >= 17
    for name in names:
        assert hasattr(L, name), f"{name} declared in lbmgpu.h but not exported"
    assert set(names) == set(lbmgpu.EXPORTS)


def test_exports_are_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", lbmgpu.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for name in declared_functions():
        assert name in syms


def test_bad_descriptors_rejected_without_cuda():
    L = lbmgpu.lib()
    h = ctypes.c_void_p()
    d = lbmgpu.Desc()
    d.abi_version = 999
    assert L.lbmgpu_create(ctypes.byref(d), ctypes.byref(h)) == -7
    assert L.lbmgpu_create(None, ctypes.byref(h)) == -1
    d.abi_version = lbmgpu.ABI_VERSION
    d.Nx = d.Ny = d.Nz = 2
    assert L.lbmgpu_create(ctypes.byref(d), ctypes.byref(h)) == -1
    for fn in ("lbmgpu_destroy", "lbmgpu_init", "lbmgpu_collide", "lbmgpu_streaming", "lbmgpu_tms_bc",
               "lbmgpu_calculate_moment", "lbmgpu_synchronize"):
        assert getattr(L, fn)(None) == -1
    assert lbmgpu.error_string(-4).startswith("phase")


def test_mixture_layout_matches_reference_class():
    assert lbmgpu.MIXTURE_SC == cases.MIXTURE_SC
    assert lbmgpu.MIXTURE_SC.itemsize == sc.lib().orc_sc_sizeof()
    if refsc.available():
        lay = refsc.layout()
        assert lay["size"] == lbmgpu.MIXTURE_SC.itemsize
        for k, v in lay.items():
            if k != "size":
                assert lbmgpu.MIXTURE_SC.fields[k][1] == v, k


def test_device_velocity_set_matches_reference(tmp_path):
    """The packed direction table of csrc/d3q27.cuh, compiled for the host, against the
    reference's cx/cy/cz/opposite arrays (src/headers/lbm.hpp:49-53)."""
    src = tmp_path / "dirs.cpp"
    src.write_text('#include "d3q27.cuh"\n#include <cstdio>\nint main(){for(int l=0;l<27;++l)'
                   'std::printf("%d %d %d %d\\n",lbm::cx(l),lbm::cy(l),lbm::cz(l),lbm::opp(l));}\n')
    exe = tmp_path / "dirs"
    csrc = os.path.join(ROOT, "lattice-boltzmann-method_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-D__host__=", "-D__device__=", "-D__forceinline__=inline", "-I", csrc,
                    str(src), "-o", str(exe)], check=True)
    rows = np.array([list(map(int, l.split())) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                                      check=True).stdout.split("\n") if l])
    cx = [0, +1, -1, 0, 0, 0, 0, +1, -1, +1, -1, 0, 0, +1, -1, +1, -1, 0, 0, +1, -1, +1, -1, +1, -1, -1, +1]
    cy = [0, 0, 0, +1, -1, 0, 0, +1, -1, 0, 0, +1, -1, -1, +1, 0, 0, +1, -1, +1, -1, +1, -1, -1, +1, +1, -1]
    cz = [0, 0, 0, 0, 0, +1, -1, 0, 0, +1, -1, +1, -1, 0, 0, -1, +1, -1, +1, +1, -1, -1, +1, +1, -1, +1, -1]
    opposite = [0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25]
    np.testing.assert_array_equal(rows[:, 0], cx)
    np.testing.assert_array_equal(rows[:, 1], cy)
    np.testing.assert_array_equal(rows[:, 2], cz)
    np.testing.assert_array_equal(rows[:, 3], opposite)
