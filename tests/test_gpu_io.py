"""Restart and VTK output from the device state through the C ABI, against the reference's
own writers and reader (oracle/_ref/libref_mc*.so: write_restart / read_restart,
src/restart_file.cpp:274-440, and OutputVTK, src/output.cpp:9-210):
  * the restart file lbmgpu_write_restart writes is byte for byte the file the reference's
    write_restart writes from the same state (the device state downloaded into the
    reference's arrays), and the reference's read_restart reads it back to that state;
  * the VTK file lbmgpu_write_vtk packs on the device is byte for byte the reference's
    OutputVTK file of the same state (its OUTPUT_SI and OUTPUT_MASSFRAC build);
  * a restart the reference writes after 5 steps, read by lbmgpu_read_restart and continued
    5 steps on the GPU, matches the reference continuing from the same point (1e-12).
Cases: the 8^3 periodic mixing layer and the reacting 10x6x4 channel with characteristic
outflow and TMS walls (FP64); the write paths also in the FP32 storage mode."""
import os

import numpy as np
import pytest

import lbmgpu
import mech
import workloads as W
from mc_common import rel
from oracle import refmc

pytestmark = pytest.mark.gpu


def case(name):
    m = mech.h2_air_9()
    if name == "mix8":
        return m, *W.mixing_layer_mc(m, N=8), False
    return m, *W.flame_channel_mc(m, NX=10, NY=6, NZ=4), True


def gpu_state(m, mix, sp, reaction, steps, precision=lbmgpu.FP64):
    lat = lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                         chem=lbmgpu.CHEM_REF_EXPLICIT if reaction else lbmgpu.CHEM_OFF, precision=precision)
    lat.upload(mix, sp)
    lat.init()
    lat.step(steps)
    assert lat.synchronize() == 0
    return lat


def reference_from(m, c, s, reaction):
    N3 = [x - 2 for x in c.shape]
    ref = refmc.RefMC(*N3, m, W.FLAME_UNITS, W.MIXTURE_MC, W.SPECIES, reaction=reaction)
    ref.cells[...] = c
    for a in range(len(s)):
        ref.species[a][...] = s[a]
    return ref


def in_dir(path, fn):
    cwd = os.getcwd()
    os.chdir(path)
    try:
        return fn()
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("name,precision", [("mix8", lbmgpu.FP64), ("chan", lbmgpu.FP64), ("chan", lbmgpu.FP32)])
def test_restart_and_vtk_written_from_the_device_equal_the_reference_writers(name, precision, tmp_path):
    m, mix, sp, reaction = case(name)
    lat = gpu_state(m, mix, sp, reaction, 5, precision)
    info = lbmgpu.RestartInfo(dx=1, dy=1, dz=1, step=5, Ra=0.0, permeability=999999.0)  # the LBM defaults
    ours_rst = str(tmp_path / "ours.dat")
    ours_vtk = str(tmp_path / "ours.vtr")
    lat.write_restart(ours_rst, info)
    lat.write_vtk(ours_vtk, dx=1, flags=lbmgpu.VTK_SI | lbmgpu.VTK_MASSFRAC)
    # the same state in the reference's arrays (the download sets every field the
    # reference's writers read; the arrays start as zeros with the cell types)
    c = np.zeros_like(mix)
    c["type"] = mix["type"]
    s = [np.zeros_like(a) for a in sp]
    lat.download(c, s)
    lat.close()
    ref = reference_from(m, c, s, reaction)
    in_dir(tmp_path, lambda: (ref.write_restart(5), ref.output_vtk(5)))
    ref.close()
    assert open(ours_rst, "rb").read() == open(tmp_path / "restart000005.dat", "rb").read()
    assert open(ours_vtk, "rb").read() == open(tmp_path / "field000005.vtr", "rb").read()
    # and the reference reads our file back to the same state
    back = refmc.RefMC.from_restart(ours_rst, m, W.FLAME_UNITS, W.MIXTURE_MC, W.SPECIES, reaction=reaction)
    assert back.cells.tobytes() == c.tobytes()
    for a in range(len(s)):
        assert back.species[a].tobytes() == s[a].tobytes()
    back.close()


@pytest.mark.parametrize("name", ["mix8", "chan"])
def test_reference_restart_read_and_continued_on_the_gpu(name, tmp_path):
    m, mix, sp, reaction = case(name)
    ref = reference_from(m, mix, sp, reaction)
    ref.init()
    ref.loop(5)
    in_dir(tmp_path, lambda: ref.write_restart(5))
    ref.loop(5)
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_REF_EXPLICIT if reaction else lbmgpu.CHEM_OFF) as lat:
        info = lat.read_restart(str(tmp_path / "restart000005.dat"))
        assert (info.step, info.dx, info.permeability) == (5, 1, 999999.0)
        lat.step(5)
        assert lat.synchronize() == 0
        c = mix.copy()
        s = [a.copy() for a in sp]
        lat.download(c, s)
    fl = mix["type"] == W.TYPE_F
    tol = 1e-12 if name == "mix8" else 1e-9  # the channel's boundary cells: the reference's FMA sensitivity
    vs = max(np.abs(ref.cells[k][fl]).max() for k in "uvw")
    for k in ("rho", "u", "v", "w", "temp", "p", "rhoe"):
        assert rel(c[k][fl], ref.cells[k][fl], vs if k in "uvw" else None) < tol, k
    for a in range(len(sp)):
        assert rel(s[a]["rho"][fl], ref.species[a]["rho"][fl]) < tol, a
    ref.close()


def test_read_restart_rejects_a_mismatched_lattice(tmp_path):
    m, mix, sp, reaction = case("mix8")
    lat = gpu_state(m, mix, sp, reaction, 1)
    path = str(tmp_path / "r.dat")
    lat.write_restart(path, lbmgpu.RestartInfo(dx=1, dy=1, dz=1, step=1, Ra=0.0, permeability=1.0))
    lat.close()
    m2, mix2, sp2, _ = case("chan")
    with lbmgpu.Lattice(*mix2.shape, mech=m2, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES,
                        dx_dt=W.FLAME_UNITS) as other:
        with pytest.raises(lbmgpu.LbmGpuError):
            other.read_restart(path)
