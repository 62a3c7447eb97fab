"""Restart and VTK output from the device state through the C ABI, against the reference's
own writers and reader (oracle/_ref/libref_mc*.so: write_restart / read_restart,
src/restart_file.cpp:274-440, and OutputVTK, src/output.cpp:9-210):
  * the restart file lbmgpu_write_restart writes is the file the reference's write_restart
    writes from the same state (the device state downloaded into the reference's arrays):
    the same header bytes and every record field equal (the reference's records also carry
    6 uninitialised padding bytes after the cell type), and the reference's read_restart
    reads it back to that state;
  * the VTK file lbmgpu_write_vtk packs on the device is byte for byte the reference's
    OutputVTK file of the same state (its OUTPUT_SI and OUTPUT_MASSFRAC build);
  * a restart the reference writes after 5 steps, read by lbmgpu_read_restart and continued
    5 steps on the GPU, matches the reference continuing from the same point (1e-12; the
    boundary case within the reference's own drift at those steps).
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


def read_restart_file(path, ns):
    """(header bytes, mixture records, species records) of a multicomponent restart file in
    the reference's layout; records as the structured arrays the fields are compared on (the
    reference's records carry uninitialised padding bytes after the cell type)."""
    raw = open(path, "rb").read()
    p = 8 * 4 + 8
    for _ in range(ns):
        p += 8 + int(np.frombuffer(raw[p:p + 8], np.uint64)[0])
    p += 8
    rec = np.dtype([("m", W.MIXTURE_MC)] + [(f"s{a}", W.SPECIES) for a in range(ns)])
    body = np.frombuffer(raw[p:], dtype=rec)
    return raw[:p], body["m"], [body[f"s{a}"] for a in range(ns)]


def same_records(a, b):
    return all(np.array_equal(a[f], b[f]) for f in a.dtype.names)


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
    h1, m1, s1 = read_restart_file(ours_rst, len(sp))
    h2, m2, s2 = read_restart_file(tmp_path / "restart000005.dat", len(sp))
    assert h1 == h2 and len(m1) == mix.size
    assert same_records(m1, m2) and all(same_records(x, y) for x, y in zip(s1, s2))
    assert open(ours_vtk, "rb").read() == open(tmp_path / "field000005.vtr", "rb").read()
    # and the reference reads our file back to the same state
    back = refmc.RefMC.from_restart(ours_rst, m, W.FLAME_UNITS, W.MIXTURE_MC, W.SPECIES, reaction=reaction)
    assert same_records(back.cells, c)
    for a in range(len(s)):
        assert same_records(back.species[a], s[a])
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
    # the channel's boundary cells: the reference's own sensitivity to last-bit differences
    # (its two builds drift 5e-7 apart between steps 5 and 10 of this case)
    tol = 1e-12 if name == "mix8" else 2e-6
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
