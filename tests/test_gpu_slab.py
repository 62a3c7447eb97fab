"""Slab decomposition along x through the C ABI on one GPU: two handles, each holding one
slab of a multicomponent lattice (lbmgpu_set_halo), stepped through the phase calls with
their halo planes exchanged through device buffers (lbmgpu_halo_pack / lbmgpu_halo_unpack,
the host ordering the two handles' streams) -- the schedule the multi-GPU driver runs over
NCCL, here with both slabs on one device and no kernel waiting on another.  In FP64 the
two slabs' cells equal the single-domain run through the same library bit for bit; in the
FP32 storage mode (each slab shifts its populations by its own plane means) within the
FP32 mode's bounds.  Cases: a reacting H2/air mixing layer periodic in x, cut through the
interface, and config 4's turbulent reacting layer (characteristic outflow y faces, stiff
chemistry) at 16^3."""
import numpy as np
import pytest

import lbmgpu
import mech
import workloads as W

pytestmark = pytest.mark.gpu
STEPS = 8


def case(name):
    m = mech.h2_air_9()
    if name == "mixing":
        mix, sp = W.mixing_layer_mc(m, N=16, T_hi=1800.0)
        return m, mix, sp, W.FLAME_UNITS, lbmgpu.CHEM_REF_EXPLICIT, 6
    # 16 cells per energy-containing wavelength, the layer 4 cells wide
    mix, sp = W.turbulent_layer_mc(m, N=16, k0=1.0, width=4.0)
    return m, mix, sp, W.TURB_UNITS, lbmgpu.CHEM_ROSENBROCK, 9


def new(m, mix, units, chem, prec):
    return lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=units, chem=chem,
                          precision=prec)


def single(name, prec):
    m, mix, sp, units, chem, cut = case(name)
    with new(m, mix, units, chem, prec) as lat:
        lat.upload(mix, sp)
        lat.init()
        for _ in range(STEPS):
            lat.collide_species()
            lat.collide()
            lat.streaming()
            lat.tms_bc()
            lat.calculate_moment()
        assert lat.synchronize() == 0
        c, s = mix.copy(), [a.copy() for a in sp]
        lat.download(c, s)
    return c, s


def slabs(name, prec):
    import torch
    m, mix, sp, units, chem, cut = case(name)
    Nx = mix.shape[0]
    parts = [(1, cut - 1), (cut, Nx - 2)]
    lats, views = [], []
    for a, b in parts:
        sl = slice(a - 1, b + 2)
        lm, ls = np.ascontiguousarray(mix[sl]), [np.ascontiguousarray(x[sl]) for x in sp]
        lat = new(m, lm, units, chem, prec)
        lat.set_halo(1, 1, Nx)
        lat.upload(lm, ls)
        lat.init()
        lats.append(lat)
        views.append((lm, ls))
    bufs = {}
    for what in (lbmgpu.HALO_POPULATIONS, lbmgpu.HALO_RECORD):
        nb = lats[0].halo_bytes(what)
        bufs[what] = [[torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(2)] for _ in range(2)]

    def exchange(what):
        # slab r packs face 1 for its upper neighbour and face 0 for its lower one
        for r, lat in enumerate(lats):
            lat.halo_pack(1, what, bufs[what][r][1].data_ptr())
            lat.halo_pack(0, what, bufs[what][r][0].data_ptr())
        for lat in lats:
            lat.synchronize()
        for r, lat in enumerate(lats):
            down, up = (r - 1) % 2, (r + 1) % 2
            lat.halo_unpack(0, what, bufs[what][down][1].data_ptr())
            lat.halo_unpack(1, what, bufs[what][up][0].data_ptr())
        for lat in lats:
            lat.synchronize()

    for _ in range(STEPS):
        for lat in lats:
            lat.collide_species()
            lat.collide()
        exchange(lbmgpu.HALO_POPULATIONS)
        for lat in lats:
            lat.streaming()
            lat.tms_bc()
            lat.calculate_moment()
        exchange(lbmgpu.HALO_RECORD)
    out = []
    for (a, b), lat, (lm, ls) in zip(parts, lats, views):
        assert lat.synchronize() == 0
        lat.download(lm, ls)
        out.append((a, b, lm, ls))
        lat.close()
    return out


FIELDS = ("rho", "u", "v", "w", "temp", "p", "rhoe", "HRR", "g", "gpc")


@pytest.mark.parametrize("name", ["mixing", "turbulent"])
def test_gpu_slabs_equal_the_single_domain_fp64(name):
    c, s = single(name, lbmgpu.FP64)
    for a, b, lm, ls in slabs(name, lbmgpu.FP64):
        fl = lm["type"][1:-1] == W.TYPE_F
        for k in FIELDS:
            assert np.array_equal(lm[k][1:-1][fl], c[k][a:b + 1][fl]), (k, a)
        for q in range(len(s)):
            for k in ("rho", "u", "v", "w", "X", "f", "fpc"):
                assert np.array_equal(ls[q][k][1:-1][fl], s[q][k][a:b + 1][fl]), (q, k, a)


def test_gpu_slabs_fp32_within_fp32_bounds():
    name = "mixing"
    c, s = single(name, lbmgpu.FP64)
    for a, b, lm, ls in slabs(name, lbmgpu.FP32):
        fl = lm["type"][1:-1] == W.TYPE_F
        for k in ("rho", "temp", "p", "rhoe"):
            want = c[k][a:b + 1][fl]
            assert np.max(np.abs(lm[k][1:-1][fl] - want)) / np.max(np.abs(want)) < 1e-5, k
        vs = max(np.max(np.abs(c[k][a:b + 1][fl])) for k in "uvw")
        for k in "uvw":
            assert np.max(np.abs(lm[k][1:-1][fl] - c[k][a:b + 1][fl])) / vs < 1e-4, k
        for q in range(len(s)):
            Y = ls[q]["rho"][1:-1][fl] / lm["rho"][1:-1][fl]
            Yw = s[q]["rho"][a:b + 1][fl] / c["rho"][a:b + 1][fl]
            assert np.max(np.abs(Y - Yw)) < 1e-5, q
