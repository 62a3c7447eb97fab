"""GPU parity of the multicomponent path through the C ABI: the reference's own
multicomponent solver (fixtures from oracle/_ref/libref_mc*.so on the Cantera-API shim)
against liblbmgpu.so on the same seeded inputs.  FP64; tolerance 1e-12 relative for the
fields, populations and species moments (1e-10 for the heat release rate)."""
import os

import numpy as np
import pytest

import lbmgpu
import workloads as W
from mc_common import GOLDEN, NS, case, digest, rel

pytestmark = pytest.mark.gpu


def lattice(m, mix, reaction):
    return lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                          chem=lbmgpu.CHEM_REF_EXPLICIT if reaction else lbmgpu.CHEM_OFF)


def run(m, mix, sp, reaction, cps, phases=False):
    out = {}
    with lattice(m, mix, reaction) as lat:
        lat.upload(mix, sp)
        lat.init()
        done = 0
        for cp in cps:
            for _ in range(cp - done):
                if phases:
                    lat.collide_species()
                    lat.collide()
                    lat.streaming()
                    lat.tms_bc()
                    lat.calculate_moment()
            if not phases:
                lat.step(cp - done)
            done = cp
            assert lat.synchronize() == 0
            c = mix.copy()
            s = [a.copy() for a in sp]
            lat.download(c, s)
            out[cp] = (c, s)
    return out


@pytest.mark.parametrize("fixture,phases", [("mc_mix8.npz", False), ("mc_mix8.npz", True), ("mc_react8.npz", False)])
def test_gpu_mc_matches_reference(fixture, phases):
    m, mix, sp, reaction, cps = case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture))
    assert digest(mix, sp) == str(gold["input_sha256"])
    res = run(m, mix, sp, reaction, cps, phases)
    fl = mix["type"] == 0
    idx = tuple(gold["pop_cells"].T)
    for cp in cps:
        c, s = res[cp]
        vs = max(np.abs(gold[f"{k}_{cp}"][fl]).max() for k in "uvw")
        for k in ("rho", "u", "v", "w", "temp", "p", "rhoe"):
            assert rel(c[k][fl], gold[f"{k}_{cp}"][fl], vs if k in "uvw" else None) < 1e-12, (k, cp)
        if reaction:
            assert rel(c["HRR"][fl], gold[f"HRR_{cp}"][fl]) < 1e-10
        for a in range(NS):
            assert rel(s[a]["rho"][fl], gold[f"sp_rho_{cp}"][a][fl]) < 1e-12
            assert rel(s[a]["X"][fl], gold[f"sp_X_{cp}"][a][fl]) < 1e-12
            assert rel(s[a]["f"][idx], gold[f"sp_f_{cp}"][a]) < 1e-12
            assert rel(s[a]["fpc"][idx], gold[f"sp_fpc_{cp}"][a]) < 1e-12
        assert rel(c["g"][idx], gold[f"g_{cp}"]) < 1e-12
        assert rel(c["p_tensor"][idx], gold[f"p_tensor_{cp}"]) < 1e-12


def test_gpu_mc_rejects_boundary_types_and_orders_phases():
    m, mix, sp, reaction, cps = case("mc_mix8.npz")
    with lattice(m, mix, False) as lat:
        bad = mix.copy()
        bad["type"][0, 3, 3] = W.TYPE_O
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.upload(bad, sp)
        lat.upload(mix, sp)
        lat.init()
        with pytest.raises(lbmgpu.LbmGpuError):
            lat.collide()  # Collide_Species first
        lat.collide_species()
        lat.collide()
        lat.streaming()
        lat.tms_bc()
        lat.calculate_moment()
        assert lat.synchronize() == 0


@pytest.mark.parametrize("fixture", ["mc_mix8.npz", "mc_react8.npz"])
def test_gpu_mc_fp32_storage_within_tolerance(fixture):
    """FP32 population storage on the device against the device's FP64 mode after 200
    steps: rho, T, p, rhoe within 1e-5 relative, u within 5e-5 of the largest velocity,
    every Y_k within 1e-5 absolute."""
    m, mix, sp, reaction, _ = case(fixture)
    res = {}
    for prec in (lbmgpu.FP64, lbmgpu.FP32):
        with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                            chem=lbmgpu.CHEM_REF_EXPLICIT if reaction else lbmgpu.CHEM_OFF, precision=prec) as lat:
            lat.upload(mix, sp)
            lat.init()
            lat.step(200)
            assert lat.synchronize() == 0
            c = mix.copy()
            s = [a.copy() for a in sp]
            lat.download(c, s)
            res[prec] = (c, s)
    (c64, s64), (c32, s32) = res[lbmgpu.FP64], res[lbmgpu.FP32]
    fl = mix["type"] == 0
    for k in ("rho", "temp", "p", "rhoe"):
        assert rel(c32[k][fl], c64[k][fl]) < 1e-5, k
    vs = max(np.abs(c64[k][fl]).max() for k in "uvw")
    for k in "uvw":
        assert rel(c32[k][fl], c64[k][fl], vs) < 5e-5, k
    for a in range(NS):
        Y64 = s64[a]["rho"][fl] / c64["rho"][fl]
        Y32 = s32[a]["rho"][fl] / c32["rho"][fl]
        assert np.abs(Y64 - Y32).max() < 1e-5, a


def test_gpu_mc_rosenbrock_matches_host_build(tmp_path):
    """CHEM_ROSENBROCK on the device against the same per-cell functions built for the host
    (FP64, 10 steps of the reacting fixture); the adaptive sub-step control is the only
    place where rounding differences could change a decision, hence 1e-7."""
    from mc_common import SP0, build_host_lib, host_run
    m, mix, sp, _, _ = case("mc_react8.npz")
    R, st = host_run(build_host_lib(tmp_path), m, mix, sp, lbmgpu.CHEM_ROSENBROCK, 10)
    assert st == 0
    with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                        chem=lbmgpu.CHEM_ROSENBROCK) as lat:
        lat.upload(mix, sp)
        lat.init()
        lat.step(10)
        assert lat.synchronize() == 0
        c = mix.copy()
        s = [a.copy() for a in sp]
        lat.download(c, s)
    fl = mix["type"] == 0
    f1 = fl.reshape(-1)
    for q, k in ((0, "rho"), (4, "temp"), (5, "p"), (6, "rhoe"), (13, "HRR")):
        assert rel(c[k][fl], R[q][f1]) < 1e-7, k
    for a in range(NS):
        assert rel(s[a]["rho"][fl], R[SP0 + 8 * a][f1]) < 1e-7, a


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_gpu_mc_boundaries_match_reference(fixture):
    """Characteristic outflow (NSCBC) / inflow (inline LODI) ghosts and TMS solid walls
    through the C ABI against the reference on the Cantera-API shim: 1e-12 after one step
    (fields and the streamed populations of the sampled cells, half of them boundary
    cells), 1e-10 after two, 1e-4 after twenty -- the reference's upwind choice on the sign
    of near-zero diffusion velocities makes later steps depend on last-bit rounding."""
    from test_mc_host import BC_TOL, bc_case
    m, mix, sp, reaction = bc_case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture))
    assert digest(mix, sp) == str(gold["input_sha256"])
    res = run(m, mix, sp, reaction, list(BC_TOL))
    fl = mix["type"] == 0
    idx = tuple(gold["pop_cells"].T)
    for cp, tol in BC_TOL.items():
        c, s = res[cp]
        vs = max(np.abs(gold[f"{k}_{cp}"][fl]).max() for k in "uvw")
        for k in ("rho", "u", "v", "w", "temp", "p", "rhoe"):
            assert rel(c[k][fl], gold[f"{k}_{cp}"][fl], vs if k in "uvw" else None) < tol, (k, cp)
        for a in range(NS):
            assert rel(s[a]["rho"][fl], gold[f"sp_rho_{cp}"][a][fl]) < tol, (a, cp)
        if cp == 1:
            for a in range(NS):
                assert rel(s[a]["f"][idx], gold[f"sp_f_{cp}"][a]) < tol
                assert rel(s[a]["fpc"][idx], gold[f"sp_fpc_{cp}"][a]) < tol
            assert rel(c["g"][idx], gold[f"g_{cp}"]) < tol


def test_gpu_mc_rejects_noncharacteristic_open_types():
    """TYPE_O / TYPE_I (order-dependent in the reference) are refused at upload."""
    from test_mc_host import bc_case
    m, mix, sp, reaction = bc_case("mc_inflow.npz")
    for t in (W.TYPE_O, W.TYPE_I):
        bad = mix.copy()
        bad["type"][0] = t
        with lattice(m, bad, False) as lat:
            with pytest.raises(lbmgpu.LbmGpuError):
                lat.upload(bad, sp)


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_gpu_mc_fp32_storage_with_boundaries(fixture):
    """FP32 population storage with characteristic inflow/outflow and TMS walls (the
    boundary cells' kept populations are stored in float too) against the FP64 mode after
    20 steps: 1e-5 relative for rho, T, p, rhoE, 1e-4 of the largest velocity, 1e-5
    absolute for every Y_k."""
    from test_mc_host import bc_case
    m, mix, sp, reaction = bc_case(fixture)
    res = {}
    for prec in (lbmgpu.FP64, lbmgpu.FP32):
        with lbmgpu.Lattice(*mix.shape, mech=m, dtype=W.MIXTURE_MC, species_dtype=W.SPECIES, dx_dt=W.FLAME_UNITS,
                            chem=lbmgpu.CHEM_REF_EXPLICIT if reaction else lbmgpu.CHEM_OFF, precision=prec) as lat:
            lat.upload(mix, sp)
            lat.init()
            lat.step(20)
            assert lat.synchronize() == 0
            c = mix.copy()
            s = [a.copy() for a in sp]
            lat.download(c, s)
            res[prec] = (c, s)
    (c64, s64), (c32, s32) = res[lbmgpu.FP64], res[lbmgpu.FP32]
    fl = mix["type"] == 0
    for k in ("rho", "temp", "p", "rhoe"):
        assert rel(c32[k][fl], c64[k][fl]) < 1e-5, k
    vs = max(np.abs(c64[k][fl]).max() for k in "uvw")
    for k in "uvw":
        assert rel(c32[k][fl], c64[k][fl], vs) < 1e-4, k
    for a in range(NS):
        assert np.abs(s64[a]["rho"][fl] / c64["rho"][fl] - s32[a]["rho"][fl] / c32["rho"][fl]).max() < 1e-5, a
