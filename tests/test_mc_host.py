"""The device's multicomponent per-cell functions (csrc/mc_cell.cuh), built for the host,
against the reference's own multicomponent solver (fixtures from oracle/_ref/libref_mc*.so
on the Cantera-API shim).  Same inputs, FP64, tolerance 1e-12 relative; the reacting cases
with the H2/air mechanism (9 species) and with the reference's two-step CH4 and C3H8
mechanisms (6 species, fractional reaction orders)."""
import os

import numpy as np
import pytest

from mc_common import GOLDEN, NS, SP0, build_host_lib, case, digest, host_run, rel


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    return build_host_lib(tmp_path_factory.mktemp("mchost"))


@pytest.mark.parametrize("fixture", ["mc_mix8.npz", "mc_react8.npz", "mc_ch4_react8.npz", "mc_c3h8_react8.npz"])
def test_host_cells_match_reference(hostlib, fixture):
    m, mix, sp, reaction, cps = case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture))
    assert digest(mix, sp) == str(gold["input_sha256"])
    fl = (mix["type"] == 0).reshape(-1)
    for cp in cps:
        R, st = host_run(hostlib, m, mix, sp, reaction, cp)
        assert st == 0
        assert rel(R[0][fl], gold[f"rho_{cp}"].reshape(-1)[fl]) < 1e-12
        vs = max(np.abs(gold[f"{k}_{cp}"].reshape(-1)[fl]).max() for k in "uvw")
        for q, k in ((1, "u"), (2, "v"), (3, "w")):
            assert rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl], vs) < 1e-12, k
        assert rel(R[4][fl], gold[f"temp_{cp}"].reshape(-1)[fl]) < 1e-12
        assert rel(R[5][fl], gold[f"p_{cp}"].reshape(-1)[fl]) < 1e-12
        assert rel(R[6][fl], gold[f"rhoe_{cp}"].reshape(-1)[fl]) < 1e-12
        for a in range(len(sp)):
            assert rel(R[SP0 + 8 * a][fl], gold[f"sp_rho_{cp}"][a].reshape(-1)[fl]) < 1e-12, a
            assert rel(R[SP0 + 8 * a + 4][fl], gold[f"sp_X_{cp}"][a].reshape(-1)[fl]) < 1e-12, a
        if reaction:
            assert rel(R[13][fl], gold[f"HRR_{cp}"].reshape(-1)[fl]) < 1e-10


# FP32 population storage (shifted, records FP64) against the FP64 run of the same
# per-cell functions after 200 steps.  Measured on these fixtures: rho, T, p, rhoe within
# 1e-6 relative, u within 6e-6 of the largest velocity, Y within 3e-7 absolute.
FP32_STEPS = 200
FP32_TOL = {"scalar": 1e-5, "u": 5e-5, "Y": 1e-5}


def fp32_errors(R32, R64, fl):
    err = {}
    for q, k in ((0, "rho"), (4, "temp"), (5, "p"), (6, "rhoe")):
        err[k] = rel(R32[q][fl], R64[q][fl])
    vs = max(np.abs(R64[q][fl]).max() for q in (1, 2, 3))
    err["u"] = max(rel(R32[q][fl], R64[q][fl], vs) for q in (1, 2, 3))
    Y64 = np.array([R64[SP0 + 8 * a][fl] / R64[0][fl] for a in range(NS)])
    Y32 = np.array([R32[SP0 + 8 * a][fl] / R32[0][fl] for a in range(NS)])
    err["Y"] = float(np.abs(Y64 - Y32).max())
    return err


@pytest.mark.parametrize("fixture", ["mc_mix8.npz", "mc_react8.npz"])
def test_host_fp32_storage_within_tolerance(hostlib, fixture):
    m, mix, sp, reaction, _ = case(fixture)
    fl = (mix["type"] == 0).reshape(-1)
    R64, s64 = host_run(hostlib, m, mix, sp, reaction, FP32_STEPS)
    R32, s32 = host_run(hostlib, m, mix, sp, reaction, FP32_STEPS, "fp32", shift=True)
    assert s64 == 0 and s32 == 0
    err = fp32_errors(R32, R64, fl)
    for k, e in err.items():
        assert e < FP32_TOL["u" if k == "u" else ("Y" if k == "Y" else "scalar")], (k, e)
    # and the unshifted storage is no better (the shift is what the mode is for)
    R0, _ = host_run(hostlib, m, mix, sp, reaction, FP32_STEPS, "fp32", shift=False)
    assert fp32_errors(R0, R64, fl)["u"] >= err["u"]


def element_totals(m, R, fl):
    rho_a = np.array([R[SP0 + 8 * a][fl] for a in range(NS)])
    W = np.array([m.W[k] for k in range(NS)])
    E = np.array([[m.elements[k][e] for e in range(3)] for k in range(NS)], float)  # H, O, N
    return ((rho_a / W[:, None]).T @ E).sum(0)


def test_host_rosenbrock_chemistry_tracks_reference_scheme(hostlib):
    """CHEM_ROSENBROCK (ROS2 over the whole step) against the reference's explicit scheme on
    the reacting fixture: at dt = 1 ns both resolve the chemistry, so after 10 steps the
    states agree to the explicit scheme's truncation error, and the stiff integrator adds no
    element drift of its own (the drift of both comes from the species floor of 1e-8)."""
    m, mix, sp, _, _ = case("mc_react8.npz")
    fl = (mix["type"] == 0).reshape(-1)
    R0, _ = host_run(hostlib, m, mix, sp, 0, 0)
    e0 = element_totals(m, R0, fl)
    R1, s1 = host_run(hostlib, m, mix, sp, 1, 10)
    R2, s2 = host_run(hostlib, m, mix, sp, 2, 10)
    assert s1 == 0 and s2 == 0
    assert rel(R2[4][fl], R1[4][fl]) < 1e-5
    for a in range(NS):
        Y1 = R1[SP0 + 8 * a][fl] / R1[0][fl]
        Y2 = R2[SP0 + 8 * a][fl] / R2[0][fl]
        assert np.abs(Y1 - Y2).max() < 1e-6, a
    assert rel(R2[13][fl], R1[13][fl]) < 1e-2
    assert np.abs(R2[13][fl]).max() > 0.0
    d1 = np.abs(element_totals(m, R1, fl) - e0) / e0
    d2 = np.abs(element_totals(m, R2, fl) - e0) / e0
    assert np.all(np.abs(d2 - d1) < 1e-8), (d1, d2)


# Boundary fixtures (characteristic inflow/outflow and TMS walls).  The reference's energy
# collision picks the upwind side of its species-gradient term from the sign of each
# species' diffusion velocity (src/lbm-collision.cpp:282-284); in uniform-composition
# regions that velocity is rounding noise, so last-bit differences (FMA contraction,
# summation order) flip the stencil and the runs drift apart at a rate the reference
# itself sets.  The first steps are compared tightly, step 20 to 1e-4.
BC_TOL = {1: 1e-12, 2: 1e-10, 20: 1e-4}


def bc_case(fixture):
    import workloads as Wk
    m = mech_h2()
    if fixture == "mc_chan.npz":
        mix, sp = Wk.flame_channel_mc(m, NX=10, NY=6, NZ=4)
        return m, mix, sp, 1
    mix, sp = Wk.inflow_layer_mc(m, NX=10, NY=6, NZ=6)
    return m, mix, sp, 0


def mech_h2():
    import mech
    return mech.h2_air_9()


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_host_boundary_cells_match_reference(hostlib, fixture):
    m, mix, sp, reaction = bc_case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture))
    assert digest(mix, sp) == str(gold["input_sha256"])
    fl = (mix["type"] == 0).reshape(-1)
    for cp, tol in BC_TOL.items():
        R, st = host_run(hostlib, m, mix, sp, reaction, cp)
        assert st == 0
        for q, k in ((0, "rho"), (4, "temp"), (5, "p"), (6, "rhoe")):
            assert rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl]) < tol, (k, cp)
        vs = max(np.abs(gold[f"{k}_{cp}"].reshape(-1)[fl]).max() for k in "uvw")
        for q, k in ((1, "u"), (2, "v"), (3, "w")):
            assert rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl], vs) < tol, (k, cp)
        for a in range(NS):
            assert rel(R[SP0 + 8 * a][fl], gold[f"sp_rho_{cp}"][a].reshape(-1)[fl]) < tol, (a, cp)
        if reaction:
            assert rel(R[13][fl], gold[f"HRR_{cp}"].reshape(-1)[fl]) < max(tol, 1e-10), cp


@pytest.fixture(scope="module")
def hostlib_nofma(tmp_path_factory):
    return build_host_lib(tmp_path_factory.mktemp("mchost_nofma"), contract=False)


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_host_boundary_cells_match_reference_without_fma(hostlib_nofma, fixture):
    """The boundary cases with floating-point contraction off on both sides: the per-cell
    functions (host build, -ffp-contract=off) against the reference's own solver built the
    same way (mc_*_nofma.npz) agree to 1e-12 through 20 steps -- the NSCBC outflow, the
    inline LODI inflow, the TMS walls and the reacting cells are the reference's formulas
    operation for operation.  With contraction on, the two sides place their fused
    multiply-adds differently and drift apart exactly as two builds of the reference do
    (next test)."""
    from mc_common import bc_errors
    m, mix, sp, reaction = bc_case(fixture)
    gold = np.load(os.path.join(GOLDEN, fixture.replace(".npz", "_nofma.npz")))
    assert digest(mix, sp) == str(gold["input_sha256"])
    fl = (mix["type"] == 0).reshape(-1)
    for cp in (1, 2, 5, 10, 20):
        R, st = host_run(hostlib_nofma, m, mix, sp, reaction, cp)
        assert st == 0
        e = bc_errors(R, gold, cp, fl, reaction)
        assert max(e.values()) < 1e-12, (cp, e)


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_reference_boundary_drift_bounds_the_tolerance(hostlib, fixture):
    """The reference against itself: its solver built with and without floating-point
    contraction (mc_*.npz vs mc_*_nofma.npz, same inputs) agrees to 1e-14 after 2 steps and
    then drifts apart -- the energy collision's upwind switch on near-zero diffusion
    velocities (src/lbm-collision.cpp:282-284) amplifies last-bit differences -- to 4e-7
    (channel) and 8e-6 (inflow) by step 20.  The host build with contraction drifts from
    the contracted reference by no more than that, and BC_TOL[20] sits above it."""
    from mc_common import bc_errors, fixture_drift
    m, mix, sp, reaction = bc_case(fixture)
    g_fma = np.load(os.path.join(GOLDEN, fixture))
    g_off = np.load(os.path.join(GOLDEN, fixture.replace(".npz", "_nofma.npz")))
    fl = (mix["type"] == 0).reshape(-1)
    assert fixture_drift(g_fma, g_off, 2, fl) < 1e-13
    drift = fixture_drift(g_fma, g_off, 20, fl)
    assert 1e-8 < drift < BC_TOL[20], drift
    R, st = host_run(hostlib, m, mix, sp, reaction, 20)
    assert st == 0
    e = max(bc_errors(R, g_fma, 20, fl, False).values())
    assert e <= 2.0 * drift + 1e-12, (e, drift)


@pytest.mark.parametrize("fixture", ["mc_chan.npz", "mc_inflow.npz"])
def test_host_fp32_storage_with_boundaries(hostlib, fixture):
    """FP32 population storage (incl. the boundary cells' kept populations) against FP64
    after 20 steps of the boundary fixtures.  The FP64 runs themselves drift apart at the
    1e-6 level under last-bit changes here (see BC_TOL), so the bounds are those of the
    boundary parity: 1e-5 relative for rho, T, p, rhoE, 1e-4 of the largest velocity,
    1e-5 absolute for Y."""
    m, mix, sp, reaction = bc_case(fixture)
    fl = (mix["type"] == 0).reshape(-1)
    R64, s64 = host_run(hostlib, m, mix, sp, reaction, 20)
    R32, s32 = host_run(hostlib, m, mix, sp, reaction, 20, "fp32", shift=True)
    assert s64 == 0 and s32 == 0
    err = fp32_errors(R32, R64, fl)
    for k, e in err.items():
        assert e < {"u": 1e-4, "Y": 1e-5}.get(k, 1e-5), (k, e)


def test_surrogate_correction_conserves_elements_exactly(hostlib):
    """sur_conserve (the correction the surrogate's prediction gets before use) with the
    projector sur_projector forms from the mechanism: after it, sum_k E_ek / W_k dY_k = 0
    for H, O, N to rounding; the projector is I - A^T (A A^T)^-1 A over the elements the
    species carry (numpy, to 1e-12); a prediction that already conserves the elements comes
    back unchanged (to rounding)."""
    import ctypes
    import mech
    m = mech.h2_air_9()
    E = np.array([[m.elements[k][e] / m.W[k] for k in range(NS)] for e in range(4)])
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    proj = np.zeros(NS * NS)
    hostlib.sur_projector_host(ctypes.byref(m), P(proj))
    proj = proj.reshape(NS, NS)
    A = E[np.abs(E).sum(1) > 0]
    want = np.eye(NS) - A.T @ np.linalg.solve(A @ A.T, A)
    assert np.abs(proj - want).max() <= 1e-12 * np.abs(want).max()
    rng = np.random.default_rng(17)
    for trial in range(200):
        dY0 = rng.normal(size=NS) * 10.0 ** rng.uniform(-9, -3, NS)
        dY = dY0.copy()
        hostlib.sur_conserve_host(P(np.ascontiguousarray(proj)), P(dY))
        scale = np.abs(E).max(1) * np.abs(dY0).max()
        assert np.all(np.abs(E @ dY) <= 1e-13 * scale + 1e-300), (trial, E @ dY)
    # a conserving prediction is kept
    null = np.linalg.svd(A)[2][A.shape[0]:].T  # basis of element-conserving changes
    dY0 = null @ rng.normal(size=null.shape[1]) * 1e-5
    dY = dY0.copy()
    hostlib.sur_conserve_host(P(np.ascontiguousarray(proj)), P(dY))
    assert np.abs(dY - dY0).max() <= 1e-12 * np.abs(dY0).max()
