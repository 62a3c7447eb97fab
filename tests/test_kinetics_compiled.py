"""The H2/air mechanism compiled to straight-line code (gen_kinetics.py ->
csrc/kinetics_h2_air_9.cuh, the kinetics the device's stiff chemistry runs when a handle's
mechanism is that one) against the table-driven kinetics of gas.cuh, host builds without
contraction of multiply-adds:
  * the reactor right-hand side (net production with Arrhenius, third-body, Troe fall-off and
    equilibrium reverse rates; dT/dt) equals rate_factors + reactor_rhs_k bit for bit on
    states on both sides of the NASA polynomials' switch temperature, lean to rich, trace
    radicals to equilibrium products;
  * the analytic Jacobian (jac: the species and temperature columns) equals the Jacobian of the
    tables' right-hand side by Richardson-extrapolated central differences, to the differences'
    own accuracy (the best of four step sizes, 1e-6 of the row's largest entry);
  * one ROS2 advance (the device integrator's compile-time-sized form over the compiled
    kinetics and their analytic Jacobian) takes the same
    sub-steps as the host integrator over the tables (finite differences throughout) and
    lands within 1e-10 in every mass fraction and 1e-9 relative in T, five orders inside the
    integrator's own tolerance (rtol 1e-5) -- ROS2 is a W-method, the Jacobian's
    approximation moves rounding only, which grows with the sub-steps of the longest advances
    (~1e-12 after 200) -- on the states of the turbulent
    reacting layer's mixing and ignition, over its lattice time step and over longer steps
    that take many sub-steps;
  * `matches` accepts the mechanism it was generated from and rejects one with any quantity
    the kinetics read changed by one unit in the last place;
  * the committed header is what the generator writes for the committed mechanism."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import mech
from mc_common import CSRC, ROOT

D = ctypes.c_double
DP = ctypes.POINTER(ctypes.c_double)
PKG = os.path.join(ROOT, "lattice-boltzmann-method_b200")


@pytest.fixture(scope="module")
def kh(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("kin") / "libkh.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I", CSRC,
                    os.path.join(ROOT, "tests", "host", "kin_host.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    L.kh_tables.restype = vp
    L.kh_tables.argtypes = [vp]
    L.kh_free.argtypes = [vp]
    L.kh_matches.argtypes = [vp]
    for f in ("kh_rhs_tables", "kh_rhs_dense"):
        getattr(L, f).argtypes = [vp, D, DP, DP]
    L.kh_rhs_compiled.argtypes = [D, DP, DP]
    for f in ("kh_ros2_tables", "kh_ros2_dense"):
        getattr(L, f).argtypes = [vp, D, DP, DP, D]
    L.kh_ros2_compiled.argtypes = [D, DP, DP, D]
    L.kh_jac_compiled.argtypes = [D, DP, DP, DP]
    L.kh_sys_full.argtypes = [ctypes.POINTER(ctypes.c_int)]
    return L


def p(a):
    return a.ctypes.data_as(DP)


def states(m, n, seed=7):
    """n reactor states (rho, Y_0..Y_8, T): temperatures 300-2800 K (both NASA ranges), fuel
    fractions from pure air to pure H2, radicals from 1e-12 to 1e-2, water and HO2 / H2O2
    as in burnt and igniting gas, at 0.5-5 atm."""
    rng = np.random.default_rng(seed)
    names = m.species_names()
    W = np.array([m.W[k] for k in range(m.n_species)])
    out = []
    for i in range(n):
        X = np.zeros(m.n_species)
        phi = rng.uniform(0.0, 1.0)
        X[names.index("H2")] = phi
        X[names.index("O2")] = (1 - phi) * 0.21
        X[names.index("N2")] = (1 - phi) * 0.79
        for s_ in ("H", "O", "OH", "HO2", "H2O2"):
            X[names.index(s_)] = 10 ** rng.uniform(-12, -2)
        X[names.index("H2O")] = rng.uniform(0, 0.3) * (i % 3 != 0)
        X /= X.sum()
        Y = X * W / (X * W).sum()
        T = rng.uniform(300.0, 2800.0) if i % 7 else 1000.0 - 1e-9 * (i % 2)
        P = 101325.0 * rng.uniform(0.5, 5.0)
        rho = P * (X * W).sum() / (8314.46261815324 * T)
        out.append((rho, np.concatenate([Y, [T]])))
    return out


def layer_states(kh, t, m):
    """The states the turbulent reacting layer's cells go through: H2-laden air at 1500 K
    blended with air at 300 K (mixture fraction s, the other species at mole fraction 1e-6,
    1 atm), and each blend's constant-volume evolution sampled after advances of 1 ns growing to
    10 us (up to an advance that reaches the integrator's sub-step cap)."""
    names = m.species_names()
    W = np.array([m.W[k] for k in range(m.n_species)])
    out = []
    for s in np.linspace(0.0, 1.0, 9):
        Y = np.zeros(m.n_species)
        Y[names.index("H2")] = 0.03 * s
        Y[names.index("O2")] = 0.233 * (1 - Y[names.index("H2")])
        Y[names.index("N2")] = 0.767 * (1 - Y[names.index("H2")])
        X = Y / W
        X /= X.sum()
        for a, nm in enumerate(names):
            if nm not in ("H2", "O2", "N2"):
                X[a] = 1e-6
        X[names.index("H2")] = max(X[names.index("H2")], 1e-6)
        X /= X.sum()
        Y = X * W / (X * W).sum()
        T = np.array([300.0 + 1200.0 * s])
        rho = 101325.0 * (X * W).sum() / (8314.46261815324 * T[0])
        out.append((rho, np.concatenate([Y, T])))
        for dt in [1e-9] * 5 + [1e-8] * 5 + [1e-7] * 5 + [1e-6] * 10 + [1e-5] * 10:
            if kh.kh_ros2_tables(t, rho, p(Y), p(T), dt) < 0:
                break  # the sub-step cap: the trajectory ends here
            out.append((rho, np.concatenate([Y, T])))
    return out


def test_compiled_rhs_equals_the_tables_bit_for_bit(kh):
    m = mech.h2_air_9()
    t = kh.kh_tables(ctypes.addressof(m))
    try:
        for rho, y in states(m, 400):
            Ft = np.zeros(10)
            Fc = np.zeros(10)
            Fd = np.zeros(10)
            kh.kh_rhs_tables(t, rho, p(y), p(Ft))
            kh.kh_rhs_compiled(rho, p(y), p(Fc))
            kh.kh_rhs_dense(t, rho, p(y), p(Fd))
            assert np.array_equal(Ft, Fc), (y, Ft - Fc)
            # the dense table form sums in species order: rounding apart
            assert np.all(np.abs(Fd - Ft) <= 1e-9 * np.abs(Ft).max() + 1e-300)
    finally:
        kh.kh_free(t)


def test_analytic_jacobian_matches_finite_differences(kh):
    """Over the unknowns of the iteration system (every component but the inert N2, whose
    right-hand side is zero everywhere) the analytic Jacobian is the tables' finite
    differences."""
    m = mech.h2_air_9()
    full = (ctypes.c_int * 10)()
    nsys = kh.kh_sys_full(full)
    sys_ = list(full[:nsys])
    names = m.species_names()
    assert [c for c in range(10) if c not in sys_] == [names.index("N2")]
    t = kh.kh_tables(ctypes.addressof(m))
    try:
        for rho, y in states(m, 120, seed=3):
            J = np.zeros((10, 10))
            Fj = np.zeros(10)
            Ft = np.zeros(10)
            kh.kh_jac_compiled(rho, p(y), p(J), p(Fj))
            # the right-hand side formed with the Jacobian is the tables' one, bit for bit
            kh.kh_rhs_tables(t, rho, p(y), p(Ft))
            assert np.array_equal(Fj, Ft), (y, Fj - Ft)
            assert Ft[names.index("N2")] == 0.0
            scale = np.abs(J[sys_]).max(axis=1) + 1e-300
            for j in sys_:
                def F(d):
                    yy = y.copy()
                    yy[j] += d
                    out = np.zeros(10)
                    kh.kh_rhs_tables(t, rho, p(yy), p(out))
                    return out
                best = np.inf
                for r in (1e-3, 1e-4, 1e-5, 1e-6):
                    h = (max(abs(y[j]), 1e-6) if j < 9 else y[j]) * r
                    d1 = (F(h) - F(-h)) / (2 * h)
                    d2 = (F(h / 2) - F(-h / 2)) / h
                    best = min(best, (np.abs(J[sys_, j] - ((4 * d2 - d1) / 3)[sys_]) / scale).max())
                assert best < 1e-6, (j, best)
    finally:
        kh.kh_free(t)


@pytest.mark.parametrize("dt", [5e-10, 1e-7, 2e-6])
def test_compiled_ros2_matches_the_host_integrator(kh, dt):
    m = mech.h2_air_9()
    t = kh.kh_tables(ctypes.addressof(m))
    subs = []
    try:
        for rho, y in layer_states(kh, t, m):
            Ya, Ta = y[:9].copy(), np.array([y[9]])
            Yb, Tb = y[:9].copy(), np.array([y[9]])
            na = kh.kh_ros2_tables(t, rho, p(Ya), p(Ta), dt)
            nb = kh.kh_ros2_compiled(rho, p(Yb), p(Tb), dt)
            # the same sub-steps (or both at the cap) and the same state to rounding
            assert na == nb
            assert np.abs(Ya - Yb).max() <= 1e-10 and abs(Ta[0] - Tb[0]) <= 1e-9 * Ta[0], (Ya - Yb, Ta - Tb)
            subs.append(na)
    finally:
        kh.kh_free(t)
    subs = np.array(subs)
    assert len(subs) > 200 and np.mean(subs > 0) > 0.75
    if dt >= 2e-6:
        assert subs.max() > 5  # the long steps exercise the step-size control


def test_matches_accepts_its_mechanism_and_rejects_any_change(kh):
    m = mech.h2_air_9()
    assert kh.kh_matches(ctypes.addressof(m)) == 1

    def bumped(fn):
        mm = mech.h2_air_9()
        fn(mm)
        return kh.kh_matches(ctypes.addressof(mm))

    up = lambda x: float(np.nextafter(x, np.inf))
    edits = [
        lambda mm: mm.A.__setitem__(5, up(mm.A[5])),
        lambda mm: mm.b.__setitem__(1, up(mm.b[1])),
        lambda mm: mm.Ea.__setitem__(2, up(mm.Ea[2])),
        lambda mm: mm.W.__setitem__(3, up(mm.W[3])),
        lambda mm: mm.nasa_lo[4].__setitem__(2, up(mm.nasa_lo[4][2])),
        lambda mm: mm.nasa_hi[8].__setitem__(6, up(mm.nasa_hi[8][6])),
        lambda mm: mm.T_mid.__setitem__(0, up(mm.T_mid[0])),
        lambda mm: mm.eff[0].__setitem__(4, up(mm.eff[0][4])),
        lambda mm: mm.troe[21].__setitem__(0, up(mm.troe[21][0])),
        lambda mm: mm.A0.__setitem__(8, up(mm.A0[8])),
        lambda mm: mm.reversible.__setitem__(3, 0),
        lambda mm: mm.nu_reac[3].__setitem__(0, 1.0),
        lambda mm: setattr(mm, "n_reactions", mm.n_reactions - 1),
    ]
    for i, e in enumerate(edits):
        assert bumped(e) == 0, i


def test_committed_header_is_generated_from_the_committed_mechanism():
    sys.path.insert(0, PKG)
    import gen_kinetics
    m = mech.load_json(os.path.join(PKG, "data", "h2_air_9.json"))
    text = gen_kinetics.generate(m, "h2_air_9")
    assert text == open(os.path.join(CSRC, "kinetics_h2_air_9.cuh")).read()
