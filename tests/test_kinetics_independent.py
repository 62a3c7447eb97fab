"""The device's kinetics (csrc/gas.cuh, built for the host as oracle/libgasprobe.so) against
an independent evaluation of the same mechanism (tests/golden/kin_h2_air_9.npz, written by
tests/golden/make_kinetics.py: its own parse of the reference's src/reaction-mech/nh3.yaml
and a numpy restatement of NASA-7 thermo, Arrhenius / third-body / Troe fall-off rates and
equilibrium-constant reverse rates, sharing no code with gas.cuh or mech.py).

The reference obtains these rates from Cantera (getNetProductionRates, called at
src/lbm-collision.cpp:382-384), which is not installed here; this pins the restatement to
the mechanism file and the published rate laws instead, on 1000 seeded states (T 300-2500
K, p 0.5-5 atm, mass fractions over six decades):
  * every reaction's forward and reverse rate of progress, 1e-10 relative;
  * every species' net production rate, 1e-10 of the gross rate through that species;
  * the constant-volume ignition delay of stoichiometric H2-air at 1 atm and 1000 K
    (the time of the largest dT/dt) from the device's stiff integrator (ROS2, rtol 1e-5,
    0.2 us steps) within 1 % of the independent SciPy BDF integration (191 us)."""
import ctypes
import os

import numpy as np
import pytest

import mech

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "kin_h2_air_9.npz")
D = ctypes.c_double
DP = ctypes.POINTER(D)


@pytest.fixture(scope="module")
def gp():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "libgasprobe.so"))
    L.gp_rates_of_progress.argtypes = [D, DP, DP, DP]
    L.gp_wdot.argtypes = [D, DP, DP]
    L.gp_ros2.argtypes = [D, DP, DP, D]
    L.gp_ros2.restype = ctypes.c_int
    L.gp_n_reactions.restype = ctypes.c_int
    m = mech.h2_air_9()
    L.gp_set_mech(ctypes.byref(m))
    L.mech = m
    return L


def ptr(a):
    return a.ctypes.data_as(DP)


def equations(m):
    """The mechanism table's reactions written as the fixture writes them."""
    names = m.species_names()
    out = []
    for r in range(m.n_reactions):
        lhs = " + ".join(f"{m.nu_reac[r][j]:g} {names[m.reac[r][j]]}" for j in range(m.n_reac[r]))
        rhs = " + ".join(f"{m.nu_prod[r][j]:g} {names[m.prod[r][j]]}" for j in range(m.n_prod[r]))
        out.append((lhs, rhs))
    return out


def canon(side):
    terms = {}
    for t in side.split(" + "):
        c, s = t.split()
        terms[s] = terms.get(s, 0.0) + float(c)
    return tuple(sorted(terms.items()))


def test_mechanism_table_matches_the_independent_parse(gp):
    g = np.load(GOLD)
    assert list(g["species"]) == gp.mech.species_names()
    mine = [(canon(a), canon(b)) for a, b in equations(gp.mech)]
    theirs = [tuple(canon(x) for x in e.split(" <=> ")) for e in g["equations"]]
    assert mine == theirs


def test_rates_of_progress_match_independent_evaluation(gp):
    g = np.load(GOLD)
    nr = gp.gp_n_reactions()
    names = gp.mech.species_names()
    nu = np.zeros((len(names), nr))  # |stoichiometric coefficient| of species k in reaction r
    for r, (lhs, rhs) in enumerate(equations(gp.mech)):
        for side in (lhs, rhs):
            for s_, c in canon(side):
                nu[names.index(s_), r] += c
    qf_all, qr_all, wd_all = g["qf"], g["qr"], g["wdot"]
    worst_q = worst_w = 0.0
    for i in range(len(g["T"])):
        C = np.ascontiguousarray(g["C"][i])
        qf = np.zeros(nr)
        qr = np.zeros(nr)
        gp.gp_rates_of_progress(float(g["T"][i]), ptr(C), ptr(qf), ptr(qr))
        for q, want in ((qf, qf_all[i]), (qr, qr_all[i])):
            scale = np.maximum(np.abs(want), 1e-300)
            worst_q = max(worst_q, float(np.max(np.abs(q - want) / scale)))
        w = np.zeros(len(C))
        gp.gp_wdot(float(g["T"][i]), ptr(C), ptr(w))
        gross = nu @ (qf_all[i] + qr_all[i])  # the gross rate through each species
        worst_w = max(worst_w, float(np.max(np.abs(w - wd_all[i]) / np.maximum(gross, 1e-300))))
    print(f"rates of progress {worst_q:.2e}, net production {worst_w:.2e}")
    assert worst_q < 1e-10
    assert worst_w < 1e-10


def test_ignition_delay_matches_independent_integration(gp):
    g = np.load(GOLD)
    Y = np.ascontiguousarray(g["Y_ign"].copy())
    T = D(1000.0)
    rho = float(g["rho_ign"])
    dt = 0.2e-6
    ts, Ts = [0.0], [1000.0]
    for k in range(1, 10001):
        assert gp.gp_ros2(rho, ptr(Y), ctypes.byref(T), dt) > 0
        ts.append(k * dt)
        Ts.append(T.value)
    ts, Ts = np.array(ts), np.array(Ts)
    tau = ts[np.argmax(np.gradient(Ts, ts))]
    print(f"ignition delay: device integrator {tau * 1e6:.2f} us, independent {float(g['tau_ign']) * 1e6:.2f} us")
    assert abs(tau - float(g["tau_ign"])) <= 0.01 * float(g["tau_ign"])
    assert Ts[-1] > 2400.0  # burnt
