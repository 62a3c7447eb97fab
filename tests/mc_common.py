"""Helpers shared by the multicomponent tests: the seeded inputs of the fixtures and the
host build of the device's per-cell functions (tests/host/mc_host.cpp)."""
import ctypes
import hashlib
import os
import subprocess

import numpy as np

import mech
import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CSRC = os.path.join(ROOT, "lattice-boltzmann-method_b200", "csrc")
NS = 9
SP0 = 17          # first per-species record plane
NREC = SP0 + 8 * NS
CASES = {
    "mc_mix8.npz": (False, {}, [1, 40]),
    "mc_react8.npz": (True, {"T_hi": 1800.0}, [1, 30]),
    # the reference's 6-species two-step methane mechanism (CH4_2S.yaml): a CH4-laden hot
    # slab in air, fractional reaction orders, CO oxidation reversible
    "mc_ch4_react8.npz": (True, {"T_hi": 1800.0, "fuel": "CH4", "Y_H2": 0.05}, [1, 30]),
    "mc_c3h8_react8.npz": (True, {"T_hi": 1800.0, "fuel": "C3H8", "Y_H2": 0.05}, [1, 30]),
}


def case_mech(fixture):
    if "ch4" in fixture:
        return mech.ch4_2s()
    if "c3h8" in fixture:
        return mech.c3h8_2s()
    return mech.h2_air_9()


def case(fixture):
    reaction, kw, cps = CASES[fixture]
    m = case_mech(fixture)
    mix, sp = W.mixing_layer_mc(m, N=8, **kw)
    return m, mix, sp, reaction, cps


def nrec(ns):
    return SP0 + 8 * ns


def digest(mix, sp):
    h = hashlib.sha256(np.ascontiguousarray(mix).tobytes())
    for a in sp:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def rel(got, want, scale=None):
    scale = max(np.max(np.abs(want)) if scale is None else scale, 1e-300)
    return float(np.max(np.abs(got - want)) / scale)


def build_host_lib(tmpdir, contract=True):
    """The host build of the per-cell functions; contract=False compiles it without
    floating-point contraction (no fused multiply-adds), like the no-FMA reference."""
    out = os.path.join(str(tmpdir), "libmchost.so" if contract else "libmchost_nofma.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC]
                   + ([] if contract else ["-ffp-contract=off"])
                   + [os.path.join(ROOT, "tests", "host", "mc_host.cpp"), "-o", out], check=True)
    return ctypes.CDLL(out)


def bc_errors(R, gold, cp, fl, reaction):
    """Largest relative differences of the record R (host or device planes) from a fixture's
    fields after cp steps, over the fluid cells fl: rho, T, p, rhoE, velocity (against the
    largest velocity component), every species density, and HRR when reacting."""
    e = {}
    for q, k in ((0, "rho"), (4, "temp"), (5, "p"), (6, "rhoe")):
        e[k] = rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl])
    vs = max(np.abs(gold[f"{k}_{cp}"].reshape(-1)[fl]).max() for k in "uvw")
    for q, k in ((1, "u"), (2, "v"), (3, "w")):
        e[k] = rel(R[q][fl], gold[f"{k}_{cp}"].reshape(-1)[fl], vs)
    e["rho_a"] = max(rel(R[SP0 + 8 * a][fl], gold[f"sp_rho_{cp}"][a].reshape(-1)[fl])
                     for a in range(len(gold[f"sp_rho_{cp}"])))
    if reaction:
        e["HRR"] = rel(R[13][fl], gold[f"HRR_{cp}"].reshape(-1)[fl])
    return e


def fixture_drift(gold_a, gold_b, cp, fl):
    """The same differences between two fixtures of one case (two builds of the reference)."""
    R = np.zeros((NREC, fl.size))
    for q, k in ((0, "rho"), (1, "u"), (2, "v"), (3, "w"), (4, "temp"), (5, "p"), (6, "rhoe")):
        R[q] = gold_a[f"{k}_{cp}"].reshape(-1)
    for a in range(NS):
        R[SP0 + 8 * a] = gold_a[f"sp_rho_{cp}"][a].reshape(-1)
    return max(bc_errors(R, gold_b, cp, fl, False).values())


def soa_state(mix, sp):
    """The device record planes of an AoS state (the planes the upload fills from it; the
    face-difference terms stay zero until Init computes them)."""
    nc = mix.size
    ns = len(sp)
    rec = np.zeros((nrec(ns), nc))
    f = lambda a: np.ascontiguousarray(a).reshape(-1)  # noqa: E731
    for q, k in enumerate(["rho", "u", "v", "w", "temp", "p", "rhoe"]):
        rec[q] = f(mix[k])
    P = mix["p_tensor"].reshape(-1, 9)
    for q, (a, b) in enumerate([(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]):
        rec[7 + q] = P[:, 3 * a + b]
    rec[13] = f(mix["HRR"])
    for a in range(ns):
        base = SP0 + 8 * a
        rec[base] = f(sp[a]["rho"])
        rec[base + 1] = f(sp[a]["u"])
        rec[base + 2] = f(sp[a]["v"])
        rec[base + 3] = f(sp[a]["w"])
        rec[base + 4] = f(sp[a]["X"])
    return rec


def host_run(L, m, mix, sp, reaction, steps, precision="fp64", shift=True, pops=False):
    """Init + `steps` steps of the host build (populations in FP64 or, "fp32", in FP32);
    returns (record planes, status)."""
    dt = np.float64 if precision == "fp64" else np.float32
    rec0 = soa_state(mix, sp)
    rec1 = rec0.copy()
    nc = mix.size
    ns = len(sp)
    pop0 = np.zeros((27 * (ns + 1), nc), dt)
    pop1 = np.zeros_like(pop0)
    typ = np.ascontiguousarray(mix["type"].astype(np.int8).reshape(-1))
    st = ctypes.c_uint(0)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    args = [*mix.shape, P(typ), ctypes.byref(m), ctypes.c_float(W.FLAME_UNITS[0]),
            ctypes.c_float(W.FLAME_UNITS[1]), int(reaction), steps, P(pop0), P(pop1), P(rec0), P(rec1)]
    fout = np.zeros((27 * (ns + 1), nc)) if pops else None
    if precision == "fp64":
        L.mc_host_run.restype = ctypes.c_int
        cur = L.mc_host_run(*args, ctypes.byref(st), P(fout) if pops else None)
    else:
        L.mc_host_run32.restype = ctypes.c_int
        cur = L.mc_host_run32(*args, int(shift), ctypes.byref(st))
    if pops:
        return (rec0, rec1)[cur], st.value, fout
    return (rec0, rec1)[cur], st.value
