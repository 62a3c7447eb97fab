"""Generates tests/golden/kin_h2_air_9.npz: an independent evaluation of the 9-species
H2/O2/N2 kinetics the device uses, for tests/test_kinetics_independent.py.

Run from the repository root with the reference tree:

    python tests/golden/make_kinetics.py --reference <reference tree>

(or with the tree in LBM_REFERENCE).  It shares no code with csrc/gas.cuh or mech.py: it
parses the reference's src/reaction-mech/nh3.yaml (the Cantera-YAML mechanism the device
table is extracted from) with PyYAML, keeps the species H2, H, O2, O, H2O, OH, H2O2, HO2, N2
and the reactions closed over them, drops third-body efficiencies of the other species,
and evaluates in numpy, from the published formulas:

* NASA 7-coefficient thermo (McBride, Gordon & Reno, NASA TM-4513);
* modified Arrhenius rates k = A T^b exp(-Ea / R T), converted from the file's units
  (cm, mol, cal/mol) to kmol, m^3, J;
* third-body rates with the collision efficiencies; Lindemann/Troe fall-off (Gilbert,
  Luther & Troe, Ber. Bunsenges. Phys. Chem. 87 (1983) 169);
* reverse rates from K_c = exp(-dG0 / R T) (p0 / R T)^dnu with p0 = 1 atm (Cantera's
  reference pressure of NASA-7 species);
* mass-action rates of progress and net production rates.

Inputs: 1000 seeded states (numpy PCG64, seed 20261205): T uniform in 300..2500 K, p
log-uniform in 0.5..5 atm, mass fractions from exponentials of normals (spread over six
decades, so trace and major species both occur), normalised.  Outputs per state: the forward
and reverse rates of progress of every reaction and the net production rates.

Also the constant-volume ignition delay of stoichiometric H2-air (X_H2 : X_O2 : X_N2 =
0.2958 : 0.1479 : 0.5563) at 1 atm and 1000 K -- the time of the largest dT/dt, integrated
with SciPy's BDF (rtol 1e-9) over the rates above -- and the temperature history.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KEEP = ["H2", "H", "O2", "O", "H2O", "OH", "H2O2", "HO2", "N2"]
R_U = 8314.46261815324      # J / (kmol K)
P_ATM = 101325.0
CAL = 4184.0                # J/kmol per cal/mol


def reference_tree():
    ref = os.environ.get("LBM_REFERENCE")
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    if not ref:
        raise SystemExit("make_kinetics.py: pass --reference <reference tree> or set LBM_REFERENCE")
    return ref


def side(text):
    """'2 OH' / 'O + O + M' / 'H2O2 (+M)' -> {species: coefficient}."""
    out = {}
    text = text.replace("(+M)", "")
    for term in text.split(" + "):
        term = term.strip()
        if not term or term == "M":
            continue
        m = re.match(r"^(\d+(?:\.\d+)?)\s+(\S+)$", term)
        c, s = (float(m.group(1)), m.group(2)) if m else (1.0, term)
        out[s] = out.get(s, 0.0) + c
    return out


class Mech:
    def __init__(self, path):
        import yaml
        doc = yaml.safe_load(open(path))
        u = doc.get("units", {})
        assert u.get("length") == "cm" and u.get("quantity") == "mol" and u.get("activation-energy") == "cal/mol"
        sp = {s["name"]: s for s in doc["species"]}
        self.names = KEEP
        self.ns = len(KEEP)
        self.W = np.zeros(self.ns)
        self.tr = np.zeros((self.ns, 3))
        self.lo = np.zeros((self.ns, 7))
        self.hi = np.zeros((self.ns, 7))
        mass = {"H": 1.008, "O": 15.999, "N": 14.007}
        for k, n in enumerate(KEEP):
            s = sp[n]
            self.W[k] = sum(mass[e] * c for e, c in s["composition"].items())
            self.tr[k] = s["thermo"]["temperature-ranges"]
            self.lo[k], self.hi[k] = s["thermo"]["data"]
        self.rx = []
        for r in doc["reactions"]:
            lhs, rhs = r["equation"].split("<=>") if "<=>" in r["equation"] else r["equation"].split("=>")
            reac, prod = side(lhs), side(rhs)
            if not set(reac) | set(prod) <= set(KEEP):
                continue
            kind = r.get("type", "elementary")
            order = sum(reac.values())
            d = {"reac": reac, "prod": prod, "kind": kind, "rev": "<=>" in r["equation"]}
            if kind == "falloff":
                d["hi"] = self.arr(r["high-P-rate-constant"], order)
                d["lo"] = self.arr(r["low-P-rate-constant"], order + 1)
                t = r.get("Troe")
                d["troe"] = None if t is None else (t["A"], t["T3"], t["T1"], t.get("T2"))
            else:
                d["k"] = self.arr(r["rate-constant"], order + (1 if kind == "three-body" else 0))
            if kind in ("three-body", "falloff"):
                eff = np.ones(self.ns)
                for s_, e in r.get("efficiencies", {}).items():
                    if s_ in KEEP:
                        eff[KEEP.index(s_)] = e
                d["eff"] = eff
            self.rx.append(d)

    @staticmethod
    def arr(p, order):
        """(A in kmol, m^3, s; b; Ea in J/kmol) from the file's cm / mol / cal/mol."""
        return (p["A"] * 1e-3 ** (order - 1), p["b"], p["Ea"] * CAL)

    def nasa(self, T):
        """(cp/R, h/RT, s/R) arrays of shape (ns,) at T."""
        a = np.where((T < self.tr[:, 1])[:, None], self.lo, self.hi)
        cp = a[:, 0] + a[:, 1] * T + a[:, 2] * T ** 2 + a[:, 3] * T ** 3 + a[:, 4] * T ** 4
        h = a[:, 0] + a[:, 1] * T / 2 + a[:, 2] * T ** 2 / 3 + a[:, 3] * T ** 3 / 4 + a[:, 4] * T ** 4 / 5 + a[:, 5] / T
        s = a[:, 0] * np.log(T) + a[:, 1] * T + a[:, 2] * T ** 2 / 2 + a[:, 3] * T ** 3 / 3 + a[:, 4] * T ** 4 / 4 + a[:, 6]
        return cp, h, s

    def rates(self, T, C):
        """Forward and reverse rates of progress (kmol/m^3/s) of every reaction, and the net
        production rates of every species, at T (K) and concentrations C (kmol/m^3)."""
        _, h, s = self.nasa(T)
        g = h - s
        qf = np.zeros(len(self.rx))
        qr = np.zeros(len(self.rx))
        for i, r in enumerate(self.rx):
            arrh = lambda p: p[0] * T ** p[1] * np.exp(-p[2] / (R_U * T))  # noqa: E731
            if r["kind"] == "falloff":
                kinf, k0 = arrh(r["hi"]), arrh(r["lo"])
                M = float(r["eff"] @ C)
                Pr = k0 * M / kinf
                F = 1.0
                if r["troe"] is not None:
                    A, T3, T1, T2 = r["troe"]
                    Fc = (1 - A) * np.exp(-T / T3) + A * np.exp(-T / T1) + (np.exp(-T2 / T) if T2 is not None else 0.0)
                    lf = np.log10(Fc)
                    c = -0.4 - 0.67 * lf
                    n = 0.75 - 1.27 * lf
                    lp = np.log10(Pr)
                    F = 10.0 ** (lf / (1.0 + ((lp + c) / (n - 0.14 * (lp + c))) ** 2))
                kf = kinf * Pr / (1.0 + Pr) * F
            else:
                kf = arrh(r["k"])
                if r["kind"] == "three-body":
                    kf = kf * float(r["eff"] @ C)
            qf[i] = kf * np.prod([C[KEEP.index(s_)] ** v for s_, v in r["reac"].items()])
            if r["rev"]:
                dg = sum(v * g[KEEP.index(s_)] for s_, v in r["prod"].items()) - \
                    sum(v * g[KEEP.index(s_)] for s_, v in r["reac"].items())
                dnu = sum(r["prod"].values()) - sum(r["reac"].values())
                Kc = np.exp(-dg) * (P_ATM / (R_U * T)) ** dnu
                qr[i] = kf / Kc * np.prod([C[KEEP.index(s_)] ** v for s_, v in r["prod"].items()])
        w = np.zeros(self.ns)
        for i, r in enumerate(self.rx):
            q = qf[i] - qr[i]
            for s_, v in r["reac"].items():
                w[KEEP.index(s_)] -= v * q
            for s_, v in r["prod"].items():
                w[KEEP.index(s_)] += v * q
        return qf, qr, w


def ignition(mech, T0=1000.0, p0=P_ATM):
    """Constant-volume adiabatic reactor: dY/dt = w W / rho, dT/dt = -sum e_k w_k / (rho cv)."""
    from scipy.integrate import solve_ivp
    X = np.zeros(mech.ns)
    for n, x in (("H2", 0.2958), ("O2", 0.1479), ("N2", 0.5563)):
        X[KEEP.index(n)] = x
    X /= X.sum()
    Wm = X @ mech.W
    Y0 = X * mech.W / Wm
    rho = p0 * Wm / (R_U * T0)

    def f(t, y):
        Y, T = y[:-1], y[-1]
        C = rho * Y / mech.W
        _, _, w = mech.rates(T, C)
        cp, h, _ = mech.nasa(T)
        cv = R_U * np.sum(Y * (cp - 1.0) / mech.W)
        e = R_U * T * (h - 1.0)  # J/kmol
        return np.concatenate([w * mech.W / rho, [-np.sum(e * w) / (rho * cv)]])

    sol = solve_ivp(f, (0.0, 2e-3), np.concatenate([Y0, [T0]]), method="BDF", rtol=1e-9, atol=1e-14,
                    dense_output=True)
    t = np.linspace(0.0, 2e-3, 200001)
    T = sol.sol(t)[-1]
    dT = np.gradient(T, t)
    return t[np.argmax(dT)], rho, Y0, t[::1000], T[::1000]


def main():
    mech = Mech(os.path.join(reference_tree(), "src", "reaction-mech", "nh3.yaml"))
    rng = np.random.Generator(np.random.PCG64(20261205))
    n = 1000
    T = rng.uniform(300.0, 2500.0, n)
    p = P_ATM * np.exp(rng.uniform(np.log(0.5), np.log(5.0), n))
    Y = np.exp(rng.normal(0.0, 3.0, (n, mech.ns)))
    Y /= Y.sum(1, keepdims=True)
    C = np.zeros((n, mech.ns))
    QF = np.zeros((n, len(mech.rx)))
    QR = np.zeros((n, len(mech.rx)))
    WD = np.zeros((n, mech.ns))
    for i in range(n):
        Wm = 1.0 / np.sum(Y[i] / mech.W)
        rho = p[i] * Wm / (R_U * T[i])
        C[i] = rho * Y[i] / mech.W
        QF[i], QR[i], WD[i] = mech.rates(T[i], C[i])
    tau, rho_ig, Y_ig, t_hist, T_hist = ignition(mech)
    eqs = [" + ".join(f"{v:g} {s}" for s, v in r["reac"].items()) + " <=> "
           + " + ".join(f"{v:g} {s}" for s, v in r["prod"].items()) for r in mech.rx]
    np.savez_compressed(os.path.join(HERE, "kin_h2_air_9.npz"), species=np.array(KEEP), equations=np.array(eqs),
                        T=T, p=p, Y=Y, C=C, qf=QF, qr=QR, wdot=WD, W=mech.W, tau_ign=tau, rho_ign=rho_ig,
                        Y_ign=Y_ig, t_hist=t_hist, T_hist=T_hist)
    print(f"{len(mech.rx)} reactions, ignition delay {tau * 1e6:.2f} us")


if __name__ == "__main__":
    main()
