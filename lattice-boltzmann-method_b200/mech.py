"""Loader of the repository's Cantera-YAML gas mechanisms into the flat ``lbmgpu_mech``
tables of include/lbmgpu.h (SI units: kmol, m, s, J, K).

It replaces ``Cantera::newSolution(file, phase)`` (reference src/lbm-main.cpp:84) for the
subset of the YAML format the reference's mechanisms use (src/reaction-mech/*.yaml, written
by Cantera 3.0.0's ck2yaml): ``ideal-gas`` thermo with NASA-7 polynomials, ``gas``
transport parameters, and elementary / ``three-body`` / ``falloff`` (Lindemann and Troe)
reactions with optional ``duplicate`` and ``efficiencies`` entries.

``load(path, species)`` extracts the listed species, keeps the reactions closed over them
and drops third-body efficiencies of absent species (the reference's 9-species H2/O2/N2
set comes from nh3.yaml this way).
"""
import ctypes
import re

import yaml

MAX_SPECIES = 12
MAX_REACTIONS = 48
MAX_RSPEC = 3
RXN_ELEMENTARY, RXN_THREEBODY, RXN_FALLOFF = 0, 1, 2
GEOM = {"atom": 0, "linear": 1, "nonlinear": 2}

# IUPAC standard atomic weights (kg/kmol) of the elements these mechanisms contain
ATOMIC_WEIGHT = {"H": 1.008, "O": 15.999, "N": 14.007, "Ar": 39.95, "He": 4.002602, "C": 12.011}
ELEMENT_SLOT = {"H": 0, "O": 1, "N": 2, "Ar": 3, "C": 4}
MAX_ELEMENTS = 5
DEBYE = 3.33564e-30          # C m
CAL = 4.184                  # J

H2_AIR_9 = ["H2", "H", "O2", "O", "H2O", "OH", "H2O2", "HO2", "N2"]


class Mech(ctypes.Structure):
    S, R, K = MAX_SPECIES, MAX_REACTIONS, MAX_RSPEC
    _fields_ = [
        ("n_species", ctypes.c_int), ("n_reactions", ctypes.c_int),
        ("name", (ctypes.c_char * 16) * S),
        ("W", ctypes.c_double * S),
        ("T_lo", ctypes.c_double * S), ("T_mid", ctypes.c_double * S), ("T_hi", ctypes.c_double * S),
        ("nasa_lo", (ctypes.c_double * 7) * S), ("nasa_hi", (ctypes.c_double * 7) * S),
        ("geometry", ctypes.c_int * S),
        ("well_depth", ctypes.c_double * S), ("diameter", ctypes.c_double * S),
        ("dipole", ctypes.c_double * S), ("polarizability", ctypes.c_double * S),
        ("rot_relax", ctypes.c_double * S),
        ("elements", (ctypes.c_int * MAX_ELEMENTS) * S),
        ("rtype", ctypes.c_int * R), ("reversible", ctypes.c_int * R),
        ("n_reac", ctypes.c_int * R), ("n_prod", ctypes.c_int * R),
        ("reac", (ctypes.c_int * K) * R), ("prod", (ctypes.c_int * K) * R),
        ("nu_reac", (ctypes.c_double * K) * R), ("nu_prod", (ctypes.c_double * K) * R),
        ("A", ctypes.c_double * R), ("b", ctypes.c_double * R), ("Ea", ctypes.c_double * R),
        ("A0", ctypes.c_double * R), ("b0", ctypes.c_double * R), ("Ea0", ctypes.c_double * R),
        ("troe_n", ctypes.c_int * R), ("troe", (ctypes.c_double * 4) * R),
        ("eff", (ctypes.c_double * S) * R),
        ("order_reac", (ctypes.c_double * K) * R),
    ]

    def species_names(self):
        return [self.name[k].value.decode() for k in range(self.n_species)]


def _parse_side(side):
    """'H2O2 (+M)' / 'O + O + M' / '2 OH' -> ({species: coefficient}, third_body_kind)."""
    tb = None
    side = side.strip()
    if re.search(r"\(\+\s*M\s*\)", side):
        tb = "falloff"
        side = re.sub(r"\(\+\s*M\s*\)", "", side)
    out = {}
    for tok in side.split(" + "):
        tok = tok.strip()
        if not tok:
            continue
        if tok == "M":
            tb = tb or "three-body"
            continue
        m = re.match(r"^(\d+(?:\.\d+)?)\s+(\S+)$", tok) or re.match(r"^(\d+(?:\.\d+)?)(\S+)$", tok)
        if m and not tok[0].isalpha():
            nu, sp = float(m.group(1)), m.group(2)
        else:
            nu, sp = 1.0, tok
        out[sp] = out.get(sp, 0.0) + nu
    return out, tb


def _convert_A(A, order, conc_factor):
    # (cm^3/mol)^(order-1) / s  ->  (m^3/kmol)^(order-1) / s
    return A * conc_factor ** (order - 1)


def load(path, species=H2_AIR_9):
    """Reads a Cantera-YAML mechanism and returns a filled ``Mech`` for `species`."""
    doc = yaml.safe_load(open(path))
    units = doc.get("units", {})
    length = {"cm": 1e-2, "m": 1.0}[units.get("length", "m")]
    qty = {"mol": 1e-3, "kmol": 1.0}[units.get("quantity", "kmol")]
    conc_factor = length ** 3 / qty          # 1 cm^3/mol = 1e-3 m^3/kmol
    ea_unit = units.get("activation-energy", "J/kmol")
    ea_factor = {"cal/mol": CAL * 1e3, "kcal/mol": CAL * 1e6, "J/mol": 1e3, "J/kmol": 1.0}[ea_unit]

    if len(species) > MAX_SPECIES:
        raise ValueError("too many species")
    by_name = {s["name"]: s for s in doc["species"]}
    m = Mech()
    m.n_species = len(species)
    idx = {}
    for k, name in enumerate(species):
        if name not in by_name:
            raise KeyError(f"species {name} is not in {path}")
        s = by_name[name]
        idx[name] = k
        m.name[k].value = name.encode()
        comp = s["composition"]
        m.W[k] = sum(ATOMIC_WEIGHT[e] * n for e, n in comp.items())
        for e, n in comp.items():
            if e not in ELEMENT_SLOT:
                raise ValueError(f"{name}: element {e} has no slot")
            m.elements[k][ELEMENT_SLOT[e]] = int(n)
        th = s["thermo"]
        if th["model"] != "NASA7":
            raise ValueError(f"{name}: only NASA7 thermo is supported")
        tr_ = th["temperature-ranges"]
        m.T_lo[k], m.T_mid[k], m.T_hi[k] = tr_[0], tr_[1], tr_[-1]
        for j in range(7):
            m.nasa_lo[k][j] = th["data"][0][j]
            m.nasa_hi[k][j] = th["data"][1][j] if len(th["data"]) > 1 else th["data"][0][j]
        tp = s.get("transport", {})
        m.geometry[k] = GEOM[tp.get("geometry", "atom")]
        m.well_depth[k] = tp.get("well-depth", 0.0)
        m.diameter[k] = tp.get("diameter", 0.0) * 1e-10
        m.dipole[k] = tp.get("dipole", 0.0) * DEBYE
        m.polarizability[k] = tp.get("polarizability", 0.0) * 1e-30
        m.rot_relax[k] = tp.get("rotational-relaxation", 0.0)

    nr = 0
    for r in doc.get("reactions", []):
        eq = r["equation"]
        rev = "<=>" in eq or ("=" in eq and "=>" not in eq)
        lhs, rhs = re.split(r"<=>|=>|=", eq, maxsplit=1)
        reac, tb1 = _parse_side(lhs)
        prod, tb2 = _parse_side(rhs)
        if not (set(reac) | set(prod)) <= set(species):
            continue
        if nr >= MAX_REACTIONS:
            raise ValueError("too many reactions")
        kind = r.get("type", "elementary")
        if kind not in ("elementary", "three-body", "falloff"):
            raise ValueError(f"reaction type {kind} not supported: {eq}")
        if len(reac) > MAX_RSPEC or len(prod) > MAX_RSPEC:
            raise ValueError(f"too many species in {eq}")
        m.rtype[nr] = {"elementary": RXN_ELEMENTARY, "three-body": RXN_THREEBODY, "falloff": RXN_FALLOFF}[kind]
        m.reversible[nr] = int(rev)
        m.n_reac[nr] = len(reac)
        m.n_prod[nr] = len(prod)
        orders = r.get("orders", {})
        if not set(orders) <= set(reac):
            raise ValueError(f"orders of non-reactants are not supported: {eq}")
        for j, (sp, nu) in enumerate(reac.items()):
            m.reac[nr][j] = idx[sp]
            m.nu_reac[nr][j] = nu
            m.order_reac[nr][j] = float(orders.get(sp, nu))
        for j, (sp, nu) in enumerate(prod.items()):
            m.prod[nr][j] = idx[sp]
            m.nu_prod[nr][j] = nu
        # the rate constant's units follow the reaction's order (the forward orders)
        order = sum(float(orders.get(sp, nu)) for sp, nu in reac.items())
        if kind == "falloff":
            hi, lo = r["high-P-rate-constant"], r["low-P-rate-constant"]
            m.A[nr] = _convert_A(hi["A"], order, conc_factor)
            m.b[nr] = hi["b"]
            m.Ea[nr] = hi["Ea"] * ea_factor
            m.A0[nr] = _convert_A(lo["A"], order + 1, conc_factor)
            m.b0[nr] = lo["b"]
            m.Ea0[nr] = lo["Ea"] * ea_factor
            if "Troe" in r:
                t = r["Troe"]
                vals = [t["A"], t["T3"], t["T1"]] + ([t["T2"]] if "T2" in t else [])
                m.troe_n[nr] = len(vals)
                for j, v in enumerate(vals):
                    m.troe[nr][j] = v
        else:
            rc = r["rate-constant"]
            m.A[nr] = _convert_A(rc["A"], order + (1 if kind == "three-body" else 0), conc_factor)
            m.b[nr] = rc["b"]
            m.Ea[nr] = rc["Ea"] * ea_factor
        for k in range(m.n_species):
            m.eff[nr][k] = 1.0 if kind in ("three-body", "falloff") else 0.0
        for sp, e in r.get("efficiencies", {}).items():
            if sp in idx:
                m.eff[nr][idx[sp]] = e
        nr += 1
    m.n_reactions = nr
    return m


def to_dict(m):
    """The table as plain lists (JSON-serialisable)."""
    out = {}
    for name, ctype in Mech._fields_:
        v = getattr(m, name)
        if isinstance(v, int):
            out[name] = v
        elif name == "name":
            out[name] = [m.name[k].value.decode() for k in range(MAX_SPECIES)]
        else:
            out[name] = _to_list(v)
    return out


def _to_list(v):
    try:
        return [_to_list(x) for x in v]
    except TypeError:
        return v


def from_dict(d):
    m = Mech()
    d = dict(d)
    if "order_reac" not in d:  # tables written before reaction orders: the stoichiometry
        d["order_reac"] = d["nu_reac"]
    d["elements"] = [list(row) + [0] * (MAX_ELEMENTS - len(row)) for row in d["elements"]]
    for name, ctype in Mech._fields_:
        v = d[name]
        if isinstance(v, int):
            setattr(m, name, v)
        elif name == "name":
            for k, s in enumerate(v):
                m.name[k].value = s.encode()
        else:
            _fill(getattr(m, name), v)
    return m


def _fill(arr, v):
    for i, x in enumerate(v):
        if isinstance(x, list):
            _fill(arr[i], x)
        else:
            arr[i] = x


def save_json(m, path, source=""):
    import json
    d = to_dict(m)
    d["_source"] = source
    with open(path, "w") as fh:
        json.dump(d, fh, separators=(",", ":"))


def load_json(path):
    import json
    with open(path) as fh:
        return from_dict(json.load(fh))


DATA = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)), "data")
H2_AIR_9_JSON = __import__("os").path.join(DATA, "h2_air_9.json")
CH4_2S_JSON = __import__("os").path.join(DATA, "ch4_2s.json")
C3H8_2S_JSON = __import__("os").path.join(DATA, "c3h8_2s.json")
CH4_2S = ["O2", "H2O", "CH4", "CO", "CO2", "N2"]
C3H8_2S = ["CO", "C3H8", "CO2", "H2O", "N2", "O2"]

# (table, source file in the reference's src/reaction-mech, species in the phase's order)
TABLES = [(H2_AIR_9_JSON, "nh3.yaml", H2_AIR_9), (CH4_2S_JSON, "CH4_2S.yaml", CH4_2S),
          (C3H8_2S_JSON, "propane_mech.yaml", C3H8_2S)]


def h2_air_9():
    """The 9-species H2/O2/N2 mechanism (23 reactions) extracted from the reference's
    src/reaction-mech/nh3.yaml; regenerate with
    ``python lattice-boltzmann-method_b200/mech.py <reference src/reaction-mech directory>``."""
    return load_json(H2_AIR_9_JSON)


def ch4_2s():
    """The reference's 6-species, 2-step methane mechanism (src/reaction-mech/CH4_2S.yaml,
    phase CH4_BFER_mix: CH4 + 1.5 O2 => CO + 2 H2O with orders CH4^0.5 O2^0.65, and
    CO + 0.5 O2 <=> CO2)."""
    return load_json(CH4_2S_JSON)


def c3h8_2s():
    """The reference's 6-species, 2-step propane mechanism (src/reaction-mech/propane_mech.yaml:
    C3H8 + 3.5 O2 => 3 CO + 4 H2O with orders C3H8^0.8 O2^0.86, and CO + 0.5 O2 <=> CO2)."""
    return load_json(C3H8_2S_JSON)


if __name__ == "__main__":
    import sys
    os_ = __import__("os")
    os_.makedirs(DATA, exist_ok=True)
    for path, src, species in TABLES:
        m = load(os_.path.join(sys.argv[1], src), species)
        save_json(m, path, source=f"{src} (farrasarira/Lattice-Boltzmann-Method src/reaction-mech), "
                                  "species " + " ".join(species))
        # the raw struct, for C/C++ callers: fread(&mech, sizeof(lbmgpu_mech), 1, f)
        with open(path[:-5] + ".bin", "wb") as fh:
            fh.write(bytes(m))
        print("wrote", path, m.n_species, "species", m.n_reactions, "reactions")
