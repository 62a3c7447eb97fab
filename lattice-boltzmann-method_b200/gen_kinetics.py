"""Compiles a gas mechanism into straight-line CUDA/C++ kinetics: the temperature factors of
every reaction (Arrhenius rate constants, fall-off k_0 and Troe F_cent, reverse factors
1/K_c from NASA-7 Gibbs energies, the species' h/RT and c_p/R) and the constant-volume
reactor's right-hand side from them (third-body sums, fall-off blending, mass-action rates of
progress, net production, dT/dt), with every constant a literal and every species index
fixed, so that the device integrator runs it without loading tables or branching on the
mechanism's structure.

    python gen_kinetics.py data/h2_air_9.json csrc/kinetics_h2_air_9.cuh

The generated `thermo` + `rhs_t` compute what gas.cuh's rate_factors + reactor_rhs_k
(net_production_k, progress_one) compute, operation for operation and in the same order
(sums over the reaction's species in the order the mechanism lists them, the quotients of
constants that the tables path forms at run time formed here as literals with the same
rounding), so that on a host without contraction of multiply-adds the two agree bit for bit.
Only the species' thermo is kept per temperature: each reaction's rate constants are formed
where the reaction is evaluated, so no per-reaction array stays live in the integrator's
registers.  `rhs_jac` returns the same right-hand side together with the analytic Jacobian.
Terms that are exactly zero or one are dropped (an Arrhenius exponent of 0, a third-body
efficiency of 0, a stoichiometric factor of 1), which leaves every result unchanged.  It
also emits `matches(mech)`, which tells whether a handle's mechanism is the one compiled
here.  The Makefile regenerates the header when the mechanism or this script changes.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

KR = 8314.46261815324      # J / (kmol K), gas.cuh's kR
ONE_ATM = 101325.0         # Pa, gas.cuh's kOneAtm
FALLOFF, THREEBODY = 2, 1
# rhs_jac places a scheduling fence (GAS_SCHED_FENCE) before every JAC_FENCE_EVERY-th reaction:
# between fences the compiler merges the accumulations of the reactions into the same matrix
# entries, across them it keeps no reaction's terms live.  Measured on the 9-species
# integrator (one ROS2 step of 16.8 M cells): 1 -> 25.1 ms, 2 -> 24.0, 4 -> 24.3, none -> 28.1.
JAC_FENCE_EVERY = 2


def lit(x):
    """A double literal that reads back as exactly x."""
    r = repr(float(x))
    if "inf" in r or "nan" in r:
        raise ValueError(f"non-finite mechanism constant {x}")
    return r if ("." in r or "e" in r) else r + ".0"


def conc(k, nu):
    """C_k^nu as gas::conc_pow evaluates it."""
    if nu == 1.0:
        return f"C{k}"
    if nu == 2.0:
        return f"(C{k} * C{k})"
    if nu == 3.0:
        return f"(C{k} * C{k} * C{k})"
    return f"pow(C{k}, {lit(nu)})"


def arrhenius(A, b, Ea):
    """A exp(b ln T - Ea / RT) (gas::rate_factor_one) without the exactly-zero terms."""
    if b == 0.0 and Ea == 0.0:
        return lit(A)  # A * exp(0 - 0) = A * 1
    if Ea == 0.0:
        return f"{lit(A)} * exp({lit(b)} * logT)"
    if b == 0.0:
        return f"{lit(A)} * exp(-({lit(Ea)} * invRT))"  # 0 * logT - x = -x
    return f"{lit(A)} * exp({lit(b)} * logT - {lit(Ea)} * invRT)"


def troe_terms(m, r):
    """The Troe F_cent terms of reaction r as (kind, value): kind 'zero' / 'one' where the term
    is exactly 0 or 1 in double precision for every temperature between 1e-17 K and 1e4 K
    (T*** <= 1e-20 or T** >= 1e20: exp underflows to 0; T* >= 1e20: exp(-T/T*) rounds to 1),
    'exp' otherwise."""
    a, T3, T1 = m.troe[r][0], m.troe[r][1], m.troe[r][2]
    out = [("zero" if T3 <= 1e-20 else ("one" if T3 >= 1e20 else "exp"), T3),
           ("zero" if T1 <= 1e-20 else ("one" if T1 >= 1e20 else "exp"), T1)]
    if m.troe_n[r] == 4:
        T2 = m.troe[r][3]
        out.append(("zero" if T2 >= 1e20 else ("one" if T2 <= 1e-20 else "exp"), T2))
    return out


def troe_constant(m, r):
    """log10 F_cent of reaction r as a literal when every term folds (troe_terms), else None;
    the same operations in the same order as gas::rate_factor_one, so the value is the one the
    tables compute."""
    import math
    terms = troe_terms(m, r)
    if any(k == "exp" for k, _ in terms):
        return None
    a = m.troe[r][0]
    val = lambda k: 0.0 if k == "zero" else 1.0  # noqa: E731
    Fc = (1.0 - a) * val(terms[0][0]) + a * val(terms[1][0])
    if len(terms) == 3:
        Fc += val(terms[2][0])
    return lit(math.log10(max(Fc, 1e-300)))


def weighted(terms):
    """sum_j nu_j g_j accumulated from 0 in the listed order (signs: +1 products, -1 reactants)."""
    out = ""
    for sign, nu, name in terms:
        t = name if nu == 1.0 else f"{lit(nu)} * {name}"
        if not out:
            out = t if sign > 0 else f"-({t})"
        else:
            out += (" + " if sign > 0 else " - ") + t
    return out or "0.0"


def dpow(k, nu, others):
    """d/dC_k of C_k^nu * prod(others): the product of the other factors times nu C_k^(nu-1)."""
    rest = [conc(j, n) for j, n in others]
    if nu == 1.0:
        head = []
    elif nu == 2.0:
        head = [f"2.0 * C{k}"]
    elif nu == 3.0:
        head = [f"3.0 * (C{k} * C{k})"]
    else:
        head = [f"{lit(nu)} * pow(C{k}, {lit(nu - 1.0)})"]
    terms = head + rest
    return " * ".join(terms) if terms else "1.0"


def nasa_branches(m, add, body):
    """Emits `body(k, a)` for every species under its switch temperature's branch (one branch
    per distinct switch temperature, as in factors)."""
    groups = {}
    for k in range(m.n_species):
        groups.setdefault(m.T_mid[k], []).append(k)
    for Tm, ks in groups.items():
        add(f"    if (T < {lit(Tm)}) {{")
        for branch in ("lo", "hi"):
            if branch == "hi":
                add("    } else {")
            for k in ks:
                body(k, m.nasa_lo[k] if branch == "lo" else m.nasa_hi[k])
        add("    }")


class Names:
    """How the generated code names a reaction's temperature factors and a species' thermo:
    the fused functions form k_inf, k_0, log10 F_cent and the reverse factor per reaction as
    locals (kf, k0, lFc0, er) and read h/RT, g/RT, c_p/R from the Thermo struct `th`."""

    def kf(self, r):
        return "kf"

    def er(self, r):
        return "er"

    def k0(self, i):
        return "k0"

    def lfc(self, i):
        return "lFc0"

    def hrt(self, k):
        return f"th.hRT[{k}]"

    def cpr(self, k):
        return f"th.cpR[{k}]"

    def grt(self, k):
        return f"th.gRT[{k}]"


def inert_species(m):
    """The species whose net stoichiometric coefficient is zero in every reaction."""
    net = [0.0] * m.n_species
    busy = [False] * m.n_species
    for r in range(m.n_reactions):
        d = {}
        for j in range(m.n_reac[r]):
            d[m.reac[r][j]] = d.get(m.reac[r][j], 0.0) - m.nu_reac[r][j]
        for j in range(m.n_prod[r]):
            d[m.prod[r][j]] = d.get(m.prod[r][j], 0.0) + m.nu_prod[r][j]
        for k, v in d.items():
            if v != 0.0:
                busy[k] = True
    return [k for k in range(m.n_species) if not busy[k]]


def system_index(m):
    """pos[k]: the unknown of the integrator's iteration system that state component k
    (species k, or T for k = n_species) is, None for an inert species; and the components of
    the system in order."""
    inert = set(inert_species(m))
    comps = [k for k in range(m.n_species) if k not in inert] + [m.n_species]
    pos = {c: i for i, c in enumerate(comps)}
    return pos, comps


def reaction_lists(m, r):
    reac = [(m.reac[r][j], m.nu_reac[r][j]) for j in range(m.n_reac[r])]
    prod = [(m.prod[r][j], m.nu_prod[r][j]) for j in range(m.n_prod[r])]
    ordr = [(m.reac[r][j], m.order_reac[r][j]) for j in range(m.n_reac[r])]
    return reac, prod, ordr


def emit_rates(m, r, fidx, add, N):
    """The temperature factors of reaction r as locals (gas::rate_factor_one): k_inf, for a
    fall-off reaction k_0 and log10 F_cent, and for a reversible one the reverse factor
    exp(dG/RT - dnu ln(p_atm / R T)); from logT, invRT, log_cref and the species' g/RT."""
    add(f"        const double kf = {arrhenius(m.A[r], m.b[r], m.Ea[r])};")
    if m.rtype[r] == FALLOFF:
        add(f"        const double k0 = {arrhenius(m.A0[r], m.b0[r], m.Ea0[r])};")
        if m.troe_n[r] >= 3 and troe_constant(m, r) is not None:
            # every F_cent term is exactly 0 or 1 at physical temperatures (troe_terms)
            add(f"        const double lFc0 = {troe_constant(m, r)};")
        elif m.troe_n[r] >= 3:
            a, T3, T1 = m.troe[r][0], m.troe[r][1], m.troe[r][2]
            add(f"        double Fc0 = {lit(1.0 - a)} * exp(-T / {lit(T3)}) + {lit(a)} * exp(-T / {lit(T1)});")
            if m.troe_n[r] == 4:
                add(f"        Fc0 += exp({lit(-m.troe[r][3])} / T);")
            add("        const double lFc0 = log10(fmax(Fc0, 1e-300));")
        else:
            add("        const double lFc0 = 0.0;")
    if m.reversible[r]:
        terms = [(+1, m.nu_prod[r][j], N.grt(m.prod[r][j])) for j in range(m.n_prod[r])]
        terms += [(-1, m.nu_reac[r][j], N.grt(m.reac[r][j])) for j in range(m.n_reac[r])]
        dnu = 0.0
        for _, nu, _ in terms[:m.n_prod[r]]:
            dnu += nu
        for _, nu, _ in terms[m.n_prod[r]:]:
            dnu -= nu
        dG = weighted(terms)
        if dnu == 0.0:
            add(f"        const double er = exp({dG});")
        else:
            add(f"        const double er = exp(({dG}) - {lit(dnu)} * log_cref);")


def emit_rhs_reaction(m, r, fidx, add, N, names):
    """Reaction r's rate of progress and its contributions to the net production rates w_k
    (gas::progress_one, net_production_k)."""
    ns = m.n_species
    reac, prod, ordr = reaction_lists(m, r)
    eq = " + ".join(f"{nu:g} {names[k]}" for k, nu in reac) + (" <=> " if m.reversible[r] else " => ") + \
        " + ".join(f"{nu:g} {names[k]}" for k, nu in prod)
    tag = "  (+M)" if m.rtype[r] == FALLOFF else ("  + M" if m.rtype[r] == THREEBODY else "")
    add(f"        {{  // rate of progress: {eq}{tag}")
    if m.rtype[r] == 0:
        add(f"            const double kfM = {N.kf(r)};")
    else:
        effs = [(k, m.eff[r][k]) for k in range(ns) if m.eff[r][k] != 0.0]
        msum = " + ".join((f"C{k}" if e == 1.0 else f"{lit(e)} * C{k}") for k, e in effs) or "0.0"
        add(f"            const double M = {msum};")
        if m.rtype[r] == FALLOFF:
            i = fidx[r]
            add(f"            const double Pr = {N.k0(i)} * M / {N.kf(r)};")
            if m.troe_n[r] >= 3:
                add(f"            const double lFc = {N.lfc(i)};")
                add("            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;")
                add("            const double lPr = log10(fmax(Pr, 1e-300));")
                add("            const double x = (lPr + c) / (n - 0.14 * (lPr + c));")
                add(f"            const double kfM = {N.kf(r)} * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));")
            else:
                add(f"            const double kfM = {N.kf(r)} * (Pr / (1.0 + Pr)) * 1.0;")
        else:
            add(f"            const double kfM = {N.kf(r)} * M;")
    add("            const double fwd = kfM" + "".join(f" * {conc(k, nu)}" for k, nu in ordr) + ";")
    if m.reversible[r]:
        add(f"            const double rev = kfM * {N.er(r)}" + "".join(f" * {conc(k, nu)}" for k, nu in prod) + ";")
        add("            const double q = fwd - rev;")
    else:
        add("            const double q = fwd;")
    for k, nu in reac:
        add(f"            w{k} -= {'q' if nu == 1.0 else lit(nu) + ' * q'};")
    for k, nu in prod:
        add(f"            w{k} += {'q' if nu == 1.0 else lit(nu) + ' * q'};")
    add("        }")


def emit_jac_reaction(m, r, fidx, add, N):
    """Reaction r's terms of s J (JACOBIAN_DOC)."""
    ns = m.n_species
    W = [m.W[k] for k in range(ns)]
    reac, prod, ordr = reaction_lists(m, r)
    net = {}
    for k, nu in reac:
        net[k] = net.get(k, 0.0) - nu
    for k, nu in prod:
        net[k] = net.get(k, 0.0) + nu
    net = {k: v for k, v in net.items() if v != 0.0}
    rev = bool(m.reversible[r])
    dlnkf = f"({lit(m.b[r])} + {lit(m.Ea[r])} * invRT) * invT"
    ind = "            "
    add("        {  // Jacobian terms")
    pf = " * ".join(conc(k, nu) for k, nu in ordr)
    pb = " * ".join(conc(k, nu) for k, nu in prod)
    add(f"{ind}const double pf = {pf};")
    if rev:
        add(f"{ind}const double pb = {pb};")
    if m.rtype[r] == 0:
        add(f"{ind}const double kfM = {N.kf(r)};")
        add(f"{ind}const double dlnk = {dlnkf};")
    else:
        effs = [(k, m.eff[r][k]) for k in range(ns) if m.eff[r][k] != 0.0]
        msum = " + ".join((f"C{k}" if e == 1.0 else f"{lit(e)} * C{k}") for k, e in effs) or "0.0"
        add(f"{ind}const double M = {msum};")
        if m.rtype[r] == FALLOFF:
            i = fidx[r]
            add(f"{ind}const double Pr = {N.k0(i)} * M / {N.kf(r)};")
            add(f"{ind}const double ipr = 1.0 / (1.0 + Pr);")
            add(f"{ind}const double dlnkinf = {dlnkf};")
            add(f"{ind}const double dlnk0 = ({lit(m.b0[r])} + {lit(m.Ea0[r])} * invRT) * invT;")
            if m.troe_n[r] >= 3:
                add(f"{ind}const double lFc = {N.lfc(i)};")
                add(f"{ind}const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;")
                add(f"{ind}const double lPr = log10(fmax(Pr, 1e-300));")
                add(f"{ind}const double u = lPr + c, den = n - 0.14 * u;")
                add(f"{ind}const double x = u / den;")
                add(f"{ind}const double opx = 1.0 + x * x;")
                add(f"{ind}const double Fo = pow(10.0, lFc / opx);")
                add(f"{ind}const double kfM = {N.kf(r)} * (Pr * ipr) * Fo;")
                add(f"{ind}const double dkdM = {N.k0(i)} * Fo * ipr * (ipr - 2.0 * x * lFc * n / (opx * opx * den * den));")
                # temperature derivative of F_cent (zero where it is a constant)
                if troe_constant(m, r) is not None:
                    add(f"{ind}const double dlFc = 0.0;")
                else:
                    a, T3, T1 = m.troe[r][0], m.troe[r][1], m.troe[r][2]
                    terms = troe_terms(m, r)
                    fc, dfc = [], []
                    if terms[0][0] == "exp":
                        add(f"{ind}const double e3 = exp(-T / {lit(T3)});")
                        fc.append(f"{lit(1.0 - a)} * e3")
                        dfc.append(f"-{lit((1.0 - a) / T3)} * e3")
                    elif terms[0][0] == "one":
                        fc.append(lit(1.0 - a))
                    if terms[1][0] == "exp":
                        add(f"{ind}const double e1 = exp(-T / {lit(T1)});")
                        fc.append(f"{lit(a)} * e1")
                        dfc.append(f"-{lit(a / T1)} * e1")
                    elif terms[1][0] == "one":
                        fc.append(lit(a))
                    if len(terms) == 3:
                        T2 = m.troe[r][3]
                        if terms[2][0] == "exp":
                            add(f"{ind}const double e2 = exp({lit(-T2)} / T);")
                            fc.append("e2")
                            dfc.append(f"{lit(T2)} * invT * invT * e2")
                        elif terms[2][0] == "one":
                            fc.append("1.0")
                    add(f"{ind}const double Fc = fmax({' + '.join(fc) or '0.0'}, 1e-300);")
                    add(f"{ind}const double dlFc = ({' + '.join(dfc) or '0.0'}) / (Fc * 2.302585092994046);")
                add(f"{ind}const double du = (dlnk0 - dlnkinf) * 0.4342944819032518 - 0.67 * dlFc;")
                add(f"{ind}const double dden = -1.27 * dlFc - 0.14 * du;")
                add(f"{ind}const double dx = (du * den - u * dden) / (den * den);")
                add(f"{ind}const double dlnFo = 2.302585092994046 * (dlFc / opx - 2.0 * x * lFc * dx / (opx * opx));")
                add(f"{ind}const double dlnk = dlnkinf + (dlnk0 - dlnkinf) * ipr + dlnFo;")
            else:
                add(f"{ind}const double kfM = {N.kf(r)} * (Pr * ipr);")
                add(f"{ind}const double dkdM = {N.k0(i)} * ipr * ipr;")
                add(f"{ind}const double dlnk = dlnkinf + (dlnk0 - dlnkinf) * ipr;")
        else:
            add(f"{ind}const double kfM = {N.kf(r)} * M;")
            add(f"{ind}const double dkdM = {N.kf(r)};")
            add(f"{ind}const double dlnk = {dlnkf};")
    if m.rtype[r] != 0:
        if rev:
            add(f"{ind}const double g = dkdM * (pf - {N.er(r)} * pb);")
        else:
            add(f"{ind}const double g = dkdM * pf;")
    # d q / dT at fixed concentrations
    if rev:
        dnu = sum(nu for _, nu in prod) - sum(nu for _, nu in reac)
        dh = " + ".join([f"{lit(nu)} * {N.hrt(k)}" for k, nu in prod]) + " - (" + \
            " + ".join([f"{lit(nu)} * {N.hrt(k)}" for k, nu in reac]) + ")"
        add(f"{ind}const double dlner = ({lit(dnu)} - ({dh})) * invT;")
        add(f"{ind}const double dqT = kfM * (dlnk * (pf - {N.er(r)} * pb) - {N.er(r)} * dlner * pb);")
    else:
        add(f"{ind}const double dqT = kfM * dlnk * pf;")
    dq = {}
    for idx, (k, nu) in enumerate(ordr):
        others = [x for jdx, x in enumerate(ordr) if jdx != idx]
        dq.setdefault(k, []).append(("+", dpow(k, nu, others)))
    if rev:
        for idx, (k, nu) in enumerate(prod):
            others = [x for jdx, x in enumerate(prod) if jdx != idx]
            dq.setdefault(k, []).append(("-", dpow(k, nu, others)))
    effs = {k: m.eff[r][k] for k in range(ns) if m.rtype[r] != 0 and m.eff[r][k] != 0.0}
    cols = [j for j in sorted(set(dq) | set(effs)) if j in system_index(m)[0]]
    for j in cols:
        parts = []
        for sign, e in dq.get(j, []):
            if sign == "+":
                parts.append(f"+ kfM * ({e})")
            else:
                parts.append(f"- kfM * {N.er(r)} * ({e})")
        if j in effs:
            e = effs[j]
            parts.append("+ g" if e == 1.0 else f"+ {lit(e)} * g")
        expr = " ".join(parts)
        expr = expr[2:] if expr.startswith("+ ") else "-" + expr[2:]
        add(f"{ind}const double dq{j} = {expr};")
    er_terms = " + ".join(f"{lit(v)} * ({N.hrt(k)} - 1.0)" for k, v in net.items()) or "0.0"
    add(f"{ind}const double e_r = {er_terms};")
    add(f"{ind}const double eT = sT * e_r;")
    add(f"{ind}sum_eT += e_r * dqT;")
    pos, _ = system_index(m)
    for j in cols:
        if pos.get(j) is None:
            continue  # an inert species' column multiplies its zero increment
        for k, v in net.items():
            add(f"{ind}J({pos[k]}, {pos[j]}) += {lit(v * W[k] / W[j])} * s * dq{j};")
        add(f"{ind}jT{pos[j]} += {lit(1.0 / W[j])} * eT * dq{j};")
    for k, v in net.items():
        add(f"{ind}jc{pos[k]} += {lit(v * W[k])} * s_rho * dqT;")
    add("        }")


JACOBIAN_DOC = """
The Jacobian of d(Y, T)/dt at fixed density, d F_k / d Y_j and d F_k / dT, differentiating the
right-hand side's expressions.  With q_r the rates of progress, nu_kr the net coefficients and
C_j = rho Y_j / W_j:
    dF_k/dY_j = (W_k / W_j) sum_r nu_kr dq_r/dC_j,
    dF_k/dT   = (W_k / rho) sum_r nu_kr dq_r/dT,
    dF_T/dY_j = -(R T / (W_j c_v)) sum_r e_r dq_r/dC_j - F_T R (c_p,j/R - 1) / (W_j c_v),
    dF_T/dT   = -R [sum_k (c_p,k/R - 1) w_k + T sum_r e_r dq_r/dT] / (rho c_v) - F_T (dc_v/dT) / c_v,
e_r = sum_k nu_kr (h_k/RT - 1), w_k the net production rates.  dq_r/dC_j through the
mass-action products, the third-body sum M and the Troe blend F(Pr), Pr = k0 M / k_inf:
d(k_inf Pr/(1+Pr) F)/dM = k0 F/(1+Pr) [1/(1+Pr) - 2 x lFc n / ((1+x^2)^2 (n - 0.14 u)^2)],
u = log10 Pr + c, x = u / (n - 0.14 u).  dq_r/dT through d ln k/dT = (b + E_a/RT)/T for
k_f and k_0, d ln(1/K_c)/dT = (dnu - sum_k nu_kr h_k/RT)/T (d(g_k/RT)/dT = -h_k/(R T^2),
d ln(p_atm/RT)/dT = -1/T), and for a fall-off reaction d ln(Pr/(1+Pr))/dT =
(d ln k0 - d ln k_inf)/(1+Pr) and d ln F/dT = ln 10 [dlFc/(1+x^2) - 2 x lFc dx/(1+x^2)^2]
with du = (d ln k0 - d ln k_inf)/ln 10 - 0.67 dlFc (dlFc = 0 where F_cent is constant).
Every term is accumulated straight into the scaled matrix (s J, s = -gamma h for the
integrator's iteration matrix).
"""


def emit_prologue(m, add, with_jac):
    """The locals every fused function starts from: T, the thermo scalars, the
    concentrations, the net production accumulators; for the Jacobian also c_v and the T
    row's scales, and the matrix cleared."""
    ns = m.n_species
    add(f"    const double T = y[{ns}];")
    add("    const double logT = th.logT, invRT = th.invRT, log_cref = th.log_cref;")
    add("    (void)logT;")
    add("    (void)log_cref;")
    for k in range(ns):
        add(f"    const double C{k} = rho * y[{k}] * {lit(1.0 / m.W[k])};")
    for k in range(ns):
        add(f"    double w{k} = 0.0;")
    add("    double cv = 0.0;")
    for k in range(ns):
        add(f"    cv += y[{k}] * (th.cpR[{k}] - 1.0) * {lit(1.0 / m.W[k])};")
    add(f"    cv *= {lit(KR)};")
    if with_jac:
        add("    const double invT = 1.0 / T;")
        add(f"    const double sT = -s * {lit(KR)} * T / cv;  // times e_r dq_rj / W_j: the T row")
        add("    const double s_rho = s / rho;")
        add("    double sum_eT = 0.0;  // sum_r e_r dq_r/dT")
        nsys = len(system_index(m)[1])
        # the temperature row and column: every reaction adds to them, so they are summed in
        # registers (in reaction order, as into the matrix) and stored once
        add("    // the temperature row (jT) and column (jc), summed in registers and stored once")
        add("    double " + ", ".join(f"jT{q} = 0.0" for q in range(nsys - 1)) + ";")
        add("    double " + ", ".join(f"jc{q} = 0.0" for q in range(nsys - 1)) + ";")
        add("#pragma unroll")
        add(f"    for (int k = 0; k < {nsys}; ++k)")
        add("#pragma unroll")
        add(f"        for (int j = 0; j < {nsys}; ++j) J(k, j) = 0.0;")


def emit_rhs_epilogue(m, add):
    """F from the net production rates (gas::reactor_rhs_k)."""
    ns = m.n_species
    add("    double es = 0.0;")
    for k in range(ns):
        add(f"    F[{k}] = w{k} * {lit(m.W[k])} / rho;")
        add(f"    es += (th.hRT[{k}] - 1.0) * {lit(KR)} * T * w{k};")
    add(f"    F[{ns}] = -es / (rho * cv);")


def emit_jac_epilogue(m, add):
    """The T row's composition columns (the c_v term) and its T column."""
    ns = m.n_species
    pos, _ = system_index(m)
    add(f"    const double sF = s * F[{ns}] * {lit(KR)} / cv;")
    for j in range(ns):
        if pos.get(j) is not None:
            add(f"    J({pos[ns]}, {pos[j]}) = jT{pos[j]} - sF * (th.cpR[{j}] - 1.0) * {lit(1.0 / m.W[j])};")
            add(f"    J({pos[j]}, {pos[ns]}) = jc{pos[j]};")
    add("    double sw = 0.0, dcv = 0.0;  // sum_k (c_p,k/R - 1) w_k, dc_v/dT / R")
    for k in range(ns):
        add(f"    sw += (th.cpR[{k}] - 1.0) * F[{k}] * rho * {lit(1.0 / m.W[k])};")

    def dcp(k, a):
        add(f"        dcv += y[{k}] * {lit(1.0 / m.W[k])} * ({lit(a[1])} + T * ({lit(2 * a[2])} + T * ({lit(3 * a[3])} + "
            f"T * {lit(4 * a[4])})));")
    nasa_branches(m, add, dcp)
    add(f"    J({pos[ns]}, {pos[ns]}) = s * (-{lit(KR)} * (sw + T * sum_eT) / (rho * cv) - F[{ns}] * {lit(KR)} * dcv / cv);")


def generate(m, name):
    ns, nr = m.n_species, m.n_reactions
    names = m.species_names()
    falloff = [r for r in range(nr) if m.rtype[r] == FALLOFF]
    fidx = {r: i for i, r in enumerate(falloff)}
    L = []
    add = L.append
    add(f"// Generated by gen_kinetics.py from the mechanism {name} -- do not edit; `make` regenerates it.")
    add("// Its kinetics as straight-line code: gas.cuh's rate_factors and reactor_rhs_k (thermo, rhs_t)")
    add("// and their analytic Jacobian (rhs_jac) with the mechanism's constants inlined.")
    add("#pragma once")
    add("#include <math.h>")
    add('#include "gas.cuh"')
    add("")
    add(f"namespace kin_{name} {{")
    add("")
    add(f"constexpr int NS = {ns}, NR = {nr}, NF = {max(len(falloff), 1)};")
    add("")
    # ---- matches(): every quantity the kinetics read
    add("// Whether `m` is the mechanism compiled here (every quantity the kinetics read).")
    add("inline bool matches(const lbmgpu_mech &m) {")
    add(f"    if (m.n_species != {ns} || m.n_reactions != {nr}) return false;")
    for k in range(ns):
        add(f"    if (m.W[{k}] != {lit(m.W[k])} || m.T_mid[{k}] != {lit(m.T_mid[k])}) return false;")
        for i in range(7):
            add(f"    if (m.nasa_lo[{k}][{i}] != {lit(m.nasa_lo[k][i])} || m.nasa_hi[{k}][{i}] != "
                f"{lit(m.nasa_hi[k][i])}) return false;")
    for r in range(nr):
        add(f"    if (m.rtype[{r}] != {m.rtype[r]} || m.reversible[{r}] != {m.reversible[r]} || m.n_reac[{r}] != "
            f"{m.n_reac[r]} || m.n_prod[{r}] != {m.n_prod[r]}) return false;")
        for j in range(m.n_reac[r]):
            add(f"    if (m.reac[{r}][{j}] != {m.reac[r][j]} || m.nu_reac[{r}][{j}] != {lit(m.nu_reac[r][j])} || "
                f"m.order_reac[{r}][{j}] != {lit(m.order_reac[r][j])}) return false;")
        for j in range(m.n_prod[r]):
            add(f"    if (m.prod[{r}][{j}] != {m.prod[r][j]} || m.nu_prod[{r}][{j}] != {lit(m.nu_prod[r][j])}) "
                f"return false;")
        add(f"    if (m.A[{r}] != {lit(m.A[r])} || m.b[{r}] != {lit(m.b[r])} || m.Ea[{r}] != {lit(m.Ea[r])}) "
            f"return false;")
        if m.rtype[r] == FALLOFF:
            add(f"    if (m.A0[{r}] != {lit(m.A0[r])} || m.b0[{r}] != {lit(m.b0[r])} || m.Ea0[{r}] != "
                f"{lit(m.Ea0[r])} || m.troe_n[{r}] != {m.troe_n[r]}) return false;")
            for i in range(m.troe_n[r]):
                add(f"    if (m.troe[{r}][{i}] != {lit(m.troe[r][i])}) return false;")
        if m.rtype[r] != 0:
            for k in range(ns):
                add(f"    if (m.eff[{r}][{k}] != {lit(m.eff[r][k])}) return false;")
    add("    return true;")
    add("}")
    add("")
    # ---- per-temperature thermo
    add("// The species' thermo at one temperature (NASA-7): h/RT, g/RT and c_p/R, with ln T, 1/RT and")
    add("// ln(p_atm / R T); the rate constants are formed from them reaction by reaction where they")
    add("// are used (rhs_t, rhs_jac), so that no per-reaction array stays live across the kinetics.")
    add("struct Thermo {")
    add("    double hRT[NS], gRT[NS], cpR[NS], logT, invRT, log_cref;")
    add("};")
    add("")
    add("GAS_HD void thermo(double T, Thermo &th) {")
    add("    const double logT = log(T);")
    add("    th.logT = logT;")
    add(f"    th.invRT = 1.0 / ({lit(KR)} * T);")
    add(f"    th.log_cref = log({lit(ONE_ATM)} / ({lit(KR)} * T));")

    def nasa(k, a):
        add(f"        th.cpR[{k}] = {lit(a[0])} + T * ({lit(a[1])} + T * ({lit(a[2])} + T * ({lit(a[3])} + T * "
            f"{lit(a[4])})));")
        # h_RT: a1/2 + T (a2/3 + T (a3/4 + T a4 / 5)) + a5 / T
        add(f"        th.hRT[{k}] = {lit(a[0])} + T * ({lit(a[1] / 2)} + T * ({lit(a[2] / 3)} + T * "
            f"({lit(a[3] / 4)} + T * {lit(a[4])} / 5.0))) + {lit(a[5])} / T;")
        # s_R: a0 ln T + T (a1 + T (a2/2 + T (a3/3 + T a4 / 4))) + a6 (the quarter is exact)
        add(f"        th.gRT[{k}] = th.hRT[{k}] - ({lit(a[0])} * logT + T * ({lit(a[1])} + T * ({lit(a[2] / 2)} + T * "
            f"({lit(a[3] / 3)} + T * {lit(a[4] / 4)}))) + {lit(a[6])});")
    nasa_branches(m, add, nasa)
    add("}")
    add("")
    N = Names()
    # ---- right-hand side
    add("// F = d(Y_0..Y_{NS-1}, T)/dt at density rho [kg/m^3] and state y, from the thermo th at")
    add("// y's temperature (gas::rate_factors + gas::reactor_rhs_k, reaction by reaction).")
    add("GAS_HD void rhs_t(const Thermo &th, double rho, const double *y, double *F) {")
    emit_prologue(m, add, with_jac=False)
    for r in range(nr):
        add("    GAS_SCHED_FENCE();")
        add(f"    {{  // reaction {r}")
        emit_rates(m, r, fidx, add, N)
        emit_rhs_reaction(m, r, fidx, add, N, names)
        add("    }")
    emit_rhs_epilogue(m, add)
    add("}")
    add("")
    # ---- right-hand side and Jacobian together
    _, comps = system_index(m)
    inert = inert_species(m)
    add("// rhs_t, and s times the Jacobian of F with respect to (Y, T) at fixed density over the")
    add("// unknowns of the integrator's iteration system (Kinetics::sys_full): J(p, q) = s dF_a / dY_b,")
    add("// a = sys_full(p), b = sys_full(q), the temperature the last unknown.")
    if inert:
        add("// The inert species (" + ", ".join(names[k] for k in inert) + ") are not unknowns: their row is zero")
        add("// and their column multiplies a zero increment.")
    add("// Each reaction's rate constants are formed once and serve both.")
    for line in JACOBIAN_DOC.strip().split("\n"):
        add("// " + line if line else "//")
    add("template <class Mat>")
    add("GAS_HD void rhs_jac(const Thermo &th, double rho, const double *y, double *F, double s, Mat &J) {")
    emit_prologue(m, add, with_jac=True)
    for r in range(nr):
        if r % JAC_FENCE_EVERY == 0:
            add("    GAS_SCHED_FENCE();")
        add(f"    {{  // reaction {r}")
        emit_rates(m, r, fidx, add, N)
        emit_rhs_reaction(m, r, fidx, add, N, names)
        emit_jac_reaction(m, r, fidx, add, N)
        add("    }")
    emit_rhs_epilogue(m, add)
    emit_jac_epilogue(m, add)
    add("}")
    add("")
    add("// The integrator's kinetics policy (gas::ros2_advance_km): thermo once per temperature,")
    add("// the right-hand side with the analytic Jacobian at the sub-step's start, the right-hand")
    add("// side alone at its second stage.")
    add("struct Kinetics {")
    add("    using K = Thermo;")
    add("    static constexpr bool kAnalyticJacobian = true;")
    add(f"    static constexpr int kSys = {len(comps)};  // unknowns of the iteration system")
    chain = str(comps[-1])
    for i in range(len(comps) - 2, -1, -1):
        chain = f"i == {i} ? {comps[i]} : ({chain})"
    add(f"    GAS_HD static constexpr int sys_full(int i) {{ return {chain}; }}")
    add("    GAS_HD void factors(double T, Thermo &k) const { thermo(T, k); }")
    add("    GAS_HD void rhs(const Thermo &k, double rho, const double *y, double *F) const { rhs_t(k, rho, y, F); }")
    add("    template <class Mat>")
    add("    GAS_HD void rhs_jacobian(const Thermo &k, double rho, const double *y, double *F, double s, Mat &J) const {")
    add("        rhs_jac(k, rho, y, F, s, J);")
    add("    }")
    add("};")
    add("")
    add(f"}}  // namespace kin_{name}")
    return "\n".join(L) + "\n"


def main():
    import mech
    src, out = sys.argv[1], sys.argv[2]
    m = mech.load_json(src)
    name = os.path.splitext(os.path.basename(src))[0]
    text = generate(m, name)
    if not os.path.exists(out) or open(out).read() != text:
        with open(out, "w") as fh:
            fh.write(text)


if __name__ == "__main__":
    main()
