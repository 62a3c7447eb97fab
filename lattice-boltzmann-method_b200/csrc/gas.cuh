// Ideal-gas thermodynamics, mixture-averaged transport and mass-action kinetics of one
// mechanism (the physical-property evaluations the reference obtains from Cantera 3.x:
// ThermoPhase, MixTransport, GasKinetics; call sites src/lbm-collision.cpp:236-247,
// 364-467, src/lbm-moment.cpp:219-368, src/lbm-edf.cpp:177-186).
//
// Written from the published methods, in FP64, for both host and device:
//  * thermo: NASA 7-coefficient polynomials (McBride, Gordon & Reno, NASA TM-4513):
//      cp/R = a1 + a2 T + a3 T^2 + a4 T^3 + a5 T^4,  h/RT = a1 + a2 T/2 + ... + a6/T,
//      s/R = a1 ln T + a2 T + a3 T^2/2 + a4 T^3/3 + a5 T^4/4 + a7;
//    T from (u, v) by Newton iteration on u(T) (what setState_UV solves).
//  * transport: as CHEMKIN's TRANFIT and Cantera do, the kinetic-theory expressions below
//    are evaluated at 50 temperatures and fitted once (make_tables) by degree-4
//    polynomials in ln T: ln mu_k, ln lambda_k and ln(D_kj P); the per-cell evaluation is
//    then one polynomial and one exp per property.  The kinetic theory:
//    Chapman-Enskog species viscosities and binary diffusion coefficients with
//    the Neufeld, Janzen & Aziz (1972) fits of the Lennard-Jones collision integrals
//    Omega(2,2)* and Omega(1,1)*, Brokaw's dipole correction, the polar/non-polar
//    combining rules of the CHEMKIN transport formulation (Kee et al., SAND86-8246);
//    species conductivities by the Warnatz/CHEMKIN translational-rotational-vibrational
//    split with the Parker-Brau-Jonkman rotational-relaxation temperature dependence;
//    mixture viscosity by Wilke's rule, mixture conductivity by the
//    Mathur-Tondon-Saxena average.
//  * kinetics: modified Arrhenius rates, third-body and Lindemann/Troe fall-off
//    (Gilbert, Luther & Troe 1983), reverse rates from equilibrium constants of the
//    NASA-7 Gibbs energies at 1 atm.
// Transport and kinetics have no pinned reference values (Cantera is not available);
// tests check them against physical identities and literature values.
#pragma once
#include <math.h>

#include "../../include/lbmgpu.h"

#if defined(__CUDACC__)
#define GAS_HD __host__ __device__ __forceinline__
#else
#define GAS_HD inline
#endif

// A point that the compiler moves no memory access across (device code only): placed between
// the reactions of the straight-line kinetics, it keeps the accumulations into the iteration
// matrix and the scheduling of each reaction's terms local to that reaction, which bounds the
// live registers of the unrolled code.
#if defined(__CUDA_ARCH__)
#define GAS_SCHED_FENCE() __asm__ volatile("" ::: "memory")
#else
#define GAS_SCHED_FENCE() ((void)0)
#endif

namespace gas {

constexpr double kR = 8314.46261815324;       // J / (kmol K)  (Cantera::GasConstant)
constexpr double kOneAtm = 101325.0;          // Pa
constexpr double kBoltz = 1.380649e-23;       // J / K
constexpr double kNA = 6.02214076e26;         // 1 / kmol
constexpr double kPi = 3.14159265358979323846;
constexpr double kEps0 = 8.8541878128e-12;    // F / m
constexpr int MAXS = LBMGPU_MAX_SPECIES;
constexpr int MAXR = LBMGPU_MAX_REACTIONS;

// Mechanism plus the per-species and per-pair transport constants derived from it once
// on the host (make_tables).
struct Tables {
    lbmgpu_mech m;
    int ns;
    double invW[MAXS];
    // h/RT polynomial of each NASA-7 range with its quotients formed once: a1, a2/2, a3/3,
    // a4/4, a5/5, a6 (the reciprocal forms of the FP32 storage mode, h_RT_fast)
    double hcoef[MAXS][2][6];
    double visc_pref[MAXS];            // mu_k = visc_pref * sqrt(T) / Omega22(T/eps_k, delta_k)
    double eps[MAXS];                  // epsilon/k_B of the species, K
    double delta[MAXS];                // reduced dipole moment delta*_k
    double diff_pref[MAXS][MAXS];      // D_kj * P = diff_pref * T^1.5 / Omega11(T/eps_kj, delta_kj)
    double eps_pair[MAXS][MAXS];
    double delta_pair[MAXS][MAXS];
    double cvrot_R[MAXS];              // rotational heat capacity / R
    double zrot298_F298[MAXS];         // Z_rot(298) F(298), Z_rot(T) = this / F(T)
    // fits in x = ln T - kFitX0 (Horner order c[4] x^4 + ... + c[0])
    double fit_visc[MAXS][5];          // ln mu_k           [Pa s]
    double fit_cond[MAXS][5];          // ln lambda_k       [W/(m K)]
    double fit_diff[MAXS][MAXS][5];    // ln (D_kj * P)     [m^2 Pa / s]
    // per-species constants of the lattice collision, set by the device setup
    double Ra_lat[MAXS];               // units.cp(R / W_a)
    double sqrt4W[MAXS][MAXS];         // sqrt(sqrt(W_b / W_a))   (Wilke factor, reference order)
    double wilke_den[MAXS][MAXS];      // sqrt(8 (1 + W_a / W_b))
    float inv_wilke_den_f[MAXS][MAXS]; // 1 / wilke_den and W_a / W_b in FP32 (the FP32 storage
    float W_ratio_f[MAXS][MAXS];       // mode's transport)
    // dense stoichiometry (species k of reaction r; 0 where k does not take part): reactant and
    // product coefficients and their net difference, for the compile-time-unrolled kinetics
    double nu_f[MAXR][MAXS], nu_b[MAXR][MAXS], nu_net[MAXR][MAXS], dnu[MAXR];
    double ord_f[MAXR][MAXS];  // forward reaction orders (mech.order_reac) by species
};

constexpr double kFitTlo = 200.0, kFitThi = 3500.0, kFitX0 = 7.0;
constexpr int kFitN = 50;

GAS_HD double sq(double x) { return x * x; }

// ---- collision integrals (Neufeld, Janzen & Aziz 1972) with Brokaw's polar term ----
GAS_HD double omega22(double Ts, double delta) {
    const double o = 1.16145 * pow(Ts, -0.14874) + 0.52487 * exp(-0.77320 * Ts) + 2.16178 * exp(-2.43787 * Ts);
    return o + 0.2 * delta * delta / Ts;
}
GAS_HD double omega11(double Ts, double delta) {
    const double o = 1.06036 * pow(Ts, -0.15610) + 0.19300 * exp(-0.47635 * Ts) + 1.03587 * exp(-1.52996 * Ts) +
                     1.76474 * exp(-3.89411 * Ts);
    return o + 0.19 * delta * delta / Ts;
}

// Parker-Brau-Jonkman temperature function of the rotational collision number.
GAS_HD double parker_F(double eps_over_T) {
    const double x = eps_over_T;
    return 1.0 + 0.5 * pow(kPi, 1.5) * sqrt(x) + (0.25 * kPi * kPi + 2.0) * x + pow(kPi, 1.5) * x * sqrt(x);
}

inline void make_tables_base(const lbmgpu_mech &m, Tables &t) {
    t.m = m;
    t.ns = m.n_species;
    for (int k = 0; k < t.ns; ++k) {
        t.invW[k] = 1.0 / m.W[k];
        for (int r = 0; r < 2; ++r) {
            const double *a = r == 0 ? m.nasa_lo[k] : m.nasa_hi[k];
            const double c[6] = {a[0], a[1] / 2, a[2] / 3, a[3] / 4, a[4] / 5, a[5]};
            for (int i = 0; i < 6; ++i) t.hcoef[k][r][i] = c[i];
        }
        const double mk = m.W[k] / kNA;                 // kg per molecule
        const double s = m.diameter[k];
        t.visc_pref[k] = (5.0 / 16.0) * sqrt(kPi * mk * kBoltz) / (kPi * s * s);
        t.eps[k] = m.well_depth[k];
        const double epsJ = m.well_depth[k] * kBoltz;
        t.delta[k] = (epsJ > 0 && s > 0) ? 0.5 * m.dipole[k] * m.dipole[k] / (4.0 * kPi * kEps0 * epsJ * s * s * s) : 0.0;
        t.cvrot_R[k] = m.geometry[k] == LBMGPU_GEOM_ATOM ? 0.0 : (m.geometry[k] == LBMGPU_GEOM_LINEAR ? 1.0 : 1.5);
        t.zrot298_F298[k] = m.rot_relax[k] * parker_F(m.well_depth[k] / 298.0);
    }
    for (int k = 0; k < t.ns; ++k)
        for (int j = 0; j < t.ns; ++j) {
            double epsk = m.well_depth[k], epsj = m.well_depth[j];
            double sk = m.diameter[k], sj = m.diameter[j];
            double xi = 1.0;
            // polar / non-polar pair: induced-dipole correction of the combining rules
            const bool pk = m.dipole[k] > 0, pj = m.dipole[j] > 0;
            if (pk != pj) {
                const int p = pk ? k : j, n = pk ? j : k;
                const double alpha_n = m.polarizability[n] / (m.diameter[n] * m.diameter[n] * m.diameter[n]);
                const double epsp = m.well_depth[p] * kBoltz, sp3 = pow(m.diameter[p], 3);
                const double mu_p = m.dipole[p] / sqrt(4.0 * kPi * kEps0 * epsp * sp3);
                xi = 1.0 + 0.25 * alpha_n * mu_p * mu_p * sqrt(m.well_depth[p] / m.well_depth[n]);
            }
            t.eps_pair[k][j] = sqrt(epsk * epsj) * xi * xi;
            const double skj = 0.5 * (sk + sj) * pow(xi, -1.0 / 6.0);
            const double mred = (m.W[k] * m.W[j] / (m.W[k] + m.W[j])) / kNA;
            t.diff_pref[k][j] = (3.0 / 16.0) * sqrt(2.0 * kPi * pow(kBoltz, 3) / mred) / (kPi * skj * skj);
            t.delta_pair[k][j] = sqrt(t.delta[k] * t.delta[j]);
        }
}

// ---- thermo ----------------------------------------------------------------------
GAS_HD const double *nasa(const Tables &t, int k, double T) {
    return T < t.m.T_mid[k] ? t.m.nasa_lo[k] : t.m.nasa_hi[k];
}
GAS_HD double cp_R(const Tables &t, int k, double T) {
    const double *a = nasa(t, k, T);
    return a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4])));
}
GAS_HD double h_RT(const Tables &t, int k, double T) {
    const double *a = nasa(t, k, T);
    return a[0] + T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5))) + a[5] / T;
}
GAS_HD double s_R(const Tables &t, int k, double T) {
    const double *a = nasa(t, k, T);
    return a[0] * log(T) + T * (a[1] + T * (a[2] / 2 + T * (a[3] / 3 + T * a[4] / 4))) + a[6];
}

// mean molar mass from mass fractions (1 / sum Y/W; Cantera's meanMolecularWeight with
// normalised fractions)
GAS_HD double meanW_Y(const Tables &t, const double *Y) {
    double s = 0.0, sy = 0.0;
    for (int k = 0; k < t.ns; ++k) {
        s += Y[k] * t.invW[k];
        sy += Y[k];
    }
    return sy / s;
}
GAS_HD double cp_mass(const Tables &t, const double *Y, double T) {
    double c = 0.0;
    for (int k = 0; k < t.ns; ++k) c += Y[k] * cp_R(t, k, T) * t.invW[k];
    return c * kR;
}
GAS_HD double int_energy_mass(const Tables &t, const double *Y, double T) {
    double u = 0.0;
    for (int k = 0; k < t.ns; ++k) u += Y[k] * (h_RT(t, k, T) - 1.0) * t.invW[k];
    return u * kR * T;
}
GAS_HD double cv_mass(const Tables &t, const double *Y, double T) {
    double c = 0.0;
    for (int k = 0; k < t.ns; ++k) c += Y[k] * (cp_R(t, k, T) - 1.0) * t.invW[k];
    return c * kR;
}

// h/RT with the coefficients' quotients formed once and 1/T given: the same polynomial as
// h_RT with products in place of its divisions (the FP32 storage mode's moment solve, where
// the result differs from h_RT by rounding).
GAS_HD double h_RT_fast(const Tables &t, int k, double T, double invT) {
    const double *c = t.hcoef[k][T < t.m.T_mid[k] ? 0 : 1];
    return c[0] + T * (c[1] + T * (c[2] + T * (c[3] + T * c[4]))) + c[5] * invT;
}

// T_from_u with h_RT_fast and one reciprocal per iteration: the same damped Newton iteration
// and stopping rule, for NS species (t.ns) known at compile time so that Y stays in registers.
template <int NS>
GAS_HD int T_from_u_fast(const Tables &t, const double *Y, double u, double T0, double rtol, int maxit, double &T) {
    T = T0 > 0 ? T0 : 300.0;
    for (int it = 0; it < maxit; ++it) {
        const double invT = 1.0 / T;
        double e = 0.0, c = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            e += Y[k] * (h_RT_fast(t, k, T, invT) - 1.0) * t.invW[k];
            c += Y[k] * (cp_R(t, k, T) - 1.0) * t.invW[k];
        }
        double dT = -(e * kR * T - u) / (c * kR);
        if (dT > 500.0) dT = 500.0;
        if (dT < -0.5 * T) dT = -0.5 * T;
        T += dT;
        if (fabs(dT) <= rtol * T) return it + 1;
    }
    return -1;
}

// T with int_energy_mass(Y, T) = u: damped Newton from T0, at most `maxit` iterations.
// Returns the number of iterations, or -1 when the iteration cap was reached.
GAS_HD int T_from_u(const Tables &t, const double *Y, double u, double T0, double rtol, int maxit, double &T) {
    T = T0 > 0 ? T0 : 300.0;
    for (int it = 0; it < maxit; ++it) {
        const double f = int_energy_mass(t, Y, T) - u;
        const double cv = cv_mass(t, Y, T);
        double dT = -f / cv;
        if (dT > 500.0) dT = 500.0;
        if (dT < -0.5 * T) dT = -0.5 * T;
        T += dT;
        if (fabs(dT) <= rtol * T) return it + 1;
    }
    return -1;
}

// ---- transport: kinetic theory (evaluated at setup only) ---------------------------
inline double species_visc_kt(const Tables &t, int k, double T) {
    return t.visc_pref[k] * sqrt(T) / omega22(T / t.eps[k], t.delta[k]);
}
inline double binary_diff_kt(const Tables &t, int k, int j, double T, double P) {
    return t.diff_pref[k][j] * T * sqrt(T) / (P * omega11(T / t.eps_pair[k][j], t.delta_pair[k][j]));
}

// ---- transport: fitted (per cell) --------------------------------------------------
GAS_HD double fit_eval(const double *c, double x) { return c[0] + x * (c[1] + x * (c[2] + x * (c[3] + x * c[4]))); }
// the same polynomial in FP32 arithmetic (the FP32 storage mode's transport)
GAS_HD float fit_eval_f(const double *c, float x) {
    return (float)c[0] + x * ((float)c[1] + x * ((float)c[2] + x * ((float)c[3] + x * (float)c[4])));
}
GAS_HD double lnT_x(double T) { return log(T) - kFitX0; }
GAS_HD double species_visc(const Tables &t, int k, double T) { return exp(fit_eval(t.fit_visc[k], lnT_x(T))); }
GAS_HD double species_visc_x(const Tables &t, int k, double x) { return exp(fit_eval(t.fit_visc[k], x)); }
// D_kj at (T, P), m^2/s
GAS_HD double binary_diff(const Tables &t, int k, int j, double T, double P) {
    return exp(fit_eval(t.fit_diff[k][j], lnT_x(T))) / P;
}
GAS_HD double binary_diff_x(const Tables &t, int k, int j, double x, double P) {
    return exp(fit_eval(t.fit_diff[k][j], x)) / P;
}

// Wilke weights phi[a][b] = (1 + sqrt(mu_a/mu_b) (W_b/W_a)^(1/4))^2 / sqrt(8 (1 + W_a/W_b)),
// formed for b >= a and mirrored through phi[b][a] = mu_b/mu_a W_a/W_b phi[a][b] -- the
// way the reference's species collision forms them (src/lbm-collision.cpp:408-417); the
// mixture viscosity uses the same matrix.
GAS_HD void wilke_phi(const Tables &t, const double *mu, double (*phi)[MAXS]) {
    for (int a = 0; a < t.ns; ++a)
        for (int b = a; b < t.ns; ++b) {
            const double f1 = 1.0 + sqrt(mu[a] / mu[b]) * t.sqrt4W[a][b];
            phi[a][b] = f1 * f1 / t.wilke_den[a][b];
            phi[b][a] = mu[b] / mu[a] * t.m.W[a] / t.m.W[b] * phi[a][b];
        }
}

// Wilke's mixing rule: mu = sum_k X_k mu_k / sum_j X_j phi_kj.
GAS_HD double wilke_from_phi(const Tables &t, const double *X, const double *mu, const double (*phi)[MAXS]) {
    double s = 0.0;
    for (int k = 0; k < t.ns; ++k) {
        double d = 0.0;
        for (int j = 0; j < t.ns; ++j) d += X[j] * phi[k][j];
        s += X[k] * mu[k] / d;
    }
    return s;
}

GAS_HD double wilke(const Tables &t, const double *X, const double *mu) {
    double phi[MAXS][MAXS];
    wilke_phi(t, mu, phi);
    return wilke_from_phi(t, X, mu, phi);
}

// Species thermal conductivity (Warnatz / CHEMKIN), W/(m K), from kinetic theory.
inline double species_cond_kt(const Tables &t, int k, double T, double P, double mu_k) {
    const double W = t.m.W[k];
    const double rho = P * W / (kR * T);
    const double Dkk = binary_diff_kt(t, k, k, T, P);
    const double rdm = rho * Dkk / mu_k;
    const double cv_R = cp_R(t, k, T) - 1.0;
    if (t.m.geometry[k] == LBMGPU_GEOM_ATOM) return mu_k / W * kR * 2.5 * 1.5;
    const double cvrot = t.cvrot_R[k];
    const double cvvib = cv_R - 1.5 - cvrot;
    const double zrot = t.zrot298_F298[k] / parker_F(t.eps[k] / T);
    const double A = 2.5 - rdm;
    const double B = zrot + (2.0 / kPi) * (5.0 / 3.0 * cvrot + rdm);
    const double ftr = 2.5 * (1.0 - (2.0 / kPi) * (cvrot / 1.5) * (A / B));
    const double frot = rdm * (1.0 + (2.0 / kPi) * (A / B));
    return mu_k / W * kR * (ftr * 1.5 + frot * cvrot + rdm * cvvib);
}

GAS_HD double species_cond(const Tables &t, int k, double T) { return exp(fit_eval(t.fit_cond[k], lnT_x(T))); }
GAS_HD double species_cond_x(const Tables &t, int k, double x) { return exp(fit_eval(t.fit_cond[k], x)); }

// Mixture conductivity (Mathur-Tondon-Saxena average of the species values).
GAS_HD double mix_cond(const Tables &t, const double *X, double T, double P, const double *mu) {
    (void)P;
    (void)mu;
    double s1 = 0.0, s2 = 0.0;
    for (int k = 0; k < t.ns; ++k) {
        const double lk = species_cond(t, k, T);
        s1 += X[k] * lk;
        s2 += X[k] / lk;
    }
    return 0.5 * (s1 + 1.0 / s2);
}

// ---- kinetics ----------------------------------------------------------------------
// The temperature-only factors of the net production rates at one T: the Arrhenius rate
// (k_inf for fall-off reactions), the fall-off k_0 and log10 F_cent (Troe), the reverse
// factor exp(dG/RT - dnu ln(p_atm / R T)) = 1 / K_c, and the species' h/RT and cp/R.  A
// stiff integrator evaluates the rates at many compositions but few temperatures (its
// finite-difference Jacobian perturbs one species at a time), so it computes these once
// per temperature (rate_factors) and the composition-dependent part per call
// (net_production_k); net_production does both, with the same arithmetic.
struct RateT {
    double kf[MAXR], k0[MAXR], lFc[MAXR], er[MAXR];
    double hRT[MAXS], cpR[MAXS];
};

// The temperature-only factors of reaction r (see RateT); k0 and lFc are 0 unless the
// reaction falls off, er is 0 unless it is reversible.
GAS_HD void rate_factor_one(const Tables &t, int r, double T, double logT, double invRT, double log_cref,
                            const double *g_RT, double &kf, double &k0, double &lFc, double &er) {
    const lbmgpu_mech &m = t.m;
    kf = m.A[r] * exp(m.b[r] * logT - m.Ea[r] * invRT);
    k0 = 0.0;
    lFc = 0.0;
    er = 0.0;
    if (m.rtype[r] == LBMGPU_RXN_FALLOFF) {
        k0 = m.A0[r] * exp(m.b0[r] * logT - m.Ea0[r] * invRT);
        if (m.troe_n[r] >= 3) {
            const double a = m.troe[r][0], T3 = m.troe[r][1], T1 = m.troe[r][2];
            double Fc = (1.0 - a) * exp(-T / T3) + a * exp(-T / T1);
            if (m.troe_n[r] == 4) Fc += exp(-m.troe[r][3] / T);
            lFc = log10(fmax(Fc, 1e-300));
        }
    }
    if (m.reversible[r]) {
        double dG = 0.0, dnu = 0.0;
        for (int j = 0; j < m.n_prod[r]; ++j) {
            dG += m.nu_prod[r][j] * g_RT[m.prod[r][j]];
            dnu += m.nu_prod[r][j];
        }
        for (int j = 0; j < m.n_reac[r]; ++j) {
            dG -= m.nu_reac[r][j] * g_RT[m.reac[r][j]];
            dnu -= m.nu_reac[r][j];
        }
        er = exp(dG - dnu * log_cref);
    }
}

GAS_HD void rate_factors(const Tables &t, double T, RateT &K) {
    double g_RT[MAXS];
    for (int k = 0; k < t.ns; ++k) {
        K.hRT[k] = h_RT(t, k, T);
        K.cpR[k] = cp_R(t, k, T);
        g_RT[k] = K.hRT[k] - s_R(t, k, T);
    }
    const double logT = log(T), invRT = 1.0 / (kR * T);
    const double log_cref = log(kOneAtm / (kR * T));
    for (int r = 0; r < t.m.n_reactions; ++r)
        rate_factor_one(t, r, T, logT, invRT, log_cref, g_RT, K.kf[r], K.k0[r], K.lFc[r], K.er[r]);
}

// C^nu of a mass-action factor: a product for the integer orders 1 to 3 (the elementary
// stoichiometries of the mechanisms), otherwise pow of the concentration clipped at zero (a
// fractional order of a global step, or a half-integer stoichiometric coefficient, has no
// real value at the slightly negative concentrations a transported species can take).
GAS_HD double conc_pow(double C, double nu) {
    if (nu == 1.0) return C;
    if (nu == 2.0) return C * C;
    if (nu == 3.0) return C * C * C;
    return pow(fmax(C, 0.0), nu);
}

// Forward and reverse rates of progress (kmol/m^3/s) of reaction r from its temperature
// factors (rate_factor_one) and the concentrations C[k] (kmol/m^3).
GAS_HD void progress_one(const Tables &t, int r, const double *C, double kf, double k0, double lFc, double er,
                         double &fwd_out, double &rev_out) {
    const lbmgpu_mech &m = t.m;
    double M = 1.0;
    if (m.rtype[r] != LBMGPU_RXN_ELEMENTARY) {
        M = 0.0;
        for (int k = 0; k < t.ns; ++k) M += m.eff[r][k] * C[k];
    }
    if (m.rtype[r] == LBMGPU_RXN_FALLOFF) {
        const double Pr = k0 * M / kf;
        double F = 1.0;
        if (m.troe_n[r] >= 3) {
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double x = (lPr + c) / (n - 0.14 * (lPr + c));
            F = pow(10.0, lFc / (1.0 + x * x));
        }
        kf = kf * (Pr / (1.0 + Pr)) * F;
        M = 1.0;
    }
    double fwd = kf * M, rev = 0.0;
    for (int j = 0; j < m.n_reac[r]; ++j) fwd *= conc_pow(C[m.reac[r][j]], m.order_reac[r][j]);
    if (m.reversible[r]) {
        rev = kf * M * er;  // kf / Kc
        for (int j = 0; j < m.n_prod[r]; ++j) rev *= conc_pow(C[m.prod[r][j]], m.nu_prod[r][j]);
    }
    fwd_out = fwd;
    rev_out = rev;
}

// The same from the factors of rate_factors.
GAS_HD void rate_of_progress(const Tables &t, const RateT &K, const double *C, int r, double &fwd_out,
                             double &rev_out) {
    progress_one(t, r, C, K.kf[r], K.k0[r], K.lFc[r], K.er[r], fwd_out, rev_out);
}

// Net molar production rates wdot[k] (kmol/m^3/s) from the factors of rate_factors and
// the concentrations C[k] (kmol/m^3).
GAS_HD void net_production_k(const Tables &t, const RateT &K, const double *C, double *wdot) {
    const lbmgpu_mech &m = t.m;
    for (int k = 0; k < t.ns; ++k) wdot[k] = 0.0;
    for (int r = 0; r < m.n_reactions; ++r) {
        double fwd, rev;
        rate_of_progress(t, K, C, r, fwd, rev);
        const double q = fwd - rev;
        for (int j = 0; j < m.n_reac[r]; ++j) wdot[m.reac[r][j]] -= m.nu_reac[r][j] * q;
        for (int j = 0; j < m.n_prod[r]; ++j) wdot[m.prod[r][j]] += m.nu_prod[r][j] * q;
    }
}

// Net molar production rates wdot[k] (kmol/m^3/s) at (T, concentrations C[k] kmol/m^3).
GAS_HD void net_production(const Tables &t, double T, const double *C, double *wdot) {
    RateT K;
    rate_factors(t, T, K);
    net_production_k(t, K, C, wdot);
}

// Least-squares polynomial fit (degree 4) of y(x) on n points; normal equations solved
// by Gaussian elimination with partial pivoting (host, setup only).
inline void polyfit4(const double *x, const double *y, int n, double *c) {
    double A[5][6] = {};
    for (int i = 0; i < n; ++i) {
        double p[5] = {1.0, x[i], x[i] * x[i], x[i] * x[i] * x[i], x[i] * x[i] * x[i] * x[i]};
        for (int r = 0; r < 5; ++r) {
            for (int q = 0; q < 5; ++q) A[r][q] += p[r] * p[q];
            A[r][5] += p[r] * y[i];
        }
    }
    for (int col = 0; col < 5; ++col) {
        int piv = col;
        for (int r = col + 1; r < 5; ++r)
            if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
        for (int q = 0; q < 6; ++q) {
            const double tmp = A[col][q];
            A[col][q] = A[piv][q];
            A[piv][q] = tmp;
        }
        for (int r = col + 1; r < 5; ++r) {
            const double f = A[r][col] / A[col][col];
            for (int q = col; q < 6; ++q) A[r][q] -= f * A[col][q];
        }
    }
    for (int r = 4; r >= 0; --r) {
        double v = A[r][5];
        for (int q = r + 1; q < 5; ++q) v -= A[r][q] * c[q];
        c[r] = v / A[r][r];
    }
}

// Host-side construction of the derived constants and the transport fits.
inline void make_tables(const lbmgpu_mech &m, Tables &t) {
    make_tables_base(m, t);
    double x[kFitN], y[kFitN];
    const double P = kOneAtm;
    for (int k = 0; k < t.ns; ++k) {
        for (int i = 0; i < kFitN; ++i) {
            const double T = kFitTlo + (kFitThi - kFitTlo) * i / (kFitN - 1);
            x[i] = log(T) - kFitX0;
            y[i] = log(species_visc_kt(t, k, T));
        }
        polyfit4(x, y, kFitN, t.fit_visc[k]);
        for (int i = 0; i < kFitN; ++i) {
            const double T = kFitTlo + (kFitThi - kFitTlo) * i / (kFitN - 1);
            y[i] = log(species_cond_kt(t, k, T, P, species_visc_kt(t, k, T)));
        }
        polyfit4(x, y, kFitN, t.fit_cond[k]);
        for (int j = 0; j < t.ns; ++j) {
            for (int i = 0; i < kFitN; ++i) {
                const double T = kFitTlo + (kFitThi - kFitTlo) * i / (kFitN - 1);
                y[i] = log(binary_diff_kt(t, k, j, T, P) * P);
            }
            polyfit4(x, y, kFitN, t.fit_diff[k][j]);
        }
    }
    for (int a = 0; a < t.ns; ++a)
        for (int b = 0; b < t.ns; ++b) {
            t.sqrt4W[a][b] = sqrt(sqrt(m.W[b] / m.W[a]));
            t.W_ratio_f[a][b] = (float)(m.W[a] / m.W[b]);
            t.wilke_den[a][b] = sqrt(8.0 * (1.0 + m.W[a] / m.W[b]));
            t.inv_wilke_den_f[a][b] = (float)(1.0 / t.wilke_den[a][b]);
        }
    for (int a = 0; a < t.ns; ++a) t.Ra_lat[a] = 0.0;
    for (int r = 0; r < MAXR; ++r) {
        t.dnu[r] = 0.0;
        for (int k = 0; k < MAXS; ++k) t.nu_f[r][k] = t.nu_b[r][k] = t.nu_net[r][k] = t.ord_f[r][k] = 0.0;
    }
    for (int r = 0; r < m.n_reactions; ++r) {
        for (int j = 0; j < m.n_reac[r]; ++j) t.nu_f[r][m.reac[r][j]] += m.nu_reac[r][j];
        for (int j = 0; j < m.n_reac[r]; ++j) t.ord_f[r][m.reac[r][j]] += m.order_reac[r][j];
        for (int j = 0; j < m.n_prod[r]; ++j) t.nu_b[r][m.prod[r][j]] += m.nu_prod[r][j];
        for (int k = 0; k < t.ns; ++k) {
            t.nu_net[r][k] = t.nu_b[r][k] - t.nu_f[r][k];
            t.dnu[r] += t.nu_net[r][k];
        }
    }
}

}  // namespace gas
