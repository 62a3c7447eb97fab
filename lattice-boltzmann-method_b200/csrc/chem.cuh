// Stiff per-cell chemistry over one lattice time step: the constant-volume,
// constant-internal-energy reactor
//     dY_k/dt = wdot_k W_k / rho,
//     dT/dt   = -sum_k e_k wdot_k W_k / (rho c_v),   e_k = h_k - R T / W_k (per mass),
// integrated with the two-stage L-stable Rosenbrock method ROS2 (Verwer, Spee, Blom &
// Hundsdorfer, SIAM J. Sci. Comput. 20 (1999) 1456; gamma = 1 + 1/sqrt 2):
//     (I - gamma h J) k1 = F(y)
//     (I - gamma h J) k2 = F(y + h k1) - 2 k1
//     y+ = y + 3/2 h k1 + 1/2 h k2,   error estimate e = 1/2 h (k1 + k2)  (vs. the embedded
//     first-order y + h k1),
// with a finite-difference Jacobian, a partial-pivot LU of the (nS+1)^2 system in FP64,
// step-size control on the error norm, and a hard cap on the number of sub-steps (the
// caller raises a status bit when it is reached; nothing spins).
#pragma once
#include <math.h>

#include <type_traits>

#include "gas.cuh"

namespace gas {

constexpr int kChemMaxSub = 256;

// right-hand side of the reactor state y = (Y_0..Y_{ns-1}, T) at density rho (kg/m^3),
// with the temperature factors K = rate_factors(t, y[ns])
GAS_HD void reactor_rhs_k(const Tables &t, const RateT &K, double rho, const double *y, double *F) {
    const int ns = t.ns;
    double C[MAXS], w[MAXS];
    const double T = y[ns];
    for (int k = 0; k < ns; ++k) C[k] = rho * y[k] * t.invW[k];
    net_production_k(t, K, C, w);
    double cv = 0.0, s = 0.0;
    for (int k = 0; k < ns; ++k) {
        F[k] = w[k] * t.m.W[k] / rho;
        cv += y[k] * (K.cpR[k] - 1.0) * t.invW[k];
        s += (K.hRT[k] - 1.0) * kR * T * w[k];   // e_k W_k = h_k,molar - R T
    }
    cv *= kR;
    F[ns] = -s / (rho * cv);
}

// The reactor's right-hand side with NS species known at compile time, for the device's
// one-thread-per-cell integrator: the temperature factors of each reaction evaluated inside
// the reaction loop (no per-reaction arrays), log T taken once for the species entropies,
// and the mass-action products and species sums over the dense stoichiometry tables, so that
// every array is indexed by compile-time constants and stays in registers.  The same rate
// laws as net_production; the products and sums run in species order instead of the order
// the reaction lists its species, which moves results by rounding only.
template <int NS>
GAS_HD void reactor_rhs_dense(const Tables &t, double rho, const double *y, double *F) {
    const lbmgpu_mech &m = t.m;
    const double T = y[NS];
    const double logT = log(T), invT = 1.0 / T, invRT = 1.0 / (kR * T);
    const double log_cref = log(kOneAtm / (kR * T));
    double C[NS], w[NS], hRT[NS], gRT[NS], cv = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        const double *a = T < m.T_mid[k] ? m.nasa_lo[k] : m.nasa_hi[k];
        const double cpR = a[0] + T * (a[1] + T * (a[2] + T * (a[3] + T * a[4])));
        cv += y[k] * (cpR - 1.0) * t.invW[k];
        hRT[k] = a[0] + T * (a[1] / 2 + T * (a[2] / 3 + T * (a[3] / 4 + T * a[4] / 5))) + a[5] * invT;
        gRT[k] = hRT[k] - (a[0] * logT + T * (a[1] + T * (a[2] / 2 + T * (a[3] / 3 + T * a[4] / 4))) + a[6]);
        C[k] = rho * y[k] * t.invW[k];
        w[k] = 0.0;
    }
    for (int r = 0; r < m.n_reactions; ++r) {
        double kf = m.A[r] * exp(m.b[r] * logT - m.Ea[r] * invRT);
        double M = 1.0;
        if (m.rtype[r] != LBMGPU_RXN_ELEMENTARY) {
            M = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) M += m.eff[r][k] * C[k];
        }
        if (m.rtype[r] == LBMGPU_RXN_FALLOFF) {
            const double k0 = m.A0[r] * exp(m.b0[r] * logT - m.Ea0[r] * invRT);
            const double Pr = k0 * M / kf;
            double F = 1.0;
            if (m.troe_n[r] >= 3) {
                const double a = m.troe[r][0], T3 = m.troe[r][1], T1 = m.troe[r][2];
                double Fc = (1.0 - a) * exp(-T / T3) + a * exp(-T / T1);
                if (m.troe_n[r] == 4) Fc += exp(-m.troe[r][3] * invT);
                const double lFc = log10(fmax(Fc, 1e-300));
                const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
                const double lPr = log10(fmax(Pr, 1e-300));
                const double x = (lPr + c) / (n - 0.14 * (lPr + c));
                F = pow(10.0, lFc / (1.0 + x * x));
            }
            kf = kf * (Pr / (1.0 + Pr)) * F;
            M = 1.0;
        }
        double fwd = kf * M, rev = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k)
            if (t.ord_f[r][k] != 0.0) fwd *= conc_pow(C[k], t.ord_f[r][k]);
        if (m.reversible[r]) {
            double dG = 0.0;
#pragma unroll
            for (int k = 0; k < NS; ++k) dG += t.nu_net[r][k] * gRT[k];
            rev = kf * M * exp(dG - t.dnu[r] * log_cref);
#pragma unroll
            for (int k = 0; k < NS; ++k)
                if (t.nu_b[r][k] != 0.0) rev *= conc_pow(C[k], t.nu_b[r][k]);
        }
        const double q = fwd - rev;
#pragma unroll
        for (int k = 0; k < NS; ++k) w[k] += t.nu_net[r][k] * q;
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        F[k] = w[k] * m.W[k] / rho;
        s += (hRT[k] - 1.0) * kR * T * w[k];
    }
    cv *= kR;
    F[NS] = -s / (rho * cv);
}

GAS_HD void reactor_rhs(const Tables &t, double rho, const double *y, double *F) {
    RateT K;
    rate_factors(t, y[t.ns], K);
    reactor_rhs_k(t, K, rho, y, F);
}

// LU with partial pivoting of an n x n matrix (row-major, stride MAXS+1); returns false
// on a zero pivot.
GAS_HD bool lu_factor(double (*M)[MAXS + 1], int n, int *piv) {
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (fabs(M[r][c]) > fabs(M[p][c])) p = r;
        piv[c] = p;
        if (M[p][c] == 0.0) return false;
        if (p != c)
            for (int q = 0; q < n; ++q) {
                const double tmp = M[c][q];
                M[c][q] = M[p][q];
                M[p][q] = tmp;
            }
        for (int r = c + 1; r < n; ++r) {
            const double f = M[r][c] / M[c][c];
            M[r][c] = f;
            for (int q = c + 1; q < n; ++q) M[r][q] -= f * M[c][q];
        }
    }
    return true;
}

// The iteration matrix of the compile-time-sized integrators: an N x N array of the thread
// (registers, or local memory where the pivoting indexes it), or a view of the thread's
// matrix in shared memory, element (r, c) at p[(r N + c) stride] so that the threads of a
// warp touch consecutive words.
template <int N>
struct RegMat {
    double a[N][N];
    GAS_HD double &operator()(int r, int c) { return a[r][c]; }
    GAS_HD double operator()(int r, int c) const { return a[r][c]; }
};
template <int N>
struct SharedMat {
    double *p;
    int stride;
    GAS_HD double &operator()(int r, int c) const { return p[(r * N + c) * stride]; }
};

// lu_factor / lu_solve for a matrix of compile-time size N (the device integrator): the same
// partial pivoting and elimination, each pivot inverted once (dinv) so that the multipliers and
// the back substitution multiply instead of dividing.  Every loop is unrolled, so piv, dinv
// and b are indexed by constants only: a row interchange with a register matrix, and the
// interchanges applied to b, select among the candidate rows instead of indexing by the
// pivot (an index known only at run time would put the array in local memory).
template <class Mat>
struct MatRowsAddressable : std::false_type {};
template <int N>
struct MatRowsAddressable<SharedMat<N>> : std::true_type {};

template <int N, class Mat>
GAS_HD bool lu_factor_n(Mat &M, int *piv, double *dinv) {
#pragma unroll
    for (int c = 0; c < N; ++c) {
        int p = c;
        double best = fabs(M(c, c));
#pragma unroll
        for (int r = c + 1; r < N; ++r) {
            const double v = fabs(M(r, c));
            if (v > best) {
                best = v;
                p = r;
            }
        }
        piv[c] = p;
        if (best == 0.0) return false;
        if (p != c) {
            if constexpr (MatRowsAddressable<Mat>::value) {
#pragma unroll
                for (int q = 0; q < N; ++q) {
                    const double tmp = M(c, q);
                    M(c, q) = M(p, q);
                    M(p, q) = tmp;
                }
            } else {
#pragma unroll
                for (int r = c + 1; r < N; ++r)
                    if (r == p)
#pragma unroll
                        for (int q = 0; q < N; ++q) {
                            const double tmp = M(c, q);
                            M(c, q) = M(r, q);
                            M(r, q) = tmp;
                        }
            }
        }
        const double inv = 1.0 / M(c, c);
        dinv[c] = inv;
#pragma unroll
        for (int r = c + 1; r < N; ++r) {
            const double f = M(r, c) * inv;
            M(r, c) = f;
#pragma unroll
            for (int q = c + 1; q < N; ++q) M(r, q) -= f * M(c, q);
        }
    }
    return true;
}
template <int N, class Mat>
GAS_HD void lu_solve_n(const Mat &M, const int *piv, const double *dinv, double *b) {
#pragma unroll
    for (int c = 0; c < N; ++c) {
        const int p = piv[c];
#pragma unroll
        for (int q = c + 1; q < N; ++q)
            if (q == p) {
                const double tmp = b[c];
                b[c] = b[q];
                b[q] = tmp;
            }
    }
#pragma unroll
    for (int r = 1; r < N; ++r)
#pragma unroll
        for (int q = 0; q < r; ++q) b[r] -= M(r, q) * b[q];
#pragma unroll
    for (int r = N - 1; r >= 0; --r) {
        double v = b[r];
#pragma unroll
        for (int q = r + 1; q < N; ++q) v -= M(r, q) * b[q];
        b[r] = v * dinv[r];
    }
}

// The factorisation swaps whole rows (multipliers included), so all interchanges are
// applied to b before the forward substitution.
GAS_HD void lu_solve(const double (*M)[MAXS + 1], int n, const int *piv, double *b) {
    for (int c = 0; c < n; ++c) {
        const double tmp = b[c];
        b[c] = b[piv[c]];
        b[piv[c]] = tmp;
    }
    for (int r = 1; r < n; ++r)
        for (int q = 0; q < r; ++q) b[r] -= M[r][q] * b[q];
    for (int r = n - 1; r >= 0; --r) {
        double v = b[r];
        for (int q = r + 1; q < n; ++q) v -= M[r][q] * b[q];
        b[r] = v / M[r][r];
    }
}

// Advances (Y, T) over dt seconds at constant density rho.  Returns the number of
// accepted sub-steps, or -1 if the sub-step cap was reached (state is left at the last
// accepted point).
GAS_HD int ros2_advance(const Tables &t, double rho, double *Y, double &T, double dt, double rtol = 1e-5,
                        double atol = 1e-10, double atol_T = 1e-3) {
    const int ns = t.ns, n = ns + 1;
    const double gam = 1.0 + 1.0 / sqrt(2.0);
    double y[MAXS + 1], F0[MAXS + 1], Fp[MAXS + 1], yp[MAXS + 1], k1[MAXS + 1], k2[MAXS + 1];
    double M[MAXS + 1][MAXS + 1];
    int piv[MAXS + 1];
    for (int k = 0; k < ns; ++k) y[k] = Y[k];
    y[ns] = T;
    double tt = 0.0, h = dt;
    int acc = 0;
    bool done = false;
    for (int it = 0; it < kChemMaxSub && !done; ++it) {
        const bool last = tt + h >= dt;
        if (last) h = dt - tt;
        // the temperature factors at y serve F0 and the species columns; the temperature
        // column and the second stage take their own
        RateT K;
        rate_factors(t, y[ns], K);
        reactor_rhs_k(t, K, rho, y, F0);
        // finite-difference Jacobian, column by column
        for (int c = 0; c < n; ++c) {
            for (int q = 0; q < n; ++q) yp[q] = y[q];
            const double eps = c < ns ? 1e-8 * fmax(fabs(y[c]), 1e-6) : 1e-7 * y[c];
            yp[c] += eps;
            if (c == ns) rate_factors(t, yp[ns], K);
            reactor_rhs_k(t, K, rho, yp, Fp);
            for (int r = 0; r < n; ++r) M[r][c] = -gam * h * (Fp[r] - F0[r]) / eps;
        }
        for (int r = 0; r < n; ++r) M[r][r] += 1.0;
        if (!lu_factor(M, n, piv)) {
            h *= 0.25;
            continue;
        }
        for (int q = 0; q < n; ++q) k1[q] = F0[q];
        lu_solve(M, n, piv, k1);
        for (int q = 0; q < n; ++q) yp[q] = y[q] + h * k1[q];
        rate_factors(t, yp[ns], K);
        reactor_rhs_k(t, K, rho, yp, Fp);
        for (int q = 0; q < n; ++q) k2[q] = Fp[q] - 2.0 * k1[q];
        lu_solve(M, n, piv, k2);
        double err = 0.0;
        for (int q = 0; q < n; ++q) {
            const double ynew = y[q] + 1.5 * h * k1[q] + 0.5 * h * k2[q];
            const double sc = (q < ns ? atol : atol_T) + rtol * fmax(fabs(y[q]), fabs(ynew));
            const double e = 0.5 * h * (k1[q] + k2[q]) / sc;
            err = fmax(err, fabs(e));
            yp[q] = ynew;
        }
        if (err <= 1.0) {
            for (int q = 0; q < n; ++q) y[q] = yp[q];
            tt = last ? dt : tt + h;  // the last step lands on dt exactly
            done = last;
            ++acc;
        }
        // second-order controller with safety factor, growth limited to 4x, shrink to 1/5
        const double fac = err > 0.0 ? 0.9 / sqrt(err) : 4.0;
        h *= fmin(4.0, fmax(0.2, fac));
    }
    for (int k = 0; k < ns; ++k) Y[k] = y[k];
    T = y[ns];
    return done ? acc : -1;
}

// The kinetics policies ros2_advance_k takes: `K` what is formed once per temperature,
// `factors(T, K)` forms it, `rhs(K, rho, y, F)` is the reactor's right-hand side at y from K at
// y's temperature; with kAnalyticJacobian, `rhs_jacobian(K, rho, y, F, s, J)` writes that
// right-hand side and s times the Jacobian dF/d(Y, T) (its columns are finite differences
// otherwise).  TableKinetics evaluates any mechanism from the tables, recomputing its factors
// inside each right-hand side (reactor_rhs_dense: nothing per reaction kept between calls); a
// mechanism compiled to straight-line code (gen_kinetics.py) provides its own policy, whose K
// is the species' thermo and whose rate constants are formed reaction by reaction.
template <int NS>
struct TableKinetics {
    static constexpr bool kAnalyticJacobian = false;
    const Tables &t;
    struct K {};
    GAS_HD void factors(double, K &) const {}
    GAS_HD void rhs(const K &, double rho, const double *y, double *F) const { reactor_rhs_dense<NS>(t, rho, y, F); }
};

// The tables with the temperature factors kept between right-hand sides (rate_factors +
// reactor_rhs_k, ros2_advance's evaluation): one RateT per temperature, which a thread holds in
// local memory.
struct CachedTableKinetics {
    static constexpr bool kAnalyticJacobian = false;
    const Tables &t;
    using K = RateT;
    GAS_HD void factors(double T, RateT &k) const { rate_factors(t, T, k); }
    GAS_HD void rhs(const RateT &k, double rho, const double *y, double *F) const { reactor_rhs_k(t, k, rho, y, F); }
};

// The unknowns of ros2_advance_km's iteration system: every component of (Y_0..Y_{NS-1}, T),
// unless the kinetics policy names fewer (kSys, and sys_full(i) the state component of unknown
// i, ascending, T last).  A species whose net stoichiometric coefficient is zero in every
// reaction (N2 in the H2/air mechanism) has a zero right-hand side and a zero Jacobian row: its
// row of I - gamma h J is the identity row, so its stage increments are zero and its column,
// which multiplies them, drops out as well.
template <class Kin, int N, class = void>
struct SysMap {
    static constexpr int size = N;
    GAS_HD static constexpr int full(int i) { return i; }
};
template <class Kin, int N>
struct SysMap<Kin, N, std::void_t<decltype(Kin::kSys)>> {
    static constexpr int size = Kin::kSys;
    GAS_HD static constexpr int full(int i) { return Kin::sys_full(i); }
};

// ros2_advance with the species count known at compile time and the kinetics a policy, for
// the device's one-thread-per-cell kernels: the same method, step control, factorisation and
// sequence of right-hand sides (the species columns of the Jacobian at the unperturbed
// temperature's factors, the temperature column and the second stage at their own), its
// vectors sized and its loops unrolled so that they stay in registers.  A policy with an
// analytic Jacobian replaces the finite differences and their right-hand sides (ROS2 is a
// W-method: its order holds for any Jacobian approximation, so the two differ by the
// differences' truncation and rounding in the step-size decisions).
template <int NS, class Kin, class Mat>
GAS_HD int ros2_advance_km(const Kin &kin, Mat &M, double rho, double *Y, double &T, double dt, double rtol = 1e-5,
                           double atol = 1e-10, double atol_T = 1e-3) {
    constexpr int ns = NS, n = NS + 1;
    using Sys = SysMap<Kin, n>;
    constexpr int m = Sys::size;  // unknowns of the iteration system (M is m x m)
    const double gam = 1.0 + 1.0 / sqrt(2.0);
    double y[n], F0[n], Fp[n], yp[n], k1[m], k2[m], dinv[m];
    int piv[m];
    for (int k = 0; k < ns; ++k) y[k] = Y[k];
    y[ns] = T;
    double tt = 0.0, h = dt;
    int acc = 0;
    bool done = false;
    for (int it = 0; it < kChemMaxSub && !done; ++it) {
        const bool last = tt + h >= dt;
        if (last) h = dt - tt;
        // one set of temperature factors, formed at y, then at the temperature column's (finite
        // differences) and the second stage's temperatures in turn
        typename Kin::K Kf;
        kin.factors(y[ns], Kf);
        if constexpr (Kin::kAnalyticJacobian) {
            kin.rhs_jacobian(Kf, rho, y, F0, -gam * h, M);
        } else {
            static_assert(m == n, "finite-difference Jacobians cover the whole state");
            kin.rhs(Kf, rho, y, F0);
            // the species columns in a rolled loop (one inlined right-hand side); the perturbed
            // component is selected by comparison so that yp stays in registers
#pragma unroll 1
            for (int c = 0; c < ns; ++c) {
                double yc = y[0];
#pragma unroll
                for (int q = 1; q < ns; ++q)
                    if (q == c) yc = y[q];
                const double eps = 1e-8 * fmax(fabs(yc), 1e-6);
#pragma unroll
                for (int q = 0; q < n; ++q) yp[q] = q == c ? y[q] + eps : y[q];
                kin.rhs(Kf, rho, yp, Fp);
#pragma unroll
                for (int r = 0; r < n; ++r) M(r, c) = -gam * h * (Fp[r] - F0[r]) / eps;
            }
        }
        if constexpr (!Kin::kAnalyticJacobian) {  // the temperature column
            const double eps = 1e-7 * y[ns];
#pragma unroll
            for (int q = 0; q < n; ++q) yp[q] = y[q];
            yp[ns] += eps;
            kin.factors(yp[ns], Kf);
            kin.rhs(Kf, rho, yp, Fp);
#pragma unroll
            for (int r = 0; r < n; ++r) M(r, ns) = -gam * h * (Fp[r] - F0[r]) / eps;
        }
        for (int r = 0; r < m; ++r) M(r, r) += 1.0;
        if (!lu_factor_n<m>(M, piv, dinv)) {
            h *= 0.25;
            continue;
        }
#pragma unroll
        for (int q = 0; q < m; ++q) k1[q] = F0[Sys::full(q)];
        lu_solve_n<m>(M, piv, dinv, k1);
#pragma unroll
        for (int q = 0; q < n; ++q) yp[q] = y[q];
#pragma unroll
        for (int q = 0; q < m; ++q) yp[Sys::full(q)] = y[Sys::full(q)] + h * k1[q];
        kin.factors(yp[ns], Kf);
        kin.rhs(Kf, rho, yp, Fp);
#pragma unroll
        for (int q = 0; q < m; ++q) k2[q] = Fp[Sys::full(q)] - 2.0 * k1[q];
        lu_solve_n<m>(M, piv, dinv, k2);
        double err = 0.0;
#pragma unroll
        for (int q = 0; q < m; ++q) {
            const int c = Sys::full(q);
            const double ynew = y[c] + 1.5 * h * k1[q] + 0.5 * h * k2[q];
            const double sc = (c < ns ? atol : atol_T) + rtol * fmax(fabs(y[c]), fabs(ynew));
            const double e = 0.5 * h * (k1[q] + k2[q]) / sc;
            err = fmax(err, fabs(e));
            yp[c] = ynew;
        }
        if (err <= 1.0) {
#pragma unroll
            for (int q = 0; q < n; ++q) y[q] = yp[q];
            tt = last ? dt : tt + h;
            done = last;
            ++acc;
        }
        const double fac = err > 0.0 ? 0.9 / sqrt(err) : 4.0;
        h *= fmin(4.0, fmax(0.2, fac));
    }
    for (int k = 0; k < ns; ++k) Y[k] = y[k];
    T = y[ns];
    return done ? acc : -1;
}

// ros2_advance_km with the iteration matrix in the thread's own array.
template <int NS, class Kin>
GAS_HD int ros2_advance_k(const Kin &kin, double rho, double *Y, double &T, double dt, double rtol = 1e-5,
                          double atol = 1e-10, double atol_T = 1e-3) {
    RegMat<SysMap<Kin, NS + 1>::size> M;
    return ros2_advance_km<NS>(kin, M, rho, Y, T, dt, rtol, atol, atol_T);
}

// ros2_advance_k over the tables of any mechanism of NS species.
template <int NS>
GAS_HD int ros2_advance_n(const Tables &t, double rho, double *Y, double &T, double dt, double rtol = 1e-5,
                          double atol = 1e-10, double atol_T = 1e-3) {
    return ros2_advance_k<NS>(TableKinetics<NS>{t}, rho, Y, T, dt, rtol, atol, atol_T);
}

#if defined(__CUDACC__)
// ros2_advance for one cell by a group of G lanes (G a power of two <= 32, the group's
// lanes consecutive and aligned within the warp; every lane passes the same arguments).
// The n + 1 right-hand sides of a sub-step's finite-difference Jacobian (column c
// perturbed, c < n, and the unperturbed one, index n) are dealt out round robin, index
// j to lane j % G; each lane then assembles the Jacobian from the group's columns by
// shuffles and runs the same factorisation, stages and step control -- the arithmetic of
// ros2_advance_k value for value, with the Jacobian's evaluations side by side.  The
// kinetics policy as for ros2_advance_k; CachedTableKinetics gives ros2_advance's values.
template <int NS, int G, class Kin>
__device__ int ros2_advance_group(const Kin &kin, double rho, double *Y, double &T, double dt, double rtol = 1e-5,
                                  double atol = 1e-10, double atol_T = 1e-3) {
    constexpr int ns = NS, n = NS + 1;
    constexpr int kPer = (n + G) / G;  // right-hand sides per lane, at most
    const int lane = (int)(threadIdx.x & 31u), g = lane & (G - 1);
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (lane & ~(G - 1));
    const double gam = 1.0 + 1.0 / sqrt(2.0);
    double y[n], F0[n], Fp[n], yp[n], k1[n], k2[n];
    double Fc[kPer][n], ec[kPer];  // this lane's right-hand sides and their steps
    RegMat<n> M;
    double dinv[n];
    int piv[n];
    for (int k = 0; k < ns; ++k) y[k] = Y[k];
    y[ns] = T;
    double tt = 0.0, h = dt;
    int acc = 0;
    bool done = false;
    for (int it = 0; it < kChemMaxSub && !done; ++it) {
        const bool last = tt + h >= dt;
        if (last) h = dt - tt;
        typename Kin::K K0;
        bool k_at_y = false;  // K0 holds the factors at y's temperature
#pragma unroll
        for (int m = 0; m < kPer; ++m) {
            const int c = g + m * G;  // column c < n, or the unperturbed right-hand side c == n
            if (c > n) break;
            double yc = y[0];
#pragma unroll
            for (int q = 1; q < n; ++q)
                if (q == c) yc = y[q];
            double eps = 1.0;
            if (c < n) eps = c < ns ? 1e-8 * fmax(fabs(yc), 1e-6) : 1e-7 * yc;
#pragma unroll
            for (int q = 0; q < n; ++q) yp[q] = q == c ? y[q] + eps : y[q];
            ec[m] = eps;
            if (c == ns) {
                typename Kin::K Kt;
                kin.factors(yp[ns], Kt);
                kin.rhs(Kt, rho, yp, Fc[m]);
            } else {
                if (!k_at_y) {
                    kin.factors(y[ns], K0);
                    k_at_y = true;
                }
                kin.rhs(K0, rho, yp, Fc[m]);
            }
        }
#pragma unroll
        for (int r = 0; r < n; ++r) F0[r] = __shfl_sync(gmask, Fc[n / G][r], n % G, G);
#pragma unroll
        for (int m = 0; m < kPer; ++m)  // this lane's Jacobian columns
            if (g + m * G < n)
#pragma unroll
                for (int r = 0; r < n; ++r) Fc[m][r] = -gam * h * (Fc[m][r] - F0[r]) / ec[m];
#pragma unroll
        for (int c = 0; c < n; ++c)
#pragma unroll
            for (int r = 0; r < n; ++r) M(r, c) = __shfl_sync(gmask, Fc[c / G][r], c % G, G);
        for (int r = 0; r < n; ++r) M(r, r) += 1.0;
        if (!lu_factor_n<n>(M, piv, dinv)) {
            h *= 0.25;
            continue;
        }
#pragma unroll
        for (int q = 0; q < n; ++q) k1[q] = F0[q];
        lu_solve_n<n>(M, piv, dinv, k1);
#pragma unroll
        for (int q = 0; q < n; ++q) yp[q] = y[q] + h * k1[q];
        {
            typename Kin::K K2;
            kin.factors(yp[ns], K2);
            kin.rhs(K2, rho, yp, Fp);
        }
#pragma unroll
        for (int q = 0; q < n; ++q) k2[q] = Fp[q] - 2.0 * k1[q];
        lu_solve_n<n>(M, piv, dinv, k2);
        double err = 0.0;
#pragma unroll
        for (int q = 0; q < n; ++q) {
            const double ynew = y[q] + 1.5 * h * k1[q] + 0.5 * h * k2[q];
            const double sc = (q < ns ? atol : atol_T) + rtol * fmax(fabs(y[q]), fabs(ynew));
            const double e = 0.5 * h * (k1[q] + k2[q]) / sc;
            err = fmax(err, fabs(e));
            yp[q] = ynew;
        }
        if (err <= 1.0) {
#pragma unroll
            for (int q = 0; q < n; ++q) y[q] = yp[q];
            tt = last ? dt : tt + h;
            done = last;
            ++acc;
        }
        const double fac = err > 0.0 ? 0.9 / sqrt(err) : 4.0;
        h *= fmin(4.0, fmax(0.2, fac));
    }
    for (int k = 0; k < ns; ++k) Y[k] = y[k];
    T = y[ns];
    return done ? acc : -1;
}
#endif

}  // namespace gas
