// Multicomponent boundary cells ("special": a fluid cell with a solid, adiabatic,
// free-slip, inflow or outflow cell upstream along some direction): streaming with the
// reference's per-type rules, the Tamm-Mott-Smith boundary treatment (characteristic
// outflow with NSCBC, characteristic inflow with the inline LODI relaxation, solid wall),
// then the moments.  Host/device, like mc_cell.cuh.
//
// Reference path (farrasarira/Lattice-Boltzmann-Method, MULTICOMP on):
//   LBM::Streaming                      src/lbm-streaming.cpp:3-119
//   LBM::TMS_BC outflow pass            src/lbm-bc.cpp:126-340   (TYPE_O_C branch)
//   LBM::TMS_BC inflow pass             src/lbm-bc.cpp:463-808   (TYPE_I_C branch)
//   LBM::TMS_BC solid pass              src/lbm-bc.cpp:941-1110
//   impose_NSCBC and its helpers        src/impose_nscbc.cpp:45-546
//   calculate_feq_geq (multicomponent)  src/lbm-edf.cpp:168-209
//   calculate_temp                      src/lbm-moment.cpp:540-553
//   fd_uw                               src/FD.cpp:64-74
// Within one cell the passes run in the reference's order (outflow, inflow, solid); they
// read the previous step's record of the cell and its neighbours and no other cell's
// populations, so a per-cell kernel reproduces the reference's sweep.  The reference's
// non-characteristic TYPE_O / TYPE_I treatment rewrites a neighbour's moments in place
// from inside the sweep (calculate_moment_point), which makes it order dependent; those
// two types are not accepted by this path.
#pragma once
#include "mc_cell.cuh"

namespace lbm {

constexpr double kNscbcSigmaOut = 0.25;  // NSCBC_SIGMA_OUT, src/headers/defines.hpp:101
constexpr double kLodiSigmaIn = 5.0;     // sigma of the inline LODI inflow, src/lbm-bc.cpp:520

template <class AT>
MC_HD int mc_type_at(const AT &A, int i, int j, int k) {
    return A.type[(long)i * A.si + (long)j * A.sj + k];
}
template <class AT>
MC_HD long mc_idx(const AT &A, int i, int j, int k) {
    return (long)i * A.si + (long)j * A.sj + k;
}

// calculate_feq_geq of the multicomponent build (src/lbm-edf.cpp:168-195): the per-axis
// factors of every species' target set (velocity vela[a], theta_a = R T / W_a) and of
// the energy set (velocity vel, theta = R T / W, internal energy of the state); the
// Cantera state is (T, rho, Y = rhoa / rho).  Returns T in SI, the temperature the
// reference's Cantera object is left at.
template <int NS>
MC_HD double mc_target_axes(const gas::Tables &t, const UnitsF &U, double rho, const double *rhoa,
                            const double vel[3], const double (*vela)[3], double T_lat, AxisF<double> *Fa,
                            AxisG<double> &G) {
    double y[NS], Y[NS], X[NS];
    for (int a = 0; a < NS; ++a) y[a] = rhoa[a] / rho;
    const double W = set_mass_fractions<NS>(t, y, Y, X);
    const double T_si = si_temp(U, (float)T_lat);
    const double e = u_energy_mass(U, (float)gas::int_energy_mass(t, Y, T_si));
    const double theta = u_energy_mass(U, (float)(gas::kR * T_si / W));
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < NS; ++a) {
        const double tha = u_energy_mass(U, (float)(gas::kR * T_si / t.m.W[a]));
        axis_feq(Fa[a], vela ? vela[a] : vel, tha, zero);
    }
    axis_geq(G, e, theta, vel);
    return T_si;
}

// calculate_temp (src/lbm-moment.cpp:540-553): T from the internal energy per mass and
// the composition rho_a / rho; the Newton iteration of setState_UV starts from T0_si
// (the state the Cantera object holds) with Cantera 3's default tolerance (1e-9).
template <int NS, class AT>
MC_HD double mc_calc_temp(const AT &A, double Uint, double rho, const double *rhoa, double T0_si) {
    double y[NS], Y[NS], X[NS];
    for (int a = 0; a < NS; ++a) y[a] = rhoa[a] / rho;
    set_mass_fractions<NS>(*A.tab, y, Y, X);
    double T;
    if (gas::T_from_u(*A.tab, Y, si_energy_mass(A.U, (float)Uint), T0_si, 1e-9, 100, T) < 0)
        atomic_status(A.status, LBMGPU_ST_NEWTON);
    return u_temp(A.U, (float)T);
}

// The Cantera state set by (setMassFractions(rho_a/rho), setState_DP(rho, p)) of a
// record entry: T, frozen sound speed (lattice units), cp/cv and the mixture gas
// constant in lattice units.
struct McDP {
    double T, c, gamma, Rmix;
};
template <int NS>
MC_HD McDP mc_state_dp(const gas::Tables &t, const UnitsF &U, double rho_l, double p_l, const double *y) {
    double Y[NS], X[NS];
    const double W = set_mass_fractions<NS>(t, y, Y, X);
    McDP s;
    const double rho_si = si_rho(U, (float)rho_l);
    const double P_si = si_p(U, (float)p_l);
    s.T = P_si * W / (rho_si * gas::kR);
    const double cp = gas::cp_mass(t, Y, s.T), cv = gas::cv_mass(t, Y, s.T);
    s.c = u_u(U, (float)sqrt(cp / cv * gas::kR * s.T / W));
    s.gamma = cp / cv;
    s.Rmix = u_cp(U, (float)(gas::kR / W));
    return s;
}

// The macroscopic fields the boundary formulas read from the previous step's record.
struct McFields {
    double rho, u[3], p, T;
};
template <class AT>
MC_HD McFields mc_fields(const AT &A, long m) {
    const typename AT::R *R = A.rec_cur;
    McFields f;
    f.rho = rec(A, R, RM_RHO, m);
    f.u[0] = rec(A, R, RM_U, m);
    f.u[1] = rec(A, R, RM_V, m);
    f.u[2] = rec(A, R, RM_W, m);
    f.p = rec(A, R, RM_P, m);
    f.T = rec(A, R, RM_T, m);
    return f;
}
template <int NS, class AT>
MC_HD void mc_Y_of(const AT &A, long m, double *y) {
    const double r = rec(A, A.rec_cur, RM_RHO, m);
    for (int a = 0; a < NS; ++a) y[a] = rec(A, A.rec_cur, rs(a, RS_RHO), m) / r;
}

// Derivatives of (p, u, v, w, rho, Y_a) along axis d (impose_nscbc.cpp:111-166 and
// :168-276): one-sided second order (mode +1 forward, -1 backward) or central (mode 0).
template <int NS, class AT>
MC_HD void mc_deriv(const AT &A, int i, int j, int k, int d, int mode, double D[5], double *dY) {
    const int e[3] = {d == 0, d == 1, d == 2};
    auto at = [&](int s) { return mc_idx(A, i + s * e[0], j + s * e[1], k + s * e[2]); };
    const typename AT::R *R = A.rec_cur;
    const int pl[5] = {RM_P, RM_U, RM_V, RM_W, RM_RHO};
    if (mode == 1) {
        const long m0 = at(0), m1 = at(1), m2 = at(2);
        for (int q = 0; q < 5; ++q)
            D[q] = (-1.5 * rec(A, R, pl[q], m0) + 2.0 * rec(A, R, pl[q], m1) - 0.5 * rec(A, R, pl[q], m2)) / 1.0;
        for (int a = 0; a < NS; ++a)
            dY[a] = (-1.5 * rec(A, R, rs(a, RS_RHO), m0) / rec(A, R, RM_RHO, m0) +
                     2.0 * rec(A, R, rs(a, RS_RHO), m1) / rec(A, R, RM_RHO, m1) -
                     0.5 * rec(A, R, rs(a, RS_RHO), m2) / rec(A, R, RM_RHO, m2)) /
                    1.0;
    } else if (mode == -1) {
        const long m0 = at(0), m1 = at(-1), m2 = at(-2);
        for (int q = 0; q < 5; ++q)
            D[q] = (1.5 * rec(A, R, pl[q], m0) - 2.0 * rec(A, R, pl[q], m1) + 0.5 * rec(A, R, pl[q], m2)) / 1.0;
        for (int a = 0; a < NS; ++a)
            dY[a] = (1.5 * rec(A, R, rs(a, RS_RHO), m0) / rec(A, R, RM_RHO, m0) -
                     2.0 * rec(A, R, rs(a, RS_RHO), m1) / rec(A, R, RM_RHO, m1) +
                     0.5 * rec(A, R, rs(a, RS_RHO), m2) / rec(A, R, RM_RHO, m2)) /
                    1.0;
    } else {
        const long mp = at(1), mm = at(-1);
        for (int q = 0; q < 5; ++q) D[q] = (rec(A, R, pl[q], mp) - rec(A, R, pl[q], mm)) / (2.0 * 1.0);
        for (int a = 0; a < NS; ++a)
            dY[a] = (rec(A, R, rs(a, RS_RHO), mp) / rec(A, R, RM_RHO, mp) -
                     rec(A, R, rs(a, RS_RHO), mm) / rec(A, R, RM_RHO, mm)) /
                    (2.0 * 1.0);
    }
}

// impose_NSCBC for a TYPE_O_C ghost (impose_nscbc.cpp:45-110, compute_waves :315-391,
// update_bc_cells :477-546): the boundary cell's state advanced one step with the LODI
// relations, the incoming acoustic wave replaced by the pressure relaxation toward the
// ghost's pressure with the transverse correction of Yoo & Im.  idir: axis 0..2 of the
// boundary normal, isign: its direction into the domain.
template <int NS, class AT>
MC_HD void mc_nscbc_outflow(const AT &A, int i, int j, int k, int idir, int isign, double &rho_out, double *rhoa_out,
                            double vel_out[3], double &T_out) {
    const gas::Tables &t = *A.tab;
    const long n = mc_idx(A, i, j, k);
    const McFields c0 = mc_fields(A, n);
    const int Nax[3] = {A.Nx_glob, A.Ny, A.Nz};  // the domain's lengths (x: the whole decomposed domain)
    const int ijk[3] = {i, j, k};
    // derivatives: [axis][p, u, v, w, rho]
    double D[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}, {0, 0, 0, 0, 0}};
    double dYn[NS], dYt[NS];
    mc_deriv<NS>(A, i, j, k, idir, isign, D[idir], dYn);
    bool any_t = false;
    for (int d = 0; d < 3; ++d) {
        if (d == idir || !(Nax[d] - 2 > 3)) continue;
        any_t = true;
        int mode;
        int lo[3] = {i, j, k}, hi[3] = {i, j, k};
        lo[d] -= 1;
        hi[d] += 1;
        if (mc_type_at(A, lo[0], lo[1], lo[2]) != T_F)
            mode = 1;
        else if (d != 2 && mc_type_at(A, hi[0], hi[1], hi[2]) != T_F)
            mode = -1;  // the z branch of the reference tests k-1 twice, so never this case
        else
            mode = 0;
        (void)ijk;
        mc_deriv<NS>(A, i, j, k, d, mode, D[d], dYt);
    }
    double y[NS];
    mc_Y_of<NS>(A, n, y);
    const McDP st = mc_state_dp<NS>(t, A.U, c0.rho, c0.p, y);
    const double c = st.c, rho = c0.rho, p = c0.p;
    const double u = c0.u[0], v = c0.u[1], w = c0.u[2];
    // transverse terms T1, T5 (compute_tranverse_terms, impose_nscbc.cpp:278-313)
    double T1 = 0.0, T5 = 0.0;
    if (any_t) {
        const double gam = st.gamma;
        // D[axis][0 p, 1 u, 2 v, 3 w]
        if (idir == 0) {
            T1 = (v * (D[1][0] - rho * c * D[1][1])) + (w * (D[2][0] - rho * c * D[2][1])) +
                 (gam * p * (D[1][2] + D[2][3]));
            T5 = (v * (D[1][0] + rho * c * D[1][1])) + (w * (D[2][0] + rho * c * D[2][1])) +
                 (gam * p * (D[1][2] + D[2][3]));
        } else if (idir == 1) {
            T1 = (u * (D[0][0] - rho * c * D[0][2])) + (w * (D[2][0] - rho * c * D[2][2])) +
                 (gam * p * (D[0][1] + D[2][3]));
            T5 = (u * (D[0][0] + rho * c * D[0][2])) + (w * (D[2][0] + rho * c * D[2][2])) +
                 (gam * p * (D[0][1] + D[2][3]));
        } else {
            T1 = (u * (D[0][0] - rho * c * D[0][3])) + (v * (D[1][0] - rho * c * D[1][3])) +
                 (gam * p * (D[0][1] + D[1][2]));
            T5 = (u * (D[0][0] + rho * c * D[0][3])) + (v * (D[1][0] + rho * c * D[1][3])) +
                 (gam * p * (D[0][1] + D[1][2]));
        }
    }
    // waves (compute_waves)
    const double mach = sqrt(u * u + v * v + w * w) / c;
    const double un = c0.u[idir];
    const double dp = D[idir][0], dun = D[idir][1 + idir], drho = D[idir][4];
    double L1 = (un - c) * (dp - rho * c * dun);
    double L5 = (un + c) * (dp + rho * c * dun);
    const double Ls = un * (c * c * drho - dp);
    double Lt[3];  // L2, L3, L4
    for (int d = 0; d < 3; ++d) Lt[d] = (d == idir) ? Ls : un * D[idir][1 + d];
    double L6[NS];
    for (int a = 0; a < NS; ++a) L6[a] = un * dYn[a];
    int gb[3] = {i, j, k};
    gb[idir] -= isign;
    const double P_target = rec(A, A.rec_cur, RM_P, mc_idx(A, gb[0], gb[1], gb[2]));
    const double beta = mach;
    if (mach < 1.0) {
        const double Kout = kNscbcSigmaOut * (1.0 - mach * mach) * (c / Nax[idir]);
        if (isign == 1)
            L5 = Kout * (p - P_target) - (1.0 - beta) * T5;
        else
            L1 = Kout * (p - P_target) - (1.0 - beta) * T1;
    }
    // update of the boundary cell (update_bc_cells)
    const double dt = A.dt;
    double dv[3];
    const double drho_t = (Lt[idir] + 0.5 * (L1 + L5)) / (c * c);
    for (int d = 0; d < 3; ++d) dv[d] = (d == idir) ? (L5 - L1) / (2.0 * c * rho) : Lt[d];
    const double dpt = 0.5 * (L1 + L5);
    rho_out = rho - dt * drho_t;
    for (int d = 0; d < 3; ++d) vel_out[d] = c0.u[d] - dt * dv[d];
    const double p_out = p - dt * dpt;
    for (int a = 0; a < NS; ++a) rhoa_out[a] = (y[a] - dt * L6[a]) * rho_out;
    double y2[NS], Y2[NS], X2[NS];
    for (int a = 0; a < NS; ++a) y2[a] = rhoa_out[a] / rho_out;
    const double W2 = set_mass_fractions<NS>(t, y2, Y2, X2);
    const double T = (double)si_p(A.U, (float)p_out) * W2 / ((double)si_rho(A.U, (float)rho_out) * gas::kR);
    T_out = u_temp(A.U, (float)T);
}

// fd_uw (src/FD.cpp:64-74): first-order one-sided difference into the domain.
MC_HD double mc_fd_uw(double s0, double s1, double vel) { return vel < 0 ? (s0 - s1) / 1.0 : (-s0 + s1) / 1.0; }

// The inline LODI inflow of a TYPE_I_C ghost (src/lbm-bc.cpp:519-690) and the common
// constant-(T, p) re-evaluation of the inflow state (:676-690).
template <int NS, class AT>
MC_HD void mc_lodi_inflow(const AT &A, int i, int j, int k, int l_if, double &rho_in, double *rhoa_in,
                          double vel_in[3], double &T_in, double &p_in) {
    const gas::Tables &t = *A.tab;
    const long n = mc_idx(A, i, j, k);
    const McFields c0 = mc_fields(A, n);
    double y[NS];
    mc_Y_of<NS>(A, n, y);
    const McDP st = mc_state_dp<NS>(t, A.U, c0.rho, c0.p, y);
    const double c = st.c;
    const int cxl = cx(l_if), cyl = cy(l_if), czl = cz(l_if);
    const int d = cxl != 0 ? 0 : (cyl != 0 ? 1 : 2);
    const int cd = d == 0 ? cxl : (d == 1 ? cyl : czl);
    const long m1 = mc_idx(A, i + cxl, j + cyl, k + czl);
    const long mb = mc_idx(A, i - cxl, j - cyl, k - czl);
    const McFields c1 = mc_fields(A, m1), cb = mc_fields(A, mb);
    const double dun = mc_fd_uw(c0.u[d], c1.u[d], cd);
    const double dp = mc_fd_uw(c0.p, c1.p, cd);
    double dY[NS];
    for (int a = 0; a < NS; ++a)
        dY[a] = mc_fd_uw(rec(A, A.rec_cur, rs(a, RS_RHO), n) / c0.rho, rec(A, A.rec_cur, rs(a, RS_RHO), m1) / c1.rho,
                         cd);
    const int Nd = d == 0 ? A.Nx_glob : (d == 1 ? A.Ny : A.Nz);
    const double rho = c0.rho, un = c0.u[d];
    // the two tangential axes in the reference's order per branch: x -> (y, z), y -> (z, x),
    // z -> (x, y)
    const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
    const double L1a = (un - c) * (dp - rho * c * dun);
    const double L2 = kLodiSigmaIn * c / Nd * rho * st.Rmix * (c0.T - cb.T);
    const double L3 = kLodiSigmaIn * c / Nd * (c0.u[t1] - cb.u[t1]);
    const double L4 = kLodiSigmaIn * c / Nd * (c0.u[t2] - cb.u[t2]);
    const double L5a = (un + c) * (dp + rho * c * dun);
    const double relax_K = kLodiSigmaIn * c * c / Nd * rho * (1.0 - (un / c) * (un / c));
    double L1 = L1a, L5 = L5a;
    // left boundary: the z branch of the reference tests cy here (so a z face always
    // takes the right-boundary form)
    const bool left = (d == 2 ? cyl : cd) > 0;
    if (left)
        L5 = relax_K * (un - cb.u[d]);
    else
        L1 = relax_K * (un - cb.u[d]);
    const double d1 = 1.0 / (c * c) * (L2 + 0.5 * (L5 + L1));
    const double d2 = 1.0 / (2.0 * rho * c) * (L5 - L1);
    const double d5 = 0.5 * (L5 + L1);
    const double dt = A.dt;
    rho_in = rho - dt * d1;
    vel_in[d] = un - dt * d2;
    vel_in[t1] = c0.u[t1] - dt * L3;
    vel_in[t2] = c0.u[t2] - dt * L4;
    p_in = c0.p - dt * d5;
    for (int a = 0; a < NS; ++a)
        rhoa_in[a] = (rec(A, A.rec_cur, rs(a, RS_RHO), n) / c0.rho - dt * un * dY[a]) * rho_in;
    double y2[NS], Y2[NS], X2[NS];
    for (int a = 0; a < NS; ++a) y2[a] = rhoa_in[a] / rho_in;
    double W2 = set_mass_fractions<NS>(t, y2, Y2, X2);
    const double T = (double)si_p(A.U, (float)p_in) * W2 / ((double)si_rho(A.U, (float)rho_in) * gas::kR);
    T_in = u_temp(A.U, (float)T);
    // setState_TP(T_in, p_in): density of the state, species in the un-normalised ratios
    for (int a = 0; a < NS; ++a) y2[a] = rhoa_in[a] / rho_in;
    W2 = set_mass_fractions<NS>(t, y2, Y2, X2);
    const double dens = (double)si_p(A.U, (float)p_in) * W2 / (gas::kR * (double)si_temp(A.U, (float)T_in));
    rho_in = u_rho(A.U, (float)dens);
    for (int a = 0; a < NS; ++a) rhoa_in[a] = y2[a] * rho_in;
}

// Local state of the cell with the boundary directions (upstream type accepted by
// `isb`) taken from the target set (Fa, G at rho_t, rhoa_t), the others from f
// (src/lbm-bc.cpp:233-306 and the matching blocks of the other passes).
template <int NS, class AT, class IsB>
MC_HD void mc_local_state(const AT &A, int i, int j, int k, const IsB &isb, const double (*f)[27],
                          const AxisF<double> *Fa, const AxisG<double> &G, double rho_t, const double *rhoa_t,
                          double &rho_loc, double *rhoa_loc, double vel_loc[3], double (*vela_loc)[3],
                          double &Uint) {
    double rhoe_loc = 0.0;
    for (int a = 0; a < NS; ++a) {
        rhoa_loc[a] = 0.0;
        vela_loc[a][0] = vela_loc[a][1] = vela_loc[a][2] = 0.0;
    }
    for (int l = 0; l < 27; ++l) {
        const bool b = isb(mc_type_at(A, i - cx(l), j - cy(l), k - cz(l)));
        for (int a = 0; a < NS; ++a) {
            const double fv = b ? feq_l(l, rhoa_t[a], Fa[a]) : f[a][l];
            rhoa_loc[a] += fv;
            vela_loc[a][0] += fv * cx(l);
            vela_loc[a][1] += fv * cy(l);
            vela_loc[a][2] += fv * cz(l);
        }
        rhoe_loc += b ? geq_l(l, rho_t, G) : f[NS][l];
    }
    rho_loc = 0.0;
    vel_loc[0] = vel_loc[1] = vel_loc[2] = 0.0;
    for (int a = 0; a < NS; ++a) {
        rho_loc += rhoa_loc[a];
        for (int d = 0; d < 3; ++d) vel_loc[d] += vela_loc[a][d];
        for (int d = 0; d < 3; ++d) vela_loc[a][d] = rhoa_loc[a] > 0.0 ? vela_loc[a][d] / rhoa_loc[a] : 0.0;
    }
    for (int d = 0; d < 3; ++d) vel_loc[d] = rho_loc > 0 ? vel_loc[d] / rho_loc : 0.0;
    Uint = rhoe_loc / rho_loc;
    for (int a = 0; a < NS; ++a)
        Uint = Uint - 0.5 * rhoa_loc[a] / rho_loc *
                          (vela_loc[a][0] * vela_loc[a][0] + vela_loc[a][1] * vela_loc[a][1] +
                           vela_loc[a][2] * vela_loc[a][2]);
}

MC_HD bool mc_face_dir(int l) { return csq(l) == 1; }

// Streaming, boundary treatment and moments of one special cell b (cell n).
template <int NS, class AT>
MC_HDN void mc_special_cell(const AT &A, long n, long b) {
    const gas::Tables &t = *A.tab;
    int i, j, k;
    cell_ijk(n, A.si, A.sj, i, j, k);
    double f[NS + 1][27];
    // ---- streaming (src/lbm-streaming.cpp:15-107)
    for (int l = 0; l < 27; ++l) {
        int in = i - cx(l), jn = j - cy(l), kn = k - cz(l);
        const int tn = mc_type_at(A, in, jn, kn);
        if (tn == T_S || tn == T_A) {  // bounce-back; g only off adiabatic cells
            for (int a = 0; a < NS; ++a) f[a][l] = ldpop(A, A.pop_src, 27 * a + opp(l), n);
            f[NS][l] = tn == T_A ? ldpop(A, A.pop_src, 27 * NS + opp(l), n)
                                 : ldpop_b(A, A.bst_cur, 27 * NS + l, b);
        } else if (tn == T_FS) {  // specular reflection (dirSlip, src/lbm-bc.cpp:1352-1399)
            int cxp = cx(l), cyp = cy(l), czp = cz(l), ip = in, jp = jn, kp = kn;
            if (mc_type_at(A, in, j, k) == T_FS) {
                cxp = -cxp;
                ip = i;
            } else if (mc_type_at(A, i, jn, k) == T_FS) {
                cyp = -cyp;
                jp = j;
            } else if (mc_type_at(A, i, j, kn) == T_FS) {
                czp = -czp;
                kp = k;
            }
            if (!((ip == 0 && A.halo_lo) || (ip == A.Nx - 1 && A.halo_hi))) ip = ((ip - 1 + (A.Nx - 2)) % (A.Nx - 2)) + 1;
            jp = ((jp - 1 + (A.Ny - 2)) % (A.Ny - 2)) + 1;
            kp = ((kp - 1 + (A.Nz - 2)) % (A.Nz - 2)) + 1;
            int lp = l;
            for (int q = 0; q < 27; ++q)
                if (cx(q) == cxp && cy(q) == cyp && cz(q) == czp) lp = q;
            const long src = mc_idx(A, ip, jp, kp);
            for (int a = 0; a <= NS; ++a) f[a][l] = ldpop(A, A.pop_src, 27 * a + lp, src);
        } else if (tn == T_O || tn == T_O_C || tn == T_I || tn == T_I_C) {  // kept
            for (int a = 0; a <= NS; ++a) f[a][l] = ldpop_b(A, A.bst_cur, 27 * a + l, b);
        } else {  // periodic wrap through the ghost layer
            if (in == 0 && !A.halo_lo) in = A.Nx - 2; else if (in == A.Nx - 1 && !A.halo_hi) in = 1;
            if (jn == 0) jn = A.Ny - 2; else if (jn == A.Ny - 1) jn = 1;
            if (kn == 0) kn = A.Nz - 2; else if (kn == A.Nz - 1) kn = 1;
            const long src = mc_idx(A, in, jn, kn);
            for (int a = 0; a <= NS; ++a) f[a][l] = ldpop(A, A.pop_src, 27 * a + l, src);
        }
    }

    AxisF<double> Fo[NS], Fl[NS];
    AxisG<double> Go, Gl;
    double rho_loc, rhoa_loc[NS], vel_loc[3], vela_loc[NS][3], Uint;
    // ---- outflow pass: the first direction with an outflow ghost upstream and fluid
    // downstream, acted on only when it is a face direction
    {
        int li = -1;
        for (int l = 0; l < 27 && li < 0; ++l) {
            const int tu = mc_type_at(A, i - cx(l), j - cy(l), k - cz(l));
            if ((tu == T_O || tu == T_O_C) && mc_type_at(A, i + cx(l), j + cy(l), k + cz(l)) == T_F) li = l;
        }
        if (li >= 0 && mc_face_dir(li)) {
            const int d = cx(li) != 0 ? 0 : (cy(li) != 0 ? 1 : 2);
            const int sg = d == 0 ? cx(li) : (d == 1 ? cy(li) : cz(li));
            double rho_o, rhoa_o[NS], vel_o[3], T_o;
            mc_nscbc_outflow<NS>(A, i, j, k, d, sg, rho_o, rhoa_o, vel_o, T_o);
            const double Tsi = mc_target_axes<NS>(t, A.U, rho_o, rhoa_o, vel_o, nullptr, T_o, Fo, Go);
            auto isb = [](int ty) { return ty == T_O || ty == T_O_C; };
            mc_local_state<NS>(A, i, j, k, isb, f, Fo, Go, rho_o, rhoa_o, rho_loc, rhoa_loc, vel_loc, vela_loc, Uint);
            const double Tl = mc_calc_temp<NS>(A, Uint, rho_loc, rhoa_loc, Tsi);
            mc_target_axes<NS>(t, A.U, rho_loc, rhoa_loc, vel_loc, vela_loc, Tl, Fl, Gl);
            for (int l = 0; l < 27; ++l) {
                const bool bd = isb(mc_type_at(A, i - cx(l), j - cy(l), k - cz(l)));
                for (int a = 0; a < NS; ++a) {
                    const double fo = feq_l(l, rhoa_o[a], Fo[a]), fl = feq_l(l, rhoa_loc[a], Fl[a]);
                    f[a][l] = bd ? 2 * fo - fl : fo + f[a][l] - fl;
                }
                const double go = geq_l(l, rho_o, Go), gl = geq_l(l, rho_loc, Gl);
                f[NS][l] = bd ? 2 * go - gl : go + f[NS][l] - gl;
            }
        }
    }
    // ---- inflow pass
    {
        int li = -1;
        for (int l = 0; l < 27 && li < 0; ++l) {
            const int tu = mc_type_at(A, i - cx(l), j - cy(l), k - cz(l));
            if ((tu == T_I || tu == T_I_C) && mc_type_at(A, i + cx(l), j + cy(l), k + cz(l)) == T_F) li = l;
        }
        if (li >= 0 && mc_face_dir(li)) {
            double rho_i, rhoa_i[NS], vel_i[3], T_i, p_i;
            mc_lodi_inflow<NS>(A, i, j, k, li, rho_i, rhoa_i, vel_i, T_i, p_i);
            const double Tsi = mc_target_axes<NS>(t, A.U, rho_i, rhoa_i, vel_i, nullptr, T_i, Fo, Go);
            auto isb = [](int ty) { return ty == T_I || ty == T_I_C; };
            mc_local_state<NS>(A, i, j, k, isb, f, Fo, Go, rho_i, rhoa_i, rho_loc, rhoa_loc, vel_loc, vela_loc, Uint);
            const double Tl = mc_calc_temp<NS>(A, Uint, rho_loc, rhoa_loc, Tsi);
            mc_target_axes<NS>(t, A.U, rho_loc, rhoa_loc, vel_loc, vela_loc, Tl, Fl, Gl);
            AxisF<double> Ft[NS];
            AxisG<double> Gt;
            mc_target_axes<NS>(t, A.U, rho_loc, rhoa_loc, vel_i, nullptr, T_i, Ft, Gt);
            for (int l = 0; l < 27; ++l) {
                const bool bd = isb(mc_type_at(A, i - cx(l), j - cy(l), k - cz(l)));
                for (int a = 0; a < NS; ++a) {
                    const double fi = feq_l(l, rhoa_i[a], Fo[a]), fl = feq_l(l, rhoa_loc[a], Fl[a]),
                                 ft = feq_l(l, rhoa_loc[a], Ft[a]);
                    f[a][l] = bd ? ft + fi - fl : ft + f[a][l] - fl;
                }
                const double gi = geq_l(l, rho_i, Go), gl = geq_l(l, rho_loc, Gl), gt = geq_l(l, rho_loc, Gt);
                f[NS][l] = bd ? gt + gi - gl : gt + f[NS][l] - gl;
            }
        }
    }
    // ---- solid pass: half-way interpolated target, q = 0.5
    {
        int nd = 0;
        double vt[3] = {0, 0, 0}, Tt = 0, vat[NS][3];
        for (int a = 0; a < NS; ++a) vat[a][0] = vat[a][1] = vat[a][2] = 0.0;
        const double q = 0.5;
        for (int l = 0; l < 27; ++l) {
            if (mc_type_at(A, i - cx(l), j - cy(l), k - cz(l)) != T_S ||
                mc_type_at(A, i + cx(l), j + cy(l), k + cz(l)) != T_F)
                continue;
            ++nd;
            const long hi = mc_idx(A, i + cx(l), j + cy(l), k + cz(l));
            const long lo = mc_idx(A, i - cx(l), j - cy(l), k - cz(l));
            const McFields h = mc_fields(A, hi), o = mc_fields(A, lo);
            for (int d = 0; d < 3; ++d) vt[d] += (q * h.u[d] + o.u[d]) / (1.0 + q);
            Tt += (q * h.T + o.T) / (1.0 + q);
            // the species target mixes the fluid side's species velocity with the solid
            // cell's mixture velocity, as the reference does (src/lbm-bc.cpp:998-1000)
            for (int a = 0; a < NS; ++a)
                for (int d = 0; d < 3; ++d)
                    vat[a][d] += (q * rec(A, A.rec_cur, rs(a, RS_UX + d), hi) + o.u[d]) / (1.0 + q);
        }
        if (nd > 0) {
            double rho_bb = 0.0, rhoa_bb[NS];
            for (int a = 0; a < NS; ++a) {
                rhoa_bb[a] = 0.0;
                for (int l = 0; l < 27; ++l) rhoa_bb[a] += f[a][l];
                rho_bb += rhoa_bb[a];
            }
            for (int d = 0; d < 3; ++d) vt[d] = 1.0 / nd * vt[d];
            Tt = 1.0 / nd * Tt;
            for (int a = 0; a < NS; ++a)
                for (int d = 0; d < 3; ++d) vat[a][d] = 1.0 / nd * vat[a][d];
            const double Tsi = mc_target_axes<NS>(t, A.U, rho_bb, rhoa_bb, vt, vat, Tt, Fo, Go);
            auto isb = [](int ty) { return ty == T_S; };
            mc_local_state<NS>(A, i, j, k, isb, f, Fo, Go, rho_bb, rhoa_bb, rho_loc, rhoa_loc, vel_loc, vela_loc, Uint);
            const double Tl = mc_calc_temp<NS>(A, Uint, rho_loc, rhoa_loc, Tsi);
            mc_target_axes<NS>(t, A.U, rho_loc, rhoa_loc, vel_loc, vela_loc, Tl, Fl, Gl);
            for (int l = 0; l < 27; ++l) {
                const bool bd = isb(mc_type_at(A, i - cx(l), j - cy(l), k - cz(l)));
                for (int a = 0; a < NS; ++a) {
                    const double fo = feq_l(l, rhoa_bb[a], Fo[a]), fl = feq_l(l, rhoa_loc[a], Fl[a]);
                    f[a][l] = bd ? 2 * fo - fl : fo + f[a][l] - fl;
                }
                const double go = geq_l(l, rho_bb, Go), gl = geq_l(l, rho_loc, Gl);
                f[NS][l] = bd ? 2 * go - gl : go + f[NS][l] - gl;
            }
        }
    }
    // ---- moments, and the populations kept for the collision and the next streaming
    mc_moments_cell<NS>(A, n, [&](int a, int l) { return f[a][l]; });
    for (int a = 0; a <= NS; ++a)
        for (int l = 0; l < 27; ++l) stpop_b(A, A.bst_nxt, 27 * a + l, b, f[a][l]);
}

}  // namespace lbm
