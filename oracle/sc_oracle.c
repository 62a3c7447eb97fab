/* Plain-C oracle, single-component thermal D3Q27 path.  TEST INFRASTRUCTURE ONLY
 * (see lbm_oracle.h).  Every routine restates the reference routine named beside it,
 * operating on the reference's own AoS cell layout. */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* D3Q27 velocity set in the reference's direction order (src/headers/lbm.hpp:49-53). */
static const int CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
static const int CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};

static int opp_dir(int l) {
    for (int m = 0; m < 27; ++m)
        if (CX[m] == -CX[l] && CY[m] == -CY[l] && CZ[m] == -CZ[l]) return m;
    return -1;
}

size_t orc_sc_sizeof(void) { return sizeof(orc_mix_sc); }

void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ---------------------------------------------------------------------------------
 * Equilibria
 * ------------------------------------------------------------------------------- */

/* One-axis factor of the product-form equilibrium: c = 0 -> 1 - zeta,
 * c = +-1 -> (+-xi + zeta)/2.  Reference: calculate_feq, lbm.hpp:276-305. */
static double axis_psi(int c, double xi, double zeta) {
    if (c == 0) return 1.0 - zeta;
    return (c * xi + zeta) * 0.5;
}

double orc_feq(int l, double rho, const double u[3], double theta, const double corr[3]) {
    const int c[3] = {CX[l], CY[l], CZ[l]};
    double r = rho;
    for (int a = 0; a < 3; ++a) r *= axis_psi(c[a], u[a], theta + u[a] * u[a] + corr[a]);
    return r;
}

/* Energy equilibrium of the reference's expanded polynomial (lbm-edf.cpp:38-98).
 * The polynomial equals, for every direction,
 *   rho * [ E*Psi + theta * sum_a u_a dPsi/dxi_a + sum_a (theta^2 + 2 theta u_a^2) dPsi/dzeta_a ]
 * with E = U + |u|^2/2 and Psi the product-form factor at xi = u, zeta_a = theta + u_a^2:
 * the unique first-order correction of E*Psi that reproduces the moments
 * rho*E, rho*H*u and rho*(H*P/rho + theta*u u) with H = E + theta.  (Checked symbolically
 * against all 27 reference polynomials.) */
double orc_geq(int l, double rho, double U, double theta, const double u[3]) {
    const int c[3] = {CX[l], CY[l], CZ[l]};
    double ps[3], dxi[3], dze[3];
    for (int a = 0; a < 3; ++a) {
        ps[a] = axis_psi(c[a], u[a], theta + u[a] * u[a]);
        dxi[a] = 0.5 * c[a];
        dze[a] = (c[a] == 0) ? -1.0 : 0.5;
    }
    const double E = U + 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    double r = E * ps[0] * ps[1] * ps[2];
    r += theta * (u[0] * dxi[0] * ps[1] * ps[2] + u[1] * ps[0] * dxi[1] * ps[2] + u[2] * ps[0] * ps[1] * dxi[2]);
    r += (theta * theta + 2.0 * theta * u[0] * u[0]) * dze[0] * ps[1] * ps[2];
    r += (theta * theta + 2.0 * theta * u[1] * u[1]) * ps[0] * dze[1] * ps[2];
    r += (theta * theta + 2.0 * theta * u[2] * u[2]) * ps[0] * ps[1] * dze[2];
    return rho * r;
}

/* Moment-form energy equilibrium used by the single-component Init
 * (lbm-edf.cpp:100-138): Hermite-like expansion in (rhoe, q, R) weighted by the
 * rest-frame product weights, plus a diagonal correction on the rest and unit-speed
 * directions. */
double orc_geq_moment(int l, double rhoe, const double q[3], const double R[9], double theta) {
    const double c[3] = {(double)CX[l], (double)CY[l], (double)CZ[l]};
    double val = rhoe + (q[0] * c[0] + q[1] * c[1] + q[2] * c[2]) / theta;
    double contr = 0.0;
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
            double A = R[3 * a + b] - (a == b ? rhoe * theta : 0.0);
            double B = c[a] * c[b] - (a == b ? theta : 0.0);
            contr += A * B;
        }
    val += contr / (2.0 * theta * theta);
    double wgt = 1.0;
    for (int m = 0; m < 3; ++m) wgt *= (c[m] == 0.0) ? (1.0 - theta) : theta / 2.0;
    val *= wgt;
    const double c2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    for (int m = 0; m < 3; ++m) {
        double Bm = (c2 == 0.0) ? 1.0 : (c2 == 1.0 ? -0.5 * fabs(c[m]) : 0.0);
        double Zm = (1.0 - 3.0 * theta) / (2.0 * theta) * (R[4 * m] - theta * rhoe);
        val += Bm * Zm;
    }
    return val;
}

/* Quasi-equilibrium shift on the six unit-speed directions (lbm-edf.cpp:140-150). */
double orc_gstr(int l, double geq, const double dq[3]) {
    const int c2 = CX[l] * CX[l] + CY[l] * CY[l] + CZ[l] * CZ[l];
    if (c2 != 1) return geq;
    return geq + 0.5 * (CX[l] * dq[0] + CY[l] * dq[1] + CZ[l] * dq[2]);
}

/* ---------------------------------------------------------------------------------
 * Finite differences (FD.hpp:108-127, FD.cpp:5-23, 64-74)
 * ------------------------------------------------------------------------------- */
static int wall_like(int t) {
    return t == ORC_S || t == ORC_A || t == ORC_FS || t == ORC_P || t == ORC_O || t == ORC_O_C;
}

double orc_fd_central(double sl, double sc, double sr, double dx, double vel, int tl, int tr) {
    (void)vel;
    if (wall_like(tl)) return (tr == ORC_P) ? 0.0 : (sr - sc) / dx;
    if (wall_like(tr)) return (tl == ORC_P) ? 0.0 : (sc - sl) / dx;
    return (sr - sl) / (2 * dx);
}

static int upwind_blocked(int t) { return wall_like(t) || t == ORC_I || t == ORC_I_C; }

double orc_fd_fuw(double sl, double sc, double sr, double dx, double vel, int tl, int tr) {
    if (vel > 0) return upwind_blocked(tl) ? 0.0 : (sc - sl) / dx;
    return upwind_blocked(tr) ? 0.0 : (sr - sc) / dx;
}

double orc_fd_uw(double s0, double s1, double s2, double dx, double vel) {
    (void)s2;
    return (vel < 0) ? (s0 - s1) / dx : (s1 - s0) / dx;
}

/* ---------------------------------------------------------------------------------
 * Per-step phases
 * ------------------------------------------------------------------------------- */
#define IDX(g, i, j, k) (((size_t)(i) * (size_t)(g)->Ny + (size_t)(j)) * (size_t)(g)->Nz + (size_t)(k))

/* BC target populations from (rho, u, T) (lbm-edf.cpp:153-164). */
static void feq_geq_sc(const orc_sc_grid *g, double *f, double *ge, double rho, const double vel[3], double T) {
    const double theta = g->R * T;
    const double cv = g->R / (g->gamma - 1.0);
    const double U = cv * T;
    const double zero[3] = {0, 0, 0};
    for (int l = 0; l < 27; ++l) {
        f[l] = orc_feq(l, rho, vel, theta, zero);
        ge[l] = orc_geq(l, rho, U, theta, vel);
    }
}

/* LBM::Init, single component (lbm-init.cpp:8-82).  f starts at rest (zero velocity)
 * while the g heat flux carries the setup velocity; the moments are left for the first
 * Collide to use as they stand. */
void orc_sc_init(orc_mix_sc *cells, const orc_sc_grid *g) {
    const long ncell = (long)g->Nx * g->Ny * g->Nz;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < ncell; ++n) {
        orc_mix_sc *m = &cells[n];
        if (!(m->type == ORC_F || m->type == ORC_S || m->type == ORC_I || m->type == ORC_O || m->type == ORC_Q))
            continue;
        const double vel0[3] = {0.0, 0.0, 0.0};
        m->rho = m->p / (g->R * m->temp);
        const double theta = g->R * m->temp;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) m->p_tensor[a][b] = (a == b) ? m->p : 0.0;
        const double cv = g->R / (g->gamma - 1.0);
        const double cp = cv + g->R;
        m->rhoe = m->rho * (cv * m->temp);
        const double H = cp * m->temp;
        double Rt[9];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Rt[3 * a + b] = H * m->p_tensor[a][b];
        const double q[3] = {H * m->rho * m->u, H * m->rho * m->v, H * m->rho * m->w};
        const double zero[3] = {0, 0, 0};
        for (int l = 0; l < 27; ++l) {
            m->f[l] = orc_feq(l, m->rho, vel0, theta, zero);
            m->g[l] = orc_geq_moment(l, m->rhoe, q, Rt, theta);
        }
    }
}

/* Momentum-flux deviation term rho*u_a*(1 - 3 R T) - rho*u_a^3 whose face-centred
 * difference corrects the equilibria (lbm-collision.cpp:65-67). */
static double qdev(const orc_mix_sc *m, int a, double R) {
    const double ua = (a == 0) ? m->u : (a == 1 ? m->v : m->w);
    return m->rho * ua * (1.0 - 3.0 * R * m->temp) - m->rho * ua * ua * ua;
}

/* LBM::Collide, single component (lbm-collision.cpp:9-99). */
void orc_sc_collide(orc_mix_sc *cells, const orc_sc_grid *g) {
    const double dt = g->dt;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->Nx; ++i)
        for (int j = 0; j < g->Ny; ++j)
            for (int k = 0; k < g->Nz; ++k) {
                orc_mix_sc *m = &cells[IDX(g, i, j, k)];
                if (m->type != ORC_F) continue;
                const double cv = g->R / (g->gamma - 1.0);
                const double cp = cv + g->R;
                const double theta = g->R * m->temp;
                const double mu = g->nu * m->rho;
                const double kappa = mu * cp / g->prtl;
                const double om1 = 2 * m->p * cp * dt / (m->p * cp * dt + 2 * kappa);
                const double om = 2 * m->p * dt / (m->p * dt + 2 * mu);
                const double vel[3] = {m->u, m->v, m->w};
                const double Uint = m->rhoe / m->rho - 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
                double eqP[3][3];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) eqP[a][b] = (a == b ? m->p : 0.0) + m->rho * vel[a] * vel[b];
                const orc_mix_sc *nb_lo[3] = {&cells[IDX(g, i - 1, j, k)], &cells[IDX(g, i, j - 1, k)], &cells[IDX(g, i, j, k - 1)]};
                const orc_mix_sc *nb_hi[3] = {&cells[IDX(g, i + 1, j, k)], &cells[IDX(g, i, j + 1, k)], &cells[IDX(g, i, j, k + 1)]};
                double dQ[3];
                for (int a = 0; a < 3; ++a)
                    dQ[a] = orc_fd_central(qdev(nb_lo[a], a, g->R), qdev(m, a, g->R), qdev(nb_hi[a], a, g->R), 1.0, vel[a],
                                           nb_lo[a]->type, nb_hi[a]->type);
                double dq[3], corr[3];
                for (int b = 0; b < 3; ++b) {
                    double s = 0.0;
                    for (int a = 0; a < 3; ++a) s += vel[a] * (m->p_tensor[a][b] - eqP[a][b]);
                    dq[b] = s + 0.5 * dt * vel[b] * dQ[b];
                    corr[b] = dt * (2 - om) / (2 * m->rho * om) * dQ[b];
                }
                for (int l = 0; l < 27; ++l) {
                    const double fe = orc_feq(l, m->rho, vel, theta, corr);
                    m->fpc[l] = (1.0 - om) * m->f[l] + om * fe;
                    const double ge = orc_geq(l, m->rho, Uint, theta, vel);
                    const double gs = orc_gstr(l, ge, dq);
                    m->gpc[l] = m->g[l] + om1 * (ge - m->g[l]) + (om - om1) * (ge - gs);
                }
            }
}

/* Specular partner of direction l for a free-slip neighbour (LBM::dirSlip,
 * lbm-bc.cpp:1352-1399): flips the first axis (x, then y, then z) along which the
 * axis neighbour is a free-slip cell, and wraps the source cell periodically. */
static void dir_slip(const orc_mix_sc *cells, const orc_sc_grid *g, int l, int i, int j, int k, int *lp, int *ip, int *jp, int *kp) {
    const int inb = i - CX[l], jnb = j - CY[l], knb = k - CZ[l];
    int cxp = CX[l], cyp = CY[l], czp = CZ[l];
    *ip = inb;
    *jp = jnb;
    *kp = knb;
    if (cells[IDX(g, inb, j, k)].type == ORC_FS) {
        cxp = -CX[l];
        *ip = i;
    } else if (cells[IDX(g, i, jnb, k)].type == ORC_FS) {
        cyp = -CY[l];
        *jp = j;
    } else if (cells[IDX(g, i, j, knb)].type == ORC_FS) {
        czp = -CZ[l];
        *kp = k;
    }
    *ip = ((*ip - 1 + (g->Nx - 2)) % (g->Nx - 2)) + 1;
    *jp = ((*jp - 1 + (g->Ny - 2)) % (g->Ny - 2)) + 1;
    *kp = ((*kp - 1 + (g->Nz - 2)) % (g->Nz - 2)) + 1;
    *lp = l;
    for (int a = 0; a < 27; ++a)
        if (CX[a] == cxp && CY[a] == cyp && CZ[a] == czp) {
            *lp = a;
            break;
        }
}

/* LBM::Streaming (lbm-streaming.cpp:3-119): pull from the upstream neighbour with
 * bounce-back off solid (f only) and adiabatic (f and g) cells, specular reflection off
 * free-slip cells, no change next to inflow/outflow cells, periodic wrap at ghosts. */
void orc_sc_streaming(orc_mix_sc *cells, const orc_sc_grid *g) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->Nx; ++i)
        for (int j = 0; j < g->Ny; ++j)
            for (int k = 0; k < g->Nz; ++k) {
                orc_mix_sc *m = &cells[IDX(g, i, j, k)];
                if (m->type != ORC_F) continue;
                for (int l = 0; l < 27; ++l) {
                    int in = i - CX[l], jn = j - CY[l], kn = k - CZ[l];
                    const int tn = cells[IDX(g, in, jn, kn)].type;
                    if (tn == ORC_S) {
                        m->f[l] = m->fpc[opp_dir(l)];
                    } else if (tn == ORC_FS) {
                        int lp, ip, jp, kp;
                        dir_slip(cells, g, l, i, j, k, &lp, &ip, &jp, &kp);
                        m->f[l] = cells[IDX(g, ip, jp, kp)].fpc[lp];
                        m->g[l] = cells[IDX(g, ip, jp, kp)].gpc[lp];
                    } else if (tn == ORC_A) {
                        m->f[l] = m->fpc[opp_dir(l)];
                        m->g[l] = m->gpc[opp_dir(l)];
                    } else if (tn == ORC_O || tn == ORC_O_C || tn == ORC_I || tn == ORC_I_C) {
                        /* populations keep their previous values; TMS_BC rebuilds them */
                    } else {
                        if (in == 0) in = g->Nx - 2; else if (in == g->Nx - 1) in = 1;
                        if (jn == 0) jn = g->Ny - 2; else if (jn == g->Ny - 1) jn = 1;
                        if (kn == 0) kn = g->Nz - 2; else if (kn == g->Nz - 1) kn = 1;
                        m->f[l] = cells[IDX(g, in, jn, kn)].fpc[l];
                        m->g[l] = cells[IDX(g, in, jn, kn)].gpc[l];
                    }
                }
            }
}

/* Local moments of a cell whose populations along boundary directions (upstream
 * neighbour of type btype) are replaced by the target set ft/gt, and the temperature
 * they imply (lbm-bc.cpp:381-410 and the matching inflow/solid blocks). */
static void local_state(const orc_mix_sc *cells, const orc_sc_grid *g, int i, int j, int k, int btype,
                        const double *ft, const double *gt, double *rho_o, double vel_o[3], double *T_o) {
    const orc_mix_sc *m = &cells[IDX(g, i, j, k)];
    double rho = 0, ru = 0, rv = 0, rw = 0, re = 0;
    for (int l = 0; l < 27; ++l) {
        const int tn = cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type;
        const double fv = (tn == btype) ? ft[l] : m->f[l];
        const double gv = (tn == btype) ? gt[l] : m->g[l];
        rho += fv;
        ru += fv * CX[l];
        rv += fv * CY[l];
        rw += fv * CZ[l];
        re += gv;
    }
    vel_o[0] = ru / rho;
    vel_o[1] = rv / rho;
    vel_o[2] = rw / rho;
    const double Uint = re / rho - 0.5 * (vel_o[0] * vel_o[0] + vel_o[1] * vel_o[1] + vel_o[2] * vel_o[2]);
    *T_o = Uint / (g->R / (g->gamma - 1.0));
    *rho_o = rho;
}

/* LBM::TMS_BC, single component (lbm-bc.cpp:341-460 outflow, 809-938 inflow,
 * 1111-1229 solid): Tamm-Mott-Smith replacement f <- f_tgt + f - f_loc, with the
 * boundary directions rebuilt from the target state. */
void orc_sc_tms_bc(orc_mix_sc *cells, const orc_sc_grid *g) {
    /* outflow */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->Nx; ++i)
        for (int j = 0; j < g->Ny; ++j)
            for (int k = 0; k < g->Nz; ++k) {
                orc_mix_sc *m = &cells[IDX(g, i, j, k)];
                if (m->type != ORC_F) continue;
                int li = -1;
                for (int l = 0; l < 27; ++l)
                    if (cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type == ORC_O &&
                        cells[IDX(g, i + CX[l], j + CY[l], k + CZ[l])].type == ORC_F) {
                        li = l;
                        break;
                    }
                if (li < 0) continue;
                const orc_mix_sc *in_nb = &cells[IDX(g, i + CX[li], j + CY[li], k + CZ[li])];
                const orc_mix_sc *gh = &cells[IDX(g, i - CX[li], j - CY[li], k - CZ[li])];
                const double vel_out[3] = {in_nb->u, in_nb->v, in_nb->w};
                const double T_out = in_nb->temp;
                const double rho_out = gh->p / (g->R * T_out);
                double fo[27], go[27], fl[27], gl[27], rl, vl[3], Tl;
                feq_geq_sc(g, fo, go, rho_out, vel_out, T_out);
                local_state(cells, g, i, j, k, ORC_O, fo, go, &rl, vl, &Tl);
                feq_geq_sc(g, fl, gl, rl, vl, Tl);
                for (int l = 0; l < 27; ++l) {
                    if (cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type == ORC_O) {
                        m->f[l] = 2 * fo[l] - fl[l];
                        m->g[l] = 2 * go[l] - gl[l];
                    } else {
                        m->f[l] = fo[l] + m->f[l] - fl[l];
                        m->g[l] = go[l] + m->g[l] - gl[l];
                    }
                }
            }
    /* inflow */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->Nx; ++i)
        for (int j = 0; j < g->Ny; ++j)
            for (int k = 0; k < g->Nz; ++k) {
                orc_mix_sc *m = &cells[IDX(g, i, j, k)];
                if (m->type != ORC_F) continue;
                int li = -1;
                for (int l = 0; l < 27; ++l)
                    if (cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type == ORC_I &&
                        cells[IDX(g, i + CX[l], j + CY[l], k + CZ[l])].type == ORC_F) {
                        li = l;
                        break;
                    }
                if (li < 0) continue;
                const orc_mix_sc *gh = &cells[IDX(g, i - CX[li], j - CY[li], k - CZ[li])];
                const orc_mix_sc *in_nb = &cells[IDX(g, i + CX[li], j + CY[li], k + CZ[li])];
                const double vel_in[3] = {gh->u, gh->v, gh->w};
                const double T_in = gh->temp;
                const double rho_in = in_nb->p / (g->R * T_in);
                double fi[27], gi[27], fl[27], gl[27], ft[27], gt[27], rl, vl[3], Tl;
                feq_geq_sc(g, fi, gi, rho_in, vel_in, T_in);
                local_state(cells, g, i, j, k, ORC_I, fi, gi, &rl, vl, &Tl);
                feq_geq_sc(g, fl, gl, rl, vl, Tl);
                feq_geq_sc(g, ft, gt, rl, vel_in, T_in);
                for (int l = 0; l < 27; ++l) {
                    if (cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type == ORC_I) {
                        m->f[l] = ft[l] + fi[l] - fl[l];
                        m->g[l] = gt[l] + gi[l] - gl[l];
                    } else {
                        m->f[l] = ft[l] + m->f[l] - fl[l];
                        m->g[l] = gt[l] + m->g[l] - gl[l];
                    }
                }
            }
    /* solid walls, half-way interpolated target (q = 0.5) */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < g->Nx; ++i)
        for (int j = 0; j < g->Ny; ++j)
            for (int k = 0; k < g->Nz; ++k) {
                orc_mix_sc *m = &cells[IDX(g, i, j, k)];
                if (m->type != ORC_F) continue;
                int nd = 0;
                double vt[3] = {0, 0, 0}, Tt = 0;
                const double q = 0.5;
                for (int l = 0; l < 27; ++l) {
                    const orc_mix_sc *lo = &cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])];
                    const orc_mix_sc *hi = &cells[IDX(g, i + CX[l], j + CY[l], k + CZ[l])];
                    if (lo->type == ORC_S && hi->type == ORC_F) {
                        ++nd;
                        vt[0] += (q * hi->u + lo->u) / (1.0 + q);
                        vt[1] += (q * hi->v + lo->v) / (1.0 + q);
                        vt[2] += (q * hi->w + lo->w) / (1.0 + q);
                        Tt += (q * hi->temp + lo->temp) / (1.0 + q);
                    }
                }
                if (nd == 0) continue;
                double rho_bb = 0;
                for (int l = 0; l < 27; ++l) rho_bb += m->f[l];
                for (int a = 0; a < 3; ++a) vt[a] = 1.0 / nd * vt[a];
                Tt = 1.0 / nd * Tt;
                double ft[27], gt[27], fl[27], gl[27], rl, vl[3], Tl;
                feq_geq_sc(g, ft, gt, rho_bb, vt, Tt);
                local_state(cells, g, i, j, k, ORC_S, ft, gt, &rl, vl, &Tl);
                feq_geq_sc(g, fl, gl, rl, vl, Tl);
                for (int l = 0; l < 27; ++l) {
                    if (cells[IDX(g, i - CX[l], j - CY[l], k - CZ[l])].type == ORC_S) {
                        m->f[l] = 2 * ft[l] - fl[l];
                        m->g[l] = 2 * gt[l] - gl[l];
                    } else {
                        m->f[l] = ft[l] + m->f[l] - fl[l];
                        m->g[l] = gt[l] + m->g[l] - gl[l];
                    }
                }
            }
}

/* LBM::calculate_moment, single component (lbm-moment.cpp:11-125). */
void orc_sc_moment(orc_mix_sc *cells, const orc_sc_grid *g) {
    const long ncell = (long)g->Nx * g->Ny * g->Nz;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < ncell; ++n) {
        orc_mix_sc *m = &cells[n];
        if (m->type != ORC_F) continue;
        double rho = 0, j[3] = {0, 0, 0}, P[3][3] = {{0}}, re = 0, qf[3] = {0, 0, 0};
        for (int l = 0; l < 27; ++l) {
            const double c[3] = {(double)CX[l], (double)CY[l], (double)CZ[l]};
            const double fv = m->f[l], gv = m->g[l];
            rho += fv;
            for (int a = 0; a < 3; ++a) {
                j[a] += fv * c[a];
                qf[a] += gv * c[a];
                for (int b = a; b < 3; ++b) P[a][b] += fv * c[a] * c[b];
            }
            re += gv;
        }
        P[1][0] = P[0][1];
        P[2][0] = P[0][2];
        P[2][1] = P[1][2];
        memcpy(m->p_tensor, P, sizeof(P));
        m->rho = rho;
        m->u = j[0] / rho;
        m->v = j[1] / rho;
        m->w = j[2] / rho;
        m->rhoe = re;
        for (int a = 0; a < 3; ++a) m->energy_flux[a] = qf[a];
        const double Uint = re / rho - 0.5 * (m->u * m->u + m->v * m->v + m->w * m->w);
        m->temp = Uint / (g->R / (g->gamma - 1.0));
        m->p = m->rho * g->R * m->temp;
    }
}

void orc_sc_loop(orc_mix_sc *cells, const orc_sc_grid *g, int nsteps) {
    for (int s = 0; s < nsteps; ++s) {
        orc_sc_collide(cells, g);
        orc_sc_streaming(cells, g);
        orc_sc_tms_bc(cells, g);
        orc_sc_moment(cells, g);
    }
}
