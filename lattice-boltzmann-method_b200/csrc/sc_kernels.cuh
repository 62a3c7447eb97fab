// Single-component thermal D3Q27 step kernels (the reference with MULTICOMP off).
//
// Device state (structure of arrays; cell index n = (i*Ny + j)*Nz + k, k fastest, ghosts
// included so the neighbour arithmetic is the reference's):
//   pop[2] : 54 planes of ncell doubles -- f directions 0..26, then g directions 0..26.
//            The post-collision populations fpc/gpc of the last step, or -- right after an
//            upload or Init ("local" mode) -- the populations f/g themselves.
//   mom[2] : M_N planes -- the per-cell record the collision and the neighbours read:
//            rho, u, v, w, T, p; the face-difference term Q_a = rho u_a (1 - 3 R T) - rho u_a^3
//            for a = x, y, z (src/lbm-collision.cpp:65-67); and the two collision inputs
//            that need the full pressure tensor and rho*E:
//              S_b = sum_a u_a (P_ab - P^eq_ab)   (src/lbm-collision.cpp:72-74 without the FD part)
//              Uint = rhoE/rho - |u|^2/2         (src/lbm-collision.cpp:40)
//            Double-buffered: the boundary step of step n+1 reads step n's record while
//            the moment step writes step n+1's.
//   bst[2] : 54 values per "special" cell (a fluid cell with a solid, adiabatic, free-slip,
//            inflow or outflow neighbour upstream): its post-boundary populations f, g.
//            Populations along inflow/outflow (f and g) and solid (g) directions persist
//            from step to step in the reference (src/lbm-streaming.cpp:25-32, 63-87).
//
// One time step = k_sc_collide (pop[cur] -> pop[nxt]) + k_sc_stream_moment and
// k_sc_stream_moment_special (pull pop[nxt], boundary treatment, moments -> mom[nxt],
// bst[nxt]); then cur <-> nxt.
#pragma once
#include <cstdint>
#include "d3q27.cuh"

namespace lbm {

enum : int {
    M_RHO = 0, M_U = 1, M_V = 2, M_W = 3, M_T = 4, M_P = 5, M_QX = 6, M_QY = 7, M_QZ = 8,
    M_SX = 9, M_SY = 10, M_SZ = 11, M_UINT = 12, M_N = 13
};

struct ScGeom {
    int Nx, Ny, Nz;
    long ncell;
    long sj, si;  // strides of j and i (Nz, Ny*Nz)
};

struct ScPhys {
    double nu, R, gamma, prtl, dt, cv, cp;
};

__device__ __forceinline__ void raise_status(unsigned *flags, unsigned bits) { atomicOr(flags, bits); }

__device__ __forceinline__ long nb_index(const ScGeom &g, long n, int dx, int dy, int dz) {
    return n + dx * g.si + dy * g.sj + dz;
}

__device__ __forceinline__ int type_at(const ScGeom &g, const int8_t *__restrict__ type, int i, int j, int k) {
    return type[(long)i * g.si + (long)j * g.sj + k];
}

// Source-cell offsets of the pull for a cell none of whose upstream neighbours is a
// boundary cell: per axis, the upstream coordinate for c = 0, +1, -1 with the reference's
// periodic wrap (a neighbour index of 0 maps to N-2, N-1 maps to 1;
// src/lbm-streaming.cpp:101-105).  The 27 source cells are then sums of one entry per axis,
// with no branch and no type lookup.
struct PullSrc {
    int X[3], Y[3], Z[3];  // cell offsets (a single-component lattice has < 2^31 cells)
};

__device__ __forceinline__ void pull_src(const ScGeom &g, long n, PullSrc &s) {
    int i, j, k;
    cell_ijk(n, g.si, g.sj, i, j, k);
    const int im = (i - 1 == 0) ? g.Nx - 2 : i - 1, ip = (i + 1 == g.Nx - 1) ? 1 : i + 1;
    const int jm = (j - 1 == 0) ? g.Ny - 2 : j - 1, jp = (j + 1 == g.Ny - 1) ? 1 : j + 1;
    const int km = (k - 1 == 0) ? g.Nz - 2 : k - 1, kp = (k + 1 == g.Nz - 1) ? 1 : k + 1;
    s.X[0] = i * (int)g.si;
    s.X[1] = im * (int)g.si;
    s.X[2] = ip * (int)g.si;
    s.Y[0] = j * (int)g.sj;
    s.Y[1] = jm * (int)g.sj;
    s.Y[2] = jp * (int)g.sj;
    s.Z[0] = k;
    s.Z[1] = km;
    s.Z[2] = kp;
}

__device__ __forceinline__ int pull_at(const PullSrc &s, int l) {
    return s.X[cidx(cx(l))] + s.Y[cidx(cy(l))] + s.Z[cidx(cz(l))];
}

// Specular partner of direction l off a free-slip neighbour (reference LBM::dirSlip,
// src/lbm-bc.cpp:1352-1399).
__device__ __forceinline__ void dir_slip(const ScGeom &g, const int8_t *__restrict__ type, int l, int i, int j,
                                         int k, int &lp, long &src) {
    const int inb = i - cx(l), jnb = j - cy(l), knb = k - cz(l);
    int cxp = cx(l), cyp = cy(l), czp = cz(l);
    int ip = inb, jp = jnb, kp = knb;
    if (type_at(g, type, inb, j, k) == T_FS) {
        cxp = -cxp;
        ip = i;
    } else if (type_at(g, type, i, jnb, k) == T_FS) {
        cyp = -cyp;
        jp = j;
    } else if (type_at(g, type, i, j, knb) == T_FS) {
        czp = -czp;
        kp = k;
    }
    ip = ((ip - 1 + (g.Nx - 2)) % (g.Nx - 2)) + 1;
    jp = ((jp - 1 + (g.Ny - 2)) % (g.Ny - 2)) + 1;
    kp = ((kp - 1 + (g.Nz - 2)) % (g.Nz - 2)) + 1;
    lp = l;
#pragma unroll
    for (int a = 0; a < 27; ++a)
        if (cx(a) == cxp && cy(a) == cyp && cz(a) == czp) lp = a;
    src = (long)ip * g.si + (long)jp * g.sj + kp;
}

// Streaming of a special cell (reference LBM::Streaming, src/lbm-streaming.cpp:3-119):
// bounce-back off solid (f only) and adiabatic (f and g) cells, specular reflection off
// free-slip cells, populations kept (`stale`) along inflow/outflow directions, periodic
// wrap otherwise.
__device__ __forceinline__ void pull_special(const ScGeom &g, const int8_t *__restrict__ type, long n,
                                             const double *__restrict__ pop, const double *__restrict__ stale,
                                             long nb_stride, double f[27], double ge[27]) {
    const long nc = g.ncell;
    int i, j, k;
    cell_ijk(n, g.si, g.sj, i, j, k);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        int in = i - cx(l), jn = j - cy(l), kn = k - cz(l);
        const int tn = type_at(g, type, in, jn, kn);
        if (tn == T_S) {
            f[l] = pop[(long)opp(l) * nc + n];
            ge[l] = stale[(long)(27 + l) * nb_stride];
        } else if (tn == T_FS) {
            int lp;
            long src;
            dir_slip(g, type, l, i, j, k, lp, src);
            f[l] = pop[(long)lp * nc + src];
            ge[l] = pop[(long)(27 + lp) * nc + src];
        } else if (tn == T_A) {
            f[l] = pop[(long)opp(l) * nc + n];
            ge[l] = pop[(long)(27 + opp(l)) * nc + n];
        } else if (tn == T_O || tn == T_O_C || tn == T_I || tn == T_I_C) {
            f[l] = stale[(long)l * nb_stride];
            ge[l] = stale[(long)(27 + l) * nb_stride];
        } else {
            if (in == 0) in = g.Nx - 2; else if (in == g.Nx - 1) in = 1;
            if (jn == 0) jn = g.Ny - 2; else if (jn == g.Ny - 1) jn = 1;
            if (kn == 0) kn = g.Nz - 2; else if (kn == g.Nz - 1) kn = 1;
            const long s = (long)in * g.si + (long)jn * g.sj + kn;
            f[l] = pop[(long)l * nc + s];
            ge[l] = pop[(long)(27 + l) * nc + s];
        }
    }
}

// Target populations of a prescribed (rho, u, T) (reference calculate_feq_geq,
// src/lbm-edf.cpp:153-164).
__device__ __forceinline__ void target_sc(const ScPhys &P, double rho, const double vel[3], double T, double ft[27],
                                          double gt[27]) {
    const double theta = P.R * T;
    const double zero[3] = {0.0, 0.0, 0.0};
    AxisF<double> F;
    axis_feq(F, vel, theta, zero);
    AxisG<double> G;
    axis_geq(G, P.cv * T, theta, vel);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        ft[l] = feq_l(l, rho, F);
        gt[l] = geq_l(l, rho, G);
    }
}

// Local state of the cell with boundary directions (upstream type `bt`) replaced by the
// target set, and its temperature (src/lbm-bc.cpp:381-410, 874-903, 1167-1196).
__device__ __forceinline__ void local_state_sc(const ScGeom &g, const ScPhys &P, const int8_t *__restrict__ type, int i,
                                               int j, int k, int bt, const double f[27], const double ge[27],
                                               const double ft[27], const double gt[27], double &rho_o, double vel[3],
                                               double &T_o) {
    double rho = 0, ru = 0, rv = 0, rw = 0, re = 0;
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const bool b = type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == bt;
        const double fv = b ? ft[l] : f[l];
        const double gv = b ? gt[l] : ge[l];
        rho += fv;
        ru += fv * cx(l);
        rv += fv * cy(l);
        rw += fv * cz(l);
        re += gv;
    }
    vel[0] = ru / rho;
    vel[1] = rv / rho;
    vel[2] = rw / rho;
    const double Uint = re / rho - 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    T_o = Uint / P.cv;
    rho_o = rho;
}

// Tamm-Mott-Smith boundary treatment of one fluid cell (reference LBM::TMS_BC, single
// component: outflow src/lbm-bc.cpp:341-460, inflow :809-938, solid :1111-1229), applied
// in the reference's pass order.  `mom` holds the previous step's record.
static __device__ void tms_cell_sc(const ScGeom &g, const ScPhys &P, const int8_t *__restrict__ type,
                            const double *__restrict__ mom, long n, double f[27], double ge[27]) {
    const long nc = g.ncell;
    int i, j, k;
    cell_ijk(n, g.si, g.sj, i, j, k);
    double ft[27], gt[27], fl[27], gl[27];
    // ---- outflow: first direction with an outflow cell upstream and fluid downstream
    {
        int li = -1;
        long ni = n, ng = n;
#pragma unroll
        for (int l = 26; l >= 0; --l)
            if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_O &&
                type_at(g, type, i + cx(l), j + cy(l), k + cz(l)) == T_F) {
                li = l;
                ni = nb_index(g, n, cx(l), cy(l), cz(l));
                ng = nb_index(g, n, -cx(l), -cy(l), -cz(l));
            }
        if (li >= 0) {
            const double vel[3] = {mom[M_U * nc + ni], mom[M_V * nc + ni], mom[M_W * nc + ni]};
            const double T_out = mom[M_T * nc + ni];
            const double rho_out = mom[M_P * nc + ng] / (P.R * T_out);
            target_sc(P, rho_out, vel, T_out, ft, gt);
            double rl, vl[3], Tl;
            local_state_sc(g, P, type, i, j, k, T_O, f, ge, ft, gt, rl, vl, Tl);
            target_sc(P, rl, vl, Tl, fl, gl);
#pragma unroll
            for (int l = 0; l < 27; ++l) {
                if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_O) {
                    f[l] = 2 * ft[l] - fl[l];
                    ge[l] = 2 * gt[l] - gl[l];
                } else {
                    f[l] = ft[l] + f[l] - fl[l];
                    ge[l] = gt[l] + ge[l] - gl[l];
                }
            }
        }
    }
    // ---- inflow
    {
        int li = -1;
        long ni = n, ng = n;
#pragma unroll
        for (int l = 26; l >= 0; --l)
            if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_I &&
                type_at(g, type, i + cx(l), j + cy(l), k + cz(l)) == T_F) {
                li = l;
                ni = nb_index(g, n, cx(l), cy(l), cz(l));
                ng = nb_index(g, n, -cx(l), -cy(l), -cz(l));
            }
        if (li >= 0) {
            const double vin[3] = {mom[M_U * nc + ng], mom[M_V * nc + ng], mom[M_W * nc + ng]};
            const double T_in = mom[M_T * nc + ng];
            const double rho_in = mom[M_P * nc + ni] / (P.R * T_in);
            double fi[27], gi[27];
            target_sc(P, rho_in, vin, T_in, fi, gi);
            double rl, vl[3], Tl;
            local_state_sc(g, P, type, i, j, k, T_I, f, ge, fi, gi, rl, vl, Tl);
            target_sc(P, rl, vl, Tl, fl, gl);
            target_sc(P, rl, vin, T_in, ft, gt);
#pragma unroll
            for (int l = 0; l < 27; ++l) {
                if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_I) {
                    f[l] = ft[l] + fi[l] - fl[l];
                    ge[l] = gt[l] + gi[l] - gl[l];
                } else {
                    f[l] = ft[l] + f[l] - fl[l];
                    ge[l] = gt[l] + ge[l] - gl[l];
                }
            }
        }
    }
    // ---- solid walls, half-way interpolated target (q = 0.5)
    {
        int nd = 0;
        double vt[3] = {0, 0, 0}, Tt = 0;
        const double q = 0.5;
#pragma unroll
        for (int l = 0; l < 27; ++l) {
            if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_S &&
                type_at(g, type, i + cx(l), j + cy(l), k + cz(l)) == T_F) {
                const long hi = nb_index(g, n, cx(l), cy(l), cz(l));
                const long lo = nb_index(g, n, -cx(l), -cy(l), -cz(l));
                ++nd;
                vt[0] += (q * mom[M_U * nc + hi] + mom[M_U * nc + lo]) / (1.0 + q);
                vt[1] += (q * mom[M_V * nc + hi] + mom[M_V * nc + lo]) / (1.0 + q);
                vt[2] += (q * mom[M_W * nc + hi] + mom[M_W * nc + lo]) / (1.0 + q);
                Tt += (q * mom[M_T * nc + hi] + mom[M_T * nc + lo]) / (1.0 + q);
            }
        }
        if (nd > 0) {
            double rho_bb = 0;
#pragma unroll
            for (int l = 0; l < 27; ++l) rho_bb += f[l];
            const double inv = 1.0 / nd;
            vt[0] = inv * vt[0];
            vt[1] = inv * vt[1];
            vt[2] = inv * vt[2];
            Tt = inv * Tt;
            target_sc(P, rho_bb, vt, Tt, ft, gt);
            double rl, vl[3], Tl;
            local_state_sc(g, P, type, i, j, k, T_S, f, ge, ft, gt, rl, vl, Tl);
            target_sc(P, rl, vl, Tl, fl, gl);
#pragma unroll
            for (int l = 0; l < 27; ++l) {
                if (type_at(g, type, i - cx(l), j - cy(l), k - cz(l)) == T_S) {
                    f[l] = 2 * ft[l] - fl[l];
                    ge[l] = 2 * gt[l] - gl[l];
                } else {
                    f[l] = ft[l] + f[l] - fl[l];
                    ge[l] = gt[l] + ge[l] - gl[l];
                }
            }
        }
    }
}

// Sums of the moments of one cell: rho, j, P (upper triangle), rhoe, q.
struct ScSums {
    double rho, j[3], P[6], re, q[3];
};

__device__ __forceinline__ void sums_init(ScSums &s) {
    s.rho = 0;
    s.re = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        s.j[a] = 0;
        s.q[a] = 0;
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) s.P[a] = 0;
}

// Adds direction l's populations (in the reference's summation order, lbm-moment.cpp:35-53).
__device__ __forceinline__ void sums_add(ScSums &s, int l, double fv, double gv) {
    s.rho += fv;
    if (cx(l)) s.j[0] += cx(l) * fv;
    if (cy(l)) s.j[1] += cy(l) * fv;
    if (cz(l)) s.j[2] += cz(l) * fv;
    if (cx(l)) s.P[0] += fv;
    if (cx(l) * cy(l)) s.P[1] += cx(l) * cy(l) * fv;
    if (cx(l) * cz(l)) s.P[2] += cx(l) * cz(l) * fv;
    if (cy(l)) s.P[3] += fv;
    if (cy(l) * cz(l)) s.P[4] += cy(l) * cz(l) * fv;
    if (cz(l)) s.P[5] += fv;
    s.re += gv;
    if (cx(l)) s.q[0] += cx(l) * gv;
    if (cy(l)) s.q[1] += cy(l) * gv;
    if (cz(l)) s.q[2] += cz(l) * gv;
}

__device__ __forceinline__ void sums_sc(const double f[27], const double ge[27], ScSums &s) {
    sums_init(s);
#pragma unroll
    for (int l = 0; l < 27; ++l) sums_add(s, l, f[l], ge[l]);
}

// The face-difference quantity of the collision's FD correction (src/lbm-collision.cpp:65-67).
__device__ __forceinline__ double qdev(double rho, double ua, double T, double R) {
    return rho * ua * (1.0 - 3.0 * R * T) - rho * (ua * ua * ua);
}

// The collision inputs that need the full pressure tensor and rho*E
// (src/lbm-collision.cpp:40-54, 72-74): S_b = sum_a u_a (P_ab - (p delta_ab + rho u_a u_b)),
// Uint = rhoE/rho - |u|^2/2.
__device__ __forceinline__ void coll_inputs(double rho, const double u[3], double p, const double P6[6], double rhoe,
                                            double S[3], double &Uint) {
    const double Pf[3][3] = {{P6[0], P6[1], P6[2]}, {P6[1], P6[3], P6[4]}, {P6[2], P6[4], P6[5]}};
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) s += u[a] * (Pf[a][b] - ((a == b ? p : 0.0) + rho * u[a] * u[b]));
        S[b] = s;
    }
    Uint = rhoe / rho - 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
}

// Stores the step record of a fluid cell from its post-stream moment sums (reference
// LBM::calculate_moment, src/lbm-moment.cpp:11-125), with the state checks.
__device__ __forceinline__ void store_record_sc(const ScGeom &g, const ScPhys &P, long n, const ScSums &s,
                                                double *__restrict__ mom, unsigned *status) {
    const long nc = g.ncell;
    const double rho = s.rho;
    const double u[3] = {s.j[0] / rho, s.j[1] / rho, s.j[2] / rho};
    const double Uint0 = s.re / rho - 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double T = Uint0 / P.cv;
    const double p = rho * P.R * T;
    double S[3], Uint;
    coll_inputs(rho, u, p, s.P, s.re, S, Uint);
    mom[M_RHO * nc + n] = rho;
    mom[M_U * nc + n] = u[0];
    mom[M_V * nc + n] = u[1];
    mom[M_W * nc + n] = u[2];
    mom[M_T * nc + n] = T;
    mom[M_P * nc + n] = p;
    mom[M_QX * nc + n] = qdev(rho, u[0], T, P.R);
    mom[M_QY * nc + n] = qdev(rho, u[1], T, P.R);
    mom[M_QZ * nc + n] = qdev(rho, u[2], T, P.R);
    mom[M_SX * nc + n] = S[0];
    mom[M_SY * nc + n] = S[1];
    mom[M_SZ * nc + n] = S[2];
    mom[M_UINT * nc + n] = Uint;
    if (!isfinite(rho) || !isfinite(T) || !isfinite(u[0]) || !isfinite(u[1]) || !isfinite(u[2]))
        raise_status(status, LBMGPU_ST_NAN);
    else if (!(rho > 0.0) || !(T > 0.0))
        raise_status(status, LBMGPU_ST_NEG_STATE);
}

}  // namespace lbm
