// Single-component thermal D3Q27 step kernels (reference: MULTICOMP off).
//
// Device state (structure of arrays, cell index n = (i*Ny + j)*Nz + k, k fastest, ghosts
// included so the index arithmetic is the reference's):
//   pop[2]  : 54 planes of ncell values -- f directions 0..26, then g directions 0..26.
//             Holds the post-collision populations fpc/gpc of the last step (or, right
//             after an upload/Init, the populations f/g themselves: "local" mode).
//   mom[2]  : 6 planes -- rho, u, v, w, temp, p (the moments the neighbours and the
//             boundary treatment read).  Double-buffered: the boundary step of step n+1
//             reads step n's moments while the moment step writes step n+1's.
//   minit   : 7 planes -- P00 P01 P02 P11 P12 P22 rhoe, used only by the first collision
//             after an upload/Init (the reference's first Collide uses the moments Init
//             left, which are not those of the populations: src/lbm-init.cpp:21-60).
//   bst[2]  : 54 values per boundary cell -- post-boundary populations f, g of cells next
//             to solid/inflow/outflow cells, whose populations along those directions
//             persist from step to step (src/lbm-streaming.cpp:25-32, 63-87).
//
// One time step = collide kernel (reads pop[cur], writes pop[nxt]) + stream/boundary/
// moment kernel (pulls pop[nxt], writes mom[nxt], bst[nxt]); then cur <-> nxt.
#pragma once
#include <cstdint>
#include "d3q27.cuh"

namespace lbm {

enum : int { M_RHO = 0, M_U = 1, M_V = 2, M_W = 3, M_T = 4, M_P = 5, M_N = 6 };
enum : uint8_t { CF_FLUID = 1, CF_SLOW = 2, CF_BOUND = 4 };

struct ScGeom {
    int Nx, Ny, Nz;
    long ncell;
    long sj, si;  // strides of j and i (Nz, Ny*Nz)
};

struct ScPhys {
    double nu, R, gamma, prtl, dt, cv, cp;
};

struct ScStatusPtr {
    unsigned *flags;
};

__device__ __forceinline__ void raise_status(unsigned *flags, unsigned bits) { atomicOr(flags, bits); }

__device__ __forceinline__ long nb_index(const ScGeom &g, long n, int dx, int dy, int dz) {
    return n + dx * g.si + dy * g.sj + dz;
}

// Specular partner of direction l off a free-slip neighbour (reference LBM::dirSlip,
// src/lbm-bc.cpp:1352-1399).
__device__ __forceinline__ void dir_slip(const ScGeom &g, const int8_t *__restrict__ type, int l, int i, int j,
                                         int k, int &lp, long &src) {
    const int inb = i - cx(l), jnb = j - cy(l), knb = k - cz(l);
    int cxp = cx(l), cyp = cy(l), czp = cz(l);
    int ip = inb, jp = jnb, kp = knb;
    if (type[(long)inb * g.si + (long)j * g.sj + k] == T_FS) {
        cxp = -cxp;
        ip = i;
    } else if (type[(long)i * g.si + (long)jnb * g.sj + k] == T_FS) {
        cyp = -cyp;
        jp = j;
    } else if (type[(long)i * g.si + (long)j * g.sj + knb] == T_FS) {
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

// Streaming (reference LBM::Streaming, src/lbm-streaming.cpp:3-119) of one fluid cell
// into f[27], g[27], pulling post-collision values from `pop`.  `stale` (boundary cells
// only) holds the cell's previous post-boundary populations, which persist along
// directions whose upstream neighbour is an inflow/outflow cell (f and g) or a solid
// cell (g only).
template <typename R>
__device__ __forceinline__ void pull_cell(const ScGeom &g, const int8_t *__restrict__ type, uint8_t cflag, long n,
                                          const R *__restrict__ pop, const R *__restrict__ stale, long nb_stride,
                                          R f[27], R ge[27]) {
    const long nc = g.ncell;
    if (!(cflag & CF_SLOW)) {
#pragma unroll
        for (int l = 0; l < 27; ++l) {
            const long s = nb_index(g, n, -cx(l), -cy(l), -cz(l));
            f[l] = pop[(long)l * nc + s];
            ge[l] = pop[(long)(27 + l) * nc + s];
        }
        return;
    }
    const int i = (int)(n / g.si);
    const int j = (int)((n / g.sj) % g.Ny);
    const int k = (int)(n % g.Nz);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        int in = i - cx(l), jn = j - cy(l), kn = k - cz(l);
        const int tn = type[(long)in * g.si + (long)jn * g.sj + kn];
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

__device__ __forceinline__ int type_at(const ScGeom &g, const int8_t *__restrict__ type, int i, int j, int k) {
    return type[(long)i * g.si + (long)j * g.sj + k];
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
// in the reference's pass order.  `mom` holds the moments of the previous step.
__device__ void tms_cell_sc(const ScGeom &g, const ScPhys &P, const int8_t *__restrict__ type,
                            const double *__restrict__ mom, long n, double f[27], double ge[27]) {
    const long nc = g.ncell;
    const int i = (int)(n / g.si);
    const int j = (int)((n / g.sj) % g.Ny);
    const int k = (int)(n % g.Nz);
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

__device__ __forceinline__ void sums_sc(const double f[27], const double ge[27], ScSums &s) {
    s.rho = 0;
    s.re = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        s.j[a] = 0;
        s.q[a] = 0;
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) s.P[a] = 0;
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const double fv = f[l], gv = ge[l];
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
}

}  // namespace lbm
