// lbmgpu: B200 (sm_100a) device implementation of the D3Q27 thermal LBM time step and
// the C ABI declared in include/lbmgpu.h.
//
// Reference path replaced (farrasarira/Lattice-Boltzmann-Method, single component):
//   LBM::Collide            src/lbm-collision.cpp:9-99     -> k_sc_collide
//   LBM::Streaming          src/lbm-streaming.cpp:3-119    -> k_sc_stream_moment (pull)
//   LBM::TMS_BC             src/lbm-bc.cpp:341-460, 809-938, 1111-1229 -> k_sc_stream_moment
//   LBM::calculate_moment   src/lbm-moment.cpp:11-125      -> k_sc_stream_moment
//   LBM::Init               src/lbm-init.cpp:8-82          -> k_sc_init
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/lbmgpu.h"
#include "handle.cuh"
#include "mc_ops.cuh"
#include "sc_kernels.cuh"
#include "sums.cuh"
#include "halo.cuh"

using namespace lbm;
using lbmh::MixOff;

namespace {

using lbmh::kBlock;
using lbmh::PK_UPLOADED;
using lbmh::PK_INIT;
using lbmh::PK_STEPPED;

__device__ __forceinline__ bool wall_like(int t) {
    return t == T_S || t == T_A || t == T_FS || t == T_P || t == T_O || t == T_O_C;
}

// fd_central (reference src/headers/FD.hpp:108-127) with dx = 1.
__device__ __forceinline__ double fd_central(double sl, double sc, double sr, int tl, int tr) {
    if (wall_like(tl)) return (tr == T_P) ? 0.0 : (sr - sc);
    if (wall_like(tr)) return (tl == T_P) ? 0.0 : (sc - sl);
    return (sr - sl) / 2.0;
}

// ----------------------------------------------------------------------------------
// Collision (reference LBM::Collide, single component, src/lbm-collision.cpp:9-99).
// Reads the step record of the cell and the Q terms of its six face neighbours, then
// streams through the 27 directions: fetch f_l, g_l (pulled from the last collision's
// output, or the special-cell store, or -- in local mode -- in place), relax, store.
// ----------------------------------------------------------------------------------
// Population q (0..53: f then g) of cell n at the start of the collision: in place
// (local mode), from the special-cell store, or pulled from the upstream cell.
__device__ __forceinline__ double fetch_pop(const double *__restrict__ src, const double *__restrict__ bst, long nc,
                                            long nb, long n, long b, const PullSrc &ps, int q, bool local,
                                            bool special) {
    if (local) return src[(long)q * nc + n];
    if (special) return bst[(long)q * nb + b];
    return src[(long)q * nc + pull_at(ps, q % 27)];
}

template <bool LOCAL>
__global__ void __launch_bounds__(kBlock, 4)
    k_sc_collide(ScGeom g, ScPhys P, const int8_t *__restrict__ type, const uint8_t *__restrict__ cflag,
                 const int *__restrict__ bid, const double *__restrict__ src, double *__restrict__ dst,
                 const double *__restrict__ mom, const double *__restrict__ bst, long nb, unsigned *status) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.ncell) return;
    const uint8_t cf = cflag[n];
    if (!(cf & CF_FLUID)) return;
    const long nc = g.ncell;

    const double rho = mom[M_RHO * nc + n];
    const double vel[3] = {mom[M_U * nc + n], mom[M_V * nc + n], mom[M_W * nc + n]};
    const double T = mom[M_T * nc + n];
    const double p = mom[M_P * nc + n];
    const double S[3] = {mom[M_SX * nc + n], mom[M_SY * nc + n], mom[M_SZ * nc + n]};
    const double Uint = mom[M_UINT * nc + n];

    const double dt = P.dt;
    const double theta = P.R * T;
    const double mu = P.nu * rho;
    const double kappa = mu * P.cp / P.prtl;
    const double om1 = 2 * p * P.cp * dt / (p * P.cp * dt + 2 * kappa);
    const double om = 2 * p * dt / (p * dt + 2 * mu);
    if (!(1.0 / om > 0.5) || !(1.0 / om1 > 0.5)) raise_status(status, LBMGPU_ST_TAU_UNSTABLE);

    double dq[3], corr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const long off = a == 0 ? g.si : (a == 1 ? g.sj : 1);
        const long nlo = n - off, nhi = n + off;
        const double *Q = mom + (long)(M_QX + a) * nc;
        const double dQ = fd_central(Q[nlo], Q[n], Q[nhi], type[nlo], type[nhi]);
        dq[a] = S[a] + 0.5 * dt * vel[a] * dQ;
        corr[a] = dt * (2 - om) / (2 * rho * om) * dQ;
    }
    AxisF<double> F;
    axis_feq(F, vel, theta, corr);
    AxisG<double> G;
    axis_geq(G, Uint, theta, vel);

    const bool special = cf & CF_SPECIAL;
    PullSrc ps;
    if (!LOCAL && !special) pull_src(g, n, ps);
    const long b = special ? (long)bid[n] : 0;
    // Each population set is fetched with all 27 loads issued back to back before any is
    // used (the kernel is bound by memory latency; this keeps 27 loads in flight per
    // thread), then relaxed and stored.
    double v[27];
#pragma unroll
    for (int l = 0; l < 27; ++l) v[l] = fetch_pop(src, bst, nc, nb, n, b, ps, l, LOCAL, special);
#pragma unroll
    for (int l = 0; l < 27; ++l) dst[(long)l * nc + n] = (1.0 - om) * v[l] + om * feq_l(l, rho, F);
#pragma unroll
    for (int l = 0; l < 27; ++l) v[l] = fetch_pop(src, bst, nc, nb, n, b, ps, 27 + l, LOCAL, special);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const double gq = geq_l(l, rho, G);
        const double gs = (csq(l) == 1) ? gq + 0.5 * (cx(l) * dq[0] + cy(l) * dq[1] + cz(l) * dq[2]) : gq;
        dst[(long)(27 + l) * nc + n] = v[l] + om1 * (gq - v[l]) + (om - om1) * (gq - gs);
    }
}

// ----------------------------------------------------------------------------------
// Streaming + moments for the cells with no boundary neighbour (reference LBM::Streaming
// and LBM::calculate_moment, src/lbm-streaming.cpp:88-117, src/lbm-moment.cpp:11-125).
// ----------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock, 4)
    k_sc_stream_moment(ScGeom g, ScPhys P, const uint8_t *__restrict__ cflag, const double *__restrict__ src,
                       double *__restrict__ mom_nxt, unsigned *status) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.ncell) return;
    if (cflag[n] != CF_FLUID) return;  // not fluid, or special (k_sc_stream_moment_special)
    const long nc = g.ncell;
    PullSrc ps;
    pull_src(g, n, ps);
    ScSums s;
    sums_init(s);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const long sidx = pull_at(ps, l);
        sums_add(s, l, src[(long)l * nc + sidx], src[(long)(27 + l) * nc + sidx]);
    }
    store_record_sc(g, P, n, s, mom_nxt, status);
}

// The same for the special cells (compact list): streaming with bounce-back, free-slip
// and persisting populations, the TMS boundary treatment (reference LBM::TMS_BC), moments.
__global__ void __launch_bounds__(kBlock)
    k_sc_stream_moment_special(ScGeom g, ScPhys P, const int8_t *__restrict__ type, const long *__restrict__ blist,
                               const double *__restrict__ src, const double *__restrict__ mom_cur,
                               double *__restrict__ mom_nxt, const double *__restrict__ bst_cur,
                               double *__restrict__ bst_nxt, long nb, unsigned *status) {
    const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const long n = blist[b];
    double f[27], ge[27];
    pull_special(g, type, n, src, bst_cur + b, nb, f, ge);
    tms_cell_sc(g, P, type, mom_cur, n, f, ge);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        bst_nxt[(long)l * nb + b] = f[l];
        bst_nxt[(long)(27 + l) * nb + b] = ge[l];
    }
    ScSums s;
    sums_sc(f, ge, s);
    store_record_sc(g, P, n, s, mom_nxt, status);
}

// ----------------------------------------------------------------------------------
// Init (reference LBM::Init, single component, src/lbm-init.cpp:8-82)
// ----------------------------------------------------------------------------------
// Moment-form energy equilibrium (reference calculate_geq(l, rhoe, q, R, theta),
// src/lbm-edf.cpp:100-138) for a diagonal R tensor R = r*I (all Init ever passes).
__device__ __forceinline__ double geq_moment_diag(int l, double rhoe, const double q[3], double rdiag, double theta) {
    const double c[3] = {(double)cx(l), (double)cy(l), (double)cz(l)};
    double val = rhoe + (q[0] * c[0] + q[1] * c[1] + q[2] * c[2]) / theta;
    double contr = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) contr += (rdiag - rhoe * theta) * (c[a] * c[a] - theta);
    val += contr / (2.0 * theta * theta);
    double wgt = 1.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) wgt *= (c[m] == 0.0) ? (1.0 - theta) : theta / 2.0;
    val *= wgt;
    const int c2 = csq(l);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const double Bm = (c2 == 0) ? 1.0 : (c2 == 1 ? -0.5 * fabs(c[m]) : 0.0);
        val += Bm * ((1.0 - 3.0 * theta) / (2.0 * theta) * (rdiag - theta * rhoe));
    }
    return val;
}

__device__ __forceinline__ void put_record_both(double *m0, double *m1, long nc, long n, int field, double v) {
    m0[(long)field * nc + n] = v;
    m1[(long)field * nc + n] = v;
}

__global__ void __launch_bounds__(kBlock)
    k_sc_init(ScGeom g, ScPhys P, const int8_t *__restrict__ type, const uint8_t *__restrict__ cflag,
              const int *__restrict__ bid, double *__restrict__ pop, double *__restrict__ mom0,
              double *__restrict__ mom1, double *__restrict__ bst, long nb) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.ncell) return;
    const int t = type[n];
    if (!(t == T_F || t == T_S || t == T_I || t == T_O || t == T_Q)) return;
    const long nc = g.ncell;
    const double p = mom0[M_P * nc + n];
    const double T = mom0[M_T * nc + n];
    const double rho = p / (P.R * T);
    const double u[3] = {mom0[M_U * nc + n], mom0[M_V * nc + n], mom0[M_W * nc + n]};
    put_record_both(mom0, mom1, nc, n, M_RHO, rho);
#pragma unroll
    for (int a = 0; a < 3; ++a) put_record_both(mom0, mom1, nc, n, M_QX + a, qdev(rho, u[a], T, P.R));
    if (!(cflag[n] & CF_FLUID)) return;
    const double theta = P.R * T;
    const double rhoe = rho * (P.cv * T);
    const double H = P.cp * T;
    const double P6[6] = {p, 0.0, 0.0, p, 0.0, p};
    double S[3], Uint;
    coll_inputs(rho, u, p, P6, rhoe, S, Uint);
#pragma unroll
    for (int a = 0; a < 3; ++a) put_record_both(mom0, mom1, nc, n, M_SX + a, S[a]);
    put_record_both(mom0, mom1, nc, n, M_UINT, Uint);
    const double q[3] = {H * rho * u[0], H * rho * u[1], H * rho * u[2]};
    const double vel0[3] = {0.0, 0.0, 0.0}, zero[3] = {0.0, 0.0, 0.0};
    AxisF<double> F;
    axis_feq(F, vel0, theta, zero);
    const long b = (cflag[n] & CF_SPECIAL) ? bid[n] : -1;
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const double fv = feq_l(l, rho, F);
        const double gv = geq_moment_diag(l, rhoe, q, H * p, theta);
        pop[(long)l * nc + n] = fv;
        pop[(long)(27 + l) * nc + n] = gv;
        if (b >= 0) {
            bst[(long)l * nb + b] = fv;
            bst[(long)(27 + l) * nb + b] = gv;
        }
    }
}

// ----------------------------------------------------------------------------------
// AoS <-> SoA packing for upload/download (the caller's MIXTURE records)
// ----------------------------------------------------------------------------------

__device__ __forceinline__ double ld(const char *rec, long off) { return *reinterpret_cast<const double *>(rec + off); }
__device__ __forceinline__ void st(char *rec, long off, double v) { *reinterpret_cast<double *>(rec + off) = v; }

__global__ void k_sc_unpack(ScGeom g, ScPhys P, MixOff o, const char *__restrict__ stage, long n0, long n1,
                            const uint8_t *__restrict__ cflag, const int *__restrict__ bid, double *__restrict__ pop,
                            double *__restrict__ mom0, double *__restrict__ mom1, double *__restrict__ bst, long nb) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    const char *rec = stage + (n - n0) * o.size;
    const long nc = g.ncell;
    const double rho = ld(rec, o.rho), T = ld(rec, o.temp), p = ld(rec, o.p);
    const double u[3] = {ld(rec, o.u), ld(rec, o.v), ld(rec, o.w)};
    put_record_both(mom0, mom1, nc, n, M_RHO, rho);
    put_record_both(mom0, mom1, nc, n, M_U, u[0]);
    put_record_both(mom0, mom1, nc, n, M_V, u[1]);
    put_record_both(mom0, mom1, nc, n, M_W, u[2]);
    put_record_both(mom0, mom1, nc, n, M_T, T);
    put_record_both(mom0, mom1, nc, n, M_P, p);
    for (int a = 0; a < 3; ++a) put_record_both(mom0, mom1, nc, n, M_QX + a, qdev(rho, u[a], T, P.R));
    if (!(cflag[n] & CF_FLUID)) return;
    const int pi[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    double P6[6];
    for (int a = 0; a < 6; ++a) P6[a] = ld(rec, o.p_tensor + 8 * (3 * pi[a][0] + pi[a][1]));
    double S[3], Uint;
    coll_inputs(rho, u, p, P6, ld(rec, o.rhoe), S, Uint);
    for (int a = 0; a < 3; ++a) put_record_both(mom0, mom1, nc, n, M_SX + a, S[a]);
    put_record_both(mom0, mom1, nc, n, M_UINT, Uint);
    const long b = (cflag[n] & CF_SPECIAL) ? bid[n] : -1;
    for (int l = 0; l < 27; ++l) {
        const double fv = ld(rec, o.f + 8 * l), gv = ld(rec, o.g + 8 * l);
        pop[(long)l * nc + n] = fv;
        pop[(long)(27 + l) * nc + n] = gv;
        if (b >= 0) {
            bst[(long)l * nb + b] = fv;
            bst[(long)(27 + l) * nb + b] = gv;
        }
    }
}

template <int MODE>
__global__ void k_sc_pack(ScGeom g, ScPhys P, MixOff o, char *__restrict__ stage, long n0, long n1,
                          const int8_t *__restrict__ type, const uint8_t *__restrict__ cflag,
                          const int *__restrict__ bid, const double *__restrict__ pop, const double *__restrict__ mom,
                          const double *__restrict__ bst, long nb) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    char *rec = stage + (n - n0) * o.size;
    const long nc = g.ncell;
    const long offs[6] = {o.rho, o.u, o.v, o.w, o.temp, o.p};
    const int fld[6] = {M_RHO, M_U, M_V, M_W, M_T, M_P};
    for (int m = 0; m < 6; ++m) st(rec, offs[m], mom[(long)fld[m] * nc + n]);
    const uint8_t cf = cflag[n];
    if (!(cf & CF_FLUID)) return;
    const bool special = cf & CF_SPECIAL;
    PullSrc ps;
    if (MODE == PK_STEPPED && !special) pull_src(g, n, ps);
    const long b = special ? (long)bid[n] : 0;
    ScSums s;
    sums_init(s);
    for (int l = 0; l < 27; ++l) {
        double fv, gv;
        if (MODE != PK_STEPPED) {
            fv = pop[(long)l * nc + n];
            gv = pop[(long)(27 + l) * nc + n];
        } else if (special) {
            fv = bst[(long)l * nb + b];
            gv = bst[(long)(27 + l) * nb + b];
        } else {
            const long sidx = pull_at(ps, l);
            fv = pop[(long)l * nc + sidx];
            gv = pop[(long)(27 + l) * nc + sidx];
        }
        st(rec, o.f + 8 * l, fv);
        st(rec, o.g + 8 * l, gv);
        if (MODE == PK_STEPPED) {
            st(rec, o.fpc + 8 * l, pop[(long)l * nc + n]);
            st(rec, o.gpc + 8 * l, pop[(long)(27 + l) * nc + n]);
            sums_add(s, l, fv, gv);
        }
    }
    const int full[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    if (MODE == PK_STEPPED) {
        for (int a = 0; a < 9; ++a) st(rec, o.p_tensor + 8 * a, s.P[full[a]]);
        st(rec, o.rhoe, s.re);
        for (int a = 0; a < 3; ++a) st(rec, o.energy_flux + 8 * a, s.q[a]);
    } else if (MODE == PK_INIT) {
        // Init leaves p_tensor = p I and rhoe = rho cv T (src/lbm-init.cpp:30-43)
        const double p = mom[M_P * nc + n], rho = mom[M_RHO * nc + n], T = mom[M_T * nc + n];
        for (int a = 0; a < 9; ++a) st(rec, o.p_tensor + 8 * a, (a % 4 == 0) ? p : 0.0);
        st(rec, o.rhoe, rho * (P.cv * T));
    }
}

}  // namespace

namespace {
using namespace lbmh;

int launch_collide(lbmgpu *h) {
    if (h->ns > 0) return lbmh::mc_launch_collide(h);
    const int c = h->cur, x = 1 - c;
    EvPair ep{};
    ev_begin(h, K_COLLIDE, ep);
    if (h->pack_mode != PK_STEPPED)
        k_sc_collide<true><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(
            h->g, h->P, h->type, h->cflag, h->bid, h->pop[c], h->pop[x], h->mom[c], h->bst[c], h->nb, h->status);
    else
        k_sc_collide<false><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(
            h->g, h->P, h->type, h->cflag, h->bid, h->pop[c], h->pop[x], h->mom[c], h->bst[c], h->nb, h->status);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

int launch_stream_moment(lbmgpu *h) {
    if (h->ns > 0) return lbmh::mc_launch_stream(h);
    const int c = h->cur, x = 1 - c;
    EvPair ep{};
    ev_begin(h, K_STREAM_MOMENT, ep);
    k_sc_stream_moment<<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(h->g, h->P, h->cflag, h->pop[x],
                                                                        h->mom[x], h->status);
    ev_end(h, ep);
    CK(cudaGetLastError());
    if (h->nb > 0) {
        EvPair eb{};
        ev_begin(h, K_OTHER, eb);
        k_sc_stream_moment_special<<<grid_for(h->nb), kBlock, 0, h->stream>>>(
            h->g, h->P, h->type, h->blist, h->pop[x], h->mom[c], h->mom[x], h->bst[c], h->bst[x], h->nb, h->status);
        ev_end(h, eb);
        CK(cudaGetLastError());
    }
    h->cur = x;
    h->pack_mode = PK_STEPPED;
    return 0;
}

// Every index the kernels follow must lie inside the tables.
bool valid_mech(const lbmgpu_mech &m) {
    if (m.n_species < 1 || m.n_species > LBMGPU_MAX_SPECIES) return false;
    if (m.n_reactions < 0 || m.n_reactions > LBMGPU_MAX_REACTIONS) return false;
    for (int k = 0; k < m.n_species; ++k)
        if (!(m.W[k] > 0) || !(m.T_mid[k] > 0) || !(m.diameter[k] > 0) || !(m.well_depth[k] > 0)) return false;
    for (int r = 0; r < m.n_reactions; ++r) {
        if (m.rtype[r] < 0 || m.rtype[r] > 2) return false;
        if (m.n_reac[r] < 1 || m.n_reac[r] > LBMGPU_MAX_RSPEC || m.n_prod[r] < 1 || m.n_prod[r] > LBMGPU_MAX_RSPEC)
            return false;
        for (int j = 0; j < m.n_reac[r]; ++j)
            if (m.reac[r][j] < 0 || m.reac[r][j] >= m.n_species || !(m.order_reac[r][j] >= 0.0) ||
                !(m.order_reac[r][j] <= 4.0))
                return false;
        for (int j = 0; j < m.n_prod[r]; ++j)
            if (m.prod[r][j] < 0 || m.prod[r][j] >= m.n_species) return false;
        if (m.troe_n[r] != 0 && m.troe_n[r] != 3 && m.troe_n[r] != 4) return false;
    }
    return true;
}

bool valid_layout(const lbmgpu_mixture_layout &m) {
    const long need[] = {m.type, m.f, m.fpc, m.p_tensor, m.rho, m.u, m.v, m.w, m.p, m.g, m.gpc, m.rhoe,
                         m.energy_flux, m.temp};
    if (m.size == 0 || (m.size % 8) != 0) return false;
    for (long o : need)
        if (o < 0 || (size_t)o >= m.size) return false;
    const long dbl[] = {m.f, m.fpc, m.p_tensor, m.rho, m.u, m.v, m.w, m.p, m.g, m.gpc, m.rhoe, m.energy_flux, m.temp};
    for (long o : dbl)
        if (o % 8) return false;
    // every field must lie inside the record: arrays of 27, 9 and 3 doubles, scalars, a short type
    const long ext[][2] = {{m.f, 216}, {m.fpc, 216}, {m.g, 216}, {m.gpc, 216}, {m.p_tensor, 72}, {m.energy_flux, 24},
                           {m.rho, 8}, {m.u, 8}, {m.v, 8}, {m.w, 8}, {m.p, 8}, {m.rhoe, 8}, {m.temp, 8}, {m.type, 2}};
    for (const auto &e : ext)
        if ((size_t)(e[0] + e[1]) > m.size) return false;
    return true;
}

}  // namespace

using namespace lbmh;

extern "C" {

const char *lbmgpu_error_string(int code) {
    switch (code) {
        case LBMGPU_OK: return "ok";
        case LBMGPU_E_ARG: return "invalid argument or descriptor";
        case LBMGPU_E_CUDA: return "CUDA runtime error";
        case LBMGPU_E_NODEV: return "no usable CUDA device or kernel image (sm_100a build)";
        case LBMGPU_E_PHASE: return "phase called out of the reference's step order";
        case LBMGPU_E_STATE: return "no state uploaded yet";
        case LBMGPU_E_UNSUPPORTED: return "configuration not supported";
        case LBMGPU_E_VERSION: return "descriptor abi_version mismatch";
        case LBMGPU_E_IO: return "file could not be opened, read or written";
        default: return code > 0 ? "device status bits raised" : "unknown error";
    }
}

int lbmgpu_create(const lbmgpu_desc *desc, lbmgpu_t **out) {
    if (!desc || !out) return LBMGPU_E_ARG;
    *out = nullptr;
    if (desc->abi_version != LBMGPU_ABI_VERSION) return LBMGPU_E_VERSION;
    if (desc->Nx < 3 || desc->Ny < 3 || desc->Nz < 3) return LBMGPU_E_ARG;
    if (desc->precision != LBMGPU_FP64 && desc->precision != LBMGPU_FP32) return LBMGPU_E_ARG;
    if (desc->precision == LBMGPU_FP32 && desc->n_species == 0) return LBMGPU_E_UNSUPPORTED;  // FP32: multicomponent
    if (desc->dt_sim <= 0) return LBMGPU_E_ARG;
    if (desc->n_species == 0) {
        if (!(desc->gamma > 1.0) || !(desc->gas_const > 0.0) || !(desc->prtl > 0.0) || !(desc->nu >= 0.0))
            return LBMGPU_E_ARG;
        if (!valid_layout(desc->mix)) return LBMGPU_E_ARG;
    } else {
        if (!desc->mech || desc->mech->n_species != desc->n_species) return LBMGPU_E_ARG;
        if (!valid_mech(*desc->mech)) return LBMGPU_E_ARG;
        if (!lbmh::mc_ns_built(desc->n_species)) return LBMGPU_E_UNSUPPORTED;  // the kernels' species counts
        if (desc->chem_mode != LBMGPU_CHEM_OFF && desc->chem_mode != LBMGPU_CHEM_REF_EXPLICIT &&
            desc->chem_mode != LBMGPU_CHEM_ROSENBROCK)
            return LBMGPU_E_UNSUPPORTED;
        if (!(desc->units_m > 0.f) || !(desc->units_kg > 0.f) || !(desc->units_s > 0.f) || !(desc->units_K > 0.f))
            return LBMGPU_E_ARG;
    }
    if ((double)desc->Nx * desc->Ny * desc->Nz > 2147483647.0) return LBMGPU_E_UNSUPPORTED;  // 32-bit cell offsets
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        (void)cudaGetLastError();
        return LBMGPU_E_NODEV;
    }
    if (desc->device < 0 || desc->device >= ndev) return LBMGPU_E_ARG;
    CK(cudaSetDevice(desc->device));
    lbmgpu *h = new (std::nothrow) lbmgpu();
    if (!h) return LBMGPU_E_ARG;
    h->d = *desc;
    h->g.Nx = desc->Nx;
    h->g.Ny = desc->Ny;
    h->g.Nz = desc->Nz;
    h->g.sj = desc->Nz;
    h->g.si = (long)desc->Ny * desc->Nz;
    h->g.ncell = (long)desc->Nx * desc->Ny * desc->Nz;
    h->P.nu = desc->nu;
    h->P.R = desc->gas_const;
    h->P.gamma = desc->gamma;
    h->P.prtl = desc->prtl;
    h->P.dt = desc->dt_sim;
    h->P.cv = desc->gas_const / (desc->gamma - 1.0);
    h->P.cp = h->P.cv + desc->gas_const;
    const lbmgpu_mixture_layout &m = desc->mix;
    h->mo = MixOff{(long)m.size, m.type, m.f,   m.fpc,  m.p_tensor,    m.rho,  m.u,  m.v,
                   m.w,           m.p,    m.g,   m.gpc,  m.rhoe,        m.energy_flux, m.temp, m.HRR};
    const long nc = h->g.ncell;
    int rc = 0;
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_fail(e);
    if (!rc) rc = dalloc(h, &h->type, nc);
    if (!rc) rc = dalloc(h, &h->cflag, nc);
    if (!rc) rc = dalloc(h, &h->bid, nc);
    if (desc->n_species == 0) {
        for (int b = 0; b < 2 && !rc; ++b) rc = dalloc(h, &h->pop[b], 54 * (size_t)nc);
        for (int b = 0; b < 2 && !rc; ++b) rc = dalloc(h, &h->mom[b], (size_t)M_N * nc);
    } else if (!rc) {
        rc = lbmh::mc_setup(h);
    }
    if (!rc) rc = dalloc(h, &h->status, 1);
    // load the reduction kernels' module and the fixed scratch of lbmgpu_sums_noalloc now,
    // while allocating is allowed (lazy module loading would do it at their first use)
    if (!rc) rc = lbmh::sums_preload();
    if (!rc) rc = lbmh::noalloc_prepare();
    if (!rc) {
        e = cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->stream);
        if (e != cudaSuccess) rc = cuda_fail(e);
    }
    if (!rc) {
        // staging for AoS transfers: up to 256 MiB of records (mixture + species) per chunk
        const size_t per_cell = m.size + (size_t)desc->n_species * desc->spc.size;
        h->stage_cells = std::max<size_t>(1, std::min<size_t>((size_t)nc, (256u << 20) / per_cell));
        h->stage_bytes = h->stage_cells * per_cell;
        rc = dalloc(h, &h->stage, h->stage_bytes);
        if (!rc) {
            e = cudaMallocHost(reinterpret_cast<void **>(&h->bounce), h->stage_bytes);
            if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&h->bounce2), h->stage_bytes);
            if (e != cudaSuccess) rc = cuda_fail(e);
        }
    }
    if (rc) {
        lbmgpu_destroy(h);
        return rc;
    }
    *out = h;
    return LBMGPU_OK;
}

int lbmgpu_destroy(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    cudaSetDevice(h->d.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto &e : h->pending) h->pool.push_back(e);
    for (auto &e : h->pool) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    cudaFree(h->type);
    cudaFree(h->cflag);
    cudaFree(h->bid);
    cudaFree(h->blist);
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->pop[b]);
        cudaFree(h->mom[b]);
        cudaFree(h->bst[b]);
    }
    cudaFree(h->status);
    cudaFree(h->sum_scratch);
    cudaFree(h->stage);
    if (h->bounce) cudaFreeHost(h->bounce);
    if (h->bounce2) cudaFreeHost(h->bounce2);
    lbmh::mc_release(h);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    (void)cudaGetLastError();
    delete h;
    return LBMGPU_OK;
}

int lbmgpu_upload(lbmgpu_t *h, const void *mixture_aos, const void *const *species_aos) {
    if (!h || !mixture_aos) return LBMGPU_E_ARG;
    if (h->ns > 0) return lbmh::mc_upload(h, mixture_aos, species_aos);
    CK(cudaSetDevice(h->d.device));
    const ScGeom &g = h->g;
    const long nc = g.ncell;
    const size_t rs = h->mo.size;
    const char *host = static_cast<const char *>(mixture_aos);
    // cell types and the per-cell classification, computed on the host once per upload
    std::vector<int8_t> ty(nc);
    for (long n = 0; n < nc; ++n) {
        short t;
        std::memcpy(&t, host + n * rs + h->mo.type, sizeof(short));
        if (t < 0 || t > 9) return LBMGPU_E_ARG;
        ty[n] = (int8_t)t;
    }
    std::vector<uint8_t> cf(nc, 0);
    std::vector<int> bidh(nc, -1);
    std::vector<long> blh;
    long nb = 0;
    for (int i = 0; i < g.Nx; ++i)
        for (int j = 0; j < g.Ny; ++j)
            for (int k = 0; k < g.Nz; ++k) {
                const long n = (long)i * g.si + (long)j * g.sj + k;
                if (ty[n] != T_F) continue;
                if (i == 0 || j == 0 || k == 0 || i == g.Nx - 1 || j == g.Ny - 1 || k == g.Nz - 1)
                    return LBMGPU_E_ARG;  // a fluid cell on the outermost layer has no ghost neighbour
                // special: a boundary cell upstream (solid, adiabatic, free-slip, inflow,
                // outflow); the others stream with the branch-free periodic pull
                uint8_t c = CF_FLUID;
                for (int l = 0; l < 27; ++l) {
                    const long s = n - (long)cx(l) * g.si - (long)cy(l) * g.sj - cz(l);
                    const int t = ty[s];
                    if (t == T_S || t == T_A || t == T_FS || t == T_I || t == T_O || t == T_I_C || t == T_O_C)
                        c |= CF_SPECIAL;
                }
                if (c & CF_SPECIAL) {
                    bidh[n] = (int)nb++;
                    blh.push_back(n);
                }
                cf[n] = c;
            }
    // (re)size the boundary store
    if (nb != h->nb || !h->bst[0]) {
        for (int b = 0; b < 2; ++b) {
            if (h->bst[b]) {
                cudaFree(h->bst[b]);
                h->bytes -= 54 * (size_t)h->nb * sizeof(double);
                h->bst[b] = nullptr;
            }
        }
        if (h->blist) {
            cudaFree(h->blist);
            h->bytes -= (size_t)std::max<long>(h->nb, 1) * sizeof(long);
            h->blist = nullptr;
        }
        h->nb = nb;
        for (int b = 0; b < 2; ++b) {
            int rc = dalloc(h, &h->bst[b], 54 * (size_t)std::max<long>(nb, 1));
            if (rc) return rc;
        }
        int rc = dalloc(h, &h->blist, (size_t)std::max<long>(nb, 1));
        if (rc) return rc;
    }
    if (nb > 0) CK(cudaMemcpyAsync(h->blist, blh.data(), nb * sizeof(long), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->type, ty.data(), nc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->cflag, cf.data(), nc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->bid, bidh.data(), nc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    for (long n0 = 0; n0 < nc; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(nc, n0 + (long)h->stage_cells);
        CK(cudaMemcpyAsync(h->stage, host + n0 * rs, (n1 - n0) * rs, cudaMemcpyHostToDevice, h->stream));
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        k_sc_unpack<<<grid_for(n1 - n0), kBlock, 0, h->stream>>>(g, h->P, h->mo, h->stage, n0, n1, h->cflag,
                                                                 h->bid, h->pop[0], h->mom[0], h->mom[1], h->bst[0],
                                                                 h->nb);
        ev_end(h, ep);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->stream));
    h->pack_mode = PK_UPLOADED;
    h->have_state = true;
    h->phase = lbmh::PH_BOUNDARY;
    return LBMGPU_OK;
}

int lbmgpu_upload_planes(lbmgpu_t *h, int i0, int i1, const void *mixture_aos, const void *const *species_aos) {
    if (!h || !mixture_aos) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    return lbmh::mc_upload_planes(h, i0, i1, mixture_aos, species_aos);
}

int lbmgpu_download_planes(lbmgpu_t *h, int i0, int i1, void *mixture_aos, void *const *species_aos) {
    if (!h || !mixture_aos) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    return lbmh::mc_download_planes(h, i0, i1, mixture_aos, species_aos);
}

int lbmgpu_set_halo(lbmgpu_t *h, int lo, int hi, int nx_global) {
    if (!h) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    if (nx_global < h->g.Nx || (lo != 0 && lo != 1) || (hi != 0 && hi != 1)) return LBMGPU_E_ARG;
    h->halo_lo = lo;
    h->halo_hi = hi;
    h->nx_glob = nx_global;
    h->have_state = false;  // the classification of the cells changes: upload again
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    return LBMGPU_OK;
}

int lbmgpu_halo_bytes(lbmgpu_t *h, int what, size_t *bytes) {
    if (!h || !bytes || (what != LBMGPU_HALO_POPULATIONS && what != LBMGPU_HALO_RECORD)) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    *bytes = (size_t)lbm::halo_values(what, h->ns) * h->g.Ny * h->g.Nz * sizeof(double);
    return LBMGPU_OK;
}

static int halo_call(lbmgpu_t *h, int face, int what, const void *buf, bool pack) {
    if (!h || !buf || (face != 0 && face != 1)) return LBMGPU_E_ARG;
    if (what != LBMGPU_HALO_POPULATIONS && what != LBMGPU_HALO_RECORD) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (!pack && !(face == 0 ? h->halo_lo : h->halo_hi)) return LBMGPU_E_ARG;  // no halo on that face
    // populations between Collide and calculate_moment, the record between steps
    const bool collided = h->phase == lbmh::PH_COLLIDED || h->phase == lbmh::PH_STREAMED || h->phase == lbmh::PH_BC;
    if (what == LBMGPU_HALO_POPULATIONS ? !collided : h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    return lbmh::mc_halo(h, face, what, static_cast<double *>(const_cast<void *>(buf)), pack);
}

int lbmgpu_halo_pack(lbmgpu_t *h, int face, int what, void *dev_buf) { return halo_call(h, face, what, dev_buf, true); }

int lbmgpu_halo_unpack(lbmgpu_t *h, int face, int what, const void *dev_buf) {
    return halo_call(h, face, what, dev_buf, false);
}

int lbmgpu_get_stream(lbmgpu_t *h, void **stream) {
    if (!h || !stream) return LBMGPU_E_ARG;
    *stream = static_cast<void *>(h->stream);
    return LBMGPU_OK;
}

int lbmgpu_download(lbmgpu_t *h, void *mixture_aos, void *const *species_aos) {
    if (!h || !mixture_aos) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    if (h->ns > 0) return lbmh::mc_download(h, mixture_aos, species_aos);
    CK(cudaSetDevice(h->d.device));
    const ScGeom &g = h->g;
    const long nc = g.ncell;
    const size_t rs = h->mo.size;
    char *host = static_cast<char *>(mixture_aos);
    std::vector<int8_t> ty(nc);
    CK(cudaMemcpyAsync(ty.data(), h->type, nc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int c = h->cur;
    const long mof[6] = {h->mo.rho, h->mo.u, h->mo.v, h->mo.w, h->mo.temp, h->mo.p};
    for (long n0 = 0; n0 < nc; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(nc, n0 + (long)h->stage_cells);
        CK(cudaMemsetAsync(h->stage, 0, (size_t)(n1 - n0) * rs, h->stream));  // zero padding bytes
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        const unsigned gb = grid_for(n1 - n0);
        if (h->pack_mode == PK_STEPPED)
            k_sc_pack<PK_STEPPED><<<gb, kBlock, 0, h->stream>>>(g, h->P, h->mo, h->stage, n0, n1, h->type, h->cflag,
                                                                h->bid, h->pop[c], h->mom[c], h->bst[c], h->nb);
        else if (h->pack_mode == PK_INIT)
            k_sc_pack<PK_INIT><<<gb, kBlock, 0, h->stream>>>(g, h->P, h->mo, h->stage, n0, n1, h->type, h->cflag,
                                                             h->bid, h->pop[c], h->mom[c], h->bst[c], h->nb);
        else
            k_sc_pack<PK_UPLOADED><<<gb, kBlock, 0, h->stream>>>(g, h->P, h->mo, h->stage, n0, n1, h->type,
                                                                 h->cflag, h->bid, h->pop[c], h->mom[c], h->bst[c],
                                                                 h->nb);
        ev_end(h, ep);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->bounce, h->stage, (n1 - n0) * rs, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        // merge: fluid cells take the whole record except the type; the others only
        // their stored moments (ghost populations are not represented on the device)
        for (long n = n0; n < n1; ++n) {
            const char *srec = h->bounce + (n - n0) * rs;
            char *drec = host + n * rs;
            if (ty[n] == T_F && h->pack_mode == PK_STEPPED) {
                // every field of a stepped fluid cell was produced: the whole record but the type
                short t;
                std::memcpy(&t, drec + h->mo.type, sizeof(short));
                std::memcpy(drec, srec, rs);
                std::memcpy(drec + h->mo.type, &t, sizeof(short));
            } else {
                for (int m = 0; m < 6; ++m) std::memcpy(drec + mof[m], srec + mof[m], sizeof(double));
                if (ty[n] == T_F) {
                    std::memcpy(drec + h->mo.f, srec + h->mo.f, 27 * sizeof(double));
                    std::memcpy(drec + h->mo.g, srec + h->mo.g, 27 * sizeof(double));
                    if (h->pack_mode == PK_INIT) {
                        std::memcpy(drec + h->mo.p_tensor, srec + h->mo.p_tensor, 9 * sizeof(double));
                        std::memcpy(drec + h->mo.rhoe, srec + h->mo.rhoe, sizeof(double));
                    }
                }
            }
        }
    }
    return LBMGPU_OK;
}

int lbmgpu_init(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    if (h->ns > 0) return lbmh::mc_init(h);
    if (h->cur != 0) {
        // Init always rebuilds the state in buffer 0 from the stored moments
        const long nc = h->g.ncell;
        CK(cudaMemcpyAsync(h->mom[0], h->mom[1], (size_t)M_N * nc * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->stream));
        h->cur = 0;
    }
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_sc_init<<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(h->g, h->P, h->type, h->cflag, h->bid, h->pop[0],
                                                              h->mom[0], h->mom[1], h->bst[0], h->nb);
    ev_end(h, ep);
    CK(cudaGetLastError());
    h->pack_mode = PK_INIT;
    return LBMGPU_OK;
}

// Multicomponent: Collide_Species and Collide run as one fused kernel, launched by
// lbmgpu_collide; Collide_Species must come first (src/lbm-main.cpp:157-163).
int lbmgpu_collide_species(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;  // single component: no species phase in the loop
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    h->phase = PH_SPECIES;
    return LBMGPU_OK;
}

int lbmgpu_collide(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != (h->ns > 0 ? PH_SPECIES : lbmh::PH_BOUNDARY)) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    int rc = launch_collide(h);
    if (rc) return rc;
    h->phase = PH_COLLIDED;
    return LBMGPU_OK;
}

int lbmgpu_streaming(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (h->phase != PH_COLLIDED) return LBMGPU_E_PHASE;
    h->phase = PH_STREAMED;
    return LBMGPU_OK;
}

int lbmgpu_tms_bc(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (h->phase != PH_STREAMED) return LBMGPU_E_PHASE;
    h->phase = PH_BC;
    return LBMGPU_OK;
}

int lbmgpu_calculate_moment(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    if (h->phase != PH_BC) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    int rc = launch_stream_moment(h);
    if (rc) return rc;
    h->phase = lbmh::PH_BOUNDARY;
    return LBMGPU_OK;
}

int lbmgpu_step(lbmgpu_t *h, int nsteps) {
    if (!h || nsteps < 0) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    for (int s = 0; s < nsteps; ++s) {
        int rc = launch_collide(h);
        if (!rc) rc = launch_stream_moment(h);
        if (rc) return rc;
    }
    return LBMGPU_OK;
}

int lbmgpu_time_steps(lbmgpu_t *h, int nsteps, double *ms) {
    if (!h || !ms || nsteps < 0) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != lbmh::PH_BOUNDARY) return LBMGPU_E_PHASE;
    CK(cudaSetDevice(h->d.device));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    int rc = 0;
    cudaError_t e = cudaEventRecord(a, h->stream);
    if (e != cudaSuccess) rc = cuda_fail(e);
    for (int s = 0; s < nsteps && !rc; ++s) {
        rc = launch_collide(h);
        if (!rc) rc = launch_stream_moment(h);
    }
    if (!rc) {
        e = cudaEventRecord(b, h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float t = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
        if (e != cudaSuccess) rc = cuda_fail(e);
        *ms = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

int lbmgpu_synchronize(lbmgpu_t *h) {
    if (!h) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    CK(cudaStreamSynchronize(h->stream));
    ev_drain(h);
    unsigned f = 0;
    CK(cudaMemcpyAsync(&f, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return (int)f;
}

int lbmgpu_status(lbmgpu_t *h, uint32_t *flags, int clear) {
    if (!h || !flags) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    CK(cudaStreamSynchronize(h->stream));
    unsigned f = 0;
    CK(cudaMemcpyAsync(&f, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *flags = f;
    if (clear) {
        CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return LBMGPU_OK;
}

int lbmgpu_profile(lbmgpu_t *h, int enable) {
    if (!h) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    CK(cudaStreamSynchronize(h->stream));
    ev_drain(h);
    h->prof = enable != 0;
    for (int k = 0; k < K_NKINDS; ++k) {
        h->launches[k] = 0;
        h->ms[k] = 0.0;
    }
    return LBMGPU_OK;
}

int lbmgpu_kernel_times(lbmgpu_t *h, int nkinds, long *launches, double *ms) {
    if (!h || nkinds < 0 || (nkinds > 0 && (!launches || !ms))) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    CK(cudaStreamSynchronize(h->stream));
    ev_drain(h);
    for (int k = 0; k < nkinds && k < K_NKINDS; ++k) {
        launches[k] = h->launches[k];
        ms[k] = h->ms[k];
    }
    return K_NKINDS;
}

int lbmgpu_units_from_dx_dt(float dx, float dt, float *out4) {
    if (!out4 || !(dx > 0.f) || !(dt > 0.f)) return LBMGPU_E_ARG;
    const lbm::UnitsF u = lbm::units_from_dx_dt(dx, dt);
    out4[0] = u.m;
    out4[1] = u.kg;
    out4[2] = u.s;
    out4[3] = u.K;
    return LBMGPU_OK;
}

int lbmgpu_device_bytes(lbmgpu_t *h, size_t *bytes) {
    if (!h || !bytes) return LBMGPU_E_ARG;
    *bytes = h->bytes;
    return LBMGPU_OK;
}

}  // extern "C"
