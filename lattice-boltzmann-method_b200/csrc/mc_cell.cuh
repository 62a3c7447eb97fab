// Multicomponent thermal D3Q27 step, per-cell logic (the reference with MULTICOMP on).
// Every function here is host/device: the kernels in mc.cu call them once per cell, and
// the tests build them for the host to compare with the reference's own solver.
//
// Device state (structure of arrays, cell index n = (i*Ny + j)*Nz + k); populations stored
// as AT::P (double: the bit-faithful FP64 mode; float: the FP32 mode), records as AT::R:
//   pop[2]: 27*(NS+1) planes -- species a, direction l at plane 27a + l; the energy
//           population g at plane 27 NS + l.  Post-collision values of the last step, or
//           (after an upload or Init, "local" mode) the populations themselves; the other
//           buffer then keeps the uploaded fpc, which the reference's skip rule for
//           vanishing species (src/lbm-collision.cpp:512-513) leaves in place.  With a
//           shift table a population is stored as its deviation from the plane's shift
//           (the mean of that population over the fluid cells at upload or Init) and
//           decoded to FP64 for all arithmetic.
//   rec[2]: mc_nrec(NS) planes per cell -- the state calculate_moment leaves
//           (src/lbm-moment.cpp:193-377): rho, u, v, w, T, p, rhoE, the pressure tensor
//           (6), HRR; the mixture face-difference term Q_a (src/lbm-collision.cpp:296-300,
//           with the composition gas constant a neighbour's value carries); then per
//           species rho_a, u_a (3: the Stefan-Maxwell velocities), X_a and the species
//           face-difference term Q_{a,x|y|z} (src/lbm-collision.cpp:487-489).  The
//           neighbours of a cell read only the Q terms of their axis, rho_a and rho.
#pragma once
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "d3q27.cuh"
#include "chem.cuh"
#include "kinetics_h2_air_9.cuh"
#include "surrogate.cuh"
#include "gas.cuh"
#include "units.cuh"

#if defined(__CUDACC__)
#define MC_HD __host__ __device__ __forceinline__
#define MC_HDN __host__ __device__
#else
#define MC_HD inline
#define MC_HDN inline
#endif

namespace lbm {

constexpr double kSpeciesMin = 1e-8;   // SPECIES_MIN, src/headers/defines.hpp:96

enum : int {
    RM_RHO = 0, RM_U = 1, RM_V = 2, RM_W = 3, RM_T = 4, RM_P = 5, RM_RHOE = 6, RM_P00 = 7,  // P00 P01 P02 P11 P12 P22
    RM_HRR = 13, RM_QX = 14, RM_SP = 17, RM_SPN = 8                                          // per species block
};
enum : int { RS_RHO = 0, RS_UX = 1, RS_X = 4, RS_QX = 5 };
MC_HD int mc_nrec(int ns) { return RM_SP + RM_SPN * ns; }
MC_HD int rs(int a, int f) { return RM_SP + RM_SPN * a + f; }

enum : int { CHEM_OFF = 0, CHEM_REF_EXPLICIT = 1, CHEM_ROSENBROCK = 2 };

template <typename P_, typename R_>
struct McArgsT {
    using P = P_;          // population storage type
    using R = R_;          // record storage type
    int Nx, Ny, Nz;
    long ncell, sj, si;
    int ns, dt, chem;
    // slab decomposition along x: the low / high x ghost plane is a halo holding the
    // neighbouring slab's cells (no periodic wrap through it), and the domain's global x
    // length with ghosts, for the boundary formulas' domain lengths
    int halo_lo, halo_hi, Nx_glob;
    UnitsF U;
    const gas::Tables *tab;
    const int8_t *type;
    const uint8_t *cflag;
    const P *pop_src;      // collide: pop[cur]; stream: the collide's output
    P *pop_dst;            // collide: pop[nxt]
    const P *pop_prev;     // collide: fpc of the previous step (skip rule); null in local mode
    const R *rec_cur;
    R *rec_nxt;
    const double *shift;   // per population plane, or null (no shift)
    unsigned *status;
    int local;
    // cells with a boundary upstream ("special"): compact index, and their streamed and
    // boundary-treated populations, 27 (NS+1) planes of nb entries
    const int *bid;
    const P *bst_cur;      // of the current step (collide, and the stale directions)
    P *bst_nxt;            // written by the boundary-cell kernel (k_mc_special)
    long nb;
    double *props;         // collision parameters per cell (mc_props_cell -> mc_relax_*)
    SurArgs sur;           // chemistry surrogate (LBMGPU_CHEM_ROSENBROCK only)
};
using McArgs = McArgsT<double, double>;

template <class AT, typename T>
MC_HD double rec(const AT &A, const T *r, int plane, long n) {
    return (double)r[(long)plane * A.ncell + n];
}
template <class AT, typename T>
MC_HD void put(const AT &A, T *r, int plane, long n, double v) {
    r[(long)plane * A.ncell + n] = (T)v;
}
template <class AT, typename T>
MC_HD double ldpop(const AT &A, const T *p, int plane, long idx) {
    const double v = (double)p[(long)plane * A.ncell + idx];
    return A.shift ? v + A.shift[plane] : v;
}
template <class AT, typename T>
MC_HD void stpop(const AT &A, T *p, int plane, long idx, double v) {
    p[(long)plane * A.ncell + idx] = (T)(A.shift ? v - A.shift[plane] : v);
}
// the same for the compact special-cell store (planes of nb entries)
template <class AT, typename T>
MC_HD double ldpop_b(const AT &A, const T *p, int plane, long b) {
    const double v = (double)p[(long)plane * A.nb + b];
    return A.shift ? v + A.shift[plane] : v;
}
template <class AT, typename T>
MC_HD void stpop_b(const AT &A, T *p, int plane, long b, double v) {
    p[(long)plane * A.nb + b] = (T)(A.shift ? v - A.shift[plane] : v);
}

// Adds `flag` (0 or 1) to a counter; on the device one atomic per warp.
MC_HD void count_flag(double *c, bool flag) {
#if defined(__CUDA_ARCH__)
    const unsigned act = __activemask();
    const unsigned votes = __ballot_sync(act, flag);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(act) - 1) && votes) atomicAdd(c, (double)__popc(votes));
#else
    *c += flag ? 1.0 : 0.0;
#endif
}
MC_HD void add_max(double *sum, double *mx, double v) {
#if defined(__CUDA_ARCH__)
    atomicAdd(sum, v);
    atomicMax(reinterpret_cast<unsigned long long *>(mx), (unsigned long long)__double_as_longlong(v));
#else
    *sum += v;
    if (v > *mx) *mx = v;
#endif
}

MC_HD void atomic_status(unsigned *s, unsigned bits) {
#if defined(__CUDA_ARCH__)
    atomicOr(s, bits);
#else
    *s |= bits;
#endif
}

// Per-species constants of the lattice collision that depend on the units (host, setup).
inline void set_lattice_constants(gas::Tables &t, const UnitsF &U) {
    for (int a = 0; a < t.ns; ++a) t.Ra_lat[a] = u_cp(U, (float)(gas::kR / t.m.W[a]));
}

MC_HD bool fluid_like(int t) { return t == T_F || t == T_I || t == T_O || t == T_I_C || t == T_O_C; }

MC_HD bool mc_wall_like(int t) {
    return t == T_S || t == T_A || t == T_FS || t == T_P || t == T_O || t == T_O_C;
}
// fd_central (src/headers/FD.hpp:108-127), dx = 1
MC_HD double mc_fd_central(double sl, double sc, double sr, int tl, int tr) {
    if (mc_wall_like(tl)) return (tr == T_P) ? 0.0 : (sr - sc);
    if (mc_wall_like(tr)) return (tl == T_P) ? 0.0 : (sc - sl);
    return (sr - sl) / 2.0;
}
// fd_fuw (src/FD.cpp:5-23), dx = 1
MC_HD bool fuw_blocked(int t) { return mc_wall_like(t) || t == T_I || t == T_I_C; }
MC_HD double mc_fd_fuw(double sl, double sc, double sr, double vel, int tl, int tr) {
    if (vel > 0) return fuw_blocked(tl) ? 0.0 : (sc - sl);
    return fuw_blocked(tr) ? 0.0 : (sr - sc);
}

// Periodic pull sources of a cell with no boundary neighbour (src/lbm-streaming.cpp:88-117):
// per axis the upstream coordinate for c = 0, +1, -1 with the reference's wrap (none through
// an x halo plane, which holds the neighbouring slab's cells).
struct McPull {
    long X[3], Y[3], Z[3];
};
template <class AT>
MC_HD void mc_pull(const AT &A, long n, McPull &p) {
    int i, j, k;
    cell_ijk(n, A.si, A.sj, i, j, k);
    const int im = (i - 1 == 0 && !A.halo_lo) ? A.Nx - 2 : i - 1;
    const int ip = (i + 1 == A.Nx - 1 && !A.halo_hi) ? 1 : i + 1;
    const int jm = (j - 1 == 0) ? A.Ny - 2 : j - 1, jp = (j + 1 == A.Ny - 1) ? 1 : j + 1;
    const int km = (k - 1 == 0) ? A.Nz - 2 : k - 1, kp = (k + 1 == A.Nz - 1) ? 1 : k + 1;
    p.X[0] = (long)i * A.si;
    p.X[1] = (long)im * A.si;
    p.X[2] = (long)ip * A.si;
    p.Y[0] = (long)j * A.sj;
    p.Y[1] = (long)jm * A.sj;
    p.Y[2] = (long)jp * A.sj;
    p.Z[0] = k;
    p.Z[1] = km;
    p.Z[2] = kp;
}
MC_HD long pull_idx(const McPull &p, int l) { return p.X[cidx(cx(l))] + p.Y[cidx(cy(l))] + p.Z[cidx(cz(l))]; }

// Cantera's setMassFractions: clip negatives, normalise.  Returns the mean molar mass.
template <int NS>
MC_HD double set_mass_fractions(const gas::Tables &t, const double *y, double *Y, double *X) {
    double s = 0.0;
    for (int k = 0; k < NS; ++k) {
        Y[k] = y[k] > 0.0 ? y[k] : 0.0;
        s += Y[k];
    }
    for (int k = 0; k < NS; ++k) Y[k] /= s;
    double sw = 0.0;
    for (int k = 0; k < NS; ++k) sw += Y[k] / t.m.W[k];
    const double W = 1.0 / sw;
    for (int k = 0; k < NS; ++k) X[k] = Y[k] / t.m.W[k] * W;
    return W;
}

// set_mass_fractions with products by reciprocals in place of its divisions (the FP32 storage
// mode's moment solve; rounding-level differences).
template <int NS>
MC_HD double set_mass_fractions_fast(const gas::Tables &t, const double *y, double *Y, double *X) {
    double s = 0.0;
    for (int k = 0; k < NS; ++k) {
        Y[k] = y[k] > 0.0 ? y[k] : 0.0;
        s += Y[k];
    }
    const double is = 1.0 / s;
    double sw = 0.0;
    for (int k = 0; k < NS; ++k) {
        Y[k] *= is;
        sw += Y[k] * t.invW[k];
    }
    const double W = 1.0 / sw;
    for (int k = 0; k < NS; ++k) X[k] = Y[k] * t.invW[k] * W;
    return W;
}

// The face-difference terms a cell offers its neighbours: species Q_{a,d} with the species
// gas constant (src/lbm-collision.cpp:487-489) and the mixture Q_d with the composition
// gas constant a neighbour uses (src/lbm-collision.cpp:207-215, 296-300; zero gas constant
// for cells that are not fluid-like).
template <int NS, class AT>
MC_HD void store_face_terms(const AT &A, typename AT::R *R, long n, int ty, double rho, const double u[3], double T,
                            const double *rho_a, const double (*ua)[3]) {
    const gas::Tables &t = *A.tab;
    double gc = 0.0;
    if (fluid_like(ty)) {
        double sYW = 0.0, sY = 0.0;
        for (int a = 0; a < NS; ++a) {
            const double Ya = rho_a[a] / rho;
            sYW += Ya / t.m.W[a];
            sY += Ya;
        }
        gc = (double)u_cp(A.U, (float)(gas::kR * sYW / sY));
    }
    for (int d = 0; d < 3; ++d)
        put(A, R, RM_QX + d, n, rho * u[d] * (1.0 - 3.0 * gc * T) - rho * (u[d] * u[d] * u[d]));
    for (int a = 0; a < NS; ++a) {
        const double Ra = t.Ra_lat[a];
        for (int d = 0; d < 3; ++d)
            put(A, R, rs(a, RS_QX + d), n,
                rho_a[a] * ua[a][d] * (1.0 - 3.0 * Ra * T) - rho_a[a] * (ua[a][d] * ua[a][d] * ua[a][d]));
    }
}

// Collision parameter planes (written by mc_props_cell, below).
template <int NS> MC_HD constexpr int pr_om(int a) { return a; }
template <int NS> MC_HD constexpr int pr_f(int a, int d) { return NS + 3 * a + d; }
template <int NS> MC_HD constexpr int pr_drho(int a) { return 4 * NS + a; }
template <int NS> MC_HD constexpr int pr_omm() { return 5 * NS; }
template <int NS> MC_HD constexpr int pr_om1() { return 5 * NS + 1; }
template <int NS> MC_HD constexpr int pr_theta() { return 5 * NS + 2; }
template <int NS> MC_HD constexpr int pr_uint() { return 5 * NS + 3; }
template <int NS> MC_HD constexpr int pr_dq(int d) { return 5 * NS + 4 + d; }
// the lattice binary diffusion coefficients D_ab (b < a) at the record's state: the
// collision uses them for the Maxwell-Stefan shift, and the moment solve that follows
// for its Stefan-Maxwell matrix -- both evaluate them at the same (T, p, composition)
template <int NS> MC_HD constexpr int pr_d(int a, int b) { return 5 * NS + 7 + a * (a - 1) / 2 + b; }
// the mixture gas constant R / W in lattice units (the energy-flux terms' Q_c)
template <int NS> MC_HD constexpr int pr_gc() { return 5 * NS + 7 + NS * (NS - 1) / 2; }
template <int NS> MC_HD constexpr int pr_count() { return pr_gc<NS>() + 1; }

// ------------------------------------------------------------------------------------
// Moments (the multicomponent LBM::calculate_moment, src/lbm-moment.cpp:193-377) of one
// fluid cell from its streamed populations, in two parts: the population sums (per
// species: rho_a, j_a and its share of the P tensor; the energy set's sum), then the
// per-cell solve from the sums (Stefan-Maxwell species velocities, temperature, record).
// The P tensor is summed species by species (each species' share over its 27 directions,
// then the shares in species order) on every path, so the interior split into a gather
// kernel and a solve kernel gives the same bits as the one-pass function.
// ------------------------------------------------------------------------------------
constexpr int kGsPerSpecies = 10;  // rho_a, j_a (3), P-tensor share (6)
template <int NS> MC_HD constexpr int gs_count() { return kGsPerSpecies * NS + 1; }

// The sums of one cell held in registers (the one-pass path); SumsAt reads the same
// values from the gathered planes where they are used.
template <int NS>
struct McSums {
    double ra[NS], ja[NS][3], p6[6], re;
    MC_HD double rho_a(int a) const { return ra[a]; }
    MC_HD double j(int a, int d) const { return ja[a][d]; }
    MC_HD double P6(int q) const { return p6[q]; }
    MC_HD double rhoe() const { return re; }
};

// The sums of one species' streamed populations fv[27]: s = (rho_a, j_a (3), P share (6)).
MC_HD void species_sums(const double *fv, double *s) {
    double r = 0, jx = 0, jy = 0, jz = 0, p[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        r += fv[l];
        jx += fv[l] * cx(l);
        jy += fv[l] * cy(l);
        jz += fv[l] * cz(l);
        if (cx(l)) p[0] += fv[l];
        if (cx(l) * cy(l)) p[1] += cx(l) * cy(l) * fv[l];
        if (cx(l) * cz(l)) p[2] += cx(l) * cz(l) * fv[l];
        if (cy(l)) p[3] += fv[l];
        if (cy(l) * cz(l)) p[4] += cy(l) * cz(l) * fv[l];
        if (cz(l)) p[5] += fv[l];
    }
    s[0] = r;
    s[1] = jx;
    s[2] = jy;
    s[3] = jz;
    for (int q = 0; q < 6; ++q) s[4 + q] = p[q];
}

// The gathered sum planes of cell n (k_mc_gather): species a at planes 10a..10a+9, the
// energy sum at 10 NS; the P tensor adds the species' shares in species order.
template <int NS>
struct SumsAt {
    const double *gs;
    long ncell, n;
    MC_HD double at(int plane) const { return gs[(long)plane * ncell + n]; }
    MC_HD double rho_a(int a) const { return at(kGsPerSpecies * a); }
    MC_HD double j(int a, int d) const { return at(kGsPerSpecies * a + 1 + d); }
    MC_HD double P6(int q) const {
        double v = 0.0;
        for (int a = 0; a < NS; ++a) v += at(kGsPerSpecies * a + 4 + q);
        return v;
    }
    MC_HD double rhoe() const { return at(kGsPerSpecies * NS); }
};

template <int NS, class AT, class Sums>
MC_HDN void mc_moments_finish(const AT &A, long n, const Sums &S);

// The Stefan-Maxwell system A u_a = j_a (lbm-moment.cpp:302-341): every entry of row a is
// -dt/2 p X_a X_b / D_ab in that order, so the lower triangle (b < a, holding D_ab on entry)
// is the matrix's own entry and the diagonal takes row a's entries, b = 0..NS-1, as the
// reference subtracts them; rows go in order, row a reading the D_ab of the rows below it
// (still untouched) and its own slots before replacing them; then a dense in-place lower
// Cholesky factor and the two triangular solves per axis, in arithmetic C (double: the
// reference's, every division a division -- the boundary cells' upwind differences switch
// on the sign of near-zero diffusion velocities, so a reciprocal in place of a quotient
// moves results by 1e-9 within two steps).
template <int NS, typename C>
MC_HD void mc_stefan_maxwell(int dt, double p_old, const double *Xold, const double *rho_s, const double (*j_a)[3],
                             double (*Ld)[NS], double (*usm)[3]) {
    C L[NS][NS];
    for (int a = 0; a < NS; ++a)
        for (int b = 0; b < a; ++b) L[a][b] = (C)Ld[a][b];
    for (int a = 0; a < NS; ++a) {
        C d = (C)(rho_s[a] == 0.0 ? 1.0 : rho_s[a]);
        for (int b = 0; b < NS; ++b) {
            if (b == a) continue;
            const C D = b < a ? L[a][b] : L[b][a];
            const C m = (C)-1.0 * (C)dt / (C)2.0 * (C)p_old * (C)Xold[a] * (C)Xold[b] / D;
            if (b < a) L[a][b] = m;
            d -= m;
        }
        L[a][a] = d;
    }
    for (int c = 0; c < NS; ++c) {  // in-place lower Cholesky factor
        C d = L[c][c];
        for (int q = 0; q < c; ++q) d -= L[c][q] * L[c][q];
        L[c][c] = sqrt(d);
        for (int r = c + 1; r < NS; ++r) {
            C s = L[r][c];
            for (int q = 0; q < c; ++q) s -= L[r][q] * L[c][q];
            L[r][c] = s / L[c][c];
        }
    }
    for (int dmn = 0; dmn < 3; ++dmn) {
        C y[NS], x[NS];
        for (int r = 0; r < NS; ++r) {
            C s = (C)j_a[r][dmn];
            for (int q = 0; q < r; ++q) s -= L[r][q] * y[q];
            y[r] = s / L[r][r];
        }
        for (int r = NS - 1; r >= 0; --r) {
            C s = y[r];
            for (int q = r + 1; q < NS; ++q) s -= L[q][r] * x[q];
            x[r] = s / L[r][r];
        }
        for (int r = 0; r < NS; ++r) usm[r][dmn] = (double)x[r];
    }
}

// The same system for the FP32 storage mode, where the result need not reproduce the
// reference's roundings: the matrix is symmetric (each pair's entry -dt/2 p X_a X_b / D_ab
// formed once, one division), and the Cholesky factor's pivots are inverted once, so the
// factorisation and the solves multiply instead of dividing -- 36 divisions and 9 square roots
// in place of 171 divisions and 9 square roots.  Every loop is unrolled, so the factor and the
// vectors are indexed by constants and stay out of local memory (1.92 -> 1.57 ms at 128^3,
// with the temperature iteration's species loop unrolled as well).
template <int NS>
MC_HD void mc_stefan_maxwell_fast(int dt, double p_old, const double *Xold, const double *rho_s,
                                  const double (*j_a)[3], double (*Ld)[NS], double (*usm)[3]) {
    double L[NS][NS];
    const double k = -0.5 * (double)dt * p_old;
#pragma unroll
    for (int a = 0; a < NS; ++a) L[a][a] = rho_s[a] == 0.0 ? 1.0 : rho_s[a];
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int b = 0; b < a; ++b) {
            const double m = k * Xold[a] * Xold[b] / Ld[a][b];
            L[a][b] = m;
            L[a][a] -= m;
            L[b][b] -= m;
        }
    double inv[NS];
#pragma unroll
    for (int c = 0; c < NS; ++c) {  // in-place lower Cholesky factor, reciprocal pivots
        double d = L[c][c];
#pragma unroll
        for (int q = 0; q < c; ++q) d -= L[c][q] * L[c][q];
        inv[c] = 1.0 / sqrt(d);
#pragma unroll
        for (int r = c + 1; r < NS; ++r) {
            double sum = L[r][c];
#pragma unroll
            for (int q = 0; q < c; ++q) sum -= L[r][q] * L[c][q];
            L[r][c] = sum * inv[c];
        }
    }
#pragma unroll
    for (int dmn = 0; dmn < 3; ++dmn) {
        double y[NS], x[NS];
#pragma unroll
        for (int r = 0; r < NS; ++r) {
            double sum = j_a[r][dmn];
#pragma unroll
            for (int q = 0; q < r; ++q) sum -= L[r][q] * y[q];
            y[r] = sum * inv[r];
        }
#pragma unroll
        for (int r = NS - 1; r >= 0; --r) {
            double sum = y[r];
#pragma unroll
            for (int q = r + 1; q < NS; ++q) sum -= L[q][r] * x[q];
            x[r] = sum * inv[r];
        }
#pragma unroll
        for (int r = 0; r < NS; ++r) usm[r][dmn] = x[r];
    }
}

template <int NS, class AT, class Pop>
MC_HDN void mc_moments_cell(const AT &A, long n, const Pop &pop) {
    McSums<NS> S;
    for (int q = 0; q < 6; ++q) S.p6[q] = 0.0;
    for (int a = 0; a < NS; ++a) {
        double fv[27], s[kGsPerSpecies];
#pragma unroll
        for (int l = 0; l < 27; ++l) fv[l] = pop(a, l);
        species_sums(fv, s);
        S.ra[a] = s[0];
        for (int d = 0; d < 3; ++d) S.ja[a][d] = s[1 + d];
        for (int q = 0; q < 6; ++q) S.p6[q] += s[4 + q];
    }
    double rhoe = 0.0;
#pragma unroll
    for (int l = 0; l < 27; ++l) rhoe += pop(NS, l);
    S.re = rhoe;
    mc_moments_finish<NS>(A, n, S);
}

template <int NS, class AT, class Sums>
MC_HDN void mc_moments_finish(const AT &A, long n, const Sums &S) {
    const gas::Tables &t = *A.tab;
    // -- old temperature, where the reference's Newton iteration starts (lbm-moment.cpp:219-221);
    // the old state's diffusion coefficients come from the collision parameters
    const double T_si = si_temp(A.U, (float)rec(A, A.rec_cur, RM_T, n));

    // the diffusion coefficients first (one load per pair, into the lower triangle that
    // the Stefan-Maxwell entries then replace row by row), the momenta next
    double L[NS][NS];  // lower triangle and diagonal only
    for (int a = 0; a < NS; ++a)
        for (int b = 0; b < a; ++b) L[a][b] = A.props[(long)pr_d<NS>(a, b) * A.ncell + n];
    double j_a[NS][3];
    double rho = 0, ru = 0, rv = 0, rw = 0, rho_s[NS];
    for (int a = 0; a < NS; ++a) {
        const double ra = S.rho_a(a);
        for (int d = 0; d < 3; ++d) j_a[a][d] = S.j(a, d);
        rho_s[a] = ra > kSpeciesMin ? ra : kSpeciesMin;
        rho += ra;
        ru += j_a[a][0];
        rv += j_a[a][1];
        rw += j_a[a][2];
    }
    const double u = ru / rho, v = rv / rho, w = rw / rho;

    // -- Stefan-Maxwell species velocities (mc_stefan_maxwell) with the D_ab the collision of
    // this step evaluated at the same old state (T, p, Y)
    const double p_old = rec(A, A.rec_cur, RM_P, n);
    double Xold[NS];
    for (int a = 0; a < NS; ++a) Xold[a] = rec(A, A.rec_cur, rs(a, RS_X), n);
    // FP64 in both storage modes (an FP32 solve moved the characteristic-inflow case's
    // temperature by 2e-5 against FP64 within 20 steps -- its boundary cells amplify last-bit
    // changes -- twice the FP32 mode's bound); the FP32 storage mode takes the reciprocal
    // forms of the solve, the mass fractions and the temperature iteration, which differ
    // from the reference's divisions by rounding
    constexpr bool fast = sizeof(typename AT::P) == sizeof(float);
    double usm[NS][3];
    if constexpr (fast)
        mc_stefan_maxwell_fast<NS>(A.dt, p_old, Xold, rho_s, j_a, L, usm);
    else
        mc_stefan_maxwell<NS, double>(A.dt, p_old, Xold, rho_s, j_a, L, usm);

    // -- temperature from the internal energy (setState_UV, lbm-moment.cpp:346-368)
    double Yr[NS], Y[NS], X[NS];
    double Wn;
    if constexpr (fast) {
        const double ir = 1.0 / rho;
        for (int a = 0; a < NS; ++a) Yr[a] = rho_s[a] * ir;
        Wn = set_mass_fractions_fast<NS>(t, Yr, Y, X);
    } else {
        for (int a = 0; a < NS; ++a) Yr[a] = rho_s[a] / rho;
        Wn = set_mass_fractions<NS>(t, Yr, Y, X);
    }
    const double rhoe = S.rhoe();
    double e = rhoe / rho;
    for (int a = 0; a < NS; ++a)
        e = e - 0.5 * rho_s[a] / rho * (usm[a][0] * usm[a][0] + usm[a][1] * usm[a][1] + usm[a][2] * usm[a][2]);
    const double u_si = si_energy_mass(A.U, (float)e);
    const double vol = 1.0 / (double)si_rho(A.U, (float)rho);
    const double rho_n_si = 1.0 / vol;
    double Tn;
    const int it = fast ? gas::T_from_u_fast<NS>(t, Y, u_si, T_si, 1e-14, 100, Tn)
                        : gas::T_from_u(t, Y, u_si, T_si, 1e-14, 100, Tn);
    if (it < 0) atomic_status(A.status, LBMGPU_ST_NEWTON);
    const double Pn = rho_n_si * gas::kR * Tn / Wn;
    const double Tl = u_temp(A.U, (float)Tn);

    typename AT::R *R = A.rec_nxt;
    put(A, R, RM_RHO, n, rho);
    put(A, R, RM_U, n, u);
    put(A, R, RM_V, n, v);
    put(A, R, RM_W, n, w);
    put(A, R, RM_T, n, Tl);
    put(A, R, RM_P, n, u_p(A.U, (float)Pn));
    put(A, R, RM_RHOE, n, rhoe);
    for (int q = 0; q < 6; ++q) put(A, R, RM_P00 + q, n, S.P6(q));
    for (int a = 0; a < NS; ++a) {
        put(A, R, rs(a, RS_RHO), n, rho_s[a]);
        for (int d = 0; d < 3; ++d) put(A, R, rs(a, RS_UX + d), n, usm[a][d]);
        put(A, R, rs(a, RS_X), n, X[a]);
    }
    const double um[3] = {u, v, w};
    store_face_terms<NS>(A, R, n, T_F, rho, um, Tl, rho_s, usm);
    if (!isfinite(rho) || !isfinite(Tn) || !isfinite(u) || !isfinite(v) || !isfinite(w))
        atomic_status(A.status, LBMGPU_ST_NAN);
    else if (!(rho > 0.0) || !(Tn > 0.0))
        atomic_status(A.status, LBMGPU_ST_NEG_STATE);
}

// Streaming + moments of a fluid cell of the periodic interior (no boundary upstream):
// every population pulled from its upstream neighbour.
template <int NS, class AT>
MC_HDN void mc_stream_moment_cell(const AT &A, long n) {
    McPull pp;
    mc_pull(A, n, pp);
    mc_moments_cell<NS>(A, n, [&](int a, int l) { return ldpop(A, A.pop_src, 27 * a + l, pull_idx(pp, l)); });
}

// ------------------------------------------------------------------------------------
// Collision: species (LBM::Collide_Species, src/lbm-collision.cpp:334-526) and energy
// (LBM::Collide, src/lbm-collision.cpp:191-332), in two parts:
//   mc_props_cell    per cell: chemistry, transport, relaxation rates, the Maxwell-Stefan
//                    velocity shift and the energy-flux correction -> the props planes;
//   mc_relax_species per (cell, species) and mc_relax_energy per cell: the BGK update of
//                    the 27 populations of one set from the props planes.
// Props planes (FP64, per cell): om_a (NS), F_a,d (3 NS), drho_a (NS), omega, omega_1,
// theta, U, dq_d (3, written by mc_eflux_cell), D_ab (NS (NS-1) / 2), R / W.
// ------------------------------------------------------------------------------------

// The chemistry of LBMGPU_CHEM_ROSENBROCK for one cell: the constant-(rho, e) reactor
// over the whole lattice step with ROS2 (chem.cuh); the density change and the heat
// release enter the collision the same way as the reference's explicit increments.
//
// With the surrogate on (sur.mode 1) the network's dY, dT replace the integrator, made
// exactly element-conserving (sur_conserve); cells outside the training box, non-finite
// predictions and the audited cells need the integrator (the audited ones also score the
// prediction against it).  With `defer` and a list (sur.ilist) such cells are only
// appended to the list -- k_mc_chem_list integrates them afterwards in dense warps --
// otherwise they are integrated here.  Teacher steps (mode 0) can write samples.
//
// G > 1 (device, the integrator list): a group of G lanes handles the cell together --
// every lane runs this function with the same arguments, the integration is
// ros2_advance_group, and only the group's first lane writes the results.
// KIN (device): the kinetics policy of a mechanism compiled to straight-line code
// (gen_kinetics.py) when the handle's mechanism is that one, void for the tables.
// SMAT (device, G = 1, KIN): the integrator's iteration matrix in the dynamic shared memory
// the kernel was launched with, (NS + 1)^2 doubles per thread of the block.
// PRED (false: a launch made while the surrogate's predictions are not in use): the
// prediction, its gate and its audit compiled out, so nothing of them stays live across the
// integration.
template <int NS, class AT, bool CAN_INTEGRATE = true, int G = 1, class KIN = void, bool SMAT = false,
          bool PRED = true>
MC_HDN void mc_chem_ros2(const AT &A, long n, double rho, const double *rho_a, const double *Y, double T_si,
                         double rho_si, double P_si, bool defer) {
    const gas::Tables &t = *A.tab;
#if defined(__CUDA_ARCH__)
    const bool lead = G == 1 || (threadIdx.x & (G - 1)) == 0;
#else
    const bool lead = true;
#endif
    const SurArgs &S = A.sur;
    const double dt_si = (double)A.dt * (double)A.U.s;
    double Yc[gas::MAXS], Tc = T_si, Yp[NS], Tp = T_si;
    bool have_pred = false;
    if (PRED && S.mode == 1 && !S.gate[n]) {
        // the prediction is used if it is finite, every output lies within kSurOutGate
        // standard deviations of the training targets, and after the element projection no
        // mass fraction goes below -kSurNegTol; otherwise the integrator takes the cell
        // the row's NS + 1 outputs in whole 16-byte words (rows are kSurOutPad floats, 64 B)
        constexpr int kWords = (NS + 4) / 4;
        float pr[4 * kWords];
#if defined(__CUDA_ARCH__)
        const float4 *pw = reinterpret_cast<const float4 *>(S.pred + n * kSurOutPad);
#pragma unroll
        for (int q = 0; q < kWords; ++q) {
            const float4 v = pw[q];
            pr[4 * q] = v.x;
            pr[4 * q + 1] = v.y;
            pr[4 * q + 2] = v.z;
            pr[4 * q + 3] = v.w;
        }
#else
        for (int q = 0; q < 4 * kWords; ++q) pr[q] = S.pred[n * kSurOutPad + q];
#endif
        const SurNorm &nm = *S.nrm;
        double dY[NS];
        // |pred - mean| <= kSurOutGate std (the standard deviations are positive)
        have_pred = isfinite(pr[NS]) && fabsf(pr[NS] - nm.y_mean[NS]) <= kSurOutGate * nm.y_std[NS];
#pragma unroll
        for (int a = 0; a < NS; ++a) {
            dY[a] = (double)pr[a];
            have_pred = have_pred && isfinite(dY[a]) && fabsf(pr[a] - nm.y_mean[a]) <= kSurOutGate * nm.y_std[a];
        }
        if (have_pred) {
            sur_conserve<NS>(S.proj, dY);
            for (int a = 0; a < NS; ++a) have_pred = have_pred && Y[a] + dY[a] >= -kSurNegTol;
        }
        for (int a = 0; a < NS; ++a) Yp[a] = Y[a] + dY[a];
        Tp = T_si + (double)pr[NS];
    }
    const bool audit = have_pred && S.audit_period > 0 && (unsigned)(n % S.audit_period) == S.audit_phase;
    if (PRED && S.mode == 1 && (defer || !S.ilist)) {
        count_flag(&S.audit[3], audit);
        count_flag(&S.audit[4], have_pred && !audit);
        count_flag(&S.audit[5], !have_pred);
    }
    if (!have_pred || audit) {
        if (!CAN_INTEGRATE || (defer && S.ilist)) {
#if defined(__CUDA_ARCH__)
            S.ilist[atomicAdd(S.icount, 1u)] = (int)n;
#else
            S.ilist[(*S.icount)++] = (int)n;
#endif
            return;
        }
        if (CAN_INTEGRATE) {
            for (int a = 0; a < NS; ++a) Yc[a] = Y[a];
            int rc;
#if defined(__CUDA_ARCH__)
            if constexpr (G > 1 && !std::is_void_v<KIN>)
                rc = gas::ros2_advance_group<NS, G>(KIN{}, rho_si, Yc, Tc, dt_si);
            else if constexpr (G > 1)
                rc = gas::ros2_advance_group<NS, G>(gas::CachedTableKinetics{t}, rho_si, Yc, Tc, dt_si);
            else if constexpr (!std::is_void_v<KIN> && SMAT) {
                extern __shared__ double mc_chem_smem[];
                gas::SharedMat<gas::SysMap<KIN, NS + 1>::size> Ms{mc_chem_smem + threadIdx.x, (int)blockDim.x};
                rc = gas::ros2_advance_km<NS>(KIN{}, Ms, rho_si, Yc, Tc, dt_si);
            } else if constexpr (!std::is_void_v<KIN>)
                rc = gas::ros2_advance_k<NS>(KIN{}, rho_si, Yc, Tc, dt_si);
            else
                rc = gas::ros2_advance_n<NS>(t, rho_si, Yc, Tc, dt_si);
#else
            rc = gas::ros2_advance(t, rho_si, Yc, Tc, dt_si);
#endif
            if (rc < 0 && lead) atomic_status(A.status, LBMGPU_ST_CHEM);
        }
    } else {
        for (int a = 0; a < NS; ++a) Yc[a] = Yp[a];
        Tc = Tp;
    }
    if (!lead) return;
    if (audit) {  // L1 error of the predicted dY and L1 size of the integrator's dY
        double num = 0.0, den = 0.0;
        for (int a = 0; a < NS; ++a) {
            num += fabs(Yp[a] - Yc[a]);
            den += fabs(Yc[a] - Y[a]);
        }
        add_max(&S.audit[0], &S.audit[2], num);
#if defined(__CUDA_ARCH__)
        atomicAdd(&S.audit[1], den);
#else
        S.audit[1] += den;
#endif
    }
    if (S.ds_x && (!have_pred || audit) && (long)(n % S.ds_stride) == S.ds_phase) {
        const long row = S.ds_base + n / S.ds_stride;
        if (row < S.ds_cap) {
            sur_features<NS>(T_si, P_si, Y, dt_si, S.ds_x + row * kSurIn);
            for (int a = 0; a < NS; ++a) S.ds_y[row * kSurOut + a] = (float)(Yc[a] - Y[a]);
            S.ds_y[row * kSurOut + NS] = (float)(Tc - T_si);
            S.ds_valid[row] = 1;
        }
    }
    // the heat release -sum_k h_k dρ_k from the reciprocal forms (h_RT_fast, 1/W_k): this
    // stiff-chemistry mode has no reference rounding to reproduce
    double hrr = 0.0;
    const double invTc = 1.0 / Tc;
    for (int a = 0; a < NS; ++a) {
        const double dr = rho * (Yc[a] - Y[a]);
        hrr += -1.0 * (double)u_energy_mass(A.U, (float)(gas::h_RT_fast(t, a, Tc, invTc) * gas::kR * Tc * t.invW[a])) * dr;
        A.props[(long)pr_drho<NS>(a) * A.ncell + n] = dr;
    }
    put(A, A.rec_nxt, RM_HRR, n, hrr);
}

// The chemistry state of a cell from the record, as the collision forms it (Cantera's
// setMassFractions + setState_TD, lbm-collision.cpp:364-367), in the reciprocal forms
// (set_mass_fractions_fast): the stiff-chemistry mode has no reference rounding to reproduce.
template <int NS, class AT>
MC_HD void mc_chem_state(const AT &A, long n, double &rho, double *rho_a, double *Y, double &T_si, double &rho_si,
                         double &P_si) {
    const gas::Tables &t = *A.tab;
    rho = rec(A, A.rec_cur, RM_RHO, n);
    double Yr[NS], X[NS];
    const double ir = 1.0 / rho;
    for (int a = 0; a < NS; ++a) {
        rho_a[a] = rec(A, A.rec_cur, rs(a, RS_RHO), n);
        Yr[a] = rho_a[a] * ir;
    }
    const double W = set_mass_fractions_fast<NS>(t, Yr, Y, X);
    T_si = si_temp(A.U, (float)rec(A, A.rec_cur, RM_T, n));
    rho_si = si_rho(A.U, (float)rho);
    P_si = rho_si * gas::kR * T_si / W;
}

// The transport part of the collision parameters (lbm-collision.cpp:402-471 species rates and
// Maxwell-Stefan force, :231-316 energy rates) in FP64, the reference's arithmetic and order
// (the FP64 storage mode, bit-faithful).
template <int NS, class AT>
MC_HDN void mc_transport_f64(const AT &A, long n, double p, const double *rho_a, const double (*ua)[3],
                             const double *Xs, const double *Y, const double *X, double W, double T_si, double P_si,
                             double Uint) {
    const gas::Tables &t = *A.tab;
    double *Pr = A.props;
    auto prp = [&](int plane, double v) { Pr[(long)plane * A.ncell + n] = v; };
    const double dt = A.dt;
    // -- species viscosities; Wilke weights phi_ab = (1 + sqrt(mu_a/mu_b) (W_b/W_a)^1/4)^2 /
    // sqrt(8 (1 + W_a/W_b)) formed for b >= a and mirrored, phi_ba = mu_b/mu_a W_a/W_b phi_ab
    // (lbm-collision.cpp:402-430).  Each weight enters the two row sums the reference forms
    // with it -- sum_b Xs_b phi_ab for the species rates, sum_b X_b phi_ab for the mixture
    // viscosity -- pair by pair; every row still receives its terms in the order b = 0..NS-1.
    const double xT = gas::lnT_x(T_si);
    double mu_k[NS];
    for (int a = 0; a < NS; ++a) mu_k[a] = gas::species_visc_x(t, a, xT);
    double den_s[NS], den_m[NS];
    for (int a = 0; a < NS; ++a) den_s[a] = den_m[a] = 0.0;
    for (int a = 0; a < NS; ++a)
        for (int b = a; b < NS; ++b) {
            const double f1 = 1.0 + sqrt(mu_k[a] / mu_k[b]) * t.sqrt4W[a][b];
            const double pab = f1 * f1 / t.wilke_den[a][b];
            const double pba = mu_k[b] / mu_k[a] * t.m.W[a] / t.m.W[b] * pab;
            if (b == a) {
                den_s[a] = den_s[a] + Xs[a] * pba;
                den_m[a] += X[a] * pba;
            } else {
                den_s[a] = den_s[a] + Xs[b] * pab;
                den_m[a] += X[b] * pab;
                den_s[b] = den_s[b] + Xs[a] * pba;
                den_m[b] += X[a] * pba;
            }
        }
    for (int a = 0; a < NS; ++a) {
        const double visc = Xs[a] * (double)u_mu(A.U, (float)mu_k[a]) / den_s[a];
        prp(pr_om<NS>(a), 2 * Xs[a] * p * dt / (Xs[a] * p * dt + 2 * visc));
    }

    // -- Maxwell-Stefan force (lbm-collision.cpp:433-471); the diagonal term vanishes
    double F[NS][3];
    for (int a = 0; a < NS; ++a)
        for (int d = 0; d < 3; ++d) F[a][d] = 0.0;
    for (int a = 0; a < NS; ++a)
        for (int b = 0; b < a; ++b) {
            const double D = u_nu(A.U, (float)gas::binary_diff_x(t, a, b, xT, P_si));
            prp(pr_d<NS>(a, b), D);
            // the reference's -p X_a X_b / D_ab, once per ordered pair
            const double kab = -1.0 * p * Xs[a] * Xs[b] / D, kba = -1.0 * p * Xs[b] * Xs[a] / D;
            for (int d = 0; d < 3; ++d) {
                F[a][d] += kab * (ua[a][d] - ua[b][d]);
                F[b][d] += kba * (ua[b][d] - ua[a][d]);
            }
        }
    for (int a = 0; a < NS; ++a)
        for (int d = 0; d < 3; ++d) prp(pr_f<NS>(a, d), F[a][d] * dt / rho_a[a]);

    // -- energy collision parameters (lbm-collision.cpp:231-316): the relaxation rates here,
    // the energy-flux terms (neighbour differences) in mc_eflux_cell
    double mu = 0.0;  // Wilke mixture viscosity sum_k X_k mu_k / sum_j X_j phi_kj
    for (int k = 0; k < NS; ++k) mu += X[k] * mu_k[k] / den_m[k];
    const double cp = u_cp(A.U, (float)gas::cp_mass(t, Y, T_si));
    const double gasconstant = u_cp(A.U, (float)(gas::kR / W));
    mu = u_mu(A.U, (float)mu);
    const double lam = u_cond(A.U, (float)gas::mix_cond(t, X, T_si, P_si, mu_k));
    const double theta = u_energy_mass(A.U, (float)(gas::kR * T_si / W));
    const double om1 = 2 * p * cp * dt / (p * cp * dt + 2 * lam);
    const double om = 2 * p * dt / (p * dt + 2 * mu);
    if (!(1.0 / om > 0.5) || !(1.0 / om1 > 0.5)) atomic_status(A.status, LBMGPU_ST_TAU_UNSTABLE);
    prp(pr_omm<NS>(), om);
    prp(pr_om1<NS>(), om1);
    prp(pr_theta<NS>(), theta);
    prp(pr_uint<NS>(), Uint);
    prp(pr_gc<NS>(), gasconstant);
}

// The same parameters for the FP32 storage mode, in FP32 arithmetic: species viscosities,
// conductivities and binary diffusion coefficients (exp of the ln T fits), the Wilke
// weights, c_p and the mixture conductivity -- quantities the reference itself rounds to
// float at its unit conversions (units.hpp:10) -- with the Maxwell-Stefan force accumulated
// in FP64 (its terms are differences of nearly equal species velocities).  The Wilke pairs
// take products of per-species square roots and reciprocals in place of the quotients.
template <int NS, class AT>
MC_HDN void mc_transport_f32(const AT &A, long n, double p, const double *rho_a, const double (*ua)[3],
                             const double *Xs, const double *Y, const double *X, double W, double T_si, double P_si,
                             double Uint) {
    const gas::Tables &t = *A.tab;
    double *Pr = A.props;
    auto prp = [&](int plane, double v) { Pr[(long)plane * A.ncell + n] = v; };
    const float dt = (float)A.dt, pf = (float)p;
    const float xT = (float)gas::lnT_x(T_si);
    // per species: mu_k, sqrt(mu_k) and their reciprocals, so that the Wilke pairs multiply;
    // every loop unrolled, so that these arrays live in registers
    float mu_k[NS], imu[NS], smu[NS], ismu[NS], Xsf[NS], Xf[NS];
#pragma unroll
    for (int a = 0; a < NS; ++a) {
        mu_k[a] = expf(gas::fit_eval_f(t.fit_visc[a], xT));
        imu[a] = 1.f / mu_k[a];
        smu[a] = sqrtf(mu_k[a]);
        ismu[a] = 1.f / smu[a];
        Xsf[a] = (float)Xs[a];
        Xf[a] = (float)X[a];
    }
    float den_s[NS], den_m[NS];
#pragma unroll
    for (int a = 0; a < NS; ++a) den_s[a] = den_m[a] = 0.f;
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int b = a; b < NS; ++b) {
            const float f1 = 1.f + smu[a] * ismu[b] * (float)t.sqrt4W[a][b];
            const float pab = f1 * f1 * t.inv_wilke_den_f[a][b];
            const float pba = mu_k[b] * imu[a] * t.W_ratio_f[a][b] * pab;
            if (b == a) {
                den_s[a] += Xsf[a] * pba;
                den_m[a] += Xf[a] * pba;
            } else {
                den_s[a] += Xsf[b] * pab;
                den_m[a] += Xf[b] * pab;
                den_s[b] += Xsf[a] * pba;
                den_m[b] += Xf[a] * pba;
            }
        }
#pragma unroll
    for (int a = 0; a < NS; ++a) {
        const float visc = Xsf[a] * u_mu(A.U, mu_k[a]) / den_s[a];
        prp(pr_om<NS>(a), (double)(2.f * Xsf[a] * pf * dt / (Xsf[a] * pf * dt + 2.f * visc)));
    }
    double F[NS][3];
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) F[a][d] = 0.0;
    const float inv_P = 1.f / (float)P_si;
#pragma unroll
    for (int a = 0; a < NS; ++a)
#pragma unroll
        for (int b = 0; b < a; ++b) {
            const float D = u_nu(A.U, expf(gas::fit_eval_f(t.fit_diff[a][b], xT)) * inv_P);
            prp(pr_d<NS>(a, b), (double)D);
            const double k = (double)(-pf * Xsf[a] * Xsf[b] / D);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double du = ua[a][d] - ua[b][d];
                F[a][d] += k * du;
                F[b][d] -= k * du;
            }
        }
#pragma unroll
    for (int a = 0; a < NS; ++a) {
        const double s = (double)dt / rho_a[a];
#pragma unroll
        for (int d = 0; d < 3; ++d) prp(pr_f<NS>(a, d), F[a][d] * s);
    }
    float mu = 0.f, cpm = 0.f, s1 = 0.f, s2 = 0.f;
    const float Tf = (float)T_si;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        mu += Xf[k] * mu_k[k] / den_m[k];
        const double *c = T_si < t.m.T_mid[k] ? t.m.nasa_lo[k] : t.m.nasa_hi[k];
        cpm += (float)Y[k] * ((float)c[0] + Tf * ((float)c[1] + Tf * ((float)c[2] + Tf * ((float)c[3] + Tf * (float)c[4])))) *
               (float)t.invW[k];
        const float lk = expf(gas::fit_eval_f(t.fit_cond[k], xT));
        s1 += Xf[k] * lk;
        s2 += Xf[k] / lk;
    }
    const float cp = u_cp(A.U, cpm * (float)gas::kR);
    const float gasconstant = u_cp(A.U, (float)(gas::kR / W));
    const float muf = u_mu(A.U, mu);
    const float lam = u_cond(A.U, 0.5f * (s1 + 1.f / s2));
    const double theta = u_energy_mass(A.U, (float)(gas::kR * T_si / W));
    const double om1 = (double)(2.f * pf * cp * dt / (pf * cp * dt + 2.f * lam));
    const double om = (double)(2.f * pf * dt / (pf * dt + 2.f * muf));
    if (!(1.0 / om > 0.5) || !(1.0 / om1 > 0.5)) atomic_status(A.status, LBMGPU_ST_TAU_UNSTABLE);
    prp(pr_omm<NS>(), om);
    prp(pr_om1<NS>(), om1);
    prp(pr_theta<NS>(), theta);
    prp(pr_uint<NS>(), Uint);
    prp(pr_gc<NS>(), (double)gasconstant);
}

template <int NS, int CHEM, class AT>
MC_HDN void mc_props_cell(const AT &A, long n) {
    const gas::Tables &t = *A.tab;
    const typename AT::R *Rc = A.rec_cur;
    double *Pr = A.props;
    auto prp = [&](int plane, double v) { Pr[(long)plane * A.ncell + n] = v; };
    const double rho = rec(A, Rc, RM_RHO, n);
    const double um[3] = {rec(A, Rc, RM_U, n), rec(A, Rc, RM_V, n), rec(A, Rc, RM_W, n)};
    const double Tl = rec(A, Rc, RM_T, n), p = rec(A, Rc, RM_P, n), rhoe = rec(A, Rc, RM_RHOE, n);
    double rho_a[NS], ua[NS][3], Xs[NS];
    for (int a = 0; a < NS; ++a) {
        rho_a[a] = rec(A, Rc, rs(a, RS_RHO), n);
        for (int d = 0; d < 3; ++d) ua[a][d] = rec(A, Rc, rs(a, RS_UX + d), n);
        Xs[a] = rec(A, Rc, rs(a, RS_X), n);
    }
    // Cantera state (lbm-collision.cpp:364-367 and :236-238); the FP32 storage mode takes the
    // reciprocal forms (rounding-level differences, as in its moment solve)
    constexpr bool fast = sizeof(typename AT::P) == sizeof(float);
    double Yr[NS], Y[NS], X[NS];
    double W;
    if constexpr (fast) {
        const double ir = 1.0 / rho;
        for (int a = 0; a < NS; ++a) Yr[a] = rho_a[a] * ir;
        W = set_mass_fractions_fast<NS>(t, Yr, Y, X);
    } else {
        for (int a = 0; a < NS; ++a) Yr[a] = rho_a[a] / rho;
        W = set_mass_fractions<NS>(t, Yr, Y, X);
    }
    const double T_si = si_temp(A.U, (float)Tl);
    const double rho_si = si_rho(A.U, (float)rho);
    const double P_si = rho_si * gas::kR * T_si / W;
    const double dt = A.dt;

    // internal energy without the species kinetic energy (lbm-collision.cpp:260-263, 373-376)
    double Uint = rhoe / rho;
    for (int a = 0; a < NS; ++a)
        Uint = Uint - 0.5 * rho_a[a] / rho * (ua[a][0] * ua[a][0] + ua[a][1] * ua[a][1] + ua[a][2] * ua[a][2]);

    // -- chemistry: two explicit half steps with T from (u, v) in between (lbm-collision.cpp:370-399)
    if (CHEM == CHEM_REF_EXPLICIT) {
        double drho[NS];
        for (int a = 0; a < NS; ++a) drho[a] = 0.0;
        double Tc = T_si, rc = rho_si, Yc[NS], Xc[NS];
        for (int a = 0; a < NS; ++a) Yc[a] = Y[a];
        for (int sub = 0; sub < 2; ++sub) {
            double C[gas::MAXS], wd[gas::MAXS];
            for (int a = 0; a < NS; ++a) C[a] = rc * Yc[a] / t.m.W[a];
            gas::net_production(t, Tc, C, wd);
            for (int a = 0; a < NS; ++a) drho[a] += dt / 2.0 * (double)u_rho_dot(A.U, (float)(wd[a] * t.m.W[a]));
            double yy[NS];
            for (int a = 0; a < NS; ++a) yy[a] = (rho_a[a] + drho[a]) / rho;
            set_mass_fractions<NS>(t, yy, Yc, Xc);
            const double vol = 1.0 / (double)si_rho(A.U, (float)rho);
            rc = 1.0 / vol;
            double Tn;
            if (gas::T_from_u(t, Yc, si_energy_mass(A.U, (float)Uint), Tc, 1e-14, 100, Tn) < 0)
                atomic_status(A.status, LBMGPU_ST_NEWTON);
            Tc = Tn;
        }
        double hrr = 0.0;
        for (int a = 0; a < NS; ++a) {
            hrr += -1.0 * (double)u_energy_mass(A.U, (float)(gas::h_RT(t, a, Tc) * gas::kR * Tc / t.m.W[a])) * drho[a];
            prp(pr_drho<NS>(a), drho[a]);
        }
        put(A, A.rec_nxt, RM_HRR, n, hrr);
    } else if (CHEM == CHEM_ROSENBROCK) {  // the host build; the device runs it in k_mc_chem
        double rc, rac[NS], Yc[NS], Tc, rhoc, Pc;  // the state as k_mc_chem forms it
        mc_chem_state<NS>(A, n, rc, rac, Yc, Tc, rhoc, Pc);
        mc_chem_ros2<NS>(A, n, rc, rac, Yc, Tc, rhoc, Pc, true);
    }

    if constexpr (sizeof(typename AT::P) == sizeof(float))
        mc_transport_f32<NS>(A, n, p, rho_a, ua, Xs, Y, X, W, T_si, P_si, Uint);
    else
        mc_transport_f64<NS>(A, n, p, rho_a, ua, Xs, Y, X, W, T_si, P_si, Uint);
}

// The energy-flux terms of the energy collision (lbm-collision.cpp:265-316): the enthalpy
// diffusion q_diff and the upwind mass-fraction correction q_corr summed over the species,
// the heat-flux difference and the pressure-tensor term -> dq (3 planes), from the rates
// mc_props_cell wrote.  A kernel of its own: it is mostly neighbour loads, which hide
// behind each other at the occupancy of a small kernel.
template <int NS, class AT>
MC_HDN void mc_eflux_cell(const AT &A, long n) {
    const gas::Tables &t = *A.tab;
    const typename AT::R *Rc = A.rec_cur;
    double *Pr = A.props;
    auto prg = [&](int plane) { return Pr[(long)plane * A.ncell + n]; };
    auto prp = [&](int plane, double v) { Pr[(long)plane * A.ncell + n] = v; };
    const double rho = rec(A, Rc, RM_RHO, n);
    const double um[3] = {rec(A, Rc, RM_U, n), rec(A, Rc, RM_V, n), rec(A, Rc, RM_W, n)};
    const double Tl = rec(A, Rc, RM_T, n), p = rec(A, Rc, RM_P, n);
    const double T_si = si_temp(A.U, (float)Tl);
    const double dt = A.dt;
    const double om = prg(pr_omm<NS>()), om1 = prg(pr_om1<NS>()), gasconstant = prg(pr_gc<NS>());
    long nbl[3], nbh[3];
    int tl[3], th[3];
    for (int d = 0; d < 3; ++d) {
        const long off = d == 0 ? A.si : (d == 1 ? A.sj : 1);
        nbl[d] = n - off;
        nbh[d] = n + off;
        tl[d] = A.type[nbl[d]];
        th[d] = A.type[nbh[d]];
    }
    double qd[3] = {0, 0, 0}, qc[3] = {0, 0, 0};
    const double rl[3] = {rec(A, Rc, RM_RHO, nbl[0]), rec(A, Rc, RM_RHO, nbl[1]), rec(A, Rc, RM_RHO, nbl[2])};
    const double rh[3] = {rec(A, Rc, RM_RHO, nbh[0]), rec(A, Rc, RM_RHO, nbh[1]), rec(A, Rc, RM_RHO, nbh[2])};
    // the FP32 storage mode: reciprocal densities and enthalpy quotients (rounding-level
    // differences, as in its moment solve)
    constexpr bool fast = sizeof(typename AT::P) == sizeof(float);
    double irl[3], irh[3];
    const double ir = fast ? 1.0 / rho : 0.0, invT = fast ? 1.0 / T_si : 0.0;
    for (int d = 0; d < 3; ++d) {
        irl[d] = fast ? 1.0 / rl[d] : 0.0;
        irh[d] = fast ? 1.0 / rh[d] : 0.0;
    }
    for (int a = 0; a < NS; ++a) {
        const double ha =
            fast ? u_energy_mass(A.U, (float)(gas::h_RT_fast(t, a, T_si, invT) * gas::kR * T_si * t.invW[a]))
                 : u_energy_mass(A.U, (float)(gas::h_RT(t, a, T_si) * gas::kR * T_si / t.m.W[a]));
        const int pr = rs(a, RS_RHO);
        const double rho_a = rec(A, Rc, pr, n);
        const double ua[3] = {rec(A, Rc, rs(a, RS_UX), n), rec(A, Rc, rs(a, RS_UX + 1), n),
                              rec(A, Rc, rs(a, RS_UX + 2), n)};
        for (int d = 0; d < 3; ++d) {
            qd[d] += om1 / (-om + om1) * ha * rho_a * (ua[d] - um[d]);
            const double Yl = fast ? rec(A, Rc, pr, nbl[d]) * irl[d] : rec(A, Rc, pr, nbl[d]) / rl[d];
            const double Yc = fast ? rho_a * ir : rho_a / rho;
            const double Yh = fast ? rec(A, Rc, pr, nbh[d]) * irh[d] : rec(A, Rc, pr, nbh[d]) / rh[d];
            const double dY = mc_fd_fuw(Yl, Yc, Yh, ua[d] - um[d], tl[d], th[d]);
            qc[d] += 0.5 * (2.0 - om1) / (-om + om1) * dt * p * ha * dY;
        }
    }
    double P6[6];
    for (int q = 0; q < 6; ++q) P6[q] = rec(A, Rc, RM_P00 + q, n);
    const double Pf[3][3] = {{P6[0], P6[1], P6[2]}, {P6[1], P6[3], P6[4]}, {P6[2], P6[4], P6[5]}};
    for (int d = 0; d < 3; ++d) {
        const double Qc = rho * um[d] * (1.0 - 3.0 * gasconstant * Tl) - rho * (um[d] * um[d] * um[d]);
        const double dQ = mc_fd_central(rec(A, Rc, RM_QX + d, nbl[d]), Qc, rec(A, Rc, RM_QX + d, nbh[d]), tl[d], th[d]);
        double s = 0.0;
        for (int b = 0; b < 3; ++b) s += um[b] * (Pf[b][d] - ((b == d ? p : 0.0) + rho * um[b] * um[d]));
        prp(pr_dq<NS>(d), s + qd[d] + qc[d] + 0.5 * dt * um[d] * dQ);
    }
}

// The cell's populations of one set after streaming and boundary treatment: in place
// (local mode), from the special-cell store, or pulled from the upstream cells.  The
// mode is resolved once into a base pointer, a plane stride and a per-axis offset table,
// so the 27 loads are branch-free and issue back to back.
template <class AT>
struct McFetch {
    using P = typename AT::P;
    const P *src;
    long stride;
    int X[3], Y[3], Z[3];
    const double *shift;
    MC_HD McFetch(const AT &A, long n) : shift(A.shift) {
        const bool special = !A.local && (A.cflag[n] & CF_SPECIAL);
        if (A.local || special) {
            const int base = special ? A.bid[n] : (int)n;
            src = special ? A.bst_cur : A.pop_src;
            stride = special ? A.nb : A.ncell;
            for (int c = 0; c < 3; ++c) {
                X[c] = base;
                Y[c] = 0;
                Z[c] = 0;
            }
        } else {
            McPull pp;
            mc_pull(A, n, pp);
            src = A.pop_src;
            stride = A.ncell;
            for (int c = 0; c < 3; ++c) {
                X[c] = (int)pp.X[c];
                Y[c] = (int)pp.Y[c];
                Z[c] = (int)pp.Z[c];
            }
        }
    }
    MC_HD double operator()(int plane, int l) const {
        const double v = (double)src[(long)plane * stride + (X[cidx(cx(l))] + Y[cidx(cy(l))] + Z[cidx(cz(l))])];
        return shift ? v + shift[plane] : v;
    }
};

// BGK update of species a at cell n (lbm-collision.cpp:446-519).
template <int NS, class AT>
MC_HDN void mc_relax_species(const AT &A, long n, int a) {
    const gas::Tables &t = *A.tab;
    const typename AT::R *Rc = A.rec_cur;
    const double *Pr = A.props;
    auto prg = [&](int plane) { return Pr[(long)plane * A.ncell + n]; };
    const double rho_a = rec(A, Rc, rs(a, RS_RHO), n);
    const double um[3] = {rec(A, Rc, RM_U, n), rec(A, Rc, RM_V, n), rec(A, Rc, RM_W, n)};
    const double Tl = rec(A, Rc, RM_T, n);
    const double om = prg(pr_om<NS>(a));
    const double dt = A.dt;
    // loads that do not depend on the fetch mode first: the face terms and neighbour types,
    // the shift parameters and the chemistry source
    double qf[3][3];
    int tyl[3], tyh[3];
    for (int d = 0; d < 3; ++d) {
        const long off = d == 0 ? A.si : (d == 1 ? A.sj : 1);
        const int pq = rs(a, RS_QX + d);
        qf[d][0] = rec(A, Rc, pq, n - off);
        qf[d][1] = rec(A, Rc, pq, n);
        qf[d][2] = rec(A, Rc, pq, n + off);
        tyl[d] = A.type[n - off];
        tyh[d] = A.type[n + off];
    }
    const double fsh[3] = {prg(pr_f<NS>(a, 0)), prg(pr_f<NS>(a, 1)), prg(pr_f<NS>(a, 2))};
    const double drho = A.chem != CHEM_OFF ? prg(pr_drho<NS>(a)) : 0.0;
    const McFetch<AT> fetch(A, n);
    double fv[27];
#pragma unroll
    for (int l = 0; l < 27; ++l) fv[l] = fetch(27 * a + l, l);
    // bare species velocity sum f c / rho_a (lbm-collision.cpp:446-454)
    double ux[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        ux[0] += fv[l] * cx(l);
        ux[1] += fv[l] * cy(l);
        ux[2] += fv[l] * cz(l);
    }
    for (int d = 0; d < 3; ++d) ux[d] = ux[d] / rho_a;
    const double theta = t.Ra_lat[a] * Tl;
    double corr[3];
    for (int d = 0; d < 3; ++d) {  // FD of the face terms the moment kernels stored (lbm-collision.cpp:487-497)
        const double dQ = mc_fd_central(qf[d][0], qf[d][1], qf[d][2], tyl[d], tyh[d]);
        corr[d] = dt * (2.0 - om) / (2.0 * rho_a * om) * dQ;
    }
    AxisF<double> Fe, Fd, Fr;
    axis_feq(Fe, ux, theta, corr);
    const double udu[3] = {ux[0] + fsh[0], ux[1] + fsh[1], ux[2] + fsh[2]};
    axis_feq(Fd, udu, theta, corr);
    const double zero[3] = {0.0, 0.0, 0.0};
    axis_feq(Fr, um, theta, zero);
    const bool skip_all = rho_a <= kSpeciesMin && A.chem == CHEM_OFF;
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const int plane = 27 * a + l;
        const double fr = A.chem != CHEM_OFF ? feq_l(l, drho, Fr) : 0.0;
        if (skip_all || (rho_a <= kSpeciesMin && fr <= 0.0)) {
            if (!A.local) A.pop_dst[(long)plane * A.ncell + n] = A.pop_prev[(long)plane * A.ncell + n];
            continue;
        }
        const double fe = feq_l(l, rho_a, Fe);
        const double fd = feq_l(l, rho_a, Fd);
        stpop(A, A.pop_dst, plane, n, fv[l] + om * (fe - fv[l]) + (fd - fe) + fr);
    }
}

// Update of the energy populations at cell n (lbm-collision.cpp:317-324).
template <int NS, class AT>
MC_HDN void mc_relax_energy(const AT &A, long n) {
    const typename AT::R *Rc = A.rec_cur;
    const double *Pr = A.props;
    auto prg = [&](int plane) { return Pr[(long)plane * A.ncell + n]; };
    const double rho = rec(A, Rc, RM_RHO, n);
    const double um[3] = {rec(A, Rc, RM_U, n), rec(A, Rc, RM_V, n), rec(A, Rc, RM_W, n)};
    const double om = prg(pr_omm<NS>()), om1 = prg(pr_om1<NS>());
    const double dq[3] = {prg(pr_dq<NS>(0)), prg(pr_dq<NS>(1)), prg(pr_dq<NS>(2))};
    AxisG<double> G;
    axis_geq(G, prg(pr_uint<NS>()), prg(pr_theta<NS>()), um);
    const McFetch<AT> fetch(A, n);
    double gv[27];
#pragma unroll
    for (int l = 0; l < 27; ++l) gv[l] = fetch(27 * NS + l, l);
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        const double gq = geq_l(l, rho, G);
        const double gs = (csq(l) == 1) ? gq + 0.5 * (cx(l) * dq[0] + cy(l) * dq[1] + cz(l) * dq[2]) : gq;
        stpop(A, A.pop_dst, 27 * NS + l, n, gv[l] + om1 * (gq - gv[l]) + (om - om1) * (gq - gs));
    }
}

// The whole collision of one cell (host build and tests): props, then every set.
template <int NS, class AT>
MC_HDN void mc_collide_cell(const AT &A, long n) {
    if (A.chem == CHEM_REF_EXPLICIT)
        mc_props_cell<NS, CHEM_REF_EXPLICIT>(A, n);
    else if (A.chem == CHEM_ROSENBROCK)
        mc_props_cell<NS, CHEM_ROSENBROCK>(A, n);
    else
        mc_props_cell<NS, CHEM_OFF>(A, n);
    mc_eflux_cell<NS>(A, n);
    for (int a = 0; a < NS; ++a) mc_relax_species<NS>(A, n, a);
    mc_relax_energy<NS>(A, n);
}

// ------------------------------------------------------------------------------------
// Init (reference LBM::Init, multicomponent, src/lbm-init.cpp:85-146).  Writes the
// record planes it changes into both record buffers and the populations into pop0.
// ------------------------------------------------------------------------------------
template <int NS, class AT>
MC_HDN void mc_init_cell(const AT &A, long n, typename AT::R *rec0, typename AT::R *rec1, typename AT::P *pop0) {
    const int ty = A.type[n];
    if (!(ty == T_F || ty == T_I || ty == T_I_C || ty == T_O || ty == T_O_C)) return;
    const gas::Tables &t = *A.tab;
    double X[NS], Y[NS];
    double s = 0.0;
    for (int a = 0; a < NS; ++a) {
        const double xa = rec(A, rec0, rs(a, RS_X), n);
        X[a] = xa > 0.0 ? xa : 0.0;
        s += X[a];
    }
    double W = 0.0;
    for (int a = 0; a < NS; ++a) {
        X[a] /= s;
        W += X[a] * t.m.W[a];
    }
    for (int a = 0; a < NS; ++a) Y[a] = X[a] * t.m.W[a] / W;
    const double Tl = rec(A, rec0, RM_T, n);
    const double T_si = si_temp(A.U, (float)Tl);
    const double P_si = si_p(A.U, (float)rec(A, rec0, RM_P, n));
    const double dens = P_si * W / (gas::kR * T_si);
    const double rho = u_rho(A.U, (float)dens);
    const double vel[3] = {rec(A, rec0, RM_U, n), rec(A, rec0, RM_V, n), rec(A, rec0, RM_W, n)};
    const double U = u_energy_mass(A.U, (float)gas::int_energy_mass(t, Y, T_si));
    const double rhoe = rho * (U + 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]));
    const double theta = u_energy_mass(A.U, (float)(gas::kR * T_si / W));
    typename AT::R *R2[2] = {rec0, rec1};
    for (int b = 0; b < 2; ++b) {
        put(A, R2[b], RM_RHO, n, rho);
        put(A, R2[b], RM_RHOE, n, rhoe);
    }
    const bool fluid = ty == T_F;
    AxisG<double> G;
    axis_geq(G, U, theta, vel);
    if (fluid)
        for (int l = 0; l < 27; ++l) stpop(A, pop0, 27 * NS + l, n, geq_l(l, rho, G));
    const double zero[3] = {0.0, 0.0, 0.0};
    double ra_all[NS], ua_all[NS][3];
    for (int a = 0; a < NS; ++a) {
        double ra = Y[a] * rho;
        ra = ra > kSpeciesMin ? ra : kSpeciesMin;
        ra_all[a] = ra;
        const double tha = u_energy_mass(A.U, (float)(gas::kR * T_si / t.m.W[a]));
        for (int b = 0; b < 2; ++b) {
            put(A, R2[b], rs(a, RS_RHO), n, ra);
            for (int d = 0; d < 3; ++d) put(A, R2[b], rs(a, RS_UX + d), n, vel[d]);
        }
        for (int d = 0; d < 3; ++d) ua_all[a][d] = vel[d];
        if (fluid) {
            AxisF<double> Fe;
            axis_feq(Fe, vel, tha, zero);
            for (int l = 0; l < 27; ++l) stpop(A, pop0, 27 * a + l, n, feq_l(l, ra, Fe));
        }
    }
    for (int b = 0; b < 2; ++b) store_face_terms<NS>(A, R2[b], n, ty, rho, vel, Tl, ra_all, ua_all);
}

}  // namespace lbm
