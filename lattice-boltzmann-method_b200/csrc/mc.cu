// lbmgpu, multicomponent path: device kernels around the per-cell functions of
// mc_cell.cuh and the handle operations for n_species > 0.
//
// Reference path replaced (farrasarira/Lattice-Boltzmann-Method, MULTICOMP on):
//   LBM::Collide_Species + LBM::Collide   src/lbm-collision.cpp:191-526 -> k_mc_props, k_mc_chem (stiff
//                                          chemistry or the surrogate's use; the surrogate's kernels,
//                                          k_mc_chem_list), k_mc_eflux, k_mc_relax
//   LBM::Streaming + LBM::calculate_moment src/lbm-streaming.cpp, src/lbm-moment.cpp:193-377
//                                          -> k_mc_gather (pull + population sums per
//                                             (cell, set)) and k_mc_solve (per cell)
//   LBM::Init                              src/lbm-init.cpp:85-146 -> k_mc_init
//   LBM::Streaming + LBM::TMS_BC + LBM::calculate_moment of the cells with a boundary
//   upstream (src/lbm-bc.cpp:122-1110, src/impose_nscbc.cpp) -> k_mc_special
// Cell types: fluid, periodic ghosts, solid (TMS wall), adiabatic, free-slip, and the
// characteristic inflow/outflow ghosts TYPE_I_C / TYPE_O_C.  The reference's
// non-characteristic TYPE_I / TYPE_O rewrite a neighbour's moments from inside the
// boundary sweep (order dependent) and are rejected at upload with LBMGPU_E_UNSUPPORTED.
//
// Storage: FP64 (bit-faithful to the reference) or FP32 (LBMGPU_FP32: populations in
// float as deviations from a per-plane shift; the per-cell record stays FP64, and all
// arithmetic is FP64).
#include <algorithm>
#include <cstring>
#include <vector>

#include "halo.cuh"
#include "handle.cuh"
#include "mc_bc.cuh"
#include "mc_cell.cuh"
#include "surrogate_host.cuh"

namespace {

using namespace lbm;
using namespace lbmh;

constexpr int NS9 = 9;

// collision parameters of every fluid cell, one instance per chemistry mode
// FP32 storage: the transport runs in FP32, and four blocks per SM (at most 128 registers)
// keep more cells in flight than the FP64 instance's register budget allows
template <int NS, int CHEM, typename S>
__global__ void __launch_bounds__(kBlock, sizeof(S) == sizeof(float) ? 4 : 3) k_mc_props(McArgsT<S, double> A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || !(A.cflag[n] & CF_FLUID)) return;
    mc_props_cell<NS, CHEM>(A, n);
}

// The cells the surrogate leaves to the integrator (sur.ilist), G lanes per cell: the
// lanes of a group evaluate the finite-difference Jacobian's columns side by side
// (gas::ros2_advance_group), so the listed cells do not wait on serial integrations of one
// lane each.  A short list (up to kChemShortList cells: latency-bound) takes 8 lanes per
// cell, a long one 4 (the group's redundant factorisation then costs more than the
// latency it saves); the choice is made on the device from the list's length.
constexpr unsigned kChemShortList = 5000;
template <int NS, int G, typename S, class KIN>
__device__ __forceinline__ void chem_list_groups(const McArgsT<S, double> &A, unsigned cnt) {
    const unsigned groups = gridDim.x * blockDim.x / G;
    for (unsigned i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < cnt; i += groups) {
        const long n = A.sur.ilist[i];
        double rho, rho_a[NS], Y[NS], T_si, rho_si, P_si;
        mc_chem_state<NS>(A, n, rho, rho_a, Y, T_si, rho_si, P_si);
        mc_chem_ros2<NS, McArgsT<S, double>, true, G, KIN>(A, n, rho, rho_a, Y, T_si, rho_si, P_si, false);
    }
}
// With a compiled mechanism (KIN: analytic species Jacobian, two right-hand sides per
// sub-step besides it) a cell is one lane's work.
template <int NS, typename S, class KIN = void>
__global__ void __launch_bounds__(kBlock) k_mc_chem_list(McArgsT<S, double> A) {
    const unsigned cnt = *A.sur.icount;
    if constexpr (!std::is_void_v<KIN>)
        chem_list_groups<NS, 1, S, KIN>(A, cnt);
    else if (cnt <= kChemShortList)
        chem_list_groups<NS, 8, S, KIN>(A, cnt);
    else
        chem_list_groups<NS, 4, S, KIN>(A, cnt);
}

// Chemistry of every fluid cell for LBMGPU_CHEM_ROSENBROCK handles, one thread per cell,
// beside the transport part of the collision parameters (k_mc_props<CHEM_OFF>), from the
// state the collision forms from the record (mc_chem_state):
//   SUR = false: the stiff integrator (ROS2) itself;
//   SUR = true : the surrogate's prediction where the gate passes it (element projection,
//                output gate), the cells it does not cover and the audited ones appended
//                to the integrator list for k_mc_chem_list.
// A kernel of its own, so that its time (with the surrogate's kernels) is the chemistry's
// share of the step, and the transport kernel keeps its own occupancy.
// One thread per cell.  The integrator's vectors are sized by the species count at compile
// time (ros2_advance_n) so that they stay in registers; its iteration matrix and the rate
// factors stay per-thread local memory, and the bound of two blocks per SM keeps that
// working set (about 2 kB per thread) inside L2 instead of streaming it through HBM.
// KIN: the compiled kinetics of the handle's mechanism (gen_kinetics.py), void for the tables.
template <int NS, bool SUR, typename S, class KIN = void>
__global__ void __launch_bounds__(kBlock, 2) k_mc_chem(McArgsT<S, double> A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || !(A.cflag[n] & CF_FLUID)) return;
    double rho, rho_a[NS], Y[NS], T_si, rho_si, P_si;
    mc_chem_state<NS>(A, n, rho, rho_a, Y, T_si, rho_si, P_si);
    mc_chem_ros2<NS, McArgsT<S, double>, !SUR, 1, KIN>(A, n, rho, rho_a, Y, T_si, rho_si, P_si, SUR);
}

// The energy-flux terms of the collision (mc_eflux_cell), after the collision parameters.
template <int NS, typename S>
__global__ void __launch_bounds__(kBlock) k_mc_eflux(McArgsT<S, double> A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || !(A.cflag[n] & CF_FLUID)) return;
    mc_eflux_cell<NS>(A, n);
}

// BGK update: blockIdx.y selects the population set (species 0..NS-1, NS = energy), the
// x dimension the cells, so a warp reads one set's planes at 32 consecutive cells
template <int NS, typename S>
__global__ void __launch_bounds__(kBlock, 4) k_mc_relax(McArgsT<S, double> A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || !(A.cflag[n] & CF_FLUID)) return;
    const int a = blockIdx.y;
    if (a < NS)
        mc_relax_species<NS>(A, n, a);
    else
        mc_relax_energy<NS>(A, n);
}

// the cells with a boundary upstream, one thread each (compact list)
template <int NS, typename S>
__global__ void __launch_bounds__(kBlock) k_mc_special(McArgsT<S, double> A, const long *__restrict__ blist) {
    const long b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= A.nb) return;
    mc_special_cell<NS>(A, blist[b], b);
}

// the special cells' current populations into the compact store (after upload and Init)
template <typename S>
__global__ void k_mc_fill_bst(long ncell, long nb, int np, const long *__restrict__ blist, const S *__restrict__ pop,
                              S *__restrict__ bst) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)np * nb) return;
    const int q = (int)(i / nb);
    const long b = i - (long)q * nb;
    bst[i] = pop[(long)q * ncell + blist[b]];
}

// Interior cells (no boundary upstream): the pull of one population set per thread
// (blockIdx.y = species, NS = the energy set) and its sums into the gsum planes --
// species a: rho_a, j_a, its P-tensor share at planes 10a..10a+9; the energy set's sum at
// plane 10 NS.  A warp reads one set's planes at 32 consecutive cells.
template <int NS, typename S>
__global__ void __launch_bounds__(kBlock, 4) k_mc_gather(McArgsT<S, double> A, double *__restrict__ gs) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || A.cflag[n] != CF_FLUID) return;
    const int a = blockIdx.y;
    McPull pp;
    mc_pull(A, n, pp);
    if (a < NS) {
        double fv[27], s[kGsPerSpecies];
#pragma unroll
        for (int l = 0; l < 27; ++l) fv[l] = ldpop(A, A.pop_src, 27 * a + l, pull_idx(pp, l));
        species_sums(fv, s);
#pragma unroll
        for (int q = 0; q < kGsPerSpecies; ++q) gs[(long)(kGsPerSpecies * a + q) * A.ncell + n] = s[q];
    } else {
        double e = 0.0;
#pragma unroll
        for (int l = 0; l < 27; ++l) e += ldpop(A, A.pop_src, 27 * NS + l, pull_idx(pp, l));
        gs[(long)(kGsPerSpecies * NS) * A.ncell + n] = e;
    }
}

// Interior cells: the moment solve from the gathered sums (species velocities from the
// Stefan-Maxwell system, temperature, the record) -- the same bits as mc_stream_moment_cell.
template <int NS, typename S>
__global__ void __launch_bounds__(kBlock, 2) k_mc_solve(McArgsT<S, double> A, const double *__restrict__ gs) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || A.cflag[n] != CF_FLUID) return;
    const SumsAt<NS> Sm{gs, A.ncell, n};
    mc_moments_finish<NS>(A, n, Sm);
}

template <int NS, typename S>
__global__ void __launch_bounds__(kBlock) k_mc_init(McArgsT<S, double> A, double *rec0, double *rec1, S *pop0) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell) return;
    mc_init_cell<NS>(A, n, rec0, rec1, pop0);
}

// FP32 storage: new per-plane shift = mean over the fluid cells of the decoded population
// (one block per plane, fixed reduction order, so the result is deterministic) ...
constexpr int kMeanBlock = 256;
template <typename S>
__global__ void __launch_bounds__(kMeanBlock) k_plane_mean(McArgsT<S, double> A, const S *pop, double *shift_new,
                                                           long nfluid) {
    __shared__ double red[kMeanBlock];
    const int q = blockIdx.x;
    double s = 0.0;
    for (long n = threadIdx.x; n < A.ncell; n += kMeanBlock)
        if (A.cflag[n] & CF_FLUID) s += ldpop(A, pop, q, n);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kMeanBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) shift_new[q] = nfluid > 0 ? red[0] / (double)nfluid : 0.0;
}

// ... and both population buffers re-encoded from the old shift to the new one.
template <typename S>
__global__ void k_reshift(long total, long ncell, S *p0, S *p1, const double *old_s, const double *new_s) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int q = (int)(i / ncell);
    const double d = old_s[q] - new_s[q];
    p0[i] = (S)((double)p0[i] + d);
    p1[i] = (S)((double)p1[i] + d);
}

__device__ __forceinline__ double ldd(const char *rec, long off) { return *reinterpret_cast<const double *>(rec + off); }
__device__ __forceinline__ void std_(char *rec, long off, double v) { *reinterpret_cast<double *>(rec + off) = v; }

// Staging layout of a chunk of cnt cells: cnt mixture records, then cnt records of each
// species in turn.
template <int NS, typename S>
__global__ void k_mc_unpack(McArgsT<S, double> A, MixOff mo, SpOff so, const char *__restrict__ stage, long n0, long n1,
                            double *rec0, double *rec1, S *pop0, S *pop1) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    const long cnt = n1 - n0;
    const char *mr = stage + (n - n0) * mo.size;
    auto pr = [&](int plane, double v) {
        put(A, rec0, plane, n, v);
        put(A, rec1, plane, n, v);
    };
    const double rho = ldd(mr, mo.rho), T = ldd(mr, mo.temp);
    const double um[3] = {ldd(mr, mo.u), ldd(mr, mo.v), ldd(mr, mo.w)};
    pr(RM_RHO, rho);
    pr(RM_U, um[0]);
    pr(RM_V, um[1]);
    pr(RM_W, um[2]);
    pr(RM_T, T);
    pr(RM_P, ldd(mr, mo.p));
    pr(RM_RHOE, ldd(mr, mo.rhoe));
    const int pi[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int q = 0; q < 6; ++q) pr(RM_P00 + q, ldd(mr, mo.p_tensor + 8 * (3 * pi[q][0] + pi[q][1])));
    pr(RM_HRR, ldd(mr, mo.HRR));
    const bool fluid = A.type[n] == T_F;  // the cell classification follows the whole upload
    double rho_a[NS], ua[NS][3];
    for (int a = 0; a < NS; ++a) {
        const char *sr = stage + cnt * mo.size + ((long)a * cnt + (n - n0)) * so.size;
        rho_a[a] = ldd(sr, so.rho);
        ua[a][0] = ldd(sr, so.u);
        ua[a][1] = ldd(sr, so.v);
        ua[a][2] = ldd(sr, so.w);
        pr(rs(a, RS_RHO), rho_a[a]);
        for (int d = 0; d < 3; ++d) pr(rs(a, RS_UX + d), ua[a][d]);
        pr(rs(a, RS_X), ldd(sr, so.X));
        if (fluid)
            for (int l = 0; l < 27; ++l) {
                stpop(A, pop0, 27 * a + l, n, ldd(sr, so.f + 8 * l));
                stpop(A, pop1, 27 * a + l, n, ldd(sr, so.fpc + 8 * l));
            }
    }
    store_face_terms<NS>(A, rec0, n, A.type[n], rho, um, T, rho_a, ua);
    store_face_terms<NS>(A, rec1, n, A.type[n], rho, um, T, rho_a, ua);
    if (fluid)
        for (int l = 0; l < 27; ++l) {
            stpop(A, pop0, 27 * NS + l, n, ldd(mr, mo.g + 8 * l));
            stpop(A, pop1, 27 * NS + l, n, ldd(mr, mo.gpc + 8 * l));
        }
}

// pop_now: what the cell's populations are taken from (pulled when `stepped`, in place
// otherwise); pop_pc: the post-collision populations (fpc, gpc).
template <int NS, typename S>
__global__ void k_mc_pack(McArgsT<S, double> A, MixOff mo, SpOff so, char *__restrict__ stage, long n0, long n1,
                          const double *rec, const S *pop_now, const S *pop_pc, const S *bst, int stepped) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    const long cnt = n1 - n0;
    char *mr = stage + (n - n0) * mo.size;
    auto get = [&](int plane) { return (double)rec[(long)plane * A.ncell + n]; };
    std_(mr, mo.rho, get(RM_RHO));
    std_(mr, mo.u, get(RM_U));
    std_(mr, mo.v, get(RM_V));
    std_(mr, mo.w, get(RM_W));
    std_(mr, mo.temp, get(RM_T));
    std_(mr, mo.p, get(RM_P));
    std_(mr, mo.rhoe, get(RM_RHOE));
    std_(mr, mo.HRR, get(RM_HRR));
    const int full[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int q = 0; q < 9; ++q) std_(mr, mo.p_tensor + 8 * q, get(RM_P00 + full[q]));
    const bool fluid = A.cflag[n] & CF_FLUID;
    const bool special = stepped && (A.cflag[n] & CF_SPECIAL);
    const long bs = special ? (long)A.bid[n] : 0;
    McPull pp;
    mc_pull(A, n, pp);
    // the cell's populations: kept in the special-cell store, pulled, or in place
    auto now = [&](int plane, int l) {
        if (special) return ldpop_b(A, bst, plane, bs);
        return ldpop(A, pop_now, plane, stepped ? pull_idx(pp, l) : n);
    };
    for (int a = 0; a < NS; ++a) {
        char *sr = stage + cnt * mo.size + ((long)a * cnt + (n - n0)) * so.size;
        std_(sr, so.rho, get(rs(a, RS_RHO)));
        std_(sr, so.u, get(rs(a, RS_UX)));
        std_(sr, so.v, get(rs(a, RS_UX + 1)));
        std_(sr, so.w, get(rs(a, RS_UX + 2)));
        std_(sr, so.X, get(rs(a, RS_X)));
        if (!fluid) continue;
        for (int l = 0; l < 27; ++l) {
            const int plane = 27 * a + l;
            std_(sr, so.f + 8 * l, now(plane, l));
            std_(sr, so.fpc + 8 * l, ldpop(A, pop_pc, plane, n));
        }
    }
    if (!fluid) return;
    double q3[3] = {0, 0, 0};
    for (int l = 0; l < 27; ++l) {
        const int plane = 27 * NS + l;
        const double gv = now(plane, l);
        std_(mr, mo.g + 8 * l, gv);
        std_(mr, mo.gpc + 8 * l, ldpop(A, pop_pc, plane, n));
        q3[0] += gv * cx(l);
        q3[1] += gv * cy(l);
        q3[2] += gv * cz(l);
    }
    for (int q = 0; q < 3; ++q) std_(mr, mo.energy_flux + 8 * q, q3[q]);
}

template <typename S>
McArgsT<S, double> base_args(lbmgpu *h) {
    McArgsT<S, double> A{};
    A.Nx = h->g.Nx;
    A.halo_lo = h->halo_lo;
    A.halo_hi = h->halo_hi;
    A.Nx_glob = h->nx_glob > 0 ? h->nx_glob : h->g.Nx;
    A.Ny = h->g.Ny;
    A.Nz = h->g.Nz;
    A.ncell = h->g.ncell;
    A.sj = h->g.sj;
    A.si = h->g.si;
    A.ns = h->ns;
    A.dt = h->d.dt_sim;
    A.chem = h->chem;
    A.U = h->U;
    A.tab = h->tab;
    A.type = h->type;
    A.cflag = h->cflag;
    A.status = h->status;
    A.shift = h->fp32 ? h->shift[0] : nullptr;
    A.bid = h->bid;
    A.nb = h->nb;
    A.props = h->props;
    return A;
}

// The two storage types' buffers behind one accessor.
template <typename S> S *popb(lbmgpu *h, int b);
template <> double *popb<double>(lbmgpu *h, int b) { return h->pop[b]; }
template <> float *popb<float>(lbmgpu *h, int b) { return h->pop32[b]; }
template <typename S> S *bstb(lbmgpu *h, int b);
template <> double *bstb<double>(lbmgpu *h, int b) { return h->bst[b]; }
template <> float *bstb<float>(lbmgpu *h, int b) { return h->bst32[b]; }

// the special cells' populations of pop[cur] into bst[cur]
template <typename S>
int fill_bst(lbmgpu *h) {
    if (h->nb == 0) return 0;
    const int np = 27 * (h->ns + 1);
    const long total = (long)np * h->nb;
    k_mc_fill_bst<S><<<grid_for(total), kBlock, 0, h->stream>>>(h->g.ncell, h->nb, np, h->blist, popb<S>(h, h->cur),
                                                                bstb<S>(h, h->cur));
    CK(cudaGetLastError());
    return 0;
}

bool valid_mc_layout(const lbmgpu_mixture_layout &m, const lbmgpu_species_layout &s) {
    if (m.size == 0 || m.size % 8 || s.size == 0 || s.size % 8) return false;
    const long mext[][2] = {{m.p_tensor, 72}, {m.rho, 8}, {m.u, 8},  {m.v, 8},    {m.w, 8},
                            {m.p, 8},         {m.g, 216}, {m.gpc, 216}, {m.rhoe, 8}, {m.energy_flux, 24},
                            {m.temp, 8},      {m.HRR, 8}};
    for (const auto &e : mext)
        if (e[0] < 0 || e[0] % 8 || (size_t)(e[0] + e[1]) > m.size) return false;
    if (m.type < 0 || (size_t)(m.type + 2) > m.size) return false;
    const long sext[][2] = {{s.X, 8}, {s.rho, 8}, {s.f, 216}, {s.fpc, 216}, {s.u, 8}, {s.v, 8}, {s.w, 8}};
    for (const auto &e : sext)
        if (e[0] < 0 || e[0] % 8 || (size_t)(e[0] + e[1]) > s.size) return false;
    return true;
}

// FP32 storage: move both population buffers onto the mean of the current state.
int rebase_shift(lbmgpu *h) {
    if (!h->fp32) return 0;
    McArgsT<float, double> A = base_args<float>(h);
    const int np = 27 * (h->ns + 1);
    k_plane_mean<float><<<np, kMeanBlock, 0, h->stream>>>(A, h->pop32[h->cur], h->shift[1], h->nfluid);
    CK(cudaGetLastError());
    const long total = (long)np * h->g.ncell;
    k_reshift<float><<<grid_for(total), kBlock, 0, h->stream>>>(total, h->g.ncell, h->pop32[0], h->pop32[1],
                                                                h->shift[0], h->shift[1]);
    CK(cudaGetLastError());
    std::swap(h->shift[0], h->shift[1]);
    return 0;
}

// The records of cells [c0, c1) -- the caller's arrays start at cell c0 -- into the device
// state, one staging chunk at a time.
template <typename S>
int upload_t(lbmgpu *h, const char *hm, const void *const *species, long c0, long c1) {
    const size_t ms = h->mo.size, ss = h->so.size;
    McArgsT<S, double> A = base_args<S>(h);
    for (long n0 = c0; n0 < c1; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(c1, n0 + (long)h->stage_cells), cnt = n1 - n0;
        CK(cudaMemcpyAsync(h->stage, hm + (n0 - c0) * ms, cnt * ms, cudaMemcpyHostToDevice, h->stream));
        for (int a = 0; a < h->ns; ++a)
            CK(cudaMemcpyAsync(h->stage + cnt * ms + (size_t)a * cnt * ss,
                               static_cast<const char *>(species[a]) + (n0 - c0) * ss, cnt * ss,
                               cudaMemcpyHostToDevice, h->stream));
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        k_mc_unpack<NS9, S><<<grid_for(cnt), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[0],
                                                                     h->mom[1], popb<S>(h, 0), popb<S>(h, 1));
        ev_end(h, ep);
        CK(cudaGetLastError());
    }
    return 0;
}

template <typename S>
int pack_chunk(lbmgpu *h, long n0, long n1, bool stepped) {
    McArgsT<S, double> A = base_args<S>(h);
    const int c = h->cur;
    const S *pc = stepped ? popb<S>(h, c) : popb<S>(h, 1 - c);
    // the records' padding bytes come out as zeros, not as what the staging held before
    CK(cudaMemsetAsync(h->stage, 0, (size_t)(n1 - n0) * (h->mo.size + (size_t)h->ns * h->so.size), h->stream));
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_mc_pack<NS9, S><<<grid_for(n1 - n0), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[c],
                                                                   popb<S>(h, c), pc, bstb<S>(h, c), stepped ? 1 : 0);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

template <typename S>
int init_t(lbmgpu *h) {
    McArgsT<S, double> A = base_args<S>(h);
    const int c = h->cur;
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_mc_init<NS9, S><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A, h->mom[c], h->mom[1 - c],
                                                                      popb<S>(h, c));
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

template <typename S>
int collide_t(lbmgpu *h) {
    const int c = h->cur, x = 1 - c;
    McArgsT<S, double> A = base_args<S>(h);
    const bool local = h->pack_mode != PK_STEPPED;
    A.pop_src = popb<S>(h, c);
    A.pop_dst = popb<S>(h, x);
    A.pop_prev = local ? nullptr : popb<S>(h, c);
    A.rec_cur = h->mom[c];
    A.rec_nxt = h->mom[x];
    A.local = local ? 1 : 0;
    A.bst_cur = bstb<S>(h, c);
    const int rs_ = sur_prepare_t<S>(h, A);
    if (rs_) return rs_;
    EvPair ep{};
    ev_begin(h, K_PROPS, ep);
    const unsigned gp = grid_for(h->g.ncell);
    if (h->chem == CHEM_REF_EXPLICIT)
        k_mc_props<NS9, CHEM_REF_EXPLICIT, S><<<gp, kBlock, 0, h->stream>>>(A);
    else
        k_mc_props<NS9, CHEM_OFF, S><<<gp, kBlock, 0, h->stream>>>(A);  // ROS2 / surrogate: k_mc_chem
    ev_end(h, ep);
    CK(cudaGetLastError());
    if (h->chem == CHEM_ROSENBROCK) {
        EvPair ec{};
        ev_begin(h, K_CHEM, ec);
        using KinH2 = kin_h2_air_9::Kinetics;
        if (A.sur.mode == 1 && A.sur.ilist)
            k_mc_chem<NS9, true, S><<<gp, kBlock, 0, h->stream>>>(A);
        else if (h->kin == KIN_H2_AIR_9)
            k_mc_chem<NS9, false, S, KinH2><<<gp, kBlock, 0, h->stream>>>(A);
        else
            k_mc_chem<NS9, false, S><<<gp, kBlock, 0, h->stream>>>(A);
        ev_end(h, ec);
        CK(cudaGetLastError());
    }
    if (A.sur.ilist) {
        EvPair ei{};
        ev_begin(h, K_SURROGATE, ei);
        if (h->kin == KIN_H2_AIR_9)
            k_mc_chem_list<NS9, S, kin_h2_air_9::Kinetics><<<148 * 8, kBlock, 0, h->stream>>>(A);
        else
            k_mc_chem_list<NS9, S><<<148 * 8, kBlock, 0, h->stream>>>(A);
        ev_end(h, ei);
        CK(cudaGetLastError());
    }
    EvPair ee{};
    ev_begin(h, K_EFLUX, ee);
    k_mc_eflux<NS9, S><<<gp, kBlock, 0, h->stream>>>(A);
    ev_end(h, ee);
    CK(cudaGetLastError());
    EvPair er{};
    ev_begin(h, K_COLLIDE, er);
    k_mc_relax<NS9, S><<<dim3(grid_for(h->g.ncell), NS9 + 1), kBlock, 0, h->stream>>>(A);
    ev_end(h, er);
    CK(cudaGetLastError());
    return 0;
}

template <typename S>
int stream_t(lbmgpu *h) {
    const int c = h->cur, x = 1 - c;
    McArgsT<S, double> A = base_args<S>(h);
    A.pop_src = popb<S>(h, x);
    A.rec_cur = h->mom[c];
    A.rec_nxt = h->mom[x];
    // The boundary cells run on the side stream beside the interior's gather and solve:
    // the two sets of cells are disjoint, and both read only the post-collision populations
    // and the previous records, so the latency-bound boundary kernel overlaps them; the
    // handle's stream waits for it before anything that follows.
    if (h->nb > 0) {
        McArgsT<S, double> B = A;
        B.bst_cur = bstb<S>(h, c);
        B.bst_nxt = bstb<S>(h, x);
        CK(cudaEventRecord(h->fork, h->stream));
        CK(cudaStreamWaitEvent(h->side, h->fork, 0));
        EvPair eb{};
        ev_begin(h, K_OTHER, eb, h->side);
        k_mc_special<NS9, S><<<(unsigned)((h->nb + 31) / 32), 32, 0, h->side>>>(B, h->blist);
        ev_end(h, eb, h->side);
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->join, h->side));
    }
    EvPair ep{};
    ev_begin(h, K_STREAM_MOMENT, ep);
    k_mc_gather<NS9, S><<<dim3(grid_for(h->g.ncell), NS9 + 1), kBlock, 0, h->stream>>>(A, h->gsum);
    ev_end(h, ep);
    CK(cudaGetLastError());
    EvPair es{};
    ev_begin(h, K_SOLVE, es);
    k_mc_solve<NS9, S><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A, h->gsum);
    ev_end(h, es);
    CK(cudaGetLastError());
    if (h->nb > 0) CK(cudaStreamWaitEvent(h->stream, h->join, 0));
    return 0;
}

// Slab faces (halo.cuh): one thread per cell of the face plane.
template <int NS, typename S>
__global__ void k_halo_pack(McArgsT<S, double> A, const S *pop, const double *rec, int face, int what,
                            double *__restrict__ buf) {
    const long jk = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (jk >= (long)A.Ny * A.Nz) return;
    halo_pack_cell<NS>(A, pop, rec, face, what, jk, buf);
}
template <int NS, typename S>
__global__ void k_halo_unpack(McArgsT<S, double> A, S *pop, double *rec, int face, int what,
                              const double *__restrict__ buf) {
    const long jk = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (jk >= (long)A.Ny * A.Nz) return;
    halo_unpack_cell<NS>(A, pop, rec, face, what, jk, buf);
}

// populations: the post-collision buffer the coming stream reads (between Collide and
// calculate_moment); record: the current step's record (between steps)
template <typename S>
int halo_t(lbmgpu *h, int face, int what, double *buf, bool pack) {
    McArgsT<S, double> A = base_args<S>(h);
    S *pop = popb<S>(h, 1 - h->cur);
    double *rec = h->mom[h->cur];
    const long plane = (long)h->g.Ny * h->g.Nz;
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    if (pack)
        k_halo_pack<NS9, S><<<grid_for(plane), kBlock, 0, h->stream>>>(A, pop, rec, face, what, buf);
    else
        k_halo_unpack<NS9, S><<<grid_for(plane), kBlock, 0, h->stream>>>(A, pop, rec, face, what, buf);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

}  // namespace

namespace lbmh {

int mc_halo(lbmgpu *h, int face, int what, double *buf, bool pack) {
    return h->fp32 ? halo_t<float>(h, face, what, buf, pack) : halo_t<double>(h, face, what, buf, pack);
}

int mc_setup(lbmgpu *h) {
    const lbmgpu_desc &d = h->d;
    if (!valid_mc_layout(d.mix, d.spc)) return LBMGPU_E_ARG;
    h->ns = d.n_species;
    h->mech = *d.mech;
    h->nrec = mc_nrec(h->ns);
    h->chem = d.chem_mode;
    h->fp32 = d.precision == LBMGPU_FP32;
    h->U = UnitsF{d.units_m, d.units_kg, d.units_s, d.units_K};
    const lbmgpu_species_layout &s = d.spc;
    h->so = SpOff{(long)s.size, s.X, s.rho, s.f, s.fpc, s.u, s.v, s.w};
    const long nc = h->g.ncell;
    const size_t np = 27 * (size_t)(h->ns + 1);
    for (int b = 0; b < 2; ++b) {
        int rc = h->fp32 ? dalloc(h, &h->pop32[b], np * nc) : dalloc(h, &h->pop[b], np * nc);
        if (rc) return rc;
        rc = dalloc(h, &h->mom[b], (size_t)h->nrec * nc);
        if (rc) return rc;
        if (b == 0) {
            rc = dalloc(h, &h->props, (size_t)pr_count<NS9>() * nc);
            if (rc) return rc;
            rc = dalloc(h, &h->gsum, (size_t)gs_count<NS9>() * nc);
            if (rc) return rc;
        }
        // the face-difference planes of cells the kernels never write (ghosts) are read
        // but not used, and the ghosts' populations are never read; zero them all so they
        // hold no stale bits
        CK(cudaMemset(h->mom[b], 0, (size_t)h->nrec * nc * sizeof(double)));
        CK(cudaMemset(h->fp32 ? (void *)h->pop32[b] : (void *)h->pop[b], 0,
                      np * nc * (h->fp32 ? sizeof(float) : sizeof(double))));
        if (h->fp32) {
            rc = dalloc(h, &h->shift[b], np);
            if (rc) return rc;
            CK(cudaMemset(h->shift[b], 0, np * sizeof(double)));
        }
    }
    h->kin = kin_h2_air_9::matches(*d.mech) ? KIN_H2_AIR_9 : KIN_TABLES;
    gas::Tables *ht = new gas::Tables();
    gas::make_tables(*d.mech, *ht);
    set_lattice_constants(*ht, h->U);
    int rc = dalloc(h, &h->tab, 1);
    if (!rc) {
        cudaError_t e = cudaMemcpy(h->tab, ht, sizeof(gas::Tables), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = cuda_fail(e);
    }
    delete ht;
    return rc;
}

void mc_release(lbmgpu *h) {
    sur_release(h);
    if (h->tab) cudaFree(h->tab);
    h->tab = nullptr;
    cudaFree(h->props);
    h->props = nullptr;
    cudaFree(h->gsum);
    h->gsum = nullptr;
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->pop32[b]);
        cudaFree(h->bst32[b]);
        cudaFree(h->shift[b]);
        h->pop32[b] = nullptr;
        h->bst32[b] = nullptr;
        h->shift[b] = nullptr;
    }
}

// Classification of the whole lattice once every plane is on the device: fluid cells,
// the cells with a boundary upstream (compact list), the boundary store, the FP32 shift.
static int mc_finish_upload(lbmgpu *h) {
    const lbm::ScGeom &g = h->g;
    const long nc = g.ncell;
    const std::vector<int8_t> &ty = h->htype;
    std::vector<uint8_t> cf(nc, 0);
    long nfluid = 0, nb = 0;
    std::vector<int> bidh(nc, -1);
    std::vector<long> blh;
    for (int i = 0; i < g.Nx; ++i)
        for (int j = 0; j < g.Ny; ++j)
            for (int k = 0; k < g.Nz; ++k) {
                const long n = (long)i * g.si + (long)j * g.sj + k;
                if (ty[n] != T_F) continue;
                // a halo plane holds the neighbouring slab's cells: never updated here
                if ((i == 0 && h->halo_lo) || (i == g.Nx - 1 && h->halo_hi)) continue;
                if (i == 0 || j == 0 || k == 0 || i == g.Nx - 1 || j == g.Ny - 1 || k == g.Nz - 1)
                    return LBMGPU_E_ARG;
                uint8_t c = CF_FLUID;
                for (int l = 0; l < 27; ++l) {
                    const int t = ty[n - (long)cx(l) * g.si - (long)cy(l) * g.sj - cz(l)];
                    if (t != T_F && t != T_P) c |= CF_SPECIAL;
                }
                if (c & CF_SPECIAL) {
                    bidh[n] = (int)nb++;
                    blh.push_back(n);
                }
                cf[n] = c;
                ++nfluid;
            }
    // the boundary formulas read up to two cells inward along an axis
    if (nb > 0 && (g.Nx < 5 || g.Ny < 5 || g.Nz < 5)) return LBMGPU_E_UNSUPPORTED;
    h->nfluid = nfluid;
    if (nb != h->nb || !h->blist) {
        const size_t np = 27 * (size_t)(h->ns + 1), es = h->fp32 ? sizeof(float) : sizeof(double);
        for (int b = 0; b < 2; ++b) {
            void *&p = h->fp32 ? reinterpret_cast<void *&>(h->bst32[b]) : reinterpret_cast<void *&>(h->bst[b]);
            if (p) {
                cudaFree(p);
                h->bytes -= np * (size_t)std::max<long>(h->nb, 1) * es;
                p = nullptr;
            }
        }
        if (h->blist) {
            cudaFree(h->blist);
            h->bytes -= (size_t)std::max<long>(h->nb, 1) * sizeof(long);
            h->blist = nullptr;
        }
        h->nb = nb;
        for (int b = 0; b < 2; ++b) {
            const int rc = h->fp32 ? dalloc(h, &h->bst32[b], np * (size_t)std::max<long>(nb, 1))
                                   : dalloc(h, &h->bst[b], np * (size_t)std::max<long>(nb, 1));
            if (rc) return rc;
        }
        const int rc = dalloc(h, &h->blist, (size_t)std::max<long>(nb, 1));
        if (rc) return rc;
    }
    if (nb > 0) CK(cudaMemcpyAsync(h->blist, blh.data(), nb * sizeof(long), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->bid, bidh.data(), nc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->cflag, cf.data(), nc, cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    int rc = rebase_shift(h);
    if (rc) return rc;
    rc = h->fp32 ? fill_bst<float>(h) : fill_bst<double>(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    h->pack_mode = PK_UPLOADED;
    h->have_state = true;
    h->phase = PH_BOUNDARY;
    return LBMGPU_OK;
}

int mc_upload_planes(lbmgpu *h, int i0, int i1, const void *mix, const void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    const lbm::ScGeom &g = h->g;
    if (i0 < 0 || i1 > g.Nx || i0 >= i1) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const long c0 = (long)i0 * g.si, c1 = (long)i1 * g.si;
    const size_t ms = h->mo.size;
    const char *hm = static_cast<const char *>(mix);
    if ((long)h->htype.size() != g.ncell) h->htype.assign(g.ncell, 0);
    if ((int)h->plane_have.size() != g.Nx) h->plane_have.assign(g.Nx, 0);
    for (long n = c0; n < c1; ++n) {
        short t;
        std::memcpy(&t, hm + (n - c0) * ms + h->mo.type, sizeof(short));
        if (t < 0 || t > 9) return LBMGPU_E_ARG;
        if (t == T_I || t == T_O || t == T_Q) return LBMGPU_E_UNSUPPORTED;
        h->htype[n] = (int8_t)t;
    }
    // a new upload begins: the state is incomplete until every plane has arrived again
    if (h->planes_have == 0) h->have_state = false;
    CK(cudaMemcpyAsync(h->type + c0, h->htype.data() + c0, c1 - c0, cudaMemcpyHostToDevice, h->stream));
    int rc = h->fp32 ? upload_t<float>(h, hm, species, c0, c1) : upload_t<double>(h, hm, species, c0, c1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    for (int i = i0; i < i1; ++i)
        if (!h->plane_have[i]) {
            h->plane_have[i] = 1;
            ++h->planes_have;
        }
    if (h->planes_have < g.Nx) return LBMGPU_OK;
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    return mc_finish_upload(h);
}

int mc_upload(lbmgpu *h, const void *mix, const void *const *species) {
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    return mc_upload_planes(h, 0, h->g.Nx, mix, species);
}

int mc_download_planes(lbmgpu *h, int i0, int i1, void *mix, void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    if (i0 < 0 || i1 > h->g.Nx || i0 >= i1) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const long c0 = (long)i0 * h->g.si, c1 = (long)i1 * h->g.si;
    const size_t ms = h->mo.size, ss = h->so.size;
    std::vector<uint8_t> cf(c1 - c0);
    CK(cudaMemcpyAsync(cf.data(), h->cflag + c0, c1 - c0, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const bool stepped = h->pack_mode == PK_STEPPED;
    const long mfld[] = {h->mo.rho, h->mo.u, h->mo.v, h->mo.w, h->mo.p, h->mo.temp, h->mo.rhoe, h->mo.HRR};
    const long sfld[] = {h->so.X, h->so.rho, h->so.u, h->so.v, h->so.w};
    char *hm = static_cast<char *>(mix);
    for (long n0 = c0; n0 < c1; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(c1, n0 + (long)h->stage_cells), cnt = n1 - n0;
        const int rc = h->fp32 ? pack_chunk<float>(h, n0, n1, stepped) : pack_chunk<double>(h, n0, n1, stepped);
        if (rc) return rc;
        const size_t bytes = cnt * (ms + (size_t)h->ns * ss);
        CK(cudaMemcpyAsync(h->bounce, h->stage, bytes, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (long n = n0; n < n1; ++n) {
            const char *srec = h->bounce + (n - n0) * ms;
            char *drec = hm + (n - c0) * ms;
            const bool fluid = cf[n - c0] & CF_FLUID;
            if (fluid) {
                short t;
                std::memcpy(&t, drec + h->mo.type, sizeof(short));
                std::memcpy(drec, srec, ms);
                std::memcpy(drec + h->mo.type, &t, sizeof(short));
            } else {
                for (long o : mfld) std::memcpy(drec + o, srec + o, sizeof(double));
                std::memcpy(drec + h->mo.p_tensor, srec + h->mo.p_tensor, 9 * sizeof(double));
            }
            for (int a = 0; a < h->ns; ++a) {
                const char *ssrc = h->bounce + cnt * ms + ((size_t)a * cnt + (n - n0)) * ss;
                char *sdst = static_cast<char *>(species[a]) + (n - c0) * ss;
                if (fluid)
                    std::memcpy(sdst, ssrc, ss);
                else
                    for (long o : sfld) std::memcpy(sdst + o, ssrc + o, sizeof(double));
            }
        }
    }
    return LBMGPU_OK;
}

int mc_download(lbmgpu *h, void *mix, void *const *species) { return mc_download_planes(h, 0, h->g.Nx, mix, species); }

int mc_init(lbmgpu *h) {
    int rc = h->fp32 ? init_t<float>(h) : init_t<double>(h);
    if (rc) return rc;
    rc = rebase_shift(h);
    if (rc) return rc;
    rc = h->fp32 ? fill_bst<float>(h) : fill_bst<double>(h);
    if (rc) return rc;
    h->pack_mode = PK_INIT;
    return LBMGPU_OK;
}

int mc_launch_collide(lbmgpu *h) { return h->fp32 ? collide_t<float>(h) : collide_t<double>(h); }

int mc_launch_stream(lbmgpu *h) {
    const int rc = h->fp32 ? stream_t<float>(h) : stream_t<double>(h);
    if (rc) return rc;
    h->cur = 1 - h->cur;
    h->pack_mode = PK_STEPPED;
    sur_after_step(h);
    return 0;
}

}  // namespace lbmh
