// lbmgpu, multicomponent path: the device kernels around the per-cell functions of
// mc_cell.cuh and their launches, for one species count NS (McOps<NS>, instantiated in
// mc_ns<NS>.cu; the handle operations that dispatch to them are in mc.cu).
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
#pragma once
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "halo.cuh"
#include "handle.cuh"
#include "mc_bc.cuh"
#include "mc_cell.cuh"
#include "mc_ops.cuh"
#include "surrogate_host.cuh"

namespace {

using namespace lbm;
using namespace lbmh;

// collision parameters of every fluid cell, one instance per chemistry mode; three blocks per
// SM (168 registers).  FP32 storage: the transport runs in FP32 with its species loops
// unrolled, so its per-species arrays live in registers (at 128 registers, four blocks per SM,
// they spilled: 2.00 ms against 1.21 ms at 128^3)
template <int NS, int CHEM, typename S>
__global__ void __launch_bounds__(kBlock, 3) k_mc_props(McArgsT<S, double> A) {
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
// The stiff integrator's iteration matrix in shared memory, m^2 doubles per thread of a block
// (kernels over a compiled mechanism; m the unknowns of its iteration system, gas::SysMap: 9
// for the H2/air mechanism, whose N2 is inert): two blocks of 128 threads per SM hold 162 kB,
// where the thread's own array would live in local memory (its pivoted rows are indexed at
// run time) and spill through L2; what the blocks leave of the SM's 256 kB serves as L1.
constexpr bool kChemSharedMat = true;
template <int NS, class KIN>
constexpr size_t chem_smem_bytes() {
    constexpr size_t m = gas::SysMap<KIN, NS + 1>::size;
    return kChemSharedMat ? m * m * kBlock * sizeof(double) : 0;
}
constexpr unsigned kChemShortList = 5000;
template <int NS, int G, typename S, class KIN, bool SMAT = false>
__device__ __forceinline__ void chem_list_groups(const McArgsT<S, double> &A, unsigned cnt) {
    const unsigned groups = gridDim.x * blockDim.x / G;
    for (unsigned i = (blockIdx.x * blockDim.x + threadIdx.x) / G; i < cnt; i += groups) {
        const long n = A.sur.ilist[i];
        double rho, rho_a[NS], Y[NS], T_si, rho_si, P_si;
        mc_chem_state<NS>(A, n, rho, rho_a, Y, T_si, rho_si, P_si);
        mc_chem_ros2<NS, McArgsT<S, double>, true, G, KIN, SMAT>(A, n, rho, rho_a, Y, T_si, rho_si, P_si, false);
    }
}
// With a compiled mechanism (KIN: analytic species Jacobian, two right-hand sides per
// sub-step besides it) a cell is one lane's work, its iteration matrix in shared memory as in
// k_mc_chem (launched with chem_smem_bytes).
template <int NS, typename S, class KIN = void>
__global__ void __launch_bounds__(kBlock, 2) k_mc_chem_list(McArgsT<S, double> A) {
    const unsigned cnt = *A.sur.icount;
    if constexpr (!std::is_void_v<KIN>)
        chem_list_groups<NS, 1, S, KIN, kChemSharedMat>(A, cnt);
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
// time (ros2_advance_k) so that they stay in registers, two blocks per SM.  KIN: the compiled
// kinetics of the handle's mechanism (gen_kinetics.py), void for the tables; with it the
// iteration matrix of each thread lives in shared memory (kChemSharedMat), otherwise in the
// thread's local memory.
// The surrogate's instance (SUR: no integrator in it) holds far less per thread and runs four
// blocks per SM.
// PRED false: launched only while the surrogate's predictions are not in use (mode != 1).
template <int NS, bool SUR, typename S, class KIN = void, bool PRED = true>
__global__ void __launch_bounds__(kBlock, SUR ? 4 : 2) k_mc_chem(McArgsT<S, double> A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || !(A.cflag[n] & CF_FLUID)) return;
    double rho, rho_a[NS], Y[NS], T_si, rho_si, P_si;
    mc_chem_state<NS>(A, n, rho, rho_a, Y, T_si, rho_si, P_si);
    constexpr bool smat = kChemSharedMat && !std::is_void_v<KIN>;
    mc_chem_ros2<NS, McArgsT<S, double>, !SUR, 1, KIN, smat, PRED>(A, n, rho, rho_a, Y, T_si, rho_si, P_si, SUR);
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

// The stiff chemistry over the compiled kinetics of the handle's mechanism, where the library
// has them for it (kinetics_h2_air_9.cuh): every cell (k_mc_chem) or the integrator list
// (k_mc_chem_list).  Returns false when the handle's mechanism is not compiled.
template <int NS, typename S>
bool launch_compiled_chem(lbmgpu *h, const McArgsT<S, double> &A, unsigned grid, bool list) {
    if constexpr (NS == kin_h2_air_9::NS) {
        using KinH2 = kin_h2_air_9::Kinetics;
        if (h->kin != KIN_H2_AIR_9) return false;
        constexpr size_t sm = chem_smem_bytes<NS, KinH2>();
        // the launches below report a refused attribute as a launch error
        if (list) {
            if (sm > 48 * 1024)
                (void)cudaFuncSetAttribute(k_mc_chem_list<NS, S, KinH2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sm);
            k_mc_chem_list<NS, S, KinH2><<<grid, kBlock, sm, h->stream>>>(A);
        } else if (A.sur.mode == 1) {
            if (sm > 48 * 1024)
                (void)cudaFuncSetAttribute(k_mc_chem<NS, false, S, KinH2>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_mc_chem<NS, false, S, KinH2><<<grid, kBlock, sm, h->stream>>>(A);
        } else {
            if (sm > 48 * 1024)
                (void)cudaFuncSetAttribute(k_mc_chem<NS, false, S, KinH2, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            k_mc_chem<NS, false, S, KinH2, false><<<grid, kBlock, sm, h->stream>>>(A);
        }
        return true;
    }
    return false;
}

// The records of cells [c0, c1) -- the caller's arrays start at cell c0 -- into the device
// state, one staging chunk at a time.
template <int NS, typename S>
int upload_t(lbmgpu *h, const char *hm, const void *const *species, long c0, long c1) {
    const size_t ms = h->mo.size, ss = h->so.size;
    McArgsT<S, double> A = base_args<S>(h);
    // pageable caller memory goes through the pinned bounce buffer, filled by host threads
    // (a copy from pageable memory would otherwise be staged by the driver, one thread);
    // page-locked caller memory is copied directly
    bool pinned = host_pinned(hm);
    for (int a = 0; a < h->ns; ++a) pinned = pinned && host_pinned(species[a]);
    for (long n0 = c0; n0 < c1; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(c1, n0 + (long)h->stage_cells), cnt = n1 - n0;
        if (pinned) {
            CK(cudaMemcpyAsync(h->stage, hm + (n0 - c0) * ms, cnt * ms, cudaMemcpyHostToDevice, h->stream));
            for (int a = 0; a < h->ns; ++a)
                CK(cudaMemcpyAsync(h->stage + cnt * ms + (size_t)a * cnt * ss,
                                   static_cast<const char *>(species[a]) + (n0 - c0) * ss, cnt * ss,
                                   cudaMemcpyHostToDevice, h->stream));
        } else {
            CK(cudaStreamSynchronize(h->stream));  // the bounce buffer's previous chunk has gone
            const long nb = (long)h->ns + 1;       // the mixture block, then each species' block
            host_parallel_for(nb * 64, [&](long lo, long hi) {
                for (long q = lo; q < hi; ++q) {
                    const long blk = q / 64, part = q % 64;
                    const size_t sz = blk == 0 ? ms : ss;
                    const char *src = blk == 0 ? hm : static_cast<const char *>(species[blk - 1]);
                    char *dst = h->bounce + (blk == 0 ? 0 : cnt * ms + (size_t)(blk - 1) * cnt * ss);
                    const long r0 = cnt * part / 64, r1 = cnt * (part + 1) / 64;
                    std::memcpy(dst + r0 * sz, src + (n0 - c0 + r0) * sz, (r1 - r0) * sz);
                }
            }, 1);
            CK(cudaMemcpyAsync(h->stage, h->bounce, cnt * (ms + (size_t)h->ns * ss), cudaMemcpyHostToDevice,
                               h->stream));
        }
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        k_mc_unpack<NS, S><<<grid_for(cnt), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[0],
                                                                     h->mom[1], popb<S>(h, 0), popb<S>(h, 1));
        ev_end(h, ep);
        CK(cudaGetLastError());
    }
    return 0;
}

template <int NS, typename S>
int pack_chunk(lbmgpu *h, long n0, long n1, bool stepped) {
    McArgsT<S, double> A = base_args<S>(h);
    const int c = h->cur;
    const S *pc = stepped ? popb<S>(h, c) : popb<S>(h, 1 - c);
    // the records' padding bytes come out as zeros, not as what the staging held before
    CK(cudaMemsetAsync(h->stage, 0, (size_t)(n1 - n0) * (h->mo.size + (size_t)h->ns * h->so.size), h->stream));
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_mc_pack<NS, S><<<grid_for(n1 - n0), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[c],
                                                                   popb<S>(h, c), pc, bstb<S>(h, c), stepped ? 1 : 0);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

template <int NS, typename S>
int init_t(lbmgpu *h) {
    McArgsT<S, double> A = base_args<S>(h);
    const int c = h->cur;
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_mc_init<NS, S><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A, h->mom[c], h->mom[1 - c],
                                                                      popb<S>(h, c));
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

template <int NS, typename S>
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
        k_mc_props<NS, CHEM_REF_EXPLICIT, S><<<gp, kBlock, 0, h->stream>>>(A);
    else
        k_mc_props<NS, CHEM_OFF, S><<<gp, kBlock, 0, h->stream>>>(A);  // ROS2 / surrogate: k_mc_chem
    ev_end(h, ep);
    CK(cudaGetLastError());
    if (h->chem == CHEM_ROSENBROCK) {
        EvPair ec{};
        ev_begin(h, K_CHEM, ec);
        if (A.sur.mode == 1 && A.sur.ilist)
            k_mc_chem<NS, true, S><<<gp, kBlock, 0, h->stream>>>(A);
        else if (!launch_compiled_chem<NS, S>(h, A, gp, false))
            k_mc_chem<NS, false, S><<<gp, kBlock, 0, h->stream>>>(A);
        ev_end(h, ec);
        CK(cudaGetLastError());
    }
    if (A.sur.ilist) {
        EvPair ei{};
        ev_begin(h, K_SURROGATE, ei);
        if (!launch_compiled_chem<NS, S>(h, A, 148 * 8, true))
            k_mc_chem_list<NS, S><<<148 * 8, kBlock, 0, h->stream>>>(A);
        ev_end(h, ei);
        CK(cudaGetLastError());
    }
    EvPair ee{};
    ev_begin(h, K_EFLUX, ee);
    k_mc_eflux<NS, S><<<gp, kBlock, 0, h->stream>>>(A);
    ev_end(h, ee);
    CK(cudaGetLastError());
    EvPair er{};
    ev_begin(h, K_COLLIDE, er);
    k_mc_relax<NS, S><<<dim3(grid_for(h->g.ncell), NS + 1), kBlock, 0, h->stream>>>(A);
    ev_end(h, er);
    CK(cudaGetLastError());
    return 0;
}

template <int NS, typename S>
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
        k_mc_special<NS, S><<<(unsigned)((h->nb + 31) / 32), 32, 0, h->side>>>(B, h->blist);
        ev_end(h, eb, h->side);
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->join, h->side));
    }
    EvPair ep{};
    ev_begin(h, K_STREAM_MOMENT, ep);
    k_mc_gather<NS, S><<<dim3(grid_for(h->g.ncell), NS + 1), kBlock, 0, h->stream>>>(A, h->gsum);
    ev_end(h, ep);
    CK(cudaGetLastError());
    EvPair es{};
    ev_begin(h, K_SOLVE, es);
    k_mc_solve<NS, S><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A, h->gsum);
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
template <int NS, typename S>
int halo_t(lbmgpu *h, int face, int what, double *buf, bool pack) {
    McArgsT<S, double> A = base_args<S>(h);
    S *pop = popb<S>(h, 1 - h->cur);
    double *rec = h->mom[h->cur];
    const long plane = (long)h->g.Ny * h->g.Nz;
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    if (pack)
        k_halo_pack<NS, S><<<grid_for(plane), kBlock, 0, h->stream>>>(A, pop, rec, face, what, buf);
    else
        k_halo_unpack<NS, S><<<grid_for(plane), kBlock, 0, h->stream>>>(A, pop, rec, face, what, buf);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

}  // namespace

namespace lbmh {

template <int NS>
int McOps<NS>::upload(lbmgpu *h, const char *hm, const void *const *species, long c0, long c1) {
    return h->fp32 ? upload_t<NS, float>(h, hm, species, c0, c1) : upload_t<NS, double>(h, hm, species, c0, c1);
}
template <int NS>
int McOps<NS>::pack(lbmgpu *h, long n0, long n1, bool stepped) {
    return h->fp32 ? pack_chunk<NS, float>(h, n0, n1, stepped) : pack_chunk<NS, double>(h, n0, n1, stepped);
}
template <int NS>
int McOps<NS>::init(lbmgpu *h) {
    return h->fp32 ? init_t<NS, float>(h) : init_t<NS, double>(h);
}
template <int NS>
int McOps<NS>::collide(lbmgpu *h) {
    return h->fp32 ? collide_t<NS, float>(h) : collide_t<NS, double>(h);
}
template <int NS>
int McOps<NS>::stream(lbmgpu *h) {
    return h->fp32 ? stream_t<NS, float>(h) : stream_t<NS, double>(h);
}
template <int NS>
int McOps<NS>::halo(lbmgpu *h, int face, int what, double *buf, bool pack) {
    return h->fp32 ? halo_t<NS, float>(h, face, what, buf, pack) : halo_t<NS, double>(h, face, what, buf, pack);
}

}  // namespace lbmh
