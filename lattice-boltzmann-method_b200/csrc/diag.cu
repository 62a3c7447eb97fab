// lbmgpu_diagnostics: run diagnostics of the current state reduced on the device, so a
// driver can log them every step without downloading the lattice.
//
// The first three are the reference's OutputKeEns (src/output.cpp:212-275) over the fluid
// cells: the kinetic-energy sum  sum rho |u|^2  (:232-233), the enstrophy sum
// sum rho |curl u|^2  with central differences whose neighbour indices wrap inside the
// interior [1, N-2] of each axis (:235-262, the wrap test for the upper neighbour only runs
// when the lower one did not wrap, as there), and the total energy  sum rho E  (:265).
// Then the heat-release sum  sum HRR  (the per-cell field the chemistry writes,
// src/lbm-collision.cpp:395-398) and the peak and minimum temperature -- what a reacting run
// is assessed by.  All in lattice units.  Deterministic: fixed grid-strided cell sets per
// block, warp shuffles, then the blocks in order; the partials use the handle's reduction
// scratch (allocated on the first call of this or lbmgpu_sums).
#include <algorithm>
#include <cfloat>

#include "handle.cuh"
#include "mc_cell.cuh"
#include "sums.cuh"

namespace lbmh {

namespace {

using namespace lbm;

constexpr int kDiag = 6;  // LBMGPU_DIAG_COUNT
static_assert(kDiag <= kSumMax, "diagnostics partials reuse the sums scratch");

struct DiagSrc {
    const double *rec;
    const uint8_t *cflag;
    long ncell, si, sj;
    int Nx, Ny, Nz, ns;
    int halo_lo, halo_hi;  // x halo planes of a slab (lbmgpu_set_halo)
    double cv;  // single component: R / (gamma - 1)
};

// The reference's wrapped neighbours of index i on an axis of N cells (output.cpp:235-249).
__device__ __forceinline__ void wrap_nb(int i, int N, int &lo, int &hi) {
    hi = i + 1;
    lo = i - 1;
    if (lo < 1)
        lo = N - 2;
    else if (hi > N - 2)
        hi = 1;
}

__device__ __forceinline__ void cell_diag(const DiagSrc &S, long n, double *v) {
    const long nc = S.ncell;
    const double *R = S.rec;
    const double rho = R[RM_RHO * nc + n];
    const double u = R[RM_U * nc + n], w = R[RM_W * nc + n], vv = R[RM_V * nc + n];
    const double uu = u * u + vv * vv + w * w;
    v[0] = rho * uu;
    int i, j, k;
    cell_ijk(n, S.si, S.sj, i, j, k);
    int ia, ib, ja, jb, ka, kb;
    wrap_nb(i, S.Nx, ib, ia);
    if (i == 1 && S.halo_lo) ib = 0;  // an x halo plane holds the neighbouring slab's cells
    if (i == S.Nx - 2 && S.halo_hi) ia = S.Nx - 1;
    wrap_nb(j, S.Ny, jb, ja);
    wrap_nb(k, S.Nz, kb, ka);
    auto at = [&](int plane, int ii, int jj, int kk) { return R[plane * nc + (long)ii * S.si + (long)jj * S.sj + kk]; };
    const double uy = (at(RM_U, i, ja, k) - at(RM_U, i, jb, k)) / 2;
    const double uz = (at(RM_U, i, j, ka) - at(RM_U, i, j, kb)) / 2;
    const double vx = (at(RM_V, ia, j, k) - at(RM_V, ib, j, k)) / 2;
    const double vz = (at(RM_V, i, j, ka) - at(RM_V, i, j, kb)) / 2;
    const double wx = (at(RM_W, ia, j, k) - at(RM_W, ib, j, k)) / 2;
    const double wy = (at(RM_W, i, ja, k) - at(RM_W, i, jb, k)) / 2;
    const double vort = (wy - vz) * (wy - vz) + (uz - wx) * (uz - wx) + (vx - uy) * (vx - uy);
    v[1] = rho * vort;
    const double T = R[RM_T * nc + n];
    if (S.ns == 0) {  // single-component record (sc_kernels.cuh): E from T and u, no heat release
        v[2] = rho * (S.cv * T + 0.5 * uu);
        v[3] = 0.0;
    } else {
        v[2] = R[RM_RHOE * nc + n];
        v[3] = R[RM_HRR * nc + n];
    }
    v[4] = T;
    v[5] = T;
}

__device__ __forceinline__ double combine(int q, double a, double b) {
    return q == 4 ? fmax(a, b) : (q == 5 ? fmin(a, b) : a + b);
}

__global__ void __launch_bounds__(kSumBlock) k_diag_partials(DiagSrc S, double *__restrict__ partials) {
    __shared__ double warp_part[kSumBlock / 32][kDiag];
    double acc[kDiag] = {0.0, 0.0, 0.0, 0.0, -DBL_MAX, DBL_MAX}, v[kDiag];
    for (long n = (long)blockIdx.x * kSumBlock + threadIdx.x; n < S.ncell; n += (long)gridDim.x * kSumBlock) {
        if (!(S.cflag[n] & CF_FLUID)) continue;
        cell_diag(S, n, v);
#pragma unroll
        for (int q = 0; q < kDiag; ++q) acc[q] = combine(q, acc[q], v[q]);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kDiag; ++q) {
        double x = acc[q];
        for (int off = 16; off > 0; off >>= 1) x = combine(q, x, __shfl_down_sync(0xffffffffu, x, off));
        if (lane == 0) warp_part[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x < kDiag) {
        const int q = threadIdx.x;
        double x = warp_part[0][q];
        for (int w = 1; w < kSumBlock / 32; ++w) x = combine(q, x, warp_part[w][q]);
        partials[(long)blockIdx.x * kDiag + q] = x;
    }
}

__global__ void k_diag_final(const double *__restrict__ partials, int nblocks, double *__restrict__ out) {
    const int q = threadIdx.x;
    if (q >= kDiag) return;
    double x = partials[q];
    for (int b = 1; b < nblocks; ++b) x = combine(q, x, partials[(long)b * kDiag + q]);
    out[q] = x;
}

}  // namespace

}  // namespace lbmh

using namespace lbmh;

extern "C" {

int lbmgpu_diagnostics(lbmgpu_t *h, double *out, int n_out) {
    if (!h || !out) return LBMGPU_E_ARG;
    if (n_out < kDiag) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    CK(cudaSetDevice(h->d.device));
    if (!h->sum_scratch) {  // shared with lbmgpu_sums: partials of every block, then the totals
        const int rc = dalloc(h, &h->sum_scratch, (size_t)kSumMaxBlocks * kSumMax + kSumMax);
        if (rc) return rc;
    }
    DiagSrc S;
    S.rec = h->mom[h->cur];
    S.cflag = h->cflag;
    S.ncell = h->g.ncell;
    S.Nx = h->g.Nx;
    S.halo_lo = h->halo_lo;
    S.halo_hi = h->halo_hi;
    S.Ny = h->g.Ny;
    S.Nz = h->g.Nz;
    S.sj = h->g.sj;
    S.si = h->g.si;
    S.ns = h->ns;
    S.cv = h->P.cv;
    const int G = sums_grid(h);
    double *out_dev = h->sum_scratch + (size_t)kSumMaxBlocks * kSumMax;
    k_diag_partials<<<G, kSumBlock, 0, h->stream>>>(S, h->sum_scratch);
    CK(cudaGetLastError());
    k_diag_final<<<1, 32, 0, h->stream>>>(h->sum_scratch, G, out_dev);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, out_dev, kDiag * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

}  // extern "C"
