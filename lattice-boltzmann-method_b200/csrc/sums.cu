// lbmgpu_sums: FP64 totals of the conserved quantities over the fluid cells of the
// current state -- the global mass, momentum and energy sums (and, multicomponent, the
// species masses and the element totals) that the reference's diagnostics reduce on the
// host (OutputKeEns, src/output.cpp) and that conservation checks need every few steps.
//
// Two kernels, deterministic: each block of the first reduces a fixed, grid-strided set of
// cells (warp shuffles, then the warps in order) into its slot of a partials buffer; one
// block of the second adds the partials in block order.  The partials buffer is device
// scratch owned by the handle, allocated on the first call.
#include <algorithm>

#include "handle.cuh"
#include "mc_cell.cuh"
#include "sums.cuh"

namespace lbmh {

namespace {

using namespace lbm;

// Values of cell n, in the order of the output: mass, momentum (3), total energy, then
// (multicomponent) the species masses and the element totals.
struct SumSrc {
    const double *rec;
    const uint8_t *cflag;
    const gas::Tables *tab;  // multicomponent, else null
    long ncell;
    int ns, nsum;
    double cv;               // single component: R / (gamma - 1)
};

__device__ __forceinline__ void cell_values(const SumSrc &S, long n, double *v) {
    const long nc = S.ncell;
    if (S.ns == 0) {  // single-component record (sc_kernels.cuh)
        const double rho = S.rec[M_RHO * nc + n];
        const double u = S.rec[M_U * nc + n], w_ = S.rec[M_W * nc + n], vv = S.rec[M_V * nc + n];
        v[0] = rho;
        v[1] = rho * u;
        v[2] = rho * vv;
        v[3] = rho * w_;
        v[4] = rho * (S.cv * S.rec[M_T * nc + n] + 0.5 * (u * u + vv * vv + w_ * w_));
        return;
    }
    const double rho = S.rec[RM_RHO * nc + n];
    v[0] = rho;
    v[1] = rho * S.rec[RM_U * nc + n];
    v[2] = rho * S.rec[RM_V * nc + n];
    v[3] = rho * S.rec[RM_W * nc + n];
    v[4] = S.rec[RM_RHOE * nc + n];
    for (int e = 0; e < kSumElements; ++e) v[5 + S.ns + e] = 0.0;
    for (int a = 0; a < S.ns; ++a) {
        const double ra = S.rec[(long)rs(a, RS_RHO) * nc + n];
        v[5 + a] = ra;
        const double mol = ra / S.tab->m.W[a];
        for (int e = 0; e < kSumElements; ++e) v[5 + S.ns + e] += mol * S.tab->m.elements[a][e];
    }
}

__global__ void __launch_bounds__(kSumBlock) k_sum_partials(SumSrc S, double *__restrict__ partials) {
    __shared__ double warp_part[kSumBlock / 32][kSumMax];
    double acc[kSumMax], v[kSumMax];
    for (int k = 0; k < kSumMax; ++k) acc[k] = 0.0;
    for (long n = (long)blockIdx.x * kSumBlock + threadIdx.x; n < S.ncell; n += (long)gridDim.x * kSumBlock) {
        if (!(S.cflag[n] & CF_FLUID)) continue;
        cell_values(S, n, v);
        for (int k = 0; k < S.nsum; ++k) acc[k] += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < S.nsum; ++k) {
        double x = acc[k];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) warp_part[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < S.nsum) {
        double x = 0.0;
        for (int w = 0; w < kSumBlock / 32; ++w) x += warp_part[w][threadIdx.x];
        partials[(long)blockIdx.x * S.nsum + threadIdx.x] = x;
    }
}

__global__ void k_sum_final(const double *__restrict__ partials, int nblocks, int nsum, double *__restrict__ out) {
    const int k = threadIdx.x;
    if (k >= nsum) return;
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b) x += partials[(long)b * nsum + k];
    out[k] = x;
}

}  // namespace

int sums_count(const lbmgpu *h) { return h->ns > 0 ? 5 + h->ns + kSumElements : 5; }

int sums_preload() {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, k_sum_partials));
    CK(cudaFuncGetAttributes(&fa, k_sum_final));
    return 0;
}

int sums_grid(const lbmgpu *h) {
    return (int)std::max<long>(1, std::min<long>((h->g.ncell + kSumBlock - 1) / kSumBlock, kSumMaxBlocks));
}

int sums_launch(lbmgpu *h, double *partials, double *out_dev) {
    SumSrc S;
    S.rec = h->mom[h->cur];
    S.cflag = h->cflag;
    S.tab = h->ns > 0 ? h->tab : nullptr;
    S.ncell = h->g.ncell;
    S.ns = h->ns;
    S.nsum = sums_count(h);
    S.cv = h->P.cv;
    const int G = sums_grid(h);
    k_sum_partials<<<G, kSumBlock, 0, h->stream>>>(S, partials);
    CK(cudaGetLastError());
    k_sum_final<<<1, 32, 0, h->stream>>>(partials, G, S.nsum, out_dev);
    CK(cudaGetLastError());
    return 0;
}

}  // namespace lbmh

using namespace lbmh;

extern "C" {

int lbmgpu_sums_count(const lbmgpu_t *h) { return h ? sums_count(h) : LBMGPU_E_ARG; }

int lbmgpu_sums(lbmgpu_t *h, double *out, int n_out) {
    if (!h || !out) return LBMGPU_E_ARG;
    const int K = sums_count(h);
    if (n_out < K) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    CK(cudaSetDevice(h->d.device));
    if (!h->sum_scratch) {  // partials of every block, then the K totals
        const int rc = dalloc(h, &h->sum_scratch, (size_t)kSumMaxBlocks * kSumMax + kSumMax);
        if (rc) return rc;
    }
    double *out_dev = h->sum_scratch + (size_t)kSumMaxBlocks * kSumMax;
    const int rc = sums_launch(h, h->sum_scratch, out_dev);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, out_dev, K * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

}  // extern "C"
