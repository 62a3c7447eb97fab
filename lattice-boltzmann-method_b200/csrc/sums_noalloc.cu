// lbmgpu_sums_noalloc: lbmgpu_sums (sums.cu) with its reduction scratch in a fixed
// file-scope device array instead of handle memory, so the call allocates nothing.
//
// Why: lbmgpu_sums allocates its scratch with cudaMalloc on its first call.  Some callers
// cannot allocate at that point:
//   - a run whose lattice was sized to fill the device's memory: the conservation check
//     added afterwards finds no room for even a small cudaMalloc;
//   - a monitoring loop that reads the totals between steps while other streams on the
//     device are busy: cudaMalloc / cudaFree synchronise the whole device and would stall
//     that work;
//   - a host that hands all device memory to its own pool after setup and forbids further
//     runtime allocation.
// The scratch is a file-scope __device__ array of the library.  Under CUDA's lazy module
// loading (the default) the module holding it -- and the module holding the reduction
// kernels -- would load at first use and allocate their code and data then; so every
// lbmgpu_create loads both on its device (noalloc_prepare, sums_preload), while allocation
// is still allowed, and no later call of this entry point allocates.
//
// Limits and rules:
//   - Scratch size: kSumMaxBlocks * kSumMax partials + kSumMax totals = 1184 * 22 + 22
//     doubles (208,560 bytes) per device, held from the first handle's creation on that
//     device until the process exits.  The reduction grid is capped at kSumMaxBlocks
//     blocks, so every lattice fits; n_out above LBMGPU_SUMS_MAX (or below the handle's
//     lbmgpu_sums_count) is rejected with LBMGPU_E_ARG.
//   - Nothing in the scratch has to start at zero: each call's first kernel writes every
//     partial the second kernel reads, and the second writes every total the copy reads.
//   - One scratch per device per process: calls whose work overlaps on the same device
//     (two handles on different streams, or two host threads) race on it.  Callers must
//     serialise them -- one stream, or host-side ordering.
//   - Each call looks the scratch's address up again (cudaGetSymbolAddress on the loaded
//     module does not allocate), so no address outlives the context it belongs to.  A
//     cudaDeviceReset destroys the context together with every handle's memory; handles
//     created after it prepare the new context the same way.
#include "handle.cuh"
#include "sums.cuh"

static_assert(lbmh::kSumMax == LBMGPU_SUMS_MAX, "scratch sized for LBMGPU_SUMS_MAX totals");

static __device__ __align__(256) double g_sums_scratch[lbmh::kSumMaxBlocks * lbmh::kSumMax + lbmh::kSumMax];

namespace lbmh {

int noalloc_prepare() {
    void *p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_sums_scratch));
    return 0;
}

}  // namespace lbmh

extern "C" int lbmgpu_sums_noalloc(lbmgpu_t *h, double *out, int n_out) {
    if (!h || !out) return LBMGPU_E_ARG;
    const int K = lbmh::sums_count(h);
    if (n_out < K || n_out > LBMGPU_SUMS_MAX) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    CK(cudaSetDevice(h->d.device));
    void *p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_sums_scratch));
    double *scratch = static_cast<double *>(p);
    double *out_dev = scratch + (size_t)lbmh::kSumMaxBlocks * lbmh::kSumMax;
    const int rc = lbmh::sums_launch(h, scratch, out_dev);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, out_dev, K * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}
