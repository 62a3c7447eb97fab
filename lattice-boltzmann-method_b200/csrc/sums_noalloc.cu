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
// The scratch here is part of the library's device image, so it exists as soon as the
// module is loaded.
//
// Limits and rules:
//   - Scratch size: kSumMaxBlocks * kSumMax partials + kSumMax totals = 1184 * 21 + 21
//     doubles (199,080 bytes) per device.  The reduction grid is capped at kSumMaxBlocks
//     blocks, so every lattice fits; n_out above LBMGPU_SUMS_MAX (or below the handle's
//     lbmgpu_sums_count) is rejected with LBMGPU_E_ARG.
//   - Nothing in the scratch has to start at zero: each call's first kernel writes every
//     partial the second kernel reads, and the second writes every total the copy reads.
//   - One scratch per device per process: calls whose work overlaps on the same device
//     (two handles on different streams, or two host threads) race on it.  Callers must
//     serialise them -- one stream, or host-side ordering.
//   - The first call on each device resolves the scratch's address with
//     cudaGetSymbolAddress (with that device current); make that first call before any
//     stream capture begins.
#include <mutex>

#include "handle.cuh"
#include "sums.cuh"

static_assert(lbmh::kSumMax == LBMGPU_SUMS_MAX, "scratch sized for LBMGPU_SUMS_MAX totals");

static __device__ __align__(256) double g_sums_scratch[lbmh::kSumMaxBlocks * lbmh::kSumMax + lbmh::kSumMax];

namespace {

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Address of the device copy of g_sums_scratch on `device`, resolved once per device.
int scratch_on(int device, double **out) {
    if (device < 0 || device >= kMaxDevices) return LBMGPU_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        CK(cudaSetDevice(device));
        void *p = nullptr;
        CK(cudaGetSymbolAddress(&p, g_sums_scratch));
        g_scratch_addr[device] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[device];
    return 0;
}

}  // namespace

extern "C" int lbmgpu_sums_noalloc(lbmgpu_t *h, double *out, int n_out) {
    if (!h || !out) return LBMGPU_E_ARG;
    const int K = lbmh::sums_count(h);
    if (n_out < K || n_out > LBMGPU_SUMS_MAX) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    double *scratch = nullptr;
    int rc = scratch_on(h->d.device, &scratch);
    if (rc) return rc;
    CK(cudaSetDevice(h->d.device));
    double *out_dev = scratch + (size_t)lbmh::kSumMaxBlocks * lbmh::kSumMax;
    rc = lbmh::sums_launch(h, scratch, out_dev);
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, out_dev, K * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}
