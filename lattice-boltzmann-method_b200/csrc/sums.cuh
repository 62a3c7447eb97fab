// Shared constants and host helpers of the conserved-sums reduction (sums.cu).
#pragma once

struct lbmgpu;

namespace lbmh {

constexpr int kSumBlock = 256;              // threads per block of the partials kernel
constexpr int kSumMaxBlocks = 148 * 8;      // grid cap: 8 blocks per SM of a B200
constexpr int kSumElements = 4;             // H, O, N, Ar (lbmgpu_mech.elements)
constexpr int kSumMax = 5 + 12 + kSumElements;  // LBMGPU_SUMS_MAX

int sums_count(const lbmgpu *h);
int sums_grid(const lbmgpu *h);
// Enqueues both kernels on the handle's stream: block partials into `partials`
// (sums_grid(h) * sums_count(h) doubles), the totals into out_dev.
int sums_launch(lbmgpu *h, double *partials, double *out_dev);

}  // namespace lbmh
