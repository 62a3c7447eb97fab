// Shared constants and host helpers of the conserved-sums reduction (sums.cu).
#pragma once

#include "../../include/lbmgpu.h"

struct lbmgpu;

namespace lbmh {

constexpr int kSumBlock = 256;              // threads per block of the partials kernel
constexpr int kSumMaxBlocks = 148 * 8;      // grid cap: 8 blocks per SM of a B200
constexpr int kSumElements = LBMGPU_MAX_ELEMENTS;  // H, O, N, Ar, C (lbmgpu_mech.elements)
constexpr int kSumMax = 5 + 12 + kSumElements;  // LBMGPU_SUMS_MAX

int sums_count(const lbmgpu *h);
int sums_grid(const lbmgpu *h);
// Enqueues both kernels on the handle's stream: block partials into `partials`
// (sums_grid(h) * sums_count(h) doubles), the totals into out_dev.
int sums_launch(lbmgpu *h, double *partials, double *out_dev);
// Loads the module holding the two reduction kernels on the current device (under lazy
// module loading it would otherwise load, and allocate its code, at the first launch).
int sums_preload();
// Resolves the fixed scratch of lbmgpu_sums_noalloc on the current device (sums_noalloc.cu):
// loads its module so that no later call allocates.  Called at handle creation.
int noalloc_prepare();

}  // namespace lbmh
