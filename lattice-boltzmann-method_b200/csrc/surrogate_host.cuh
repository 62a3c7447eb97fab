// Host-side hooks of the chemistry surrogate (surrogate.cu) used by the multicomponent
// step (mc.cu).
#pragma once
#include "mc_cell.cuh"

struct lbmgpu;

namespace lbmh {

struct SurState;
int sur_create(lbmgpu *h);
void sur_release(lbmgpu *h);
// Fills A.sur for the collision-parameter kernel; with the surrogate on, first launches
// the feature and network kernels on the handle's stream.
template <typename S>
int sur_prepare_t(lbmgpu *h, lbm::McArgsT<S, double> &A);
// Advances the sample cursor and the step counter after a completed step.
void sur_after_step(lbmgpu *h);

}  // namespace lbmh
