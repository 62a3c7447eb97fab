// The multicomponent kernels and launches for 9 species (mc_kernels.cuh).
#include "mc_kernels.cuh"

template struct lbmh::McOps<9>;
