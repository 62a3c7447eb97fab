// The multicomponent kernels and launches for 6 species (mc_kernels.cuh).
#include "mc_kernels.cuh"

template struct lbmh::McOps<6>;
