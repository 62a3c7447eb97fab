// Multicomponent launch plumbing shared by the handle operations (mc.cu) and the kernel
// instances for each species count (mc_kernels.cuh, instantiated in mc_ns<N>.cu): the
// kernel arguments of a handle, its population buffers by storage type, and McOps<NS>, the
// launches of one species count.  mc_by_ns dispatches a handle to the instance for its
// species count: the mechanisms the reference ships have 9 (H2/O2/N2, from nh3.yaml) and 6
// species (the two-step CH4_2S.yaml and propane_mech.yaml).
#pragma once
#include <type_traits>

#include "handle.cuh"
#include "mc_cell.cuh"

namespace lbmh {

template <typename S>
lbm::McArgsT<S, double> base_args(lbmgpu *h) {
    lbm::McArgsT<S, double> A{};
    A.Nx = h->g.Nx;
    A.halo_lo = h->halo_lo;
    A.halo_hi = h->halo_hi;
    A.Nx_glob = h->nx_glob > 0 ? h->nx_glob : h->g.Nx;
    A.Ny = h->g.Ny;
    A.Nz = h->g.Nz;
    A.ncell = h->g.ncell;
    A.sj = h->g.sj;
    A.si = h->g.si;
    A.ns = h->ns;
    A.dt = h->d.dt_sim;
    A.chem = h->chem;
    A.U = h->U;
    A.tab = h->tab;
    A.type = h->type;
    A.cflag = h->cflag;
    A.status = h->status;
    A.shift = h->fp32 ? h->shift[0] : nullptr;
    A.bid = h->bid;
    A.nb = h->nb;
    A.props = h->props;
    return A;
}

// The two storage types' buffers behind one accessor.
template <typename S>
S *popb(lbmgpu *h, int b) {
    if constexpr (std::is_same_v<S, float>)
        return h->pop32[b];
    else
        return h->pop[b];
}
template <typename S>
S *bstb(lbmgpu *h, int b) {
    if constexpr (std::is_same_v<S, float>)
        return h->bst32[b];
    else
        return h->bst[b];
}

// The launches of one species count (both storage types).
template <int NS>
struct McOps {
    // the records of cells [c0, c1) (the caller's arrays start at cell c0) into the state
    static int upload(lbmgpu *h, const char *hm, const void *const *species, long c0, long c1);
    // cells [n0, n1) into the staging buffer in the caller's record layout
    static int pack(lbmgpu *h, long n0, long n1, bool stepped);
    static int init(lbmgpu *h);
    static int collide(lbmgpu *h);
    static int stream(lbmgpu *h);
    static int halo(lbmgpu *h, int face, int what, double *buf, bool pack);
    static constexpr int props_planes() { return lbm::pr_count<NS>(); }
    static constexpr int gsum_planes() { return lbm::gs_count<NS>(); }
};
extern template struct McOps<9>;
extern template struct McOps<6>;

// f(McOps<ns>{}) for the species counts the kernels are built for; LBMGPU_E_UNSUPPORTED
// for any other.
constexpr bool mc_ns_built(int ns) { return ns == 9 || ns == 6; }
template <class F>
int mc_by_ns(int ns, F &&f) {
    switch (ns) {
    case 9:
        return f(McOps<9>{});
    case 6:
        return f(McOps<6>{});
    default:
        return LBMGPU_E_UNSUPPORTED;
    }
}

}  // namespace lbmh
