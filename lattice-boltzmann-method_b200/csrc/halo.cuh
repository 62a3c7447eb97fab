// Slab decomposition along x (multi-GPU): what crosses a slab face each time step, per cell
// of the face plane.  Host/device functions -- the device kernels (halo.cu) and the host
// build of the tests call the same code.
//
// A slab's lattice holds its own x-planes 1 .. Nx-2 and, where lbmgpu_set_halo marks them,
// halo planes 0 and Nx-1 that hold the neighbouring slab's edge plane (the global
// periodic ghost planes of the decomposed domain become halos too: the first and the last
// slab exchange with each other).  Two exchanges per step keep every halo as the single
// domain would see that plane:
//   * after the collision, the post-collision populations the next stream pulls across the
//     face: the low halo (plane 0) needs the 9 directions with c_x = +1 of the lower
//     neighbour's last plane, the high halo (plane Nx-1) the 9 with c_x = -1 of the upper
//     neighbour's first plane -- 9 (NS + 1) values per face cell;
//   * after the moments, the whole per-cell record of the edge plane (the neighbours' face
//     terms, densities and states the FD stencils and boundary formulas read).
// Buffers are FP64, plane-major: value q of face cell jk (jk = j Nz + k) at q * Ny Nz + jk;
// populations decoded (value + shift in the FP32 storage mode) so slabs need not share a
// shift.  Pack face 0 sends plane 1 to the lower neighbour (its face 1), pack face 1 sends
// plane Nx-2 to the upper neighbour (its face 0).
#pragma once
#include "mc_cell.cuh"

namespace lbm {

enum : int { HALO_POPULATIONS = 0, HALO_RECORD = 1 };

// the m-th (m = 0..8) direction with c_x == cxs, in direction order
MC_HD int halo_dir(int cxs, int m) {
    int c = 0;
    for (int l = 0; l < 27; ++l)
        if (cx(l) == cxs) {
            if (c == m) return l;
            ++c;
        }
    return -1;
}

// values per face cell of one exchange
MC_HD int halo_values(int what, int ns) { return what == HALO_POPULATIONS ? 9 * (ns + 1) : mc_nrec(ns); }

// pack: plane 1 (face 0) or Nx-2 (face 1); the populations leaving through that face
template <int NS, class AT>
MC_HD void halo_pack_cell(const AT &A, const typename AT::P *pop, const typename AT::R *recb, int face, int what,
                          long jk, double *buf) {
    const long plane = (long)A.Ny * A.Nz;
    const long n = (long)(face == 0 ? 1 : A.Nx - 2) * A.si + jk;
    if (what == HALO_POPULATIONS) {
        const int cxs = face == 0 ? -1 : 1;
        for (int s = 0; s <= NS; ++s)
            for (int m = 0; m < 9; ++m)
                buf[(long)(9 * s + m) * plane + jk] = ldpop(A, pop, 27 * s + halo_dir(cxs, m), n);
    } else {
        for (int q = 0; q < mc_nrec(NS); ++q) buf[(long)q * plane + jk] = rec(A, recb, q, n);
    }
}

// unpack into the halo plane 0 (face 0) or Nx-1 (face 1): the populations entering
// through that face
template <int NS, class AT>
MC_HD void halo_unpack_cell(const AT &A, typename AT::P *pop, typename AT::R *recp, int face, int what, long jk,
                            const double *buf) {
    const long plane = (long)A.Ny * A.Nz;
    const long n = (long)(face == 0 ? 0 : A.Nx - 1) * A.si + jk;
    if (what == HALO_POPULATIONS) {
        const int cxs = face == 0 ? 1 : -1;
        for (int s = 0; s <= NS; ++s)
            for (int m = 0; m < 9; ++m) stpop(A, pop, 27 * s + halo_dir(cxs, m), n, buf[(long)(9 * s + m) * plane + jk]);
    } else {
        for (int q = 0; q < mc_nrec(NS); ++q) put(A, recp, q, n, buf[(long)q * plane + jk]);
    }
}

}  // namespace lbm
