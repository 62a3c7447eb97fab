// D3Q27 lattice constants and the per-axis factorised equilibria shared by all kernels.
#pragma once
#include <cstdint>

// The per-cell functions are also built for the host (tests); there the CUDA execution
// space qualifiers are empty.
#if !defined(__CUDACC__) && !defined(__host__)
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace lbm {

// Cell-type codes, identical to the reference's (src/headers/defines.hpp:140-149): the
// caller's cell arrays carry them unchanged.
enum CellType : int {
    T_F = 0, T_S = 1, T_P = 2, T_A = 3, T_FS = 4, T_I = 5, T_O = 6, T_I_C = 7, T_O_C = 8, T_Q = 9
};

// Lattice indices (i, j, k) of cell n = i si + j sj + k with sj = Nz, si = Ny Nz.
// lbmgpu_create admits lattices of fewer than 2^31 cells, so 32-bit unsigned division
// gives the same integers as 64-bit division at a fraction of its cost.
__host__ __device__ __forceinline__ void cell_ijk(long n, long si, long sj, int &i, int &j, int &k) {
    const unsigned u = (unsigned)n, usi = (unsigned)si, usj = (unsigned)sj;
    const unsigned ui = u / usi, r = u - ui * usi, uj = r / usj;
    i = (int)ui;
    j = (int)uj;
    k = (int)(r - uj * usj);
}

// Per-cell flags of the device's cell classification: a fluid cell, and one with a
// boundary cell (anything but fluid or a periodic ghost) upstream along some direction.
enum : uint8_t { CF_FLUID = 1, CF_SPECIAL = 2 };

// Direction l of the reference's D3Q27 ordering (src/headers/lbm.hpp:49-53), packed two
// bits per axis (0 -> 0, 1 -> +1, 2 -> -1), x in bits 0-1, y in 2-3, z in 4-5.  All loops
// over l are unrolled, so these fold to immediates.
__host__ __device__ constexpr uint8_t dir_code(int l) {
    constexpr uint8_t code[27] = {
        0x00, 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x05, 0x0A, 0x11, 0x22, 0x14, 0x28, 0x09,
        0x06, 0x21, 0x12, 0x24, 0x18, 0x15, 0x2A, 0x25, 0x1A, 0x19, 0x26, 0x16, 0x29};
    return code[l];
}
__host__ __device__ constexpr int dec2(int b) { return b == 1 ? 1 : (b == 2 ? -1 : 0); }
__host__ __device__ constexpr int cx(int l) { return dec2(dir_code(l) & 3); }
__host__ __device__ constexpr int cy(int l) { return dec2((dir_code(l) >> 2) & 3); }
__host__ __device__ constexpr int cz(int l) { return dec2((dir_code(l) >> 4) & 3); }
__host__ __device__ constexpr int csq(int l) { return cx(l) * cx(l) + cy(l) * cy(l) + cz(l) * cz(l); }
__host__ __device__ constexpr int opp(int l) { return l == 0 ? 0 : ((l & 1) ? l + 1 : l - 1); }
// index 0,1,2 of the per-axis factor tables for c = 0, +1, -1
__host__ __device__ constexpr int cidx(int c) { return c == 0 ? 0 : (c == 1 ? 1 : 2); }

// Per-axis factors of the product-form equilibrium (reference calculate_feq,
// src/headers/lbm.hpp:276-305): psi_0 = 1 - zeta, psi_+-1 = (+-xi + zeta)/2.
template <typename R>
struct AxisF {
    R v[3][3];  // [axis][c index]
};

template <typename R>
__host__ __device__ __forceinline__ void axis_feq(AxisF<R> &F, const R u[3], R theta, const R corr[3]) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const R z = theta + u[a] * u[a] + corr[a];
        F.v[a][0] = R(1) - z;
        F.v[a][1] = (u[a] + z) * R(0.5);
        F.v[a][2] = (-u[a] + z) * R(0.5);
    }
}

template <typename R>
__host__ __device__ __forceinline__ R feq_l(int l, R rho, const AxisF<R> &F) {
    return rho * F.v[0][cidx(cx(l))] * F.v[1][cidx(cy(l))] * F.v[2][cidx(cz(l))];
}

// Energy equilibrium (the reference's expanded polynomial, src/lbm-edf.cpp:38-98),
// factorised: g_l = rho [E Px Py Pz + Ax Py Pz + Px Ay Pz + Px Py Az] with
// P_a = psi(c_a; u_a, theta + u_a^2), A_a = theta u_a dpsi/dxi + (theta^2 + 2 theta u_a^2) dpsi/dzeta,
// E = U + |u|^2/2.  This is the first-order correction of E*Psi that reproduces the
// reference's total-energy, energy-flux and second-moment constraints; it equals the
// reference polynomial identically (checked symbolically for all 27 directions).
template <typename R>
struct AxisG {
    R P[3][3], A[3][3];
    R E;
};

template <typename R>
__host__ __device__ __forceinline__ void axis_geq(AxisG<R> &G, R U, R theta, const R u[3]) {
    G.E = U + R(0.5) * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const R z = theta + u[a] * u[a];
        const R s = theta * theta + R(2) * theta * u[a] * u[a];
        const R tu = theta * u[a] * R(0.5);
        G.P[a][0] = R(1) - z;
        G.P[a][1] = (u[a] + z) * R(0.5);
        G.P[a][2] = (-u[a] + z) * R(0.5);
        G.A[a][0] = -s;
        G.A[a][1] = tu + s * R(0.5);
        G.A[a][2] = -tu + s * R(0.5);
    }
}

template <typename R>
__host__ __device__ __forceinline__ R geq_l(int l, R rho, const AxisG<R> &G) {
    const int ix = cidx(cx(l)), iy = cidx(cy(l)), iz = cidx(cz(l));
    const R px = G.P[0][ix], py = G.P[1][iy], pz = G.P[2][iz];
    const R r = G.E * px * py * pz + G.A[0][ix] * py * pz + px * G.A[1][iy] * pz + px * py * G.A[2][iz];
    return rho * r;
}

}  // namespace lbm
