// Chemistry surrogate shared between the per-cell kernels (mc_cell.cuh) and the network
// kernels (surrogate.cu): the input features of a cell, the per-step arguments the
// collision-parameter kernel reads, and the network's fixed shape.
//
// The surrogate replaces the stiff integrator of LBMGPU_CHEM_ROSENBROCK over one lattice
// step: (T, ln p, Y_0..Y_8, dt) -> (dY_0..dY_8, dT).  A small MLP, 12 -> 128 -> 128 -> 128
// -> 10 with GELU hidden layers, BF16 weights and activations, FP32 accumulation.  Inputs
// and outputs are standardised with the training set's mean and standard deviation.
#pragma once
#include <stdint.h>

#include "gas.cuh"

namespace lbm {

constexpr int kSurIn = 12, kSurInPad = 16;    // features, padded to one MMA k-slice
constexpr int kSurHid = 128;                  // hidden width
constexpr int kSurOut = 10, kSurOutPad = 16;  // outputs, padded to two MMA n-tiles
constexpr int kSurLd = kSurHid + 8;           // row stride (bf16) of the 128-wide weights: no bank conflicts

// Standardisation of the features and targets, and the box of the training features the
// gate accepts (expanded by 5 % of its width on both sides).
struct SurNorm {
    float x_mean[kSurInPad], x_std[kSurInPad], x_lo[kSurInPad], x_hi[kSurInPad];
    float y_mean[kSurOutPad], y_std[kSurOutPad];
};

// What the collision-parameter kernel needs of the surrogate in one step.
struct SurArgs {
    int mode;                  // 0: integrator (teacher); 1: surrogate with integrator fallback
    const float *pred;         // [ncell][kSurOutPad] predicted dY_k, dT (SI), mode 1
    const uint8_t *gate;       // per cell 1: features outside the training box -> integrator
    double *audit;             // [0] sum of |dY_net - dY_int|_1, [1] sum of |dY_int|_1, [2] max
                               // of the former (bits), [3] audited, [4] predicted, [5] integrated
    unsigned audit_period;     // 1 in audit_period cells (by a hash of cell and step) is audited
    unsigned step;
    const double *elem;        // [4][9] atoms of element e per unit mass of species k: E_ek / W_k
    // sample collection (teacher steps): cells with n % ds_stride == ds_phase write their
    // (features, targets) to row ds_base + n / ds_stride while below ds_cap
    float *ds_x, *ds_y;        // [ds_cap][kSurIn], [ds_cap][kSurOut]
    uint8_t *ds_valid;
    long ds_base, ds_cap;
    int ds_stride, ds_phase;
    double dt_si;              // the lattice time step in seconds
    int *ilist;                // cells left to the integrator (mode 1), appended by the
    unsigned *icount;          //   collision-parameter kernel, integrated by k_mc_chem_list
};

// Features of a cell: T (K), ln p (p in Pa), the normalised mass fractions, dt (s).
template <int NS>
__host__ __device__ inline void sur_features(double T_si, double P_si, const double *Y, double dt_si, float *x) {
    x[0] = (float)T_si;
    x[1] = (float)log(P_si);
    for (int a = 0; a < NS; ++a) x[2 + a] = (float)Y[a];
    x[2 + NS] = (float)dt_si;
}

// The predicted change dY made exactly element-conserving: species already at the floor
// (rho_a <= floor) whose prediction is negative are held at zero change -- the LBM would
// drop such a change (the species collision's skip rule), which is what would break the
// balance -- and the others take the smallest correction that restores
//   sum_k E_ek / W_k dY_k = 0   for every element e,
// dY_free -= A_f^T (A_f A_f^T)^-1 A_f dY_free over the elements the free species carry.
template <int NS>
__host__ __device__ inline void sur_conserve(const double *elem, const double *rho_a, double floor_rho, double *dY) {
    bool fixed[NS];
    for (int k = 0; k < NS; ++k) {
        fixed[k] = rho_a[k] <= floor_rho && dY[k] < 0.0;
        if (fixed[k]) dY[k] = 0.0;
    }
    // elements carried by some free species
    int rows[4], ne = 0;
    for (int e = 0; e < 4; ++e) {
        bool any = false;
        for (int k = 0; k < NS; ++k) any = any || (!fixed[k] && elem[e * NS + k] != 0.0);
        if (any) rows[ne++] = e;
    }
    if (ne == 0) return;
    double G[4][5];  // [G | r]
    for (int i = 0; i < ne; ++i) {
        for (int j = 0; j < ne; ++j) {
            double g = 0.0;
            for (int k = 0; k < NS; ++k)
                if (!fixed[k]) g += elem[rows[i] * NS + k] * elem[rows[j] * NS + k];
            G[i][j] = g;
        }
        double r = 0.0;
        for (int k = 0; k < NS; ++k) r += elem[rows[i] * NS + k] * dY[k];
        G[i][ne] = r;
    }
    for (int c = 0; c < ne; ++c) {  // Gaussian elimination with partial pivoting (G is SPD)
        int p = c;
        for (int r = c + 1; r < ne; ++r)
            if (fabs(G[r][c]) > fabs(G[p][c])) p = r;
        for (int q = 0; q <= ne; ++q) {
            const double tmp = G[c][q];
            G[c][q] = G[p][q];
            G[p][q] = tmp;
        }
        for (int r = c + 1; r < ne; ++r) {
            const double f = G[r][c] / G[c][c];
            for (int q = c; q <= ne; ++q) G[r][q] -= f * G[c][q];
        }
    }
    double lam[4];
    for (int r = ne - 1; r >= 0; --r) {
        double v = G[r][ne];
        for (int q = r + 1; q < ne; ++q) v -= G[r][q] * lam[q];
        lam[r] = v / G[r][r];
    }
    for (int k = 0; k < NS; ++k) {
        if (fixed[k]) continue;
        double corr = 0.0;
        for (int i = 0; i < ne; ++i) corr += elem[rows[i] * NS + k] * lam[i];
        dY[k] -= corr;
    }
}

__host__ __device__ inline unsigned sur_hash(unsigned a, unsigned b) {
    unsigned h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u + (a << 6) + (a >> 2));
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

}  // namespace lbm
