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
constexpr int kSurInX = 2 * kSurInPad;        // a feature row as the network reads it: the BF16
                                              // value of each standardised feature, then the BF16
                                              // remainder (feature - value), two k-slices whose sum
                                              // carries the feature to ~16 significant bits
constexpr int kSurHid = 128;                  // hidden width
constexpr int kSurOut = 10, kSurOutPad = 16;  // outputs, padded to two MMA n-tiles
constexpr int kSurLd = kSurHid + 8;           // row stride (bf16) of the 128-wide weights: no bank conflicts

// Standardisation of the features and targets, and the box of the training features the
// gate accepts (expanded by 5 % of its width on both sides).
constexpr float kSurOutGate = 16.f;    // predictions beyond 16 standard deviations of the
                                       // training targets go to the integrator
constexpr double kSurNegTol = 1e-12;   // ... and so do those that drive a mass fraction below -1e-12
struct SurNorm {
    float x_mean[kSurInPad], x_std[kSurInPad], x_lo[kSurInPad], x_hi[kSurInPad];
    float y_mean[kSurOutPad], y_std[kSurOutPad];
};

// What the collision-parameter kernel needs of the surrogate in one step.
struct SurArgs {
    int mode;                  // 0: integrator (teacher); 1: surrogate with integrator fallback
    const float *pred;         // [ncell][kSurOutPad] predicted dY_k, dT (SI), mode 1
    const uint8_t *gate;       // per cell 1: features outside the training box -> integrator
    const SurNorm *nrm;        // the standardisation (output gate)
    double *audit;             // [0] sum of |dY_net - dY_int|_1, [1] sum of |dY_int|_1, [2] max
                               // of the former (bits), [3] audited, [4] predicted, [5] integrated
    unsigned audit_period;     // every audit_period-th cell (n % audit_period == audit_phase,
    unsigned audit_phase;      //   the phase moving from step to step) is audited
    unsigned step;
    const double *proj;        // [9][9] projector onto element-conserving changes (sur_projector)
    // sample collection: integrated cells with n % ds_stride == ds_phase write their
    // (features, targets) to row ds_base + n / ds_stride while below ds_cap -- teacher steps
    // at the collection stride, surrogate steps at the audit stride and phase (the audited
    // cells and those outside the training box on it: states the integrator takes anyway)
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

// The orthogonal projector onto element-conserving changes of the mass fractions,
//   P = I - A^T (A A^T)^-1 A,   A_ek = E_ek / W_k (atoms of element e per unit mass of k),
// over the elements some species carries; A P = 0, so P dY conserves every element to
// rounding, and a dY that already conserves them comes back unchanged.  Formed once on the
// host from the mechanism (Gauss-Jordan elimination with partial pivoting on the small,
// symmetric positive definite A A^T); proj is row-major [NS][NS].
template <int NS>
inline void sur_projector(const double (*elements)[LBMGPU_MAX_ELEMENTS], const double *W, double *proj) {
    constexpr int kE = LBMGPU_MAX_ELEMENTS;
    double A[kE][NS];
    int ne = 0;
    for (int e = 0; e < kE; ++e) {
        bool any = false;
        for (int k = 0; k < NS; ++k) any = any || elements[k][e] != 0.0;
        if (!any) continue;
        for (int k = 0; k < NS; ++k) A[ne][k] = elements[k][e] / W[k];
        ++ne;
    }
    double G[kE][2 * kE];  // [A A^T | I] -> [I | (A A^T)^-1]
    for (int i = 0; i < ne; ++i)
        for (int j = 0; j < ne; ++j) {
            double g = 0.0;
            for (int k = 0; k < NS; ++k) g += A[i][k] * A[j][k];
            G[i][j] = g;
            G[i][ne + j] = i == j ? 1.0 : 0.0;
        }
    for (int c = 0; c < ne; ++c) {
        int p = c;
        for (int r = c + 1; r < ne; ++r)
            if (fabs(G[r][c]) > fabs(G[p][c])) p = r;
        for (int q = 0; q < 2 * ne; ++q) {
            const double tmp = G[c][q];
            G[c][q] = G[p][q];
            G[p][q] = tmp;
        }
        const double piv = G[c][c];
        for (int q = 0; q < 2 * ne; ++q) G[c][q] /= piv;
        for (int r = 0; r < ne; ++r) {
            if (r == c) continue;
            const double f = G[r][c];
            for (int q = 0; q < 2 * ne; ++q) G[r][q] -= f * G[c][q];
        }
    }
    for (int k = 0; k < NS; ++k)
        for (int l = 0; l < NS; ++l) {
            double v = k == l ? 1.0 : 0.0;
            for (int i = 0; i < ne; ++i)
                for (int j = 0; j < ne; ++j) v -= A[i][k] * G[i][ne + j] * A[j][l];
            proj[k * NS + l] = v;
        }
}

// The predicted change dY made exactly element-conserving: dY <- P dY (the smallest
// correction in the L2 sense).  Species at the density floor are treated like the others:
// the LBM's species collision drops a negative change of a floored species whichever
// chemistry produced it, so the surrogate's change goes through the same rule as the
// integrator's.
template <int NS>
__host__ __device__ inline void sur_conserve(const double *proj, double *dY) {
    double out[NS];
    for (int k = 0; k < NS; ++k) {
        double v = 0.0;
        for (int l = 0; l < NS; ++l) v += proj[k * NS + l] * dY[l];
        out[k] = v;
    }
    for (int k = 0; k < NS; ++k) dY[k] = out[k];
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
