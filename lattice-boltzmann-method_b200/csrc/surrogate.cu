// Chemistry surrogate: network kernels, training and the C entry points.
//
// No counterpart in the reference (whose chemistry is Cantera's explicit rates): an MLP
// that learns the stiff ROS2 integrator's step (T, ln p, Y_k, dt) -> (dY_k, dT) from
// samples the integrator itself writes while the run proceeds (mc_cell.cuh, teacher
// steps), then stands in for it with an input-box gate, an exactly element-conserving
// correction of the prediction (sur_conserve, surrogate.cuh) and an audited sample
// (mc_cell.cuh, mode 1).
//
// Tensor-core kernels, BF16 operands with FP32 accumulation:
//   k_sur_mlp_tc  the whole network for 128-cell tiles on the 5th-generation tensor cores:
//                 tcgen05.mma from shared-memory operand tiles into a tensor-memory
//                 accumulator, one commit per layer on an mbarrier, the bias/GELU epilogue
//                 from tcgen05.ld back into shared memory as the next layer's operand; the
//                 first layer takes each standardised feature as a BF16 value plus a BF16
//                 remainder, two k-slices against the same W1, so the inputs (T above all:
//                 BF16 alone would round 1700 K by several kelvin) enter at ~16 bits;
//   k_gemm_tn     C = A B^T for training (forward, input gradients, weight gradients),
//                 tcgen05 with the same shared-memory layout, 128 x 64 tiles;
//   elementwise bias/GELU forward and backward, the MSE loss gradient, column sums for
//   the bias gradients, Adam on FP32 master weights with BF16 copies.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "handle.cuh"
#include "mc_cell.cuh"
#include "surrogate_host.cuh"

namespace lbmh {

using namespace lbm;

namespace {

constexpr int kW1 = kSurHid * kSurInPad;       // elements of the padded weight tensors
constexpr int kW2 = kSurHid * kSurLd;
constexpr int kW4 = kSurOutPad * kSurLd;
constexpr int kNParams = kW1 + 2 * kW2 + kW4 + 3 * kSurHid + kSurOutPad;

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const unsigned *>(&v);
}

// GELU in its tanh form (Hendrycks & Gimpel, arXiv:1606.08415):
//   gelu(z) = z/2 (1 + tanh(u)),  u = sqrt(2/pi) (z + 0.044715 z^3),
// the tanh from the hardware's approximate tanh (relative error about 2^-11, below the BF16
// rounding of the activations), the same function in training and inference.
__host__ __device__ __forceinline__ float tanh_fast(float u) {
#if defined(__CUDA_ARCH__)
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return t;
#else
    return tanhf(u);
#endif
}
// u = z (c + c' z^2), gelu = z/2 + (z/2) tanh(u), c = sqrt(2/pi), c' = 0.044715 c: the same
// fused multiply-adds in the scalar form (training) and the packed pair form (inference).
constexpr float kGeluC = 0.7978845608028654f;     // sqrt(2 / pi)
constexpr float kGeluC3 = 0.7978845608028654f * 0.044715f;
__host__ __device__ __forceinline__ float gelu_f(float z) {
    const float u = z * fmaf(z * z, kGeluC3, kGeluC);
    const float hz = 0.5f * z;
    return fmaf(hz, tanh_fast(u), hz);
}
__device__ inline float gelu_grad(float z) {
    const float z2 = z * z;
    const float t = tanh_fast(z * fmaf(z2, kGeluC3, kGeluC));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * fmaf(z2, 3.0f * kGeluC3, kGeluC);
}
// gelu_f of two values with the packed FP32 pair instructions of sm_100 (the tanh stays scalar)
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 u = __fmul2_rn(z, __ffma2_rn(__fmul2_rn(z, z), make_float2(kGeluC3, kGeluC3),
                                              make_float2(kGeluC, kGeluC)));
    const float2 hz = __fmul2_rn(z, make_float2(0.5f, 0.5f));
    return __ffma2_rn(hz, make_float2(tanh_fast(u.x), tanh_fast(u.y)), hz);
}

// The first padding slot of a network input row carries 1.0 as value and as "remainder": the
// tensor-core network multiplies it by the first layer's bias, split into a BF16 value and a
// BF16 remainder (k_sur_mlp_tc), so the bias is added inside the MMA.
constexpr int kSurBiasSlot = kSurIn;
static_assert(kSurBiasSlot < kSurInPad && kSurBiasSlot % 2 == 0, "a padding slot at an even index");
__device__ __forceinline__ unsigned bias_slot_pair(unsigned pair) {  // (1.0, the odd slot's value)
    return (pair & 0xFFFF0000u) | (unsigned)__bfloat16_as_ushort(__float2bfloat16(1.0f));
}

// A standardised feature into slot q of a network input row: its BF16 value and the BF16
// remainder.
__device__ __forceinline__ void put_split(__nv_bfloat16 *row, int q, float v) {
    const __nv_bfloat16 hi = __float2bfloat16(v);
    row[q] = hi;
    row[kSurInPad + q] = __float2bfloat16(v - __bfloat162float(hi));
}

// -------------------------------------------------------------------------------------
// Inference: features of every cell, then the fused network.
// -------------------------------------------------------------------------------------
template <int NS, typename S>
__global__ void k_sur_features(McArgsT<S, double> A, const SurNorm *__restrict__ nrm, __nv_bfloat16 *__restrict__ X,
                               uint8_t *__restrict__ gate, long mpad) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= mpad) return;
    float x[kSurInPad] = {};
    bool out_of_box = true;
    if (n < A.ncell && (A.cflag[n] & CF_FLUID)) {
        const gas::Tables &t = *A.tab;
        const double rho = rec(A, A.rec_cur, RM_RHO, n);
        double Yr[NS], Y[NS], Xm[NS];
        for (int a = 0; a < NS; ++a) Yr[a] = rec(A, A.rec_cur, rs(a, RS_RHO), n) / rho;
        const double W = set_mass_fractions<NS>(t, Yr, Y, Xm);
        const double T_si = si_temp(A.U, (float)rec(A, A.rec_cur, RM_T, n));
        const double rho_si = si_rho(A.U, (float)rho);
        const double P_si = rho_si * gas::kR * T_si / W;
        sur_features<NS>(T_si, P_si, Y, (double)A.dt * (double)A.U.s, x);
        out_of_box = false;
        for (int q = 0; q < kSurIn; ++q) {
            const float w = nrm->x_hi[q] - nrm->x_lo[q];
            if (w > 0.f && (x[q] < nrm->x_lo[q] - 0.05f * w || x[q] > nrm->x_hi[q] + 0.05f * w)) out_of_box = true;
            x[q] = (x[q] - nrm->x_mean[q]) / nrm->x_std[q];
        }
    }
    // the row (kSurInPad values, then their remainders) as four 16-byte stores, so a warp
    // writes 2 kB of consecutive rows
    unsigned hv[kSurInPad / 2], lv[kSurInPad / 2];
#pragma unroll
    for (int q = 0; q < kSurInPad; q += 2) {
        const __nv_bfloat16 h0 = __float2bfloat16(x[q]), h1 = __float2bfloat16(x[q + 1]);
        const __nv_bfloat162 hh = __halves2bfloat162(h0, h1);
        const __nv_bfloat162 ll = __floats2bfloat162_rn(x[q] - __bfloat162float(h0), x[q + 1] - __bfloat162float(h1));
        hv[q / 2] = *reinterpret_cast<const unsigned *>(&hh);
        lv[q / 2] = *reinterpret_cast<const unsigned *>(&ll);
    }
    hv[kSurBiasSlot / 2] = bias_slot_pair(hv[kSurBiasSlot / 2]);
    lv[kSurBiasSlot / 2] = bias_slot_pair(lv[kSurBiasSlot / 2]);
    uint4 *row = reinterpret_cast<uint4 *>(X + n * kSurInX);
    static_assert(kSurInPad == 16 && kSurInX == 32, "a row is 16 values and 16 remainders");
    row[0] = make_uint4(hv[0], hv[1], hv[2], hv[3]);
    row[1] = make_uint4(hv[4], hv[5], hv[6], hv[7]);
    row[2] = make_uint4(lv[0], lv[1], lv[2], lv[3]);
    row[3] = make_uint4(lv[4], lv[5], lv[6], lv[7]);
    if (n < A.ncell) gate[n] = out_of_box ? 1 : 0;
}

// Raw features (rows of kSurIn floats) -> standardised network input rows.
__global__ void k_sur_standardise(const float *__restrict__ x, long m, long mpad, const SurNorm *__restrict__ nrm,
                                  __nv_bfloat16 *__restrict__ X) {
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= mpad) return;
    for (int q = 0; q < kSurInPad; ++q) {
        float v = 0.f;
        if (r < m && q < kSurIn) v = (x[r * kSurIn + q] - nrm->x_mean[q]) / nrm->x_std[q];
        put_split(X + r * kSurInX, q, v);
    }
    X[r * kSurInX + kSurBiasSlot] = __float2bfloat16(1.0f);
    X[r * kSurInX + kSurInPad + kSurBiasSlot] = __float2bfloat16(1.0f);
}

struct SurNet {  // device pointers of the BF16 weights and FP32 biases
    const __nv_bfloat16 *w1, *w2, *w3, *w4;
    const float *b1, *b2, *b3, *b4;
};



// -------------------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05): 128 cells per tile = the MMA's
// M.  The four weight tiles sit in shared memory once per CTA; per layer one thread issues
// tcgen05.mma (BF16 operands from shared memory, FP32 accumulator of 128 lanes x N columns
// in tensor memory) and commits it to an mbarrier; after the wait each thread -- one per
// cell row, warp w reading tensor-memory lanes 32w..32w+31 -- takes its row with
// tcgen05.ld, adds the bias, applies GELU and writes the BF16 row back to shared memory as
// the next layer's A operand.  Shared-memory operands are K-major without swizzle: element
// (r, k) of an R x K tile at byte (r / 8) (16 K) + (k / 8) 128 + (r % 8) 16 + (k % 8) 2,
// i.e. 8 x 16-byte core matrices, the two of one 16-wide K step 128 bytes apart (leading
// offset) and 8-row groups 16 K bytes apart (stride offset).  Every wait has a time limit:
// past it the kernel raises LBMGPU_ST_SURROGATE, waits once more for its own tensor-core
// work, frees its tensor memory and returns.
// -------------------------------------------------------------------------------------
constexpr int kTcRows = 128;       // cells per tile (MMA M), one thread each
constexpr int kTcGroups = 3;       // independent tile groups per CTA (one warpgroup each)
constexpr uint32_t kTcCols = 128;  // tensor-memory columns per group: the widest accumulator
// tensor memory is allocated in powers of two columns (32..512): the groups' columns rounded up
constexpr uint32_t kTcAlloc = kTcCols * kTcGroups <= 256 ? 256u : 512u;
static_assert(kTcCols * kTcGroups <= kTcAlloc && kTcAlloc <= 512, "the groups' accumulators fit tensor memory");
// The hidden activations carry one more 16-wide K slice (kTcK): columns 128 and 129 hold 1.0
// and the next layer's weights there its bias split into a BF16 value and a BF16 remainder,
// so the MMA adds the bias; the input rows do the same in their padding slot (kSurBiasSlot).
constexpr int kTcK = kSurHid + 16;
constexpr int kTcW1 = 0, kTcW2 = kTcW1 + kSurHid * kSurInX * 2, kTcW3 = kTcW2 + kSurHid * kTcK * 2,
              kTcW4 = kTcW3 + kSurHid * kTcK * 2, kTcG = kTcW4 + kSurOutPad * kTcK * 2,  // weights, shared
              kTcA = 0, kTcX = kTcA + kTcRows * kTcK * 2, kTcGBytes = kTcX + kTcRows * kSurInX * 2,  // per group
              kTcB = kTcG + kTcGroups * kTcGBytes, kTcBar = kTcB + 2 * kSurOutPad * 4,
              kTcErr = kTcBar + 8 * kTcGroups, kTcSlot = kTcErr + 4 * kTcGroups, kTcSmem = kTcSlot + 8;
static_assert(kTcSmem <= 227 * 1024, "one CTA's shared memory");
static_assert(kTcG % 16 == 0 && kTcGBytes % 16 == 0 && kTcX % 16 == 0 && kTcBar % 8 == 0,
              "operand tiles 16-byte, mbarriers 8-byte aligned");

__device__ __forceinline__ uint32_t tc_off(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
// shared-memory matrix descriptor: start, leading offset 128 B, stride offset, version 1
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void group_bar(int g) {  // the 128 threads of tile group g
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kTcRows) : "memory");
}
__device__ __forceinline__ void tc_sync(int g) {  // group's shared writes visible to the tensor core, in step
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    group_bar(g);
    tc_fence_after();
}
// One layer: D (tensor memory) = A (rows x K, shared) B^T (N x K, shared), K / 16 MMAs, then
// the commit that arrives on the mbarrier when they are done.
__device__ __forceinline__ void tc_layer(uint32_t tmem, uint32_t a, uint32_t b, int K, int N, uint32_t bar) {
    const uint32_t idesc = tc_idesc(N);
    for (int s = 0; s < K / 16; ++s) {
        const uint64_t ad = tc_desc(a + 256u * s, (uint32_t)K * 16u), bd = tc_desc(b + 256u * s, (uint32_t)K * 16u);
        const uint32_t acc = s > 0;
        asm volatile(
            "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// Waits for the mbarrier phase `parity`, at most ~1 s of wall time.
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    uint64_t t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 1000000000ull) return false;
    }
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// X [mpad][kSurInX] network input rows -> pred [mpad][16] in SI units (outputs 10..15 zero).
// kTcGroups warpgroups per CTA work on their own tiles (own operand buffers, mbarrier and
// tensor-memory columns) against the shared weights, so one group's epilogue overlaps the
// other's tensor-core work and epilogue.
__global__ void __launch_bounds__(kTcRows *kTcGroups, 1)
    k_sur_mlp_tc(SurNet net, const SurNorm *__restrict__ nrm, const __nv_bfloat16 *__restrict__ X,
                 float *__restrict__ pred, long mpad, unsigned *__restrict__ status) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, g = tid / kTcRows, t = tid % kTcRows;
    const int nthr = kTcRows * kTcGroups;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm);
    float *bb = reinterpret_cast<float *>(sm + kTcB);  // y_mean, y_std
    // weights into the canonical layout: W1 as [W1 | W1] (values and remainders), W2, W3, W4;
    // each layer's bias as a BF16 value and remainder in the K slice its input's 1.0 meets
    auto split = [](float b, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
        hi = __float2bfloat16(b);
        lo = __float2bfloat16(b - __bfloat162float(hi));
    };
    for (int i = tid; i < kSurHid * (kSurInX / 8); i += nthr) {
        const int r = i / (kSurInX / 8), c = i % (kSurInX / 8);
        union {
            uint4 v;
            __nv_bfloat16 e[8];
        } u;
        u.v = *reinterpret_cast<const uint4 *>(net.w1 + r * kSurInPad + (c % 2) * 8);
        if (c % 2 == kSurBiasSlot / 8) {  // the bias slot: value half, remainder half
            __nv_bfloat16 hi, lo;
            split(net.b1[r], hi, lo);
            u.e[kSurBiasSlot % 8] = c < 2 ? hi : lo;
        }
        *reinterpret_cast<uint4 *>(sm + kTcW1 + tc_off(r, c * 8, kSurInX)) = u.v;
    }
    auto hidden_w = [&](int off, const __nv_bfloat16 *w, const float *b, int rows) {
        for (int i = tid; i < rows * (kTcK / 8); i += nthr) {
            const int r = i / (kTcK / 8), c = i % (kTcK / 8);
            union {
                uint4 v;
                __nv_bfloat16 e[8];
            } u;
            u.v = make_uint4(0u, 0u, 0u, 0u);
            if (c < kSurHid / 8) {
                u.v = *reinterpret_cast<const uint4 *>(w + r * kSurLd + c * 8);
            } else if (c == kSurHid / 8) {
                split(b[r], u.e[0], u.e[1]);
            }
            *reinterpret_cast<uint4 *>(sm + off + tc_off(r, c * 8, kTcK)) = u.v;
        }
    };
    hidden_w(kTcW2, net.w2, net.b2, kSurHid);
    hidden_w(kTcW3, net.w3, net.b3, kSurHid);
    hidden_w(kTcW4, net.w4, net.b4, kSurOutPad);
    if (tid < kSurOutPad) {
        bb[tid] = nrm->y_mean[tid];
        bb[kSurOutPad + tid] = nrm->y_std[tid];
    }
    volatile int *err = reinterpret_cast<volatile int *>(sm + kTcErr);
    if (tid < kTcGroups) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(base + kTcBar + 8u * tid) : "memory");
        err[tid] = 0;
    }
    if (tid == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kTcSlot),
                     "r"(kTcAlloc)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *reinterpret_cast<volatile uint32_t *>(sm + kTcSlot);
    const uint32_t tmem = tbase + kTcCols * (uint32_t)g;                     // this group's accumulator
    const uint32_t trow = tmem + ((uint32_t)((warp % 4) * 32) << 16);        // this warp's lane quarter
    const uint32_t bar = base + kTcBar + 8u * (uint32_t)g;
    const uint32_t gA = base + kTcG + (uint32_t)(g * kTcGBytes) + kTcA, gX = base + kTcG + (uint32_t)(g * kTcGBytes) + kTcX;
    unsigned char *smA = sm + kTcG + g * kTcGBytes + kTcA, *smX = sm + kTcG + g * kTcGBytes + kTcX;
    const float *ym = bb, *ys = bb + kSurOutPad;
    {  // the activations' bias slice: 1.0 in columns 128 and 129, zeros after (never rewritten)
        const __nv_bfloat162 one2 = __floats2bfloat162_rn(1.0f, 1.0f);
        const unsigned one = *reinterpret_cast<const unsigned *>(&one2);
        *reinterpret_cast<uint4 *>(smA + tc_off(t, kSurHid, kTcK)) = make_uint4(one, 0u, 0u, 0u);
        *reinterpret_cast<uint4 *>(smA + tc_off(t, kSurHid + 8, kTcK)) = make_uint4(0u, 0u, 0u, 0u);
    }
    const uint32_t wl[4] = {base + kTcW1, base + kTcW2, base + kTcW3, base + kTcW4};
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (mpad + kTcRows - 1) / kTcRows;
    for (long tile = (long)blockIdx.x * kTcGroups + g; tile < ntiles && ok; tile += (long)gridDim.x * kTcGroups) {
        const long row = tile * kTcRows + t;
#pragma unroll
        for (int c = 0; c < kSurInX / 8; ++c) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (row < mpad) v = *reinterpret_cast<const uint4 *>(X + row * kSurInX + c * 8);
            *reinterpret_cast<uint4 *>(smX + tc_off(t, c * 8, kSurInX)) = v;
        }
        tc_sync(g);
        for (int L = 0; L < 4 && ok; ++L) {
            if (t == 0)
                tc_layer(tmem, L == 0 ? gX : gA, wl[L], L == 0 ? kSurInX : kTcK, L == 3 ? kSurOutPad : kSurHid, bar);
            if (!tc_wait(bar, phase)) err[g] = 1;
            group_bar(g);
            tc_fence_after();
            ok = err[g] == 0;
            if (!ok) break;
            phase ^= 1u;
            if (L < 3) {  // GELU of the accumulator (the bias is in it), BF16 into the next operand
#pragma unroll 1
                for (int cb = 0; cb < kSurHid / 32; ++cb) {
                    uint32_t r[32];
                    tc_ld32(trow + (uint32_t)(cb * 32), r);
                    tc_wait_ld();
#pragma unroll
                    for (int j = 0; j < 32; j += 8) {
                        uint4 o;
                        const int k = cb * 32 + j;
                        float2 a;
                        a = gelu2(make_float2(__uint_as_float(r[j]), __uint_as_float(r[j + 1])));
                        o.x = pack_bf16(a.x, a.y);
                        a = gelu2(make_float2(__uint_as_float(r[j + 2]), __uint_as_float(r[j + 3])));
                        o.y = pack_bf16(a.x, a.y);
                        a = gelu2(make_float2(__uint_as_float(r[j + 4]), __uint_as_float(r[j + 5])));
                        o.z = pack_bf16(a.x, a.y);
                        a = gelu2(make_float2(__uint_as_float(r[j + 6]), __uint_as_float(r[j + 7])));
                        o.w = pack_bf16(a.x, a.y);
                        *reinterpret_cast<uint4 *>(smA + tc_off(t, k, kTcK)) = o;
                    }
                }
            } else {
                uint32_t r[16];
                tc_ld16(trow, r);
                tc_wait_ld();
                if (row < mpad) {
#pragma unroll
                    for (int c = 0; c < kSurOutPad; c += 4) {
                        float4 o;
                        o.x = __uint_as_float(r[c]) * ys[c] + ym[c];
                        o.y = __uint_as_float(r[c + 1]) * ys[c + 1] + ym[c + 1];
                        o.z = __uint_as_float(r[c + 2]) * ys[c + 2] + ym[c + 2];
                        o.w = __uint_as_float(r[c + 3]) * ys[c + 3] + ym[c + 3];
                        *reinterpret_cast<float4 *>(pred + row * kSurOutPad + c) = o;
                    }
                }
            }
            tc_sync(g);
        }
    }
    if (!ok) {  // the tensor core may still be working on the timed-out layer: one more bounded wait
        if (t == 0) atomicOr(status, (unsigned)LBMGPU_ST_SURROGATE);
        tc_wait(bar, phase);
        tc_fence_after();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTcAlloc)
                     : "memory");
}

// -------------------------------------------------------------------------------------
// Training kernels.
// -------------------------------------------------------------------------------------
// C[M][N] (FP32, ldc) = A[M][K] B[N][K]^T (accum: C +=) on tcgen05, for training: A and B
// BF16 row-major with leading dimensions lda, ldb (multiples of 8), K a multiple of 16.  A
// CTA computes a 128 x 64 tile: K in chunks of 64 staged by its 128 threads into shared
// memory in the canonical layout of the network kernel (rows and columns past M, N, K
// zero-filled), four tcgen05.mma per chunk into a tensor-memory accumulator, a commit to the
// stage's mbarrier; two stages, so that the next chunk is staged while the tensor core works
// on this one (a stage is refilled after a bounded wait for the MMAs that read it two chunks
// earlier).  The epilogue reads the accumulator with tcgen05.ld.  With gridDim.z > 1 block z
// takes the z-th of gridDim.z equal slices of K (each a multiple of 16) and writes its partial
// product to C + z zstride (split K, summed afterwards by k_sum_splits).
constexpr int kGmM = 128, kGmN = 64, kGmK = 64;
constexpr int kGmStage = kGmM * kGmK * 2 + kGmN * kGmK * 2;  // A then B of one chunk
constexpr int kGmA = 0, kGmB = kGmM * kGmK * 2, kGmBar = 2 * kGmStage, kGmSlot = kGmBar + 16,
              kGmSmem = kGmSlot + 8;
static_assert(kGmStage % 128 == 0 && kGmBar % 8 == 0, "stage buffers 128-byte, mbarriers 8-byte aligned");
__global__ void __launch_bounds__(128) k_gemm_tn(const __nv_bfloat16 *__restrict__ Am, int lda,
                                                 const __nv_bfloat16 *__restrict__ Bm, int ldb, float *__restrict__ C,
                                                 int ldc, int M, int N, int K, int accum, long zstride,
                                                 unsigned *__restrict__ status) {
    extern __shared__ __align__(128) unsigned char gsm[];
    unsigned char *sm = gsm;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm);
    const int m0 = blockIdx.y * kGmM, n0 = blockIdx.x * kGmN;
    const int kc = K / (int)gridDim.z, kbeg = (int)blockIdx.z * kc;
    C += (long)blockIdx.z * zstride;
    const uint32_t bar0 = base + kGmBar;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + kGmSlot),
                     "r"((uint32_t)kGmN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(sm + kGmSlot);
    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};  // a commit of the stage not yet waited for
    bool ok = true;
    int it = 0;
    for (int k0 = kbeg; k0 < kbeg + kc && ok; k0 += kGmK, ++it) {
        const int st = it & 1;
        const uint32_t bar = bar0 + 8u * (uint32_t)st;
        if (pending[st]) {  // the MMAs of chunk it - 2 read this stage
            ok = __syncthreads_and(tc_wait(bar, phase[st])) != 0;
            tc_fence_after();
            if (!ok) break;
            phase[st] ^= 1u;
            pending[st] = false;
        }
        unsigned char *sa = sm + st * kGmStage + kGmA, *sb = sm + st * kGmStage + kGmB;
        // stage the chunk: A rows m0.., B rows n0.., 16-byte pieces (8 elements of K)
        for (int i = tid; i < kGmM * (kGmK / 8); i += 128) {
            const int r = i / (kGmK / 8), c = i % (kGmK / 8), k = k0 + c * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m0 + r < M && k < kbeg + kc) v = *reinterpret_cast<const uint4 *>(Am + (long)(m0 + r) * lda + k);
            *reinterpret_cast<uint4 *>(sa + tc_off(r, c * 8, kGmK)) = v;
        }
        for (int i = tid; i < kGmN * (kGmK / 8); i += 128) {
            const int r = i / (kGmK / 8), c = i % (kGmK / 8), k = k0 + c * 8;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (n0 + r < N && k < kbeg + kc) v = *reinterpret_cast<const uint4 *>(Bm + (long)(n0 + r) * ldb + k);
            *reinterpret_cast<uint4 *>(sb + tc_off(r, c * 8, kGmK)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t idesc = tc_idesc(kGmN);
            const uint32_t abase = base + (uint32_t)(st * kGmStage + kGmA), bbase = base + (uint32_t)(st * kGmStage + kGmB);
            for (int s = 0; s < kGmK / 16; ++s) {
                const uint64_t ad = tc_desc(abase + 256u * s, kGmK * 16u);
                const uint64_t bd = tc_desc(bbase + 256u * s, kGmK * 16u);
                const uint32_t acc = (k0 > kbeg || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        pending[st] = true;
    }
    // drain: the commits still outstanding (the last of each stage), each wait bounded; also
    // after a timed-out wait, so that no MMA is left running when the tensor memory is freed
    for (int s2 = 0; s2 < 2; ++s2)
        if (pending[s2]) {
            const bool done = __syncthreads_and(tc_wait(bar0 + 8u * (uint32_t)s2, phase[s2])) != 0;
            tc_fence_after();
            ok = ok && done;
        }
    if (ok && kc > 0) {  // epilogue: row m0 + tid of the tile, 64 columns in four loads
        const long r = m0 + tid;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int cb = 0; cb < kGmN / 16; ++cb) {
            uint32_t v[16];
            tc_ld16(trow + (uint32_t)(cb * 16), v);
            tc_wait_ld();
            if (r < M)
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int c = n0 + cb * 16 + j;
                    if (c < N) {
                        float *dst = C + r * ldc + c;
                        *dst = __uint_as_float(v[j]) + (accum ? *dst : 0.f);
                    }
                }
        }
    }
    if (!ok && tid == 0) atomicOr(status, (unsigned)LBMGPU_ST_SURROGATE);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kGmN) : "memory");
}

// out[r][c] = sum_z part[z][r][c] over the split-K slices, in slice order, for the
// cols real columns of rows of width ld (the padding columns of out are left alone).
__global__ void k_sum_splits(const float *__restrict__ part, int splits, long n, int cols, int ld,
                             float *__restrict__ out) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n || (int)(e % ld) >= cols) return;
    float v = 0.f;
    for (int z = 0; z < splits; ++z) v += part[(long)z * n + e];
    out[e] = v;
}

// Z = C + b; H = GELU(Z) in BF16 (rows of width W).
__global__ void k_bias_gelu(const float *__restrict__ C, const float *__restrict__ b, float *__restrict__ Z,
                            __nv_bfloat16 *__restrict__ H, long rows, int W) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * W) return;
    const float z = C[i] + b[i % W];
    Z[i] = z;
    H[i] = __float2bfloat16(gelu_f(z));
}

// Output layer: out = C + b4; dOut = 2 (out - y) / (valid * kSurOut) on the valid rows and
// real outputs, 0 elsewhere; the squared errors summed per block into part[].
__global__ void k_out_loss(const float *__restrict__ C, const float *__restrict__ b4, const float *__restrict__ Yt,
                           const uint8_t *__restrict__ valid, float nvalid, float *__restrict__ dOut,
                           double *__restrict__ part, long rows) {
    __shared__ double red[256];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double se = 0.0;
    if (i < rows * kSurOutPad) {
        const long r = i / kSurOutPad;
        const int c = (int)(i % kSurOutPad);
        float g = 0.f;
        if (c < kSurOut && valid[r]) {
            const float e = C[i] + b4[c] - Yt[i];
            se = (double)e * e;
            g = 2.f * e / (nvalid * kSurOut);
        }
        dOut[i] = g;
    }
    red[threadIdx.x] = se;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// dZ = dH * GELU'(Z) (FP32 in, BF16 and FP32 out).
__global__ void k_gelu_bwd(const float *__restrict__ dH, const float *__restrict__ Z, float *__restrict__ dZ,
                           __nv_bfloat16 *__restrict__ dZb, long n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = dH[i] * gelu_grad(Z[i]);
    dZ[i] = g;
    dZb[i] = __float2bfloat16(g);
}

__global__ void k_f32_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, long n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}

// out[c][r] = in[r][c] (BF16), in: rows x cols with leading dimension ldi, out: ldo.
__global__ void k_transpose_bf16(const __nv_bfloat16 *__restrict__ in, int ldi, __nv_bfloat16 *__restrict__ out,
                                 int ldo, int rows, int cols) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = by + y, c = bx + threadIdx.x;
        tile[y][threadIdx.x] = (r < rows && c < cols) ? in[(long)r * ldi + c] : __float2bfloat16(0.f);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = bx + y, r = by + threadIdx.x;
        if (c < cols && r < rows) out[(long)c * ldo + r] = tile[threadIdx.x][y];
    }
}

// db[c] = sum_r dZ[r][c] for a block of 32 columns: lane = column, warp w sums rows
// w, w + 8, ... in order (a warp reads 32 consecutive floats of a row), then the 8 warp
// sums are added in warp order -- a fixed order, so the result does not vary run to run.
constexpr int kColsumWarps = 8;
__global__ void __launch_bounds__(32 * kColsumWarps) k_colsum(const float *__restrict__ dZ, long rows, int W,
                                                               float *__restrict__ db) {
    __shared__ double part[kColsumWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, c = blockIdx.x * 32 + lane;
    double s = 0.0;
    if (c < W)
        for (long r = warp; r < rows; r += kColsumWarps) s += dZ[r * W + c];
    part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && c < W) {
        double t = 0.0;
        for (int w = 0; w < kColsumWarps; ++w) t += part[w][lane];
        db[c] = (float)t;
    }
}

// Adam on FP32 master parameters; the BF16 copy (if any) follows.  g at gradient stride.
__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, __nv_bfloat16 *__restrict__ wb, long n, float lr, float b1,
                       float b2, float c1, float c2, float eps) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

// Batch rows from the sample set: network input rows and standardised FP32 targets.
__global__ void k_gather_batch(const float *__restrict__ dx, const float *__restrict__ dy, const int *__restrict__ idx,
                               int nb, int B, const SurNorm *__restrict__ nrm, __nv_bfloat16 *__restrict__ Xb,
                               float *__restrict__ Yb, uint8_t *__restrict__ vb) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const bool ok = r < nb;
    const long s = ok ? idx[r] : 0;
    for (int q = 0; q < kSurInPad; ++q) {
        const float v = (ok && q < kSurIn) ? (dx[s * kSurIn + q] - nrm->x_mean[q]) / nrm->x_std[q] : 0.f;
        put_split(Xb + (long)r * kSurInX, q, v);
    }
    for (int q = 0; q < kSurOutPad; ++q)
        Yb[(long)r * kSurOutPad + q] = (ok && q < kSurOut) ? (dy[s * kSurOut + q] - nrm->y_mean[q]) / nrm->y_std[q] : 0.f;
    vb[r] = ok ? 1 : 0;
}

// State-space augmentation.  New row i takes a random valid row of the sample set (the
// source, drawn from the list src_rows of the n_src valid rows), multiplies each mass
// fraction below y_trace by exp(U(-span_y, span_y)) and T by exp(U(-span_t, span_t)) at
// the source's density, renormalises the mass fractions, and labels the perturbed state
// with the integrator over the source's dt.  Rows whose integration fails are left invalid.
__global__ void k_sur_augment(const gas::Tables *__restrict__ tab, float *__restrict__ ds_x, float *__restrict__ ds_y,
                              uint8_t *__restrict__ ds_valid, const int *__restrict__ src_rows, long n_src, long base,
                              long n_new, float span_y, float span_t, float y_trace, unsigned seed) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_new) return;
    const long row = base + i;
    unsigned hs = sur_hash((unsigned)i, seed);
    const long src = src_rows[((unsigned long long)hs * (unsigned long long)n_src) >> 32];
    const gas::Tables &t = *tab;
    const float *xs = ds_x + src * kSurIn;
    const double dt = xs[2 + 9];
    double T = xs[0], Y[gas::MAXS], iw = 0.0;
    for (int k = 0; k < 9; ++k) {
        Y[k] = xs[2 + k];
        iw += Y[k] / t.m.W[k];
    }
    const double rho = exp((double)xs[1]) / (gas::kR * T * iw);
    auto uni = [&](unsigned salt) {  // uniform in [-1, 1)
        hs = sur_hash(hs, salt);
        return (double)hs * (2.0 / 4294967296.0) - 1.0;
    };
    double sum = 0.0;
    for (int k = 0; k < 9; ++k) {
        const double f = exp(span_y * uni(k + 1));
        if (Y[k] < y_trace) Y[k] *= f;
        sum += Y[k];
    }
    iw = 0.0;
    for (int k = 0; k < 9; ++k) {
        Y[k] /= sum;
        iw += Y[k] / t.m.W[k];
    }
    T *= exp(span_t * uni(97));
    sur_features<9>(T, rho * gas::kR * T * iw, Y, dt, ds_x + row * kSurIn);
    double Yc[gas::MAXS], Tc = T;
    for (int k = 0; k < 9; ++k) Yc[k] = Y[k];
    if (gas::ros2_advance(t, rho, Yc, Tc, dt) < 0) {
        ds_valid[row] = 0;
        return;
    }
    for (int k = 0; k < 9; ++k) ds_y[row * kSurOut + k] = (float)(Yc[k] - Y[k]);
    ds_y[row * kSurOut + 9] = (float)(Tc - T);
    ds_valid[row] = 1;
}

inline unsigned blocks(long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// k_gemm_tn over the whole C (splits > 1: split K, partials zstride apart).
void gemm_tn(lbmgpu *h, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *Bm, int ldb, float *C, int ldc, int M,
             int N, int K, int accum = 0, int splits = 1, long zstride = 0) {
    cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, kGmSmem);
    k_gemm_tn<<<dim3((N + kGmN - 1) / kGmN, (M + kGmM - 1) / kGmM, splits), 128, kGmSmem, h->stream>>>(
        A, lda, Bm, ldb, C, ldc, M, N, K, accum, zstride, h->status);
}

}  // namespace

// -------------------------------------------------------------------------------------
// Host side.
// -------------------------------------------------------------------------------------
struct SurState {
    // parameters: FP32 master (w), Adam moments (m, v), gradients (g), BF16 copies of the
    // weight tensors; one contiguous block each in the order w1 w2 w3 w4 b1 b2 b3 b4
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    __nv_bfloat16 *wb = nullptr;
    SurNorm *nrm = nullptr;
    SurNorm nrm_h{};
    double *proj = nullptr;
    double *audit = nullptr;
    // samples
    float *ds_x = nullptr, *ds_y = nullptr;
    uint8_t *ds_valid = nullptr;
    long ds_cap = 0, ds_next = 0;
    int collect = 0, stride = 64, collect_steps = 0, step_stride = 64;
    // inference
    __nv_bfloat16 *feat = nullptr;
    uint8_t *gate = nullptr;
    float *pred = nullptr;
    int *ilist = nullptr;
    unsigned *icount = nullptr;
    long mpad = 0;
    int enabled = 0;
    unsigned audit_period = 100;
    unsigned step = 0;
    bool trained = false;
    long adam_t = 0, train_steps = 0;
    double last_loss = 0.0;
};

namespace {

size_t off_w(int t) {  // element offset of tensor t (0..3 weights, 4..7 biases)
    const size_t sz[8] = {kW1, kW2, kW2, kW4, kSurHid, kSurHid, kSurHid, kSurOutPad};
    size_t o = 0;
    for (int i = 0; i < t; ++i) o += sz[i];
    return o;
}

void default_norm(SurNorm &n) {
    for (int q = 0; q < kSurInPad; ++q) {
        n.x_mean[q] = 0.f;
        n.x_std[q] = 1.f;
        n.x_lo[q] = 0.f;
        n.x_hi[q] = 0.f;
    }
    for (int q = 0; q < kSurOutPad; ++q) {
        n.y_mean[q] = 0.f;
        n.y_std[q] = 1.f;
    }
}

int upload_params(lbmgpu *h) {  // FP32 master -> BF16 copies of the weight tensors
    SurState &s = *h->sur;
    const long nw = (long)off_w(4);
    k_f32_to_bf16<<<blocks(nw), 256, 0, h->stream>>>(s.w, s.wb, nw);
    CK(cudaGetLastError());
    return 0;
}

int init_params(lbmgpu *h, unsigned seed) {  // Kaiming-uniform weights, zero biases, fresh Adam
    SurState &s = *h->sur;
    std::vector<float> w(kNParams, 0.f);
    std::mt19937_64 rng(seed);
    const int fan_in[4] = {kSurIn, kSurHid, kSurHid, kSurHid};
    const int rows[4] = {kSurHid, kSurHid, kSurHid, kSurOut};
    const int ld[4] = {kSurInPad, kSurLd, kSurLd, kSurLd};
    for (int t = 0; t < 4; ++t) {
        const double bound = std::sqrt(6.0 / fan_in[t]) * (t == 3 ? 0.1 : 1.0);
        std::uniform_real_distribution<double> U(-bound, bound);
        for (int r = 0; r < rows[t]; ++r)
            for (int k = 0; k < fan_in[t]; ++k) w[off_w(t) + (size_t)r * ld[t] + k] = (float)U(rng);
    }
    CK(cudaMemcpyAsync(s.w, w.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(s.m, 0, kNParams * sizeof(float), h->stream));
    CK(cudaMemsetAsync(s.v, 0, kNParams * sizeof(float), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    s.adam_t = 0;
    return upload_params(h);
}

SurNet net_of(const SurState &s) {
    SurNet n;
    n.w1 = s.wb + off_w(0);
    n.w2 = s.wb + off_w(1);
    n.w3 = s.wb + off_w(2);
    n.w4 = s.wb + off_w(3);
    n.b1 = s.w + off_w(4);
    n.b2 = s.w + off_w(5);
    n.b3 = s.w + off_w(6);
    n.b4 = s.w + off_w(7);
    return n;
}

int run_mlp(lbmgpu *h, const __nv_bfloat16 *X, float *pred, long mpad) {
    SurState &s = *h->sur;
    CK(cudaFuncSetAttribute(k_sur_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    const long ntiles = (mpad + kTcRows - 1) / kTcRows;
    const unsigned grid = (unsigned)std::max<long>(1, std::min<long>((ntiles + kTcGroups - 1) / kTcGroups, 148));
    k_sur_mlp_tc<<<grid, kTcRows * kTcGroups, kTcSmem, h->stream>>>(net_of(s), s.nrm, X, pred, mpad, h->status);
    CK(cudaGetLastError());
    return 0;
}

}  // namespace

int sur_create(lbmgpu *h) {
    if (h->sur) return 0;
    if (h->ns != 9) return LBMGPU_E_UNSUPPORTED;
    SurState *s = new SurState();
    h->sur = s;
    int rc = 0;
    if (!rc) rc = dalloc(h, &s->w, kNParams);
    if (!rc) rc = dalloc(h, &s->m, kNParams);
    if (!rc) rc = dalloc(h, &s->v, kNParams);
    if (!rc) rc = dalloc(h, &s->g, kNParams);
    if (!rc) rc = dalloc(h, &s->wb, off_w(4));
    if (!rc) rc = dalloc(h, &s->nrm, 1);
    if (!rc) rc = dalloc(h, &s->proj, 9 * 9);
    if (!rc) rc = dalloc(h, &s->audit, 6);
    if (rc) return rc;
    CK(cudaMemsetAsync(s->g, 0, kNParams * sizeof(float), h->stream));
    CK(cudaMemsetAsync(s->audit, 0, 6 * sizeof(double), h->stream));
    default_norm(s->nrm_h);
    CK(cudaMemcpyAsync(s->nrm, &s->nrm_h, sizeof(SurNorm), cudaMemcpyHostToDevice, h->stream));
    double el[9][LBMGPU_MAX_ELEMENTS], W[9], proj[9 * 9];
    for (int k = 0; k < 9; ++k) {
        W[k] = h->mech.W[k];
        for (int e = 0; e < LBMGPU_MAX_ELEMENTS; ++e) el[k][e] = h->mech.elements[k][e];
    }
    sur_projector<9>(el, W, proj);
    CK(cudaMemcpyAsync(s->proj, proj, sizeof proj, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return init_params(h, 20261203u);
}

void sur_release(lbmgpu *h) {
    SurState *s = h->sur;
    if (!s) return;
    cudaFree(s->w);
    cudaFree(s->m);
    cudaFree(s->v);
    cudaFree(s->g);
    cudaFree(s->wb);
    cudaFree(s->nrm);
    cudaFree(s->proj);
    cudaFree(s->audit);
    cudaFree(s->ds_x);
    cudaFree(s->ds_y);
    cudaFree(s->ds_valid);
    cudaFree(s->feat);
    cudaFree(s->gate);
    cudaFree(s->pred);
    cudaFree(s->ilist);
    cudaFree(s->icount);
    delete s;
    h->sur = nullptr;
}

// Fills the per-step surrogate arguments of the collision-parameter kernel; with the
// surrogate on, computes every cell's features and the network's predictions first.
template <typename S>
int sur_prepare_t(lbmgpu *h, McArgsT<S, double> &A) {
    SurArgs &a = A.sur;
    std::memset(&a, 0, sizeof a);
    SurState *s = h->sur;
    if (!s || h->chem != CHEM_ROSENBROCK) return 0;
    a.proj = s->proj;
    a.audit = s->audit;
    a.audit_period = s->audit_period;
    a.audit_phase = s->audit_period ? (unsigned)((7919ull * s->step) % s->audit_period) : 0u;
    a.step = s->step;
    a.dt_si = (double)h->d.dt_sim * (double)h->U.s;
    if (s->collect && s->ds_x) {
        a.ds_x = s->ds_x;
        a.ds_y = s->ds_y;
        a.ds_valid = s->ds_valid;
        a.ds_cap = s->ds_cap;
        // surrogate steps collect on the audit stride (the states the integrator takes
        // anyway), teacher steps on the collection stride
        const bool online = s->enabled && s->audit_period > 0;
        s->step_stride = online ? (int)s->audit_period : s->stride;
        a.ds_stride = s->step_stride;
        a.ds_phase = online ? (int)a.audit_phase : (int)((7L * s->collect_steps) % s->stride);
        a.ds_base = s->ds_next;
    }
    if (s->enabled) {
        const long mpad = ((h->g.ncell + 15) / 16) * 16;
        if (mpad != s->mpad) {
            cudaFree(s->feat);
            cudaFree(s->gate);
            cudaFree(s->pred);
            cudaFree(s->ilist);
            cudaFree(s->icount);
            s->feat = nullptr;
            s->gate = nullptr;
            s->pred = nullptr;
            s->ilist = nullptr;
            s->icount = nullptr;
            int rc = dalloc(h, &s->feat, (size_t)mpad * kSurInX);
            if (!rc) rc = dalloc(h, &s->gate, (size_t)mpad);
            if (!rc) rc = dalloc(h, &s->pred, (size_t)mpad * kSurOutPad);
            if (!rc) rc = dalloc(h, &s->ilist, (size_t)mpad);
            if (!rc) rc = dalloc(h, &s->icount, 1);
            if (rc) return rc;
            s->mpad = mpad;
        }
        EvPair ep{};
        ev_begin(h, K_SURROGATE, ep);
        k_sur_features<9, S><<<blocks(mpad, 128), 128, 0, h->stream>>>(A, s->nrm, s->feat, s->gate, mpad);
        CK(cudaGetLastError());
        const int rc = run_mlp(h, s->feat, s->pred, mpad);
        ev_end(h, ep);
        if (rc) return rc;
        CK(cudaMemsetAsync(s->icount, 0, sizeof(unsigned), h->stream));
        a.mode = 1;
        a.pred = s->pred;
        a.gate = s->gate;
        a.nrm = s->nrm;
        a.ilist = s->ilist;
        a.icount = s->icount;
    }
    return 0;
}
template int sur_prepare_t<double>(lbmgpu *, McArgsT<double, double> &);
template int sur_prepare_t<float>(lbmgpu *, McArgsT<float, double> &);

void sur_after_step(lbmgpu *h) {
    SurState *s = h->sur;
    if (!s || h->chem != CHEM_ROSENBROCK) return;
    if (s->collect && s->ds_x) {
        s->ds_next += (h->g.ncell + s->step_stride - 1) / s->step_stride;
        s->collect_steps += 1;
        if (s->ds_next >= s->ds_cap) s->collect = 0;  // full
    }
    s->step += 1;
}

}  // namespace lbmh

using namespace lbmh;

namespace {

int sur_check(lbmgpu *h) {
    if (!h) return LBMGPU_E_ARG;
    if (h->ns == 0) return LBMGPU_E_UNSUPPORTED;
    CK(cudaSetDevice(h->d.device));
    return sur_create(h);
}

// Standardisation from the valid samples: mean and standard deviation per feature and
// target (floor 1e-12 of the mean's scale, 1 for a constant feature), the feature box.
int fit_norm(lbmgpu *h, long n) {
    SurState &s = *h->sur;
    std::vector<float> x((size_t)n * kSurIn), y((size_t)n * kSurOut);
    std::vector<uint8_t> v(n);
    CK(cudaMemcpyAsync(x.data(), s.ds_x, x.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(y.data(), s.ds_y, y.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(v.data(), s.ds_valid, n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    SurNorm &N = s.nrm_h;
    default_norm(N);
    long cnt = 0;
    std::vector<double> sx(kSurIn, 0.0), sxx(kSurIn, 0.0), sy(kSurOut, 0.0), syy(kSurOut, 0.0);
    std::vector<double> lo(kSurIn, 1e300), hi(kSurIn, -1e300);
    for (long r = 0; r < n; ++r) {
        if (!v[r]) continue;
        ++cnt;
        for (int q = 0; q < kSurIn; ++q) {
            const double a = x[r * kSurIn + q];
            sx[q] += a;
            sxx[q] += a * a;
            lo[q] = std::min(lo[q], a);
            hi[q] = std::max(hi[q], a);
        }
        for (int q = 0; q < kSurOut; ++q) {
            const double a = y[r * kSurOut + q];
            sy[q] += a;
            syy[q] += a * a;
        }
    }
    if (cnt < 2) return LBMGPU_E_STATE;
    for (int q = 0; q < kSurIn; ++q) {
        const double mu = sx[q] / cnt, var = std::max(0.0, sxx[q] / cnt - mu * mu);
        N.x_mean[q] = (float)mu;
        N.x_std[q] = var > 1e-24 * (mu * mu + 1e-300) ? (float)std::sqrt(var) : 1.f;
        N.x_lo[q] = (float)lo[q];
        N.x_hi[q] = (float)hi[q];
    }
    for (int q = 0; q < kSurOut; ++q) {
        const double mu = sy[q] / cnt, var = std::max(0.0, syy[q] / cnt - mu * mu);
        N.y_mean[q] = (float)mu;
        N.y_std[q] = var > 0.0 ? (float)std::sqrt(var) : 1.f;
    }
    CK(cudaMemcpyAsync(s.nrm, &N, sizeof(SurNorm), cudaMemcpyHostToDevice, h->stream));
    return 0;
}

int ensure_samples(lbmgpu *h, long cap) {
    SurState &s = *h->sur;
    if (s.ds_cap >= cap && s.ds_x) return 0;
    cudaFree(s.ds_x);
    cudaFree(s.ds_y);
    cudaFree(s.ds_valid);
    s.ds_x = s.ds_y = nullptr;
    s.ds_valid = nullptr;
    int rc = dalloc(h, &s.ds_x, (size_t)cap * kSurIn);
    if (!rc) rc = dalloc(h, &s.ds_y, (size_t)cap * kSurOut);
    if (!rc) rc = dalloc(h, &s.ds_valid, (size_t)cap);
    if (rc) return rc;
    CK(cudaMemsetAsync(s.ds_valid, 0, (size_t)cap, h->stream));
    s.ds_cap = cap;
    s.ds_next = 0;
    return 0;
}

// Grows the sample set to at least cap rows, keeping the rows written so far.
int grow_samples(lbmgpu *h, long cap) {
    SurState &s = *h->sur;
    if (s.ds_cap >= cap && s.ds_x) return 0;
    const long keep = s.ds_x ? std::min(s.ds_next, s.ds_cap) : 0;
    float *x = nullptr, *y = nullptr;
    uint8_t *v = nullptr;
    int rc = dalloc(h, &x, (size_t)cap * kSurIn);
    if (!rc) rc = dalloc(h, &y, (size_t)cap * kSurOut);
    if (!rc) rc = dalloc(h, &v, (size_t)cap);
    if (rc) {
        cudaFree(x);
        cudaFree(y);
        cudaFree(v);
        return rc;
    }
    CK(cudaMemsetAsync(v, 0, (size_t)cap, h->stream));
    if (keep) {
        CK(cudaMemcpyAsync(x, s.ds_x, (size_t)keep * kSurIn * 4, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(y, s.ds_y, (size_t)keep * kSurOut * 4, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(v, s.ds_valid, (size_t)keep, cudaMemcpyDeviceToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(s.ds_x);
    cudaFree(s.ds_y);
    cudaFree(s.ds_valid);
    s.ds_x = x;
    s.ds_y = y;
    s.ds_valid = v;
    s.ds_cap = cap;
    s.ds_next = keep;
    return 0;
}

}  // namespace

extern "C" {

int lbmgpu_surrogate_collect(lbmgpu_t *h, int enable, int stride, long capacity) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (h->chem != CHEM_ROSENBROCK) return LBMGPU_E_UNSUPPORTED;
    SurState &s = *h->sur;
    if (!enable) {
        s.collect = 0;
        return LBMGPU_OK;
    }
    if (stride < 1 || capacity < 16) return LBMGPU_E_ARG;
    rc = grow_samples(h, capacity);  // keeps the rows collected so far
    if (rc) return rc;
    s.stride = stride;
    s.collect = s.ds_next < s.ds_cap ? 1 : 0;
    return LBMGPU_OK;
}

int lbmgpu_surrogate_load_samples(lbmgpu_t *h, const float *x, const float *y, long n) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (!x || !y || n < 2) return LBMGPU_E_ARG;
    rc = ensure_samples(h, n);
    if (rc) return rc;
    SurState &s = *h->sur;
    CK(cudaMemcpyAsync(s.ds_x, x, (size_t)n * kSurIn * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(s.ds_y, y, (size_t)n * kSurOut * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(s.ds_valid, 1, (size_t)n, h->stream));
    if (s.ds_cap > n) CK(cudaMemsetAsync(s.ds_valid + n, 0, (size_t)(s.ds_cap - n), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    s.ds_next = n;
    s.collect = 0;
    return LBMGPU_OK;
}

int lbmgpu_surrogate_samples(lbmgpu_t *h, float *x, float *y, unsigned char *valid, long n) {
    int rc = sur_check(h);
    if (rc) return rc;
    SurState &s = *h->sur;
    if (n < 0 || n > std::min(s.ds_next, s.ds_cap) || (n > 0 && (!x || !y || !valid))) return LBMGPU_E_ARG;
    if (n == 0) return LBMGPU_OK;
    CK(cudaMemcpyAsync(x, s.ds_x, (size_t)n * kSurIn * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(y, s.ds_y, (size_t)n * kSurOut * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(valid, s.ds_valid, (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

int lbmgpu_surrogate_augment(lbmgpu_t *h, long n, float span_y, float span_t, float y_trace, unsigned seed) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (h->chem != CHEM_ROSENBROCK) return LBMGPU_E_UNSUPPORTED;
    SurState &s = *h->sur;
    if (n < 1 || !(span_y >= 0.f) || !(span_t >= 0.f) || !(y_trace >= 0.f)) return LBMGPU_E_ARG;
    const long n_rows = s.ds_x ? std::min(s.ds_next, s.ds_cap) : 0;
    if (n_rows < 1) return LBMGPU_E_STATE;
    std::vector<uint8_t> v(n_rows);
    CK(cudaMemcpyAsync(v.data(), s.ds_valid, n_rows, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> src;
    for (long r = 0; r < n_rows; ++r)
        if (v[r]) src.push_back((int)r);
    if (src.empty()) return LBMGPU_E_STATE;
    rc = grow_samples(h, n_rows + n);
    if (rc) return rc;
    int *src_d = nullptr;
    rc = dalloc(h, &src_d, src.size());
    if (rc) return rc;
    CK(cudaMemcpyAsync(src_d, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    k_sur_augment<<<blocks(n, 128), 128, 0, h->stream>>>(h->tab, s.ds_x, s.ds_y, s.ds_valid, src_d, (long)src.size(),
                                                         n_rows, n, span_y, span_t, y_trace, seed);
    const cudaError_t e = cudaGetLastError();
    const cudaError_t e2 = cudaStreamSynchronize(h->stream);
    cudaFree(src_d);
    CK(e);
    CK(e2);
    s.ds_next = n_rows + n;
    s.collect = 0;
    return LBMGPU_OK;
}

int lbmgpu_surrogate_train(lbmgpu_t *h, int epochs, int batch, float lr, unsigned seed, int refit, double *loss) {
    int rc = sur_check(h);
    if (rc) return rc;
    SurState &s = *h->sur;
    if (epochs < 0 || batch < 64 || batch % 64 || !(lr > 0.f)) return LBMGPU_E_ARG;
    const long n = std::min(s.ds_next, s.ds_cap);
    if (!s.ds_x || n < 2) return LBMGPU_E_STATE;
    if (refit || !s.trained) {
        rc = fit_norm(h, n);
        if (rc) return rc;
    }
    // valid rows, shuffled per epoch with a seeded generator
    std::vector<uint8_t> v(n);
    CK(cudaMemcpyAsync(v.data(), s.ds_valid, n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> rows;
    for (long r = 0; r < n; ++r)
        if (v[r]) rows.push_back((int)r);
    if (rows.size() < 2) return LBMGPU_E_STATE;
    const int B = batch;
    // batch buffers
    int *idx = nullptr;
    __nv_bfloat16 *Xb = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr, *dZb = nullptr, *T1 = nullptr,
                  *T2 = nullptr, *Wt = nullptr;
    float *Yb = nullptr, *C = nullptr, *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *dA = nullptr, *dZ = nullptr;
    uint8_t *vb = nullptr;
    double *part = nullptr;
    const long BH = (long)B * kSurHid;
    const unsigned nparts = blocks((long)B * kSurOutPad);
    const long nbatch = ((long)rows.size() + B - 1) / B, total = std::max<long>(1, (long)epochs * nbatch);
    int ksplit = 1;  // slices of the batch for the weight gradients: each a multiple of 16 rows
    for (int c : {32, 16, 8, 4, 2})
        if ((B / 16) % c == 0) {
            ksplit = c;
            break;
        }
    float *Gp = nullptr;  // the weight gradients' split-K partials
    auto all = [&]() {
        int r = dalloc(h, &idx, rows.size());
        if (!r) r = dalloc(h, &Xb, (size_t)B * kSurInX);
        if (!r) r = dalloc(h, &Yb, (size_t)B * kSurOutPad);
        if (!r) r = dalloc(h, &vb, B);
        if (!r) r = dalloc(h, &H1, BH);
        if (!r) r = dalloc(h, &H2, BH);
        if (!r) r = dalloc(h, &H3, BH);
        if (!r) r = dalloc(h, &Z1, BH);
        if (!r) r = dalloc(h, &Z2, BH);
        if (!r) r = dalloc(h, &Z3, BH);
        if (!r) r = dalloc(h, &C, BH);
        if (!r) r = dalloc(h, &dA, BH);
        if (!r) r = dalloc(h, &dZ, BH);
        if (!r) r = dalloc(h, &dZb, BH);
        if (!r) r = dalloc(h, &T1, BH);
        if (!r) r = dalloc(h, &T2, BH);
        if (!r) r = dalloc(h, &Wt, (size_t)kSurHid * kSurLd);
        if (!r) r = dalloc(h, &part, (size_t)nparts * nbatch);
        if (!r) r = dalloc(h, &Gp, (size_t)ksplit * kSurHid * kSurLd);
        if (!r && cudaMemsetAsync(Gp, 0, (size_t)ksplit * kSurHid * kSurLd * sizeof(float), h->stream)) r = LBMGPU_E_CUDA;
        return r;
    };
    rc = all();
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    SurNet net = net_of(s);
    double epoch_loss = 0.0;
    const int ldw[4] = {kSurInPad, kSurLd, kSurLd, kSurLd};
    const int kin[4] = {kSurInPad, kSurHid, kSurHid, kSurHid};
    const int nout[4] = {kSurHid, kSurHid, kSurHid, kSurOutPad};
    dim3 tb(32, 8);
    // the step size decays from lr to 0 along a half cosine over the call's Adam steps
    long step_in_call = 0;
    std::vector<double> parts((size_t)nparts * nbatch);
    for (int ep = 0; ep < epochs && !rc; ++ep) {
        // the epoch's order in one copy; the batches run without waiting for the host, and
        // the per-batch squared-error partials come back once at the end of the epoch
        std::shuffle(rows.begin(), rows.end(), rng);
        if (cudaMemcpyAsync(idx, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream)) {
            rc = LBMGPU_E_CUDA;
            break;
        }
        long sum_n = 0;
        long bi = 0;
        for (size_t b0 = 0; b0 < rows.size() && !rc; b0 += B, ++bi) {
            const int nb = (int)std::min<size_t>(B, rows.size() - b0);
            k_gather_batch<<<blocks(B), 256, 0, h->stream>>>(s.ds_x, s.ds_y, idx + b0, nb, B, s.nrm, Xb, Yb, vb);
            // forward
            const __nv_bfloat16 *in = Xb;
            __nv_bfloat16 *Hs[3] = {H1, H2, H3};
            float *Zs[3] = {Z1, Z2, Z3};
            const __nv_bfloat16 *Ws[4] = {net.w1, net.w2, net.w3, net.w4};
            const float *bs[4] = {net.b1, net.b2, net.b3, net.b4};
            for (int L = 0; L < 3; ++L) {
                gemm_tn(h, in, L == 0 ? kSurInX : kSurHid, Ws[L], ldw[L], C, kSurHid, B, nout[L], kin[L]);
                if (L == 0)  // the remainders' share of the first layer
                    gemm_tn(h, Xb + kSurInPad, kSurInX, Ws[0], ldw[0], C, kSurHid, B, nout[0], kin[0], 1);
                k_bias_gelu<<<blocks(BH), 256, 0, h->stream>>>(C, bs[L], Zs[L], Hs[L], B, kSurHid);
                in = Hs[L];
            }
            gemm_tn(h, H3, kSurHid, net.w4, kSurLd, C, kSurOutPad, B, kSurOutPad, kSurHid);
            k_out_loss<<<nparts, 256, 0, h->stream>>>(C, net.b4, Yb, vb, (float)nb, dA, part + (size_t)bi * nparts, B);
            // backward: dA holds dL/d(pre-activation) of the current layer (FP32), rows x nout
            float *gw[4] = {s.g + off_w(0), s.g + off_w(1), s.g + off_w(2), s.g + off_w(3)};
            float *gb[4] = {s.g + off_w(4), s.g + off_w(5), s.g + off_w(6), s.g + off_w(7)};
            for (int L = 3; L >= 0; --L) {
                const int no = nout[L], ki = kin[L];
                // bias gradient
                k_colsum<<<(no + 31) / 32, 32 * kColsumWarps, 0, h->stream>>>(dA, B, no, gb[L]);
                // dZ^T [no][B] and input^T [ki][B] for the weight gradient dW = dZ^T in
                k_f32_to_bf16<<<blocks((long)B * no), 256, 0, h->stream>>>(dA, dZb, (long)B * no);
                k_transpose_bf16<<<dim3((no + 31) / 32, (B + 31) / 32), tb, 0, h->stream>>>(dZb, no, T1, B, B, no);
                const __nv_bfloat16 *inp = L == 0 ? Xb : Hs[L - 1];
                k_transpose_bf16<<<dim3((ki + 31) / 32, (B + 31) / 32), tb, 0, h->stream>>>(
                    inp, L == 0 ? kSurInX : kSurHid, T2, B, B, ki);  // layer 0: the values' columns
                // split K (the batch) so the small weight-gradient tile keeps every SM busy
                const long gsz = (long)no * ldw[L];
                gemm_tn(h, T1, B, T2, B, Gp, ldw[L], no, ki, B, 0, ksplit, gsz);
                k_sum_splits<<<blocks(gsz), 256, 0, h->stream>>>(Gp, ksplit, gsz, ki, ldw[L], gw[L]);
                if (L == 0) break;
                // dH_prev = dZ W  (W^T [ki][no] as the B operand), then through GELU'
                k_transpose_bf16<<<dim3((ki + 31) / 32, (no + 31) / 32), tb, 0, h->stream>>>(Ws[L], ldw[L], Wt, kSurLd,
                                                                                              no, ki);
                gemm_tn(h, dZb, no, Wt, kSurLd, C, kSurHid, B, ki, no);
                k_gelu_bwd<<<blocks(BH), 256, 0, h->stream>>>(C, Zs[L - 1], dA, T1, BH);
            }
            // Adam step over every parameter (padding entries have zero gradient)
            s.adam_t += 1;
            const float lr_t =
                (float)(0.5 * lr * (1.0 + std::cos(3.14159265358979323846 * (double)step_in_call / (double)total)));
            ++step_in_call;
            const float c1 = 1.f - (float)std::pow(b1, (double)s.adam_t), c2 = 1.f - (float)std::pow(b2, (double)s.adam_t);
            for (int t = 0; t < 8; ++t) {
                const size_t sz[8] = {kW1, kW2, kW2, kW4, kSurHid, kSurHid, kSurHid, kSurOutPad};
                const size_t o = off_w(t);
                k_adam<<<blocks((long)sz[t]), 256, 0, h->stream>>>(s.w + o, s.m + o, s.v + o, s.g + o,
                                                                   t < 4 ? s.wb + o : nullptr, (long)sz[t], lr_t, b1, b2,
                                                                   c1, c2, eps);
            }
            if (cudaGetLastError() != cudaSuccess) {
                rc = LBMGPU_E_CUDA;
                break;
            }
            sum_n += (long)nb * kSurOut;
            s.train_steps += 1;
        }
        if (rc) break;
        if (cudaMemcpyAsync(parts.data(), part, (size_t)nparts * bi * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream) ||
            cudaStreamSynchronize(h->stream)) {
            rc = LBMGPU_E_CUDA;
            break;
        }
        double sum_se = 0.0;
        for (long q = 0; q < (long)nparts * bi; ++q) sum_se += parts[q];
        epoch_loss = sum_n ? sum_se / sum_n : 0.0;
    }
    cudaFree(idx);
    cudaFree(Xb);
    cudaFree(Yb);
    cudaFree(vb);
    cudaFree(H1);
    cudaFree(H2);
    cudaFree(H3);
    cudaFree(Z1);
    cudaFree(Z2);
    cudaFree(Z3);
    cudaFree(C);
    cudaFree(dA);
    cudaFree(dZ);
    cudaFree(dZb);
    cudaFree(T1);
    cudaFree(T2);
    cudaFree(Wt);
    cudaFree(part);
    cudaFree(Gp);
    if (rc) return rc;
    s.trained = true;
    s.last_loss = epoch_loss;
    if (loss) *loss = epoch_loss;
    return LBMGPU_OK;
}

int lbmgpu_surrogate_enable(lbmgpu_t *h, int enable, int audit_period) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (h->chem != CHEM_ROSENBROCK) return LBMGPU_E_UNSUPPORTED;
    if (audit_period < 0) return LBMGPU_E_ARG;
    SurState &s = *h->sur;
    if (enable && !s.trained) return LBMGPU_E_STATE;
    s.enabled = enable ? 1 : 0;
    s.audit_period = (unsigned)audit_period;
    CK(cudaMemsetAsync(s.audit, 0, 6 * sizeof(double), h->stream));  // the report counts from here
    return LBMGPU_OK;
}

int lbmgpu_surrogate_eval(lbmgpu_t *h, const float *x, long n, float *y) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (!x || !y || n < 1) return LBMGPU_E_ARG;
    SurState &s = *h->sur;
    const long mpad = ((n + 15) / 16) * 16;
    float *xd = nullptr, *pd = nullptr;
    __nv_bfloat16 *X = nullptr;
    rc = dalloc(h, &xd, (size_t)n * kSurIn);
    if (!rc) rc = dalloc(h, &X, (size_t)mpad * kSurInX);
    if (!rc) rc = dalloc(h, &pd, (size_t)mpad * kSurOutPad);
    if (!rc && cudaMemcpyAsync(xd, x, (size_t)n * kSurIn * 4, cudaMemcpyHostToDevice, h->stream)) rc = LBMGPU_E_CUDA;
    if (!rc) {
        k_sur_standardise<<<blocks(mpad), 256, 0, h->stream>>>(xd, n, mpad, s.nrm, X);
        rc = run_mlp(h, X, pd, mpad);
    }
    std::vector<float> out;
    if (!rc) {
        out.resize((size_t)mpad * kSurOutPad);
        if (cudaMemcpyAsync(out.data(), pd, out.size() * 4, cudaMemcpyDeviceToHost, h->stream) ||
            cudaStreamSynchronize(h->stream))
            rc = LBMGPU_E_CUDA;
    }
    cudaFree(xd);
    cudaFree(X);
    cudaFree(pd);
    if (rc) return rc;
    for (long r = 0; r < n; ++r)
        for (int q = 0; q < kSurOut; ++q) y[r * kSurOut + q] = out[r * kSurOutPad + q];
    return LBMGPU_OK;
}

int lbmgpu_surrogate_params(lbmgpu_t *h, float *buf, long n, int set) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (!buf || n < LBMGPU_SUR_NPARAMS) return LBMGPU_E_ARG;
    SurState &s = *h->sur;
    // packed layout: W1 [128][12], b1, W2 [128][128], b2, W3, b3, W4 [10][128], b4 [10],
    // x_mean [12], x_std [12], x_lo [12], x_hi [12], y_mean [10], y_std [10]
    std::vector<float> w(kNParams);
    CK(cudaMemcpyAsync(w.data(), s.w, kNParams * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int rows[4] = {kSurHid, kSurHid, kSurHid, kSurOut};
    const int cols[4] = {kSurIn, kSurHid, kSurHid, kSurHid};
    const int ld[4] = {kSurInPad, kSurLd, kSurLd, kSurLd};
    const int nb[4] = {kSurHid, kSurHid, kSurHid, kSurOut};
    long p = 0;
    for (int t = 0; t < 4; ++t) {
        for (int r = 0; r < rows[t]; ++r)
            for (int k = 0; k < cols[t]; ++k, ++p) {
                float &d = w[off_w(t) + (size_t)r * ld[t] + k];
                if (set) d = buf[p]; else buf[p] = d;
            }
        for (int r = 0; r < nb[t]; ++r, ++p) {
            float &d = w[off_w(4 + t) + r];
            if (set) d = buf[p]; else buf[p] = d;
        }
    }
    SurNorm &N = s.nrm_h;
    float *fields[6] = {N.x_mean, N.x_std, N.x_lo, N.x_hi, N.y_mean, N.y_std};
    const int len[6] = {kSurIn, kSurIn, kSurIn, kSurIn, kSurOut, kSurOut};
    for (int f = 0; f < 6; ++f)
        for (int q = 0; q < len[f]; ++q, ++p) {
            if (set) fields[f][q] = buf[p]; else buf[p] = fields[f][q];
        }
    if (set) {
        CK(cudaMemcpyAsync(s.w, w.data(), kNParams * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(s.nrm, &N, sizeof(SurNorm), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemsetAsync(s.m, 0, kNParams * sizeof(float), h->stream));
        CK(cudaMemsetAsync(s.v, 0, kNParams * sizeof(float), h->stream));
        s.adam_t = 0;
        rc = upload_params(h);
        if (rc) return rc;
        CK(cudaStreamSynchronize(h->stream));
        s.trained = true;
    }
    return LBMGPU_OK;
}

int lbmgpu_surrogate_grads(lbmgpu_t *h, float *buf, long n) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (!buf || n < LBMGPU_SUR_NPARAMS) return LBMGPU_E_ARG;
    SurState &s = *h->sur;
    if (s.train_steps == 0) return LBMGPU_E_STATE;
    // the gradient buffer of the last minibatch, in the packed parameter layout
    std::vector<float> g(kNParams);
    CK(cudaMemcpyAsync(g.data(), s.g, kNParams * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int rows[4] = {kSurHid, kSurHid, kSurHid, kSurOut};
    const int cols[4] = {kSurIn, kSurHid, kSurHid, kSurHid};
    const int ld[4] = {kSurInPad, kSurLd, kSurLd, kSurLd};
    const int nb[4] = {kSurHid, kSurHid, kSurHid, kSurOut};
    long p = 0;
    for (int t = 0; t < 4; ++t) {
        for (int r = 0; r < rows[t]; ++r)
            for (int k = 0; k < cols[t]; ++k, ++p) buf[p] = g[off_w(t) + (size_t)r * ld[t] + k];
        for (int r = 0; r < nb[t]; ++r, ++p) buf[p] = g[off_w(4 + t) + r];
    }
    for (; p < LBMGPU_SUR_NPARAMS; ++p) buf[p] = 0.f;
    return LBMGPU_OK;
}

int lbmgpu_surrogate_stats(lbmgpu_t *h, lbmgpu_surrogate_report *out) {
    int rc = sur_check(h);
    if (rc) return rc;
    if (!out) return LBMGPU_E_ARG;
    SurState &s = *h->sur;
    double a[6];
    CK(cudaMemcpyAsync(a, s.audit, sizeof a, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    out->samples = std::min(s.ds_next, s.ds_cap);
    out->train_steps = s.train_steps;
    out->last_loss = s.last_loss;
    out->cells_audited = (long)a[3];
    out->cells_predicted = (long)a[4];
    out->cells_integrated = (long)a[5];
    out->audit_rel_err = a[1] > 0 ? a[0] / a[1] : 0.0;
    out->audit_max_abs_err = a[2];
    out->audit_dY = a[1];
    out->enabled = s.enabled;
    out->collecting = s.collect;
    return LBMGPU_OK;
}

}  // extern "C"
