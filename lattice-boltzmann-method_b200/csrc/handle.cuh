// The lbmgpu handle: device state of one LBM object plus the host-side helpers shared by
// the single-component (lbmgpu.cu) and multicomponent (mc.cu) translation units.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "../../include/lbmgpu.h"
#include "gas.cuh"
#include "sc_kernels.cuh"
#include "units.cuh"

namespace lbmh {

struct SurState;  // chemistry surrogate (surrogate.cu)
constexpr int kBlock = 128;

enum Phase { PH_BOUNDARY = 0, PH_COLLIDED = 1, PH_STREAMED = 2, PH_BC = 3, PH_SPECIES = 4 };
// per-kernel timing classes; multicomponent: K_COLLIDE is the population update
// (k_mc_relax), K_STREAM_MOMENT the pull and population sums of the interior cells
// (k_mc_gather), K_PROPS the collision parameters (k_mc_props), K_SURROGATE the chemistry
// surrogate's features, network and integrator list, K_SOLVE the interior cells' moment
// solve (k_mc_solve), K_EFLUX the energy-flux terms of the collision (k_mc_eflux), K_CHEM
// the stiff chemistry of every cell (k_mc_chem, ROS2 without the surrogate)
enum KernelKind {
    K_COLLIDE = 0, K_STREAM_MOMENT = 1, K_OTHER = 2, K_PROPS = 3, K_SURROGATE = 4, K_SOLVE = 5, K_EFLUX = 6,
    K_CHEM = 7, K_NKINDS = 8
};
// The stiff chemistry's kinetics: the mechanism tables (any mechanism), or the H2/air
// mechanism compiled to straight-line code (kinetics_h2_air_9.cuh) when the handle's
// mechanism is that one.
enum Kinetics : int { KIN_TABLES = 0, KIN_H2_AIR_9 = 1 };
// What pop[cur] holds: the uploaded populations, the ones Init built, or post-collision
// values after at least one step.
enum PackMode : int { PK_UPLOADED = 0, PK_INIT = 1, PK_STEPPED = 2 };

struct EvPair {
    cudaEvent_t a, b;
    int kind;
};

// Byte offsets of the caller's MIXTURE fields (-1: absent).
struct MixOff {
    long size, type, f, fpc, p_tensor, rho, u, v, w, p, g, gpc, rhoe, energy_flux, temp, HRR;
};
struct SpOff {
    long size, X, rho, f, fpc, u, v, w;
};

}  // namespace lbmh

struct lbmgpu {
    lbmgpu_desc d{};
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;           // multicomponent: the boundary cells beside the interior
    cudaEvent_t fork = nullptr, join = nullptr;
    lbm::ScGeom g{};
    lbm::ScPhys P{};
    lbmh::MixOff mo{};
    lbmh::SpOff so{};
    int8_t *type = nullptr;
    uint8_t *cflag = nullptr;
    int *bid = nullptr;
    long *blist = nullptr;
    long nb = 0;
    double *pop[2] = {nullptr, nullptr};
    double *mom[2] = {nullptr, nullptr};  // single component: the step record; multicomponent: rec
    double *bst[2] = {nullptr, nullptr};
    unsigned *status = nullptr;
    char *stage = nullptr;
    size_t stage_cells = 0;
    size_t stage_bytes = 0;
    char *bounce = nullptr;  // pinned host bounce buffers for downloads (the second lets the
    char *bounce2 = nullptr; //   device pack the next chunk while the host merges one)
    int cur = 0;
    int pack_mode = lbmh::PK_UPLOADED;
    bool have_state = false;
    int phase = lbmh::PH_BOUNDARY;
    bool prof = false;
    std::vector<lbmh::EvPair> pending, pool;
    long launches[lbmh::K_NKINDS] = {};
    double ms[lbmh::K_NKINDS] = {};
    size_t bytes = 0;
    // multicomponent
    int ns = 0;
    int nrec = 0;
    int chem = 0;
    lbm::UnitsF U{};
    gas::Tables *tab = nullptr;  // device copy
    bool fp32 = false;           // FP32 population storage: pop32 instead of pop
    float *pop32[2] = {nullptr, nullptr};
    float *bst32[2] = {nullptr, nullptr};
    double *shift[2] = {nullptr, nullptr};  // FP32: per-plane population shift (current, scratch)
    double *sum_scratch = nullptr;          // lbmgpu_sums: block partials and totals
    double *props = nullptr;                // multicomponent collision parameters
    double *gsum = nullptr;                 // multicomponent: the interior cells' population sums
    lbmh::SurState *sur = nullptr;          // chemistry surrogate, created on first use
    lbmgpu_mech mech{};                     // multicomponent: the caller's mechanism, copied at create
    int kin = 0;                            // KIN_*: the stiff chemistry's kinetics
    long nfluid = 0;
    // plane-range uploads (multicomponent): the cell types on the host, and which x-planes
    // have arrived since the last complete upload
    std::vector<int8_t> htype;
    std::vector<char> plane_have;
    int planes_have = 0;
    // slab decomposition along x (lbmgpu_set_halo): halo planes and the global x length
    int halo_lo = 0, halo_hi = 0, nx_glob = 0;
};

namespace lbmh {

inline int cuda_fail(cudaError_t e) {
    (void)cudaGetLastError();
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDevice || e == cudaErrorNoDevice ||
        e == cudaErrorInsufficientDriver)
        return LBMGPU_E_NODEV;
    return LBMGPU_E_CUDA;
}

#define CK(x)                                        \
    do {                                             \
        cudaError_t e_ = (x);                        \
        if (e_ != cudaSuccess) return lbmh::cuda_fail(e_); \
    } while (0)

template <typename T>
int dalloc(lbmgpu *h, T **p, size_t count) {
    CK(cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)));
    h->bytes += count * sizeof(T);
    return 0;
}

inline void ev_begin(lbmgpu *h, int kind, EvPair &ep, cudaStream_t st = nullptr) {
    if (!h->prof) return;
    if (h->pool.empty()) {
        EvPair e{};
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
        h->pool.push_back(e);
    }
    ep = h->pool.back();
    h->pool.pop_back();
    ep.kind = kind;
    cudaEventRecord(ep.a, st ? st : h->stream);
}

inline void ev_end(lbmgpu *h, EvPair &ep, cudaStream_t st = nullptr) {
    if (!h->prof) return;
    cudaEventRecord(ep.b, st ? st : h->stream);
    h->pending.push_back(ep);
}

inline void ev_drain(lbmgpu *h) {
    for (auto &e : h->pending) {
        float t = 0.f;
        if (cudaEventSynchronize(e.b) == cudaSuccess && cudaEventElapsedTime(&t, e.a, e.b) == cudaSuccess) {
            h->ms[e.kind] += t;
            h->launches[e.kind] += 1;
        }
        h->pool.push_back(e);
    }
    h->pending.clear();
}

// f(lo, hi) over [0, n) split into contiguous ranges, one per host thread (up to the
// machine's hardware threads, at most 32; ranges of at least min_items items).
template <class F>
void host_parallel_for(long n, const F &f, long min_items = 1024) {
    const long hw = std::max(1L, (long)std::thread::hardware_concurrency());
    const long nt = std::max(1L, std::min(std::min(hw, 32L), n / std::max(1L, min_items)));
    if (nt == 1) {
        f(0L, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (long t = 1; t < nt; ++t) th.emplace_back([&f, n, nt, t] { f(n * t / nt, n * (t + 1) / nt); });
    f(0L, n / nt);
    for (auto &x : th) x.join();
}

// Whether host memory at p is page-locked (registered or allocated by CUDA).
inline bool host_pinned(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

inline unsigned grid_for(long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

// multicomponent entry points (mc.cu)
int mc_setup(lbmgpu *h);
int mc_upload(lbmgpu *h, const void *mix, const void *const *species);
int mc_download(lbmgpu *h, void *mix, void *const *species);
int mc_upload_planes(lbmgpu *h, int i0, int i1, const void *mix, const void *const *species);
int mc_halo(lbmgpu *h, int face, int what, double *buf, bool pack);
int mc_download_planes(lbmgpu *h, int i0, int i1, void *mix, void *const *species);
int mc_init(lbmgpu *h);
int mc_launch_collide(lbmgpu *h);
int mc_launch_stream(lbmgpu *h);
void mc_release(lbmgpu *h);

}  // namespace lbmh
