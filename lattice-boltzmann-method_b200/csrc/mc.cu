// lbmgpu, multicomponent path: device kernels around the per-cell functions of
// mc_cell.cuh and the handle operations for n_species > 0.
//
// Reference path replaced (farrasarira/Lattice-Boltzmann-Method, MULTICOMP on):
//   LBM::Collide_Species + LBM::Collide   src/lbm-collision.cpp:191-526 -> k_mc_collide
//   LBM::Streaming + LBM::calculate_moment src/lbm-streaming.cpp, src/lbm-moment.cpp:193-377
//                                          -> k_mc_stream
//   LBM::Init                              src/lbm-init.cpp:85-146 -> k_mc_init
// This path covers periodic lattices (fluid cells and periodic ghosts); the other cell
// types are rejected at upload with LBMGPU_E_UNSUPPORTED.
#include <algorithm>
#include <cstring>
#include <vector>

#include "handle.cuh"
#include "mc_cell.cuh"

namespace {

using namespace lbm;
using lbmh::kBlock;
using lbmh::MixOff;
using lbmh::SpOff;

constexpr int NS9 = 9;

template <int NS>
__global__ void __launch_bounds__(kBlock) k_mc_collide(McArgs A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || A.cflag[n] != CF_FLUID) return;
    mc_collide_cell<NS>(A, n);
}

template <int NS>
__global__ void __launch_bounds__(kBlock) k_mc_stream(McArgs A) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell || A.cflag[n] != CF_FLUID) return;
    mc_stream_moment_cell<NS>(A, n);
}

template <int NS>
__global__ void __launch_bounds__(kBlock) k_mc_init(McArgs A, double *rec0, double *rec1, double *pop0) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= A.ncell) return;
    mc_init_cell<NS>(A, n, rec0, rec1, pop0);
}

__device__ __forceinline__ double ldd(const char *rec, long off) { return *reinterpret_cast<const double *>(rec + off); }
__device__ __forceinline__ void std_(char *rec, long off, double v) { *reinterpret_cast<double *>(rec + off) = v; }

// Staging layout of a chunk of cnt cells: cnt mixture records, then cnt records of each
// species in turn.
template <int NS>
__global__ void k_mc_unpack(McArgs A, MixOff mo, SpOff so, const char *__restrict__ stage, long n0, long n1,
                            double *rec0, double *rec1, double *pop0, double *pop1) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    const long cnt = n1 - n0, nc = A.ncell;
    const char *mr = stage + (n - n0) * mo.size;
    auto put = [&](int plane, double v) {
        rec0[(long)plane * nc + n] = v;
        rec1[(long)plane * nc + n] = v;
    };
    put(RM_RHO, ldd(mr, mo.rho));
    put(RM_U, ldd(mr, mo.u));
    put(RM_V, ldd(mr, mo.v));
    put(RM_W, ldd(mr, mo.w));
    put(RM_T, ldd(mr, mo.temp));
    put(RM_P, ldd(mr, mo.p));
    put(RM_RHOE, ldd(mr, mo.rhoe));
    const int pi[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int q = 0; q < 6; ++q) put(RM_P00 + q, ldd(mr, mo.p_tensor + 8 * (3 * pi[q][0] + pi[q][1])));
    put(RM_HRR, ldd(mr, mo.HRR));
    const bool fluid = A.cflag[n] == CF_FLUID;
    for (int a = 0; a < NS; ++a) {
        const char *sr = stage + cnt * mo.size + ((long)a * cnt + (n - n0)) * so.size;
        put(rs(a, RS_RHO), ldd(sr, so.rho));
        put(rs(a, RS_UX), ldd(sr, so.u));
        put(rs(a, RS_UX + 1), ldd(sr, so.v));
        put(rs(a, RS_UX + 2), ldd(sr, so.w));
        put(rs(a, RS_X), ldd(sr, so.X));
        double jx = 0, jy = 0, jz = 0;
        for (int l = 0; l < 27; ++l) {
            const double fv = ldd(sr, so.f + 8 * l);
            if (fluid) {
                pop0[(long)(27 * a + l) * nc + n] = fv;
                pop1[(long)(27 * a + l) * nc + n] = ldd(sr, so.fpc + 8 * l);
            }
            jx += fv * cx(l);
            jy += fv * cy(l);
            jz += fv * cz(l);
        }
        put(rs(a, RS_JX), jx);
        put(rs(a, RS_JX + 1), jy);
        put(rs(a, RS_JX + 2), jz);
    }
    if (fluid)
        for (int l = 0; l < 27; ++l) {
            pop0[(long)(27 * NS + l) * nc + n] = ldd(mr, mo.g + 8 * l);
            pop1[(long)(27 * NS + l) * nc + n] = ldd(mr, mo.gpc + 8 * l);
        }
}

// pop_now: what the cell's populations are taken from (pulled when `stepped`, in place
// otherwise); pop_pc: the post-collision populations (fpc, gpc).
template <int NS>
__global__ void k_mc_pack(McArgs A, MixOff mo, SpOff so, char *__restrict__ stage, long n0, long n1,
                          const double *rec, const double *pop_now, const double *pop_pc, int stepped) {
    const long n = n0 + (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n1) return;
    const long cnt = n1 - n0, nc = A.ncell;
    char *mr = stage + (n - n0) * mo.size;
    auto get = [&](int plane) { return rec[(long)plane * nc + n]; };
    std_(mr, mo.rho, get(RM_RHO));
    std_(mr, mo.u, get(RM_U));
    std_(mr, mo.v, get(RM_V));
    std_(mr, mo.w, get(RM_W));
    std_(mr, mo.temp, get(RM_T));
    std_(mr, mo.p, get(RM_P));
    std_(mr, mo.rhoe, get(RM_RHOE));
    std_(mr, mo.HRR, get(RM_HRR));
    const int full[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    for (int q = 0; q < 9; ++q) std_(mr, mo.p_tensor + 8 * q, get(RM_P00 + full[q]));
    const bool fluid = A.cflag[n] == CF_FLUID;
    int i, j, k;
    decode(A, n, i, j, k);
    for (int a = 0; a < NS; ++a) {
        char *sr = stage + cnt * mo.size + ((long)a * cnt + (n - n0)) * so.size;
        std_(sr, so.rho, get(rs(a, RS_RHO)));
        std_(sr, so.u, get(rs(a, RS_UX)));
        std_(sr, so.v, get(rs(a, RS_UX + 1)));
        std_(sr, so.w, get(rs(a, RS_UX + 2)));
        std_(sr, so.X, get(rs(a, RS_X)));
        if (!fluid) continue;
        for (int l = 0; l < 27; ++l) {
            const long plane = (long)(27 * a + l) * nc;
            std_(sr, so.f + 8 * l, stepped ? pop_now[plane + mc_pull_src(A, i, j, k, l)] : pop_now[plane + n]);
            std_(sr, so.fpc + 8 * l, pop_pc[plane + n]);
        }
    }
    if (!fluid) return;
    double q3[3] = {0, 0, 0};
    for (int l = 0; l < 27; ++l) {
        const long plane = (long)(27 * NS + l) * nc;
        const double gv = stepped ? pop_now[plane + mc_pull_src(A, i, j, k, l)] : pop_now[plane + n];
        std_(mr, mo.g + 8 * l, gv);
        std_(mr, mo.gpc + 8 * l, pop_pc[plane + n]);
        q3[0] += gv * cx(l);
        q3[1] += gv * cy(l);
        q3[2] += gv * cz(l);
    }
    for (int q = 0; q < 3; ++q) std_(mr, mo.energy_flux + 8 * q, q3[q]);
}

McArgs base_args(lbmgpu *h) {
    McArgs A{};
    A.Nx = h->g.Nx;
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
    return A;
}

bool valid_mc_layout(const lbmgpu_mixture_layout &m, const lbmgpu_species_layout &s) {
    if (m.size == 0 || m.size % 8 || s.size == 0 || s.size % 8) return false;
    const long mext[][2] = {{m.p_tensor, 72}, {m.rho, 8}, {m.u, 8},  {m.v, 8},    {m.w, 8},
                            {m.p, 8},         {m.g, 216}, {m.gpc, 216}, {m.rhoe, 8}, {m.energy_flux, 24},
                            {m.temp, 8},      {m.HRR, 8}};
    for (const auto &e : mext)
        if (e[0] < 0 || e[0] % 8 || (size_t)(e[0] + e[1]) > m.size) return false;
    if (m.type < 0 || (size_t)(m.type + 2) > m.size) return false;
    const long sext[][2] = {{s.X, 8}, {s.rho, 8}, {s.f, 216}, {s.fpc, 216}, {s.u, 8}, {s.v, 8}, {s.w, 8}};
    for (const auto &e : sext)
        if (e[0] < 0 || e[0] % 8 || (size_t)(e[0] + e[1]) > s.size) return false;
    return true;
}

}  // namespace

namespace lbmh {

int mc_setup(lbmgpu *h) {
    const lbmgpu_desc &d = h->d;
    if (!valid_mc_layout(d.mix, d.spc)) return LBMGPU_E_ARG;
    h->ns = d.n_species;
    h->nrec = mc_nrec(h->ns);
    h->chem = d.chem_mode;
    h->U = UnitsF{d.units_m, d.units_kg, d.units_s, d.units_K};
    const lbmgpu_species_layout &s = d.spc;
    h->so = SpOff{(long)s.size, s.X, s.rho, s.f, s.fpc, s.u, s.v, s.w};
    const long nc = h->g.ncell;
    const size_t np = 27 * (size_t)(h->ns + 1);
    for (int b = 0; b < 2; ++b) {
        int rc = dalloc(h, &h->pop[b], np * nc);
        if (rc) return rc;
        rc = dalloc(h, &h->mom[b], (size_t)h->nrec * nc);
        if (rc) return rc;
    }
    gas::Tables *ht = new gas::Tables();
    gas::make_tables(*d.mech, *ht);
    set_lattice_constants(*ht, h->U);
    int rc = dalloc(h, &h->tab, 1);
    if (!rc) {
        cudaError_t e = cudaMemcpy(h->tab, ht, sizeof(gas::Tables), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = cuda_fail(e);
    }
    delete ht;
    return rc;
}

void mc_release(lbmgpu *h) {
    if (h->tab) cudaFree(h->tab);
    h->tab = nullptr;
}

int mc_upload(lbmgpu *h, const void *mix, const void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const lbm::ScGeom &g = h->g;
    const long nc = g.ncell;
    const size_t ms = h->mo.size, ss = h->so.size;
    const char *hm = static_cast<const char *>(mix);
    std::vector<int8_t> ty(nc);
    std::vector<uint8_t> cf(nc, 0);
    for (long n = 0; n < nc; ++n) {
        short t;
        std::memcpy(&t, hm + n * ms + h->mo.type, sizeof(short));
        if (t < 0 || t > 9) return LBMGPU_E_ARG;
        if (t != T_F && t != T_P) return LBMGPU_E_UNSUPPORTED;  // periodic lattices only
        ty[n] = (int8_t)t;
    }
    for (int i = 0; i < g.Nx; ++i)
        for (int j = 0; j < g.Ny; ++j)
            for (int k = 0; k < g.Nz; ++k) {
                const long n = (long)i * g.si + (long)j * g.sj + k;
                if (ty[n] != T_F) continue;
                if (i == 0 || j == 0 || k == 0 || i == g.Nx - 1 || j == g.Ny - 1 || k == g.Nz - 1)
                    return LBMGPU_E_ARG;
                cf[n] = CF_FLUID;
            }
    CK(cudaMemcpyAsync(h->type, ty.data(), nc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->cflag, cf.data(), nc, cudaMemcpyHostToDevice, h->stream));
    McArgs A = base_args(h);
    for (long n0 = 0; n0 < nc; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(nc, n0 + (long)h->stage_cells), cnt = n1 - n0;
        CK(cudaMemcpyAsync(h->stage, hm + n0 * ms, cnt * ms, cudaMemcpyHostToDevice, h->stream));
        for (int a = 0; a < h->ns; ++a)
            CK(cudaMemcpyAsync(h->stage + cnt * ms + (size_t)a * cnt * ss,
                               static_cast<const char *>(species[a]) + n0 * ss, cnt * ss, cudaMemcpyHostToDevice,
                               h->stream));
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        k_mc_unpack<NS9><<<grid_for(cnt), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[0],
                                                                  h->mom[1], h->pop[0], h->pop[1]);
        ev_end(h, ep);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->stream));
    h->cur = 0;
    h->pack_mode = PK_UPLOADED;
    h->have_state = true;
    h->phase = PH_BOUNDARY;
    return LBMGPU_OK;
}

int mc_download(lbmgpu *h, void *mix, void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const long nc = h->g.ncell;
    const size_t ms = h->mo.size, ss = h->so.size;
    std::vector<uint8_t> cf(nc);
    CK(cudaMemcpyAsync(cf.data(), h->cflag, nc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    McArgs A = base_args(h);
    const int c = h->cur;
    const bool stepped = h->pack_mode == PK_STEPPED;
    const double *pc = stepped ? h->pop[c] : h->pop[1 - c];
    const long mfld[] = {h->mo.rho, h->mo.u, h->mo.v, h->mo.w, h->mo.p, h->mo.temp, h->mo.rhoe, h->mo.HRR};
    const long sfld[] = {h->so.X, h->so.rho, h->so.u, h->so.v, h->so.w};
    char *hm = static_cast<char *>(mix);
    for (long n0 = 0; n0 < nc; n0 += (long)h->stage_cells) {
        const long n1 = std::min<long>(nc, n0 + (long)h->stage_cells), cnt = n1 - n0;
        EvPair ep{};
        ev_begin(h, K_OTHER, ep);
        k_mc_pack<NS9><<<grid_for(cnt), kBlock, 0, h->stream>>>(A, h->mo, h->so, h->stage, n0, n1, h->mom[c],
                                                                h->pop[c], pc, stepped ? 1 : 0);
        ev_end(h, ep);
        CK(cudaGetLastError());
        const size_t bytes = cnt * (ms + (size_t)h->ns * ss);
        CK(cudaMemcpyAsync(h->bounce, h->stage, bytes, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (long n = n0; n < n1; ++n) {
            const char *srec = h->bounce + (n - n0) * ms;
            char *drec = hm + n * ms;
            if (cf[n] == CF_FLUID) {
                short t;
                std::memcpy(&t, drec + h->mo.type, sizeof(short));
                std::memcpy(drec, srec, ms);
                std::memcpy(drec + h->mo.type, &t, sizeof(short));
                for (int q = 0; q < 9; ++q) (void)q;
            } else {
                for (long o : mfld) std::memcpy(drec + o, srec + o, sizeof(double));
                std::memcpy(drec + h->mo.p_tensor, srec + h->mo.p_tensor, 9 * sizeof(double));
            }
            for (int a = 0; a < h->ns; ++a) {
                const char *ssrc = h->bounce + cnt * ms + ((size_t)a * cnt + (n - n0)) * ss;
                char *sdst = static_cast<char *>(species[a]) + n * ss;
                if (cf[n] == CF_FLUID)
                    std::memcpy(sdst, ssrc, ss);
                else
                    for (long o : sfld) std::memcpy(sdst + o, ssrc + o, sizeof(double));
            }
        }
    }
    return LBMGPU_OK;
}

int mc_init(lbmgpu *h) {
    McArgs A = base_args(h);
    const int c = h->cur;
    EvPair ep{};
    ev_begin(h, K_OTHER, ep);
    k_mc_init<NS9><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A, h->mom[c], h->mom[1 - c], h->pop[c]);
    ev_end(h, ep);
    CK(cudaGetLastError());
    h->pack_mode = PK_INIT;
    return LBMGPU_OK;
}

int mc_launch_collide(lbmgpu *h) {
    const int c = h->cur, x = 1 - c;
    McArgs A = base_args(h);
    const bool local = h->pack_mode != PK_STEPPED;
    A.pop_src = h->pop[c];
    A.pop_dst = h->pop[x];
    A.pop_prev = local ? nullptr : h->pop[c];
    A.rec_cur = h->mom[c];
    A.rec_nxt = h->mom[x];
    A.local = local ? 1 : 0;
    EvPair ep{};
    ev_begin(h, K_COLLIDE, ep);
    k_mc_collide<NS9><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A);
    ev_end(h, ep);
    CK(cudaGetLastError());
    return 0;
}

int mc_launch_stream(lbmgpu *h) {
    const int c = h->cur, x = 1 - c;
    McArgs A = base_args(h);
    A.pop_src = h->pop[x];
    A.rec_cur = h->mom[c];
    A.rec_nxt = h->mom[x];
    EvPair ep{};
    ev_begin(h, K_STREAM_MOMENT, ep);
    k_mc_stream<NS9><<<grid_for(h->g.ncell), kBlock, 0, h->stream>>>(A);
    ev_end(h, ep);
    CK(cudaGetLastError());
    h->cur = x;
    h->pack_mode = PK_STEPPED;
    return 0;
}

}  // namespace lbmh
