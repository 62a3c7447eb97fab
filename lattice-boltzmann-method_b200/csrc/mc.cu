// lbmgpu, multicomponent path: the handle operations for n_species > 0 -- set-up, the
// record uploads and downloads, Init and the phase launches, each dispatched by the
// handle's species count to the kernels built for it (McOps<NS>: mc_kernels.cuh,
// instantiated in mc_ns9.cu and mc_ns6.cu) -- and the kernels that do not depend on the
// species count (the boundary store, the FP32 shift).
//
// Cell types: fluid, periodic ghosts, solid (TMS wall), adiabatic, free-slip, and the
// characteristic inflow/outflow ghosts TYPE_I_C / TYPE_O_C.  The reference's
// non-characteristic TYPE_I / TYPE_O rewrite a neighbour's moments from inside the
// boundary sweep (order dependent) and are rejected at upload with LBMGPU_E_UNSUPPORTED.
//
// Storage: FP64 (bit-faithful to the reference) or FP32 (LBMGPU_FP32: populations in
// float as deviations from a per-plane shift; the per-cell record stays FP64, the
// transport properties are evaluated in FP32, everything else in FP64).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "handle.cuh"
#include "mc_bc.cuh"
#include "mc_cell.cuh"
#include "mc_ops.cuh"
#include "surrogate_host.cuh"

namespace {

using namespace lbm;
using namespace lbmh;

// the special cells' current populations into the compact store (after upload and Init)
template <typename S>
__global__ void k_mc_fill_bst(long ncell, long nb, int np, const long *__restrict__ blist, const S *__restrict__ pop,
                              S *__restrict__ bst) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)np * nb) return;
    const int q = (int)(i / nb);
    const long b = i - (long)q * nb;
    bst[i] = pop[(long)q * ncell + blist[b]];
}

// FP32 storage: new per-plane shift = mean over the fluid cells of the decoded population
// (one block per plane, fixed reduction order, so the result is deterministic) ...
constexpr int kMeanBlock = 256;
template <typename S>
__global__ void __launch_bounds__(kMeanBlock) k_plane_mean(McArgsT<S, double> A, const S *pop, double *shift_new,
                                                           long nfluid) {
    __shared__ double red[kMeanBlock];
    const int q = blockIdx.x;
    double s = 0.0;
    for (long n = threadIdx.x; n < A.ncell; n += kMeanBlock)
        if (A.cflag[n] & CF_FLUID) s += ldpop(A, pop, q, n);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kMeanBlock / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) shift_new[q] = nfluid > 0 ? red[0] / (double)nfluid : 0.0;
}

// ... and both population buffers re-encoded from the old shift to the new one.
template <typename S>
__global__ void k_reshift(long total, long ncell, S *p0, S *p1, const double *old_s, const double *new_s) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int q = (int)(i / ncell);
    const double d = old_s[q] - new_s[q];
    p0[i] = (S)((double)p0[i] + d);
    p1[i] = (S)((double)p1[i] + d);
}

// the special cells' populations of pop[cur] into bst[cur]
template <typename S>
int fill_bst(lbmgpu *h) {
    if (h->nb == 0) return 0;
    const int np = 27 * (h->ns + 1);
    const long total = (long)np * h->nb;
    k_mc_fill_bst<S><<<grid_for(total), kBlock, 0, h->stream>>>(h->g.ncell, h->nb, np, h->blist, popb<S>(h, h->cur),
                                                                bstb<S>(h, h->cur));
    CK(cudaGetLastError());
    return 0;
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

// FP32 storage: move both population buffers onto the mean of the current state.
int rebase_shift(lbmgpu *h) {
    if (!h->fp32) return 0;
    McArgsT<float, double> A = base_args<float>(h);
    const int np = 27 * (h->ns + 1);
    k_plane_mean<float><<<np, kMeanBlock, 0, h->stream>>>(A, h->pop32[h->cur], h->shift[1], h->nfluid);
    CK(cudaGetLastError());
    const long total = (long)np * h->g.ncell;
    k_reshift<float><<<grid_for(total), kBlock, 0, h->stream>>>(total, h->g.ncell, h->pop32[0], h->pop32[1],
                                                                h->shift[0], h->shift[1]);
    CK(cudaGetLastError());
    std::swap(h->shift[0], h->shift[1]);
    return 0;
}

}  // namespace

namespace lbmh {

int mc_halo(lbmgpu *h, int face, int what, double *buf, bool pack) {
    return mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::halo(h, face, what, buf, pack); });
}

int mc_setup(lbmgpu *h) {
    const lbmgpu_desc &d = h->d;
    if (!valid_mc_layout(d.mix, d.spc)) return LBMGPU_E_ARG;
    h->ns = d.n_species;
    h->mech = *d.mech;
    h->nrec = mc_nrec(h->ns);
    h->chem = d.chem_mode;
    h->fp32 = d.precision == LBMGPU_FP32;
    h->U = UnitsF{d.units_m, d.units_kg, d.units_s, d.units_K};
    const lbmgpu_species_layout &s = d.spc;
    h->so = SpOff{(long)s.size, s.X, s.rho, s.f, s.fpc, s.u, s.v, s.w};
    const long nc = h->g.ncell;
    const size_t np = 27 * (size_t)(h->ns + 1);
    for (int b = 0; b < 2; ++b) {
        int rc = h->fp32 ? dalloc(h, &h->pop32[b], np * nc) : dalloc(h, &h->pop[b], np * nc);
        if (rc) return rc;
        rc = dalloc(h, &h->mom[b], (size_t)h->nrec * nc);
        if (rc) return rc;
        if (b == 0) {
            rc = dalloc(h, &h->props, (size_t)mc_by_ns(h->ns, [](auto ops) { return decltype(ops)::props_planes(); }) * nc);
            if (rc) return rc;
            rc = dalloc(h, &h->gsum, (size_t)mc_by_ns(h->ns, [](auto ops) { return decltype(ops)::gsum_planes(); }) * nc);
            if (rc) return rc;
        }
        // the face-difference planes of cells the kernels never write (ghosts) are read
        // but not used, and the ghosts' populations are never read; zero them all so they
        // hold no stale bits
        CK(cudaMemset(h->mom[b], 0, (size_t)h->nrec * nc * sizeof(double)));
        CK(cudaMemset(h->fp32 ? (void *)h->pop32[b] : (void *)h->pop[b], 0,
                      np * nc * (h->fp32 ? sizeof(float) : sizeof(double))));
        if (h->fp32) {
            rc = dalloc(h, &h->shift[b], np);
            if (rc) return rc;
            CK(cudaMemset(h->shift[b], 0, np * sizeof(double)));
        }
    }
    h->kin = kin_h2_air_9::matches(*d.mech) ? KIN_H2_AIR_9 : KIN_TABLES;
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
    sur_release(h);
    if (h->tab) cudaFree(h->tab);
    h->tab = nullptr;
    cudaFree(h->props);
    h->props = nullptr;
    cudaFree(h->gsum);
    h->gsum = nullptr;
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->pop32[b]);
        cudaFree(h->bst32[b]);
        cudaFree(h->shift[b]);
        h->pop32[b] = nullptr;
        h->bst32[b] = nullptr;
        h->shift[b] = nullptr;
    }
}

// Classification of the whole lattice once every plane is on the device: fluid cells,
// the cells with a boundary upstream (compact list), the boundary store, the FP32 shift.
static int mc_finish_upload(lbmgpu *h) {
    const lbm::ScGeom &g = h->g;
    const long nc = g.ncell;
    const std::vector<int8_t> &ty = h->htype;
    std::vector<uint8_t> cf(nc, 0);
    long nfluid = 0, nb = 0;
    std::vector<int> bidh(nc, -1);
    std::vector<long> blh;
    // classification by host threads, x-plane by x-plane: the flags and each plane's counts,
    // then the special cells' compact indices in cell order from the planes' offsets
    std::vector<long> pf(g.Nx, 0), ps(g.Nx, 0);
    std::vector<uint8_t> bad(g.Nx, 0);
    host_parallel_for(g.Nx, [&](long lo, long hi) {
        for (long i = lo; i < hi; ++i)
            for (int j = 0; j < g.Ny; ++j)
                for (int k = 0; k < g.Nz; ++k) {
                    const long n = i * g.si + (long)j * g.sj + k;
                    if (ty[n] != T_F) continue;
                    // a halo plane holds the neighbouring slab's cells: never updated here
                    if ((i == 0 && h->halo_lo) || (i == g.Nx - 1 && h->halo_hi)) continue;
                    if (i == 0 || j == 0 || k == 0 || i == g.Nx - 1 || j == g.Ny - 1 || k == g.Nz - 1) {
                        bad[i] = 1;
                        continue;
                    }
                    uint8_t c = CF_FLUID;
                    for (int l = 0; l < 27; ++l) {
                        const int t = ty[n - (long)cx(l) * g.si - (long)cy(l) * g.sj - cz(l)];
                        if (t != T_F && t != T_P) c |= CF_SPECIAL;
                    }
                    ps[i] += (c & CF_SPECIAL) ? 1 : 0;
                    cf[n] = c;
                    ++pf[i];
                }
    }, 1);
    for (int i = 0; i < g.Nx; ++i) {
        if (bad[i]) return LBMGPU_E_ARG;
        nfluid += pf[i];
        const long base = nb;
        nb += ps[i];
        ps[i] = base;  // the plane's first compact index
    }
    blh.resize(nb);
    host_parallel_for(g.Nx, [&](long lo, long hi) {
        for (long i = lo; i < hi; ++i) {
            long b = ps[i];
            for (long n = i * g.si; n < (i + 1) * g.si; ++n)
                if (cf[n] & CF_SPECIAL) {
                    bidh[n] = (int)b;
                    blh[b++] = n;
                }
        }
    }, 1);
    // the boundary formulas read up to two cells inward along an axis
    if (nb > 0 && (g.Nx < 5 || g.Ny < 5 || g.Nz < 5)) return LBMGPU_E_UNSUPPORTED;
    h->nfluid = nfluid;
    if (nb != h->nb || !h->blist) {
        const size_t np = 27 * (size_t)(h->ns + 1), es = h->fp32 ? sizeof(float) : sizeof(double);
        for (int b = 0; b < 2; ++b) {
            void *&p = h->fp32 ? reinterpret_cast<void *&>(h->bst32[b]) : reinterpret_cast<void *&>(h->bst[b]);
            if (p) {
                cudaFree(p);
                h->bytes -= np * (size_t)std::max<long>(h->nb, 1) * es;
                p = nullptr;
            }
        }
        if (h->blist) {
            cudaFree(h->blist);
            h->bytes -= (size_t)std::max<long>(h->nb, 1) * sizeof(long);
            h->blist = nullptr;
        }
        h->nb = nb;
        for (int b = 0; b < 2; ++b) {
            const int rc = h->fp32 ? dalloc(h, &h->bst32[b], np * (size_t)std::max<long>(nb, 1))
                                   : dalloc(h, &h->bst[b], np * (size_t)std::max<long>(nb, 1));
            if (rc) return rc;
        }
        const int rc = dalloc(h, &h->blist, (size_t)std::max<long>(nb, 1));
        if (rc) return rc;
    }
    if (nb > 0) CK(cudaMemcpyAsync(h->blist, blh.data(), nb * sizeof(long), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->bid, bidh.data(), nc * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->cflag, cf.data(), nc, cudaMemcpyHostToDevice, h->stream));
    h->cur = 0;
    int rc = rebase_shift(h);
    if (rc) return rc;
    rc = h->fp32 ? fill_bst<float>(h) : fill_bst<double>(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    h->pack_mode = PK_UPLOADED;
    h->have_state = true;
    h->phase = PH_BOUNDARY;
    return LBMGPU_OK;
}

int mc_upload_planes(lbmgpu *h, int i0, int i1, const void *mix, const void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    const lbm::ScGeom &g = h->g;
    if (i0 < 0 || i1 > g.Nx || i0 >= i1) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const long c0 = (long)i0 * g.si, c1 = (long)i1 * g.si;
    const size_t ms = h->mo.size;
    const char *hm = static_cast<const char *>(mix);
    if ((long)h->htype.size() != g.ncell) h->htype.assign(g.ncell, 0);
    if ((int)h->plane_have.size() != g.Nx) h->plane_have.assign(g.Nx, 0);
    // the cell types, read by host threads; the first refusal found (by cell) is returned
    std::vector<long> bad(2, c1);  // first cell with an invalid / unsupported type
    {
        std::mutex mx;
        host_parallel_for(c1 - c0, [&](long lo, long hi) {
            long b0 = c1, b1 = c1;
            for (long n = c0 + lo; n < c0 + hi; ++n) {
                short t;
                std::memcpy(&t, hm + (n - c0) * ms + h->mo.type, sizeof(short));
                if (t < 0 || t > 9) {
                    b0 = std::min(b0, n);
                    break;
                }
                if (t == T_I || t == T_O || t == T_Q) {
                    b1 = std::min(b1, n);
                    break;
                }
                h->htype[n] = (int8_t)t;
            }
            std::lock_guard<std::mutex> g(mx);
            bad[0] = std::min(bad[0], b0);
            bad[1] = std::min(bad[1], b1);
        });
    }
    if (bad[0] < c1 || bad[1] < c1) return bad[0] <= bad[1] ? LBMGPU_E_ARG : LBMGPU_E_UNSUPPORTED;
    // a new upload begins: the state is incomplete until every plane has arrived again
    if (h->planes_have == 0) h->have_state = false;
    CK(cudaMemcpyAsync(h->type + c0, h->htype.data() + c0, c1 - c0, cudaMemcpyHostToDevice, h->stream));
    int rc = mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::upload(h, hm, species, c0, c1); });
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    for (int i = i0; i < i1; ++i)
        if (!h->plane_have[i]) {
            h->plane_have[i] = 1;
            ++h->planes_have;
        }
    if (h->planes_have < g.Nx) return LBMGPU_OK;
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    return mc_finish_upload(h);
}

int mc_upload(lbmgpu *h, const void *mix, const void *const *species) {
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    return mc_upload_planes(h, 0, h->g.Nx, mix, species);
}

int mc_download_planes(lbmgpu *h, int i0, int i1, void *mix, void *const *species) {
    if (!species) return LBMGPU_E_ARG;
    for (int a = 0; a < h->ns; ++a)
        if (!species[a]) return LBMGPU_E_ARG;
    if (i0 < 0 || i1 > h->g.Nx || i0 >= i1) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    const long c0 = (long)i0 * h->g.si, c1 = (long)i1 * h->g.si;
    const size_t ms = h->mo.size, ss = h->so.size;
    std::vector<uint8_t> cf(c1 - c0);
    CK(cudaMemcpyAsync(cf.data(), h->cflag + c0, c1 - c0, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const bool stepped = h->pack_mode == PK_STEPPED;
    const long mfld[] = {h->mo.rho, h->mo.u, h->mo.v, h->mo.w, h->mo.p, h->mo.temp, h->mo.rhoe, h->mo.HRR};
    const long sfld[] = {h->so.X, h->so.rho, h->so.u, h->so.v, h->so.w};
    char *hm = static_cast<char *>(mix);
    // chunk k is packed on the device and copied into bounce buffer k % 2; while the host
    // merges chunk k, the device packs and copies chunk k + 1 into the other buffer
    const long step = (long)h->stage_cells;
    auto issue = [&](long n0, char *dst) -> int {
        const long n1 = std::min<long>(c1, n0 + step);
        const int rc = mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::pack(h, n0, n1, stepped); });
        if (rc) return rc;
        CK(cudaMemcpyAsync(dst, h->stage, (n1 - n0) * (ms + (size_t)h->ns * ss), cudaMemcpyDeviceToHost, h->stream));
        return 0;
    };
    int rc0 = issue(c0, h->bounce);
    if (rc0) return rc0;
    for (long n0 = c0, k = 0; n0 < c1; n0 += step, ++k) {
        const long n1 = std::min<long>(c1, n0 + step), cnt = n1 - n0;
        char *const buf = (k & 1) ? h->bounce2 : h->bounce;
        CK(cudaStreamSynchronize(h->stream));  // chunk k is in buf
        if (n1 < c1) {
            rc0 = issue(n1, (k & 1) ? h->bounce : h->bounce2);
            if (rc0) return rc0;
        }
        // the merge into the caller's records (each cell's own bytes: no two threads share one)
        host_parallel_for(cnt, [&](long lo, long hi) {
            for (long n = n0 + lo; n < n0 + hi; ++n) {
                const char *srec = buf + (n - n0) * ms;
                char *drec = hm + (n - c0) * ms;
                const bool fluid = cf[n - c0] & CF_FLUID;
                if (fluid) {
                    short t;
                    std::memcpy(&t, drec + h->mo.type, sizeof(short));
                    std::memcpy(drec, srec, ms);
                    std::memcpy(drec + h->mo.type, &t, sizeof(short));
                } else {
                    for (long o : mfld) std::memcpy(drec + o, srec + o, sizeof(double));
                    std::memcpy(drec + h->mo.p_tensor, srec + h->mo.p_tensor, 9 * sizeof(double));
                }
                for (int a = 0; a < h->ns; ++a) {
                    const char *ssrc = buf + cnt * ms + ((size_t)a * cnt + (n - n0)) * ss;
                    char *sdst = static_cast<char *>(species[a]) + (n - c0) * ss;
                    if (fluid)
                        std::memcpy(sdst, ssrc, ss);
                    else
                        for (long o : sfld) std::memcpy(sdst + o, ssrc + o, sizeof(double));
                }
            }
        });
    }
    CK(cudaStreamSynchronize(h->stream));
    return LBMGPU_OK;
}

int mc_download(lbmgpu *h, void *mix, void *const *species) { return mc_download_planes(h, 0, h->g.Nx, mix, species); }

int mc_init(lbmgpu *h) {
    int rc = mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::init(h); });
    if (rc) return rc;
    rc = rebase_shift(h);
    if (rc) return rc;
    rc = h->fp32 ? fill_bst<float>(h) : fill_bst<double>(h);
    if (rc) return rc;
    h->pack_mode = PK_INIT;
    return LBMGPU_OK;
}

int mc_launch_collide(lbmgpu *h) {
    return mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::collide(h); });
}

int mc_launch_stream(lbmgpu *h) {
    const int rc = mc_by_ns(h->ns, [&](auto ops) { return decltype(ops)::stream(h); });
    if (rc) return rc;
    h->cur = 1 - h->cur;
    h->pack_mode = PK_STEPPED;
    sur_after_step(h);
    return 0;
}

}  // namespace lbmh
