// lbmgpu I/O from the device state: the reference's restart file (write_restart /
// read_restart, src/restart_file.cpp:274-440) and its VTK output (OutputVTK,
// src/output.cpp:9-210).
//
// Restart: the reference's binary layout -- ints dx, dy, dz, Nx, Ny, Nz, dt_sim, step; single
// component the doubles nu, gas constant, gamma, Ra, Prandtl and then every cell's MIXTURE
// record; multicomponent the size_t species count, each species name (size_t length + the
// characters), the double permeability and then per cell the MIXTURE record followed by one
// SPECIES record per species -- cells in [i][j][k] order, records in the caller's layout
// (the sizeof of its MIXTURE / SPECIES classes).  Multicomponent files are written and read
// a few x-planes at a time through the plane-range download / upload, so a lattice whose
// AoS copy does not fit in host memory still round-trips.
//
// VTK: the RectilinearGrid file OutputVTK writes, byte for byte: the XML header with the
// same appended-data offsets, then Float32 arrays (cell data in x-fastest order) of density,
// velocity, cell type, temperature, pressure and, multicomponent, heat release, each
// species' mass or mole fraction and each species' x velocity relative to the mixture,
// then the vertex coordinates i * dx.  The cell arrays are packed on the device from the
// record planes in one kernel and copied to the host once.  SI units (OUTPUT_SI) and mass
// fractions (OUTPUT_MASSFRAC), the reference's compile-time switches, are flags here.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.cuh"
#include "mc_cell.cuh"
#include "sc_kernels.cuh"

using namespace lbm;
using namespace lbmh;

namespace {

constexpr int kIoPlanes = 8;  // x-planes per multicomponent restart chunk

struct VtkSrc {
    const double *rec;
    const int8_t *type;
    long ncell, si, sj;
    int Nx, Ny, Nz, ns, flags;
    UnitsF U;
};

// One cell's values into the arrays of the VTK file's appended data (cell data only),
// each array at its offset in `out`, cells in x-fastest order.
__global__ void k_vtk_pack(VtkSrc S, float *__restrict__ out) {
    const long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= S.ncell) return;
    int i, j, k;
    cell_ijk(n, S.si, S.sj, i, j, k);
    const long o = ((long)k * S.Ny + j) * S.Nx + i, N = S.ncell;
    const bool si = S.flags & LBMGPU_VTK_SI;
    const double *R = S.rec;
    const bool mc = S.ns > 0;
    const double rho = R[(mc ? RM_RHO : M_RHO) * N + n];
    const double u = R[(mc ? RM_U : M_U) * N + n], v = R[(mc ? RM_V : M_V) * N + n], w = R[(mc ? RM_W : M_W) * N + n];
    const double T = R[(mc ? RM_T : M_T) * N + n], p = R[(mc ? RM_P : M_P) * N + n];
    out[o] = si ? si_rho(S.U, (float)rho) : (float)rho;
    out[N + 3 * o] = si ? si_u(S.U, (float)u) : (float)u;
    out[N + 3 * o + 1] = si ? si_u(S.U, (float)v) : (float)v;
    out[N + 3 * o + 2] = si ? si_u(S.U, (float)w) : (float)w;
    out[4 * N + o] = (float)(int)S.type[n];
    out[5 * N + o] = si ? si_temp(S.U, (float)T) : (float)T;
    out[6 * N + o] = si ? si_p(S.U, (float)p) : (float)p;
    if (!mc) return;
    const double hrr = R[RM_HRR * N + n];
    out[7 * N + o] = si ? si_hrr(S.U, (float)hrr) : (float)hrr;
    for (int a = 0; a < S.ns; ++a) {
        const double ra = R[(long)rs(a, RS_RHO) * N + n];
        out[(8 + a) * N + o] = (S.flags & LBMGPU_VTK_MASSFRAC) ? (float)(ra / rho) : (float)R[(long)rs(a, RS_X) * N + n];
        const double du = R[(long)rs(a, RS_UX) * N + n] - u;
        out[(8 + S.ns + a) * N + o] = si ? si_u(S.U, (float)du) : (float)du;
    }
}

int vtk_arrays(const lbmgpu *h) { return h->ns > 0 ? 8 + 2 * h->ns : 7; }

struct File {
    FILE *f = nullptr;
    explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

bool wr(FILE *f, const void *p, size_t n) { return std::fwrite(p, 1, n, f) == n; }
bool rd(FILE *f, void *p, size_t n) { return std::fread(p, 1, n, f) == n; }

// the restart header's species names: the handle's mechanism names, in its order
std::vector<std::string> species_names(const lbmgpu *h) {
    std::vector<std::string> out;
    for (int a = 0; a < h->ns; ++a) out.emplace_back(h->mech.name[a]);
    return out;
}

}  // namespace

extern "C" {

int lbmgpu_vtk_fields(lbmgpu_t *h, float *out, size_t n_out, int flags) {
    if (!h || !out) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if ((flags & LBMGPU_VTK_SI) && h->ns == 0) return LBMGPU_E_UNSUPPORTED;  // single component: no units
    const long nc = h->g.ncell;
    const size_t need = (size_t)(vtk_arrays(h) + 2) * nc;  // velocity is three arrays wide
    if (n_out < need) return LBMGPU_E_ARG;
    CK(cudaSetDevice(h->d.device));
    float *dbuf = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&dbuf), need * sizeof(float), h->stream));
    VtkSrc S{h->mom[h->cur], h->type, nc, h->g.si, h->g.sj, h->g.Nx, h->g.Ny, h->g.Nz, h->ns, flags, h->U};
    k_vtk_pack<<<grid_for(nc), kBlock, 0, h->stream>>>(S, dbuf);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dbuf, need * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
    cudaFreeAsync(dbuf, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? LBMGPU_OK : cuda_fail(e);
}

int lbmgpu_write_vtk(lbmgpu_t *h, const char *path, int dx, int flags) {
    if (!h || !path) return LBMGPU_E_ARG;
    const int Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz, ns = h->ns;
    const long nc = h->g.ncell;
    std::vector<float> a((size_t)(vtk_arrays(h) + 2) * nc);
    int rc = lbmgpu_vtk_fields(h, a.data(), a.size(), flags);
    if (rc) return rc;
    File F(path, "wb");
    if (!F.f) return LBMGPU_E_IO;
    FILE *fp = F.f;
    unsigned long offset = 0;
    const unsigned long cell = 4 + 1 * 4 * (unsigned long)nc, vec = 4 + 3 * 4 * (unsigned long)nc;
    std::fprintf(fp, "<?xml version=\"1.0\"?>\n");
    std::fprintf(fp, "<VTKFile type=\"RectilinearGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
                     "header_type=\"UInt32\">\n");
    std::fprintf(fp, "  <RectilinearGrid WholeExtent=\"0 %d 0 %d 0 %d\">\n", Nx, Ny, Nz);
    std::fprintf(fp, "  <Piece Extent=\"0 %d 0 %d 0 %d\">\n", Nx, Ny, Nz);
    std::fprintf(fp, "    <PointData>\n");
    std::fprintf(fp, "    </PointData>\n");
    std::fprintf(fp, "    <CellData>\n");
    auto arr = [&](const char *name, int comps, unsigned long size) {
        if (comps == 1)
            std::fprintf(fp, "      <DataArray type=\"Float32\" Name=\"%s\" format=\"appended\" offset=\"%ld\" />\n",
                         name, (long)offset);
        else
            std::fprintf(fp,
                         "      <DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"appended\" "
                         "offset=\"%ld\" />\n",
                         name, comps, (long)offset);
        offset += size;
    };
    arr("Density", 1, cell);
    arr("Velocity", 3, vec);
    arr("CellType", 1, cell);
    arr("Temperature", 1, cell);
    arr("Pressure", 1, cell);
    if (ns > 0) {
        arr("HRR", 1, cell);
        for (int s = 0; s < ns; ++s) arr((std::string("Mole Fraction ") + h->mech.name[s]).c_str(), 1, cell);
        for (int s = 0; s < ns; ++s) arr((std::string("Species Velocity ") + h->mech.name[s]).c_str(), 1, cell);
    }
    std::fprintf(fp, "    </CellData>\n");
    std::fprintf(fp, "    <Coordinates>\n");
    const int ext[3] = {Nx, Ny, Nz};
    const char *cname[3] = {"CoordinateX", "CoordinateY", "CoordinateZ"};
    for (int d = 0; d < 3; ++d) {
        std::fprintf(fp, "      <DataArray type=\"Float32\" Name=\"%s\" format=\"appended\" offset=\"%ld\" />\n",
                     cname[d], (long)offset);
        offset += 4 + 1 * 4 * (unsigned long)(ext[d] + 1);
    }
    std::fprintf(fp, "    </Coordinates>\n");
    std::fprintf(fp, "  </Piece>\n");
    std::fprintf(fp, "  </RectilinearGrid>\n");
    std::fprintf(fp, "  <AppendedData encoding=\"raw\">");
    std::fprintf(fp, "_");
    // cell arrays in the file's order: density, velocity, type, temperature, pressure, then
    // HRR and the species arrays (the packed buffer holds them in this order)
    const long sizes[5] = {nc, 3 * nc, nc, nc, nc};
    long at = 0;
    bool ok = true;
    for (int q = 0; q < 5 && ok; ++q) {
        const unsigned int bytes = (unsigned int)(4 * sizes[q]);
        ok = wr(fp, &bytes, sizeof(int)) && wr(fp, a.data() + at, 4 * sizes[q]);
        at += sizes[q];
    }
    for (int q = 0; ns > 0 && q < 1 + 2 * ns && ok; ++q) {
        const unsigned int bytes = (unsigned int)(4 * nc);
        ok = wr(fp, &bytes, sizeof(int)) && wr(fp, a.data() + at, 4 * nc);
        at += nc;
    }
    for (int d = 0; d < 3 && ok; ++d) {
        const unsigned int bytes = (unsigned int)(4 * (ext[d] + 1));
        ok = wr(fp, &bytes, sizeof(int));
        for (int q = 0; q < ext[d] + 1 && ok; ++q) {
            const float c = (float)(q * dx);
            ok = wr(fp, &c, sizeof(float));
        }
    }
    std::fprintf(fp, "  </AppendedData>\n");
    std::fprintf(fp, "</VTKFile>\n");
    return ok && !std::ferror(fp) ? LBMGPU_OK : LBMGPU_E_IO;
}

int lbmgpu_write_restart(lbmgpu_t *h, const char *path, const lbmgpu_restart_info *info) {
    if (!h || !path || !info) return LBMGPU_E_ARG;
    if (!h->have_state) return LBMGPU_E_STATE;
    if (h->phase != PH_BOUNDARY) return LBMGPU_E_PHASE;
    const int Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz, ns = h->ns;
    const long plane = (long)Ny * Nz;
    const size_t ms = h->mo.size, ss = h->so.size;
    File F(path, "wb");
    if (!F.f) return LBMGPU_E_IO;
    FILE *f = F.f;
    int head[8] = {info->dx, info->dy, info->dz, Nx, Ny, Nz, h->d.dt_sim, info->step};
    bool ok = wr(f, head, sizeof(head));
    // the cell types the records carry (the device keeps them; the download preserves the
    // type field of its destination)
    std::vector<int8_t> ty(h->g.ncell);
    CK(cudaMemcpy(ty.data(), h->type, h->g.ncell, cudaMemcpyDeviceToHost));
    if (ns == 0) {
        const double sc[5] = {h->d.nu, h->d.gas_const, h->d.gamma, info->Ra, h->d.prtl};
        ok = ok && wr(f, sc, sizeof(sc));
        std::vector<char> mix((size_t)h->g.ncell * ms, 0);
        for (long n = 0; n < h->g.ncell; ++n) {
            const short t = ty[n];
            std::memcpy(mix.data() + n * ms + h->mo.type, &t, sizeof(short));
        }
        const int rc = lbmgpu_download(h, mix.data(), nullptr);
        if (rc) return rc;
        ok = ok && wr(f, mix.data(), mix.size());
        return ok ? LBMGPU_OK : LBMGPU_E_IO;
    }
    const size_t nsp = (size_t)ns;
    ok = ok && wr(f, &nsp, sizeof(nsp));
    for (const std::string &s : species_names(h)) {
        const size_t len = s.size();
        ok = ok && wr(f, &len, sizeof(len)) && wr(f, s.data(), len);
    }
    ok = ok && wr(f, &info->permeability, sizeof(double));
    const size_t per_cell = ms + nsp * ss;
    std::vector<char> mix((size_t)kIoPlanes * plane * ms), out((size_t)kIoPlanes * plane * per_cell);
    std::vector<std::vector<char>> sp(ns, std::vector<char>((size_t)kIoPlanes * plane * ss));
    std::vector<void *> spp(ns);
    for (int a = 0; a < ns; ++a) spp[a] = sp[a].data();
    for (int i0 = 0; i0 < Nx && ok; i0 += kIoPlanes) {
        const int i1 = std::min(Nx, i0 + kIoPlanes);
        const long cnt = (long)(i1 - i0) * plane, c0 = (long)i0 * plane;
        std::fill(mix.begin(), mix.end(), 0);
        for (auto &v : sp) std::fill(v.begin(), v.end(), 0);
        for (long c = 0; c < cnt; ++c) {
            const short t = ty[c0 + c];
            std::memcpy(mix.data() + c * ms + h->mo.type, &t, sizeof(short));
        }
        const int rc = mc_download_planes(h, i0, i1, mix.data(), spp.data());
        if (rc) return rc;
        for (long c = 0; c < cnt; ++c) {
            char *o = out.data() + c * per_cell;
            std::memcpy(o, mix.data() + c * ms, ms);
            for (int a = 0; a < ns; ++a) std::memcpy(o + ms + a * ss, sp[a].data() + c * ss, ss);
        }
        ok = wr(f, out.data(), (size_t)cnt * per_cell);
    }
    return ok ? LBMGPU_OK : LBMGPU_E_IO;
}

int lbmgpu_read_restart(lbmgpu_t *h, const char *path, lbmgpu_restart_info *info) {
    if (!h || !path || !info) return LBMGPU_E_ARG;
    File F(path, "rb");
    if (!F.f) return LBMGPU_E_IO;
    FILE *f = F.f;
    const int Nx = h->g.Nx, Ny = h->g.Ny, Nz = h->g.Nz, ns = h->ns;
    const long plane = (long)Ny * Nz;
    const size_t ms = h->mo.size, ss = h->so.size;
    int head[8];
    if (!rd(f, head, sizeof(head))) return LBMGPU_E_IO;
    if (head[3] != Nx || head[4] != Ny || head[5] != Nz || head[6] != h->d.dt_sim) return LBMGPU_E_ARG;
    info->dx = head[0];
    info->dy = head[1];
    info->dz = head[2];
    info->step = head[7];
    info->Ra = 0.0;
    info->permeability = 0.0;
    if (ns == 0) {
        double sc[5];
        if (!rd(f, sc, sizeof(sc))) return LBMGPU_E_IO;
        info->Ra = sc[3];
        std::vector<char> mix((size_t)h->g.ncell * ms);
        if (!rd(f, mix.data(), mix.size())) return LBMGPU_E_IO;
        return lbmgpu_upload(h, mix.data(), nullptr);
    }
    size_t nsp = 0;
    if (!rd(f, &nsp, sizeof(nsp)) || nsp != (size_t)ns) return LBMGPU_E_ARG;
    const std::vector<std::string> names = species_names(h);
    for (size_t a = 0; a < nsp; ++a) {
        size_t len = 0;
        if (!rd(f, &len, sizeof(len)) || len > 256) return LBMGPU_E_ARG;
        std::string s(len, '\0');
        if (!rd(f, &s[0], len)) return LBMGPU_E_IO;
        if (s != names[a]) return LBMGPU_E_ARG;  // species in the handle's order
    }
    if (!rd(f, &info->permeability, sizeof(double))) return LBMGPU_E_IO;
    const size_t per_cell = ms + nsp * ss;
    std::vector<char> mix((size_t)kIoPlanes * plane * ms), in((size_t)kIoPlanes * plane * per_cell);
    std::vector<std::vector<char>> sp(ns, std::vector<char>((size_t)kIoPlanes * plane * ss));
    std::vector<const void *> spp(ns);
    for (int a = 0; a < ns; ++a) spp[a] = sp[a].data();
    h->planes_have = 0;
    std::fill(h->plane_have.begin(), h->plane_have.end(), 0);
    for (int i0 = 0; i0 < Nx; i0 += kIoPlanes) {
        const int i1 = std::min(Nx, i0 + kIoPlanes);
        const long cnt = (long)(i1 - i0) * plane;
        if (!rd(f, in.data(), (size_t)cnt * per_cell)) return LBMGPU_E_IO;
        for (long c = 0; c < cnt; ++c) {
            const char *r = in.data() + c * per_cell;
            std::memcpy(mix.data() + c * ms, r, ms);
            for (int a = 0; a < ns; ++a) std::memcpy(sp[a].data() + c * ss, r + ms + a * ss, ss);
        }
        const int rc = mc_upload_planes(h, i0, i1, mix.data(), spp.data());
        if (rc) return rc;
    }
    return LBMGPU_OK;
}

}  // extern "C"
