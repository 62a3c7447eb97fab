// Host build of the product's multicomponent per-cell functions as a stateful lattice that
// steps phase by phase, with the slab decomposition's halo exchange hooks
// (lattice-boltzmann-method_b200/csrc/halo.cuh): the tests run one such lattice per gloo rank
// and compare the decomposed run with the single domain.  FP64 storage.  Test helper only;
// the product runs these functions on the GPU (csrc/mc.cu).
#include <vector>

#include "halo.cuh"
#include "mc_bc.cuh"

namespace {

using namespace lbm;

struct HostLat {
    gas::Tables tab;
    McArgsT<double, double> A{};
    std::vector<int8_t> type;
    std::vector<uint8_t> cf;
    std::vector<int> bid;
    std::vector<long> blist;
    std::vector<double> pop[2], rec[2], bst[2], props;
    unsigned status = 0;
    int cur = 0;
    bool local = true;
};

}  // namespace

// halo_lo / halo_hi mark the x ghost planes as halos of neighbouring slabs; nx_glob is the
// decomposed domain's Nx (ghosts included).  rec_init: the record planes of the uploaded
// setup state (mc_nrec(9) planes of Nx*Ny*Nz cells).
extern "C" void *mch_create(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                            float dt, int chem, int halo_lo, int halo_hi, int nx_glob, const double *rec_init) {
    if (mech->n_species != 9) return nullptr;
    HostLat *L = new HostLat();
    gas::make_tables(*mech, L->tab);
    const UnitsF U = units_from_dx_dt(dx, dt);
    set_lattice_constants(L->tab, U);
    McArgsT<double, double> &A = L->A;
    A.Nx = Nx;
    A.Ny = Ny;
    A.Nz = Nz;
    A.halo_lo = halo_lo;
    A.halo_hi = halo_hi;
    A.Nx_glob = nx_glob;
    A.ncell = (long)Nx * Ny * Nz;
    A.sj = Nz;
    A.si = (long)Ny * Nz;
    A.ns = 9;
    A.dt = 1;
    A.chem = chem;
    A.U = U;
    A.tab = &L->tab;
    L->type.assign(type, type + A.ncell);
    A.type = L->type.data();
    A.status = &L->status;
    // the upload's classification: fluid cells outside the halo planes, and among them
    // those with a boundary cell (not fluid, not periodic ghost) upstream
    L->cf.assign(A.ncell, 0);
    L->bid.assign(A.ncell, -1);
    for (long n = 0; n < A.ncell; ++n) {
        if (type[n] != T_F) continue;
        const long i = n / A.si;
        if ((i == 0 && halo_lo) || (i == Nx - 1 && halo_hi)) continue;
        uint8_t c = CF_FLUID;
        for (int l = 0; l < 27; ++l) {
            const int t = type[n - (long)cx(l) * A.si - (long)cy(l) * A.sj - cz(l)];
            if (t != T_F && t != T_P) c |= CF_SPECIAL;
        }
        if (c & CF_SPECIAL) {
            L->bid[n] = (int)L->blist.size();
            L->blist.push_back(n);
        }
        L->cf[n] = c;
    }
    A.cflag = L->cf.data();
    A.bid = L->bid.data();
    A.nb = (long)L->blist.size();
    const long nrec = mc_nrec(9), np = 27 * 10, nb = std::max<long>(A.nb, 1);
    for (int b = 0; b < 2; ++b) {
        L->rec[b].assign(rec_init, rec_init + nrec * A.ncell);
        L->pop[b].assign((size_t)np * A.ncell, 0.0);
        L->bst[b].assign((size_t)np * nb, 0.0);
    }
    L->props.assign((size_t)pr_count<9>() * A.ncell, 0.0);
    A.props = L->props.data();
    for (long n = 0; n < A.ncell; ++n) mc_init_cell<9>(A, n, L->rec[0].data(), L->rec[1].data(), L->pop[0].data());
    for (int q = 0; q < np; ++q)
        for (long b = 0; b < A.nb; ++b) L->bst[0][(size_t)q * nb + b] = L->pop[0][(long)q * A.ncell + L->blist[b]];
    return L;
}

// LBM::Collide_Species + LBM::Collide over the slab's fluid cells
extern "C" void mch_collide(void *h) {
    HostLat *L = static_cast<HostLat *>(h);
    McArgsT<double, double> &A = L->A;
    const int nx = 1 - L->cur;
    A.pop_src = L->pop[L->cur].data();
    A.pop_dst = L->pop[nx].data();
    A.pop_prev = L->local ? nullptr : L->pop[L->cur].data();
    A.rec_cur = L->rec[L->cur].data();
    A.rec_nxt = L->rec[nx].data();
    A.local = L->local;
    A.bst_cur = L->bst[L->cur].data();
    for (long n = 0; n < A.ncell; ++n)
        if (L->cf[n] & CF_FLUID) mc_collide_cell<9>(A, n);
}

// Streaming + TMS_BC + calculate_moment: the interior cells, then the boundary cells
extern "C" void mch_stream(void *h) {
    HostLat *L = static_cast<HostLat *>(h);
    McArgsT<double, double> &A = L->A;
    const int nx = 1 - L->cur;
    A.pop_src = L->pop[nx].data();
    A.bst_nxt = L->bst[nx].data();
    for (long n = 0; n < A.ncell; ++n)
        if (L->cf[n] == CF_FLUID) mc_stream_moment_cell<9>(A, n);
    for (long b = 0; b < A.nb; ++b) mc_special_cell<9>(A, L->blist[b], b);
    L->cur = nx;
    L->local = false;
}

// halo_pack_cell / halo_unpack_cell over the face plane: populations between mch_collide and
// mch_stream (the post-collision buffer), the record between steps
extern "C" void mch_halo(void *h, int face, int what, double *buf, int pack) {
    HostLat *L = static_cast<HostLat *>(h);
    const McArgsT<double, double> &A = L->A;
    double *pop = L->pop[1 - L->cur].data();
    double *rec = L->rec[L->cur].data();
    for (long jk = 0; jk < (long)A.Ny * A.Nz; ++jk) {
        if (pack)
            halo_pack_cell<9>(A, pop, rec, face, what, jk, buf);
        else
            halo_unpack_cell<9>(A, pop, rec, face, what, jk, buf);
    }
}

extern "C" long mch_halo_values(int what) { return halo_values(what, 9); }

// the current record planes (mc_nrec(9) x Nx*Ny*Nz) and the status bits
extern "C" unsigned mch_record(void *h, double *out) {
    HostLat *L = static_cast<HostLat *>(h);
    std::copy(L->rec[L->cur].begin(), L->rec[L->cur].end(), out);
    return L->status;
}

extern "C" void mch_destroy(void *h) { delete static_cast<HostLat *>(h); }
