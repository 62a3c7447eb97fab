// Host build of the product's multicomponent per-cell functions
// (lattice-boltzmann-method_b200/csrc/mc_cell.cuh, mc_bc.cuh), driven over a lattice in the
// kernels' order (periodic interior cells and the boundary cells' compact list), so tests can compare the device logic with the reference's own solver
// on the CPU.  Test helper only; the product runs these functions on the GPU.
//
// mc_host_run: FP64 storage (9 or 6 species); with fout (27*(ns+1) planes of every cell) non-null it also
// returns the final streamed populations of the fluid cells.  mc_host_run32: populations in FP32 with (shift != 0) or
// without the per-plane shift (the mean of each population plane over the fluid cells
// after Init, as the device takes it), records in FP64.  Both return the index of the record
// buffer that holds the final state.
#include <algorithm>
#include <vector>

#include "mc_bc.cuh"

namespace {

template <int NS, typename S, typename RS>
int run_ns(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx, float dt, int chem,
           int nsteps, S *pop0, S *pop1, RS *rec0, RS *rec1, int shift, unsigned *status, double *fout) {
    using namespace lbm;
    static gas::Tables tab;
    gas::make_tables(*mech, tab);
    McArgsT<S, RS> A{};
    const UnitsF U = units_from_dx_dt(dx, dt);
    set_lattice_constants(tab, U);
    A.Nx = Nx;
    A.Nx_glob = Nx;  // one domain: no halo planes
    A.Ny = Ny;
    A.Nz = Nz;
    A.ncell = (long)Nx * Ny * Nz;
    A.sj = Nz;
    A.si = (long)Ny * Nz;
    A.ns = NS;
    A.dt = 1;
    A.chem = chem;
    A.U = U;
    A.tab = &tab;
    A.type = reinterpret_cast<const int8_t *>(type);
    A.status = status;
    // classification as the upload does it: fluid cells, and among them those with a
    // boundary cell (not fluid, not periodic ghost) upstream
    std::vector<uint8_t> cf(A.ncell, 0);
    std::vector<int> bid(A.ncell, -1);
    std::vector<long> blist;
    for (long n = 0; n < A.ncell; ++n) {
        if (type[n] != T_F) continue;
        uint8_t c = CF_FLUID;
        for (int l = 0; l < 27; ++l) {
            const int t = type[n - (long)cx(l) * A.si - (long)cy(l) * A.sj - cz(l)];
            if (t != T_F && t != T_P) c |= CF_SPECIAL;
        }
        if (c & CF_SPECIAL) {
            bid[n] = (int)blist.size();
            blist.push_back(n);
        }
        cf[n] = c;
    }
    A.cflag = cf.data();
    A.bid = bid.data();
    A.nb = (long)blist.size();
    std::vector<double> props((size_t)pr_count<NS>() * A.ncell);
    A.props = props.data();
    for (long n = 0; n < A.ncell; ++n) mc_init_cell<NS>(A, n, rec0, rec1, pop0);
    const int np = 27 * (NS + 1);
    std::vector<double> sh(np, 0.0);
    if (shift) {
        long cnt = 0;
        for (long n = 0; n < A.ncell; ++n) cnt += type[n] == 0;
        for (int q = 0; q < np; ++q) {
            double s = 0.0;
            for (long n = 0; n < A.ncell; ++n)
                if (type[n] == 0) s += (double)pop0[(long)q * A.ncell + n];
            sh[q] = s / (double)cnt;
            for (long n = 0; n < A.ncell; ++n) {
                pop0[(long)q * A.ncell + n] = (S)((double)pop0[(long)q * A.ncell + n] - sh[q]);
                pop1[(long)q * A.ncell + n] = (S)((double)pop1[(long)q * A.ncell + n] - sh[q]);
            }
        }
        A.shift = sh.data();
    }
    const long nb = std::max<long>(A.nb, 1);
    std::vector<S> bst0((size_t)np * nb), bst1((size_t)np * nb);
    for (int q = 0; q < np; ++q)
        for (long b = 0; b < A.nb; ++b) bst0[(size_t)q * nb + b] = pop0[(long)q * A.ncell + blist[b]];
    S *pop[2] = {pop0, pop1};
    S *bst[2] = {bst0.data(), bst1.data()};
    RS *rc[2] = {rec0, rec1};
    int cur = 0;
    bool local = true;
    for (int s = 0; s < nsteps; ++s) {
        const int nx = 1 - cur;
        A.pop_src = pop[cur];
        A.pop_dst = pop[nx];
        A.pop_prev = local ? nullptr : pop[cur];
        A.rec_cur = rc[cur];
        A.rec_nxt = rc[nx];
        A.local = local;
        A.bst_cur = bst[cur];
        for (long n = 0; n < A.ncell; ++n)
            if (type[n] == 0) mc_collide_cell<NS>(A, n);
        A.pop_src = pop[nx];
        A.bst_nxt = bst[nx];
        for (long n = 0; n < A.ncell; ++n)
            if (cf[n] == CF_FLUID) mc_stream_moment_cell<NS>(A, n);
        for (long b = 0; b < A.nb; ++b) mc_special_cell<NS>(A, blist[b], b);
        cur = nx;
        local = false;
    }
    // the streamed (and boundary-treated) populations of the fluid cells, as a download
    // returns them
    if (fout && nsteps > 0)
        for (long n = 0; n < A.ncell; ++n) {
            if (!(cf[n] & CF_FLUID)) continue;
            McPull pp;
            mc_pull(A, n, pp);
            for (int q = 0; q < np; ++q)
                fout[(long)q * A.ncell + n] = (cf[n] & CF_SPECIAL) ? ldpop_b(A, bst[cur], q, (long)bid[n])
                                                                 : ldpop(A, pop[cur], q, pull_idx(pp, q % 27));
        }
    return cur;
}

// the species counts the device kernels are built for
template <typename S, typename RS>
int run(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx, float dt, int chem,
        int nsteps, S *pop0, S *pop1, RS *rec0, RS *rec1, int shift, unsigned *status, double *fout) {
    if (mech->n_species == 9)
        return run_ns<9>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, shift, status, fout);
    if (mech->n_species == 6)
        return run_ns<6>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, shift, status, fout);
    return -1;
}

}  // namespace

extern "C" int mc_host_run(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                           float dt, int chem, int nsteps, double *pop0, double *pop1, double *rec0, double *rec1,
                           unsigned *status, double *fout) {
    return run<double, double>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, 0, status, fout);
}

extern "C" int mc_host_run32(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                             float dt, int chem, int nsteps, float *pop0, float *pop1, double *rec0, double *rec1,
                             int shift, unsigned *status) {
    return run<float, double>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, shift, status,
                              nullptr);
}

// The surrogate's element-conserving projector and its application (surrogate.cuh).
extern "C" void sur_projector_host(const lbmgpu_mech *mech, double *proj) {
    double el[9][LBMGPU_MAX_ELEMENTS], W[9];
    for (int k = 0; k < 9; ++k) {
        W[k] = mech->W[k];
        for (int e = 0; e < LBMGPU_MAX_ELEMENTS; ++e) el[k][e] = mech->elements[k][e];
    }
    lbm::sur_projector<9>(el, W, proj);
}

extern "C" void sur_conserve_host(const double *proj, double *dY) { lbm::sur_conserve<9>(proj, dY); }

// One ROS2 step (chem.cuh) of a constant-volume adiabatic reactor per row: rho [kg/m^3],
// Y [n][9] and T [n] [K] advanced in place over dt [s].  Returns the number of rows whose
// integration failed.
extern "C" long ros2_host(const lbmgpu_mech *mech, long n, const double *rho, double *Y, double *T, double dt) {
    static gas::Tables tab;
    gas::make_tables(*mech, tab);
    long bad = 0;
    for (long r = 0; r < n; ++r)
        if (gas::ros2_advance(tab, rho[r], Y + 9 * r, T[r], dt) < 0) ++bad;
    return bad;
}
