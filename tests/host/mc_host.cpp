// Host build of the product's multicomponent per-cell functions
// (lattice-boltzmann-method_b200/csrc/mc_cell.cuh), driven over a periodic lattice in the
// kernels' order, so tests can compare the device logic with the reference's own solver
// on the CPU.  Test helper only; the product runs these functions on the GPU.
//
// mc_host_run: FP64 storage.  mc_host_run32: populations in FP32 with (shift != 0) or
// without the per-plane shift (the mean of each population plane over the fluid cells
// after Init, as the device takes it), records in FP64.  Both return the index of the record
// buffer that holds the final state.
#include <vector>

#include "mc_cell.cuh"

namespace {

template <typename S, typename RS>
int run(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx, float dt, int chem,
        int nsteps, S *pop0, S *pop1, RS *rec0, RS *rec1, int shift, unsigned *status) {
    using namespace lbm;
    static gas::Tables tab;
    gas::make_tables(*mech, tab);
    if (mech->n_species != 9) return -1;
    McArgsT<S, RS> A{};
    const UnitsF U = units_from_dx_dt(dx, dt);
    set_lattice_constants(tab, U);
    A.Nx = Nx;
    A.Ny = Ny;
    A.Nz = Nz;
    A.ncell = (long)Nx * Ny * Nz;
    A.sj = Nz;
    A.si = (long)Ny * Nz;
    A.ns = 9;
    A.dt = 1;
    A.chem = chem;
    A.U = U;
    A.tab = &tab;
    A.type = reinterpret_cast<const int8_t *>(type);
    A.status = status;
    for (long n = 0; n < A.ncell; ++n) mc_init_cell<9>(A, n, rec0, rec1, pop0);
    const int np = 27 * 10;
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
    S *pop[2] = {pop0, pop1};
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
        for (long n = 0; n < A.ncell; ++n)
            if (type[n] == 0) mc_collide_cell<9>(A, n);
        A.pop_src = pop[nx];
        for (long n = 0; n < A.ncell; ++n)
            if (type[n] == 0) mc_stream_moment_cell<9>(A, n);
        cur = nx;
        local = false;
    }
    return cur;
}

}  // namespace

extern "C" int mc_host_run(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                           float dt, int chem, int nsteps, double *pop0, double *pop1, double *rec0, double *rec1,
                           unsigned *status) {
    return run<double, double>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, 0, status);
}

extern "C" int mc_host_run32(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                             float dt, int chem, int nsteps, float *pop0, float *pop1, double *rec0, double *rec1,
                             int shift, unsigned *status) {
    return run<float, double>(Nx, Ny, Nz, type, mech, dx, dt, chem, nsteps, pop0, pop1, rec0, rec1, shift, status);
}
