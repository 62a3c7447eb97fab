// Host build of the product's multicomponent per-cell functions
// (lattice-boltzmann-method_b200/csrc/mc_cell.cuh), driven over a periodic lattice in the
// kernels' order, so tests can compare the device logic with the reference's own solver
// on the CPU.  Test helper only; the product runs these functions on the GPU.
#include <vector>

#include "mc_cell.cuh"

extern "C" int mc_host_run(int Nx, int Ny, int Nz, const signed char *type, const lbmgpu_mech *mech, float dx,
                           float dt, int chem, int nsteps, double *pop0, double *pop1, double *rec0, double *rec1,
                           int do_init, unsigned *status) {
    using namespace lbm;
    static gas::Tables tab;
    gas::make_tables(*mech, tab);
    if (mech->n_species != 9) return -1;
    McArgs A{};
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
    if (do_init)
        for (long n = 0; n < A.ncell; ++n) mc_init_cell<9>(A, n, rec0, rec1, pop0);
    double *pop[2] = {pop0, pop1};
    double *rc[2] = {rec0, rec1};
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
