// C entry points around the reference's own MULTICOMPONENT solver, compiled from the
// reference sources against the Cantera-API shim (oracle/shim) into
// oracle/_ref/libref_mc.so (REACTION off) and libref_mcr.so (REACTION on).
// Test infrastructure only: tests/, the fixture generator and bench.py's CPU baseline.
//
// Forwarded reference routines:
//   LBM::LBM(Nx,Ny,Nz,species)    src/lbm-main.cpp:39-118
//   LBM::Init                     src/lbm-init.cpp:85-146
//   LBM::loop                     src/lbm-main.cpp:149-196
//   LBM::Collide_Species/Collide/Streaming/TMS_BC/calculate_moment
#include <cstddef>
#include <cstring>
#include <omp.h>
#include <string>
#include <vector>

#include "lbm.hpp"
#include "output.hpp"
#include "restart_file.hpp"
#include "units.hpp"

Units_Conv units;   // normally defined by the case setup (src/setup.cpp:10)

extern "C" {

void ref_mc_set_mech(const lbmgpu_mech *m) { shim_set_mechanism(m); }
void ref_mc_set_units(float dx, float dt) { units.set_m_kg_s(dx, dt); }

// MIXTURE: size, type, p_tensor, rho, u, v, w, p, g, gpc, rhoe, energy_flux, temp, HRR
// SPECIES: size, X, rho, f, fpc, u, v, w
int ref_mc_layout(size_t *out, int n) {
    size_t v[21] = {sizeof(MIXTURE), offsetof(MIXTURE, type), offsetof(MIXTURE, p_tensor),
                    offsetof(MIXTURE, rho), offsetof(MIXTURE, u), offsetof(MIXTURE, v),
                    offsetof(MIXTURE, w), offsetof(MIXTURE, p), offsetof(MIXTURE, g),
                    offsetof(MIXTURE, gpc), offsetof(MIXTURE, rhoe), offsetof(MIXTURE, energy_flux),
                    offsetof(MIXTURE, temp), offsetof(MIXTURE, HRR),
                    sizeof(SPECIES), offsetof(SPECIES, X), offsetof(SPECIES, rho), offsetof(SPECIES, f),
                    offsetof(SPECIES, fpc), offsetof(SPECIES, u), offsetof(SPECIES, v)};
    int m = n < 21 ? n : 21;
    for (int i = 0; i < m; ++i) out[i] = v[i];
    return 21;
}

void *ref_mc_create(int NX, int NY, int NZ, int ns, const char *const *names) {
    std::vector<std::string> sp;
    for (int a = 0; a < ns; ++a) sp.emplace_back(names[a]);
    return new LBM(NX, NY, NZ, sp);
}

void ref_mc_destroy(void *h) {
    LBM *lb = static_cast<LBM *>(h);
    if (!lb) return;
    MIXTURE *base = &lb->mixture[0][0][0];
    for (int i = 0; i < lb->get_Nx(); ++i) delete[] lb->mixture[i];
    delete[] lb->mixture;
    delete[] base;
    for (size_t a = 0; a < lb->species.size(); ++a) {
        SPECIES *sb = &lb->species[a][0][0][0];
        for (int i = 0; i < lb->get_Nx(); ++i) delete[] lb->species[a][i];
        delete[] lb->species[a];
        delete[] sb;
    }
    delete lb;
}

int ref_mc_nx(void *h) { return static_cast<LBM *>(h)->get_Nx(); }
int ref_mc_ny(void *h) { return static_cast<LBM *>(h)->get_Ny(); }
int ref_mc_nz(void *h) { return static_cast<LBM *>(h)->get_Nz(); }
void *ref_mc_cells(void *h) { return &static_cast<LBM *>(h)->mixture[0][0][0]; }
void *ref_mc_species(void *h, int a) { return &static_cast<LBM *>(h)->species[a][0][0][0]; }
void ref_mc_set_threads(int n) { omp_set_num_threads(n); }
void ref_mc_init(void *h) { static_cast<LBM *>(h)->Init(); }
void ref_mc_loop(void *h, int n) { static_cast<LBM *>(h)->loop(n, 100000000); }

// The reference's own writers, into the current directory: write_restart ->
// ./restart%06d.dat (src/restart_file.cpp:274-350), OutputVTK -> ./field%06d.vtr
// (src/output.cpp:9-210).
void ref_mc_write_restart(void *h, int step) {
    int s = step;
    write_restart(s, static_cast<LBM *>(h));
}
void ref_mc_output_vtk(void *h, int nout) {
    int n = nout;
    OutputVTK(n, static_cast<LBM *>(h));
}

// read_restart (src/restart_file.cpp:352-440): a new LBM object from a restart file
void *ref_mc_read_restart(const char *path) { return new LBM(read_restart(std::string(path))); }

void ref_mc_phase(void *h, int which) {
    LBM *lb = static_cast<LBM *>(h);
    switch (which) {
        case 0: lb->Collide_Species(); break;
        case 1: lb->Collide(); break;
        case 2: lb->Streaming(); break;
        case 3: lb->TMS_BC(); break;
        case 4: lb->calculate_moment(); break;
        default: break;
    }
}

}  // extern "C"
