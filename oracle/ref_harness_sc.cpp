// C entry points around the reference's own single-component solver, compiled from
// the reference sources into oracle/_ref/libref_sc.so.  Test infrastructure only:
// used by tests/, by the fixture generator under tests/golden/ and by bench.py's
// CPU-baseline leg; never linked into the product.
//
// Every function forwards to the reference's code unchanged:
//   LBM::LBM(Nx,Ny,Nz,nu)        src/lbm-main.cpp:16-35
//   LBM::Init                     src/lbm-init.cpp:8-82
//   LBM::loop                     src/lbm-main.cpp:149-196
//   LBM::Collide/Streaming/TMS_BC/calculate_moment (the loop's phases)
//   calculate_feq                 src/headers/lbm.hpp:276-305
//   calculate_geq (polynomial)    src/lbm-edf.cpp:38-98
//   calculate_geq (moment form)   src/lbm-edf.cpp:100-138
//   calculate_gstr                src/lbm-edf.cpp:140-150
//   calculate_feq_geq             src/lbm-edf.cpp:153-164
//   fd_central/fd_fuw/fd_uw       src/headers/FD.hpp:108-127, src/FD.cpp:5-23, 64-74
#include <cstddef>
#include <cstring>
#include <omp.h>
#include "lbm.hpp"
#include "units.hpp"
#include "FD.hpp"

Units_Conv units;   // normally defined by the case setup (src/setup.cpp:10)

namespace {
LBM &scratch_lbm() {
    static LBM lb(1, 1, 1, 0.01);
    return lb;
}
}  // namespace

extern "C" {

// sizeof(MIXTURE) and the byte offsets of its fields, in this order:
// size, type, f, fpc, p_tensor, rho, u, v, w, p, g, gpc, rhoe, energy_flux, temp
int ref_sc_layout(size_t *out, int n) {
    size_t v[15] = {sizeof(MIXTURE),           offsetof(MIXTURE, type),
                    offsetof(MIXTURE, f),      offsetof(MIXTURE, fpc),
                    offsetof(MIXTURE, p_tensor), offsetof(MIXTURE, rho),
                    offsetof(MIXTURE, u),      offsetof(MIXTURE, v),
                    offsetof(MIXTURE, w),      offsetof(MIXTURE, p),
                    offsetof(MIXTURE, g),      offsetof(MIXTURE, gpc),
                    offsetof(MIXTURE, rhoe),   offsetof(MIXTURE, energy_flux),
                    offsetof(MIXTURE, temp)};
    int m = n < 15 ? n : 15;
    for (int i = 0; i < m; ++i) out[i] = v[i];
    return 15;
}

void *ref_sc_create(int NX, int NY, int NZ, double nu, double R, double gamma, double prtl) {
    LBM *lb = new LBM(NX, NY, NZ, nu);
    lb->set_gasconst(R);
    lb->set_gamma(gamma);
    lb->set_prtl(prtl);
    return lb;
}

void ref_sc_destroy(void *h) {
    LBM *lb = static_cast<LBM *>(h);
    if (!lb) return;
    MIXTURE *base = &lb->mixture[0][0][0];
    for (int i = 0; i < lb->get_Nx(); ++i) delete[] lb->mixture[i];
    delete[] lb->mixture;
    delete[] base;
    delete lb;
}

void *ref_sc_cells(void *h) { return &static_cast<LBM *>(h)->mixture[0][0][0]; }

void ref_sc_set_threads(int n) { omp_set_num_threads(n); }
int ref_sc_max_threads(void) { return omp_get_max_threads(); }

void ref_sc_init(void *h) { static_cast<LBM *>(h)->Init(); }

// Runs n time steps through LBM::loop.  The output cadence is pushed past the run so
// no VTK/restart files are written (loop counts from 1 each call: src/lbm-main.cpp:153).
void ref_sc_loop(void *h, int n) { static_cast<LBM *>(h)->loop(n, 100000000); }

void ref_sc_phase(void *h, int which) {
    LBM *lb = static_cast<LBM *>(h);
    switch (which) {
        case 0: lb->Collide(); break;
        case 1: lb->Streaming(); break;
        case 2: lb->TMS_BC(); break;
        case 3: lb->calculate_moment(); break;
        default: break;
    }
}

double ref_sc_feq(int l, double rho, const double *u, double theta, const double *corr) {
    double uu[3] = {u[0], u[1], u[2]}, cc[3] = {corr[0], corr[1], corr[2]};
    return scratch_lbm().calculate_feq(l, rho, uu, theta, cc);
}

double ref_sc_geq_poly(int l, double rho, double U, double theta, const double *v) {
    double vv[3] = {v[0], v[1], v[2]};
    return scratch_lbm().calculate_geq(l, rho, U, theta, vv);
}

double ref_sc_geq_moment(int l, double rhoe, const double *q, const double *R9, double theta) {
    double qq[3] = {q[0], q[1], q[2]};
    double RR[3][3];
    std::memcpy(RR, R9, sizeof(RR));
    return scratch_lbm().calculate_geq(l, rhoe, qq, RR, theta);
}

double ref_sc_gstr(int l, double geq, const double *dq) {
    double d[3] = {dq[0], dq[1], dq[2]};
    return scratch_lbm().calculate_gstr(l, geq, d);
}

void ref_sc_feq_geq(void *h, double *f, double *g, double rho, const double *vel, double T) {
    double vv[3] = {vel[0], vel[1], vel[2]};
    static_cast<LBM *>(h)->calculate_feq_geq(f, g, rho, vv, T);
}

double ref_fd_central(double l, double c, double r, double dx, double vel, int tl, int tr) {
    return fd_central(l, c, r, dx, vel, (short)tl, (short)tr);
}
double ref_fd_fuw(double l, double c, double r, double dx, double vel, int tl, int tr) {
    return fd_fuw(l, c, r, dx, vel, (short)tl, (short)tr);
}
double ref_fd_uw(double s0, double s1, double s2, double dx, double vel) {
    return fd_uw(s0, s1, s2, dx, vel);
}

}  // extern "C"
