// Host build of the compiled H2/air kinetics (kinetics_h2_air_9.cuh, generated by
// gen_kinetics.py) beside the table-driven kinetics and integrators of gas.cuh / chem.cuh,
// for tests/test_kinetics_compiled.py.  Built without contraction of multiply-adds, so that
// both evaluate their expressions exactly as written.
#include <stdlib.h>

#include "chem.cuh"
#include "kinetics_h2_air_9.cuh"

namespace K9 = kin_h2_air_9;

extern "C" {

void *kh_tables(const lbmgpu_mech *m) {
    gas::Tables *t = new gas::Tables();
    gas::make_tables(*m, *t);
    return t;
}
void kh_free(void *t) { delete (gas::Tables *)t; }
int kh_matches(const lbmgpu_mech *m) { return K9::matches(*m) ? 1 : 0; }

// the reactor's right-hand side at (rho, y): tables (rate_factors + reactor_rhs_k), the
// dense table form the device integrator uses, and the compiled kinetics
void kh_rhs_tables(const void *t, double rho, const double *y, double *F) {
    gas::reactor_rhs(*(const gas::Tables *)t, rho, y, F);
}
void kh_rhs_dense(const void *t, double rho, const double *y, double *F) {
    gas::reactor_rhs_dense<K9::NS>(*(const gas::Tables *)t, rho, y, F);
}
void kh_rhs_compiled(double rho, const double *y, double *F) {
    K9::Thermo th;
    K9::thermo(y[K9::NS], th);
    K9::rhs_t(th, rho, y, F);
}

// one ROS2 advance over dt: the host integrator over the tables (ros2_advance), and the
// compile-time-sized integrator with the table kinetics and with the compiled kinetics
int kh_ros2_tables(const void *t, double rho, double *Y, double *T, double dt) {
    return gas::ros2_advance(*(const gas::Tables *)t, rho, Y, *T, dt);
}
int kh_ros2_dense(const void *t, double rho, double *Y, double *T, double dt) {
    return gas::ros2_advance_n<K9::NS>(*(const gas::Tables *)t, rho, Y, *T, dt);
}
int kh_ros2_compiled(double rho, double *Y, double *T, double dt) {
    return gas::ros2_advance_k<K9::NS>(K9::Kinetics{}, rho, Y, *T, dt);
}
}

extern "C" {
// the compiled kinetics' analytic Jacobian d(Y, T)/dt / d(Y, T) (row-major 10 x 10 over the
// state; the rows and columns of the inert species, which are not unknowns of the iteration
// system, are left zero) and the right-hand side rhs_jac returns with it
void kh_jac_compiled(double rho, const double *y, double *J, double *F) {
    constexpr int m = K9::Kinetics::kSys, n = K9::NS + 1;
    K9::Thermo th;
    K9::thermo(y[K9::NS], th);
    gas::RegMat<m> Jm;
    K9::rhs_jac(th, rho, y, F, 1.0, Jm);
    for (int i = 0; i < n * n; ++i) J[i] = 0.0;
    for (int r = 0; r < m; ++r)
        for (int c = 0; c < m; ++c) J[K9::Kinetics::sys_full(r) * n + K9::Kinetics::sys_full(c)] = Jm(r, c);
}
// the state components that are unknowns of the compiled kinetics' iteration system
int kh_sys_full(int *full) {
    for (int i = 0; i < K9::Kinetics::kSys; ++i) full[i] = K9::Kinetics::sys_full(i);
    return K9::Kinetics::kSys;
}
}
