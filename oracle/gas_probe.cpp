// C entry points onto the gas-property library (lattice-boltzmann-method_b200/csrc/gas.cuh)
// compiled for the host, for the property tests.  Test infrastructure only.
#include "../lattice-boltzmann-method_b200/csrc/gas.cuh"
#include "../lattice-boltzmann-method_b200/csrc/chem.cuh"

static gas::Tables g_t;

extern "C" {
void gp_set_mech(const lbmgpu_mech *m) { gas::make_tables(*m, g_t); }
double gp_species_visc(int k, double T) { return gas::species_visc(g_t, k, T); }
double gp_binary_diff(int k, int j, double T, double P) { return gas::binary_diff(g_t, k, j, T, P); }
double gp_species_cond(int k, double T, double P) {
    (void)P;
    return gas::species_cond(g_t, k, T);
}
double gp_mix_visc(const double *X, double T) {
    double mu[gas::MAXS];
    for (int k = 0; k < g_t.ns; ++k) mu[k] = gas::species_visc(g_t, k, T);
    return gas::wilke(g_t, X, mu);
}
double gp_mix_cond(const double *X, double T, double P) {
    double mu[gas::MAXS];
    for (int k = 0; k < g_t.ns; ++k) mu[k] = gas::species_visc(g_t, k, T);
    return gas::mix_cond(g_t, X, T, P, mu);
}
double gp_cp_mass(const double *Y, double T) { return gas::cp_mass(g_t, Y, T); }
double gp_cv_mass(const double *Y, double T) { return gas::cv_mass(g_t, Y, T); }
double gp_int_energy(const double *Y, double T) { return gas::int_energy_mass(g_t, Y, T); }
double gp_h_RT(int k, double T) { return gas::h_RT(g_t, k, T); }
double gp_s_R(int k, double T) { return gas::s_R(g_t, k, T); }
double gp_cp_R(int k, double T) { return gas::cp_R(g_t, k, T); }
int gp_T_from_u(const double *Y, double u, double T0, double *T) { return gas::T_from_u(g_t, Y, u, T0, 1e-14, 100, *T); }
void gp_wdot(double T, const double *C, double *w) { gas::net_production(g_t, T, C, w); }
int gp_n_reactions() { return g_t.m.n_reactions; }
void gp_rates_of_progress(double T, const double *C, double *qf, double *qr) {
    gas::RateT K;
    gas::rate_factors(g_t, T, K);
    for (int r = 0; r < g_t.m.n_reactions; ++r) gas::rate_of_progress(g_t, K, C, r, qf[r], qr[r]);
}
void gp_reactor_rhs(double rho, const double *y, double *F) { gas::reactor_rhs(g_t, rho, y, F); }
int gp_ros2(double rho, double *Y, double *T, double dt) { return gas::ros2_advance(g_t, rho, Y, *T, dt); }
}
