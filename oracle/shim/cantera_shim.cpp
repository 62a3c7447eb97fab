// Implementation of the Cantera-API shim (see cantera/core.h).  Test infrastructure only.
#include <cstring>
#include <stdexcept>

#include "cantera/core.h"

namespace {
gas::Tables g_tables;
bool g_have = false;
}  // namespace

extern "C" void shim_set_mechanism(const lbmgpu_mech *m) {
    gas::make_tables(*m, g_tables);
    g_have = true;
}

namespace Cantera {

const gas::Tables &shim_tables() {
    if (!g_have) throw std::runtime_error("cantera shim: no mechanism registered (shim_set_mechanism)");
    return g_tables;
}

size_t ThermoPhase::speciesIndex(const std::string &name) const {
    for (int k = 0; k < t_->ns; ++k)
        if (name == t_->m.name[k]) return (size_t)k;
    return npos;
}

void ThermoPhase::update_X() {
    double s = 0.0;
    for (int k = 0; k < t_->ns; ++k) s += Y_[k] / t_->m.W[k];
    W_ = 1.0 / s;
    for (int k = 0; k < t_->ns; ++k) X_[k] = Y_[k] / t_->m.W[k] * W_;
}

void ThermoPhase::setMassFractions(const double *y) {
    double s = 0.0;
    for (int k = 0; k < t_->ns; ++k) {
        Y_[k] = y[k] > 0.0 ? y[k] : 0.0;
        s += Y_[k];
    }
    for (int k = 0; k < t_->ns; ++k) Y_[k] /= s;
    update_X();
}

void ThermoPhase::setMoleFractions(const double *x) {
    double s = 0.0;
    for (int k = 0; k < t_->ns; ++k) {
        X_[k] = x[k] > 0.0 ? x[k] : 0.0;
        s += X_[k];
    }
    double w = 0.0;
    for (int k = 0; k < t_->ns; ++k) {
        X_[k] /= s;
        w += X_[k] * t_->m.W[k];
    }
    W_ = w;
    for (int k = 0; k < t_->ns; ++k) Y_[k] = X_[k] * t_->m.W[k] / w;
}

void ThermoPhase::setState_UV(double u, double v, double tol) {
    rho_ = 1.0 / v;
    double T;
    const int it = gas::T_from_u(*t_, Y_.data(), u, T_, tol > 1e-14 ? tol : 1e-14, 100, T);
    if (it < 0) throw std::runtime_error("cantera shim: setState_UV did not converge");
    T_ = T;
}

double Transport::viscosity() const {
    const gas::Tables &t = th_->tables();
    double mu[gas::MAXS];
    getSpeciesViscosities(mu);
    return gas::wilke(t, th_->X(), mu);
}

double Transport::thermalConductivity() const {
    const gas::Tables &t = th_->tables();
    double mu[gas::MAXS];
    getSpeciesViscosities(mu);
    return gas::mix_cond(t, th_->X(), th_->temperature(), th_->pressure(), mu);
}

void Transport::getSpeciesViscosities(double *mu) const {
    const gas::Tables &t = th_->tables();
    for (int k = 0; k < t.ns; ++k) mu[k] = gas::species_visc(t, k, th_->temperature());
}

void Transport::getBinaryDiffCoeffs(size_t ld, double *d) const {
    const gas::Tables &t = th_->tables();
    const double T = th_->temperature(), P = th_->pressure();
    for (int j = 0; j < t.ns; ++j)
        for (int k = 0; k < t.ns; ++k) d[ld * j + k] = gas::binary_diff(t, k, j, T, P);
}

void Kinetics::getNetProductionRates(double *wdot) const {
    const gas::Tables &t = th_->tables();
    double C[gas::MAXS];
    for (int k = 0; k < t.ns; ++k) C[k] = th_->density() * th_->Y()[k] / t.m.W[k];
    gas::net_production(t, th_->temperature(), C, wdot);
}

Solution::Solution() {
    thermo_ = std::make_shared<ThermoPhase>(&shim_tables());
    transport_ = std::make_shared<Transport>(thermo_);
    kinetics_ = std::make_shared<Kinetics>(thermo_);
}

std::shared_ptr<Solution> newSolution(const std::string &, const std::string &, const std::string &) {
    return std::make_shared<Solution>();
}

}  // namespace Cantera
