// Cantera-API shim: the subset of Cantera 3.x's C++ interface that the reference's
// multicomponent sources call (ThermoPhase, Transport, Kinetics, Solution, newSolution,
// GasConstant, OneAtm, npos; list enumerated from src/lbm-*.cpp and src/impose_nscbc.cpp).
//
// TEST INFRASTRUCTURE ONLY: it lets the reference's own LBM code compile unchanged as the
// multicomponent oracle (oracle/_ref/libref_mc.so).  Cantera itself is not available, so
// the property values come from the published-method restatement in
// lattice-boltzmann-method_b200/csrc/gas.cuh -- parity at this boundary is unpinned.
//
// Semantics follow Cantera's documented behaviour for an ideal-gas phase: the state is
// (T, rho, Y); setMassFractions/setMoleFractions clip negatives to zero, normalise and
// keep T and rho; setState_TP/DP/UV solve for the missing variable.  newSolution ignores
// its file argument and returns a solution of the mechanism registered with
// shim_set_mechanism() (the reference hard-codes Cantera's bundled h2o2.yaml, which this
// environment does not have).
#pragma once
#include <cmath>
#include <cstddef>
#include <memory>
#include <string>
#include <vector>

#include "../../../lattice-boltzmann-method_b200/csrc/gas.cuh"

extern "C" void shim_set_mechanism(const lbmgpu_mech *m);

namespace Cantera {

const double GasConstant = gas::kR;
const double OneAtm = gas::kOneAtm;
const size_t npos = static_cast<size_t>(-1);

const gas::Tables &shim_tables();

class ThermoPhase {
  public:
    explicit ThermoPhase(const gas::Tables *t) : t_(t), Y_(t->ns, 0.0), X_(t->ns, 0.0) {
        Y_[0] = 1.0;
        update_X();
    }
    size_t nSpecies() const { return t_->ns; }
    size_t speciesIndex(const std::string &name) const;
    double molecularWeight(size_t k) const { return t_->m.W[k]; }
    double meanMolecularWeight() const { return W_; }
    double temperature() const { return T_; }
    double density() const { return rho_; }
    double pressure() const { return rho_ * GasConstant * T_ / W_; }
    double RT() const { return GasConstant * T_; }
    double massFraction(size_t k) const { return Y_[k]; }
    void getMoleFractions(double *x) const {
        for (int k = 0; k < t_->ns; ++k) x[k] = X_[k];
    }
    void setMassFractions(const double *y);
    void setMoleFractions(const double *x);
    void setState_TD(double T, double rho) {
        T_ = T;
        rho_ = rho;
    }
    void setState_TP(double T, double P) {
        T_ = T;
        rho_ = P * W_ / (GasConstant * T);
    }
    void setState_DP(double rho, double P) {
        rho_ = rho;
        T_ = P * W_ / (rho * GasConstant);
    }
    void setState_UV(double u, double v, double tol = 1e-9);  // Cantera 3.x default tolerance
    double cp_mass() const { return gas::cp_mass(*t_, Y_.data(), T_); }
    double cv_mass() const { return gas::cv_mass(*t_, Y_.data(), T_); }
    double intEnergy_mass() const { return gas::int_energy_mass(*t_, Y_.data(), T_); }
    double soundSpeed() const { return std::sqrt(cp_mass() / cv_mass() * GasConstant * T_ / W_); }
    void getPartialMolarEnthalpies(double *h) const {
        for (int k = 0; k < t_->ns; ++k) h[k] = gas::h_RT(*t_, k, T_) * GasConstant * T_;
    }
    const gas::Tables &tables() const { return *t_; }
    const double *X() const { return X_.data(); }
    const double *Y() const { return Y_.data(); }

  private:
    void update_X();
    const gas::Tables *t_;
    std::vector<double> Y_, X_;
    double T_ = 300.0, rho_ = 1.0, W_ = 1.0;
};

class Transport {
  public:
    explicit Transport(std::shared_ptr<ThermoPhase> th) : th_(std::move(th)) {}
    double viscosity() const;
    double thermalConductivity() const;
    void getSpeciesViscosities(double *mu) const;
    void getBinaryDiffCoeffs(size_t ld, double *d) const;

  private:
    std::shared_ptr<ThermoPhase> th_;
};

class Kinetics {
  public:
    explicit Kinetics(std::shared_ptr<ThermoPhase> th) : th_(std::move(th)) {}
    void getNetProductionRates(double *wdot) const;

  private:
    std::shared_ptr<ThermoPhase> th_;
};

class Solution {
  public:
    Solution();
    std::shared_ptr<ThermoPhase> thermo() { return thermo_; }
    std::shared_ptr<Transport> transport() { return transport_; }
    std::shared_ptr<Kinetics> kinetics() { return kinetics_; }

  private:
    std::shared_ptr<ThermoPhase> thermo_;
    std::shared_ptr<Transport> transport_;
    std::shared_ptr<Kinetics> kinetics_;
};

std::shared_ptr<Solution> newSolution(const std::string &file, const std::string &name = "",
                                      const std::string &transport = "");

}  // namespace Cantera
