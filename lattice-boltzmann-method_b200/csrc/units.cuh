// SI <-> lattice unit conversions with the reference's rounding (reference class
// Units_Conv, src/headers/units.hpp:8-131).  The reference keeps the four base units as
// float and evaluates every conversion in float (or in double where a helper returns
// double -- sq() and cb() take and return double, src/headers/math_util.hpp), returning
// float.  Each function below performs the same operations in the same order, so a
// value crossing the boundary is rounded exactly where the reference rounds it.
#pragma once

#if defined(__CUDACC__)
#define UNITS_HD __host__ __device__ __forceinline__
#else
#define UNITS_HD inline
#endif

namespace lbm {

struct UnitsF {
    float m, kg, s, K;
};

// units.set_m_kg_s(dx, dt) (units.hpp:32-44): m = dx, kg = m^3, s = dt, K = 12000.
inline UnitsF units_from_dx_dt(float dx, float dt) {
    UnitsF u;
    u.m = (float)(dx / 1.0);
    const double md = (double)u.m;
    u.kg = (float)(1.0 / 1.0 * (md * md * md));
    u.s = (float)(dt / 1.0);
    u.K = 12000.0f;
    return u;
}

UNITS_HD double dsq(double a) { return a * a; }
UNITS_HD double dcb(double a) { return a * a * a; }

// SI -> lattice
UNITS_HD float u_temp(const UnitsF &U, float si) { return si / U.K; }
UNITS_HD float u_energy_mass(const UnitsF &U, float si) { return si * (U.s * U.s) / (U.m * U.m); }
UNITS_HD float u_u(const UnitsF &U, float si) { return si * U.s / U.m; }
UNITS_HD float u_rho(const UnitsF &U, float si) { return (float)((double)si * dcb(U.m) / (double)U.kg); }
UNITS_HD float u_rho_dot(const UnitsF &U, float si) {
    return (float)((double)si * dcb(U.m) * (double)U.s / (double)U.kg);
}
UNITS_HD float u_nu(const UnitsF &U, float si) { return (float)((double)(si * U.s) / dsq(U.m)); }
UNITS_HD float u_mu(const UnitsF &U, float si) { return si * U.s * U.m / U.kg; }
UNITS_HD float u_cond(const UnitsF &U, float si) { return si * U.s * U.s * U.s * U.K / (U.kg * U.m); }
UNITS_HD float u_cp(const UnitsF &U, float si) { return si * U.s * U.s * U.K / (U.m * U.m); }
UNITS_HD float u_p(const UnitsF &U, float si) { return (float)((double)si * ((double)U.m * dsq(U.s)) / (double)U.kg); }
UNITS_HD float u_hrr(const UnitsF &U, float si) {
    return (float)((double)si / ((double)U.kg * dsq(U.m) / dcb(U.s)));
}
// lattice -> SI
UNITS_HD float si_temp(const UnitsF &U, float t) { return t * U.K; }
UNITS_HD float si_energy_mass(const UnitsF &U, float e) { return e * (U.m * U.m) / (U.s * U.s); }
UNITS_HD float si_rho(const UnitsF &U, float r) { return (float)((double)(r * U.kg) / dcb(U.m)); }
UNITS_HD float si_p(const UnitsF &U, float p) { return (float)((double)(p * U.kg) / ((double)U.m * dsq(U.s))); }
UNITS_HD float si_u(const UnitsF &U, float u) { return u * U.m / U.s; }
UNITS_HD float si_hrr(const UnitsF &U, float h) {
    return (float)((double)h * ((double)U.kg * dsq(U.m) / dcb(U.s)));
}

}  // namespace lbm
