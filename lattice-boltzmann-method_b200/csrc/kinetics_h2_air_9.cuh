// Generated by gen_kinetics.py from the mechanism h2_air_9 -- do not edit; `make` regenerates it.
// Its kinetics as straight-line code: gas.cuh's rate_factors and reactor_rhs_k (thermo, rhs_t)
// and their analytic Jacobian (rhs_jac) with the mechanism's constants inlined.
#pragma once
#include <math.h>
#include "gas.cuh"

namespace kin_h2_air_9 {

constexpr int NS = 9, NR = 23, NF = 2;

// Whether `m` is the mechanism compiled here (every quantity the kinetics read).
inline bool matches(const lbmgpu_mech &m) {
    if (m.n_species != 9 || m.n_reactions != 23) return false;
    if (m.W[0] != 2.016 || m.T_mid[0] != 1000.0) return false;
    if (m.nasa_lo[0][0] != 2.37694204 || m.nasa_hi[0][0] != 2.90207649) return false;
    if (m.nasa_lo[0][1] != 0.00773916922 || m.nasa_hi[0][1] != 0.000868992581) return false;
    if (m.nasa_lo[0][2] != -1.88735073e-05 || m.nasa_hi[0][2] != -1.6586443e-07) return false;
    if (m.nasa_lo[0][3] != 1.95517114e-08 || m.nasa_hi[0][3] != 1.90851899e-11) return false;
    if (m.nasa_lo[0][4] != -7.17095663e-12 || m.nasa_hi[0][4] != -9.31121789e-16) return false;
    if (m.nasa_lo[0][5] != -921.173081 || m.nasa_hi[0][5] != -797.948726) return false;
    if (m.nasa_lo[0][6] != 0.547184736 || m.nasa_hi[0][6] != -0.84559132) return false;
    if (m.W[1] != 1.008 || m.T_mid[1] != 1000.0) return false;
    if (m.nasa_lo[1][0] != 2.49975925 || m.nasa_hi[1][0] != 2.49985211) return false;
    if (m.nasa_lo[1][1] != 6.73824499e-07 || m.nasa_hi[1][1] != 2.34582548e-07) return false;
    if (m.nasa_lo[1][2] != 1.11807261e-09 || m.nasa_hi[1][2] != -1.16171641e-10) return false;
    if (m.nasa_lo[1][3] != -3.70192126e-12 || m.nasa_hi[1][3] != 2.25708298e-14) return false;
    if (m.nasa_lo[1][4] != 2.14233822e-15 || m.nasa_hi[1][4] != -1.52992005e-18) return false;
    if (m.nasa_lo[1][5] != 25473.7665 || m.nasa_hi[1][5] != 25473.8024) return false;
    if (m.nasa_lo[1][6] != -0.445574009 || m.nasa_hi[1][6] != -0.445864645) return false;
    if (m.W[2] != 31.998 || m.T_mid[2] != 1000.0) return false;
    if (m.nasa_lo[2][0] != 3.78498258 || m.nasa_hi[2][0] != 3.65980488) return false;
    if (m.nasa_lo[2][1] != -0.00302002233 || m.nasa_hi[2][1] != 0.000659877372) return false;
    if (m.nasa_lo[2][2] != 9.92029171e-06 || m.nasa_hi[2][2] != -1.44158172e-07) return false;
    if (m.nasa_lo[2][3] != -9.77840434e-09 || m.nasa_hi[2][3] != 2.14656037e-11) return false;
    if (m.nasa_lo[2][4] != 3.28877702e-12 || m.nasa_hi[2][4] != -1.36503784e-15) return false;
    if (m.nasa_lo[2][5] != -1064.13589 || m.nasa_hi[2][5] != -1216.03048) return false;
    if (m.nasa_lo[2][6] != 3.64780709 || m.nasa_hi[2][6] != 3.42074148) return false;
    if (m.W[3] != 15.999 || m.T_mid[3] != 1000.0) return false;
    if (m.nasa_lo[3][0] != 3.15906526 || m.nasa_hi[3][0] != 2.55160087) return false;
    if (m.nasa_lo[3][1] != -0.00321509999 || m.nasa_hi[3][1] != -3.83085457e-05) return false;
    if (m.nasa_lo[3][2] != 6.49255543e-06 || m.nasa_hi[3][2] != 8.43197478e-10) return false;
    if (m.nasa_lo[3][3] != -5.98755115e-09 || m.nasa_hi[3][3] != 4.01267136e-12) return false;
    if (m.nasa_lo[3][4] != 2.06876117e-12 || m.nasa_hi[3][4] != -4.17476574e-16) return false;
    if (m.nasa_lo[3][5] != 29129.8453 || m.nasa_hi[3][5] != 29228.7628) return false;
    if (m.nasa_lo[3][6] != 2.09078344 || m.nasa_hi[3][6] != 4.87617014) return false;
    if (m.W[4] != 18.015 || m.T_mid[4] != 1000.0) return false;
    if (m.nasa_lo[4][0] != 4.20147551 || m.nasa_hi[4][0] != 2.73117512) return false;
    if (m.nasa_lo[4][1] != -0.00205583546 || m.nasa_hi[4][1] != 0.00295136995) return false;
    if (m.nasa_lo[4][2] != 6.56547207e-06 || m.nasa_hi[4][2] != -8.35359785e-07) return false;
    if (m.nasa_lo[4][3] != -5.5290696e-09 || m.nasa_hi[4][3] != 1.26088593e-10) return false;
    if (m.nasa_lo[4][4] != 1.78282605e-12 || m.nasa_hi[4][4] != -8.40531676e-15) return false;
    if (m.nasa_lo[4][5] != -30295.0066 || m.nasa_hi[4][5] != -29916.9082) return false;
    if (m.nasa_lo[4][6] != -0.860610906 || m.nasa_hi[4][6] != 6.55183) return false;
    if (m.W[5] != 17.007 || m.T_mid[5] != 1000.0) return false;
    if (m.nasa_lo[5][0] != 3.97585165 || m.nasa_hi[5][0] != 2.84581721) return false;
    if (m.nasa_lo[5][1] != -0.00228555291 || m.nasa_hi[5][1] != 0.00109723818) return false;
    if (m.nasa_lo[5][2] != 4.33442882e-06 || m.nasa_hi[5][2] != -2.89121101e-07) return false;
    if (m.nasa_lo[5][3] != -3.5992664e-09 || m.nasa_hi[5][3] != 4.0909991e-11) return false;
    if (m.nasa_lo[5][4] != 1.2670693e-12 || m.nasa_hi[5][4] != -2.31382258e-15) return false;
    if (m.nasa_lo[5][5] != 3393.41137 || m.nasa_hi[5][5] != 3717.0661) return false;
    if (m.nasa_lo[5][6] != -0.0355397262 || m.nasa_hi[5][6] != 5.80339915) return false;
    if (m.W[6] != 34.014 || m.T_mid[6] != 1000.0) return false;
    if (m.nasa_lo[6][0] != 4.2385416 || m.nasa_hi[6][0] != 4.5401748) return false;
    if (m.nasa_lo[6][1] != -0.000249610911 || m.nasa_hi[6][1] != 0.00415970971) return false;
    if (m.nasa_lo[6][2] != 1.59857901e-05 || m.nasa_hi[6][2] != -1.30876777e-06) return false;
    if (m.nasa_lo[6][3] != -2.06919945e-08 || m.nasa_hi[6][3] != 2.00823615e-10) return false;
    if (m.nasa_lo[6][4] != 8.2976632e-12 || m.nasa_hi[6][4] != -1.15509243e-14) return false;
    if (m.nasa_lo[6][5] != -17648.6003 || m.nasa_hi[6][5] != -17951.4029) return false;
    if (m.nasa_lo[6][6] != 3.58850097 || m.nasa_hi[6][6] != 0.855881745) return false;
    if (m.W[7] != 33.006 || m.T_mid[7] != 1000.0) return false;
    if (m.nasa_lo[7][0] != 4.2625125 || m.nasa_hi[7][0] != 4.1056401) return false;
    if (m.nasa_lo[7][1] != -0.00445642032 || m.nasa_hi[7][1] != 0.00204046836) return false;
    if (m.nasa_lo[7][2] != 2.05164934e-05 || m.nasa_hi[7][2] != -3.65877562e-07) return false;
    if (m.nasa_lo[7][3] != -2.35794011e-08 || m.nasa_hi[7][3] != 1.85973044e-11) return false;
    if (m.nasa_lo[7][4] != 9.05614257e-12 || m.nasa_hi[7][4] != 4.98818315e-16) return false;
    if (m.nasa_lo[7][5] != 262.442356 || m.nasa_hi[7][5] != 43.2898769) return false;
    if (m.nasa_lo[7][6] != 3.88223684 || m.nasa_hi[7][6] != 3.30808126) return false;
    if (m.W[8] != 28.014 || m.T_mid[8] != 1000.0) return false;
    if (m.nasa_lo[8][0] != 3.53603521 || m.nasa_hi[8][0] != 2.9380297) return false;
    if (m.nasa_lo[8][1] != -0.000158270944 || m.nasa_hi[8][1] != 0.0014183803) return false;
    if (m.nasa_lo[8][2] != -4.26984251e-07 || m.nasa_hi[8][2] != -5.03281045e-07) return false;
    if (m.nasa_lo[8][3] != 2.3754259e-09 || m.nasa_hi[8][3] != 8.07555464e-11) return false;
    if (m.nasa_lo[8][4] != -1.39708206e-12 || m.nasa_hi[8][4] != -4.76064275e-15) return false;
    if (m.nasa_lo[8][5] != -1047.49645 || m.nasa_hi[8][5] != -917.18099) return false;
    if (m.nasa_lo[8][6] != 2.94603724 || m.nasa_hi[8][6] != 5.95521985) return false;
    if (m.rtype[0] != 1 || m.reversible[0] != 1 || m.n_reac[0] != 1 || m.n_prod[0] != 1) return false;
    if (m.reac[0][0] != 0 || m.nu_reac[0][0] != 1.0 || m.order_reac[0][0] != 1.0) return false;
    if (m.prod[0][0] != 1 || m.nu_prod[0][0] != 2.0) return false;
    if (m.A[0] != 4.577000000000001e+16 || m.b[0] != -1.4 || m.Ea[0] != 436809600.0) return false;
    if (m.eff[0][0] != 2.5) return false;
    if (m.eff[0][1] != 1.0) return false;
    if (m.eff[0][2] != 1.0) return false;
    if (m.eff[0][3] != 1.0) return false;
    if (m.eff[0][4] != 12.0) return false;
    if (m.eff[0][5] != 1.0) return false;
    if (m.eff[0][6] != 1.0) return false;
    if (m.eff[0][7] != 1.0) return false;
    if (m.eff[0][8] != 1.0) return false;
    if (m.rtype[1] != 0 || m.reversible[1] != 1 || m.n_reac[1] != 2 || m.n_prod[1] != 2) return false;
    if (m.reac[1][0] != 0 || m.nu_reac[1][0] != 1.0 || m.order_reac[1][0] != 1.0) return false;
    if (m.reac[1][1] != 3 || m.nu_reac[1][1] != 1.0 || m.order_reac[1][1] != 1.0) return false;
    if (m.prod[1][0] != 1 || m.nu_prod[1][0] != 1.0) return false;
    if (m.prod[1][1] != 5 || m.nu_prod[1][1] != 1.0) return false;
    if (m.A[1] != 50.80000000000001 || m.b[1] != 2.67 || m.Ea[1] != 26325728.0) return false;
    if (m.rtype[2] != 0 || m.reversible[2] != 1 || m.n_reac[2] != 2 || m.n_prod[2] != 2) return false;
    if (m.reac[2][0] != 0 || m.nu_reac[2][0] != 1.0 || m.order_reac[2][0] != 1.0) return false;
    if (m.reac[2][1] != 5 || m.nu_reac[2][1] != 1.0 || m.order_reac[2][1] != 1.0) return false;
    if (m.prod[2][0] != 1 || m.nu_prod[2][0] != 1.0) return false;
    if (m.prod[2][1] != 4 || m.nu_prod[2][1] != 1.0) return false;
    if (m.A[2] != 43800000000.00001 || m.b[2] != 0.0 || m.Ea[2] != 29246160.0) return false;
    if (m.rtype[3] != 1 || m.reversible[3] != 1 || m.n_reac[3] != 1 || m.n_prod[3] != 1) return false;
    if (m.reac[3][0] != 3 || m.nu_reac[3][0] != 2.0 || m.order_reac[3][0] != 2.0) return false;
    if (m.prod[3][0] != 2 || m.nu_prod[3][0] != 1.0) return false;
    if (m.A[3] != 6165000000.000002 || m.b[3] != -0.5 || m.Ea[3] != 0.0) return false;
    if (m.eff[3][0] != 2.5) return false;
    if (m.eff[3][1] != 1.0) return false;
    if (m.eff[3][2] != 1.0) return false;
    if (m.eff[3][3] != 1.0) return false;
    if (m.eff[3][4] != 12.0) return false;
    if (m.eff[3][5] != 1.0) return false;
    if (m.eff[3][6] != 1.0) return false;
    if (m.eff[3][7] != 1.0) return false;
    if (m.eff[3][8] != 1.0) return false;
    if (m.rtype[4] != 0 || m.reversible[4] != 1 || m.n_reac[4] != 2 || m.n_prod[4] != 2) return false;
    if (m.reac[4][0] != 2 || m.nu_reac[4][0] != 1.0 || m.order_reac[4][0] != 1.0) return false;
    if (m.reac[4][1] != 1 || m.nu_reac[4][1] != 1.0 || m.order_reac[4][1] != 1.0) return false;
    if (m.prod[4][0] != 3 || m.nu_prod[4][0] != 1.0) return false;
    if (m.prod[4][1] != 5 || m.nu_prod[4][1] != 1.0) return false;
    if (m.A[4] != 114000000000.00003 || m.b[4] != 0.0 || m.Ea[4] != 63956624.0) return false;
    if (m.rtype[5] != 1 || m.reversible[5] != 1 || m.n_reac[5] != 2 || m.n_prod[5] != 1) return false;
    if (m.reac[5][0] != 1 || m.nu_reac[5][0] != 1.0 || m.order_reac[5][0] != 1.0) return false;
    if (m.reac[5][1] != 5 || m.nu_reac[5][1] != 1.0 || m.order_reac[5][1] != 1.0) return false;
    if (m.prod[5][0] != 4 || m.nu_prod[5][0] != 1.0) return false;
    if (m.A[5] != 3.5000000000000016e+16 || m.b[5] != -2.0 || m.Ea[5] != 0.0) return false;
    if (m.eff[5][0] != 0.73) return false;
    if (m.eff[5][1] != 1.0) return false;
    if (m.eff[5][2] != 1.0) return false;
    if (m.eff[5][3] != 1.0) return false;
    if (m.eff[5][4] != 3.65) return false;
    if (m.eff[5][5] != 1.0) return false;
    if (m.eff[5][6] != 1.0) return false;
    if (m.eff[5][7] != 1.0) return false;
    if (m.eff[5][8] != 1.0) return false;
    if (m.rtype[6] != 0 || m.reversible[6] != 1 || m.n_reac[6] != 2 || m.n_prod[6] != 1) return false;
    if (m.reac[6][0] != 3 || m.nu_reac[6][0] != 1.0 || m.order_reac[6][0] != 1.0) return false;
    if (m.reac[6][1] != 4 || m.nu_reac[6][1] != 1.0 || m.order_reac[6][1] != 1.0) return false;
    if (m.prod[6][0] != 5 || m.nu_prod[6][0] != 2.0) return false;
    if (m.A[6] != 67000.00000000001 || m.b[6] != 1.704 || m.Ea[6] != 62704771.199999996) return false;
    if (m.rtype[7] != 1 || m.reversible[7] != 1 || m.n_reac[7] != 2 || m.n_prod[7] != 1) return false;
    if (m.reac[7][0] != 3 || m.nu_reac[7][0] != 1.0 || m.order_reac[7][0] != 1.0) return false;
    if (m.reac[7][1] != 1 || m.nu_reac[7][1] != 1.0 || m.order_reac[7][1] != 1.0) return false;
    if (m.prod[7][0] != 5 || m.nu_prod[7][0] != 1.0) return false;
    if (m.A[7] != 4714000000000.002 || m.b[7] != -1.0 || m.Ea[7] != 0.0) return false;
    if (m.eff[7][0] != 2.5) return false;
    if (m.eff[7][1] != 1.0) return false;
    if (m.eff[7][2] != 1.0) return false;
    if (m.eff[7][3] != 1.0) return false;
    if (m.eff[7][4] != 12.0) return false;
    if (m.eff[7][5] != 1.0) return false;
    if (m.eff[7][6] != 1.0) return false;
    if (m.eff[7][7] != 1.0) return false;
    if (m.eff[7][8] != 1.0) return false;
    if (m.rtype[8] != 2 || m.reversible[8] != 1 || m.n_reac[8] != 1 || m.n_prod[8] != 1) return false;
    if (m.reac[8][0] != 6 || m.nu_reac[8][0] != 1.0 || m.order_reac[8][0] != 1.0) return false;
    if (m.prod[8][0] != 5 || m.nu_prod[8][0] != 2.0) return false;
    if (m.A[8] != 2000000000000.0 || m.b[8] != 0.9 || m.Ea[8] != 203965816.0) return false;
    if (m.A0[8] != 2.4900000000000005e+21 || m.b0[8] != -2.3 || m.Ea0[8] != 203965816.0 || m.troe_n[8] != 3) return false;
    if (m.troe[8][0] != 0.43) return false;
    if (m.troe[8][1] != 1e-30) return false;
    if (m.troe[8][2] != 1e+30) return false;
    if (m.eff[8][0] != 3.7) return false;
    if (m.eff[8][1] != 1.0) return false;
    if (m.eff[8][2] != 1.2) return false;
    if (m.eff[8][3] != 1.0) return false;
    if (m.eff[8][4] != 7.65) return false;
    if (m.eff[8][5] != 1.0) return false;
    if (m.eff[8][6] != 7.7) return false;
    if (m.eff[8][7] != 1.0) return false;
    if (m.eff[8][8] != 1.5) return false;
    if (m.rtype[9] != 0 || m.reversible[9] != 1 || m.n_reac[9] != 2 || m.n_prod[9] != 2) return false;
    if (m.reac[9][0] != 6 || m.nu_reac[9][0] != 1.0 || m.order_reac[9][0] != 1.0) return false;
    if (m.reac[9][1] != 1 || m.nu_reac[9][1] != 1.0 || m.order_reac[9][1] != 1.0) return false;
    if (m.prod[9][0] != 4 || m.nu_prod[9][0] != 1.0) return false;
    if (m.prod[9][1] != 5 || m.nu_prod[9][1] != 1.0) return false;
    if (m.A[9] != 24100000000.000008 || m.b[9] != 0.0 || m.Ea[9] != 16610480.0) return false;
    if (m.rtype[10] != 0 || m.reversible[10] != 1 || m.n_reac[10] != 2 || m.n_prod[10] != 2) return false;
    if (m.reac[10][0] != 6 || m.nu_reac[10][0] != 1.0 || m.order_reac[10][0] != 1.0) return false;
    if (m.reac[10][1] != 1 || m.nu_reac[10][1] != 1.0 || m.order_reac[10][1] != 1.0) return false;
    if (m.prod[10][0] != 0 || m.nu_prod[10][0] != 1.0) return false;
    if (m.prod[10][1] != 7 || m.nu_prod[10][1] != 1.0) return false;
    if (m.A[10] != 21500000.000000004 || m.b[10] != 1.0 || m.Ea[10] != 25104000.0) return false;
    if (m.rtype[11] != 0 || m.reversible[11] != 1 || m.n_reac[11] != 2 || m.n_prod[11] != 2) return false;
    if (m.reac[11][0] != 6 || m.nu_reac[11][0] != 1.0 || m.order_reac[11][0] != 1.0) return false;
    if (m.reac[11][1] != 3 || m.nu_reac[11][1] != 1.0 || m.order_reac[11][1] != 1.0) return false;
    if (m.prod[11][0] != 5 || m.nu_prod[11][0] != 1.0) return false;
    if (m.prod[11][1] != 7 || m.nu_prod[11][1] != 1.0) return false;
    if (m.A[11] != 9550.000000000002 || m.b[11] != 2.0 || m.Ea[11] != 16610480.0) return false;
    if (m.rtype[12] != 0 || m.reversible[12] != 1 || m.n_reac[12] != 2 || m.n_prod[12] != 2) return false;
    if (m.reac[12][0] != 6 || m.nu_reac[12][0] != 1.0 || m.order_reac[12][0] != 1.0) return false;
    if (m.reac[12][1] != 5 || m.nu_reac[12][1] != 1.0 || m.order_reac[12][1] != 1.0) return false;
    if (m.prod[12][0] != 4 || m.nu_prod[12][0] != 1.0) return false;
    if (m.prod[12][1] != 7 || m.nu_prod[12][1] != 1.0) return false;
    if (m.A[12] != 1740000000.0000005 || m.b[12] != 0.0 || m.Ea[12] != 1330512.0) return false;
    if (m.rtype[13] != 0 || m.reversible[13] != 1 || m.n_reac[13] != 2 || m.n_prod[13] != 2) return false;
    if (m.reac[13][0] != 6 || m.nu_reac[13][0] != 1.0 || m.order_reac[13][0] != 1.0) return false;
    if (m.reac[13][1] != 5 || m.nu_reac[13][1] != 1.0 || m.order_reac[13][1] != 1.0) return false;
    if (m.prod[13][0] != 4 || m.nu_prod[13][0] != 1.0) return false;
    if (m.prod[13][1] != 7 || m.nu_prod[13][1] != 1.0) return false;
    if (m.A[13] != 75900000000.00002 || m.b[13] != 0.0 || m.Ea[13] != 30413496.0) return false;
    if (m.rtype[14] != 0 || m.reversible[14] != 1 || m.n_reac[14] != 2 || m.n_prod[14] != 1) return false;
    if (m.reac[14][0] != 7 || m.nu_reac[14][0] != 1.0 || m.order_reac[14][0] != 1.0) return false;
    if (m.reac[14][1] != 1 || m.nu_reac[14][1] != 1.0 || m.order_reac[14][1] != 1.0) return false;
    if (m.prod[14][0] != 5 || m.nu_prod[14][0] != 2.0) return false;
    if (m.A[14] != 70790000000.00002 || m.b[14] != 0.0 || m.Ea[14] != 1234280.0) return false;
    if (m.rtype[15] != 0 || m.reversible[15] != 1 || m.n_reac[15] != 2 || m.n_prod[15] != 2) return false;
    if (m.reac[15][0] != 7 || m.nu_reac[15][0] != 1.0 || m.order_reac[15][0] != 1.0) return false;
    if (m.reac[15][1] != 1 || m.nu_reac[15][1] != 1.0 || m.order_reac[15][1] != 1.0) return false;
    if (m.prod[15][0] != 0 || m.nu_prod[15][0] != 1.0) return false;
    if (m.prod[15][1] != 2 || m.nu_prod[15][1] != 1.0) return false;
    if (m.A[15] != 11402000.000000002 || m.b[15] != 1.0827 || m.Ea[15] != 2317015.52) return false;
    if (m.rtype[16] != 0 || m.reversible[16] != 1 || m.n_reac[16] != 2 || m.n_prod[16] != 2) return false;
    if (m.reac[16][0] != 7 || m.nu_reac[16][0] != 1.0 || m.order_reac[16][0] != 1.0) return false;
    if (m.reac[16][1] != 3 || m.nu_reac[16][1] != 1.0 || m.order_reac[16][1] != 1.0) return false;
    if (m.prod[16][0] != 5 || m.nu_prod[16][0] != 1.0) return false;
    if (m.prod[16][1] != 2 || m.nu_prod[16][1] != 1.0) return false;
    if (m.A[16] != 32500000000.000008 || m.b[16] != 0.0 || m.Ea[16] != 0.0) return false;
    if (m.rtype[17] != 0 || m.reversible[17] != 1 || m.n_reac[17] != 2 || m.n_prod[17] != 2) return false;
    if (m.reac[17][0] != 5 || m.nu_reac[17][0] != 1.0 || m.order_reac[17][0] != 1.0) return false;
    if (m.reac[17][1] != 7 || m.nu_reac[17][1] != 1.0 || m.order_reac[17][1] != 1.0) return false;
    if (m.prod[17][0] != 4 || m.nu_prod[17][0] != 1.0) return false;
    if (m.prod[17][1] != 2 || m.nu_prod[17][1] != 1.0) return false;
    if (m.A[17] != 7000000000.000002 || m.b[17] != 0.0 || m.Ea[17] != -4572944.640000001) return false;
    if (m.rtype[18] != 0 || m.reversible[18] != 1 || m.n_reac[18] != 2 || m.n_prod[18] != 2) return false;
    if (m.reac[18][0] != 5 || m.nu_reac[18][0] != 1.0 || m.order_reac[18][0] != 1.0) return false;
    if (m.reac[18][1] != 7 || m.nu_reac[18][1] != 1.0 || m.order_reac[18][1] != 1.0) return false;
    if (m.prod[18][0] != 4 || m.nu_prod[18][0] != 1.0) return false;
    if (m.prod[18][1] != 2 || m.nu_prod[18][1] != 1.0) return false;
    if (m.A[18] != 450000000000.0001 || m.b[18] != 0.0 || m.Ea[18] != 45729446.4) return false;
    if (m.rtype[19] != 0 || m.reversible[19] != 1 || m.n_reac[19] != 1 || m.n_prod[19] != 2) return false;
    if (m.reac[19][0] != 7 || m.nu_reac[19][0] != 2.0 || m.order_reac[19][0] != 2.0) return false;
    if (m.prod[19][0] != 6 || m.nu_prod[19][0] != 1.0) return false;
    if (m.prod[19][1] != 2 || m.nu_prod[19][1] != 1.0) return false;
    if (m.A[19] != 100000000000.00003 || m.b[19] != 0.0 || m.Ea[19] != 46195054.472) return false;
    if (m.rtype[20] != 0 || m.reversible[20] != 1 || m.n_reac[20] != 1 || m.n_prod[20] != 2) return false;
    if (m.reac[20][0] != 7 || m.nu_reac[20][0] != 2.0 || m.order_reac[20][0] != 2.0) return false;
    if (m.prod[20][0] != 6 || m.nu_prod[20][0] != 1.0) return false;
    if (m.prod[20][1] != 2 || m.nu_prod[20][1] != 1.0) return false;
    if (m.A[20] != 190000000.00000006 || m.b[20] != 0.0 || m.Ea[20] != -5894941.3632) return false;
    if (m.rtype[21] != 2 || m.reversible[21] != 1 || m.n_reac[21] != 2 || m.n_prod[21] != 1) return false;
    if (m.reac[21][0] != 1 || m.nu_reac[21][0] != 1.0 || m.order_reac[21][0] != 1.0) return false;
    if (m.reac[21][1] != 2 || m.nu_reac[21][1] != 1.0 || m.order_reac[21][1] != 1.0) return false;
    if (m.prod[21][0] != 7 || m.nu_prod[21][0] != 1.0) return false;
    if (m.A[21] != 4650000000.000001 || m.b[21] != 0.44 || m.Ea[21] != 0.0) return false;
    if (m.A0[21] != 17370000000000.006 || m.b0[21] != -1.23 || m.Ea0[21] != 0.0 || m.troe_n[21] != 4) return false;
    if (m.troe[21][0] != 0.67) return false;
    if (m.troe[21][1] != 1e-30) return false;
    if (m.troe[21][2] != 1e+30) return false;
    if (m.troe[21][3] != 1e+30) return false;
    if (m.eff[21][0] != 1.3) return false;
    if (m.eff[21][1] != 1.0) return false;
    if (m.eff[21][2] != 1.0) return false;
    if (m.eff[21][3] != 1.0) return false;
    if (m.eff[21][4] != 10.0) return false;
    if (m.eff[21][5] != 1.0) return false;
    if (m.eff[21][6] != 1.0) return false;
    if (m.eff[21][7] != 1.0) return false;
    if (m.eff[21][8] != 1.0) return false;
    if (m.rtype[22] != 1 || m.reversible[22] != 1 || m.n_reac[22] != 2 || m.n_prod[22] != 1) return false;
    if (m.reac[22][0] != 3 || m.nu_reac[22][0] != 1.0 || m.order_reac[22][0] != 1.0) return false;
    if (m.reac[22][1] != 5 || m.nu_reac[22][1] != 1.0 || m.order_reac[22][1] != 1.0) return false;
    if (m.prod[22][0] != 7 || m.nu_prod[22][0] != 1.0) return false;
    if (m.A[22] != 10000000000.000004 || m.b[22] != 0.0 || m.Ea[22] != 0.0) return false;
    if (m.eff[22][0] != 1.0) return false;
    if (m.eff[22][1] != 1.0) return false;
    if (m.eff[22][2] != 1.0) return false;
    if (m.eff[22][3] != 1.0) return false;
    if (m.eff[22][4] != 1.0) return false;
    if (m.eff[22][5] != 1.0) return false;
    if (m.eff[22][6] != 1.0) return false;
    if (m.eff[22][7] != 1.0) return false;
    if (m.eff[22][8] != 1.0) return false;
    return true;
}

// The species' thermo at one temperature (NASA-7): h/RT, g/RT and c_p/R, with ln T, 1/RT and
// ln(p_atm / R T); the rate constants are formed from them reaction by reaction where they
// are used (rhs_t, rhs_jac), so that no per-reaction array stays live across the kinetics.
struct Thermo {
    double hRT[NS], gRT[NS], cpR[NS], logT, invRT, log_cref;
};

GAS_HD void thermo(double T, Thermo &th) {
    const double logT = log(T);
    th.logT = logT;
    th.invRT = 1.0 / (8314.46261815324 * T);
    th.log_cref = log(101325.0 / (8314.46261815324 * T));
    if (T < 1000.0) {
        th.cpR[0] = 2.37694204 + T * (0.00773916922 + T * (-1.88735073e-05 + T * (1.95517114e-08 + T * -7.17095663e-12)));
        th.hRT[0] = 2.37694204 + T * (0.00386958461 + T * (-6.291169099999999e-06 + T * (4.88792785e-09 + T * -7.17095663e-12 / 5.0))) + -921.173081 / T;
        th.gRT[0] = th.hRT[0] - (2.37694204 * logT + T * (0.00773916922 + T * (-9.43675365e-06 + T * (6.517237133333333e-09 + T * -1.7927391575e-12))) + 0.547184736);
        th.cpR[1] = 2.49975925 + T * (6.73824499e-07 + T * (1.11807261e-09 + T * (-3.70192126e-12 + T * 2.14233822e-15)));
        th.hRT[1] = 2.49975925 + T * (3.369122495e-07 + T * (3.7269087000000003e-10 + T * (-9.25480315e-13 + T * 2.14233822e-15 / 5.0))) + 25473.7665 / T;
        th.gRT[1] = th.hRT[1] - (2.49975925 * logT + T * (6.73824499e-07 + T * (5.59036305e-10 + T * (-1.2339737533333333e-12 + T * 5.35584555e-16))) + -0.445574009);
        th.cpR[2] = 3.78498258 + T * (-0.00302002233 + T * (9.92029171e-06 + T * (-9.77840434e-09 + T * 3.28877702e-12)));
        th.hRT[2] = 3.78498258 + T * (-0.001510011165 + T * (3.3067639033333336e-06 + T * (-2.444601085e-09 + T * 3.28877702e-12 / 5.0))) + -1064.13589 / T;
        th.gRT[2] = th.hRT[2] - (3.78498258 * logT + T * (-0.00302002233 + T * (4.960145855e-06 + T * (-3.2594681133333337e-09 + T * 8.22194255e-13))) + 3.64780709);
        th.cpR[3] = 3.15906526 + T * (-0.00321509999 + T * (6.49255543e-06 + T * (-5.98755115e-09 + T * 2.06876117e-12)));
        th.hRT[3] = 3.15906526 + T * (-0.001607549995 + T * (2.1641851433333333e-06 + T * (-1.4968877875e-09 + T * 2.06876117e-12 / 5.0))) + 29129.8453 / T;
        th.gRT[3] = th.hRT[3] - (3.15906526 * logT + T * (-0.00321509999 + T * (3.246277715e-06 + T * (-1.995850383333333e-09 + T * 5.171902925e-13))) + 2.09078344);
        th.cpR[4] = 4.20147551 + T * (-0.00205583546 + T * (6.56547207e-06 + T * (-5.5290696e-09 + T * 1.78282605e-12)));
        th.hRT[4] = 4.20147551 + T * (-0.00102791773 + T * (2.1884906899999998e-06 + T * (-1.3822674e-09 + T * 1.78282605e-12 / 5.0))) + -30295.0066 / T;
        th.gRT[4] = th.hRT[4] - (4.20147551 * logT + T * (-0.00205583546 + T * (3.282736035e-06 + T * (-1.8430232e-09 + T * 4.457065125e-13))) + -0.860610906);
        th.cpR[5] = 3.97585165 + T * (-0.00228555291 + T * (4.33442882e-06 + T * (-3.5992664e-09 + T * 1.2670693e-12)));
        th.hRT[5] = 3.97585165 + T * (-0.001142776455 + T * (1.4448096066666668e-06 + T * (-8.998166e-10 + T * 1.2670693e-12 / 5.0))) + 3393.41137 / T;
        th.gRT[5] = th.hRT[5] - (3.97585165 * logT + T * (-0.00228555291 + T * (2.16721441e-06 + T * (-1.1997554666666665e-09 + T * 3.16767325e-13))) + -0.0355397262);
        th.cpR[6] = 4.2385416 + T * (-0.000249610911 + T * (1.59857901e-05 + T * (-2.06919945e-08 + T * 8.2976632e-12)));
        th.hRT[6] = 4.2385416 + T * (-0.0001248054555 + T * (5.3285966999999996e-06 + T * (-5.172998625e-09 + T * 8.2976632e-12 / 5.0))) + -17648.6003 / T;
        th.gRT[6] = th.hRT[6] - (4.2385416 * logT + T * (-0.000249610911 + T * (7.99289505e-06 + T * (-6.8973315e-09 + T * 2.0744158e-12))) + 3.58850097);
        th.cpR[7] = 4.2625125 + T * (-0.00445642032 + T * (2.05164934e-05 + T * (-2.35794011e-08 + T * 9.05614257e-12)));
        th.hRT[7] = 4.2625125 + T * (-0.00222821016 + T * (6.8388311333333335e-06 + T * (-5.894850275e-09 + T * 9.05614257e-12 / 5.0))) + 262.442356 / T;
        th.gRT[7] = th.hRT[7] - (4.2625125 * logT + T * (-0.00445642032 + T * (1.02582467e-05 + T * (-7.859800366666666e-09 + T * 2.2640356425e-12))) + 3.88223684);
        th.cpR[8] = 3.53603521 + T * (-0.000158270944 + T * (-4.26984251e-07 + T * (2.3754259e-09 + T * -1.39708206e-12)));
        th.hRT[8] = 3.53603521 + T * (-7.9135472e-05 + T * (-1.4232808366666666e-07 + T * (5.93856475e-10 + T * -1.39708206e-12 / 5.0))) + -1047.49645 / T;
        th.gRT[8] = th.hRT[8] - (3.53603521 * logT + T * (-0.000158270944 + T * (-2.134921255e-07 + T * (7.918086333333333e-10 + T * -3.49270515e-13))) + 2.94603724);
    } else {
        th.cpR[0] = 2.90207649 + T * (0.000868992581 + T * (-1.6586443e-07 + T * (1.90851899e-11 + T * -9.31121789e-16)));
        th.hRT[0] = 2.90207649 + T * (0.0004344962905 + T * (-5.5288143333333333e-08 + T * (4.771297475e-12 + T * -9.31121789e-16 / 5.0))) + -797.948726 / T;
        th.gRT[0] = th.hRT[0] - (2.90207649 * logT + T * (0.000868992581 + T * (-8.2932215e-08 + T * (6.361729966666667e-12 + T * -2.3278044725e-16))) + -0.84559132);
        th.cpR[1] = 2.49985211 + T * (2.34582548e-07 + T * (-1.16171641e-10 + T * (2.25708298e-14 + T * -1.52992005e-18)));
        th.hRT[1] = 2.49985211 + T * (1.17291274e-07 + T * (-3.8723880333333334e-11 + T * (5.64270745e-15 + T * -1.52992005e-18 / 5.0))) + 25473.8024 / T;
        th.gRT[1] = th.hRT[1] - (2.49985211 * logT + T * (2.34582548e-07 + T * (-5.80858205e-11 + T * (7.523609933333334e-15 + T * -3.824800125e-19))) + -0.445864645);
        th.cpR[2] = 3.65980488 + T * (0.000659877372 + T * (-1.44158172e-07 + T * (2.14656037e-11 + T * -1.36503784e-15)));
        th.hRT[2] = 3.65980488 + T * (0.000329938686 + T * (-4.8052724e-08 + T * (5.366400925e-12 + T * -1.36503784e-15 / 5.0))) + -1216.03048 / T;
        th.gRT[2] = th.hRT[2] - (3.65980488 * logT + T * (0.000659877372 + T * (-7.2079086e-08 + T * (7.155201233333333e-12 + T * -3.4125946e-16))) + 3.42074148);
        th.cpR[3] = 2.55160087 + T * (-3.83085457e-05 + T * (8.43197478e-10 + T * (4.01267136e-12 + T * -4.17476574e-16)));
        th.hRT[3] = 2.55160087 + T * (-1.915427285e-05 + T * (2.81065826e-10 + T * (1.00316784e-12 + T * -4.17476574e-16 / 5.0))) + 29228.7628 / T;
        th.gRT[3] = th.hRT[3] - (2.55160087 * logT + T * (-3.83085457e-05 + T * (4.21598739e-10 + T * (1.33755712e-12 + T * -1.043691435e-16))) + 4.87617014);
        th.cpR[4] = 2.73117512 + T * (0.00295136995 + T * (-8.35359785e-07 + T * (1.26088593e-10 + T * -8.40531676e-15)));
        th.hRT[4] = 2.73117512 + T * (0.001475684975 + T * (-2.784532616666667e-07 + T * (3.152214825e-11 + T * -8.40531676e-15 / 5.0))) + -29916.9082 / T;
        th.gRT[4] = th.hRT[4] - (2.73117512 * logT + T * (0.00295136995 + T * (-4.176798925e-07 + T * (4.2029531e-11 + T * -2.10132919e-15))) + 6.55183);
        th.cpR[5] = 2.84581721 + T * (0.00109723818 + T * (-2.89121101e-07 + T * (4.0909991e-11 + T * -2.31382258e-15)));
        th.hRT[5] = 2.84581721 + T * (0.00054861909 + T * (-9.637370033333334e-08 + T * (1.022749775e-11 + T * -2.31382258e-15 / 5.0))) + 3717.0661 / T;
        th.gRT[5] = th.hRT[5] - (2.84581721 * logT + T * (0.00109723818 + T * (-1.445605505e-07 + T * (1.3636663666666666e-11 + T * -5.78455645e-16))) + 5.80339915);
        th.cpR[6] = 4.5401748 + T * (0.00415970971 + T * (-1.30876777e-06 + T * (2.00823615e-10 + T * -1.15509243e-14)));
        th.hRT[6] = 4.5401748 + T * (0.002079854855 + T * (-4.3625592333333335e-07 + T * (5.020590375e-11 + T * -1.15509243e-14 / 5.0))) + -17951.4029 / T;
        th.gRT[6] = th.hRT[6] - (4.5401748 * logT + T * (0.00415970971 + T * (-6.54383885e-07 + T * (6.694120500000001e-11 + T * -2.887731075e-15))) + 0.855881745);
        th.cpR[7] = 4.1056401 + T * (0.00204046836 + T * (-3.65877562e-07 + T * (1.85973044e-11 + T * 4.98818315e-16)));
        th.hRT[7] = 4.1056401 + T * (0.00102023418 + T * (-1.2195918733333333e-07 + T * (4.6493261e-12 + T * 4.98818315e-16 / 5.0))) + 43.2898769 / T;
        th.gRT[7] = th.hRT[7] - (4.1056401 * logT + T * (0.00204046836 + T * (-1.82938781e-07 + T * (6.199101466666667e-12 + T * 1.2470457875e-16))) + 3.30808126);
        th.cpR[8] = 2.9380297 + T * (0.0014183803 + T * (-5.03281045e-07 + T * (8.07555464e-11 + T * -4.76064275e-15)));
        th.hRT[8] = 2.9380297 + T * (0.00070919015 + T * (-1.6776034833333333e-07 + T * (2.01888866e-11 + T * -4.76064275e-15 / 5.0))) + -917.18099 / T;
        th.gRT[8] = th.hRT[8] - (2.9380297 * logT + T * (0.0014183803 + T * (-2.516405225e-07 + T * (2.6918515466666668e-11 + T * -1.1901606875e-15))) + 5.95521985);
    }
}

// F = d(Y_0..Y_{NS-1}, T)/dt at density rho [kg/m^3] and state y, from the thermo th at
// y's temperature (gas::rate_factors + gas::reactor_rhs_k, reaction by reaction).
GAS_HD void rhs_t(const Thermo &th, double rho, const double *y, double *F) {
    const double T = y[9];
    const double logT = th.logT, invRT = th.invRT, log_cref = th.log_cref;
    (void)logT;
    (void)log_cref;
    const double C0 = rho * y[0] * 0.49603174603174605;
    const double C1 = rho * y[1] * 0.9920634920634921;
    const double C2 = rho * y[2] * 0.03125195324707794;
    const double C3 = rho * y[3] * 0.06250390649415588;
    const double C4 = rho * y[4] * 0.055509297807382736;
    const double C5 = rho * y[5] * 0.05879931792791203;
    const double C6 = rho * y[6] * 0.029399658963956014;
    const double C7 = rho * y[7] * 0.030297521662727988;
    const double C8 = rho * y[8] * 0.03569643749553795;
    double w0 = 0.0;
    double w1 = 0.0;
    double w2 = 0.0;
    double w3 = 0.0;
    double w4 = 0.0;
    double w5 = 0.0;
    double w6 = 0.0;
    double w7 = 0.0;
    double w8 = 0.0;
    double cv = 0.0;
    cv += y[0] * (th.cpR[0] - 1.0) * 0.49603174603174605;
    cv += y[1] * (th.cpR[1] - 1.0) * 0.9920634920634921;
    cv += y[2] * (th.cpR[2] - 1.0) * 0.03125195324707794;
    cv += y[3] * (th.cpR[3] - 1.0) * 0.06250390649415588;
    cv += y[4] * (th.cpR[4] - 1.0) * 0.055509297807382736;
    cv += y[5] * (th.cpR[5] - 1.0) * 0.05879931792791203;
    cv += y[6] * (th.cpR[6] - 1.0) * 0.029399658963956014;
    cv += y[7] * (th.cpR[7] - 1.0) * 0.030297521662727988;
    cv += y[8] * (th.cpR[8] - 1.0) * 0.03569643749553795;
    cv *= 8314.46261815324;
    GAS_SCHED_FENCE();
    {  // reaction 0
        const double kf = 4.577000000000001e+16 * exp(-1.4 * logT - 436809600.0 * invRT);
        const double er = exp((2.0 * th.gRT[1] - th.gRT[0]) - 1.0 * log_cref);
        {  // rate of progress: 1 H2 <=> 2 H  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C0;
            const double rev = kfM * er * (C1 * C1);
            const double q = fwd - rev;
            w0 -= q;
            w1 += 2.0 * q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 1
        const double kf = 50.80000000000001 * exp(2.67 * logT - 26325728.0 * invRT);
        const double er = exp(th.gRT[1] + th.gRT[5] - th.gRT[0] - th.gRT[3]);
        {  // rate of progress: 1 H2 + 1 O <=> 1 H + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C0 * C3;
            const double rev = kfM * er * C1 * C5;
            const double q = fwd - rev;
            w0 -= q;
            w3 -= q;
            w1 += q;
            w5 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 2
        const double kf = 43800000000.00001 * exp(-(29246160.0 * invRT));
        const double er = exp(th.gRT[1] + th.gRT[4] - th.gRT[0] - th.gRT[5]);
        {  // rate of progress: 1 H2 + 1 OH <=> 1 H + 1 H2O
            const double kfM = kf;
            const double fwd = kfM * C0 * C5;
            const double rev = kfM * er * C1 * C4;
            const double q = fwd - rev;
            w0 -= q;
            w5 -= q;
            w1 += q;
            w4 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 3
        const double kf = 6165000000.000002 * exp(-0.5 * logT);
        const double er = exp((th.gRT[2] - 2.0 * th.gRT[3]) - -1.0 * log_cref);
        {  // rate of progress: 2 O <=> 1 O2  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * (C3 * C3);
            const double rev = kfM * er * C2;
            const double q = fwd - rev;
            w3 -= 2.0 * q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 4
        const double kf = 114000000000.00003 * exp(-(63956624.0 * invRT));
        const double er = exp(th.gRT[3] + th.gRT[5] - th.gRT[2] - th.gRT[1]);
        {  // rate of progress: 1 O2 + 1 H <=> 1 O + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C2 * C1;
            const double rev = kfM * er * C3 * C5;
            const double q = fwd - rev;
            w2 -= q;
            w1 -= q;
            w3 += q;
            w5 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 5
        const double kf = 3.5000000000000016e+16 * exp(-2.0 * logT);
        const double er = exp((th.gRT[4] - th.gRT[1] - th.gRT[5]) - -1.0 * log_cref);
        {  // rate of progress: 1 H + 1 OH <=> 1 H2O  + M
            const double M = 0.73 * C0 + C1 + C2 + C3 + 3.65 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C1 * C5;
            const double rev = kfM * er * C4;
            const double q = fwd - rev;
            w1 -= q;
            w5 -= q;
            w4 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 6
        const double kf = 67000.00000000001 * exp(1.704 * logT - 62704771.199999996 * invRT);
        const double er = exp(2.0 * th.gRT[5] - th.gRT[3] - th.gRT[4]);
        {  // rate of progress: 1 O + 1 H2O <=> 2 OH
            const double kfM = kf;
            const double fwd = kfM * C3 * C4;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w3 -= q;
            w4 -= q;
            w5 += 2.0 * q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 7
        const double kf = 4714000000000.002 * exp(-1.0 * logT);
        const double er = exp((th.gRT[5] - th.gRT[3] - th.gRT[1]) - -1.0 * log_cref);
        {  // rate of progress: 1 O + 1 H <=> 1 OH  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C3 * C1;
            const double rev = kfM * er * C5;
            const double q = fwd - rev;
            w3 -= q;
            w1 -= q;
            w5 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 8
        const double kf = 2000000000000.0 * exp(0.9 * logT - 203965816.0 * invRT);
        const double k0 = 2.4900000000000005e+21 * exp(-2.3 * logT - 203965816.0 * invRT);
        const double lFc0 = -0.36653154442041347;
        const double er = exp((2.0 * th.gRT[5] - th.gRT[6]) - 1.0 * log_cref);
        {  // rate of progress: 1 H2O2 <=> 2 OH  (+M)
            const double M = 3.7 * C0 + C1 + 1.2 * C2 + C3 + 7.65 * C4 + C5 + 7.7 * C6 + C7 + 1.5 * C8;
            const double Pr = k0 * M / kf;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double x = (lPr + c) / (n - 0.14 * (lPr + c));
            const double kfM = kf * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
            const double fwd = kfM * C6;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w6 -= q;
            w5 += 2.0 * q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 9
        const double kf = 24100000000.000008 * exp(-(16610480.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[5] - th.gRT[6] - th.gRT[1]);
        {  // rate of progress: 1 H2O2 + 1 H <=> 1 H2O + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C6 * C1;
            const double rev = kfM * er * C4 * C5;
            const double q = fwd - rev;
            w6 -= q;
            w1 -= q;
            w4 += q;
            w5 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 10
        const double kf = 21500000.000000004 * exp(1.0 * logT - 25104000.0 * invRT);
        const double er = exp(th.gRT[0] + th.gRT[7] - th.gRT[6] - th.gRT[1]);
        {  // rate of progress: 1 H2O2 + 1 H <=> 1 H2 + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C1;
            const double rev = kfM * er * C0 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w1 -= q;
            w0 += q;
            w7 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 11
        const double kf = 9550.000000000002 * exp(2.0 * logT - 16610480.0 * invRT);
        const double er = exp(th.gRT[5] + th.gRT[7] - th.gRT[6] - th.gRT[3]);
        {  // rate of progress: 1 H2O2 + 1 O <=> 1 OH + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C3;
            const double rev = kfM * er * C5 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w3 -= q;
            w5 += q;
            w7 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 12
        const double kf = 1740000000.0000005 * exp(-(1330512.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[7] - th.gRT[6] - th.gRT[5]);
        {  // rate of progress: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C5;
            const double rev = kfM * er * C4 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w5 -= q;
            w4 += q;
            w7 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 13
        const double kf = 75900000000.00002 * exp(-(30413496.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[7] - th.gRT[6] - th.gRT[5]);
        {  // rate of progress: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C5;
            const double rev = kfM * er * C4 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w5 -= q;
            w4 += q;
            w7 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 14
        const double kf = 70790000000.00002 * exp(-(1234280.0 * invRT));
        const double er = exp(2.0 * th.gRT[5] - th.gRT[7] - th.gRT[1]);
        {  // rate of progress: 1 HO2 + 1 H <=> 2 OH
            const double kfM = kf;
            const double fwd = kfM * C7 * C1;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w7 -= q;
            w1 -= q;
            w5 += 2.0 * q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 15
        const double kf = 11402000.000000002 * exp(1.0827 * logT - 2317015.52 * invRT);
        const double er = exp(th.gRT[0] + th.gRT[2] - th.gRT[7] - th.gRT[1]);
        {  // rate of progress: 1 HO2 + 1 H <=> 1 H2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C7 * C1;
            const double rev = kfM * er * C0 * C2;
            const double q = fwd - rev;
            w7 -= q;
            w1 -= q;
            w0 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 16
        const double kf = 32500000000.000008;
        const double er = exp(th.gRT[5] + th.gRT[2] - th.gRT[7] - th.gRT[3]);
        {  // rate of progress: 1 HO2 + 1 O <=> 1 OH + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C7 * C3;
            const double rev = kfM * er * C5 * C2;
            const double q = fwd - rev;
            w7 -= q;
            w3 -= q;
            w5 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 17
        const double kf = 7000000000.000002 * exp(-(-4572944.640000001 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[2] - th.gRT[5] - th.gRT[7]);
        {  // rate of progress: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C5 * C7;
            const double rev = kfM * er * C4 * C2;
            const double q = fwd - rev;
            w5 -= q;
            w7 -= q;
            w4 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 18
        const double kf = 450000000000.0001 * exp(-(45729446.4 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[2] - th.gRT[5] - th.gRT[7]);
        {  // rate of progress: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C5 * C7;
            const double rev = kfM * er * C4 * C2;
            const double q = fwd - rev;
            w5 -= q;
            w7 -= q;
            w4 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 19
        const double kf = 100000000000.00003 * exp(-(46195054.472 * invRT));
        const double er = exp(th.gRT[6] + th.gRT[2] - 2.0 * th.gRT[7]);
        {  // rate of progress: 2 HO2 <=> 1 H2O2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * (C7 * C7);
            const double rev = kfM * er * C6 * C2;
            const double q = fwd - rev;
            w7 -= 2.0 * q;
            w6 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 20
        const double kf = 190000000.00000006 * exp(-(-5894941.3632 * invRT));
        const double er = exp(th.gRT[6] + th.gRT[2] - 2.0 * th.gRT[7]);
        {  // rate of progress: 2 HO2 <=> 1 H2O2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * (C7 * C7);
            const double rev = kfM * er * C6 * C2;
            const double q = fwd - rev;
            w7 -= 2.0 * q;
            w6 += q;
            w2 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 21
        const double kf = 4650000000.000001 * exp(0.44 * logT);
        const double k0 = 17370000000000.006 * exp(-1.23 * logT);
        const double lFc0 = -0.17392519729917352;
        const double er = exp((th.gRT[7] - th.gRT[1] - th.gRT[2]) - -1.0 * log_cref);
        {  // rate of progress: 1 H + 1 O2 <=> 1 HO2  (+M)
            const double M = 1.3 * C0 + C1 + C2 + C3 + 10.0 * C4 + C5 + C6 + C7 + C8;
            const double Pr = k0 * M / kf;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double x = (lPr + c) / (n - 0.14 * (lPr + c));
            const double kfM = kf * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
            const double fwd = kfM * C1 * C2;
            const double rev = kfM * er * C7;
            const double q = fwd - rev;
            w1 -= q;
            w2 -= q;
            w7 += q;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 22
        const double kf = 10000000000.000004;
        const double er = exp((th.gRT[7] - th.gRT[3] - th.gRT[5]) - -1.0 * log_cref);
        {  // rate of progress: 1 O + 1 OH <=> 1 HO2  + M
            const double M = C0 + C1 + C2 + C3 + C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C3 * C5;
            const double rev = kfM * er * C7;
            const double q = fwd - rev;
            w3 -= q;
            w5 -= q;
            w7 += q;
        }
    }
    double es = 0.0;
    F[0] = w0 * 2.016 / rho;
    es += (th.hRT[0] - 1.0) * 8314.46261815324 * T * w0;
    F[1] = w1 * 1.008 / rho;
    es += (th.hRT[1] - 1.0) * 8314.46261815324 * T * w1;
    F[2] = w2 * 31.998 / rho;
    es += (th.hRT[2] - 1.0) * 8314.46261815324 * T * w2;
    F[3] = w3 * 15.999 / rho;
    es += (th.hRT[3] - 1.0) * 8314.46261815324 * T * w3;
    F[4] = w4 * 18.015 / rho;
    es += (th.hRT[4] - 1.0) * 8314.46261815324 * T * w4;
    F[5] = w5 * 17.007 / rho;
    es += (th.hRT[5] - 1.0) * 8314.46261815324 * T * w5;
    F[6] = w6 * 34.014 / rho;
    es += (th.hRT[6] - 1.0) * 8314.46261815324 * T * w6;
    F[7] = w7 * 33.006 / rho;
    es += (th.hRT[7] - 1.0) * 8314.46261815324 * T * w7;
    F[8] = w8 * 28.014 / rho;
    es += (th.hRT[8] - 1.0) * 8314.46261815324 * T * w8;
    F[9] = -es / (rho * cv);
}

// rhs_t, and s times the Jacobian of F with respect to (Y, T) at fixed density over the
// unknowns of the integrator's iteration system (Kinetics::sys_full): J(p, q) = s dF_a / dY_b,
// a = sys_full(p), b = sys_full(q), the temperature the last unknown.
// The inert species (N2) are not unknowns: their row is zero
// and their column multiplies a zero increment.
// Each reaction's rate constants are formed once and serve both.
// The Jacobian of d(Y, T)/dt at fixed density, d F_k / d Y_j and d F_k / dT, differentiating the
// right-hand side's expressions.  With q_r the rates of progress, nu_kr the net coefficients and
// C_j = rho Y_j / W_j:
//     dF_k/dY_j = (W_k / W_j) sum_r nu_kr dq_r/dC_j,
//     dF_k/dT   = (W_k / rho) sum_r nu_kr dq_r/dT,
//     dF_T/dY_j = -(R T / (W_j c_v)) sum_r e_r dq_r/dC_j - F_T R (c_p,j/R - 1) / (W_j c_v),
//     dF_T/dT   = -R [sum_k (c_p,k/R - 1) w_k + T sum_r e_r dq_r/dT] / (rho c_v) - F_T (dc_v/dT) / c_v,
// e_r = sum_k nu_kr (h_k/RT - 1), w_k the net production rates.  dq_r/dC_j through the
// mass-action products, the third-body sum M and the Troe blend F(Pr), Pr = k0 M / k_inf:
// d(k_inf Pr/(1+Pr) F)/dM = k0 F/(1+Pr) [1/(1+Pr) - 2 x lFc n / ((1+x^2)^2 (n - 0.14 u)^2)],
// u = log10 Pr + c, x = u / (n - 0.14 u).  dq_r/dT through d ln k/dT = (b + E_a/RT)/T for
// k_f and k_0, d ln(1/K_c)/dT = (dnu - sum_k nu_kr h_k/RT)/T (d(g_k/RT)/dT = -h_k/(R T^2),
// d ln(p_atm/RT)/dT = -1/T), and for a fall-off reaction d ln(Pr/(1+Pr))/dT =
// (d ln k0 - d ln k_inf)/(1+Pr) and d ln F/dT = ln 10 [dlFc/(1+x^2) - 2 x lFc dx/(1+x^2)^2]
// with du = (d ln k0 - d ln k_inf)/ln 10 - 0.67 dlFc (dlFc = 0 where F_cent is constant).
// Every term is accumulated straight into the scaled matrix (s J, s = -gamma h for the
// integrator's iteration matrix).
template <class Mat>
GAS_HD void rhs_jac(const Thermo &th, double rho, const double *y, double *F, double s, Mat &J) {
    const double T = y[9];
    const double logT = th.logT, invRT = th.invRT, log_cref = th.log_cref;
    (void)logT;
    (void)log_cref;
    const double C0 = rho * y[0] * 0.49603174603174605;
    const double C1 = rho * y[1] * 0.9920634920634921;
    const double C2 = rho * y[2] * 0.03125195324707794;
    const double C3 = rho * y[3] * 0.06250390649415588;
    const double C4 = rho * y[4] * 0.055509297807382736;
    const double C5 = rho * y[5] * 0.05879931792791203;
    const double C6 = rho * y[6] * 0.029399658963956014;
    const double C7 = rho * y[7] * 0.030297521662727988;
    const double C8 = rho * y[8] * 0.03569643749553795;
    double w0 = 0.0;
    double w1 = 0.0;
    double w2 = 0.0;
    double w3 = 0.0;
    double w4 = 0.0;
    double w5 = 0.0;
    double w6 = 0.0;
    double w7 = 0.0;
    double w8 = 0.0;
    double cv = 0.0;
    cv += y[0] * (th.cpR[0] - 1.0) * 0.49603174603174605;
    cv += y[1] * (th.cpR[1] - 1.0) * 0.9920634920634921;
    cv += y[2] * (th.cpR[2] - 1.0) * 0.03125195324707794;
    cv += y[3] * (th.cpR[3] - 1.0) * 0.06250390649415588;
    cv += y[4] * (th.cpR[4] - 1.0) * 0.055509297807382736;
    cv += y[5] * (th.cpR[5] - 1.0) * 0.05879931792791203;
    cv += y[6] * (th.cpR[6] - 1.0) * 0.029399658963956014;
    cv += y[7] * (th.cpR[7] - 1.0) * 0.030297521662727988;
    cv += y[8] * (th.cpR[8] - 1.0) * 0.03569643749553795;
    cv *= 8314.46261815324;
    const double invT = 1.0 / T;
    const double sT = -s * 8314.46261815324 * T / cv;  // times e_r dq_rj / W_j: the T row
    const double s_rho = s / rho;
    double sum_eT = 0.0;  // sum_r e_r dq_r/dT
    // the temperature row (jT) and column (jc), summed in registers and stored once
    double jT0 = 0.0, jT1 = 0.0, jT2 = 0.0, jT3 = 0.0, jT4 = 0.0, jT5 = 0.0, jT6 = 0.0, jT7 = 0.0;
    double jc0 = 0.0, jc1 = 0.0, jc2 = 0.0, jc3 = 0.0, jc4 = 0.0, jc5 = 0.0, jc6 = 0.0, jc7 = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int j = 0; j < 9; ++j) J(k, j) = 0.0;
    GAS_SCHED_FENCE();
    {  // reaction 0
        const double kf = 4.577000000000001e+16 * exp(-1.4 * logT - 436809600.0 * invRT);
        const double er = exp((2.0 * th.gRT[1] - th.gRT[0]) - 1.0 * log_cref);
        {  // rate of progress: 1 H2 <=> 2 H  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C0;
            const double rev = kfM * er * (C1 * C1);
            const double q = fwd - rev;
            w0 -= q;
            w1 += 2.0 * q;
        }
        {  // Jacobian terms
            const double pf = C0;
            const double pb = (C1 * C1);
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double dkdM = kf;
            const double dlnk = (-1.4 + 436809600.0 * invRT) * invT;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (1.0 - (2.0 * th.hRT[1] - (1.0 * th.hRT[0]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = kfM * (1.0) + 2.5 * g;
            const double dq1 = -kfM * er * (2.0 * C1) + g;
            const double dq2 = g;
            const double dq3 = g;
            const double dq4 = 12.0 * g;
            const double dq5 = g;
            const double dq6 = g;
            const double dq7 = g;
            const double e_r = -1.0 * (th.hRT[0] - 1.0) + 2.0 * (th.hRT[1] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(0, 0) += -1.0 * s * dq0;
            J(1, 0) += 1.0 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(0, 1) += -2.0 * s * dq1;
            J(1, 1) += 2.0 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(0, 2) += -0.06300393774610913 * s * dq2;
            J(1, 2) += 0.06300393774610913 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(0, 3) += -0.12600787549221826 * s * dq3;
            J(1, 3) += 0.12600787549221826 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(0, 4) += -0.11190674437968359 * s * dq4;
            J(1, 4) += 0.11190674437968359 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(0, 5) += -0.11853942494267065 * s * dq5;
            J(1, 5) += 0.11853942494267065 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(0, 6) += -0.05926971247133533 * s * dq6;
            J(1, 6) += 0.05926971247133533 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(0, 7) += -0.061079803672059625 * s * dq7;
            J(1, 7) += 0.061079803672059625 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc0 += -2.016 * s_rho * dqT;
            jc1 += 2.016 * s_rho * dqT;
        }
    }
    {  // reaction 1
        const double kf = 50.80000000000001 * exp(2.67 * logT - 26325728.0 * invRT);
        const double er = exp(th.gRT[1] + th.gRT[5] - th.gRT[0] - th.gRT[3]);
        {  // rate of progress: 1 H2 + 1 O <=> 1 H + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C0 * C3;
            const double rev = kfM * er * C1 * C5;
            const double q = fwd - rev;
            w0 -= q;
            w3 -= q;
            w1 += q;
            w5 += q;
        }
        {  // Jacobian terms
            const double pf = C0 * C3;
            const double pb = C1 * C5;
            const double kfM = kf;
            const double dlnk = (2.67 + 26325728.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[1] + 1.0 * th.hRT[5] - (1.0 * th.hRT[0] + 1.0 * th.hRT[3]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = kfM * (C3);
            const double dq1 = -kfM * er * (C5);
            const double dq3 = kfM * (C0);
            const double dq5 = -kfM * er * (C1);
            const double e_r = -1.0 * (th.hRT[0] - 1.0) + -1.0 * (th.hRT[3] - 1.0) + 1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(0, 0) += -1.0 * s * dq0;
            J(3, 0) += -7.936011904761905 * s * dq0;
            J(1, 0) += 0.5 * s * dq0;
            J(5, 0) += 8.436011904761905 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(0, 1) += -2.0 * s * dq1;
            J(3, 1) += -15.87202380952381 * s * dq1;
            J(1, 1) += 1.0 * s * dq1;
            J(5, 1) += 16.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(0, 3) += -0.12600787549221826 * s * dq3;
            J(3, 3) += -1.0 * s * dq3;
            J(1, 3) += 0.06300393774610913 * s * dq3;
            J(5, 3) += 1.0630039377461091 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(0, 5) += -0.11853942494267065 * s * dq5;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(1, 5) += 0.05926971247133533 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            jc0 += -2.016 * s_rho * dqT;
            jc3 += -15.999 * s_rho * dqT;
            jc1 += 1.008 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 2
        const double kf = 43800000000.00001 * exp(-(29246160.0 * invRT));
        const double er = exp(th.gRT[1] + th.gRT[4] - th.gRT[0] - th.gRT[5]);
        {  // rate of progress: 1 H2 + 1 OH <=> 1 H + 1 H2O
            const double kfM = kf;
            const double fwd = kfM * C0 * C5;
            const double rev = kfM * er * C1 * C4;
            const double q = fwd - rev;
            w0 -= q;
            w5 -= q;
            w1 += q;
            w4 += q;
        }
        {  // Jacobian terms
            const double pf = C0 * C5;
            const double pb = C1 * C4;
            const double kfM = kf;
            const double dlnk = (0.0 + 29246160.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[1] + 1.0 * th.hRT[4] - (1.0 * th.hRT[0] + 1.0 * th.hRT[5]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = kfM * (C5);
            const double dq1 = -kfM * er * (C4);
            const double dq4 = -kfM * er * (C1);
            const double dq5 = kfM * (C0);
            const double e_r = -1.0 * (th.hRT[0] - 1.0) + -1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[4] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(0, 0) += -1.0 * s * dq0;
            J(5, 0) += -8.436011904761905 * s * dq0;
            J(1, 0) += 0.5 * s * dq0;
            J(4, 0) += 8.936011904761905 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(0, 1) += -2.0 * s * dq1;
            J(5, 1) += -16.87202380952381 * s * dq1;
            J(1, 1) += 1.0 * s * dq1;
            J(4, 1) += 17.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(0, 4) += -0.11190674437968359 * s * dq4;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(1, 4) += 0.055953372189841796 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(0, 5) += -0.11853942494267065 * s * dq5;
            J(5, 5) += -1.0 * s * dq5;
            J(1, 5) += 0.05926971247133533 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            jc0 += -2.016 * s_rho * dqT;
            jc5 += -17.007 * s_rho * dqT;
            jc1 += 1.008 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
        }
    }
    {  // reaction 3
        const double kf = 6165000000.000002 * exp(-0.5 * logT);
        const double er = exp((th.gRT[2] - 2.0 * th.gRT[3]) - -1.0 * log_cref);
        {  // rate of progress: 2 O <=> 1 O2  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * (C3 * C3);
            const double rev = kfM * er * C2;
            const double q = fwd - rev;
            w3 -= 2.0 * q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = (C3 * C3);
            const double pb = C2;
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double dkdM = kf;
            const double dlnk = (-0.5 + 0.0 * invRT) * invT;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (-1.0 - (1.0 * th.hRT[2] - (2.0 * th.hRT[3]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = 2.5 * g;
            const double dq1 = g;
            const double dq2 = -kfM * er * (1.0) + g;
            const double dq3 = kfM * (2.0 * C3) + g;
            const double dq4 = 12.0 * g;
            const double dq5 = g;
            const double dq6 = g;
            const double dq7 = g;
            const double e_r = -2.0 * (th.hRT[3] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(3, 0) += -15.87202380952381 * s * dq0;
            J(2, 0) += 15.87202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(3, 1) += -31.74404761904762 * s * dq1;
            J(2, 1) += 31.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(3, 2) += -1.0 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(3, 3) += -2.0 * s * dq3;
            J(2, 3) += 2.0 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(3, 4) += -1.7761865112406328 * s * dq4;
            J(2, 4) += 1.7761865112406328 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(3, 5) += -1.8814605750573292 * s * dq5;
            J(2, 5) += 1.8814605750573292 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(3, 6) += -0.9407302875286646 * s * dq6;
            J(2, 6) += 0.9407302875286646 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(3, 7) += -0.9694600981639702 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc3 += -31.998 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 4
        const double kf = 114000000000.00003 * exp(-(63956624.0 * invRT));
        const double er = exp(th.gRT[3] + th.gRT[5] - th.gRT[2] - th.gRT[1]);
        {  // rate of progress: 1 O2 + 1 H <=> 1 O + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C2 * C1;
            const double rev = kfM * er * C3 * C5;
            const double q = fwd - rev;
            w2 -= q;
            w1 -= q;
            w3 += q;
            w5 += q;
        }
        {  // Jacobian terms
            const double pf = C2 * C1;
            const double pb = C3 * C5;
            const double kfM = kf;
            const double dlnk = (0.0 + 63956624.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[3] + 1.0 * th.hRT[5] - (1.0 * th.hRT[2] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq1 = kfM * (C2);
            const double dq2 = kfM * (C1);
            const double dq3 = -kfM * er * (C5);
            const double dq5 = -kfM * er * (C3);
            const double e_r = -1.0 * (th.hRT[2] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[3] - 1.0) + 1.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(2, 1) += -31.74404761904762 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(3, 1) += 15.87202380952381 * s * dq1;
            J(5, 1) += 16.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(2, 2) += -1.0 * s * dq2;
            J(1, 2) += -0.031501968873054564 * s * dq2;
            J(3, 2) += 0.5 * s * dq2;
            J(5, 2) += 0.5315019688730546 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(2, 3) += -2.0 * s * dq3;
            J(1, 3) += -0.06300393774610913 * s * dq3;
            J(3, 3) += 1.0 * s * dq3;
            J(5, 3) += 1.0630039377461091 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(2, 5) += -1.8814605750573292 * s * dq5;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(3, 5) += 0.9407302875286646 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            jc2 += -31.998 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc3 += 15.999 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
        }
    }
    {  // reaction 5
        const double kf = 3.5000000000000016e+16 * exp(-2.0 * logT);
        const double er = exp((th.gRT[4] - th.gRT[1] - th.gRT[5]) - -1.0 * log_cref);
        {  // rate of progress: 1 H + 1 OH <=> 1 H2O  + M
            const double M = 0.73 * C0 + C1 + C2 + C3 + 3.65 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C1 * C5;
            const double rev = kfM * er * C4;
            const double q = fwd - rev;
            w1 -= q;
            w5 -= q;
            w4 += q;
        }
        {  // Jacobian terms
            const double pf = C1 * C5;
            const double pb = C4;
            const double M = 0.73 * C0 + C1 + C2 + C3 + 3.65 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double dkdM = kf;
            const double dlnk = (-2.0 + 0.0 * invRT) * invT;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (-1.0 - (1.0 * th.hRT[4] - (1.0 * th.hRT[1] + 1.0 * th.hRT[5]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = 0.73 * g;
            const double dq1 = kfM * (C5) + g;
            const double dq2 = g;
            const double dq3 = g;
            const double dq4 = -kfM * er * (1.0) + 3.65 * g;
            const double dq5 = kfM * (C1) + g;
            const double dq6 = g;
            const double dq7 = g;
            const double e_r = -1.0 * (th.hRT[1] - 1.0) + -1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[4] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(1, 0) += -0.5 * s * dq0;
            J(5, 0) += -8.436011904761905 * s * dq0;
            J(4, 0) += 8.936011904761905 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(1, 1) += -1.0 * s * dq1;
            J(5, 1) += -16.87202380952381 * s * dq1;
            J(4, 1) += 17.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(1, 2) += -0.031501968873054564 * s * dq2;
            J(5, 2) += -0.5315019688730546 * s * dq2;
            J(4, 2) += 0.5630039377461091 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(1, 3) += -0.06300393774610913 * s * dq3;
            J(5, 3) += -1.0630039377461091 * s * dq3;
            J(4, 3) += 1.1260078754922183 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(1, 4) += -0.055953372189841796 * s * dq4;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(5, 5) += -1.0 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(1, 6) += -0.029634856235667664 * s * dq6;
            J(5, 6) += -0.5 * s * dq6;
            J(4, 6) += 0.5296348562356676 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(4, 7) += 0.5458098527540447 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc1 += -1.008 * s_rho * dqT;
            jc5 += -17.007 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 6
        const double kf = 67000.00000000001 * exp(1.704 * logT - 62704771.199999996 * invRT);
        const double er = exp(2.0 * th.gRT[5] - th.gRT[3] - th.gRT[4]);
        {  // rate of progress: 1 O + 1 H2O <=> 2 OH
            const double kfM = kf;
            const double fwd = kfM * C3 * C4;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w3 -= q;
            w4 -= q;
            w5 += 2.0 * q;
        }
        {  // Jacobian terms
            const double pf = C3 * C4;
            const double pb = (C5 * C5);
            const double kfM = kf;
            const double dlnk = (1.704 + 62704771.199999996 * invRT) * invT;
            const double dlner = (0.0 - (2.0 * th.hRT[5] - (1.0 * th.hRT[3] + 1.0 * th.hRT[4]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq3 = kfM * (C4);
            const double dq4 = kfM * (C3);
            const double dq5 = -kfM * er * (2.0 * C5);
            const double e_r = -1.0 * (th.hRT[3] - 1.0) + -1.0 * (th.hRT[4] - 1.0) + 2.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(3, 3) += -1.0 * s * dq3;
            J(4, 3) += -1.1260078754922183 * s * dq3;
            J(5, 3) += 2.1260078754922183 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(3, 4) += -0.8880932556203164 * s * dq4;
            J(4, 4) += -1.0 * s * dq4;
            J(5, 4) += 1.8880932556203165 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(4, 5) += -1.0592697124713353 * s * dq5;
            J(5, 5) += 2.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            jc3 += -15.999 * s_rho * dqT;
            jc4 += -18.015 * s_rho * dqT;
            jc5 += 34.014 * s_rho * dqT;
        }
    }
    {  // reaction 7
        const double kf = 4714000000000.002 * exp(-1.0 * logT);
        const double er = exp((th.gRT[5] - th.gRT[3] - th.gRT[1]) - -1.0 * log_cref);
        {  // rate of progress: 1 O + 1 H <=> 1 OH  + M
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C3 * C1;
            const double rev = kfM * er * C5;
            const double q = fwd - rev;
            w3 -= q;
            w1 -= q;
            w5 += q;
        }
        {  // Jacobian terms
            const double pf = C3 * C1;
            const double pb = C5;
            const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double dkdM = kf;
            const double dlnk = (-1.0 + 0.0 * invRT) * invT;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (-1.0 - (1.0 * th.hRT[5] - (1.0 * th.hRT[3] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = 2.5 * g;
            const double dq1 = kfM * (C3) + g;
            const double dq2 = g;
            const double dq3 = kfM * (C1) + g;
            const double dq4 = 12.0 * g;
            const double dq5 = -kfM * er * (1.0) + g;
            const double dq6 = g;
            const double dq7 = g;
            const double e_r = -1.0 * (th.hRT[3] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(3, 0) += -7.936011904761905 * s * dq0;
            J(1, 0) += -0.5 * s * dq0;
            J(5, 0) += 8.436011904761905 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(3, 1) += -15.87202380952381 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(5, 1) += 16.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(3, 2) += -0.5 * s * dq2;
            J(1, 2) += -0.031501968873054564 * s * dq2;
            J(5, 2) += 0.5315019688730546 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(3, 3) += -1.0 * s * dq3;
            J(1, 3) += -0.06300393774610913 * s * dq3;
            J(5, 3) += 1.0630039377461091 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(3, 4) += -0.8880932556203164 * s * dq4;
            J(1, 4) += -0.055953372189841796 * s * dq4;
            J(5, 4) += 0.9440466278101582 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(3, 6) += -0.4703651437643323 * s * dq6;
            J(1, 6) += -0.029634856235667664 * s * dq6;
            J(5, 6) += 0.5 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(3, 7) += -0.4847300490819851 * s * dq7;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(5, 7) += 0.515269950918015 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc3 += -15.999 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 8
        const double kf = 2000000000000.0 * exp(0.9 * logT - 203965816.0 * invRT);
        const double k0 = 2.4900000000000005e+21 * exp(-2.3 * logT - 203965816.0 * invRT);
        const double lFc0 = -0.36653154442041347;
        const double er = exp((2.0 * th.gRT[5] - th.gRT[6]) - 1.0 * log_cref);
        {  // rate of progress: 1 H2O2 <=> 2 OH  (+M)
            const double M = 3.7 * C0 + C1 + 1.2 * C2 + C3 + 7.65 * C4 + C5 + 7.7 * C6 + C7 + 1.5 * C8;
            const double Pr = k0 * M / kf;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double x = (lPr + c) / (n - 0.14 * (lPr + c));
            const double kfM = kf * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
            const double fwd = kfM * C6;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w6 -= q;
            w5 += 2.0 * q;
        }
        {  // Jacobian terms
            const double pf = C6;
            const double pb = (C5 * C5);
            const double M = 3.7 * C0 + C1 + 1.2 * C2 + C3 + 7.65 * C4 + C5 + 7.7 * C6 + C7 + 1.5 * C8;
            const double Pr = k0 * M / kf;
            const double ipr = 1.0 / (1.0 + Pr);
            const double dlnkinf = (0.9 + 203965816.0 * invRT) * invT;
            const double dlnk0 = (-2.3 + 203965816.0 * invRT) * invT;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double u = lPr + c, den = n - 0.14 * u;
            const double x = u / den;
            const double opx = 1.0 + x * x;
            const double Fo = pow(10.0, lFc / opx);
            const double kfM = kf * (Pr * ipr) * Fo;
            const double dkdM = k0 * Fo * ipr * (ipr - 2.0 * x * lFc * n / (opx * opx * den * den));
            const double dlFc = 0.0;
            const double du = (dlnk0 - dlnkinf) * 0.4342944819032518 - 0.67 * dlFc;
            const double dden = -1.27 * dlFc - 0.14 * du;
            const double dx = (du * den - u * dden) / (den * den);
            const double dlnFo = 2.302585092994046 * (dlFc / opx - 2.0 * x * lFc * dx / (opx * opx));
            const double dlnk = dlnkinf + (dlnk0 - dlnkinf) * ipr + dlnFo;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (1.0 - (2.0 * th.hRT[5] - (1.0 * th.hRT[6]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = 3.7 * g;
            const double dq1 = g;
            const double dq2 = 1.2 * g;
            const double dq3 = g;
            const double dq4 = 7.65 * g;
            const double dq5 = -kfM * er * (2.0 * C5) + g;
            const double dq6 = kfM * (1.0) + 7.7 * g;
            const double dq7 = g;
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + 2.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 0) += -16.87202380952381 * s * dq0;
            J(5, 0) += 16.87202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(6, 1) += -33.74404761904762 * s * dq1;
            J(5, 1) += 33.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(6, 2) += -1.0630039377461091 * s * dq2;
            J(5, 2) += 1.0630039377461091 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(6, 3) += -2.1260078754922183 * s * dq3;
            J(5, 3) += 2.1260078754922183 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(6, 4) += -1.8880932556203165 * s * dq4;
            J(5, 4) += 1.8880932556203165 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(6, 5) += -2.0 * s * dq5;
            J(5, 5) += 2.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(6, 6) += -1.0 * s * dq6;
            J(5, 6) += 1.0 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(6, 7) += -1.03053990183603 * s * dq7;
            J(5, 7) += 1.03053990183603 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc6 += -34.014 * s_rho * dqT;
            jc5 += 34.014 * s_rho * dqT;
        }
    }
    {  // reaction 9
        const double kf = 24100000000.000008 * exp(-(16610480.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[5] - th.gRT[6] - th.gRT[1]);
        {  // rate of progress: 1 H2O2 + 1 H <=> 1 H2O + 1 OH
            const double kfM = kf;
            const double fwd = kfM * C6 * C1;
            const double rev = kfM * er * C4 * C5;
            const double q = fwd - rev;
            w6 -= q;
            w1 -= q;
            w4 += q;
            w5 += q;
        }
        {  // Jacobian terms
            const double pf = C6 * C1;
            const double pb = C4 * C5;
            const double kfM = kf;
            const double dlnk = (0.0 + 16610480.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[4] + 1.0 * th.hRT[5] - (1.0 * th.hRT[6] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq1 = kfM * (C6);
            const double dq4 = -kfM * er * (C5);
            const double dq5 = -kfM * er * (C4);
            const double dq6 = kfM * (C1);
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[4] - 1.0) + 1.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 1) += -33.74404761904762 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(4, 1) += 17.87202380952381 * s * dq1;
            J(5, 1) += 16.87202380952381 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(6, 4) += -1.8880932556203165 * s * dq4;
            J(1, 4) += -0.055953372189841796 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            J(5, 4) += 0.9440466278101582 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(6, 5) += -2.0 * s * dq5;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(6, 6) += -1.0 * s * dq6;
            J(1, 6) += -0.029634856235667664 * s * dq6;
            J(4, 6) += 0.5296348562356676 * s * dq6;
            J(5, 6) += 0.5 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            jc6 += -34.014 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 10
        const double kf = 21500000.000000004 * exp(1.0 * logT - 25104000.0 * invRT);
        const double er = exp(th.gRT[0] + th.gRT[7] - th.gRT[6] - th.gRT[1]);
        {  // rate of progress: 1 H2O2 + 1 H <=> 1 H2 + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C1;
            const double rev = kfM * er * C0 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w1 -= q;
            w0 += q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C6 * C1;
            const double pb = C0 * C7;
            const double kfM = kf;
            const double dlnk = (1.0 + 25104000.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[0] + 1.0 * th.hRT[7] - (1.0 * th.hRT[6] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = -kfM * er * (C7);
            const double dq1 = kfM * (C6);
            const double dq6 = kfM * (C1);
            const double dq7 = -kfM * er * (C0);
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[0] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 0) += -16.87202380952381 * s * dq0;
            J(1, 0) += -0.5 * s * dq0;
            J(0, 0) += 1.0 * s * dq0;
            J(7, 0) += 16.37202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(6, 1) += -33.74404761904762 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(0, 1) += 2.0 * s * dq1;
            J(7, 1) += 32.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(6, 6) += -1.0 * s * dq6;
            J(1, 6) += -0.029634856235667664 * s * dq6;
            J(0, 6) += 0.05926971247133533 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(6, 7) += -1.03053990183603 * s * dq7;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(0, 7) += 0.061079803672059625 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc6 += -34.014 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc0 += 2.016 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    {  // reaction 11
        const double kf = 9550.000000000002 * exp(2.0 * logT - 16610480.0 * invRT);
        const double er = exp(th.gRT[5] + th.gRT[7] - th.gRT[6] - th.gRT[3]);
        {  // rate of progress: 1 H2O2 + 1 O <=> 1 OH + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C3;
            const double rev = kfM * er * C5 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w3 -= q;
            w5 += q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C6 * C3;
            const double pb = C5 * C7;
            const double kfM = kf;
            const double dlnk = (2.0 + 16610480.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[5] + 1.0 * th.hRT[7] - (1.0 * th.hRT[6] + 1.0 * th.hRT[3]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq3 = kfM * (C6);
            const double dq5 = -kfM * er * (C7);
            const double dq6 = kfM * (C3);
            const double dq7 = -kfM * er * (C5);
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + -1.0 * (th.hRT[3] - 1.0) + 1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 3) += -2.1260078754922183 * s * dq3;
            J(3, 3) += -1.0 * s * dq3;
            J(5, 3) += 1.0630039377461091 * s * dq3;
            J(7, 3) += 2.063003937746109 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(6, 5) += -2.0 * s * dq5;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            J(7, 5) += 1.9407302875286645 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(6, 6) += -1.0 * s * dq6;
            J(3, 6) += -0.4703651437643323 * s * dq6;
            J(5, 6) += 0.5 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(6, 7) += -1.03053990183603 * s * dq7;
            J(3, 7) += -0.4847300490819851 * s * dq7;
            J(5, 7) += 0.515269950918015 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc6 += -34.014 * s_rho * dqT;
            jc3 += -15.999 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 12
        const double kf = 1740000000.0000005 * exp(-(1330512.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[7] - th.gRT[6] - th.gRT[5]);
        {  // rate of progress: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C5;
            const double rev = kfM * er * C4 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w5 -= q;
            w4 += q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C6 * C5;
            const double pb = C4 * C7;
            const double kfM = kf;
            const double dlnk = (0.0 + 1330512.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[4] + 1.0 * th.hRT[7] - (1.0 * th.hRT[6] + 1.0 * th.hRT[5]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq4 = -kfM * er * (C7);
            const double dq5 = kfM * (C6);
            const double dq6 = kfM * (C5);
            const double dq7 = -kfM * er * (C4);
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + -1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[4] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 4) += -1.8880932556203165 * s * dq4;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            J(7, 4) += 1.8321398834304745 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(6, 5) += -2.0 * s * dq5;
            J(5, 5) += -1.0 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            J(7, 5) += 1.9407302875286645 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(6, 6) += -1.0 * s * dq6;
            J(5, 6) += -0.5 * s * dq6;
            J(4, 6) += 0.5296348562356676 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(6, 7) += -1.03053990183603 * s * dq7;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(4, 7) += 0.5458098527540447 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc6 += -34.014 * s_rho * dqT;
            jc5 += -17.007 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    {  // reaction 13
        const double kf = 75900000000.00002 * exp(-(30413496.0 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[7] - th.gRT[6] - th.gRT[5]);
        {  // rate of progress: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
            const double kfM = kf;
            const double fwd = kfM * C6 * C5;
            const double rev = kfM * er * C4 * C7;
            const double q = fwd - rev;
            w6 -= q;
            w5 -= q;
            w4 += q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C6 * C5;
            const double pb = C4 * C7;
            const double kfM = kf;
            const double dlnk = (0.0 + 30413496.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[4] + 1.0 * th.hRT[7] - (1.0 * th.hRT[6] + 1.0 * th.hRT[5]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq4 = -kfM * er * (C7);
            const double dq5 = kfM * (C6);
            const double dq6 = kfM * (C5);
            const double dq7 = -kfM * er * (C4);
            const double e_r = -1.0 * (th.hRT[6] - 1.0) + -1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[4] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(6, 4) += -1.8880932556203165 * s * dq4;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            J(7, 4) += 1.8321398834304745 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(6, 5) += -2.0 * s * dq5;
            J(5, 5) += -1.0 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            J(7, 5) += 1.9407302875286645 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(6, 6) += -1.0 * s * dq6;
            J(5, 6) += -0.5 * s * dq6;
            J(4, 6) += 0.5296348562356676 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(6, 7) += -1.03053990183603 * s * dq7;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(4, 7) += 0.5458098527540447 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc6 += -34.014 * s_rho * dqT;
            jc5 += -17.007 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 14
        const double kf = 70790000000.00002 * exp(-(1234280.0 * invRT));
        const double er = exp(2.0 * th.gRT[5] - th.gRT[7] - th.gRT[1]);
        {  // rate of progress: 1 HO2 + 1 H <=> 2 OH
            const double kfM = kf;
            const double fwd = kfM * C7 * C1;
            const double rev = kfM * er * (C5 * C5);
            const double q = fwd - rev;
            w7 -= q;
            w1 -= q;
            w5 += 2.0 * q;
        }
        {  // Jacobian terms
            const double pf = C7 * C1;
            const double pb = (C5 * C5);
            const double kfM = kf;
            const double dlnk = (0.0 + 1234280.0 * invRT) * invT;
            const double dlner = (0.0 - (2.0 * th.hRT[5] - (1.0 * th.hRT[7] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq1 = kfM * (C7);
            const double dq5 = -kfM * er * (2.0 * C5);
            const double dq7 = kfM * (C1);
            const double e_r = -1.0 * (th.hRT[7] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 2.0 * (th.hRT[5] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(7, 1) += -32.74404761904762 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(5, 1) += 33.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(7, 5) += -1.9407302875286645 * s * dq5;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(5, 5) += 2.0 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(7, 7) += -1.0 * s * dq7;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(5, 7) += 1.03053990183603 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc7 += -33.006 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc5 += 34.014 * s_rho * dqT;
        }
    }
    {  // reaction 15
        const double kf = 11402000.000000002 * exp(1.0827 * logT - 2317015.52 * invRT);
        const double er = exp(th.gRT[0] + th.gRT[2] - th.gRT[7] - th.gRT[1]);
        {  // rate of progress: 1 HO2 + 1 H <=> 1 H2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C7 * C1;
            const double rev = kfM * er * C0 * C2;
            const double q = fwd - rev;
            w7 -= q;
            w1 -= q;
            w0 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = C7 * C1;
            const double pb = C0 * C2;
            const double kfM = kf;
            const double dlnk = (1.0827 + 2317015.52 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[0] + 1.0 * th.hRT[2] - (1.0 * th.hRT[7] + 1.0 * th.hRT[1]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = -kfM * er * (C2);
            const double dq1 = kfM * (C7);
            const double dq2 = -kfM * er * (C0);
            const double dq7 = kfM * (C1);
            const double e_r = -1.0 * (th.hRT[7] - 1.0) + -1.0 * (th.hRT[1] - 1.0) + 1.0 * (th.hRT[0] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(7, 0) += -16.37202380952381 * s * dq0;
            J(1, 0) += -0.5 * s * dq0;
            J(0, 0) += 1.0 * s * dq0;
            J(2, 0) += 15.87202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(7, 1) += -32.74404761904762 * s * dq1;
            J(1, 1) += -1.0 * s * dq1;
            J(0, 1) += 2.0 * s * dq1;
            J(2, 1) += 31.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(7, 2) += -1.0315019688730545 * s * dq2;
            J(1, 2) += -0.031501968873054564 * s * dq2;
            J(0, 2) += 0.06300393774610913 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(7, 7) += -1.0 * s * dq7;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(0, 7) += 0.061079803672059625 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc7 += -33.006 * s_rho * dqT;
            jc1 += -1.008 * s_rho * dqT;
            jc0 += 2.016 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 16
        const double kf = 32500000000.000008;
        const double er = exp(th.gRT[5] + th.gRT[2] - th.gRT[7] - th.gRT[3]);
        {  // rate of progress: 1 HO2 + 1 O <=> 1 OH + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C7 * C3;
            const double rev = kfM * er * C5 * C2;
            const double q = fwd - rev;
            w7 -= q;
            w3 -= q;
            w5 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = C7 * C3;
            const double pb = C5 * C2;
            const double kfM = kf;
            const double dlnk = (0.0 + 0.0 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[5] + 1.0 * th.hRT[2] - (1.0 * th.hRT[7] + 1.0 * th.hRT[3]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq2 = -kfM * er * (C5);
            const double dq3 = kfM * (C7);
            const double dq5 = -kfM * er * (C2);
            const double dq7 = kfM * (C3);
            const double e_r = -1.0 * (th.hRT[7] - 1.0) + -1.0 * (th.hRT[3] - 1.0) + 1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(7, 2) += -1.0315019688730545 * s * dq2;
            J(3, 2) += -0.5 * s * dq2;
            J(5, 2) += 0.5315019688730546 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(7, 3) += -2.063003937746109 * s * dq3;
            J(3, 3) += -1.0 * s * dq3;
            J(5, 3) += 1.0630039377461091 * s * dq3;
            J(2, 3) += 2.0 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(7, 5) += -1.9407302875286645 * s * dq5;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(5, 5) += 1.0 * s * dq5;
            J(2, 5) += 1.8814605750573292 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(7, 7) += -1.0 * s * dq7;
            J(3, 7) += -0.4847300490819851 * s * dq7;
            J(5, 7) += 0.515269950918015 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc7 += -33.006 * s_rho * dqT;
            jc3 += -15.999 * s_rho * dqT;
            jc5 += 17.007 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    {  // reaction 17
        const double kf = 7000000000.000002 * exp(-(-4572944.640000001 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[2] - th.gRT[5] - th.gRT[7]);
        {  // rate of progress: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C5 * C7;
            const double rev = kfM * er * C4 * C2;
            const double q = fwd - rev;
            w5 -= q;
            w7 -= q;
            w4 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = C5 * C7;
            const double pb = C4 * C2;
            const double kfM = kf;
            const double dlnk = (0.0 + -4572944.640000001 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[4] + 1.0 * th.hRT[2] - (1.0 * th.hRT[5] + 1.0 * th.hRT[7]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq2 = -kfM * er * (C4);
            const double dq4 = -kfM * er * (C2);
            const double dq5 = kfM * (C7);
            const double dq7 = kfM * (C5);
            const double e_r = -1.0 * (th.hRT[5] - 1.0) + -1.0 * (th.hRT[7] - 1.0) + 1.0 * (th.hRT[4] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(5, 2) += -0.5315019688730546 * s * dq2;
            J(7, 2) += -1.0315019688730545 * s * dq2;
            J(4, 2) += 0.5630039377461091 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(7, 4) += -1.8321398834304745 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            J(2, 4) += 1.7761865112406328 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(5, 5) += -1.0 * s * dq5;
            J(7, 5) += -1.9407302875286645 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            J(2, 5) += 1.8814605750573292 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(7, 7) += -1.0 * s * dq7;
            J(4, 7) += 0.5458098527540447 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc5 += -17.007 * s_rho * dqT;
            jc7 += -33.006 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 18
        const double kf = 450000000000.0001 * exp(-(45729446.4 * invRT));
        const double er = exp(th.gRT[4] + th.gRT[2] - th.gRT[5] - th.gRT[7]);
        {  // rate of progress: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
            const double kfM = kf;
            const double fwd = kfM * C5 * C7;
            const double rev = kfM * er * C4 * C2;
            const double q = fwd - rev;
            w5 -= q;
            w7 -= q;
            w4 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = C5 * C7;
            const double pb = C4 * C2;
            const double kfM = kf;
            const double dlnk = (0.0 + 45729446.4 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[4] + 1.0 * th.hRT[2] - (1.0 * th.hRT[5] + 1.0 * th.hRT[7]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq2 = -kfM * er * (C4);
            const double dq4 = -kfM * er * (C2);
            const double dq5 = kfM * (C7);
            const double dq7 = kfM * (C5);
            const double e_r = -1.0 * (th.hRT[5] - 1.0) + -1.0 * (th.hRT[7] - 1.0) + 1.0 * (th.hRT[4] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(5, 2) += -0.5315019688730546 * s * dq2;
            J(7, 2) += -1.0315019688730545 * s * dq2;
            J(4, 2) += 0.5630039377461091 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(7, 4) += -1.8321398834304745 * s * dq4;
            J(4, 4) += 1.0 * s * dq4;
            J(2, 4) += 1.7761865112406328 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(5, 5) += -1.0 * s * dq5;
            J(7, 5) += -1.9407302875286645 * s * dq5;
            J(4, 5) += 1.0592697124713353 * s * dq5;
            J(2, 5) += 1.8814605750573292 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(7, 7) += -1.0 * s * dq7;
            J(4, 7) += 0.5458098527540447 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc5 += -17.007 * s_rho * dqT;
            jc7 += -33.006 * s_rho * dqT;
            jc4 += 18.015 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    {  // reaction 19
        const double kf = 100000000000.00003 * exp(-(46195054.472 * invRT));
        const double er = exp(th.gRT[6] + th.gRT[2] - 2.0 * th.gRT[7]);
        {  // rate of progress: 2 HO2 <=> 1 H2O2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * (C7 * C7);
            const double rev = kfM * er * C6 * C2;
            const double q = fwd - rev;
            w7 -= 2.0 * q;
            w6 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = (C7 * C7);
            const double pb = C6 * C2;
            const double kfM = kf;
            const double dlnk = (0.0 + 46195054.472 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[6] + 1.0 * th.hRT[2] - (2.0 * th.hRT[7]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq2 = -kfM * er * (C6);
            const double dq6 = -kfM * er * (C2);
            const double dq7 = kfM * (2.0 * C7);
            const double e_r = -2.0 * (th.hRT[7] - 1.0) + 1.0 * (th.hRT[6] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(7, 2) += -2.063003937746109 * s * dq2;
            J(6, 2) += 1.0630039377461091 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(7, 6) += -1.9407302875286645 * s * dq6;
            J(6, 6) += 1.0 * s * dq6;
            J(2, 6) += 0.9407302875286646 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(7, 7) += -2.0 * s * dq7;
            J(6, 7) += 1.03053990183603 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc7 += -66.012 * s_rho * dqT;
            jc6 += 34.014 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 20
        const double kf = 190000000.00000006 * exp(-(-5894941.3632 * invRT));
        const double er = exp(th.gRT[6] + th.gRT[2] - 2.0 * th.gRT[7]);
        {  // rate of progress: 2 HO2 <=> 1 H2O2 + 1 O2
            const double kfM = kf;
            const double fwd = kfM * (C7 * C7);
            const double rev = kfM * er * C6 * C2;
            const double q = fwd - rev;
            w7 -= 2.0 * q;
            w6 += q;
            w2 += q;
        }
        {  // Jacobian terms
            const double pf = (C7 * C7);
            const double pb = C6 * C2;
            const double kfM = kf;
            const double dlnk = (0.0 + -5894941.3632 * invRT) * invT;
            const double dlner = (0.0 - (1.0 * th.hRT[6] + 1.0 * th.hRT[2] - (2.0 * th.hRT[7]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq2 = -kfM * er * (C6);
            const double dq6 = -kfM * er * (C2);
            const double dq7 = kfM * (2.0 * C7);
            const double e_r = -2.0 * (th.hRT[7] - 1.0) + 1.0 * (th.hRT[6] - 1.0) + 1.0 * (th.hRT[2] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(7, 2) += -2.063003937746109 * s * dq2;
            J(6, 2) += 1.0630039377461091 * s * dq2;
            J(2, 2) += 1.0 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(7, 6) += -1.9407302875286645 * s * dq6;
            J(6, 6) += 1.0 * s * dq6;
            J(2, 6) += 0.9407302875286646 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(7, 7) += -2.0 * s * dq7;
            J(6, 7) += 1.03053990183603 * s * dq7;
            J(2, 7) += 0.9694600981639702 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc7 += -66.012 * s_rho * dqT;
            jc6 += 34.014 * s_rho * dqT;
            jc2 += 31.998 * s_rho * dqT;
        }
    }
    {  // reaction 21
        const double kf = 4650000000.000001 * exp(0.44 * logT);
        const double k0 = 17370000000000.006 * exp(-1.23 * logT);
        const double lFc0 = -0.17392519729917352;
        const double er = exp((th.gRT[7] - th.gRT[1] - th.gRT[2]) - -1.0 * log_cref);
        {  // rate of progress: 1 H + 1 O2 <=> 1 HO2  (+M)
            const double M = 1.3 * C0 + C1 + C2 + C3 + 10.0 * C4 + C5 + C6 + C7 + C8;
            const double Pr = k0 * M / kf;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double x = (lPr + c) / (n - 0.14 * (lPr + c));
            const double kfM = kf * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
            const double fwd = kfM * C1 * C2;
            const double rev = kfM * er * C7;
            const double q = fwd - rev;
            w1 -= q;
            w2 -= q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C1 * C2;
            const double pb = C7;
            const double M = 1.3 * C0 + C1 + C2 + C3 + 10.0 * C4 + C5 + C6 + C7 + C8;
            const double Pr = k0 * M / kf;
            const double ipr = 1.0 / (1.0 + Pr);
            const double dlnkinf = (0.44 + 0.0 * invRT) * invT;
            const double dlnk0 = (-1.23 + 0.0 * invRT) * invT;
            const double lFc = lFc0;
            const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
            const double lPr = log10(fmax(Pr, 1e-300));
            const double u = lPr + c, den = n - 0.14 * u;
            const double x = u / den;
            const double opx = 1.0 + x * x;
            const double Fo = pow(10.0, lFc / opx);
            const double kfM = kf * (Pr * ipr) * Fo;
            const double dkdM = k0 * Fo * ipr * (ipr - 2.0 * x * lFc * n / (opx * opx * den * den));
            const double dlFc = 0.0;
            const double du = (dlnk0 - dlnkinf) * 0.4342944819032518 - 0.67 * dlFc;
            const double dden = -1.27 * dlFc - 0.14 * du;
            const double dx = (du * den - u * dden) / (den * den);
            const double dlnFo = 2.302585092994046 * (dlFc / opx - 2.0 * x * lFc * dx / (opx * opx));
            const double dlnk = dlnkinf + (dlnk0 - dlnkinf) * ipr + dlnFo;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (-1.0 - (1.0 * th.hRT[7] - (1.0 * th.hRT[1] + 1.0 * th.hRT[2]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = 1.3 * g;
            const double dq1 = kfM * (C2) + g;
            const double dq2 = kfM * (C1) + g;
            const double dq3 = g;
            const double dq4 = 10.0 * g;
            const double dq5 = g;
            const double dq6 = g;
            const double dq7 = -kfM * er * (1.0) + g;
            const double e_r = -1.0 * (th.hRT[1] - 1.0) + -1.0 * (th.hRT[2] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(1, 0) += -0.5 * s * dq0;
            J(2, 0) += -15.87202380952381 * s * dq0;
            J(7, 0) += 16.37202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(1, 1) += -1.0 * s * dq1;
            J(2, 1) += -31.74404761904762 * s * dq1;
            J(7, 1) += 32.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(1, 2) += -0.031501968873054564 * s * dq2;
            J(2, 2) += -1.0 * s * dq2;
            J(7, 2) += 1.0315019688730545 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(1, 3) += -0.06300393774610913 * s * dq3;
            J(2, 3) += -2.0 * s * dq3;
            J(7, 3) += 2.063003937746109 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(1, 4) += -0.055953372189841796 * s * dq4;
            J(2, 4) += -1.7761865112406328 * s * dq4;
            J(7, 4) += 1.8321398834304745 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(1, 5) += -0.05926971247133533 * s * dq5;
            J(2, 5) += -1.8814605750573292 * s * dq5;
            J(7, 5) += 1.9407302875286645 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(1, 6) += -0.029634856235667664 * s * dq6;
            J(2, 6) += -0.9407302875286646 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(1, 7) += -0.030539901836029813 * s * dq7;
            J(2, 7) += -0.9694600981639702 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc1 += -1.008 * s_rho * dqT;
            jc2 += -31.998 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    GAS_SCHED_FENCE();
    {  // reaction 22
        const double kf = 10000000000.000004;
        const double er = exp((th.gRT[7] - th.gRT[3] - th.gRT[5]) - -1.0 * log_cref);
        {  // rate of progress: 1 O + 1 OH <=> 1 HO2  + M
            const double M = C0 + C1 + C2 + C3 + C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double fwd = kfM * C3 * C5;
            const double rev = kfM * er * C7;
            const double q = fwd - rev;
            w3 -= q;
            w5 -= q;
            w7 += q;
        }
        {  // Jacobian terms
            const double pf = C3 * C5;
            const double pb = C7;
            const double M = C0 + C1 + C2 + C3 + C4 + C5 + C6 + C7 + C8;
            const double kfM = kf * M;
            const double dkdM = kf;
            const double dlnk = (0.0 + 0.0 * invRT) * invT;
            const double g = dkdM * (pf - er * pb);
            const double dlner = (-1.0 - (1.0 * th.hRT[7] - (1.0 * th.hRT[3] + 1.0 * th.hRT[5]))) * invT;
            const double dqT = kfM * (dlnk * (pf - er * pb) - er * dlner * pb);
            const double dq0 = g;
            const double dq1 = g;
            const double dq2 = g;
            const double dq3 = kfM * (C5) + g;
            const double dq4 = g;
            const double dq5 = kfM * (C3) + g;
            const double dq6 = g;
            const double dq7 = -kfM * er * (1.0) + g;
            const double e_r = -1.0 * (th.hRT[3] - 1.0) + -1.0 * (th.hRT[5] - 1.0) + 1.0 * (th.hRT[7] - 1.0);
            const double eT = sT * e_r;
            sum_eT += e_r * dqT;
            J(3, 0) += -7.936011904761905 * s * dq0;
            J(5, 0) += -8.436011904761905 * s * dq0;
            J(7, 0) += 16.37202380952381 * s * dq0;
            jT0 += 0.49603174603174605 * eT * dq0;
            J(3, 1) += -15.87202380952381 * s * dq1;
            J(5, 1) += -16.87202380952381 * s * dq1;
            J(7, 1) += 32.74404761904762 * s * dq1;
            jT1 += 0.9920634920634921 * eT * dq1;
            J(3, 2) += -0.5 * s * dq2;
            J(5, 2) += -0.5315019688730546 * s * dq2;
            J(7, 2) += 1.0315019688730545 * s * dq2;
            jT2 += 0.03125195324707794 * eT * dq2;
            J(3, 3) += -1.0 * s * dq3;
            J(5, 3) += -1.0630039377461091 * s * dq3;
            J(7, 3) += 2.063003937746109 * s * dq3;
            jT3 += 0.06250390649415588 * eT * dq3;
            J(3, 4) += -0.8880932556203164 * s * dq4;
            J(5, 4) += -0.9440466278101582 * s * dq4;
            J(7, 4) += 1.8321398834304745 * s * dq4;
            jT4 += 0.055509297807382736 * eT * dq4;
            J(3, 5) += -0.9407302875286646 * s * dq5;
            J(5, 5) += -1.0 * s * dq5;
            J(7, 5) += 1.9407302875286645 * s * dq5;
            jT5 += 0.05879931792791203 * eT * dq5;
            J(3, 6) += -0.4703651437643323 * s * dq6;
            J(5, 6) += -0.5 * s * dq6;
            J(7, 6) += 0.9703651437643322 * s * dq6;
            jT6 += 0.029399658963956014 * eT * dq6;
            J(3, 7) += -0.4847300490819851 * s * dq7;
            J(5, 7) += -0.515269950918015 * s * dq7;
            J(7, 7) += 1.0 * s * dq7;
            jT7 += 0.030297521662727988 * eT * dq7;
            jc3 += -15.999 * s_rho * dqT;
            jc5 += -17.007 * s_rho * dqT;
            jc7 += 33.006 * s_rho * dqT;
        }
    }
    double es = 0.0;
    F[0] = w0 * 2.016 / rho;
    es += (th.hRT[0] - 1.0) * 8314.46261815324 * T * w0;
    F[1] = w1 * 1.008 / rho;
    es += (th.hRT[1] - 1.0) * 8314.46261815324 * T * w1;
    F[2] = w2 * 31.998 / rho;
    es += (th.hRT[2] - 1.0) * 8314.46261815324 * T * w2;
    F[3] = w3 * 15.999 / rho;
    es += (th.hRT[3] - 1.0) * 8314.46261815324 * T * w3;
    F[4] = w4 * 18.015 / rho;
    es += (th.hRT[4] - 1.0) * 8314.46261815324 * T * w4;
    F[5] = w5 * 17.007 / rho;
    es += (th.hRT[5] - 1.0) * 8314.46261815324 * T * w5;
    F[6] = w6 * 34.014 / rho;
    es += (th.hRT[6] - 1.0) * 8314.46261815324 * T * w6;
    F[7] = w7 * 33.006 / rho;
    es += (th.hRT[7] - 1.0) * 8314.46261815324 * T * w7;
    F[8] = w8 * 28.014 / rho;
    es += (th.hRT[8] - 1.0) * 8314.46261815324 * T * w8;
    F[9] = -es / (rho * cv);
    const double sF = s * F[9] * 8314.46261815324 / cv;
    J(8, 0) = jT0 - sF * (th.cpR[0] - 1.0) * 0.49603174603174605;
    J(0, 8) = jc0;
    J(8, 1) = jT1 - sF * (th.cpR[1] - 1.0) * 0.9920634920634921;
    J(1, 8) = jc1;
    J(8, 2) = jT2 - sF * (th.cpR[2] - 1.0) * 0.03125195324707794;
    J(2, 8) = jc2;
    J(8, 3) = jT3 - sF * (th.cpR[3] - 1.0) * 0.06250390649415588;
    J(3, 8) = jc3;
    J(8, 4) = jT4 - sF * (th.cpR[4] - 1.0) * 0.055509297807382736;
    J(4, 8) = jc4;
    J(8, 5) = jT5 - sF * (th.cpR[5] - 1.0) * 0.05879931792791203;
    J(5, 8) = jc5;
    J(8, 6) = jT6 - sF * (th.cpR[6] - 1.0) * 0.029399658963956014;
    J(6, 8) = jc6;
    J(8, 7) = jT7 - sF * (th.cpR[7] - 1.0) * 0.030297521662727988;
    J(7, 8) = jc7;
    double sw = 0.0, dcv = 0.0;  // sum_k (c_p,k/R - 1) w_k, dc_v/dT / R
    sw += (th.cpR[0] - 1.0) * F[0] * rho * 0.49603174603174605;
    sw += (th.cpR[1] - 1.0) * F[1] * rho * 0.9920634920634921;
    sw += (th.cpR[2] - 1.0) * F[2] * rho * 0.03125195324707794;
    sw += (th.cpR[3] - 1.0) * F[3] * rho * 0.06250390649415588;
    sw += (th.cpR[4] - 1.0) * F[4] * rho * 0.055509297807382736;
    sw += (th.cpR[5] - 1.0) * F[5] * rho * 0.05879931792791203;
    sw += (th.cpR[6] - 1.0) * F[6] * rho * 0.029399658963956014;
    sw += (th.cpR[7] - 1.0) * F[7] * rho * 0.030297521662727988;
    sw += (th.cpR[8] - 1.0) * F[8] * rho * 0.03569643749553795;
    if (T < 1000.0) {
        dcv += y[0] * 0.49603174603174605 * (0.00773916922 + T * (-3.77470146e-05 + T * (5.86551342e-08 + T * -2.868382652e-11)));
        dcv += y[1] * 0.9920634920634921 * (6.73824499e-07 + T * (2.23614522e-09 + T * (-1.1105763779999999e-11 + T * 8.56935288e-15)));
        dcv += y[2] * 0.03125195324707794 * (-0.00302002233 + T * (1.984058342e-05 + T * (-2.9335213020000002e-08 + T * 1.315510808e-11)));
        dcv += y[3] * 0.06250390649415588 * (-0.00321509999 + T * (1.298511086e-05 + T * (-1.796265345e-08 + T * 8.27504468e-12)));
        dcv += y[4] * 0.055509297807382736 * (-0.00205583546 + T * (1.313094414e-05 + T * (-1.6587208800000002e-08 + T * 7.1313042e-12)));
        dcv += y[5] * 0.05879931792791203 * (-0.00228555291 + T * (8.66885764e-06 + T * (-1.0797799199999999e-08 + T * 5.0682772e-12)));
        dcv += y[6] * 0.029399658963956014 * (-0.000249610911 + T * (3.19715802e-05 + T * (-6.20759835e-08 + T * 3.31906528e-11)));
        dcv += y[7] * 0.030297521662727988 * (-0.00445642032 + T * (4.10329868e-05 + T * (-7.07382033e-08 + T * 3.622457028e-11)));
        dcv += y[8] * 0.03569643749553795 * (-0.000158270944 + T * (-8.53968502e-07 + T * (7.1262777e-09 + T * -5.58832824e-12)));
    } else {
        dcv += y[0] * 0.49603174603174605 * (0.000868992581 + T * (-3.3172886e-07 + T * (5.72555697e-11 + T * -3.724487156e-15)));
        dcv += y[1] * 0.9920634920634921 * (2.34582548e-07 + T * (-2.32343282e-10 + T * (6.771248940000001e-14 + T * -6.1196802e-18)));
        dcv += y[2] * 0.03125195324707794 * (0.000659877372 + T * (-2.88316344e-07 + T * (6.43968111e-11 + T * -5.46015136e-15)));
        dcv += y[3] * 0.06250390649415588 * (-3.83085457e-05 + T * (1.686394956e-09 + T * (1.203801408e-11 + T * -1.669906296e-15)));
        dcv += y[4] * 0.055509297807382736 * (0.00295136995 + T * (-1.67071957e-06 + T * (3.7826577900000005e-10 + T * -3.362126704e-14)));
        dcv += y[5] * 0.05879931792791203 * (0.00109723818 + T * (-5.78242202e-07 + T * (1.22729973e-10 + T * -9.25529032e-15)));
        dcv += y[6] * 0.029399658963956014 * (0.00415970971 + T * (-2.61753554e-06 + T * (6.02470845e-10 + T * -4.62036972e-14)));
        dcv += y[7] * 0.030297521662727988 * (0.00204046836 + T * (-7.31755124e-07 + T * (5.57919132e-11 + T * 1.99527326e-15)));
        dcv += y[8] * 0.03569643749553795 * (0.0014183803 + T * (-1.00656209e-06 + T * (2.422666392e-10 + T * -1.9042571e-14)));
    }
    J(8, 8) = s * (-8314.46261815324 * (sw + T * sum_eT) / (rho * cv) - F[9] * 8314.46261815324 * dcv / cv);
}

// The integrator's kinetics policy (gas::ros2_advance_km): thermo once per temperature,
// the right-hand side with the analytic Jacobian at the sub-step's start, the right-hand
// side alone at its second stage.
struct Kinetics {
    using K = Thermo;
    static constexpr bool kAnalyticJacobian = true;
    static constexpr int kSys = 9;  // unknowns of the iteration system
    GAS_HD static constexpr int sys_full(int i) { return i == 0 ? 0 : (i == 1 ? 1 : (i == 2 ? 2 : (i == 3 ? 3 : (i == 4 ? 4 : (i == 5 ? 5 : (i == 6 ? 6 : (i == 7 ? 7 : (9)))))))); }
    GAS_HD void factors(double T, Thermo &k) const { thermo(T, k); }
    GAS_HD void rhs(const Thermo &k, double rho, const double *y, double *F) const { rhs_t(k, rho, y, F); }
    template <class Mat>
    GAS_HD void rhs_jacobian(const Thermo &k, double rho, const double *y, double *F, double s, Mat &J) const {
        rhs_jac(k, rho, y, F, s, J);
    }
};

}  // namespace kin_h2_air_9
