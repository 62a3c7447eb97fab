// Generated by gen_kinetics.py from the mechanism h2_air_9 -- do not edit; `make` regenerates it.
// Its kinetics as straight-line code: gas.cuh's rate_factors (factors) and reactor_rhs_k
// (rhs_k) with the mechanism's constants inlined.
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
    if (m.reac[0][0] != 0 || m.nu_reac[0][0] != 1.0) return false;
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
    if (m.reac[1][0] != 0 || m.nu_reac[1][0] != 1.0) return false;
    if (m.reac[1][1] != 3 || m.nu_reac[1][1] != 1.0) return false;
    if (m.prod[1][0] != 1 || m.nu_prod[1][0] != 1.0) return false;
    if (m.prod[1][1] != 5 || m.nu_prod[1][1] != 1.0) return false;
    if (m.A[1] != 50.80000000000001 || m.b[1] != 2.67 || m.Ea[1] != 26325728.0) return false;
    if (m.rtype[2] != 0 || m.reversible[2] != 1 || m.n_reac[2] != 2 || m.n_prod[2] != 2) return false;
    if (m.reac[2][0] != 0 || m.nu_reac[2][0] != 1.0) return false;
    if (m.reac[2][1] != 5 || m.nu_reac[2][1] != 1.0) return false;
    if (m.prod[2][0] != 1 || m.nu_prod[2][0] != 1.0) return false;
    if (m.prod[2][1] != 4 || m.nu_prod[2][1] != 1.0) return false;
    if (m.A[2] != 43800000000.00001 || m.b[2] != 0.0 || m.Ea[2] != 29246160.0) return false;
    if (m.rtype[3] != 1 || m.reversible[3] != 1 || m.n_reac[3] != 1 || m.n_prod[3] != 1) return false;
    if (m.reac[3][0] != 3 || m.nu_reac[3][0] != 2.0) return false;
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
    if (m.reac[4][0] != 2 || m.nu_reac[4][0] != 1.0) return false;
    if (m.reac[4][1] != 1 || m.nu_reac[4][1] != 1.0) return false;
    if (m.prod[4][0] != 3 || m.nu_prod[4][0] != 1.0) return false;
    if (m.prod[4][1] != 5 || m.nu_prod[4][1] != 1.0) return false;
    if (m.A[4] != 114000000000.00003 || m.b[4] != 0.0 || m.Ea[4] != 63956624.0) return false;
    if (m.rtype[5] != 1 || m.reversible[5] != 1 || m.n_reac[5] != 2 || m.n_prod[5] != 1) return false;
    if (m.reac[5][0] != 1 || m.nu_reac[5][0] != 1.0) return false;
    if (m.reac[5][1] != 5 || m.nu_reac[5][1] != 1.0) return false;
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
    if (m.reac[6][0] != 3 || m.nu_reac[6][0] != 1.0) return false;
    if (m.reac[6][1] != 4 || m.nu_reac[6][1] != 1.0) return false;
    if (m.prod[6][0] != 5 || m.nu_prod[6][0] != 2.0) return false;
    if (m.A[6] != 67000.00000000001 || m.b[6] != 1.704 || m.Ea[6] != 62704771.199999996) return false;
    if (m.rtype[7] != 1 || m.reversible[7] != 1 || m.n_reac[7] != 2 || m.n_prod[7] != 1) return false;
    if (m.reac[7][0] != 3 || m.nu_reac[7][0] != 1.0) return false;
    if (m.reac[7][1] != 1 || m.nu_reac[7][1] != 1.0) return false;
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
    if (m.reac[8][0] != 6 || m.nu_reac[8][0] != 1.0) return false;
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
    if (m.reac[9][0] != 6 || m.nu_reac[9][0] != 1.0) return false;
    if (m.reac[9][1] != 1 || m.nu_reac[9][1] != 1.0) return false;
    if (m.prod[9][0] != 4 || m.nu_prod[9][0] != 1.0) return false;
    if (m.prod[9][1] != 5 || m.nu_prod[9][1] != 1.0) return false;
    if (m.A[9] != 24100000000.000008 || m.b[9] != 0.0 || m.Ea[9] != 16610480.0) return false;
    if (m.rtype[10] != 0 || m.reversible[10] != 1 || m.n_reac[10] != 2 || m.n_prod[10] != 2) return false;
    if (m.reac[10][0] != 6 || m.nu_reac[10][0] != 1.0) return false;
    if (m.reac[10][1] != 1 || m.nu_reac[10][1] != 1.0) return false;
    if (m.prod[10][0] != 0 || m.nu_prod[10][0] != 1.0) return false;
    if (m.prod[10][1] != 7 || m.nu_prod[10][1] != 1.0) return false;
    if (m.A[10] != 21500000.000000004 || m.b[10] != 1.0 || m.Ea[10] != 25104000.0) return false;
    if (m.rtype[11] != 0 || m.reversible[11] != 1 || m.n_reac[11] != 2 || m.n_prod[11] != 2) return false;
    if (m.reac[11][0] != 6 || m.nu_reac[11][0] != 1.0) return false;
    if (m.reac[11][1] != 3 || m.nu_reac[11][1] != 1.0) return false;
    if (m.prod[11][0] != 5 || m.nu_prod[11][0] != 1.0) return false;
    if (m.prod[11][1] != 7 || m.nu_prod[11][1] != 1.0) return false;
    if (m.A[11] != 9550.000000000002 || m.b[11] != 2.0 || m.Ea[11] != 16610480.0) return false;
    if (m.rtype[12] != 0 || m.reversible[12] != 1 || m.n_reac[12] != 2 || m.n_prod[12] != 2) return false;
    if (m.reac[12][0] != 6 || m.nu_reac[12][0] != 1.0) return false;
    if (m.reac[12][1] != 5 || m.nu_reac[12][1] != 1.0) return false;
    if (m.prod[12][0] != 4 || m.nu_prod[12][0] != 1.0) return false;
    if (m.prod[12][1] != 7 || m.nu_prod[12][1] != 1.0) return false;
    if (m.A[12] != 1740000000.0000005 || m.b[12] != 0.0 || m.Ea[12] != 1330512.0) return false;
    if (m.rtype[13] != 0 || m.reversible[13] != 1 || m.n_reac[13] != 2 || m.n_prod[13] != 2) return false;
    if (m.reac[13][0] != 6 || m.nu_reac[13][0] != 1.0) return false;
    if (m.reac[13][1] != 5 || m.nu_reac[13][1] != 1.0) return false;
    if (m.prod[13][0] != 4 || m.nu_prod[13][0] != 1.0) return false;
    if (m.prod[13][1] != 7 || m.nu_prod[13][1] != 1.0) return false;
    if (m.A[13] != 75900000000.00002 || m.b[13] != 0.0 || m.Ea[13] != 30413496.0) return false;
    if (m.rtype[14] != 0 || m.reversible[14] != 1 || m.n_reac[14] != 2 || m.n_prod[14] != 1) return false;
    if (m.reac[14][0] != 7 || m.nu_reac[14][0] != 1.0) return false;
    if (m.reac[14][1] != 1 || m.nu_reac[14][1] != 1.0) return false;
    if (m.prod[14][0] != 5 || m.nu_prod[14][0] != 2.0) return false;
    if (m.A[14] != 70790000000.00002 || m.b[14] != 0.0 || m.Ea[14] != 1234280.0) return false;
    if (m.rtype[15] != 0 || m.reversible[15] != 1 || m.n_reac[15] != 2 || m.n_prod[15] != 2) return false;
    if (m.reac[15][0] != 7 || m.nu_reac[15][0] != 1.0) return false;
    if (m.reac[15][1] != 1 || m.nu_reac[15][1] != 1.0) return false;
    if (m.prod[15][0] != 0 || m.nu_prod[15][0] != 1.0) return false;
    if (m.prod[15][1] != 2 || m.nu_prod[15][1] != 1.0) return false;
    if (m.A[15] != 11402000.000000002 || m.b[15] != 1.0827 || m.Ea[15] != 2317015.52) return false;
    if (m.rtype[16] != 0 || m.reversible[16] != 1 || m.n_reac[16] != 2 || m.n_prod[16] != 2) return false;
    if (m.reac[16][0] != 7 || m.nu_reac[16][0] != 1.0) return false;
    if (m.reac[16][1] != 3 || m.nu_reac[16][1] != 1.0) return false;
    if (m.prod[16][0] != 5 || m.nu_prod[16][0] != 1.0) return false;
    if (m.prod[16][1] != 2 || m.nu_prod[16][1] != 1.0) return false;
    if (m.A[16] != 32500000000.000008 || m.b[16] != 0.0 || m.Ea[16] != 0.0) return false;
    if (m.rtype[17] != 0 || m.reversible[17] != 1 || m.n_reac[17] != 2 || m.n_prod[17] != 2) return false;
    if (m.reac[17][0] != 5 || m.nu_reac[17][0] != 1.0) return false;
    if (m.reac[17][1] != 7 || m.nu_reac[17][1] != 1.0) return false;
    if (m.prod[17][0] != 4 || m.nu_prod[17][0] != 1.0) return false;
    if (m.prod[17][1] != 2 || m.nu_prod[17][1] != 1.0) return false;
    if (m.A[17] != 7000000000.000002 || m.b[17] != 0.0 || m.Ea[17] != -4572944.640000001) return false;
    if (m.rtype[18] != 0 || m.reversible[18] != 1 || m.n_reac[18] != 2 || m.n_prod[18] != 2) return false;
    if (m.reac[18][0] != 5 || m.nu_reac[18][0] != 1.0) return false;
    if (m.reac[18][1] != 7 || m.nu_reac[18][1] != 1.0) return false;
    if (m.prod[18][0] != 4 || m.nu_prod[18][0] != 1.0) return false;
    if (m.prod[18][1] != 2 || m.nu_prod[18][1] != 1.0) return false;
    if (m.A[18] != 450000000000.0001 || m.b[18] != 0.0 || m.Ea[18] != 45729446.4) return false;
    if (m.rtype[19] != 0 || m.reversible[19] != 1 || m.n_reac[19] != 1 || m.n_prod[19] != 2) return false;
    if (m.reac[19][0] != 7 || m.nu_reac[19][0] != 2.0) return false;
    if (m.prod[19][0] != 6 || m.nu_prod[19][0] != 1.0) return false;
    if (m.prod[19][1] != 2 || m.nu_prod[19][1] != 1.0) return false;
    if (m.A[19] != 100000000000.00003 || m.b[19] != 0.0 || m.Ea[19] != 46195054.472) return false;
    if (m.rtype[20] != 0 || m.reversible[20] != 1 || m.n_reac[20] != 1 || m.n_prod[20] != 2) return false;
    if (m.reac[20][0] != 7 || m.nu_reac[20][0] != 2.0) return false;
    if (m.prod[20][0] != 6 || m.nu_prod[20][0] != 1.0) return false;
    if (m.prod[20][1] != 2 || m.nu_prod[20][1] != 1.0) return false;
    if (m.A[20] != 190000000.00000006 || m.b[20] != 0.0 || m.Ea[20] != -5894941.3632) return false;
    if (m.rtype[21] != 2 || m.reversible[21] != 1 || m.n_reac[21] != 2 || m.n_prod[21] != 1) return false;
    if (m.reac[21][0] != 1 || m.nu_reac[21][0] != 1.0) return false;
    if (m.reac[21][1] != 2 || m.nu_reac[21][1] != 1.0) return false;
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
    if (m.reac[22][0] != 3 || m.nu_reac[22][0] != 1.0) return false;
    if (m.reac[22][1] != 5 || m.nu_reac[22][1] != 1.0) return false;
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

// The temperature-only factors (gas::RateT): k_inf (k for non-fall-off reactions), the
// fall-off k_0 and log10 F_cent, the reverse factors exp(dG/RT - dnu ln(p_atm / R T)) and
// the species' h/RT and c_p/R.
struct Factors {
    double kf[NR], er[NR], k0[NF], lFc[NF], hRT[NS], cpR[NS];
};

GAS_HD void factors(double T, Factors &K) {
    const double logT = log(T), invRT = 1.0 / (8314.46261815324 * T);
    const double log_cref = log(101325.0 / (8314.46261815324 * T));
    double gRT[9];
    if (T < 1000.0) {
        K.cpR[0] = 2.37694204 + T * (0.00773916922 + T * (-1.88735073e-05 + T * (1.95517114e-08 + T * -7.17095663e-12)));
        K.hRT[0] = 2.37694204 + T * (0.00386958461 + T * (-6.291169099999999e-06 + T * (4.88792785e-09 + T * -7.17095663e-12 / 5.0))) + -921.173081 / T;
        gRT[0] = K.hRT[0] - (2.37694204 * logT + T * (0.00773916922 + T * (-9.43675365e-06 + T * (6.517237133333333e-09 + T * -1.7927391575e-12))) + 0.547184736);
        K.cpR[1] = 2.49975925 + T * (6.73824499e-07 + T * (1.11807261e-09 + T * (-3.70192126e-12 + T * 2.14233822e-15)));
        K.hRT[1] = 2.49975925 + T * (3.369122495e-07 + T * (3.7269087000000003e-10 + T * (-9.25480315e-13 + T * 2.14233822e-15 / 5.0))) + 25473.7665 / T;
        gRT[1] = K.hRT[1] - (2.49975925 * logT + T * (6.73824499e-07 + T * (5.59036305e-10 + T * (-1.2339737533333333e-12 + T * 5.35584555e-16))) + -0.445574009);
        K.cpR[2] = 3.78498258 + T * (-0.00302002233 + T * (9.92029171e-06 + T * (-9.77840434e-09 + T * 3.28877702e-12)));
        K.hRT[2] = 3.78498258 + T * (-0.001510011165 + T * (3.3067639033333336e-06 + T * (-2.444601085e-09 + T * 3.28877702e-12 / 5.0))) + -1064.13589 / T;
        gRT[2] = K.hRT[2] - (3.78498258 * logT + T * (-0.00302002233 + T * (4.960145855e-06 + T * (-3.2594681133333337e-09 + T * 8.22194255e-13))) + 3.64780709);
        K.cpR[3] = 3.15906526 + T * (-0.00321509999 + T * (6.49255543e-06 + T * (-5.98755115e-09 + T * 2.06876117e-12)));
        K.hRT[3] = 3.15906526 + T * (-0.001607549995 + T * (2.1641851433333333e-06 + T * (-1.4968877875e-09 + T * 2.06876117e-12 / 5.0))) + 29129.8453 / T;
        gRT[3] = K.hRT[3] - (3.15906526 * logT + T * (-0.00321509999 + T * (3.246277715e-06 + T * (-1.995850383333333e-09 + T * 5.171902925e-13))) + 2.09078344);
        K.cpR[4] = 4.20147551 + T * (-0.00205583546 + T * (6.56547207e-06 + T * (-5.5290696e-09 + T * 1.78282605e-12)));
        K.hRT[4] = 4.20147551 + T * (-0.00102791773 + T * (2.1884906899999998e-06 + T * (-1.3822674e-09 + T * 1.78282605e-12 / 5.0))) + -30295.0066 / T;
        gRT[4] = K.hRT[4] - (4.20147551 * logT + T * (-0.00205583546 + T * (3.282736035e-06 + T * (-1.8430232e-09 + T * 4.457065125e-13))) + -0.860610906);
        K.cpR[5] = 3.97585165 + T * (-0.00228555291 + T * (4.33442882e-06 + T * (-3.5992664e-09 + T * 1.2670693e-12)));
        K.hRT[5] = 3.97585165 + T * (-0.001142776455 + T * (1.4448096066666668e-06 + T * (-8.998166e-10 + T * 1.2670693e-12 / 5.0))) + 3393.41137 / T;
        gRT[5] = K.hRT[5] - (3.97585165 * logT + T * (-0.00228555291 + T * (2.16721441e-06 + T * (-1.1997554666666665e-09 + T * 3.16767325e-13))) + -0.0355397262);
        K.cpR[6] = 4.2385416 + T * (-0.000249610911 + T * (1.59857901e-05 + T * (-2.06919945e-08 + T * 8.2976632e-12)));
        K.hRT[6] = 4.2385416 + T * (-0.0001248054555 + T * (5.3285966999999996e-06 + T * (-5.172998625e-09 + T * 8.2976632e-12 / 5.0))) + -17648.6003 / T;
        gRT[6] = K.hRT[6] - (4.2385416 * logT + T * (-0.000249610911 + T * (7.99289505e-06 + T * (-6.8973315e-09 + T * 2.0744158e-12))) + 3.58850097);
        K.cpR[7] = 4.2625125 + T * (-0.00445642032 + T * (2.05164934e-05 + T * (-2.35794011e-08 + T * 9.05614257e-12)));
        K.hRT[7] = 4.2625125 + T * (-0.00222821016 + T * (6.8388311333333335e-06 + T * (-5.894850275e-09 + T * 9.05614257e-12 / 5.0))) + 262.442356 / T;
        gRT[7] = K.hRT[7] - (4.2625125 * logT + T * (-0.00445642032 + T * (1.02582467e-05 + T * (-7.859800366666666e-09 + T * 2.2640356425e-12))) + 3.88223684);
        K.cpR[8] = 3.53603521 + T * (-0.000158270944 + T * (-4.26984251e-07 + T * (2.3754259e-09 + T * -1.39708206e-12)));
        K.hRT[8] = 3.53603521 + T * (-7.9135472e-05 + T * (-1.4232808366666666e-07 + T * (5.93856475e-10 + T * -1.39708206e-12 / 5.0))) + -1047.49645 / T;
        gRT[8] = K.hRT[8] - (3.53603521 * logT + T * (-0.000158270944 + T * (-2.134921255e-07 + T * (7.918086333333333e-10 + T * -3.49270515e-13))) + 2.94603724);
    } else {
        K.cpR[0] = 2.90207649 + T * (0.000868992581 + T * (-1.6586443e-07 + T * (1.90851899e-11 + T * -9.31121789e-16)));
        K.hRT[0] = 2.90207649 + T * (0.0004344962905 + T * (-5.5288143333333333e-08 + T * (4.771297475e-12 + T * -9.31121789e-16 / 5.0))) + -797.948726 / T;
        gRT[0] = K.hRT[0] - (2.90207649 * logT + T * (0.000868992581 + T * (-8.2932215e-08 + T * (6.361729966666667e-12 + T * -2.3278044725e-16))) + -0.84559132);
        K.cpR[1] = 2.49985211 + T * (2.34582548e-07 + T * (-1.16171641e-10 + T * (2.25708298e-14 + T * -1.52992005e-18)));
        K.hRT[1] = 2.49985211 + T * (1.17291274e-07 + T * (-3.8723880333333334e-11 + T * (5.64270745e-15 + T * -1.52992005e-18 / 5.0))) + 25473.8024 / T;
        gRT[1] = K.hRT[1] - (2.49985211 * logT + T * (2.34582548e-07 + T * (-5.80858205e-11 + T * (7.523609933333334e-15 + T * -3.824800125e-19))) + -0.445864645);
        K.cpR[2] = 3.65980488 + T * (0.000659877372 + T * (-1.44158172e-07 + T * (2.14656037e-11 + T * -1.36503784e-15)));
        K.hRT[2] = 3.65980488 + T * (0.000329938686 + T * (-4.8052724e-08 + T * (5.366400925e-12 + T * -1.36503784e-15 / 5.0))) + -1216.03048 / T;
        gRT[2] = K.hRT[2] - (3.65980488 * logT + T * (0.000659877372 + T * (-7.2079086e-08 + T * (7.155201233333333e-12 + T * -3.4125946e-16))) + 3.42074148);
        K.cpR[3] = 2.55160087 + T * (-3.83085457e-05 + T * (8.43197478e-10 + T * (4.01267136e-12 + T * -4.17476574e-16)));
        K.hRT[3] = 2.55160087 + T * (-1.915427285e-05 + T * (2.81065826e-10 + T * (1.00316784e-12 + T * -4.17476574e-16 / 5.0))) + 29228.7628 / T;
        gRT[3] = K.hRT[3] - (2.55160087 * logT + T * (-3.83085457e-05 + T * (4.21598739e-10 + T * (1.33755712e-12 + T * -1.043691435e-16))) + 4.87617014);
        K.cpR[4] = 2.73117512 + T * (0.00295136995 + T * (-8.35359785e-07 + T * (1.26088593e-10 + T * -8.40531676e-15)));
        K.hRT[4] = 2.73117512 + T * (0.001475684975 + T * (-2.784532616666667e-07 + T * (3.152214825e-11 + T * -8.40531676e-15 / 5.0))) + -29916.9082 / T;
        gRT[4] = K.hRT[4] - (2.73117512 * logT + T * (0.00295136995 + T * (-4.176798925e-07 + T * (4.2029531e-11 + T * -2.10132919e-15))) + 6.55183);
        K.cpR[5] = 2.84581721 + T * (0.00109723818 + T * (-2.89121101e-07 + T * (4.0909991e-11 + T * -2.31382258e-15)));
        K.hRT[5] = 2.84581721 + T * (0.00054861909 + T * (-9.637370033333334e-08 + T * (1.022749775e-11 + T * -2.31382258e-15 / 5.0))) + 3717.0661 / T;
        gRT[5] = K.hRT[5] - (2.84581721 * logT + T * (0.00109723818 + T * (-1.445605505e-07 + T * (1.3636663666666666e-11 + T * -5.78455645e-16))) + 5.80339915);
        K.cpR[6] = 4.5401748 + T * (0.00415970971 + T * (-1.30876777e-06 + T * (2.00823615e-10 + T * -1.15509243e-14)));
        K.hRT[6] = 4.5401748 + T * (0.002079854855 + T * (-4.3625592333333335e-07 + T * (5.020590375e-11 + T * -1.15509243e-14 / 5.0))) + -17951.4029 / T;
        gRT[6] = K.hRT[6] - (4.5401748 * logT + T * (0.00415970971 + T * (-6.54383885e-07 + T * (6.694120500000001e-11 + T * -2.887731075e-15))) + 0.855881745);
        K.cpR[7] = 4.1056401 + T * (0.00204046836 + T * (-3.65877562e-07 + T * (1.85973044e-11 + T * 4.98818315e-16)));
        K.hRT[7] = 4.1056401 + T * (0.00102023418 + T * (-1.2195918733333333e-07 + T * (4.6493261e-12 + T * 4.98818315e-16 / 5.0))) + 43.2898769 / T;
        gRT[7] = K.hRT[7] - (4.1056401 * logT + T * (0.00204046836 + T * (-1.82938781e-07 + T * (6.199101466666667e-12 + T * 1.2470457875e-16))) + 3.30808126);
        K.cpR[8] = 2.9380297 + T * (0.0014183803 + T * (-5.03281045e-07 + T * (8.07555464e-11 + T * -4.76064275e-15)));
        K.hRT[8] = 2.9380297 + T * (0.00070919015 + T * (-1.6776034833333333e-07 + T * (2.01888866e-11 + T * -4.76064275e-15 / 5.0))) + -917.18099 / T;
        gRT[8] = K.hRT[8] - (2.9380297 * logT + T * (0.0014183803 + T * (-2.516405225e-07 + T * (2.6918515466666668e-11 + T * -1.1901606875e-15))) + 5.95521985);
    }
    K.kf[0] = 4.577000000000001e+16 * exp(-1.4 * logT - 436809600.0 * invRT);
    K.er[0] = exp((2.0 * gRT[1] - gRT[0]) - 1.0 * log_cref);
    K.kf[1] = 50.80000000000001 * exp(2.67 * logT - 26325728.0 * invRT);
    K.er[1] = exp(gRT[1] + gRT[5] - gRT[0] - gRT[3]);
    K.kf[2] = 43800000000.00001 * exp(-(29246160.0 * invRT));
    K.er[2] = exp(gRT[1] + gRT[4] - gRT[0] - gRT[5]);
    K.kf[3] = 6165000000.000002 * exp(-0.5 * logT);
    K.er[3] = exp((gRT[2] - 2.0 * gRT[3]) - -1.0 * log_cref);
    K.kf[4] = 114000000000.00003 * exp(-(63956624.0 * invRT));
    K.er[4] = exp(gRT[3] + gRT[5] - gRT[2] - gRT[1]);
    K.kf[5] = 3.5000000000000016e+16 * exp(-2.0 * logT);
    K.er[5] = exp((gRT[4] - gRT[1] - gRT[5]) - -1.0 * log_cref);
    K.kf[6] = 67000.00000000001 * exp(1.704 * logT - 62704771.199999996 * invRT);
    K.er[6] = exp(2.0 * gRT[5] - gRT[3] - gRT[4]);
    K.kf[7] = 4714000000000.002 * exp(-1.0 * logT);
    K.er[7] = exp((gRT[5] - gRT[3] - gRT[1]) - -1.0 * log_cref);
    K.kf[8] = 2000000000000.0 * exp(0.9 * logT - 203965816.0 * invRT);
    K.k0[0] = 2.4900000000000005e+21 * exp(-2.3 * logT - 203965816.0 * invRT);
    {
        double Fc = 0.5700000000000001 * exp(-T / 1e-30) + 0.43 * exp(-T / 1e+30);
        K.lFc[0] = log10(fmax(Fc, 1e-300));
    }
    K.er[8] = exp((2.0 * gRT[5] - gRT[6]) - 1.0 * log_cref);
    K.kf[9] = 24100000000.000008 * exp(-(16610480.0 * invRT));
    K.er[9] = exp(gRT[4] + gRT[5] - gRT[6] - gRT[1]);
    K.kf[10] = 21500000.000000004 * exp(1.0 * logT - 25104000.0 * invRT);
    K.er[10] = exp(gRT[0] + gRT[7] - gRT[6] - gRT[1]);
    K.kf[11] = 9550.000000000002 * exp(2.0 * logT - 16610480.0 * invRT);
    K.er[11] = exp(gRT[5] + gRT[7] - gRT[6] - gRT[3]);
    K.kf[12] = 1740000000.0000005 * exp(-(1330512.0 * invRT));
    K.er[12] = exp(gRT[4] + gRT[7] - gRT[6] - gRT[5]);
    K.kf[13] = 75900000000.00002 * exp(-(30413496.0 * invRT));
    K.er[13] = exp(gRT[4] + gRT[7] - gRT[6] - gRT[5]);
    K.kf[14] = 70790000000.00002 * exp(-(1234280.0 * invRT));
    K.er[14] = exp(2.0 * gRT[5] - gRT[7] - gRT[1]);
    K.kf[15] = 11402000.000000002 * exp(1.0827 * logT - 2317015.52 * invRT);
    K.er[15] = exp(gRT[0] + gRT[2] - gRT[7] - gRT[1]);
    K.kf[16] = 32500000000.000008;
    K.er[16] = exp(gRT[5] + gRT[2] - gRT[7] - gRT[3]);
    K.kf[17] = 7000000000.000002 * exp(-(-4572944.640000001 * invRT));
    K.er[17] = exp(gRT[4] + gRT[2] - gRT[5] - gRT[7]);
    K.kf[18] = 450000000000.0001 * exp(-(45729446.4 * invRT));
    K.er[18] = exp(gRT[4] + gRT[2] - gRT[5] - gRT[7]);
    K.kf[19] = 100000000000.00003 * exp(-(46195054.472 * invRT));
    K.er[19] = exp(gRT[6] + gRT[2] - 2.0 * gRT[7]);
    K.kf[20] = 190000000.00000006 * exp(-(-5894941.3632 * invRT));
    K.er[20] = exp(gRT[6] + gRT[2] - 2.0 * gRT[7]);
    K.kf[21] = 4650000000.000001 * exp(0.44 * logT);
    K.k0[1] = 17370000000000.006 * exp(-1.23 * logT);
    {
        double Fc = 0.32999999999999996 * exp(-T / 1e-30) + 0.67 * exp(-T / 1e+30);
        Fc += exp(-1e+30 / T);
        K.lFc[1] = log10(fmax(Fc, 1e-300));
    }
    K.er[21] = exp((gRT[7] - gRT[1] - gRT[2]) - -1.0 * log_cref);
    K.kf[22] = 10000000000.000004;
    K.er[22] = exp((gRT[7] - gRT[3] - gRT[5]) - -1.0 * log_cref);
}

// F = d(Y_0..Y_{NS-1}, T)/dt at density rho [kg/m^3] and state y, from the factors K at
// y's temperature (gas::reactor_rhs_k).
GAS_HD void rhs_k(const Factors &K, double rho, const double *y, double *F) {
    const double T = y[9];
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
    {  // 0: 1 H2 <=> 2 H  + M
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[0] * M;
        const double fwd = kfM * C0;
        const double rev = kfM * K.er[0] * (C1 * C1);
        const double q = fwd - rev;
        w0 -= q;
        w1 += 2.0 * q;
    }
    {  // 1: 1 H2 + 1 O <=> 1 H + 1 OH
        const double kfM = K.kf[1];
        const double fwd = kfM * C0 * C3;
        const double rev = kfM * K.er[1] * C1 * C5;
        const double q = fwd - rev;
        w0 -= q;
        w3 -= q;
        w1 += q;
        w5 += q;
    }
    {  // 2: 1 H2 + 1 OH <=> 1 H + 1 H2O
        const double kfM = K.kf[2];
        const double fwd = kfM * C0 * C5;
        const double rev = kfM * K.er[2] * C1 * C4;
        const double q = fwd - rev;
        w0 -= q;
        w5 -= q;
        w1 += q;
        w4 += q;
    }
    {  // 3: 2 O <=> 1 O2  + M
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[3] * M;
        const double fwd = kfM * (C3 * C3);
        const double rev = kfM * K.er[3] * C2;
        const double q = fwd - rev;
        w3 -= 2.0 * q;
        w2 += q;
    }
    {  // 4: 1 O2 + 1 H <=> 1 O + 1 OH
        const double kfM = K.kf[4];
        const double fwd = kfM * C2 * C1;
        const double rev = kfM * K.er[4] * C3 * C5;
        const double q = fwd - rev;
        w2 -= q;
        w1 -= q;
        w3 += q;
        w5 += q;
    }
    {  // 5: 1 H + 1 OH <=> 1 H2O  + M
        const double M = 0.73 * C0 + C1 + C2 + C3 + 3.65 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[5] * M;
        const double fwd = kfM * C1 * C5;
        const double rev = kfM * K.er[5] * C4;
        const double q = fwd - rev;
        w1 -= q;
        w5 -= q;
        w4 += q;
    }
    {  // 6: 1 O + 1 H2O <=> 2 OH
        const double kfM = K.kf[6];
        const double fwd = kfM * C3 * C4;
        const double rev = kfM * K.er[6] * (C5 * C5);
        const double q = fwd - rev;
        w3 -= q;
        w4 -= q;
        w5 += 2.0 * q;
    }
    {  // 7: 1 O + 1 H <=> 1 OH  + M
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[7] * M;
        const double fwd = kfM * C3 * C1;
        const double rev = kfM * K.er[7] * C5;
        const double q = fwd - rev;
        w3 -= q;
        w1 -= q;
        w5 += q;
    }
    {  // 8: 1 H2O2 <=> 2 OH  (+M)
        const double M = 3.7 * C0 + C1 + 1.2 * C2 + C3 + 7.65 * C4 + C5 + 7.7 * C6 + C7 + 1.5 * C8;
        const double Pr = K.k0[0] * M / K.kf[8];
        const double lFc = K.lFc[0];
        const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
        const double lPr = log10(fmax(Pr, 1e-300));
        const double x = (lPr + c) / (n - 0.14 * (lPr + c));
        const double kfM = K.kf[8] * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
        const double fwd = kfM * C6;
        const double rev = kfM * K.er[8] * (C5 * C5);
        const double q = fwd - rev;
        w6 -= q;
        w5 += 2.0 * q;
    }
    {  // 9: 1 H2O2 + 1 H <=> 1 H2O + 1 OH
        const double kfM = K.kf[9];
        const double fwd = kfM * C6 * C1;
        const double rev = kfM * K.er[9] * C4 * C5;
        const double q = fwd - rev;
        w6 -= q;
        w1 -= q;
        w4 += q;
        w5 += q;
    }
    {  // 10: 1 H2O2 + 1 H <=> 1 H2 + 1 HO2
        const double kfM = K.kf[10];
        const double fwd = kfM * C6 * C1;
        const double rev = kfM * K.er[10] * C0 * C7;
        const double q = fwd - rev;
        w6 -= q;
        w1 -= q;
        w0 += q;
        w7 += q;
    }
    {  // 11: 1 H2O2 + 1 O <=> 1 OH + 1 HO2
        const double kfM = K.kf[11];
        const double fwd = kfM * C6 * C3;
        const double rev = kfM * K.er[11] * C5 * C7;
        const double q = fwd - rev;
        w6 -= q;
        w3 -= q;
        w5 += q;
        w7 += q;
    }
    {  // 12: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
        const double kfM = K.kf[12];
        const double fwd = kfM * C6 * C5;
        const double rev = kfM * K.er[12] * C4 * C7;
        const double q = fwd - rev;
        w6 -= q;
        w5 -= q;
        w4 += q;
        w7 += q;
    }
    {  // 13: 1 H2O2 + 1 OH <=> 1 H2O + 1 HO2
        const double kfM = K.kf[13];
        const double fwd = kfM * C6 * C5;
        const double rev = kfM * K.er[13] * C4 * C7;
        const double q = fwd - rev;
        w6 -= q;
        w5 -= q;
        w4 += q;
        w7 += q;
    }
    {  // 14: 1 HO2 + 1 H <=> 2 OH
        const double kfM = K.kf[14];
        const double fwd = kfM * C7 * C1;
        const double rev = kfM * K.er[14] * (C5 * C5);
        const double q = fwd - rev;
        w7 -= q;
        w1 -= q;
        w5 += 2.0 * q;
    }
    {  // 15: 1 HO2 + 1 H <=> 1 H2 + 1 O2
        const double kfM = K.kf[15];
        const double fwd = kfM * C7 * C1;
        const double rev = kfM * K.er[15] * C0 * C2;
        const double q = fwd - rev;
        w7 -= q;
        w1 -= q;
        w0 += q;
        w2 += q;
    }
    {  // 16: 1 HO2 + 1 O <=> 1 OH + 1 O2
        const double kfM = K.kf[16];
        const double fwd = kfM * C7 * C3;
        const double rev = kfM * K.er[16] * C5 * C2;
        const double q = fwd - rev;
        w7 -= q;
        w3 -= q;
        w5 += q;
        w2 += q;
    }
    {  // 17: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
        const double kfM = K.kf[17];
        const double fwd = kfM * C5 * C7;
        const double rev = kfM * K.er[17] * C4 * C2;
        const double q = fwd - rev;
        w5 -= q;
        w7 -= q;
        w4 += q;
        w2 += q;
    }
    {  // 18: 1 OH + 1 HO2 <=> 1 H2O + 1 O2
        const double kfM = K.kf[18];
        const double fwd = kfM * C5 * C7;
        const double rev = kfM * K.er[18] * C4 * C2;
        const double q = fwd - rev;
        w5 -= q;
        w7 -= q;
        w4 += q;
        w2 += q;
    }
    {  // 19: 2 HO2 <=> 1 H2O2 + 1 O2
        const double kfM = K.kf[19];
        const double fwd = kfM * (C7 * C7);
        const double rev = kfM * K.er[19] * C6 * C2;
        const double q = fwd - rev;
        w7 -= 2.0 * q;
        w6 += q;
        w2 += q;
    }
    {  // 20: 2 HO2 <=> 1 H2O2 + 1 O2
        const double kfM = K.kf[20];
        const double fwd = kfM * (C7 * C7);
        const double rev = kfM * K.er[20] * C6 * C2;
        const double q = fwd - rev;
        w7 -= 2.0 * q;
        w6 += q;
        w2 += q;
    }
    {  // 21: 1 H + 1 O2 <=> 1 HO2  (+M)
        const double M = 1.3 * C0 + C1 + C2 + C3 + 10.0 * C4 + C5 + C6 + C7 + C8;
        const double Pr = K.k0[1] * M / K.kf[21];
        const double lFc = K.lFc[1];
        const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
        const double lPr = log10(fmax(Pr, 1e-300));
        const double x = (lPr + c) / (n - 0.14 * (lPr + c));
        const double kfM = K.kf[21] * (Pr / (1.0 + Pr)) * pow(10.0, lFc / (1.0 + x * x));
        const double fwd = kfM * C1 * C2;
        const double rev = kfM * K.er[21] * C7;
        const double q = fwd - rev;
        w1 -= q;
        w2 -= q;
        w7 += q;
    }
    {  // 22: 1 O + 1 OH <=> 1 HO2  + M
        const double M = C0 + C1 + C2 + C3 + C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[22] * M;
        const double fwd = kfM * C3 * C5;
        const double rev = kfM * K.er[22] * C7;
        const double q = fwd - rev;
        w3 -= q;
        w5 -= q;
        w7 += q;
    }
    double cv = 0.0, s = 0.0;
    F[0] = w0 * 2.016 / rho;
    cv += y[0] * (K.cpR[0] - 1.0) * 0.49603174603174605;
    s += (K.hRT[0] - 1.0) * 8314.46261815324 * T * w0;
    F[1] = w1 * 1.008 / rho;
    cv += y[1] * (K.cpR[1] - 1.0) * 0.9920634920634921;
    s += (K.hRT[1] - 1.0) * 8314.46261815324 * T * w1;
    F[2] = w2 * 31.998 / rho;
    cv += y[2] * (K.cpR[2] - 1.0) * 0.03125195324707794;
    s += (K.hRT[2] - 1.0) * 8314.46261815324 * T * w2;
    F[3] = w3 * 15.999 / rho;
    cv += y[3] * (K.cpR[3] - 1.0) * 0.06250390649415588;
    s += (K.hRT[3] - 1.0) * 8314.46261815324 * T * w3;
    F[4] = w4 * 18.015 / rho;
    cv += y[4] * (K.cpR[4] - 1.0) * 0.055509297807382736;
    s += (K.hRT[4] - 1.0) * 8314.46261815324 * T * w4;
    F[5] = w5 * 17.007 / rho;
    cv += y[5] * (K.cpR[5] - 1.0) * 0.05879931792791203;
    s += (K.hRT[5] - 1.0) * 8314.46261815324 * T * w5;
    F[6] = w6 * 34.014 / rho;
    cv += y[6] * (K.cpR[6] - 1.0) * 0.029399658963956014;
    s += (K.hRT[6] - 1.0) * 8314.46261815324 * T * w6;
    F[7] = w7 * 33.006 / rho;
    cv += y[7] * (K.cpR[7] - 1.0) * 0.030297521662727988;
    s += (K.hRT[7] - 1.0) * 8314.46261815324 * T * w7;
    F[8] = w8 * 28.014 / rho;
    cv += y[8] * (K.cpR[8] - 1.0) * 0.03569643749553795;
    s += (K.hRT[8] - 1.0) * 8314.46261815324 * T * w8;
    cv *= 8314.46261815324;
    F[9] = -s / (rho * cv);
}

// The species columns of the Jacobian of F (rhs_k) with respect to (Y, T): J[k][j] =
// dF_k / dY_j for j < NS and every row k <= NS, at fixed temperature and density, from the
// factors at y's temperature and F = rhs_k(K, rho, y).  Column NS is not written.
GAS_HD void jac_species(const Factors &K, double rho, const double *y, const double *F,
                        double (&J)[NS + 1][NS + 1]) {
    const double T = y[9];
    const double C0 = rho * y[0] * 0.49603174603174605;
    const double C1 = rho * y[1] * 0.9920634920634921;
    const double C2 = rho * y[2] * 0.03125195324707794;
    const double C3 = rho * y[3] * 0.06250390649415588;
    const double C4 = rho * y[4] * 0.055509297807382736;
    const double C5 = rho * y[5] * 0.05879931792791203;
    const double C6 = rho * y[6] * 0.029399658963956014;
    const double C7 = rho * y[7] * 0.030297521662727988;
    const double C8 = rho * y[8] * 0.03569643749553795;
    double D[9][9];  // d wdot_k / d C_j
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int j = 0; j < 9; ++j) D[k][j] = 0.0;
    {  // reaction 0
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[0] * M;
        const double dkdM = K.kf[0];
        const double g = dkdM * (C0 - K.er[0] * (C1 * C1));
        const double dq0 = kfM * (1.0) + 2.5 * g;
        const double dq1 = -kfM * K.er[0] * (2.0 * C1) + g;
        const double dq2 = g;
        const double dq3 = g;
        const double dq4 = 12.0 * g;
        const double dq5 = g;
        const double dq6 = g;
        const double dq7 = g;
        const double dq8 = g;
        D[0][0] -= dq0;
        D[0][1] -= dq1;
        D[0][2] -= dq2;
        D[0][3] -= dq3;
        D[0][4] -= dq4;
        D[0][5] -= dq5;
        D[0][6] -= dq6;
        D[0][7] -= dq7;
        D[0][8] -= dq8;
        D[1][0] += 2.0 * dq0;
        D[1][1] += 2.0 * dq1;
        D[1][2] += 2.0 * dq2;
        D[1][3] += 2.0 * dq3;
        D[1][4] += 2.0 * dq4;
        D[1][5] += 2.0 * dq5;
        D[1][6] += 2.0 * dq6;
        D[1][7] += 2.0 * dq7;
        D[1][8] += 2.0 * dq8;
    }
    {  // reaction 1
        const double kfM = K.kf[1];
        const double dq0 = kfM * (C3);
        const double dq1 = -kfM * K.er[1] * (C5);
        const double dq3 = kfM * (C0);
        const double dq5 = -kfM * K.er[1] * (C1);
        D[0][0] -= dq0;
        D[0][1] -= dq1;
        D[0][3] -= dq3;
        D[0][5] -= dq5;
        D[3][0] -= dq0;
        D[3][1] -= dq1;
        D[3][3] -= dq3;
        D[3][5] -= dq5;
        D[1][0] += dq0;
        D[1][1] += dq1;
        D[1][3] += dq3;
        D[1][5] += dq5;
        D[5][0] += dq0;
        D[5][1] += dq1;
        D[5][3] += dq3;
        D[5][5] += dq5;
    }
    {  // reaction 2
        const double kfM = K.kf[2];
        const double dq0 = kfM * (C5);
        const double dq1 = -kfM * K.er[2] * (C4);
        const double dq4 = -kfM * K.er[2] * (C1);
        const double dq5 = kfM * (C0);
        D[0][0] -= dq0;
        D[0][1] -= dq1;
        D[0][4] -= dq4;
        D[0][5] -= dq5;
        D[5][0] -= dq0;
        D[5][1] -= dq1;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[1][0] += dq0;
        D[1][1] += dq1;
        D[1][4] += dq4;
        D[1][5] += dq5;
        D[4][0] += dq0;
        D[4][1] += dq1;
        D[4][4] += dq4;
        D[4][5] += dq5;
    }
    {  // reaction 3
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[3] * M;
        const double dkdM = K.kf[3];
        const double g = dkdM * ((C3 * C3) - K.er[3] * C2);
        const double dq0 = 2.5 * g;
        const double dq1 = g;
        const double dq2 = -kfM * K.er[3] * (1.0) + g;
        const double dq3 = kfM * (2.0 * C3) + g;
        const double dq4 = 12.0 * g;
        const double dq5 = g;
        const double dq6 = g;
        const double dq7 = g;
        const double dq8 = g;
        D[3][0] -= 2.0 * dq0;
        D[3][1] -= 2.0 * dq1;
        D[3][2] -= 2.0 * dq2;
        D[3][3] -= 2.0 * dq3;
        D[3][4] -= 2.0 * dq4;
        D[3][5] -= 2.0 * dq5;
        D[3][6] -= 2.0 * dq6;
        D[3][7] -= 2.0 * dq7;
        D[3][8] -= 2.0 * dq8;
        D[2][0] += dq0;
        D[2][1] += dq1;
        D[2][2] += dq2;
        D[2][3] += dq3;
        D[2][4] += dq4;
        D[2][5] += dq5;
        D[2][6] += dq6;
        D[2][7] += dq7;
        D[2][8] += dq8;
    }
    {  // reaction 4
        const double kfM = K.kf[4];
        const double dq1 = kfM * (C2);
        const double dq2 = kfM * (C1);
        const double dq3 = -kfM * K.er[4] * (C5);
        const double dq5 = -kfM * K.er[4] * (C3);
        D[2][1] -= dq1;
        D[2][2] -= dq2;
        D[2][3] -= dq3;
        D[2][5] -= dq5;
        D[1][1] -= dq1;
        D[1][2] -= dq2;
        D[1][3] -= dq3;
        D[1][5] -= dq5;
        D[3][1] += dq1;
        D[3][2] += dq2;
        D[3][3] += dq3;
        D[3][5] += dq5;
        D[5][1] += dq1;
        D[5][2] += dq2;
        D[5][3] += dq3;
        D[5][5] += dq5;
    }
    {  // reaction 5
        const double M = 0.73 * C0 + C1 + C2 + C3 + 3.65 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[5] * M;
        const double dkdM = K.kf[5];
        const double g = dkdM * (C1 * C5 - K.er[5] * C4);
        const double dq0 = 0.73 * g;
        const double dq1 = kfM * (C5) + g;
        const double dq2 = g;
        const double dq3 = g;
        const double dq4 = -kfM * K.er[5] * (1.0) + 3.65 * g;
        const double dq5 = kfM * (C1) + g;
        const double dq6 = g;
        const double dq7 = g;
        const double dq8 = g;
        D[1][0] -= dq0;
        D[1][1] -= dq1;
        D[1][2] -= dq2;
        D[1][3] -= dq3;
        D[1][4] -= dq4;
        D[1][5] -= dq5;
        D[1][6] -= dq6;
        D[1][7] -= dq7;
        D[1][8] -= dq8;
        D[5][0] -= dq0;
        D[5][1] -= dq1;
        D[5][2] -= dq2;
        D[5][3] -= dq3;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][6] -= dq6;
        D[5][7] -= dq7;
        D[5][8] -= dq8;
        D[4][0] += dq0;
        D[4][1] += dq1;
        D[4][2] += dq2;
        D[4][3] += dq3;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][6] += dq6;
        D[4][7] += dq7;
        D[4][8] += dq8;
    }
    {  // reaction 6
        const double kfM = K.kf[6];
        const double dq3 = kfM * (C4);
        const double dq4 = kfM * (C3);
        const double dq5 = -kfM * K.er[6] * (2.0 * C5);
        D[3][3] -= dq3;
        D[3][4] -= dq4;
        D[3][5] -= dq5;
        D[4][3] -= dq3;
        D[4][4] -= dq4;
        D[4][5] -= dq5;
        D[5][3] += 2.0 * dq3;
        D[5][4] += 2.0 * dq4;
        D[5][5] += 2.0 * dq5;
    }
    {  // reaction 7
        const double M = 2.5 * C0 + C1 + C2 + C3 + 12.0 * C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[7] * M;
        const double dkdM = K.kf[7];
        const double g = dkdM * (C3 * C1 - K.er[7] * C5);
        const double dq0 = 2.5 * g;
        const double dq1 = kfM * (C3) + g;
        const double dq2 = g;
        const double dq3 = kfM * (C1) + g;
        const double dq4 = 12.0 * g;
        const double dq5 = -kfM * K.er[7] * (1.0) + g;
        const double dq6 = g;
        const double dq7 = g;
        const double dq8 = g;
        D[3][0] -= dq0;
        D[3][1] -= dq1;
        D[3][2] -= dq2;
        D[3][3] -= dq3;
        D[3][4] -= dq4;
        D[3][5] -= dq5;
        D[3][6] -= dq6;
        D[3][7] -= dq7;
        D[3][8] -= dq8;
        D[1][0] -= dq0;
        D[1][1] -= dq1;
        D[1][2] -= dq2;
        D[1][3] -= dq3;
        D[1][4] -= dq4;
        D[1][5] -= dq5;
        D[1][6] -= dq6;
        D[1][7] -= dq7;
        D[1][8] -= dq8;
        D[5][0] += dq0;
        D[5][1] += dq1;
        D[5][2] += dq2;
        D[5][3] += dq3;
        D[5][4] += dq4;
        D[5][5] += dq5;
        D[5][6] += dq6;
        D[5][7] += dq7;
        D[5][8] += dq8;
    }
    {  // reaction 8
        const double M = 3.7 * C0 + C1 + 1.2 * C2 + C3 + 7.65 * C4 + C5 + 7.7 * C6 + C7 + 1.5 * C8;
        const double Pr = K.k0[0] * M / K.kf[8];
        const double lFc = K.lFc[0];
        const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
        const double lPr = log10(fmax(Pr, 1e-300));
        const double u = lPr + c, den = n - 0.14 * u;
        const double x = u / den;
        const double Fo = pow(10.0, lFc / (1.0 + x * x));
        const double ipr = 1.0 / (1.0 + Pr);
        const double kfM = K.kf[8] * (Pr * ipr) * Fo;
        const double opx = 1.0 + x * x;
        const double dkdM = K.k0[0] * Fo * ipr * (ipr - 2.0 * x * lFc * n / (opx * opx * den * den));
        const double g = dkdM * (C6 - K.er[8] * (C5 * C5));
        const double dq0 = 3.7 * g;
        const double dq1 = g;
        const double dq2 = 1.2 * g;
        const double dq3 = g;
        const double dq4 = 7.65 * g;
        const double dq5 = -kfM * K.er[8] * (2.0 * C5) + g;
        const double dq6 = kfM * (1.0) + 7.7 * g;
        const double dq7 = g;
        const double dq8 = 1.5 * g;
        D[6][0] -= dq0;
        D[6][1] -= dq1;
        D[6][2] -= dq2;
        D[6][3] -= dq3;
        D[6][4] -= dq4;
        D[6][5] -= dq5;
        D[6][6] -= dq6;
        D[6][7] -= dq7;
        D[6][8] -= dq8;
        D[5][0] += 2.0 * dq0;
        D[5][1] += 2.0 * dq1;
        D[5][2] += 2.0 * dq2;
        D[5][3] += 2.0 * dq3;
        D[5][4] += 2.0 * dq4;
        D[5][5] += 2.0 * dq5;
        D[5][6] += 2.0 * dq6;
        D[5][7] += 2.0 * dq7;
        D[5][8] += 2.0 * dq8;
    }
    {  // reaction 9
        const double kfM = K.kf[9];
        const double dq1 = kfM * (C6);
        const double dq4 = -kfM * K.er[9] * (C5);
        const double dq5 = -kfM * K.er[9] * (C4);
        const double dq6 = kfM * (C1);
        D[6][1] -= dq1;
        D[6][4] -= dq4;
        D[6][5] -= dq5;
        D[6][6] -= dq6;
        D[1][1] -= dq1;
        D[1][4] -= dq4;
        D[1][5] -= dq5;
        D[1][6] -= dq6;
        D[4][1] += dq1;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][6] += dq6;
        D[5][1] += dq1;
        D[5][4] += dq4;
        D[5][5] += dq5;
        D[5][6] += dq6;
    }
    {  // reaction 10
        const double kfM = K.kf[10];
        const double dq0 = -kfM * K.er[10] * (C7);
        const double dq1 = kfM * (C6);
        const double dq6 = kfM * (C1);
        const double dq7 = -kfM * K.er[10] * (C0);
        D[6][0] -= dq0;
        D[6][1] -= dq1;
        D[6][6] -= dq6;
        D[6][7] -= dq7;
        D[1][0] -= dq0;
        D[1][1] -= dq1;
        D[1][6] -= dq6;
        D[1][7] -= dq7;
        D[0][0] += dq0;
        D[0][1] += dq1;
        D[0][6] += dq6;
        D[0][7] += dq7;
        D[7][0] += dq0;
        D[7][1] += dq1;
        D[7][6] += dq6;
        D[7][7] += dq7;
    }
    {  // reaction 11
        const double kfM = K.kf[11];
        const double dq3 = kfM * (C6);
        const double dq5 = -kfM * K.er[11] * (C7);
        const double dq6 = kfM * (C3);
        const double dq7 = -kfM * K.er[11] * (C5);
        D[6][3] -= dq3;
        D[6][5] -= dq5;
        D[6][6] -= dq6;
        D[6][7] -= dq7;
        D[3][3] -= dq3;
        D[3][5] -= dq5;
        D[3][6] -= dq6;
        D[3][7] -= dq7;
        D[5][3] += dq3;
        D[5][5] += dq5;
        D[5][6] += dq6;
        D[5][7] += dq7;
        D[7][3] += dq3;
        D[7][5] += dq5;
        D[7][6] += dq6;
        D[7][7] += dq7;
    }
    {  // reaction 12
        const double kfM = K.kf[12];
        const double dq4 = -kfM * K.er[12] * (C7);
        const double dq5 = kfM * (C6);
        const double dq6 = kfM * (C5);
        const double dq7 = -kfM * K.er[12] * (C4);
        D[6][4] -= dq4;
        D[6][5] -= dq5;
        D[6][6] -= dq6;
        D[6][7] -= dq7;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][6] -= dq6;
        D[5][7] -= dq7;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][6] += dq6;
        D[4][7] += dq7;
        D[7][4] += dq4;
        D[7][5] += dq5;
        D[7][6] += dq6;
        D[7][7] += dq7;
    }
    {  // reaction 13
        const double kfM = K.kf[13];
        const double dq4 = -kfM * K.er[13] * (C7);
        const double dq5 = kfM * (C6);
        const double dq6 = kfM * (C5);
        const double dq7 = -kfM * K.er[13] * (C4);
        D[6][4] -= dq4;
        D[6][5] -= dq5;
        D[6][6] -= dq6;
        D[6][7] -= dq7;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][6] -= dq6;
        D[5][7] -= dq7;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][6] += dq6;
        D[4][7] += dq7;
        D[7][4] += dq4;
        D[7][5] += dq5;
        D[7][6] += dq6;
        D[7][7] += dq7;
    }
    {  // reaction 14
        const double kfM = K.kf[14];
        const double dq1 = kfM * (C7);
        const double dq5 = -kfM * K.er[14] * (2.0 * C5);
        const double dq7 = kfM * (C1);
        D[7][1] -= dq1;
        D[7][5] -= dq5;
        D[7][7] -= dq7;
        D[1][1] -= dq1;
        D[1][5] -= dq5;
        D[1][7] -= dq7;
        D[5][1] += 2.0 * dq1;
        D[5][5] += 2.0 * dq5;
        D[5][7] += 2.0 * dq7;
    }
    {  // reaction 15
        const double kfM = K.kf[15];
        const double dq0 = -kfM * K.er[15] * (C2);
        const double dq1 = kfM * (C7);
        const double dq2 = -kfM * K.er[15] * (C0);
        const double dq7 = kfM * (C1);
        D[7][0] -= dq0;
        D[7][1] -= dq1;
        D[7][2] -= dq2;
        D[7][7] -= dq7;
        D[1][0] -= dq0;
        D[1][1] -= dq1;
        D[1][2] -= dq2;
        D[1][7] -= dq7;
        D[0][0] += dq0;
        D[0][1] += dq1;
        D[0][2] += dq2;
        D[0][7] += dq7;
        D[2][0] += dq0;
        D[2][1] += dq1;
        D[2][2] += dq2;
        D[2][7] += dq7;
    }
    {  // reaction 16
        const double kfM = K.kf[16];
        const double dq2 = -kfM * K.er[16] * (C5);
        const double dq3 = kfM * (C7);
        const double dq5 = -kfM * K.er[16] * (C2);
        const double dq7 = kfM * (C3);
        D[7][2] -= dq2;
        D[7][3] -= dq3;
        D[7][5] -= dq5;
        D[7][7] -= dq7;
        D[3][2] -= dq2;
        D[3][3] -= dq3;
        D[3][5] -= dq5;
        D[3][7] -= dq7;
        D[5][2] += dq2;
        D[5][3] += dq3;
        D[5][5] += dq5;
        D[5][7] += dq7;
        D[2][2] += dq2;
        D[2][3] += dq3;
        D[2][5] += dq5;
        D[2][7] += dq7;
    }
    {  // reaction 17
        const double kfM = K.kf[17];
        const double dq2 = -kfM * K.er[17] * (C4);
        const double dq4 = -kfM * K.er[17] * (C2);
        const double dq5 = kfM * (C7);
        const double dq7 = kfM * (C5);
        D[5][2] -= dq2;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][7] -= dq7;
        D[7][2] -= dq2;
        D[7][4] -= dq4;
        D[7][5] -= dq5;
        D[7][7] -= dq7;
        D[4][2] += dq2;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][7] += dq7;
        D[2][2] += dq2;
        D[2][4] += dq4;
        D[2][5] += dq5;
        D[2][7] += dq7;
    }
    {  // reaction 18
        const double kfM = K.kf[18];
        const double dq2 = -kfM * K.er[18] * (C4);
        const double dq4 = -kfM * K.er[18] * (C2);
        const double dq5 = kfM * (C7);
        const double dq7 = kfM * (C5);
        D[5][2] -= dq2;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][7] -= dq7;
        D[7][2] -= dq2;
        D[7][4] -= dq4;
        D[7][5] -= dq5;
        D[7][7] -= dq7;
        D[4][2] += dq2;
        D[4][4] += dq4;
        D[4][5] += dq5;
        D[4][7] += dq7;
        D[2][2] += dq2;
        D[2][4] += dq4;
        D[2][5] += dq5;
        D[2][7] += dq7;
    }
    {  // reaction 19
        const double kfM = K.kf[19];
        const double dq2 = -kfM * K.er[19] * (C6);
        const double dq6 = -kfM * K.er[19] * (C2);
        const double dq7 = kfM * (2.0 * C7);
        D[7][2] -= 2.0 * dq2;
        D[7][6] -= 2.0 * dq6;
        D[7][7] -= 2.0 * dq7;
        D[6][2] += dq2;
        D[6][6] += dq6;
        D[6][7] += dq7;
        D[2][2] += dq2;
        D[2][6] += dq6;
        D[2][7] += dq7;
    }
    {  // reaction 20
        const double kfM = K.kf[20];
        const double dq2 = -kfM * K.er[20] * (C6);
        const double dq6 = -kfM * K.er[20] * (C2);
        const double dq7 = kfM * (2.0 * C7);
        D[7][2] -= 2.0 * dq2;
        D[7][6] -= 2.0 * dq6;
        D[7][7] -= 2.0 * dq7;
        D[6][2] += dq2;
        D[6][6] += dq6;
        D[6][7] += dq7;
        D[2][2] += dq2;
        D[2][6] += dq6;
        D[2][7] += dq7;
    }
    {  // reaction 21
        const double M = 1.3 * C0 + C1 + C2 + C3 + 10.0 * C4 + C5 + C6 + C7 + C8;
        const double Pr = K.k0[1] * M / K.kf[21];
        const double lFc = K.lFc[1];
        const double c = -0.4 - 0.67 * lFc, n = 0.75 - 1.27 * lFc;
        const double lPr = log10(fmax(Pr, 1e-300));
        const double u = lPr + c, den = n - 0.14 * u;
        const double x = u / den;
        const double Fo = pow(10.0, lFc / (1.0 + x * x));
        const double ipr = 1.0 / (1.0 + Pr);
        const double kfM = K.kf[21] * (Pr * ipr) * Fo;
        const double opx = 1.0 + x * x;
        const double dkdM = K.k0[1] * Fo * ipr * (ipr - 2.0 * x * lFc * n / (opx * opx * den * den));
        const double g = dkdM * (C1 * C2 - K.er[21] * C7);
        const double dq0 = 1.3 * g;
        const double dq1 = kfM * (C2) + g;
        const double dq2 = kfM * (C1) + g;
        const double dq3 = g;
        const double dq4 = 10.0 * g;
        const double dq5 = g;
        const double dq6 = g;
        const double dq7 = -kfM * K.er[21] * (1.0) + g;
        const double dq8 = g;
        D[1][0] -= dq0;
        D[1][1] -= dq1;
        D[1][2] -= dq2;
        D[1][3] -= dq3;
        D[1][4] -= dq4;
        D[1][5] -= dq5;
        D[1][6] -= dq6;
        D[1][7] -= dq7;
        D[1][8] -= dq8;
        D[2][0] -= dq0;
        D[2][1] -= dq1;
        D[2][2] -= dq2;
        D[2][3] -= dq3;
        D[2][4] -= dq4;
        D[2][5] -= dq5;
        D[2][6] -= dq6;
        D[2][7] -= dq7;
        D[2][8] -= dq8;
        D[7][0] += dq0;
        D[7][1] += dq1;
        D[7][2] += dq2;
        D[7][3] += dq3;
        D[7][4] += dq4;
        D[7][5] += dq5;
        D[7][6] += dq6;
        D[7][7] += dq7;
        D[7][8] += dq8;
    }
    {  // reaction 22
        const double M = C0 + C1 + C2 + C3 + C4 + C5 + C6 + C7 + C8;
        const double kfM = K.kf[22] * M;
        const double dkdM = K.kf[22];
        const double g = dkdM * (C3 * C5 - K.er[22] * C7);
        const double dq0 = g;
        const double dq1 = g;
        const double dq2 = g;
        const double dq3 = kfM * (C5) + g;
        const double dq4 = g;
        const double dq5 = kfM * (C3) + g;
        const double dq6 = g;
        const double dq7 = -kfM * K.er[22] * (1.0) + g;
        const double dq8 = g;
        D[3][0] -= dq0;
        D[3][1] -= dq1;
        D[3][2] -= dq2;
        D[3][3] -= dq3;
        D[3][4] -= dq4;
        D[3][5] -= dq5;
        D[3][6] -= dq6;
        D[3][7] -= dq7;
        D[3][8] -= dq8;
        D[5][0] -= dq0;
        D[5][1] -= dq1;
        D[5][2] -= dq2;
        D[5][3] -= dq3;
        D[5][4] -= dq4;
        D[5][5] -= dq5;
        D[5][6] -= dq6;
        D[5][7] -= dq7;
        D[5][8] -= dq8;
        D[7][0] += dq0;
        D[7][1] += dq1;
        D[7][2] += dq2;
        D[7][3] += dq3;
        D[7][4] += dq4;
        D[7][5] += dq5;
        D[7][6] += dq6;
        D[7][7] += dq7;
        D[7][8] += dq8;
    }
    double cv = 0.0;
    cv += y[0] * (K.cpR[0] - 1.0) * 0.49603174603174605;
    cv += y[1] * (K.cpR[1] - 1.0) * 0.9920634920634921;
    cv += y[2] * (K.cpR[2] - 1.0) * 0.03125195324707794;
    cv += y[3] * (K.cpR[3] - 1.0) * 0.06250390649415588;
    cv += y[4] * (K.cpR[4] - 1.0) * 0.055509297807382736;
    cv += y[5] * (K.cpR[5] - 1.0) * 0.05879931792791203;
    cv += y[6] * (K.cpR[6] - 1.0) * 0.029399658963956014;
    cv += y[7] * (K.cpR[7] - 1.0) * 0.030297521662727988;
    cv += y[8] * (K.cpR[8] - 1.0) * 0.03569643749553795;
    cv *= 8314.46261815324;
    const double RT_cv = 8314.46261815324 * T / cv;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        double sT = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) sT += (K.hRT[k] - 1.0) * D[k][j];
        constexpr double Wk[9] = {2.016, 1.008, 31.998, 15.999, 18.015, 17.007, 34.014, 33.006, 28.014};
        constexpr double iWk[9] = {0.49603174603174605, 0.9920634920634921, 0.03125195324707794, 0.06250390649415588, 0.055509297807382736, 0.05879931792791203, 0.029399658963956014, 0.030297521662727988, 0.03569643749553795};
#pragma unroll
        for (int k = 0; k < 9; ++k) J[k][j] = D[k][j] * Wk[k] * iWk[j];
        J[9][j] = -(RT_cv * sT + F[9] * 8314.46261815324 * (K.cpR[j] - 1.0) / cv) * iWk[j];
    }
}

// The integrator's kinetics policy (gas::ros2_advance_k): factors once per temperature,
// right-hand sides from them, the species columns of the Jacobian analytically.
struct Kinetics {
    using K = Factors;
    static constexpr bool kAnalyticJacobian = true;
    GAS_HD void factors(double T, Factors &k) const { kin_h2_air_9::factors(T, k); }
    GAS_HD void rhs(const Factors &k, double rho, const double *y, double *F) const {
        rhs_k(k, rho, y, F);
    }
    GAS_HD void jacobian(const Factors &k, double rho, const double *y, const double *F,
                         double (&J)[NS + 1][NS + 1]) const {
        jac_species(k, rho, y, F, J);
    }
};

}  // namespace kin_h2_air_9
