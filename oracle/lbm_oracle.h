/* Plain-C CPU oracle for the D3Q27 thermal lattice-Boltzmann hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg call this library as the checker; the product (liblbmgpu.so) never
 * links or calls it.
 *
 * It restates the reference solver's per-step algorithm (farrasarira/Lattice-Boltzmann-
 * Method) in straightforward FP64 C over the reference's own array-of-structures cell
 * layout, so outputs can be compared cell by cell with both the reference library
 * (oracle/_ref) and the CUDA path's download.  Each function names the reference
 * routine it follows.
 *
 * Parity of this oracle is pinned against the reference's own sources compiled here
 * (oracle/_ref/libref_sc.so) and against the fixtures in tests/golden/.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Cell-type codes (reference src/headers/defines.hpp:140-149). */
enum { ORC_F = 0, ORC_S = 1, ORC_P = 2, ORC_A = 3, ORC_FS = 4, ORC_I = 5, ORC_O = 6,
       ORC_I_C = 7, ORC_O_C = 8, ORC_Q = 9 };

/* Single-component cell record with the byte layout of the reference's MIXTURE class
 * when MULTICOMP is off (src/headers/lbm.hpp:56-88): 1024 bytes. */
typedef struct {
    short type;
    double f[27], fpc[27];
    double p_tensor[3][3];
    double rho, u, v, w, p;
    double g[27], gpc[27];
    double rhoe;
    double energy_flux[3];
    double temp;
} orc_mix_sc;

/* Lattice sizes INCLUDING the one-cell ghost layer (LBM::Nx etc., lbm-main.cpp:19-21)
 * and the single-component gas parameters (lbm.hpp:117-121). */
typedef struct {
    int Nx, Ny, Nz;
    double nu, R, gamma, prtl;
    int dt;
} orc_sc_grid;

size_t orc_sc_sizeof(void);

/* Equilibria and helpers, exported for known-answer tests. */
double orc_feq(int l, double rho, const double u[3], double theta, const double corr[3]);
double orc_geq(int l, double rho, double U, double theta, const double u[3]);
double orc_geq_moment(int l, double rhoe, const double q[3], const double R[9], double theta);
double orc_gstr(int l, double geq, const double dq[3]);
double orc_fd_central(double l, double c, double r, double dx, double vel, int tl, int tr);
double orc_fd_fuw(double l, double c, double r, double dx, double vel, int tl, int tr);
double orc_fd_uw(double s0, double s1, double s2, double dx, double vel);

/* One phase each, in the reference's per-step order (lbm-main.cpp:163-181). */
void orc_sc_init(orc_mix_sc *cells, const orc_sc_grid *g);
void orc_sc_collide(orc_mix_sc *cells, const orc_sc_grid *g);
void orc_sc_streaming(orc_mix_sc *cells, const orc_sc_grid *g);
void orc_sc_tms_bc(orc_mix_sc *cells, const orc_sc_grid *g);
void orc_sc_moment(orc_mix_sc *cells, const orc_sc_grid *g);
/* nsteps of Collide -> Streaming -> TMS_BC -> calculate_moment. */
void orc_sc_loop(orc_mix_sc *cells, const orc_sc_grid *g, int nsteps);

void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
