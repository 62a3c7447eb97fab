/* lbmgpu -- B200 (sm_100a) implementation of the per-timestep hot path of the
 * compressible thermal D3Q27 lattice-Boltzmann solver farrasarira/Lattice-Boltzmann-Method.
 *
 * C ABI: plain pointers and sizes, no C++ or CUDA types.  One handle owns the device
 * state of one LBM object on one GPU and one CUDA stream.  Every call returns an int:
 *   0                 success
 *   negative          API misuse (LBMGPU_E_*), nothing was launched
 *   positive          device status bits (LBMGPU_ST_*) raised by the kernels
 * Nothing throws across the ABI.  A handle is not thread-safe.
 *
 * How the reference's driver reaches it: the LBM member functions that make up one time
 * step (src/headers/lbm.hpp:152-197, called in src/lbm-main.cpp:149-196) keep their
 * signatures and forward here, one call each: LBM::Collide() calls lbmgpu_collide(h), and so on.
 */
#ifndef LBMGPU_H
#define LBMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBMGPU_ABI_VERSION 2

/* ---- error codes ------------------------------------------------------------- */
#define LBMGPU_OK 0
#define LBMGPU_E_ARG (-1)        /* bad argument or descriptor                       */
#define LBMGPU_E_CUDA (-2)       /* a CUDA runtime call failed                        */
#define LBMGPU_E_NODEV (-3)      /* no usable CUDA device / kernel image              */
#define LBMGPU_E_PHASE (-4)      /* phase calls out of the reference's step order     */
#define LBMGPU_E_STATE (-5)      /* no state uploaded / initialised yet               */
#define LBMGPU_E_UNSUPPORTED (-6) /* configuration not implemented                   */
#define LBMGPU_E_VERSION (-7)    /* descriptor abi_version mismatch                   */
#define LBMGPU_E_IO (-8)         /* a file could not be opened, read or written       */

/* ---- device status bits (sticky until lbmgpu_status(..., clear=1)) ------------ */
#define LBMGPU_ST_NAN 0x1u          /* non-finite density, velocity or temperature     */
#define LBMGPU_ST_NEG_STATE 0x2u    /* density or temperature <= 0                     */
#define LBMGPU_ST_TAU_UNSTABLE 0x4u /* 1/omega <= 1/2 (the reference prints these:
                                       src/lbm-collision.cpp:33-34)                   */
#define LBMGPU_ST_NEWTON 0x8u       /* temperature Newton iteration hit its cap        */
#define LBMGPU_ST_CHEM 0x10u        /* stiff chemistry hit its sub-step cap            */
#define LBMGPU_ST_SURROGATE 0x20u   /* the surrogate network's tensor-core wait ran out */

/* ---- precision of the population storage ------------------------------------- */
#define LBMGPU_FP64 0   /* the reference's doubles; results bit-faithful                */
#define LBMGPU_FP32 1   /* multicomponent only: populations stored in float as deviations
                           from a per-plane shift (the plane's mean over the fluid cells,
                           re-taken at upload and Init), the per-cell record in float; all
                           arithmetic stays FP64.  Halves the state and its traffic.       */

/* ---- gas mechanism ------------------------------------------------------------
 * Flat tables of one ideal-gas mechanism in SI units (kmol, m, s, J, K), the data the
 * reference obtains from Cantera (src/lbm-main.cpp:79-117).  Filled by a loader from the
 * repository's Cantera-YAML mechanisms (src/reaction-mech/*.yaml): NASA-7 thermo, gas
 * transport parameters, and elementary / three-body / falloff (Lindemann, Troe) reactions
 * with mass-action rate laws.  Species are listed in the caller's order. */
#define LBMGPU_MAX_SPECIES 12
#define LBMGPU_MAX_REACTIONS 48
#define LBMGPU_MAX_RSPEC 3     /* species per side of a reaction */
#define LBMGPU_MAX_ELEMENTS 5  /* H, O, N, Ar, C */

enum { LBMGPU_RXN_ELEMENTARY = 0, LBMGPU_RXN_THREEBODY = 1, LBMGPU_RXN_FALLOFF = 2 };
enum { LBMGPU_GEOM_ATOM = 0, LBMGPU_GEOM_LINEAR = 1, LBMGPU_GEOM_NONLINEAR = 2 };

typedef struct lbmgpu_mech {
    int n_species, n_reactions;
    char name[LBMGPU_MAX_SPECIES][16];
    double W[LBMGPU_MAX_SPECIES];                 /* molar mass, kg/kmol                 */
    double T_lo[LBMGPU_MAX_SPECIES], T_mid[LBMGPU_MAX_SPECIES], T_hi[LBMGPU_MAX_SPECIES];
    double nasa_lo[LBMGPU_MAX_SPECIES][7];        /* NASA-7 coefficients below T_mid     */
    double nasa_hi[LBMGPU_MAX_SPECIES][7];        /* NASA-7 coefficients above T_mid     */
    int geometry[LBMGPU_MAX_SPECIES];             /* LBMGPU_GEOM_*                       */
    double well_depth[LBMGPU_MAX_SPECIES];        /* epsilon / k_B, K                    */
    double diameter[LBMGPU_MAX_SPECIES];          /* Lennard-Jones sigma, m              */
    double dipole[LBMGPU_MAX_SPECIES];            /* C m                                 */
    double polarizability[LBMGPU_MAX_SPECIES];    /* m^3                                 */
    double rot_relax[LBMGPU_MAX_SPECIES];         /* Z_rot at 298 K                      */
    int elements[LBMGPU_MAX_SPECIES][LBMGPU_MAX_ELEMENTS]; /* atoms of H, O, N, Ar, C      */
    int rtype[LBMGPU_MAX_REACTIONS];              /* LBMGPU_RXN_*                        */
    int reversible[LBMGPU_MAX_REACTIONS];
    int n_reac[LBMGPU_MAX_REACTIONS], n_prod[LBMGPU_MAX_REACTIONS];
    int reac[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_RSPEC], prod[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_RSPEC];
    double nu_reac[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_RSPEC], nu_prod[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_RSPEC];
    double A[LBMGPU_MAX_REACTIONS], b[LBMGPU_MAX_REACTIONS], Ea[LBMGPU_MAX_REACTIONS]; /* k (or k_inf), Ea in J/kmol */
    double A0[LBMGPU_MAX_REACTIONS], b0[LBMGPU_MAX_REACTIONS], Ea0[LBMGPU_MAX_REACTIONS]; /* falloff k_0 */
    int troe_n[LBMGPU_MAX_REACTIONS];             /* 0 Lindemann, 3 or 4 Troe parameters  */
    double troe[LBMGPU_MAX_REACTIONS][4];         /* a, T***, T*, T**                    */
    double eff[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_SPECIES]; /* third-body efficiencies      */
    /* forward reaction orders of the reactants in reac[][] (the mass-action exponents of the
     * forward rate): nu_reac unless the mechanism gives `orders` (the global CH4 and C3H8
     * steps of src/reaction-mech/CH4_2S.yaml and propane_mech.yaml); a non-integer order
     * takes the concentration clipped at zero */
    double order_reac[LBMGPU_MAX_REACTIONS][LBMGPU_MAX_RSPEC];
} lbmgpu_mech;

/* Byte offsets of the fields of the caller's MIXTURE record (src/headers/lbm.hpp:56-88).
 * Fill with sizeof/offsetof from the caller's own class; -1 marks a field the
 * configuration does not have (f/fpc are absent when MULTICOMP is on). */
typedef struct lbmgpu_mixture_layout {
    size_t size;
    long type, f, fpc, p_tensor, rho, u, v, w, p, g, gpc, rhoe, energy_flux, temp, HRR;
} lbmgpu_mixture_layout;

/* Byte offsets of the caller's SPECIES record (src/headers/lbm.hpp:90-102). */
typedef struct lbmgpu_species_layout {
    size_t size;
    long X, rho, f, fpc, u, v, w;
} lbmgpu_species_layout;

/* Chemistry of the species collision (multicomponent). */
#define LBMGPU_CHEM_OFF 0           /* REACTION off                                     */
#define LBMGPU_CHEM_REF_EXPLICIT 1  /* the reference's scheme: two explicit half steps of
                                       the net production rates with T from (u, v) in
                                       between (src/lbm-collision.cpp:370-399)          */
#define LBMGPU_CHEM_ROSENBROCK 2    /* no counterpart in the reference: the constant-
                                       density, constant-energy reactor integrated over
                                       the whole step by the L-stable two-stage
                                       Rosenbrock method ROS2 with step-size control
                                       (rtol 1e-5; at most 256 sub-steps, then
                                       LBMGPU_ST_CHEM), its density change entering the
                                       species collision like the reference's            */

typedef struct lbmgpu_desc {
    int abi_version;      /* LBMGPU_ABI_VERSION                                           */
    int device;           /* CUDA device ordinal                                          */
    int Nx, Ny, Nz;       /* lattice INCLUDING the ghost layer (LBM::Nx, lbm-main.cpp:19-21) */
    int n_species;        /* 0: single component (MULTICOMP off)                          */
    int precision;        /* LBMGPU_FP64 or LBMGPU_FP32                                   */
    int dt_sim;           /* LBM::dt_sim (lbm.hpp:113), 1 in the reference                */
    double nu;            /* single component: kinematic viscosity (lbm.hpp:117)          */
    double gas_const;     /* gas constant R (lbm.hpp:118)                                 */
    double gamma;         /* cp/cv (lbm.hpp:119)                                          */
    double prtl;          /* Prandtl number (lbm.hpp:121)                                 */
    lbmgpu_mixture_layout mix;
    /* multicomponent (n_species > 0) */
    lbmgpu_species_layout spc;
    const lbmgpu_mech *mech;  /* species in the LBM's order; copied at create            */
    float units_m, units_kg, units_s, units_K; /* the caller's Units_Conv base units
                                                  (src/headers/units.hpp:10)             */
    int chem_mode;            /* LBMGPU_CHEM_*                                           */
} lbmgpu_desc;

typedef struct lbmgpu lbmgpu_t;

/* Creates the device state for one LBM object.  Replaces the allocation done by
 * LBM::LBM(Nx,Ny,Nz,nu) (src/lbm-main.cpp:16-35). */
int lbmgpu_create(const lbmgpu_desc *desc, lbmgpu_t **out);
int lbmgpu_destroy(lbmgpu_t *h);

/* Copies the caller's AoS cell arrays to the device: the mixture records
 * (LBM::mixture_data, lbm.hpp:134) and, multicomponent, one species array per species
 * (LBM::species_data[a], lbm.hpp:136; NULL when single component).  Nx*Ny*Nz records
 * each, in the reference's [i][j][k] order, k fastest.  The next Collide uses the
 * uploaded populations and moments as they stand, exactly as the reference's first step
 * after Init or read_restart does. */
int lbmgpu_upload(lbmgpu_t *h, const void *mixture_aos, const void *const *species_aos);

/* Writes the current state back into the caller's AoS arrays at a step boundary:
 * populations (post-stream, post-boundary), post-collision populations and moments of
 * every fluid cell; the stored moments of every other cell. */
int lbmgpu_download(lbmgpu_t *h, void *mixture_aos, void *const *species_aos);

/* lbmgpu_upload / lbmgpu_download for the x-planes i0 .. i1-1 only (ghost planes counted,
 * 0 <= i0 < i1 <= Nx), multicomponent handles: the caller's arrays hold the
 * (i1 - i0) * Ny * Nz records of those planes, in the reference's order.  For lattices
 * whose AoS copy (600 + n_species * 472 bytes per cell in the reference's layout: 83 GB at
 * 258^3) does not fit in host memory at once, and for the reference's restart file, which
 * is read and written plane by plane.  Planes may arrive in any order and over any number
 * of calls; once every plane has arrived since the last complete upload, the state is
 * complete and behaves exactly as after lbmgpu_upload (until then lbmgpu_init and the
 * phases return LBMGPU_E_STATE).  The arrays may be pageable or page-locked host memory
 * (page-locked arrays are copied without the library's staging); each call returns with its
 * copies complete.  No counterpart in the reference, which holds the whole AoS in host
 * memory (src/headers/lbm.hpp:134-137). */
int lbmgpu_upload_planes(lbmgpu_t *h, int i0, int i1, const void *mixture_aos, const void *const *species_aos);
int lbmgpu_download_planes(lbmgpu_t *h, int i0, int i1, void *mixture_aos, void *const *species_aos);

/* ---- slab decomposition along x (one slab per GPU) --------------------------------
 * No counterpart in the reference, which runs on one host (OpenMP).  A slab is an LBM
 * lattice of its own whose x ghost planes may be marked as halos: each holds the
 * neighbouring slab's edge plane (where the decomposed domain is periodic in x, the first
 * and the last slab are neighbours).  Cells of a halo plane are never updated by this
 * handle; no periodic wrap runs through a halo; the boundary formulas use nx_global (the
 * whole domain's Nx, ghosts included) as the domain length along x.  Two exchanges per
 * time step keep the halos as the single domain would see those planes:
 *   LBMGPU_HALO_POPULATIONS  after lbmgpu_collide and before lbmgpu_calculate_moment: the
 *       post-collision populations that stream across the face (9 directions per
 *       population set);
 *   LBMGPU_HALO_RECORD  between time steps (after calculate_moment, before the next
 *       Collide): the whole per-cell record of the edge plane.
 * lbmgpu_halo_pack(face 0) writes this slab's first plane for the lower neighbour, whose
 * lbmgpu_halo_unpack(face 1) reads it; face 1 writes the last plane for the upper
 * neighbour's face 0.  Buffers are device memory of lbmgpu_halo_bytes bytes (FP64 values,
 * populations decoded, so slabs in the FP32 mode need not share a shift); both calls are
 * enqueued on the handle's stream, so the caller synchronises before handing a buffer to
 * its transport (NCCL send/recv, a peer copy) and after receiving.  lbmgpu_step runs no
 * exchange: slabs step through the phase calls.  Multicomponent handles only;
 * lbmgpu_set_halo takes effect at the next upload (the state must be uploaded again). */
#define LBMGPU_HALO_POPULATIONS 0
#define LBMGPU_HALO_RECORD 1
int lbmgpu_set_halo(lbmgpu_t *h, int lo, int hi, int nx_global);
int lbmgpu_halo_bytes(lbmgpu_t *h, int what, size_t *bytes);
int lbmgpu_halo_pack(lbmgpu_t *h, int face, int what, void *dev_buf);
int lbmgpu_halo_unpack(lbmgpu_t *h, int face, int what, const void *dev_buf);

/* The handle's CUDA stream (a cudaStream_t), for callers that order their own work --
 * the halo transport, timing events -- with the handle's kernels.  No counterpart in the
 * reference. */
int lbmgpu_get_stream(lbmgpu_t *h, void **stream);

/* The base units units.set_m_kg_s(dx, dt) sets (src/headers/units.hpp:32-44), with its
 * float rounding: out = {m, kg, s, K}. */
int lbmgpu_units_from_dx_dt(float dx, float dt, float *out4);

/* LBM::Init (src/lbm-init.cpp:8-82 single component, :85-146 multicomponent) on the
 * uploaded setup fields. */
int lbmgpu_init(lbmgpu_t *h);

/* The reference's per-step phases, called in its order (src/lbm-main.cpp:157-181).
 * Collide launches the collision kernel; Streaming and TMS_BC record the phase;
 * calculate_moment launches the fused streaming + boundary + moment kernel.  Calls out
 * of order return LBMGPU_E_PHASE. */
int lbmgpu_collide_species(lbmgpu_t *h);  /* LBM::Collide_Species, lbm-collision.cpp:334 */
int lbmgpu_collide(lbmgpu_t *h);          /* LBM::Collide, lbm-collision.cpp:9 / :191    */
int lbmgpu_streaming(lbmgpu_t *h);        /* LBM::Streaming, lbm-streaming.cpp:3         */
int lbmgpu_tms_bc(lbmgpu_t *h);           /* LBM::TMS_BC, lbm-bc.cpp:122                 */
int lbmgpu_calculate_moment(lbmgpu_t *h); /* LBM::calculate_moment, lbm-moment.cpp:11    */

/* nsteps complete time steps (the body of LBM::loop, lbm-main.cpp:153-194, without the
 * output cadence).  Asynchronous on the handle's stream. */
int lbmgpu_step(lbmgpu_t *h, int nsteps);

/* lbmgpu_step bracketed by CUDA events on the handle's stream: *ms receives the device
 * time of the nsteps steps (the call waits for them to finish). */
int lbmgpu_time_steps(lbmgpu_t *h, int nsteps, double *ms);

/* Waits for the handle's stream.  Returns the device status bits as a positive value. */
int lbmgpu_synchronize(lbmgpu_t *h);

/* Reads (and optionally clears) the sticky device status bits. */
int lbmgpu_status(lbmgpu_t *h, uint32_t *flags, int clear);

/* Per-kernel device timing.  When enabled, every launch is bracketed by CUDA events on
 * the handle's stream; lbmgpu_kernel_times returns, per kernel kind, the number of
 * launches and the summed device milliseconds since the last reset.
 * Kinds: 0 collide (multicomponent: the population update), 1 stream+boundary+moment
 * (multicomponent: the interior cells' pull and population sums), 2 other, 3
 * multicomponent collision parameters, 4 chemistry surrogate (features, network, the
 * integrator's cells), 5 multicomponent moment solve of the interior cells, 6
 * multicomponent energy-flux terms of the collision, 7 stiff chemistry (ROS2) of every
 * cell.  Returns the number of kinds. */
int lbmgpu_profile(lbmgpu_t *h, int enable);
int lbmgpu_kernel_times(lbmgpu_t *h, int nkinds, long *launches, double *ms);

/* FP64 totals over the fluid cells of the current state (the last complete moments),
 * no counterpart in the reference's API (its diagnostics reduce the AoS arrays on the
 * host, OutputKeEns in src/output.cpp):
 *   out[0] mass sum rho, out[1..3] momentum sum rho u, out[4] total energy (sum rhoE),
 *   multicomponent also out[5 .. 5+ns-1] the species masses sum rho_a and
 *   out[5+ns .. 5+ns+4] the element totals sum_a rho_a / W_a * (atoms of H, O, N, Ar, C),
 * all in lattice units.  lbmgpu_sums_count gives the number of values (5, or
 * 5 + n_species + 5); n_out must be at least that.  The reduction order is fixed, so
 * the totals are reproducible bit for bit.  The first call allocates the handle's
 * reduction scratch (LBMGPU_SUMS_MAX * 1185 doubles); the call waits for the stream. */
#define LBMGPU_SUMS_MAX 22
int lbmgpu_sums_count(const lbmgpu_t *h);
int lbmgpu_sums(lbmgpu_t *h, double *out, int n_out);

/* lbmgpu_sums without any device allocation, no counterpart in the reference: the
 * reduction scratch is a fixed device array of the library (208,560 bytes per device)
 * instead of handle memory, for callers that cannot allocate after setup (a lattice that
 * fills the device, a monitoring loop that must not synchronise the device through
 * cudaMalloc, a host whose pool owns all device memory).  Same values, bit for bit, as
 * lbmgpu_sums.  n_out must lie in [lbmgpu_sums_count(h), LBMGPU_SUMS_MAX], else
 * LBMGPU_E_ARG.  The scratch is shared by every handle on the device: calls that overlap
 * on one device race, so serialise them.  lbmgpu_create loads the scratch and the
 * reduction kernels on its device (CUDA loads modules lazily by default), so no call of
 * this entry point allocates; the scratch stays until the process exits, or until a
 * cudaDeviceReset, which also ends every handle on that device. */
int lbmgpu_sums_noalloc(lbmgpu_t *h, double *out, int n_out);

/* Run diagnostics of the current state, reduced on the device (FP64, lattice units, over
 * the fluid cells): out[0] sum rho |u|^2, out[1] sum rho |curl u|^2 with the wrapped
 * central differences, out[2] sum rho E -- the reference's OutputKeEns
 * (src/output.cpp:212-275), which the driver calls at output steps -- then out[3] the sum
 * of the heat-release field (src/lbm-collision.cpp:395-398; 0 for a single component),
 * out[4] the peak and out[5] the minimum temperature.  n_out >= LBMGPU_DIAG_COUNT.  Uses
 * the reduction scratch of lbmgpu_sums; waits for the stream. */
#define LBMGPU_DIAG_COUNT 6
int lbmgpu_diagnostics(lbmgpu_t *h, double *out, int n_out);

/* ---- chemistry surrogate (LBMGPU_CHEM_ROSENBROCK handles) --------------------------
 * No counterpart in the reference.  A small network learns the stiff integrator's step
 *   (T [K], ln p [Pa], Y_0..Y_8, dt [s])  ->  (dY_0..dY_8, dT [K])
 * (12 -> 128 -> 128 -> 128 -> 10, GELU, BF16 weights and activations, FP32 accumulation,
 * standardised inputs and outputs) from samples the integrator writes during the run,
 * then replaces it cell by cell: the predicted dY is projected (orthogonally) onto changes
 * that conserve every element; cells whose features leave the training box (widened by
 * 5 %), whose prediction is not finite or lies beyond 16 standard deviations of the
 * training targets, or whose projected change would take a mass fraction below -1e-12 run
 * the integrator; and every audit_period-th cell (0: none; the phase moves from step to
 * step) runs it as well, takes its result and scores the prediction (L1 error of dY).
 *
 * lbmgpu_surrogate_collect: while enabled, each step's integrator writes the features and
 *   targets of every stride-th cell (a different subset each step) to the device sample
 *   set, grown to `capacity` rows with the rows already there kept; collection stops when
 *   it is full.  During surrogate steps the rows come from the audit stride instead (the
 *   audited cells and those outside the training box on it -- states the integrator
 *   computes anyway), so the set follows the run and lbmgpu_surrogate_train can refresh
 *   the network as the run leaves the states it was trained on.
 * lbmgpu_surrogate_load_samples: replaces the sample set by n host rows (x: n x 12 raw
 *   features, y: n x 10 raw targets).
 * lbmgpu_surrogate_samples: copies the first n rows of the sample set to the host (x, y as
 *   above; valid[r] = 1 where row r was written); n <= the report's `samples`.
 * lbmgpu_surrogate_augment: appends n rows made from random valid rows of the sample set
 *   (the set grows as needed): mass fractions below y_trace multiplied by exp(U(-span_y,
 *   span_y)), T by exp(U(-span_t, span_t)), at the source row's density, renormalised,
 *   and labelled by the integrator -- states near the visited ones that the run has not
 *   reached yet, so the network learns how the step depends on each input there.
 * lbmgpu_surrogate_train: Adam (beta 0.9/0.999) on the mean squared standardised error,
 *   `epochs` passes over the samples in shuffled minibatches of `batch` (a multiple of 64)
 *   rows, the step size decaying from lr to 0 along a half cosine over the call; the
 *   standardisation and gate box are fitted on the first call or with refit; *loss = the
 *   last epoch's mean loss.
 * lbmgpu_surrogate_enable: the surrogate on (after training) or off; resets the audit
 *   counters of lbmgpu_surrogate_stats.
 * lbmgpu_surrogate_eval: the network on n host rows of raw features (x: n x 12) ->
 *   raw predictions (y: n x 10), before projection.
 * lbmgpu_surrogate_params: get (set = 0) or set the parameters, packed as W1 [128][12],
 *   b1 [128], W2 [128][128], b2, W3 [128][128], b3, W4 [10][128], b4 [10], then x_mean,
 *   x_std, x_lo, x_hi [12 each], y_mean, y_std [10 each] (LBMGPU_SUR_NPARAMS floats);
 *   setting resets Adam and marks the surrogate trained. */
#define LBMGPU_SUR_NPARAMS 36046
typedef struct lbmgpu_surrogate_report {
    long samples;             /* rows in the sample set                                   */
    long train_steps;         /* Adam steps so far                                        */
    double last_loss;         /* last epoch's mean standardised squared error             */
    long cells_predicted;     /* cell updates taken from the network                      */
    long cells_integrated;    /* cell updates the gate sent to the integrator             */
    long cells_audited;       /* cell updates integrated to score the network             */
    double audit_rel_err;     /* over the audited cells: sum |dY_net - dY_int|_1 / sum |dY_int|_1 */
    double audit_max_abs_err; /* largest |dY_net - dY_int|_1 of an audited cell           */
    double audit_dY;          /* sum |dY_int|_1 over the audited cells                   */
    int enabled, collecting;
} lbmgpu_surrogate_report;
int lbmgpu_surrogate_collect(lbmgpu_t *h, int enable, int stride, long capacity);
int lbmgpu_surrogate_load_samples(lbmgpu_t *h, const float *x, const float *y, long n);
int lbmgpu_surrogate_samples(lbmgpu_t *h, float *x, float *y, unsigned char *valid, long n);
int lbmgpu_surrogate_augment(lbmgpu_t *h, long n, float span_y, float span_t, float y_trace, unsigned seed);
int lbmgpu_surrogate_train(lbmgpu_t *h, int epochs, int batch, float lr, unsigned seed, int refit, double *loss);
int lbmgpu_surrogate_enable(lbmgpu_t *h, int enable, int audit_period);
int lbmgpu_surrogate_eval(lbmgpu_t *h, const float *x, long n, float *y);
int lbmgpu_surrogate_params(lbmgpu_t *h, float *buf, long n, int set);
int lbmgpu_surrogate_stats(lbmgpu_t *h, lbmgpu_surrogate_report *out);
/* The gradients of the loss with respect to every weight and bias over the last minibatch of
 * the last lbmgpu_surrogate_train call (computed by the tensor-core backward kernels, before
 * that minibatch's Adam step), packed as lbmgpu_surrogate_params packs the parameters; the
 * standardisation entries are 0.  LBMGPU_E_STATE before any training step. */
int lbmgpu_surrogate_grads(lbmgpu_t *h, float *buf, long n);

/* ---- restart and field output from the device state --------------------------------
 * lbmgpu_write_restart / lbmgpu_read_restart: the reference's restart file
 * (write_restart / read_restart, src/restart_file.cpp:274-440), records in the caller's
 * MIXTURE / SPECIES layout of the descriptor.  The header's dx, dy, dz, step and Ra
 * (single component) or permeability (multicomponent) come from / go to `info`; Nx, Ny, Nz,
 * dt_sim, the species count and names must match the handle (else LBMGPU_E_ARG).  Written
 * from the device state between time steps (as a download would return it: fluid cells
 * whole, other cells their stored moments and type); read back as an upload (the next
 * Collide continues from it, as the reference's run does after read_restart).
 * Multicomponent files are streamed a few x-planes at a time. */
typedef struct lbmgpu_restart_info {
    int dx, dy, dz;          /* LBM::dx, dy, dz (src/headers/lbm.hpp:107)               */
    int step;                /* the time step the state belongs to                        */
    double Ra;               /* single component: LBM::Ra                                 */
    double permeability;     /* multicomponent: LBM::permeability                         */
} lbmgpu_restart_info;
int lbmgpu_write_restart(lbmgpu_t *h, const char *path, const lbmgpu_restart_info *info);
int lbmgpu_read_restart(lbmgpu_t *h, const char *path, lbmgpu_restart_info *info);

/* lbmgpu_write_vtk: the reference's OutputVTK file (src/output.cpp:9-210, a VTK
 * RectilinearGrid with raw appended Float32 data) of the current state, byte for byte: the
 * cell arrays are packed on the device and copied to the host once.  flags:
 * LBMGPU_VTK_SI converts to SI units as the reference's OUTPUT_SI build does
 * (multicomponent handles, whose descriptor carries the units), LBMGPU_VTK_MASSFRAC writes
 * mass fractions as its OUTPUT_MASSFRAC build does (mole fractions otherwise).  dx: the
 * reference's LBM::dx (the coordinates are i * dx).
 * lbmgpu_vtk_fields: the packed cell arrays alone -- density, velocity (3 per cell), cell
 * type, temperature, pressure, then multicomponent HRR, the species fractions and the
 * species x velocities relative to the mixture, each Nx*Ny*Nz values in x-fastest order;
 * n_out >= (7 or 10 + 2 n_species) * Nx*Ny*Nz. */
#define LBMGPU_VTK_SI 1
#define LBMGPU_VTK_MASSFRAC 2
int lbmgpu_write_vtk(lbmgpu_t *h, const char *path, int dx, int flags);
int lbmgpu_vtk_fields(lbmgpu_t *h, float *out, size_t n_out, int flags);

/* Bytes of device memory held by the handle. */
int lbmgpu_device_bytes(lbmgpu_t *h, size_t *bytes);

const char *lbmgpu_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif /* LBMGPU_H */
