/* clb200.h - C ABI of the B200 lattice time-evolution library (libclb200.so).
 *
 * The reference has no FFI: its operator interface is the compile-time C++ template API
 *   Evolver<Model>::Evolver / evolve / sync      (include/CosmoInterface/evolvers/evolver.h:45,102,132)
 *   ModelInitializer<T>::initialize              (include/CosmoInterface/initializers/modelinitializer.h:47-81)
 *   Measurer<Model,T>::measure                   (include/CosmoInterface/measurements/measurer.h:87-178)
 * all called only from main (source/cosmolattice.cpp:134-188).  Each entry point below replaces
 * one of those calls (cited per function).  Everything crossing this boundary is a plain C type:
 * host arrays in, host arrays out; the library owns all device memory.
 *
 * Error convention: every int-returning function returns CLB_OK (0) or a negative CLB_E* code and
 * records a message readable with clb_last_error().  No C++ exception crosses the boundary.
 * Calls on one handle are not thread-safe; distinct handles are independent.
 */
#ifndef CLB200_H
#define CLB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------- */
#define CLB_OK            0
#define CLB_EINVAL       -1 /* bad argument / inconsistent parameters (RunParametersInconsistent) */
#define CLB_ECUDA        -2 /* CUDA runtime or cuFFT error */
#define CLB_ENOMEM       -3 /* device allocation failed */
#define CLB_ENONFINITE   -4 /* a volume average became NaN/Inf */
#define CLB_ETIMEOUT     -5 /* a bounded device-side wait gave up */
#define CLB_EUNSUPPORTED -6 /* combination not implemented (EvolverTypeNotInEvolver, ...) */
#define CLB_ESTATE       -7 /* call out of order (e.g. evolve before initialize) */

/* ---- evolver ids: same numbering as the reference enum EvolverType (evolvertype.h:37) ------ */
#define CLB_LF     0
#define CLB_VV2    1
#define CLB_VV4    2
#define CLB_VV6    3
#define CLB_VV8    4
#define CLB_VV10   5
#define CLB_VV6_2  6
/* position Verlet, PositionVerlet (positionverlet.h:45-99, positionverletparameters.h:23-46);
   every model; the adjoint pair and the tangent-linear form take the VV and LF evolvers */
#define CLB_PV2    11
#define CLB_PV4    12
#define CLB_PV6    13
#define CLB_PV8    14
#define CLB_PV10   15
#define CLB_PV6_2  16

/* ---- arithmetic forms -------------------------------------------------------------------- */
#define CLB_PREC_FP64       0 /* fields, momenta, stencils, reductions and expansion in FP64 */
#define CLB_PREC_FP32_SPLIT 1 /* fields/momenta/stencils FP32; reductions, a(t), constraints FP64 */

/* ---- sweep schedule ---------------------------------------------------------------------- */
#define CLB_PATH_FUSED     0 /* one drift+kick+averages sweep per VV stage (default)             */
#define CLB_PATH_REFERENCE 1 /* the reference's operation order: kick, <pi^2>, drift, <grad^2>,<V>,
                                kick, <pi^2> as separate sweeps (velocityverlet.h:69-113)           */

/* ---- models ---------------------------------------------------------------------------------
 * The model is chosen when the handle is created, as the reference chooses it at compile time
 * (CMakeLists.txt:133-146).  Couplings are in program units.
 *   CLB_MODEL_LPHI4   : n_scalars = 1 or 2 real singlets,
 *                       V = c[0]/4 phi^4 + c[1]/2 phi^2 chi^2            (models/lphi4.h:154-177,
 *                       with c[0] = 1 and c[1] = q reproducing the reference header exactly).
 */
#define CLB_MODEL_LPHI4 1
/*   CLB_MODEL_LPHI4U1 : one complex scalar charged under one U(1) gauge field (models/lphi4U1.h),
 *                       V = c[0] |phi|^4 (c[0] = 1 is the reference header), c[1] = g Q, the effective
 *                       charge (CouplingsManager, couplingsmanager.h:167-218).  Components, fields and
 *                       momenta alike: Re phi, Im phi, A_1, A_2, A_3 (program units; n_scalars = 0). */
#define CLB_MODEL_LPHI4U1 2
#define CLB_MODEL_LPHI4SU2U1 3

#define CLB_MAX_COUPLINGS 8

typedef struct clb_config {
  int32_t N;          /* lattice points per dimension (RunParameters::N, runparameters.h:61)     */
  double dx;          /* lattice spacing in program units (= 2 pi / (N kIR), runparameters.h:179-180) */
  double dt;          /* time step (runparameters.h:64)                                         */
  int32_t evolver;    /* CLB_LF, CLB_VV2 ... (runparameters.h:102)                              */
  int32_t expansion;  /* 1: self-consistent expansion, 0: none (runparameters.h:66)             */
  int32_t precision;  /* CLB_PREC_*                                                             */
  int32_t path;       /* CLB_PATH_*                                                             */
  int32_t device;     /* CUDA device ordinal                                                    */
  /* Fixed background (runparameters.h:90-94; with expansion only; every model, not the adjoint
   * pair or the tangent-linear form):
   * a(t) = (1 + H0/p (t - t0))^p, aDot = H0 (1 + H0/p (t - t0))^(p - 1),
   * p = 2 / (3 (1 + omega_eos) - 2 alpha)  (FixedBackgroundExpansion, fixedbackgroundexpansion.h:21-50) */
  int32_t fixed_background; /* 0: self-consistent expansion (default), 1: fixed background           */
  double omega_eos;         /* equation of state w                                                  */
  double H0;                /* initial Hubble rate in program units (H0 / omega_*)                  */
  double t0;                /* initial time (runparameters.h:68); t advances by dt per step         */
} clb_config;

typedef struct clb_model_desc {
  int32_t kind;       /* CLB_MODEL_*                                                            */
  int32_t n_scalars;  /* Ns  (abstractmodel/scalarbase.h)                                       */
  double alpha;       /* time-rescaling exponent (abstractmodel/modelparametersbase.h)          */
  double fStar;       /* field rescaling f_*                                                    */
  double omegaStar;   /* frequency rescaling omega_*                                            */
  double MPl;         /* reduced Planck mass in the same units as fStar (scalefactorbase.h:18)  */
  double couplings[CLB_MAX_COUPLINGS];
} clb_model_desc;

/* Scale-factor state in program units (abstractmodel/scalefactorbase.h:20-21). */
typedef struct clb_scalefactor {
  double aI, aSI, aIM;       /* a at integer time, at the half step, at the previous integer time */
  double aDotI, aDotSI, aDotSIM;
} clb_scalefactor;

#define CLB_MAX_ENERGIES 32
#define CLB_MAX_MEANS 8

/* One measurement at the current (synchronised) time.
 *  energies[] holds the columns of the reference's average_energies.txt after "t", in its order
 *  (energiesmeasurer.h:45-101, headers :127-150): for each scalar singlet E^kin, E^grad; then each
 *  potential term <V_k>; then E_tot.
 *  friedmann[] holds (LHS-RHS)/(LHS+RHS), LHS, RHS with expansion (hubbleconstraint.h:27-36), or
 *  energy_cons = |1 - E/E0| in friedmann[0] without expansion (energiesmeasurer.h:116-118).
 *  means[f][] per scalar singlet: <phi>, <dphi/dt>, <phi^2>, <(dphi/dt)^2>, rms(phi), rms(dphi/dt)
 *  with dphi/dt = a^(alpha-3) pi (meansmeasurer.h:28-48, scalarsingletmeasurer.h:61-66).
 *  For CLB_MODEL_LPHI4U1 the rows are: sqrt2 Re phi, sqrt2 Im phi, |phi| (with their momenta
 *  a^(alpha-3) pi), then |E| = |a^(alpha-1) pi_A| and |B| (complexscalarmeasurer.h:61-72,
 *  u1measurer.h:78-87); energies: E^kin_cmplxscal0, E^grad_cmplxscal0, E^kin_U10, E^grad_U10, <V>,
 *  E_tot (energiesmeasurer.h:62-90). */
typedef struct clb_measurement {
  double aI, aDotI, hubble;            /* scalefactormeasurer.h:37-48 */
  int32_t n_energies;
  double energies[CLB_MAX_ENERGIES];
  double friedmann[3];
  int32_t n_means;
  double means[CLB_MAX_MEANS][6];
  /* GaussLaws::checkU1 (gausslaws.h:34-53): av|LHS-RHS| / av|LHS^2 sum + RHS^2|, av|LHS|, av|RHS| */
  double gauss_u1[3];
  double gauss_su2[3];  /* lphi4SU2U1: checkSU2 (gausslaws.h:56-80), same three numbers as gauss_u1 */
} clb_measurement;

typedef struct clb_handle clb_handle;

/* Library version string. */
const char *clb_version(void);

/* Message of the last failed call on `h`; h == NULL gives the last failure of clb_create on the
 * calling thread. */
const char *clb_last_error(const clb_handle *h);

/* Allocate a lattice and its device state.  Replaces the Model constructor's field allocation
 * (abstractmodel.h:147-186, via MemoryToolBox::makeShared, source/cosmolattice.cpp:82-93) and the
 * Evolver constructor's validation (evolvers/evolver.h:45-98). */
int clb_create(const clb_config *cfg, const clb_model_desc *model, clb_handle **out);
void clb_destroy(clb_handle *h);

/* Number of real N^3 component arrays in the field and momentum buffers of clb_set_state. */
int clb_num_components(const clb_handle *h, int32_t *n_field_components, int32_t *n_momentum_components);

/* Upload a state from host memory.  fields: n_field_components x N^3 doubles, momenta likewise,
 * each component row-major (x slowest, z fastest); order: scalar singlets 0..Ns-1.  The scale
 * factor state sf may be NULL (a = 1, aDot = 0).  Mirrors the end state of the field-filling part
 * of ModelInitializer::initialize (modelinitializer.h:54-69). */
int clb_set_state(clb_handle *h, const double *fields, const double *momenta, const clb_scalefactor *sf);

/* Initial state generated on the device (replaces the host generator; the reference's
 * ModelInitializer::initialize field part, modelinitializer.h:51-69): fluctuations by
 * FluctuationsGenerator::conjugateGaussianFluctuations for singlets (fluctuationsgenerator.h:39-71,
 * 130-150), U1Initializer::addFluctuationsCScalarFromPhases for the complex scalar
 * (u1initializer.h:157-230), SU2Initializer::addFluctuationsSU2DoubletFromPhases for the doublet
 * (su2initializer.h:115-186); gauge momenta from the Gauss laws with A = 0 and unit links
 * (u1initializer.h:90-114, su2initializer.h:65-85); then the homogeneous parts.  Random numbers:
 * Philox4x64-10 with key (seed, stream) and counter (mode index, 0, 0, 0); the kz = 0 and N/2
 * planes are Hermitian.  Matter components in the model's field order: lphi4 singlets 0..Ns-1;
 * lphi4U1 Re phi, Im phi; lphi4SU2U1 S, Re phi, Im phi, Phi_1..Phi_4.  sf as in clb_set_state. */
#define CLB_IC_MAX 8
typedef struct clb_ic_params {
  uint64_t seed;
  double amplitude;          /* omega_* / f_* in the reference (fluctuationsgenerator.h:91-98)      */
  double k_cutoff;           /* modes with |k| > k_cutoff (program units) are 0                     */
  double adot;               /* aDot of the homogeneous background, in pi_k = ... - aDot phi_k       */
  double mass2[CLB_IC_MAX];  /* m^2 per matter component (program units); omega_k = sqrt(k^2 + max(m^2, 0)) */
  double fld0[CLB_IC_MAX];   /* homogeneous field values (program units)                             */
  double pi0[CLB_IC_MAX];    /* homogeneous momenta (program units)                                  */
  double charge[4];          /* lphi4U1: g Q; lphi4SU2U1: g Q of the doublet under SU(2), g Q of the
                                complex scalar and of the doublet under U(1)                         */
} clb_ic_params;
int clb_generate_state(clb_handle *h, const clb_ic_params *p, const clb_scalefactor *sf);

/* Download the state (fields, momenta may be NULL to skip). */
int clb_get_state(clb_handle *h, double *fields, double *momenta, clb_scalefactor *sf);

/* Finish initialisation: volume averages of the state (Averages::setAllAverages, averages.h:349-392),
 * and with self-consistent expansion aDot_I = sqrt(Friedmann RHS) if correct_adot == 1
 * (modelinitializer.h:74-80).  Then applies the evolver constructor: for LF,
 * aDot_SI = aDot_I - dt/2 F (leapfrog.h:35) and the synced flag.
 * correct_adot == CLB_INIT_RESTART: the state is a restarted one (SimulationManager::loadSim,
 * simulationmanager.h:69-100, then the evolver's constructor with doWeRestart set): averages only,
 * no aDot correction, and the leapfrog starts unsynced, its momenta at the half step
 * (leapfrog.h:30-36); not with a fixed background (CLB_EUNSUPPORTED). */
#define CLB_INIT_RESTART 2
int clb_initialize(clb_handle *h, int32_t correct_adot);

/* Advance n_steps time steps of dt: n_steps calls of Evolver::evolve (evolver.h:102-124). */
int clb_evolve(clb_handle *h, int64_t n_steps);

/* Evolver::sync (evolver.h:132-155): LF half-kicks the momenta to integer time; VV: no-op. */
int clb_sync(clb_handle *h);

/* Energies, Friedmann constraint and means at the current state (EnergiesMeasurer::measure,
 * MeansMeasurer::measure, ScaleFactorMeasurer::measure).  Call after clb_sync.  e0 is the initial
 * total energy used for energy_cons without expansion (ignored with expansion). */
int clb_measure(clb_handle *h, double e0, clb_measurement *out);

/* Radially binned power spectrum of scalar component `comp` at the current state
 * (PowerSpectrumMeasurer::powerSpectrum, measurements/powerspectrum.h:84-134, as called from
 * ScalarSingletMeasurer::measureSpectra, scalarsingletmeasurer.h:74-83).
 *   which: 0 the field, 1 the momentum (times a^(2 alpha - 6), scalarsingletmeasurer.h:80).
 *   ps_type: 1 (sum over the bin x kIR n dx / dk / N^5 / 2 pi) or 2 (bin average x (kIR n dx / N)^3
 *            / dk / 2 pi^2), the reference's PS_type (runparameters.h:119).
 *   ps_version: 1 n = the bin's mean |n| over its modes, 2 n = the bin centre (b + 1/2) dk.
 *   Bins: b = floor(|n| / dk) over the full N^3 grid of integer wave vectors n; modes with b >= nbins
 *   go to the last bin if fold != 0, else they are not counted.  The reference's default is
 *   nbins = floor(sqrt(3)/2 N / dk) with every mode counted (fold = 1; runparameters.h:98).
 * Outputs per bin: k_out = n kIR (may be NULL), value_out, count_out = number of modes (may be NULL).
 * The transform is cuFFT D2Z in FP64 for either storage precision. */
int clb_spectrum(clb_handle *h, int32_t which, int32_t comp, int32_t ps_type, int32_t ps_version, double dk,
                 int32_t nbins, int32_t fold, double *k_out, double *value_out, int64_t *count_out);

/* ---- per-step results and instrumentation (no reference counterpart: the reference writes these
 *      averages to text files at its output cadence, measurer.h:87-121) -------------------------- */

/* Columns of one history row: a, aDot, <pi^2>, <grad^2>, <V> at the end of each step. */
#define CLB_HIST_COLS 5

/* Rows recorded by the last clb_evolve (one per step; only with self-consistent expansion, where
 * the averages are formed during the evolution).  Copies min(max_rows, rows) rows into out (may be
 * NULL) and stores the number of rows in *n_rows. */
int clb_history(clb_handle *h, double *out, int64_t max_rows, int64_t *n_rows);

typedef struct clb_kernel_stat {
  char name[40];
  int64_t launches;       /* launches since the last reset                          */
  int64_t timed_launches; /* launches bracketed by CUDA events while profiling was on */
  double total_ms;        /* summed event time of the timed launches                */
} clb_kernel_stat;

/* Per-launch CUDA events on the handle's stream (on != 0), collected at each synchronising call. */
int clb_set_profiling(clb_handle *h, int32_t on);
int clb_reset_stats(clb_handle *h);
/* Fills up to max entries, one per kernel kind; *n = number of kinds. */
int clb_kernel_stats(clb_handle *h, clb_kernel_stat *out, int32_t max, int32_t *n);
/* Device time of the last clb_evolve call, from events recorded on its stream around its launches. */
int clb_last_evolve_ms(clb_handle *h, double *ms);
/* The cudaStream_t the handle launches on (for callers that order their own work after it). */
void *clb_cuda_stream(clb_handle *h);

/* ---- adjoint (reverse-mode) pair ----------------------------------------------------------------
 * No counterpart in the reference, which has no differentiation.  Replaces, for gradient studies,
 * a caller's finite-difference loop around Evolver::evolve (evolvers/evolver.h:102-127) and
 * EnergiesMeasurer::measure (measurements/energiesmeasurer.h:45-122).
 *
 * clb_forward runs nsteps VV or leapfrog steps from the current (initialized) state, storing the
 * full state every checkpoint_every steps (the leapfrog then syncs, LeapFrog::sync
 * evolvers/leapfrog.h:96-116, so that O is taken at integer-time momenta), and returns the
 * observable
 *     O = sum_k w_k E_k / E_tot
 * over the energy components E_k in clb_measurement order without E_tot (lphi4U1: E_kin and
 * E_grad of the complex scalar, E_el, E_mag, V; n_weights <= 5).  clb_backward then returns dO
 * with respect to the state at the forward's start (fields_bar, momenta_bar: same layout as
 * clb_set_state; either may be NULL), to the scale factor there, and to the couplings through
 * their explicit appearance in the evolution.  With through_init = 1 the start state is taken as
 * made by clb_initialize(h, 1), whose aDot = sqrt(Friedmann RHS) is differentiated as well (the
 * aDot cotangent is then 0).  The backward pass recomputes each segment from its checkpoint;
 * device memory: (nsteps/checkpoint_every + 1) states plus checkpoint_every x stages + 1 states
 * (stages: 1 for the leapfrog).  lphi4U1 with the VV evolvers and the leapfrog; the position
 * Verlet, a fixed background and other models return CLB_EUNSUPPORTED.  A leapfrog forward that
 * starts right after clb_initialize differentiates its first step's <pi^2> of the previous half
 * step (the start momenta's) and the initial aDot_{-1/2} = aDot_0 - dt/2 F (leapfrog.h:35);
 * started later, that stored average is a constant and dO_dscalefactor[1] is the cotangent of the
 * stored half-step aDot.  After clb_backward the handle holds the forward's end state again. */
typedef struct clb_adjoint_grad {
  double observable;         /* O of the forward pass                                       */
  double dO_dcouplings[8];   /* clb_model_desc.couplings order (lphi4U1: [0] c4, [1] gQ)     */
  double dO_dscalefactor[2]; /* aI, aDotI at the forward's start (0 without expansion)      */
} clb_adjoint_grad;

int clb_forward(clb_handle *h, int64_t nsteps, int32_t checkpoint_every, const double *weights, int32_t n_weights,
                double *observable);
int clb_backward(clb_handle *h, int32_t through_init, double *fields_bar, double *momenta_bar, clb_adjoint_grad *grad);
/* clb_forward with the observable O = sum_b w_b P_b, P the binned spectrum of clb_spectrum (same
 * arguments) of one component at the end state, w one weight per bin; clb_backward then returns
 * dO (the momentum spectra's a-factor differentiated too).  lphi4U1. */
int clb_forward_spectrum(clb_handle *h, int64_t nsteps, int32_t checkpoint_every, int32_t which, int32_t comp,
                         int32_t ps_type, int32_t ps_version, double dk, int32_t nbins, int32_t fold,
                         const double *bin_weights, double *observable);

/* ---- tangent-linear (forward-mode) form ---------------------------------------------------------
 * No counterpart in the reference.  Replaces a caller's central-difference pair of runs around
 * Evolver::evolve (evolvers/evolver.h:102-127) and EnergiesMeasurer::measure
 * (measurements/energiesmeasurer.h:45-122) for the derivative with respect to one coupling.
 *
 * clb_tangent_begin sets the direction: the derivatives of the couplings (clb_model_desc order;
 * lphi4SU2U1: qG, qH, gQ of phi, gQ of Phi under U(1), gQ of Phi under SU(2), c4; missing ones
 * 0), and the tangent of the current state along it (same layouts as clb_set_state; NULL: zero).
 * d/d g_SU2 is couplings_dot = {0, 0, 0, 0, Q_SU2}; d/d g_U1 is {0, 0, Q_phi, Q_Phi}.  From then on
 * clb_initialize, clb_evolve and clb_sync advance the state exactly as without it and its tangent
 * alongside (the scale factor's too, through the self-consistent expansion), in one pass with no
 * checkpoints; clb_measure refreshes the cached averages of both.  clb_tangent_observable returns
 *     O = sum_k w_k E_k / E_tot,  E_k = E_kin, E_grad of S, phi, Phi; E_el, E_mag of U(1) and SU(2); V
 * (n_weights <= 11) and its derivative along the direction at the current state.  clb_set_state
 * or clb_tangent_end ends the form.  lphi4SU2U1 only (other models: CLB_EUNSUPPORTED); device
 * memory: one more state. */
int clb_tangent_begin(clb_handle *h, const double *couplings_dot, int32_t n_couplings, const double *fields_dot,
                      const double *momenta_dot, const clb_scalefactor *sf_dot);
int clb_tangent_get_state(clb_handle *h, double *fields_dot, double *momenta_dot, clb_scalefactor *sf_dot);
int clb_tangent_observable(clb_handle *h, const double *weights, int32_t n_weights, double *observable,
                           double *d_observable);
/* The 11 energies E_k of clb_tangent_observable and their derivatives (either array may be NULL). */
int clb_tangent_energies(clb_handle *h, double *energies, double *d_energies);
/* clb_spectrum of one component and, in d_value_out, its derivative along the direction (the
 * momentum spectra's a-factor included). */
int clb_tangent_spectrum(clb_handle *h, int32_t which, int32_t comp, int32_t ps_type, int32_t ps_version, double dk,
                         int32_t nbins, int32_t fold, double *k_out, double *value_out, double *d_value_out,
                         int64_t *count_out);
int clb_tangent_end(clb_handle *h);

/* ---- batched ensemble ----------------------------------------------------------------------------
 * No counterpart in the reference (one lattice per process, source/cosmolattice.cpp:134-201).  Many
 * independent one-field lphi4 lattices (model kind CLB_MODEL_LPHI4, n_scalars 1) advance together:
 * one sweep launch per VV stage covers every member, each member keeps its own scale factor and
 * volume averages, and clb_batch_evolve runs as one CUDA graph.  Members share dt, evolver (VV
 * family), expansion mode, precision and device, and differ in N (2..1024), dx, couplings[0] and
 * state.  Member arrays are N^3 doubles as in clb_set_state; measurements as clb_measure. */
typedef struct clb_batch clb_batch;

int clb_batch_create(const clb_config *cfgs, const clb_model_desc *mds, int32_t n, clb_batch **out);
void clb_batch_destroy(clb_batch *b);
const char *clb_batch_last_error(const clb_batch *b);
int clb_batch_set_state(clb_batch *b, int32_t i, const double *fields, const double *momenta, const clb_scalefactor *sf);
int clb_batch_get_state(clb_batch *b, int32_t i, double *fields, double *momenta, clb_scalefactor *sf);
int clb_batch_initialize(clb_batch *b, int32_t correct_adot);
int clb_batch_evolve(clb_batch *b, int64_t nsteps);
int clb_batch_measure(clb_batch *b, int32_t i, double e0, clb_measurement *m);
int clb_batch_last_evolve_ms(clb_batch *b, double *ms);
int clb_batch_kernel_launches(clb_batch *b, int64_t *n);

/* Sweep configuration of the ensemble: the (z, y) tile of one sweep block, the z sites each
 * thread owns (vector loads; every member's N a multiple of it) and the x-planes each block
 * marches over.  The first clb_batch_evolve of a handle times every compiled block shape (tile z x
 * y x sites per thread: 32x4x1, 32x8x1, 32x16x1, 64x4x1, 32x8x2, 32x16x2, 64x8x2, 32x16x4, 32x32x4,
 * 64x8x4, 64x16x4) with x-runs of 8, 16, 32, 64 and N planes on the ensemble itself and keeps the
 * fastest (environment CLB_BATCH_AUTOTUNE=0: keep 32x8x1, 32 planes); later handles of the same
 * ensemble shape in the process reuse it.  clb_batch_autotune reruns it (reps timed sweeps per
 * candidate); clb_batch_set_tuning fixes a configuration.  The fields do not depend on it; the
 * volume sums are summed in a configuration-dependent order. */
typedef struct clb_batch_tuning {
  int32_t tile_z, tile_y;    /* sites of one sweep block's tile along z and y                 */
  int32_t sites_per_thread;  /* consecutive z sites per thread                                */
  int32_t planes_x;          /* x-planes per block                                            */
  int32_t candidates;        /* configurations timed (0: set, cached or default)              */
  double ms_per_sweep;       /* its time for one fused stage sweep of all members             */
  double ms_default;         /* the same for 32x8x1 tiles with 32-plane runs                  */
} clb_batch_tuning;

int clb_batch_autotune(clb_batch *b, int32_t reps, clb_batch_tuning *out);
int clb_batch_set_tuning(clb_batch *b, int32_t tile_z, int32_t tile_y, int32_t sites_per_thread, int32_t planes_x);
int clb_batch_get_tuning(clb_batch *b, clb_batch_tuning *out);

/* The form an evolve call takes.  Per-stage form: one sweep and one tail launch per VV stage,
 * captured as one CUDA graph per call (the tile of clb_batch_tuning).  Persistent form: the whole
 * call is one launch of thread-block clusters (cluster_blocks blocks each, co-scheduled), each
 * cluster taking its members, longest first to the least-loaded cluster, through every step; per
 * stage the cluster sweeps a member's tiles, synchronises on the hardware cluster barrier and
 * applies the member's scale-factor update from its sums in a fixed order.  The call is captured
 * as a one-launch graph.  There is no software wait in it (no flags, no spins).
 * The autotuner (clb_batch_autotune, or the first evolve) times whole 8-step calls of both forms
 * from a snapshot of the state, which it restores, and keeps the faster; CLB_BATCH_PERSISTENT=0 or
 * 1 in the environment fixes the form.  clb_batch_set_tuning selects the per-stage form,
 * clb_batch_set_persistent the persistent form with the given tile: (tile_z, tile_y,
 * sites_per_thread) one of (32, 8, 1), (32, 8, 2), (64, 8, 4) and (32, 4, 1), with planes_x
 * x-planes per tile.  The fields do not depend on the form; the volume sums are summed in a
 * form-dependent order. */
typedef struct clb_batch_form {
  int32_t persistent;        /* 1: persistent form, 0: per-stage graph form                   */
  int32_t tile_z, tile_y;    /* persistent form's tile (0 in the per-stage form)              */
  int32_t sites_per_thread;
  int32_t planes_x;
  int32_t clusters;          /* clusters launched                                             */
  int32_t cluster_blocks;    /* blocks per cluster                                            */
  int32_t candidates;        /* persistent configurations timed (0: set, cached or default)   */
  double ms_graph;           /* per step, timed by the autotuner (0: not timed)               */
  double ms_persistent;      /* per step, the fastest persistent configuration (0: not timed) */
} clb_batch_form;

int clb_batch_set_persistent(clb_batch *b, int32_t tile_z, int32_t tile_y, int32_t sites_per_thread, int32_t planes_x);
int clb_batch_get_form(clb_batch *b, clb_batch_form *out);

/* ---- gravitational waves -------------------------------------------------------------------------
 * The GW sector of the reference (GWsKernels::get, evolvers/kernels/gwskernels.h:27-33; the
 * sources of PITensor.h: scalar singlets, complex scalars through their U(1) covariant forward
 * differences, U(1) electric and magnetic fields; Evolver::evolve/sync with the default
 * doLFforGWs, a leapfrog staggered over the matter evolver, evolvers/evolver.h:102-138;
 * GWsInitializer, zero at the start).  The field is the traceless symmetric u_ij as five
 * components (u_11, u_12, u_13, u_22, u_23; u_33 = -u_11 - u_22), its momenta likewise.
 * clb_gws_enable: after clb_create, before clb_initialize; every model, evolver and expansion (the
 * scalar singlets on the fused path; else CLB_EUNSUPPORTED).
 * A gauge handle with GWs takes no clb_forward and no clb_tangent_begin (CLB_EUNSUPPORTED), and
 * the reverse.
 * clb_gws_set_state / clb_gws_get_state: 5 x N^3 doubles each (either may be NULL).
 * clb_gw_spectrum: the GW energy spectrum d(rho_GW/rho)/dlog k (PowerSpectrumMeasurer::
 * powerSpectrumGW, measurements/powerspectrum.h:51-71) with the TT projector of
 * GWProjectorType1/2/3 (definitions/gwsprojector.h; prj_type 1, 2 or 3), the bins and PS_type /
 * PS_version of clb_spectrum; rho_gw_over_rho (may be NULL): its sum over the bins times
 * dk / k (GWsMeasurer, measurements/gwsmeasurer.h:41-53).  Measures the energies first, as the
 * reference's Energies::rho does (which refreshes the cached averages).  Call it after clb_sync. */
int clb_gws_enable(clb_handle *h);
int clb_gws_set_state(clb_handle *h, const double *u, const double *pi);
int clb_gws_get_state(clb_handle *h, double *u, double *pi);
int clb_gw_spectrum(clb_handle *h, int32_t prj_type, int32_t ps_type, int32_t ps_version, double dk, int32_t nbins,
                    int32_t fold, double *k_out, double *value_out, int64_t *count_out, double *rho_gw_over_rho);

/* ---- allocation-free entry point (no counterpart in the reference) ----------------------------
 * For callers that cannot call cudaMalloc: a host runtime that owns the whole device memory pool
 * and hands out no more, or an embedding that forbids device allocation after start-up (a service
 * with a fixed memory budget).  Computes, for FP64 scalar-singlet lattices already in device memory, the volume
 * averages d_out[0] = <sum_f pi_f^2>, d_out[1] = <sum_f grad^2 phi_f>, d_out[2] = <V> (lphi4:
 * V = c0/4 phi^4 + q/2 phi^2 chi^2), the same sums clb_initialize and clb_measure form.
 * d_fields / d_momenta: n_scalars x N^3 doubles each (layout of clb_set_state) on the current
 * device; d_out: 3 doubles on the same device; stream: a cudaStream_t or NULL.
 * Allocates nothing: the block partials live in a fixed 192 KiB device array that every GPU
 * loading the library keeps until exit, so N is limited to 1024 (larger N returns CLB_EINVAL with
 * the reason in clb_last_error(NULL)).  The first call on a device looks up that array's address
 * (cudaGetSymbolAddress) with the device current, and again in a new context after a
 * cudaDeviceReset; make that first call before any stream capture.  A CUDA error left pending by
 * earlier work is reported (CLB_ECUDA) and left in place.  Calls return once their work is enqueued.  All calls share the array: calls that overlap on the
 * GPU (other streams or host threads) race and must be serialised by the caller. */
int clb_scalar_averages_noalloc(const double *d_fields, const double *d_momenta, int32_t N, int32_t n_scalars,
                                double dx, double c0, double q, double *d_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CLB200_H */
