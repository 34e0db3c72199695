/* tiger_chem.h -- C-ABI of the B200 finite-rate chemistry path (sm_100a).
 *
 * A drop-in for the finite-rate chemistry substep of the NGA/ARTS low-Mach solver. The
 * reference exposes two Fortran ABIs on this path (external linkage, arguments by
 * reference):
 *   - the substep  finitechem_source_chemistry(RHO_, SC_)    combustion/finitechem.f90:962-1071
 *   - the mechanism plugin  PRODRATES / COMPTHERMODATA / GETMOLARMASS / GETSPECIESNAMES /
 *     GETNSPECIES / GETNREACTIONS                            combustion/mechanism.f90:17-108
 * and, around the substep, the per-cell mixture properties (finitechem_density / _W /
 * _viscosity / _diffusivity, finitechem.f90:65-74, :324-487) and the solver-state data files
 * (core/data.f90:217-457), which have entry points here too.
 * Every entry point here takes plain pointers and sizes, returns an int status (0 = OK,
 * negative = error; tng_last_error() gives the message) and is callable from Fortran through
 * ISO_C_BINDING (see fortran/tiger_chem_gpu.f90).
 *
 * Threading: one handle per host thread; a handle owns one CUDA stream on its device.
 * No entry point falls back to the CPU: without a usable sm_100 device tng_chem_create fails.
 */
#ifndef TIGER_CHEM_H
#define TIGER_CHEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TNG_OK 0
#define TNG_ERR_ARG (-1)
#define TNG_ERR_CUDA (-2)
#define TNG_ERR_MECH (-3)
#define TNG_ERR_STATE (-4)

/* Precision of the rate evaluation. */
#define TNG_FP64 0  /* everything FP64 (agrees with the reference within 1e-10 relative) */
#define TNG_MIXED 1 /* FP32 rate products in log2 space, FP64 reverse exponents/sums/thermo */

/* Literal kinds of the mechanism constants. */
#define TNG_LIT_REF 0 /* as the reference build: default-real literals rounded to float32 */
#define TNG_LIT_F64 1 /* every literal read as a double */

/* Pointer location flags for batch calls. */
#define TNG_DEVICE_PTRS 0 /* arrays live in device memory (the fast path) */
#define TNG_HOST_PTRS 1   /* arrays live in host memory; copied through pinned staging */

typedef struct tng_cfg {
  int precision;    /* TNG_FP64 | TNG_MIXED */
  int literal_mode; /* TNG_LIT_REF | TNG_LIT_F64 */
  int device;       /* CUDA device ordinal */
  double rtol;      /* relative tolerance ('Finitechem rel. tol.', finitechem.f90:266, default 1e-6) */
  double atol;      /* absolute tolerance ('Finitechem abs. tol.', finitechem.f90:267, default 1e-12) */
  int max_steps;    /* internal steps per cell and substep (MAX_NSTEPS, finitechem.f90:1025) */
  int max_newton;   /* Newton iterations per internal step before the step is retried */
  int block_size;   /* threads per block of the rate kernel, 0 = tuned default */
  int rate_variant; /* rate-kernel variant (0 plain, 1 block-synchronised, 2 + register cap), -1 = tuned */
  int solver_warps; /* cells (warps) per block of the implicit solver: 2, 4 or 8; 0 = tuned */
  int pass_budget;  /* internal steps per cell and solver pass before the cell is re-queued; 0 = no limit */
  int max_passes;   /* passes captured in the solver's CUDA graph (the last one has no budget) */
  int solver_occupancy; /* solver blocks per SM targeted by its launch bounds (with 8 warps): 1, or 2
                           (registers capped at 128, some spilled); 0 = 1 */
  int reserved[3];
} tng_cfg;

typedef struct tng_chem tng_chem;

/* Fill cfg with the reference defaults. */
void tng_default_cfg(tng_cfg* cfg);

/* Last error message of the calling thread (copied, NUL-terminated). Returns its length. */
int tng_last_error(char* buf, int len);

/* Create a handle for a built-in mechanism ("hydrogen", "grimech30", "dme39").
 * Replaces the link-time choice of mechanism (combustion/Makefile:3-5) and finitechem_init's
 * mechanism queries (finitechem.f90:184-213). */
int tng_chem_create(const char* mechanism, const tng_cfg* cfg, tng_chem** out);
int tng_chem_destroy(tng_chem* h);

/* GETNSPECIES / GETNSPECS / GETNREACTIONS (HYDROGENF.f90:412-450) and the third-body count. */
int tng_chem_sizes(const tng_chem* h, int* nspecies, int* nslots, int* nthirdbody);
/* GETMOLARMASS (HYDROGENF.f90:366-386): W_k in kg/kmol, with the handle's literal kinds. */
int tng_chem_molar_mass(const tng_chem* h, double* wmol);
/* GETSPECIESNAMES (HYDROGENF.f90:389-409): name of species k (0-based), NUL-terminated. */
int tng_chem_species_name(const tng_chem* h, int k, char* buf, int len);
/* The handle's CUDA stream (cudaStream_t) for callers that enqueue around it. */
void* tng_chem_stream(tng_chem* h);

/* ---- Compatibility shims with the mechanism's Fortran signatures, arguments by reference, for a
 * caller that still evaluates the mechanism one cell at a time (finitechem_compute_rhs,
 * finitechem.f90:93-175); a Fortran caller writes `call tng_prodrates(CDOT, W, K, C, M, T, P)`.
 * They run on the GPU of the handle registered here (one launch and two copies per call: the
 * batch entry points above are the fast path). No status is returned, as for the Fortran
 * routines: on an error the outputs are NaN and tng_last_error has the message. */
void tng_set_mechanism_handle(tng_chem* h);
/* PRODRATES(CDOT, W, K, C, M, TEMP, PRESSURE) (HYDROGENF.f90:4-277; grimech30F.f90:4-2580):
 * CDOT[N] in kmol/m^3/s from C[N] in kmol/m^3, and the slot rates W[R] (reference literal kinds
 * only; W may be null). K and M are the reference's work arrays and are not written. */
void tng_prodrates_(double* cdot, double* w, double* k, const double* c, double* m, const double* temp,
                    const double* pressure);
/* COMPTHERMODATA(H, CP, T) (HYDROGENF.f90:514-673): h_k in J/kg and cp_k in J/(kg K) at T (the
 * NASA range switch T > 1000 K strict). */
void tng_compthermodata_(double* h, double* cp, const double* t);

/* Batched finitechem_compute_rhs (finitechem.f90:93-175, low-Mach branch) with PRODRATES,
 * GETLINDRATECOEFF and COMPTHERMODATA inside: for each of ncells cells,
 *   sol = (rho*Y_1..rho*Y_N, rho*T)  ->  rhs = (d(rho*Y_k)/dt, d(rho*T)/dt)
 * Arrays are species-major: variable v of cell i at [v*ld + i], v = 0..N, ld >= ncells.
 * p is the thermodynamic pressure in Pa (the reference uses 0.5*(P_thermo+P_thermo_old)).
 * flags: TNG_DEVICE_PTRS or TNG_HOST_PTRS. Device calls are asynchronous on the handle's
 * stream; host calls return after the results are in rhs. */
int tng_prodrates_batch(tng_chem* h, const double* sol, double* rhs, int64_t ncells, int64_t ld, double p,
                        int flags);

/* Debug variant of tng_prodrates_batch that also stores every slot's rate W_r
 * (the W(r) work array of PRODRATES) at rates[r*ld + i]; device pointers only. */
int tng_prodrates_batch_rates(tng_chem* h, const double* sol, double* rhs, double* rates, int64_t ncells, int64_t ld,
                              double p);

/* Wait for the handle's stream; returns the first asynchronous error, if any. */
int tng_chem_sync(tng_chem* h);

/* ---- autotuning (no counterpart in the reference: its kernels are the compiler's) ----------- */
#define TNG_TUNE_MAX 24
typedef struct tng_tune_result {
  int n, best;           /* candidates timed; index of the kept one */
  int a[TNG_TUNE_MAX];   /* rates: kernel variant; substep: cells (warps) per block */
  int b[TNG_TUNE_MAX];   /* rates: block size; substep: pass budget (0 = one pass, no recompaction) */
  double ms[TNG_TUNE_MAX];
} tng_tune_result;
/* Set the tunable launch parameters of a handle (as tng_cfg: rate_variant -1..2, block_size 0 =
 * default, solver_warps 0/2/4/8, or 16 for 8 warps with solver_occupancy 2; pass_budget >= 0). */
int tng_chem_set_tuning(tng_chem* h, int rate_variant, int block_size, int solver_warps, int pass_budget);
/* Time the rate kernel's variants x block sizes on the caller's cells (device pointers) and keep
 * the fastest in the handle. */
int tng_rates_autotune(tng_chem* h, const double* state, int64_t ncells, int64_t ld, double p,
                       tng_tune_result* out);
/* Time the implicit solver's cells-per-block (2, 4, 8, 16 = 8 at two blocks per SM) x pass-budget
 * (recompaction) choices on a strided
 * sample of at most `sample` of the caller's cells (device pointers; 0 = 65536) and keep the
 * fastest. Results per cell do not depend on the choice. */
int tng_substep_autotune(tng_chem* h, const double* state, int64_t ncells, int64_t ld, const double* dts, double dt,
                         double p, int64_t sample, tng_tune_result* out);

/* Statistics of one implicit substep. */
typedef struct tng_substep_stats {
  int64_t cells;         /* cells integrated */
  int64_t cells_failed;  /* cells whose integration stopped with a non-zero status */
  int64_t steps;         /* internal BDF steps, all cells */
  int64_t newton_iters;  /* Newton iterations, all cells */
  int64_t jacobians;     /* Jacobian evaluations + LU factorisations, all cells */
  int max_steps_cell;    /* largest per-cell step count */
  int max_newton_cell;   /* largest per-cell Newton iteration count */
  int passes;            /* solver passes that found work */
  int newton_hist[16];   /* cells by Newton iterations: [0], [1], [2,3], [4,7], ..., [2^14, inf) */
  double ms;             /* device time of the substep (CUDA events), host copies excluded */
} tng_substep_stats;

/* The implicit chemistry substep over a batch: the per-cell CVODE integration of
 * finitechem_source_chemistry (finitechem.f90:962-1071, CVODE calls :987-1068) on the GPU.
 * state (species-major, variable v of cell i at [v*ld + i], v = 0..N: rho*Y_k then rho*T) is
 * advanced in place over dt (dts[i] per cell when dts is non-null, else the scalar dt) at
 * pressure p with the handle's rtol/atol/max_steps. Cells are integrated by a persistent
 * work-stealing kernel; the pass loop runs as one CUDA graph. cell_nst / cell_nni / cell_status
 * (device int arrays of ncells, nullable) receive per-cell step and Newton counts and status
 * (0 ok, 1 max steps, 2 convergence failures, 3 error-test failures, 4 non-finite, 5 step too
 * small). flags: TNG_DEVICE_PTRS (state, dts and cell arrays on the device) or TNG_HOST_PTRS
 * (state and dts on the host; cell arrays must then be null). stats may be null; when given the
 * call waits for the device. */
int tng_substep_batch(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt, double p,
                      int flags, int* cell_nst, int* cell_nni, int* cell_status, tng_substep_stats* stats);

/* The same implicit substep (device pointers, one pass, no step budget) for callers that must
 * not allocate device memory during the call; no counterpart in the reference, which lets
 * CVODE allocate per cell. All scratch (tables, per-cell counters) lives in one static device
 * array: at most 262144 cells per call (TNG_ERR_ARG beyond). The first call on a device does
 * a synchronous set-up (it writes the solver tables of every built-in mechanism into the
 * array) and should precede any stream capture; later calls copy nothing and may alternate
 * mechanisms freely. Calls that overlap in time on one device race on the shared scratch:
 * order them (e.g. one stream). n_failed (host, nullable) receives the number of cells with a
 * nonzero status; when given the call waits, so it must be NULL inside a stream capture
 * (TNG_ERR_ARG otherwise). */
int tng_substep_batch_static(tng_chem* h, double* state, int64_t ncells, int64_t ld, const double* dts, double dt,
                             double p, int* n_failed);

/* Bounds of the host solver's arrays (Fortran, inclusive, column-major): RHO_(imino:imaxo,
 * jmino:jmaxo, kmino:kmaxo) and SC_(..., nscalar); the interior imin..imax etc.; 1-based scalar
 * indices of the first species, of T, and of H2O / CO / CO2 for the chemsrc diagnostics
 * (0 = absent). The species scalars are isc_sc .. isc_sc+N-1 in mechanism order. */
typedef struct tng_extent {
  int imino, imaxo, jmino, jmaxo, kmino, kmaxo;
  int imin, imax, jmin, jmax, kmin, kmax;
  int nscalar, isc_sc, isc_T;
  int isc_H2O, isc_CO, isc_CO2;
} tng_extent;

/* Drop-in for finitechem_source_chemistry(RHO_, SC_) (finitechem.f90:962-1071): for every
 * interior cell with mask(i,j) /= 1 (mask(imino:imaxo, jmino:jmaxo), nullable = no mask),
 * integrate (rho*Y, rho*T) over dt at pressure p_mid (0.5*(P_thermo + P_thermo_old)), write
 * Y and T back into sc, the heat-release rate into hr and d(rho*Y)/dt of H2O/CO/CO2 into
 * chemsrc(..., 3) (both same shape as RHO_ without/with the trailing 3; nullable). flags:
 * TNG_DEVICE_PTRS or TNG_HOST_PTRS (arrays staged through the device; the call then waits). */
int tng_chem_substep(tng_chem* h, const double* rho, double* sc, const int* mask, const tng_extent* ext, double dt,
                     double p_mid, double* hr, double* chemsrc, int flags, tng_substep_stats* stats);

/* Host-only (no device, no handle): the checks tng_chem_substep makes on a rank's extent for a
 * mechanism of nspecies species, and what it derives from it -- the number of interior cells
 * (imax-imin+1)*(jmax-jmin+1)*(kmax-kmin+1), the padded volume, and the positions of H2O / CO /
 * CO2 in the species block (-1 = absent), each output nullable. Errors as tng_chem_substep's.
 * Replaces the extent bookkeeping of finitechem_source_chemistry's loops over the rank's block
 * (finitechem.f90:993-1065) set up by partition_init (geometry/partition.f90:33-93). */
int tng_extent_plan(const tng_extent* ext, int nspecies, int64_t* n_interior, int64_t* volume, int* diag_species);

/* ---- Mixture properties around the substep, on the same Fortran arrays. Like the reference,
 * they visit every cell of the padded block (imino..imaxo, jmino..jmaxo, kmino..kmaxo) whose
 * mask(i,j) /= 1 and leave masked cells untouched; only ext's padded extents, nscalar, isc_sc
 * and isc_T are read. flags: TNG_DEVICE_PTRS (asynchronous on the handle's stream) or
 * TNG_HOST_PTRS (copied through the device; the call returns when the results are back).
 *
 * Replaces finitechem_density (combustion/finitechem.f90:324-345) with finitechem_W (:65-74):
 *   W_mix = sum(Y')/sum(Y'/W), Y' = min(max(Y,0),1);  rho = p_thermo*W_mix/(8314.34*T).
 * rho and wmix (both shaped like RHO) are each nullable. */
int tng_chem_density(tng_chem* h, double* rho, double* wmix, const double* sc, const int* mask, const tng_extent* ext,
                     double p_thermo, int flags);

/* Replaces finitechem_viscosity (finitechem.f90:351-406) and finitechem_diffusivity (:412-461),
 * with finitechem_omegamu (:467-487): T clipped to [50, 5000] K, species viscosities from the
 * mechanism's GETMUCOEFF / GETKOVEREPS fits, Wilke's mixture rule into visc (shaped like RHO),
 * and lambda/Cp_mix into diff (shaped like SC): diff(isc_sc+k-1) = lambda/Cp_mix/lewis[k],
 * diff(isc_T) = lambda/Cp_mix, and diff(isc_zmix) = lambda/Cp_mix when isc_zmix > 0. visc or
 * diff may be null (one of the two routines alone); both non-null computes them in one pass.
 * lewis: N Lewis numbers in HOST memory (the 'Lewis <species>' inputs, :293-301); null = 1. */
int tng_chem_transport(tng_chem* h, double* visc, double* diff, const double* sc, const int* mask,
                       const tng_extent* ext, const double* lewis, int isc_zmix, int flags);

/* ---- ARTS data files: the solver states the reference reads and writes (core/data.f90:217-284
 * data_read, :379-457 data_write_full3D; tools/init_flow/param.f90:113-148 through
 * library/fileio_c.c). Layout: int32 nx, ny, nz, nvars; float64 dt, time; nvars names of 8
 * blank-padded characters; each variable's nx*ny*nz doubles in Fortran order.
 *
 * Header of a file: dims = (nx, ny, nz, nvars), dt, time (nullable), and when names is non-null
 * the nvars blank-padded 8-character names into names[0 .. 8*nvars) (names_len bytes available). */
int tng_data_info(const char* path, int* dims, double* dt, double* time, char* names, int names_len);

/* Replaces data_read for one rank: the sub-block start (0-based i, j, k) / count of the named
 * variables (trailing blanks ignored) into out, variable v of block cell (i, j, k) at
 * out[v*ld + i + ci*(j + cj*k)] (the species-major layout of the batch entry points), ld >= the
 * block's cells. start/count null = the whole grid. flags: TNG_HOST_PTRS (h may be null) or
 * TNG_DEVICE_PTRS (out on h's device; the file is streamed through pinned buffers on h's
 * stream). Returns when out holds the data. */
int tng_data_read(tng_chem* h, const char* path, const char* const* vars, int nvar, const int* start,
                  const int* count, double* out, int64_t ld, int flags);

/* Replaces data_write_full3D for the whole grid dims = (nx, ny, nz): nvar variables named vars
 * (at most 8 characters) from fields[v*ld + i + nx*(j + ny*k)], with dt and time in the header.
 * flags as for tng_data_read (device fields are streamed through pinned buffers). */
int tng_data_write(tng_chem* h, const char* path, const int* dims, const char* const* vars, int nvar, double dt,
                   double time, const double* fields, int64_t ld, int flags);

/* Parity helper: the solver's own (table-driven, warp-cooperative) right-hand side and, when
 * jac is non-null, its Jacobian (cell-major, (N+1)^2 row-major per cell), device pointers. */
int tng_solver_rhs_jac(tng_chem* h, const double* state, int64_t ncells, int64_t ld, double p, double* rhs,
                       double* jac);

/* ---- Surrogate network (no counterpart in the reference: the learned replacement of the
 * substep for most cells). A multilayer perceptron x -> [Linear -> GELU] x layers -> Linear,
 * trained on the device with hand-written FP32 forward/backward/Adam kernels. Inputs and
 * outputs are row-major (rows x padded width), widths padded to multiples of 16 with zeros.
 * Parameters are one flat float array [W_0 b_0 W_1 b_1 ...], W_l row-major (out x in). */
typedef struct tng_mlp tng_mlp;
int tng_mlp_create(tng_chem* h, int n_in, int n_out, int hidden, int layers, uint64_t seed, tng_mlp** out);
int tng_mlp_destroy(tng_mlp* m);
int64_t tng_mlp_param_count(const tng_mlp* m);
/* which: 0 parameters, 1 last gradients, 2 / 3 Adam first / second moments */
int tng_mlp_get_params(tng_mlp* m, float* host, int which);
int tng_mlp_set_params(tng_mlp* m, const float* host);
/* FP32 forward on the device: X (rows x in_pad) -> Y (rows x out_pad), device pointers */
int tng_mlp_forward(tng_mlp* m, const float* X, int64_t rows, float* Y);
/* forward + backward of the weighted mean squared error; gradients stay on the device
 * (tng_mlp_get_params(which=1)), loss to *loss (host) when non-null */
int tng_mlp_grad(tng_mlp* m, const float* X, const float* T, const float* w_out, int64_t rows, float* loss);
/* Asymmetric loss: squared errors of outputs below their target are weighted by under (> 0;
 * default 1, the plain weighted MSE). The surrogate's error gate trains with under > 1. */
int tng_mlp_set_under_weight(tng_mlp* m, float under);
int tng_mlp_adam_step(tng_mlp* m, float lr);
/* minibatch training: epochs over n rows (shuffled per epoch), cosine learning-rate decay from
 * lr; per-epoch loss (last minibatch) to losses[epochs] when non-null */
int tng_mlp_train(tng_mlp* m, const float* X, const float* T, const float* w_out, int64_t n, int epochs, int batch,
                  double lr, uint64_t seed, float* losses);

/* ---- The substep through the surrogate, with fallback (no counterpart in the reference).
 * The network maps (T, log P, log10 Y_k for every species but the bath gas, log10 dt) to the
 * substep's (dT, dY_k). Its BF16 weights run on the tensor cores (FP32 accumulation); the
 * prediction then gets an FP64 element-conservation projection, clipping and renormalisation
 * of Y, and T from the enthalpy balance h(Y1, T1) = h(Y0, T0) (the low-Mach substep conserves
 * enthalpy). A cell falls back to the implicit solve (tng_substep_batch's algorithm) when a
 * feature lies outside the training range, when the network's dT disagrees with the
 * enthalpy-implied dT, or when clipping removed too much mass. Every call also re-solves
 * judge_cells sampled cells with the implicit solver and reports the surrogate's error. */
typedef struct tng_surrogate_cfg {
  int hidden;             /* width of the hidden layers (default 256) */
  int layers;             /* hidden layers (default 4) */
  uint64_t seed;          /* weight initialisation */
  double ood_margin;      /* allowed excursion beyond the training range, fraction of the range (0.02) */
  double consist_tol_K;   /* fallback when network and enthalpy temperatures differ by more (K, 5) */
  double clip_tol;        /* fallback when clipping removed more mass fraction (1e-3) */
  int judge_cells;        /* cells re-solved every call to measure the error (1024) */
  int post_mode;          /* 0: T from the enthalpy balance of the conserved Y; 1: T from the network,
                             enthalpy held by the projection of Y (default 1) */
  int target_mode;        /* training targets: 0 each output scaled by its own spread; 1 dY_k share
                             one scale (errors weighted as the dY <= tol*max(Y) criterion) (1) */
  float loss_T_weight;    /* loss weight of dT relative to one species output (0 = default 2) */
  int members;            /* networks in the ensemble, trained from different initialisations; the
                             prediction is their mean (1..4, 0 = default 2) */
  float ens_tol_K;        /* fallback when the members' temperatures spread by more (K, 0 = default 2) */
  float ens_tol_Y;        /* fallback when a mass fraction spreads by more (0 = default 5e-4) */
  float gate_tol;         /* error gate: fallback when it predicts an error above this fraction of
                             the accuracy bars (|dT|/T 1e-2, max |dY| / max Y 1e-3); 0 = the value
                             calibrated with the model */
  int reserved;
} tng_surrogate_cfg;

typedef struct tng_surrogate_stats {
  int64_t cells, accepted;
  int64_t fallback_ood, fallback_consistency, fallback_clip;
  int64_t judged;               /* sampled cells solved twice */
  double judge_max_rel_dT;      /* max |T_s - T_p| / T_p over the sample (surrogate vs implicit) */
  double judge_max_dY;          /* max |Y_s,k - Y_p,k| / max_k Y_p,k over the sample */
  double ms_infer, ms_post, ms_fallback, ms_total;  /* device times; with a judged sample, ms_fallback
                                   covers the joint implicit solve of the fallback cells and the sample */
  tng_substep_stats fallback;   /* the implicit solve of the fallback cells (cells: their number; the
                                   step and iteration counts include the judged sample, solved jointly) */
  int64_t fallback_ensemble;    /* cells whose ensemble members disagreed */
  int64_t fallback_gate;        /* cells whose predicted error (error gate) exceeded gate_tol */
} tng_surrogate_stats;

typedef struct tng_surrogate tng_surrogate;
void tng_surrogate_default_cfg(tng_surrogate_cfg* cfg);
int tng_surrogate_create(tng_chem* h, const tng_surrogate_cfg* cfg, tng_surrogate** out);
int tng_surrogate_destroy(tng_surrogate* s);
/* Train on pairs from the implicit solver: state0 before and state1 after a substep of dts[i]
 * (device pointers, species-major with leading dimension ld). */
int tng_surrogate_train(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                        int64_t ld, double p, int epochs, int batch, double lr, float* losses);
/* Hard-example refinement (after tng_surrogate_train, on the same kind of pairs): the ensemble's
 * post-processed prediction of every pair is compared with state1; pair i then enters the
 * training population 1 + min(round(boost * e_i), 16) times, e_i its larger error relative to the
 * bars, and every member is trained on that population for `epochs` more epochs (cosine
 * learning rate from lr). *population (nullable) receives the population size. */
int tng_surrogate_refine(tng_surrogate* s, const double* state0, const double* state1, const double* dts, int64_t n,
                         int64_t ld, double p, int epochs, int batch, double lr, double boost, float* losses,
                         int64_t* population);
/* The error gate: a network of the members' hidden shape with two outputs, trained to predict
 * log10 of the ensemble's own post-processed errors on these pairs relative to the bars (|dT|/T
 * over 1e-2, max |dY| / max Y over 1e-3). Under-predictions weigh `under` times more in its
 * loss. Once trained (or loaded), every substep falls a cell back when the gate predicts an
 * error above gate_tol (tng_surrogate_set_gate_tol, saved with the model). */
int tng_surrogate_train_gate(tng_surrogate* s, const double* state0, const double* state1, const double* dts,
                             int64_t n, int64_t ld, double p, int epochs, int batch, double lr, double under,
                             float* losses);
int tng_surrogate_set_gate_tol(tng_surrogate* s, double tol);
/* has_gate: 1 when an error gate is trained or loaded; tol: the gate threshold in effect. */
int tng_surrogate_gate_info(const tng_surrogate* s, int* has_gate, double* tol);
int tng_surrogate_save(const tng_surrogate* s, const char* path);
int tng_surrogate_load(tng_surrogate* s, const char* path);
/* Sizes: raw inputs/outputs, their padded widths, parameter count. */
int tng_surrogate_dims(const tng_surrogate* s, int* n_in, int* n_out, int* in_pad, int* out_pad, int64_t* nparam);
/* Parameters (FP32 master copy, layout of tng_mlp_*) to host (set = 0) or from host (set = 1). */
int tng_surrogate_params(tng_surrogate* s, float* host, int set);
/* Normalised FP32 features (n x in_pad, device) of a state batch, for checks and tooling. */
int tng_surrogate_features(tng_surrogate* s, const double* state, int64_t n, int64_t ld, const double* dts, double p,
                           float* X);
/* The surrogate's prediction without fallback (device pointers): out (species-major, ld_out)
 * receives the conserved post-processed state of every cell; reason (nullable, int per cell)
 * 0 accepted / 1 out of range / 2 inconsistent / 3 clipped / 4 ensemble disagreement / 5 error
 * gate; indicator (nullable, 5 doubles per cell): the network-vs-enthalpy temperature mismatch
 * (K), the members' temperature spread (K), their largest mass-fraction spread, and the gate's
 * predicted log10 errors of T and Y relative to the bars (-inf without a gate). dts per cell or
 * the scalar dt. */
int tng_surrogate_predict(tng_chem* h, tng_surrogate* s, const double* state, int64_t ncells, int64_t ld,
                          const double* dts, double dt, double p, double* out, int64_t ld_out, int* reason,
                          double* indicator);
/* FP32 reference forward of the network on normalised features (device pointers). */
int tng_surrogate_forward_f32(tng_surrogate* s, const float* X, int64_t n, float* Y);
/* Test hook of the inference kernel's bounded waits (no counterpart in the reference): every
 * later inference of s gives up a wait after wait_limit polls (0: the default limit), and with
 * fault = 1 each CTA's first layer withholds its completion signal, so that the epilogue's wait
 * runs out. The kernel then drains its own copies and MMAs, frees its tensor memory and reports
 * the timeout, which the call returns as TNG_ERR_CUDA. (0, 0) restores normal operation. */
int tng_surrogate_debug_waits(tng_surrogate* s, int wait_limit, int fault);
/* Tensor-core inference only: normalised predictions (n x out_pad FP32, device) of a state batch. */
int tng_surrogate_infer(tng_surrogate* s, const double* state, int64_t n, int64_t ld, const double* dts, double dt,
                        double p, float* out);
/* The substep through the surrogate with fallback; same state convention as tng_substep_batch.
 * flags: TNG_DEVICE_PTRS or TNG_HOST_PTRS. stats may be null. With host pointers and a batch of
 * 2^19 cells or more the state is uploaded in chunks that overlap the inference and
 * post-processing of the chunks already on the device (stats->ms_infer then covers both and
 * ms_post is 0), and with stats the post-processed state is downloaded during the fallback solve,
 * the solved fallback cells being patched into the host state afterwards; the results are the
 * same as with device pointers. */
int tng_substep_surrogate(tng_chem* h, tng_surrogate* s, double* state, int64_t ncells, int64_t ld, const double* dts,
                          double dt, double p, int flags, tng_surrogate_stats* stats);

/* Measurement helper (no reference counterpart): sustained FP64 FMA throughput of a device in
 * TFLOP/s (FMA = 2 flops), the denominator of the FP64-pipe roofline of the rate kernels. */
int tng_bench_fp64_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* TIGER_CHEM_H */
