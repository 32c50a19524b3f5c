/*
 * axj.h -- C-ABI of the B200 per-step hot path of the axisymmetric compressible
 * jet solver (nataraj2/AxisymmetricJet).
 *
 * The reference drives the hot path through argument-less Fortran module
 * subroutines that work on module globals:
 *     DO iteration = ...; CALL ComputeTimeStep; CALL RK4; ENDDO   (ModSolver.f90:122-125)
 * This header replaces those calls with a handle-based C interface that a
 * Fortran host binds through ISO_C_BINDING (BIND(C, name="axj_...")).
 *
 * Conventions
 *  - Every host array is Fortran column-major with z (index i) fastest:
 *    a field is Nz*Nr doubles, element (i,j) at offset (i-1) + (j-1)*Nz.
 *    A solution array pv(Nz,Nr,1,5) is 5 such fields back to back
 *    (rho, V_r, V_theta, V_z, T), exactly the reference's pv layout
 *    (ModuleVariables.f90:39, ModAllocate.f90).
 *  - Patch indices are 1-based, as produced by PatchCreation (ModPatch.f90:264-309).
 *  - The library copies host arrays in and out and never keeps a host pointer
 *    after a call returns. It owns all device memory of a handle.
 *  - Every function returns an axj_status; 0 is success. The library never
 *    exits, aborts or prints; the host decides what to do (e.g. StopTheCode).
 *  - One host thread per handle; calls on one handle are not thread-safe.
 */
#ifndef AXJ_H
#define AXJ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum axj_status {
  AXJ_OK = 0,
  AXJ_ERR_ARG = 1,          /* bad argument (null pointer, size, enum value) */
  AXJ_ERR_CUDA = 2,         /* a CUDA runtime call failed; see axj_last_error */
  AXJ_ERR_NONFINITE = 3,    /* NaN/Inf found in the state after a step */
  AXJ_ERR_DT_BLOWUP = 4,    /* every point blanked: dt == 100 (ModInputOutput.f90:424-429) */
  AXJ_ERR_TIMEOUT = 5,      /* a bounded device wait gave up */
  AXJ_ERR_BADPATCH = 6,     /* inconsistent patch / bc record */
  AXJ_ERR_BADGRID = 7,      /* grid not supported (too small, not a tensor-product z(i), r(j) grid) */
  AXJ_ERR_NOMEM = 8,        /* device allocation failed */
  AXJ_ERR_NODEVICE = 9,     /* no CUDA device / library built without sm_100a code */
  AXJ_ERR_UNSUPPORTED = 10  /* option combination not implemented */
};

/* Boundary-condition codes (ModuleVariables.f90:112-117). */
enum axj_bc {
  AXJ_BC_AXIS = 90,
  AXJ_BC_SAT_FARFIELD = 91,
  AXJ_BC_NSCBC_NONREFLECTING = 92,
  AXJ_BC_SAT_NOSLIP_WALL = 93,
  AXJ_BC_NSCBC_NOSLIP_WALL = 94,
  AXJ_BC_SPONGE = 95
};

/* One boundary patch after PatchCreation: the 4-wide strip the SBP closure rows
 * live in. Field order follows TYPE patch_type (ModuleVariables.f90:102-106). */
typedef struct axj_patch {
  int64_t i_start, i_end, j_start, j_end;
  int64_t bc;      /* enum axj_bc */
  int64_t bc_dir;  /* +1/-1: z-face at i_start/i_end; +2/-2: r-face at j_start/j_end */
} axj_patch;

/* One raw row of the bc file as read by CreateAllPatches (ModPatch.f90:132):
 * "grid bc dir istart iend jstart jend k k"; -1 means the last index. */
typedef struct axj_bc_record {
  int64_t bc, bc_dir, istart, iend, jstart, jend;
} axj_bc_record;

/* dt_mode values. */
enum axj_dt_mode {
  AXJ_DT_REFERENCE = 0, /* sqrt of the stale module scalar T, as ModInputOutput.f90:405 does */
  AXJ_DT_PHYSICAL = 1   /* sqrt of the local temperature T(i,j) */
};

/* precision values. */
enum axj_precision {
  AXJ_FP64 = 0,  /* plain FP64 end to end */
  AXJ_MIXED = 1  /* FP32 stage states/stencils, FP64 accumulation, penalties, near-axis terms, dt */
};

/* sensor values (artificial-diffusivity sensor, used when shock_capturing = 1). */
enum axj_sensor_kind {
  AXJ_SENSOR_PLAIN = 0,   /* ModShockCapturing.f90:5-106 */
  AXJ_SENSOR_LEARNED = 1, /* MLP stand-in, plain sensor as periodic judge */
  AXJ_SENSOR_HELD = 2     /* baseline of the learned sensor without the network: the plain
                             sensor's coefficients of the last judge step are held between judges */
};

#define AXJ_DEFAULT_STAGE_ROWS 8

/* Run parameters: the reference's compile-time module variables
 * (ModuleVariables.f90:4-188) as a POD struct. Fill with axj_default_params. */
typedef struct axj_params {
  double gam;                 /* 1.4          ModuleVariables.f90:66 */
  double Re;                  /* 1000         :73 */
  double Pr;                  /* 0.72         :73 */
  double CFL;                 /* 0.5          :177 */
  double sponge_start_top;    /* 12.5         :12 */
  double sponge_A_top;        /* 0.5          :12 */
  double sponge_end_left;     /* 6.0          :13 */
  double sponge_A_left;       /* 5.0          :13 */
  double C_mu, C_beta, C_kappa; /* 0,0,0      :164 */
  double forcing_alpha;       /* 6.0          :184 */
  double forcing_z0, forcing_r0, forcing_lz, forcing_lr; /* Vz_Control_Vr_Feedback.dat */
  double forcing_mat[25];     /* F(eqn,k) stored row-major: forcing_mat[(eqn-1)*5 + (k-1)] */
  int64_t do_viscous_terms;   /* 1            :71 */
  int64_t shock_capturing;    /* 0            :152 */
  int64_t control_forcing;    /* 0 (:185); 1: ControlForcingTerms feedback; 2: harmonic source (below) */
  int64_t dt_mode;            /* AXJ_DT_REFERENCE */
  int64_t precision;          /* AXJ_FP64 */
  int64_t sensor;             /* AXJ_SENSOR_PLAIN */
  int64_t judge_every;        /* learned sensor: plain-sensor judge period in steps (50) */
  double judge_threshold;     /* learned sensor: fallback where |pred-plain| > thr * local max (0.1) */
  int64_t device;             /* CUDA device ordinal the handle lives on (0) */
  /* control_forcing = 2, an extension with no counterpart in the reference (whose
   * ControlForcingTerms is steady linear feedback): azimuthal-mode-0 harmonic forcing in
   * the same Gaussian window G(z,r) = exp(-(z-z0)^2/lz^2 - (r-r0)^2/lr^2). The source
   * rhs(V_z) += A * omega * G * cos(omega * t), omega = 2 pi St U_j / D (D = 1), imposes
   * a V_z fluctuation of amplitude A * G; t is the stage time t_n + c_s dt, c = (0, 1/2,
   * 1/2, 1). */
  double harmonic_amp;        /* A (velocity units) */
  double harmonic_st;         /* Strouhal number St */
  double harmonic_uj;         /* jet velocity U_j */
  /* 0: the stencil maps, face lists and tile classes of axj_create are built on the host;
   * 1: on the device (one thread per grid row and per tile, the same rules). */
  int64_t patch_prep;
  /* Rows of the fused stage kernel's CTAs on interior tiles (32 x 16 points each): 16 (one
   * CTA per tile, two CTAs per SM) or 8 (two CTAs per tile with half the shared memory, four
   * per SM); 0 is the library's default, AXJ_DEFAULT_STAGE_ROWS. The results agree to
   * rounding (separate compilations of the same per-point code). */
  int64_t stage_rows;
  /* Learned and held sensors: the RK stages of a judge step that run the plain sensor. 0 or
   * 4: all four (the judge step is a plain step); 1: the first stage only, whose plain
   * coefficients then serve the step's four stages, as the network's do between judges. */
  int64_t judge_stages;
  int64_t reserved[1];
} axj_params;

typedef struct axj_handle axj_handle;

/* Fill p with the reference defaults (ModuleVariables.f90). */
void axj_default_params(axj_params* p);

/* Create a solver instance for one Nz x Nr block.
 * zvec, rvec, ibval: Nz*Nr each (AssignGridCoordinates, ModInputOutput.f90:69-89).
 * patches: the patch list after CreateAllPatches (ModPatch.f90:117-262).
 * Replaces: AllocateVariables, CreateAllPatches' stencil maps, SBP_operator and the
 * ComputeMetric calls of ModSolver.f90:57-76. */
int axj_create(const axj_params* params, int64_t Nz, int64_t Nr,
               const double* zvec, const double* rvec, const double* ibval,
               const axj_patch* patches, int64_t npatch, axj_handle** out);

/* Upload the solution and the target (SolnRead, ModInputOutput.f90:91-148).
 * iteration/time are tau(1)/tau(4) of the restart file (ModSolver.f90:103-106). */
int axj_set_state(axj_handle* h, const double* pv, const double* pv_target,
                  int64_t iteration, double time);

/* Download the solution pv(Nz,Nr,1,5) (feeds WriteOutput, ModInputOutput.f90:201-263). */
int axj_get_state(axj_handle* h, double* pv);

/* Current iteration counter and time held by the handle. */
int axj_get_time(axj_handle* h, int64_t* iteration, double* time);

/* ComputeTimeStep (ModInputOutput.f90:389-438): global CFL/viscous dt. */
int axj_compute_dt(axj_handle* h, double* delt);

/* RK4 (ModRungeKutta.f90:5-171) with the given delt; advances iteration and time. The
 * four stages replay a CUDA graph captured on the first call (a second one for the
 * learned sensor's judge steps); a new model (axj_mlp_set, training) drops the graphs. */
int axj_rk4_step(axj_handle* h, double delt);

/* nsteps x (ComputeTimeStep + RK4) with dt kept on the device, no host sync
 * inside; the step sequence is captured once in a CUDA graph and replayed.
 * If out_every > 0 and cb != NULL, cb(user, iteration, time, pv) is called with a
 * host copy of the state of every out_every-th iteration (the noutput hook,
 * ModRungeKutta.f90:161-165). The state is copied on the device in step order and
 * brought to pinned host memory on a second stream while the following steps run; the
 * callback for an output runs when the next output is taken or before axj_run returns,
 * in order, and pv is valid only during the callback. A step that left a non-finite
 * value or a dt blow-up makes the delivery of its output return the error instead.
 * last_dt (nullable) receives the last dt used. */
typedef void (*axj_output_cb)(void* user, int64_t iteration, double time, const double* pv);
int axj_run(axj_handle* h, int64_t nsteps, int64_t out_every, axj_output_cb cb, void* user,
            double* last_dt);

/* Measurement entry points (no counterpart in the reference, which has no timers).
 * axj_run_timed: like axj_run without output, with *ms = device time of the nsteps
 * graph replays between two CUDA events on the handle's stream.
 * axj_profile_steps: nsteps steps launched one kernel at a time with a CUDA event
 * pair around every launch group; ms[0] = dt kernel, ms[1] = sensor chain,
 * ms[2] = fused stage kernels, ms[3] = whole steps (sums over the nsteps steps);
 * launches[0..2] = kernel launches of each group. */
int axj_run_timed(axj_handle* h, int64_t nsteps, double* ms);
int axj_profile_steps(axj_handle* h, int64_t nsteps, double* ms, int64_t* launches);

/* AssignValues + ComputeRHS (ModRHS.f90:5-258) on pv (Nz*Nr*5, host) with the
 * handle's target and delt-independent terms; rhs receives Nz*Nr*5 values. The
 * handle's solution is not changed. */
int axj_rhs(axj_handle* h, const double* pv, double* rhs);

/* Compute1stDerivative(var, dirn, out) (ModDeriv.f90:5-120). dirn = 1 (z) or 2 (r). */
int axj_deriv1(axj_handle* h, const double* var, int64_t dirn, double* out);

/* Compute2ndDerivative(var, dirn, first_deriv, out) (ModDeriv.f90:123-238). */
int axj_deriv2(axj_handle* h, const double* var, int64_t dirn, const double* first_deriv,
               double* out);

/* PerformTGfilter(var, dirn, out) (ModTGfilter.f90:5-95). out is read as well:
 * blanked points keep its incoming value. If inplace != 0, var is ignored and the
 * filter runs in place on out along z, i.e. PerformTGfilter(q, 1, q) as
 * ModShockCapturing.f90:63 calls it (a recurrence along i). */
int axj_tgfilter(axj_handle* h, const double* var, int64_t dirn, int64_t inplace, double* out);

/* ComputeArtTransCoeffs' sensor (ModShockCapturing.f90:5-92) on pv: the artificial
 * coefficients mustar, betastar, kappastar (Nz*Nr each) before they are added
 * to mu/beta/lambda/kappa. */
int axj_sensor(axj_handle* h, const double* pv, double* mustar, double* betastar,
               double* kappastar);

/* ComputeTimeStep for callers that cannot allocate device memory. This entry point has
 * no counterpart in the reference. The handle-based calls above allocate their buffers
 * with cudaMalloc in axj_create; a host whose device memory is owned by someone else (a
 * framework's caching allocator, a Fortran host passing its own device arrays, a process
 * that may not grow its device footprint after start-up) cannot use them. This call
 * allocates nothing: the caller passes every array, already on the device, and the
 * reduction's scratch (per-block minima and a counter) lives in a fixed array inside the
 * library, which every GPU that loads the library holds (about 512 KB) until exit.
 *   d_pv     5 planes (rho, V_r, V_theta, V_z, T) of Nr rows, row pitch `pitch` doubles
 *   d_dxidz  Nz values of dxi/dz, d_detadr Nr values of deta/dr (ComputeMetric's 1-D metrics)
 *   d_ibval  Nz x Nr (pitch `pitch`) blanking values, or NULL for no blanked points
 *   params   CFL, Re, Pr and dt_mode are read; stale_T is the module scalar T used when
 *            dt_mode is AXJ_DT_REFERENCE
 *   d_dt     receives dt on the device (100 if every point is blanked; NaN if a point that
 *            is not blanked holds a non-finite V_r, V_z or T, or gives a NaN dt); stream is a cudaStream_t (NULL: legacy default stream)
 * At most 16,777,216 points (Nz*Nr); larger grids return AXJ_ERR_ARG with a message in
 * axj_last_error(NULL). The call is asynchronous on `stream`. The first call on a device
 * writes the tables of mu = T**0.666 (a synchronous copy into the library's own device
 * array, no allocation) and looks up the scratch array's device address with that device
 * current; make that first call before any stream capture. Calls share the scratch, so calls that overlap on the
 * GPU (different streams, no ordering) race with each other. */
int axj_compute_dt_noalloc(const double* d_pv, int64_t pitch, int64_t Nz, int64_t Nr, const double* d_dxidz,
                           const double* d_detadr, const double* d_ibval, const axj_params* params, double stale_T,
                           double* d_dt, void* stream);

/* ---- Learned artificial-diffusivity sensor (sensor = AXJ_SENSOR_LEARNED) ----------
 * No counterpart in the reference. A small MLP stands in for the evaluation of
 * betastar and kappastar (ModShockCapturing.f90:18-92): 100 inputs (4 channels x a
 * 5 x 5 (z, r) window), two hidden layers of 64 with the tanh-form GELU, 2 outputs,
 * BF16 weights and FP32 accumulation on the tensor cores at inference. The network
 * runs once per step on the first stage's input and its coefficients serve the
 * step's four stages. mustar keeps the plain sensor's value of the last judge step. The plain sensor runs on the first
 * stage of every judge_every-th step (and on the first step after axj_set_state,
 * axj_mlp_set or training) as judge: wherever |prediction - plain| exceeds
 * judge_threshold x the largest |plain| in the point's 5 x 5 window, the plain value
 * of that judge step replaces the prediction until the next judge step. The other
 * three stages of a judge step use the plain sensor throughout. */
#define AXJ_MLP_CHANNELS 4  /* dilatation, |grad rho|, |vorticity|, sqrt(deltaz*deltar) */
#define AXJ_MLP_IN 100      /* input index ch*25 + (dr+2)*5 + (dz+2), dz, dr in -2..2 */
#define AXJ_MLP_HIDDEN 64
#define AXJ_MLP_OUT 2       /* betastar, kappastar before the z ramp (1+tanh(5(z-10)))/2 */

typedef struct axj_mlp {
  float w1[AXJ_MLP_HIDDEN * AXJ_MLP_IN]; /* row-major [out][in] */
  float b1[AXJ_MLP_HIDDEN];
  float w2[AXJ_MLP_HIDDEN * AXJ_MLP_HIDDEN];
  float b2[AXJ_MLP_HIDDEN];
  float w3[AXJ_MLP_OUT * AXJ_MLP_HIDDEN];
  float b3[AXJ_MLP_OUT];
  float feat_mean[AXJ_MLP_CHANNELS];     /* input = (channel value - mean) / scale; 0 outside the grid */
  float feat_scale[AXJ_MLP_CHANNELS];
  float out_scale[AXJ_MLP_OUT];          /* coefficient = output * out_scale * ramp(z) */
} axj_mlp;

typedef struct axj_train_cfg {
  int64_t steps;              /* Adam steps (2000) */
  int64_t batch;              /* points per step (65536), drawn uniformly over the data set */
  double lr, beta1, beta2, eps; /* 1e-3, 0.9, 0.999, 1e-8 */
  int64_t seed;               /* batch-sampling seed */
  int64_t fit_normalization;  /* 1: set the feature/output normalisation from the data set first */
  int64_t reserved[6];
} axj_train_cfg;

void axj_default_train_cfg(axj_train_cfg* cfg);
/* Seeded initial model: weights and biases uniform in +-1/sqrt(fan_in), unit normalisation. */
void axj_mlp_init(axj_mlp* m, int64_t seed);
/* Install / read the handle's model (the handle needs shock_capturing = 1). */
int axj_mlp_set(axj_handle* h, const axj_mlp* m);
int axj_mlp_get(axj_handle* h, axj_mlp* m);
/* Training data on the device: room for nsnapshots snapshots (24 bytes per grid point
 * each); axj_dataset_add appends the feature channels and the plain sensor's betastar,
 * kappastar (before the ramp) of the handle's current solution. */
int axj_dataset_reserve(axj_handle* h, int64_t nsnapshots);
int axj_dataset_add(axj_handle* h);
int axj_dataset_size(axj_handle* h, int64_t* nsnapshots);
/* Train the installed model with Adam on the data set (FP32, on the device);
 * loss (nullable) receives cfg->steps batch losses (mean squared error of the
 * normalised outputs, summed over the two outputs). */
int axj_mlp_train(axj_handle* h, const axj_train_cfg* cfg, float* loss);
/* Checks: the normalised batch (X: batch x 100, T: batch x 2) that training step `step`
 * with `seed` draws; the gradient (in model layout) and loss of the installed model on
 * a given normalised batch; the feature channels of pv (4 planes of Nz*Nr); the
 * tensor-core prediction (ramp applied) on pv; judge counters since creation. */
int axj_dataset_sample(axj_handle* h, int64_t batch, int64_t seed, int64_t step, float* X, float* T);
int axj_mlp_grad(axj_handle* h, const float* X, const float* T, int64_t batch, axj_mlp* grad, float* loss);
int axj_mlp_features(axj_handle* h, const double* pv, float* feat);
int axj_mlp_predict(axj_handle* h, const double* pv, double* betastar, double* kappastar);
int axj_learned_stats(axj_handle* h, int64_t* judged_outputs, int64_t* fallbacks, int64_t* njudges);

/* ---- Batches: many instances in one launch per kernel ------------------------------
 * No counterpart in the reference (one jet per run). A batch advances n handles of
 * uneven grids and parameters together: each kernel of the step runs once for all of
 * them, as a persistent grid-stride kernel over a table of (tile, instance) entries
 * with per-instance arguments and TMA descriptors in device tables, and the whole step
 * is captured in a CUDA graph. The handles keep their state: axj_get_state etc. work
 * on them between batch calls. All handles need the same device, precision, sensor
 * kind and shock-capturing setting (and, learned, the same model), and their state
 * set. The batch does not own the handles; destroy it before them. */
typedef struct axj_batch axj_batch;
typedef struct axj_batch_tuning {
  int64_t tile_order;          /* 0: instance after instance; 1: round-robin over instances */
  int64_t stage_ctas_per_sm;   /* persistent CTAs per SM of the interior stage kernel (2) */
  int64_t sensor_ctas_per_sm;  /* persistent CTAs per SM of the interior sensor kernel (4) */
  int64_t stage_rows;          /* rows of the interior stage tiles' CTAs: 16 (32 x 16 tiles, default) or 8 */
  int64_t general_ctas_per_sm; /* persistent CTAs per SM of the general stage kernel: 1 (default; 0 = 1) or 2 */
  int64_t general_serial;      /* 0: general tiles on a side stream beside the interior launches (default);
                                  1: on the batch's stream with them */
  int64_t reserved[2];
} axj_batch_tuning;

void axj_batch_default_tuning(axj_batch_tuning* t);
int axj_batch_create(axj_handle* const* handles, int64_t n, axj_batch** out);
/* nsteps x (ComputeTimeStep + RK4) of every instance, each with its own dt. */
int axj_batch_run(axj_batch* b, int64_t nsteps);
/* As axj_batch_run, *ms = device time of the nsteps graph launches (CUDA events). */
int axj_batch_run_timed(axj_batch* b, int64_t nsteps, double* ms);
int axj_batch_set_tuning(axj_batch* b, const axj_batch_tuning* t);
int axj_batch_get_tuning(axj_batch* b, axj_batch_tuning* t);
/* Autotuner: times steps_per_trial batch steps for every candidate tuning (tile order x
 * interior stage tile shape 32 x 16 or 32 x 8 with its CTAs per SM x sensor CTAs per SM:
 * 16 trials), then, from the fastest, the general tiles' CTAs per SM and stream (3 more
 * trials); keeps the fastest and returns it in *chosen; trial_ms (nullable, room for 19)
 * receives each trial's time. The trial steps are undone: the instances' solutions,
 * times and iteration counters are restored (the learned sensor re-judges). */
int axj_batch_autotune(axj_batch* b, int64_t steps_per_trial, axj_batch_tuning* chosen, double* trial_ms,
                       int64_t* ntrials);
const char* axj_batch_last_error(const axj_batch* b);
void axj_batch_destroy(axj_batch* b);

/* Poll limit of the bounded waits (TMA completions) of the stage, sensor and filter
 * kernels on the handle's device; tries < 0 restores the default (2^20 polls, about a
 * quarter of a second), 0 makes every such wait give up at once. No counterpart in the
 * reference: it exists so that a test can make the waits give up and see the kernels
 * report AXJ_ERR_TIMEOUT and return, each after its transfers in flight have landed, with
 * the context still usable. It applies to every handle on the device; axj_set_state
 * clears a handle's error flags. */
int axj_set_wait_limit(axj_handle* h, int64_t tries);

/* Last error message of the handle (or of the last failed axj_create if h is NULL). */
const char* axj_last_error(const axj_handle* h);

void axj_destroy(axj_handle* h);

/* Host helpers (no device work). */

/* Parse a bc file (ModPatch.f90:30-63): rows of 9 integers. Fills up to max_records
 * records and sets *nrecords. */
int axj_read_bc_file(const char* path, axj_bc_record* records, int64_t max_records,
                     int64_t* nrecords);

/* PatchCreation for a single block holding the whole grid (ModPatch.f90:117-309):
 * resolve -1 to the last index and widen each face to its 4-wide strip. */
int axj_patches_from_records(const axj_bc_record* records, int64_t nrecords, int64_t Nz_grid,
                             int64_t Nr_grid, axj_patch* patches, int64_t* npatch);

/* The per-point maps of CreateAllPatches (ModPatch.f90:214-242) and of the
 * BoundaryConditions loop (ModBC.f90:25-274) exactly as axj_create builds the device
 * descriptors from them, for x = (i-1) + (j-1)*Nz: zrow[x], rrow[x] = the SBP row (0..8,
 * 4 = centred) of the z and r stencils (the last patch of a direction wins a point);
 * blank[x] = 1 where ibval == 0; nfaceops[x] = the number of face operations (SAT /
 * NSCBC patches that act at the point, in patch order) and faceop_ids[x] their 1-based
 * patch numbers, one per byte from the lowest. */
int axj_point_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, const double* ibval,
                   uint8_t* zrow, uint8_t* rrow, uint8_t* blank, uint8_t* nfaceops, uint64_t* faceop_ids);

/* The stencil maps of one block as axj_create builds them for the device: algorithm 0 is
 * the host path, 1 the per-row and per-tile functions of the device path run on the host,
 * 2 the device path itself (needs a device). desc gets Nr rows of pitch P = Nz rounded up
 * to 32 (P*Nr descriptors); faces the face-operation list (capacity faces_cap, length in
 * *nfaces); tiles the (i0, j0) pairs of the interior stage, general stage, interior
 * sensor and general sensor tiles one list after the other (capacity tiles_cap pairs,
 * lengths in counts[4]); stale[2] the 1-based point where the stale scalar T is taken. */
int axj_prep_maps(const axj_patch* patches, int64_t npatch, int64_t Nz, int64_t Nr, const double* ibval,
                  int64_t algorithm, uint32_t* desc, int32_t* faces, int64_t faces_cap, int64_t* nfaces,
                  int32_t* tiles, int64_t tiles_cap, int64_t* counts, int64_t* stale);

/* The operator tables the device kernels use, as SBP_operator forms them
 * (ModOperator.f90:5-121): SBP1(0:8,0:5) and SBP2(0:8,0:5) into sbp1[54] and sbp2[54],
 * TGfilt(0:8,0:10) into tgfilt[99], row-major (row = the SBP row). */
int axj_operator_tables(double* sbp1, double* sbp2, double* tgfilt);

/* mu = T**0.666 (ModAssign.f90:20, Tvec**0.666D0) as the FP64 kernels form it: a
 * table-driven power within 1 ulp of the correctly rounded result for T in [2^-16, 2^16),
 * evaluated on the host with the device's operations (the same bits). */
double axj_mu_of_T(double T);

/* Library build information, e.g. "axj 0.1 sm_100a". */
const char* axj_version(void);

#ifdef __cplusplus
}
#endif

#endif /* AXJ_H */
