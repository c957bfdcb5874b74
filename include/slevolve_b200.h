/*
 * slevolve_b200.h -- C ABI of the B200 (sm_100a) implementation of the SLEvolve
 * per-time-step sea-level path.
 *
 * Every entry point returns an int status (SLE_OK = 0).  On failure,
 * sle_last_error() returns a message for the calling thread.  Nothing here
 * aborts, traps or exits.  No torch or CUDA types appear in the signatures:
 * streams are passed as void* (a cudaStream_t, NULL = the handle's own stream),
 * device buffers as plain pointers.
 *
 * Layouts (identical to the reference Python package):
 *   grid    float64 [nlat][nlon], Gauss-Legendre rows north -> south.
 *   dense   complex128 [lmax+1][lmax+1] as [l][m] (interleaved re, im),
 *           zero for m > l.
 *   packed  complex128, order-major triangle: order m holds degrees
 *           l = m..lmax contiguously, offset(m) = m*(lmax+1) - m*(m-1)/2.
 *
 * Reference interfaces replaced (SLEvolve, python/slevolve/):
 *   sle_sht_*     sht.py:148-343 (SHT.__init__/analysis/synthesis, the
 *                 transform the reference documents as the GPU plug-in point,
 *                 sht.py:43-46) and sht_ducc.py:206-217 (make_sht).
 *   sle_solver_*  solver.py:521-644 (SeaLevelSolver.__init__, step 0),
 *                 solver.py:814-1144 (SeaLevelSolver.step) and the
 *                 fixed-point-preserving options of solver_opt.py:267-979
 *                 (dsl, diag, inner="extrap", reuse="warm").
 */
#ifndef SLEVOLVE_B200_H
#define SLEVOLVE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SLE_ABI_VERSION 1

enum sle_status {
  SLE_OK = 0,
  SLE_ERR_BAD_SHAPE = 1,     /* ValueError in the reference (sht.py:152-155) */
  SLE_ERR_BAD_ARG = 2,       /* ValueError (solver_opt.py:282-301) */
  SLE_ERR_OOM = 3,           /* device allocation failed */
  SLE_ERR_CUDA = 4,          /* a CUDA runtime call failed */
  SLE_ERR_NONCONVERGED = 5,  /* RuntimeError at 9999 inner iterations (solver.py:1049-1050) */
  SLE_ERR_NONFINITE = 6,     /* NaN / Inf met in the inner loop or in the inputs */
  SLE_ERR_UNSUPPORTED = 7,   /* an option of the reference this build does not provide */
  SLE_ERR_STATE = 8,         /* call out of order (e.g. step before init) */
  SLE_ERR_TIMEOUT = 9        /* a device-side wait gave up (bounded waits; results invalid) */
};

/* Arithmetic of the transforms.  FP64: FP64 end to end (matches the reference to 1e-9 m).
 * MIXED: Legendre contractions as split-TF32 (3xTF32) tensor-core GEMMs with FP32 accumulation
 * (operands rounded to FP32, then split into TF32 hi + lo: 22 significant bits) and FP32 row FFTs; the Legendre recurrence (tables computed in FP64), Gauss nodes and weights, the
 * degree-0 coefficient of every analysis and synthesis and everything outside the transforms stay
 * FP64. */
enum sle_precision { SLE_PREC_FP64 = 0, SLE_PREC_MIXED = 1 };

enum sle_layout { SLE_LAYOUT_DENSE = 0, SLE_LAYOUT_PACKED = 1 };

/* ------------------------------------------------------------------ misc */
int sle_abi_version(void);
const char* sle_last_error(void);

/* ------------------------------------------------------------ transforms */
typedef struct sle_sht sle_sht;

/* sht.py:151-255: nlat even, lmax <= nlon/2; nlon must be a power of two >= 8. */
int sle_sht_create(int nlat, int nlon, int lmax, sle_sht** out);
int sle_sht_destroy(sle_sht* plan);
/* sizes: ncoef = packed length (lmax+1)(lmax+2)/2 */
int sle_sht_info(const sle_sht* plan, int* nlat, int* nlon, int* lmax, long long* ncoef);
/* fraction of the (l, m, latitude) Legendre work that is not skipped as negligible (|P~| < 1e-35) */
int sle_sht_work_fraction(const sle_sht* plan, double* frac);
/* Gauss-Legendre nodes mu_j (north -> south) and weights, computed on the device (sht.py:65-101). */
int sle_sht_gauss(const sle_sht* plan, double* mu_host, double* w_host);
/* sht.py:274-302.  nfields grids -> nfields coefficient arrays (device pointers; the pointer
 * arrays themselves are host arrays of length nfields): 1 <= nfields <= 4 with the dense layout,
 * <= 256 with the packed one. */
int sle_sht_analysis(sle_sht* plan, int nfields, const double* const* grids_dev,
                     void* const* coeffs_dev, int layout, void* stream);
/* sht.py:305-343.  Im of the m = 0 coefficients is ignored (irfft semantics).  Field counts as
 * for sle_sht_analysis. */
int sle_sht_synthesis(sle_sht* plan, int nfields, const void* const* coeffs_dev, int layout,
                      double* const* grids_dev, void* stream);
/* Analysis of one grid into packed coefficients without any device allocation.  No counterpart
 * in the reference.  For hosts that reserve the GPU's memory for their own allocator and do not
 * let a library call cudaMalloc once they run: they create the plan while setting up and then
 * analyse through this call, whose scratch is a 4 MiB array compiled into this library (held by
 * every GPU that loads it, until exit) instead of memory from cudaMalloc.  Limits: at most 512
 * latitudes and lmax 511, else SLE_ERR_BAD_SHAPE.  The first call on a device looks up the
 * array's device address and should come before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (other streams, other threads) race and must be ordered
 * by the caller.  The arithmetic is always FP64, whatever sle_sht_set_precision selected on the
 * plan (a mixed-precision plan gives the FP64 result here). */
int sle_sht_analysis_noalloc(sle_sht* plan, const double* grid_dev, void* coeffs_packed_dev,
                             void* stream);
/* Select the arithmetic of sle_sht_analysis / sle_sht_synthesis on this plan (default FP64).
 * MIXED needs nlat a multiple of 64 and lmax <= 511; no counterpart in the reference. */
int sle_sht_set_precision(sle_sht* plan, int precision);
/* Launch shape of the mixed-precision transforms; no counterpart in the reference (its precedent
 * is the Fortran OTF/GEMM hybrid switch chosen by field count, otf_kernels.inc:463-516).
 * fields_per_launch 1..32 (a transform list is cut into launches of at most this many fields),
 * stages 2 or 4 (pipeline depth of the tensor-core kernel), fold_rows 4 or 8 (rows per block of
 * the row-FFT fold).  The results do not depend on it; slevolve_b200.tuning picks it by timing. */
typedef struct {
  int fields_per_launch;
  int stages;
  int fold_rows;
} sle_mx_tuning;
int sle_sht_set_tuning(sle_sht* plan, const sle_mx_tuning* t);
int sle_sht_get_tuning(const sle_sht* plan, sle_mx_tuning* t);
/* dense <-> packed conversion of one complex128 spectrum (device buffers) */
int sle_sht_pack(sle_sht* plan, const void* dense_dev, void* packed_dev, void* stream);
int sle_sht_unpack(sle_sht* plan, const void* packed_dev, void* dense_dev, void* stream);

/* -------------------------------------------------------------- solver */
typedef struct sle_solver sle_solver;

typedef struct {
  int nlat, nlon, lmax;
  double dt_years;          /* step length (yr), solver.py:529 */
  double epsilon1;          /* inner tolerance, solver.py:534 */
  int tpw;                  /* rotational feedback */
  int checkmarine;          /* flotation test on the ice load */
  int calcRG;               /* radial displacement / geoid */
  int opt_dsl;              /* deltasl = dsl + conserv*K00 (solver_opt.py:320-325) */
  int opt_diag;             /* degree-0 diagnostics by row sums (solver_opt.py:893-916) */
  int inner_extrap;         /* inner="extrap" first guess (solver_opt.py:148-165) */
  /* Planet (solver.py:98-110) */
  double radius, mass, rhoi, rhow, gacc, omega, moiA, moiC, kf;
  int precision;            /* sle_precision of the step's transforms */
} sle_config;

typedef struct {
  int nmodes;               /* K = max modes per degree */
  const int* nmod;          /* [lmax+1] modes of each degree */
  const double* s;          /* [K][lmax+1] inverse relaxation times (1/kyr) */
  const double* a_sl;       /* [K][lmax+1] (r' - r)/s  (solver.py:261-282) */
  const double* a_rr;       /* [K][lmax+1] r/s */
  const double* ttl;        /* [lmax+1] 4 pi a^3 / (M (2l+1)), 0 at l = 0 (solver.py:596-603) */
  const double* ttlekhl;    /* [lmax+1] ttl (1 + k_l - h_l) */
  const double* ttlhe;      /* [lmax+1] ttl h_l */
  const double* a_il;       /* [K] degree-2 rotational weights */
  const double* a_m;
  const double* a_tsl;
  const double* a_trr;
  double kTE2, hTE2, kE2;   /* tidal k, h and load k at degree 2 */
} sle_earth;

typedef struct {
  int iter;                 /* step counter (1-based) */
  int numiter;              /* inner iterations of the step */
  int status;               /* sle_status of the step */
  int gr_reguess;           /* grounded re-guesses this step */
  int gr_ice_analyses;      /* ice re-analyses this step */
  double xi;                /* last convergence ratio */
  double ocean_area, oceanBeta_area, gmslc_ocn, gmslc_ocnBeta, ice_volume;
  double il[9];             /* [3][3] */
  double mm[3];
  double lam[18];           /* [3][3] complex (re, im) */
} sle_step_info;

enum sle_field {
  SLE_F_TGRID = 0,          /* topography after the step (grid) */
  SLE_F_OCEAN = 1,          /* ocean function (grid of 0/1) */
  SLE_F_BETA = 2,           /* grounded-ice complement mask (grid of 0/1) */
  SLE_F_R = 3,              /* radial displacement (grid) */
  SLE_F_G = 4,              /* deltasl + R (grid) */
  SLE_F_DELTASL = 5,        /* sea-level change (grid) */
  SLE_F_DS_CONVERGED = 6,   /* converged ocean-load spectrum (dense complex) */
  SLE_F_LOAD_INC = 7,       /* converged load increment spectrum (dense complex) */
  SLE_F_ICESTAR = 8,        /* grounded ice (grid) */
  SLE_F_OCEAN0 = 9,         /* step-0 ocean function cxy0 (grid) */
  SLE_F_BETA0 = 10          /* step-0 grounded-ice complement beta0 (grid) */
};

int sle_solver_create(const sle_config* cfg, const sle_earth* earth, sle_solver** out);
int sle_solver_destroy(sle_solver* s);
/* step 0 (solver.py:550-581).  topo0, ice0: grids; *_on_device selects host or device pointers. */
int sle_solver_init(sle_solver* s, const double* topo0, const double* ice0, int on_device,
                    double* ocean_area0, double* oceanBeta_area0, double* ice_volume0);
/* one time step (solver.py:814-1144).  dt_years <= 0 keeps the current step length. */
int sle_solver_step(sle_solver* s, const double* ice, int on_device, double dt_years,
                    sle_step_info* info);
/* copy one output of the last step; dst is host or device memory. */
int sle_solver_get(sle_solver* s, int field, void* dst, int dst_on_device);
/* Analytic rates read-out (solver.py:464-484, 722-806; FP64 solves).  set_rate_tables(tab): the
 * weights of the following steps, host doubles [w_sl (K x (lmax+1)), w_rr (K x (lmax+1)),
 * ws_sl, ws_rr, wsphi_sl, wsphi_rr (lmax+1 each)] with K the solver's mode capacity (the
 * reference's ExactMemory.w_sl, w_rr and their sums for the step length, solver.py:293-294,
 * 347-362); NULL turns the read-out off.  While on, every step also forms, before its commit, the
 * rate spectra of sea level and radial displacement without the degree-2 rotational terms.
 * get_rates after a step: dsl, drr dense complex128 [lmax+1][lmax+1] (host); rec (20 doubles:
 * dI*_00 of the step (re, im), then the rotational totals committed before it: il (9), m (3),
 * Lambda degree 2 (3 complex)); rot (18 K doubles: the degree-2 modal states after the step's
 * advance and before its commit, r_il [K][9], r_m [K][3], r_Lambda [K][3 complex]).
 * SLE_ERR_STATE without tables. */
int sle_solver_set_rate_tables(sle_solver* s, const double* tab);
int sle_solver_get_rates(sle_solver* s, void* dsl, void* drr, double* rec, double* rot);
/* Horizontal read-out (solver.py:424-448, 687-720; output only).  set_horizontal(tab): host
 * doubles [a_hl (K x (lmax+1)) = l_k / s_k per mode and degree, then ttl l^E (lmax+1)]; NULL
 * turns it off.  While on, every step forms before its commit the potential
 * Psi = ttl l^E (rhoi dI* + rhow dS_prev + rhow load) + ttl sum_k a_hl R_k (degree 0 zero, the
 * degree-2 rotational term left to the caller).  get_horizontal after a step: psi dense
 * complex128 [lmax+1][lmax+1] (host), r_lam (6 K doubles: the degree-2 modal Lambda states,
 * [K][3 complex]) and lam12 (12 doubles: the degree-2 Lambda committed before the step and the
 * step's increment, 3 complex each).  SLE_ERR_STATE while off. */
/* Second-order load placement ("ramp", solver.py:229-240, 348-368, 450-499, 904-991, 1065-1067):
 * the step's load increment accrues linearly over the step, so each mode already holds 1 - phi_k
 * of its response at the step's end.  tab: host doubles for the coming steps' length,
 * [omphi = 1 - phi (K x (lmax+1)), ttl c_sl (lmax+1), ttl c_rr (lmax+1), c_il, c_m, c_tsl, c_trr]
 * (the reference's ExactMemory coefficients); NULL turns the placement off. */
int sle_solver_set_ramp(sle_solver* s, const double* tab);
int sle_solver_set_horizontal(sle_solver* s, const double* tab);
int sle_solver_get_horizontal(sle_solver* s, void* psi, double* r_lam, double* lam12);
/* Cross-pass warm start, reuse="warm" (solver_opt.py:400-403, 514-528, 932-947): a store in
 * device memory kept by the caller across solves of the same ice history (outer iterations,
 * run_outer.py).  ds_store: [capacity][ncoef] complex128 (packed), 16-byte aligned; mask_store:
 * [capacity][nlat*nlon] bytes.  Step k (1-based, k <= capacity) records its converged load
 * increment and ocean function at entry k-1; when k <= valid (entries of an earlier pass) the step
 * first starts from them instead of the eustatic / extrapolated guess.  ds_store = NULL: off. */
int sle_solver_set_reuse(sle_solver* s, void* ds_store, void* mask_store, int capacity, int valid);
/* the solver's own CUDA stream (as void*) */
int sle_solver_stream(sle_solver* s, void** stream);
/* Snapshot / restore of the solve's whole state as a host byte image (checkpoint, preemption,
 * migration between solvers or batch slots).  Replaces the reference's modal-state checkpoint
 * (fortran/src/modal_state_mod.f90:445-477: shapes, decay, loads and modal states to a stream
 * file) and the Python solver's swappable `state` object (tests/test_small_case.py:106); the image
 * is this library's own format: header (magic "SLES", configuration, step count, step lengths),
 * then every per-solve device buffer.  A restored solve continues bit for bit as the original
 * would have.  The image restores into any solver or batch slot of the same grid, lmax, mode
 * capacity, precision and option flags (else SLE_ERR_BAD_SHAPE); a reuse store and the read-out
 * tables (rates, horizontal, ramp) are not part of it and are set again by the caller.
 * _bytes gives the image size; dst / src are host buffers of at least that many bytes. */
int sle_solver_snapshot_bytes(const sle_solver* s, long long* nbytes);
int sle_solver_snapshot(sle_solver* s, void* dst, long long nbytes);
int sle_solver_restore(sle_solver* s, const void* src, long long nbytes);

/* ------------------------------------------------------------- batches
 * A batch holds nslots independent solves ("slots") of one grid size and configuration (the
 * sle_config flags and precision are shared; Earth model, step length, topography and ice history
 * are per slot).  One sle_batch_step advances every slot given ice in the call by one time step
 * with the launches of a single solve; slots converge independently (a converged slot is skipped
 * by the remaining inner iterations).  A slot's results do not depend on the other slots.  Slots
 * are loaded, stepped and released at any time between steps (continuous batching).  No
 * counterpart in the reference, which runs one solve per process; each slot follows
 * SeaLevelSolver.step (solver.py:814-1144). */
typedef struct sle_batch sle_batch;

/* max_modes: the largest Earth-model mode count any slot will use. */
int sle_batch_create(const sle_config* cfg, int nslots, int max_modes, sle_batch** out);
int sle_batch_destroy(sle_batch* b);
/* Load a slot: Earth model, step length (yr), then step 0 (solver.py:550-581) on topo0 / ice0. */
int sle_batch_load(sle_batch* b, int slot, const sle_earth* earth, double dt_years, const double* topo0,
                   const double* ice0, int on_device, double* ocean_area0, double* oceanBeta_area0,
                   double* ice_volume0);
/* The slot no longer steps (its memory is reused by the next load; its reuse store is dropped). */
int sle_batch_release(sle_batch* b, int slot);
/* reuse store of a slot, as sle_solver_set_reuse; kept across sle_batch_load of the slot */
int sle_batch_set_reuse(sle_batch* b, int slot, void* ds_store, void* mask_store, int capacity, int valid);
/* One step of every slot with ice[slot] != NULL (ice: array of nslots grid pointers).
 * dt_years: NULL, or nslots values (> 0 changes that slot's step length).  info: nslots records,
 * filled for the slots that stepped.  Returns SLE_OK, or the status of the first slot that failed
 * (its record says which; failed slots are not committed, the others are). */
int sle_batch_step(sle_batch* b, const double* const* ice, int on_device, const double* dt_years,
                   sle_step_info* info);
/* sle_batch_step in two halves, so that the caller can overlap a step with its own work (e.g.
 * the upload of the next step's ice on another stream): _begin enqueues the step on the batch's
 * stream and returns; _end waits for it and fills info as sle_batch_step does.  Between the two,
 * the ice buffers given to _begin must stay valid and unchanged, and no other sle_batch_* call
 * on this batch is allowed (they return SLE_ERR_STATE).  No counterpart in the reference. */
int sle_batch_step_begin(sle_batch* b, const double* const* ice, int on_device, const double* dt_years);
int sle_batch_step_end(sle_batch* b, sle_step_info* info);
/* snapshot / restore of one slot, as sle_solver_snapshot / sle_solver_restore (an image of one
 * slot restores into any slot of a batch of the same configuration, or into a solver) */
int sle_batch_snapshot_bytes(const sle_batch* b, long long* nbytes);
int sle_batch_snapshot(sle_batch* b, int slot, void* dst, long long nbytes);
int sle_batch_restore(sle_batch* b, int slot, const void* src, long long nbytes);
/* copy one output of a slot's last step (as sle_solver_get) */
int sle_batch_get(sle_batch* b, int slot, int field, void* dst, int dst_on_device);
int sle_batch_stream(sle_batch* b, void** stream);
/* launch shape of the batch's mixed-precision transforms (as sle_sht_set_tuning) */
int sle_batch_set_tuning(sle_batch* b, const sle_mx_tuning* t);
/* slots, mode capacity and the device bytes the batch's solver state occupies */
int sle_batch_info(const sle_batch* b, int* nslots, int* max_modes, long long* device_bytes);

/* ----------------------------------------------------------- ice history */
/* out[i] = (1 - w) a[i] + w b[i] for i < n, on the device, with NumPy's elementwise roundings
 * (1 - w once, two products, one sum, no fused multiply-add): the blended entry "i:j:w" of the
 * outer driver's custom ice history (run_outer.py:156-174, option --ice-seq), formed from two
 * snapshots already on the device; out must not overlap a or b.  stream: a cudaStream_t (NULL =
 * the legacy default stream).
 * SLE_ERR_BAD_ARG for a negative n or a NULL buffer with n > 0. */
int sle_ice_blend(double* out, const double* a, const double* b, double w, long long n, void* stream);

/* The water-volume residual of the segmented initial-topography guess
 * (init_topo_segmented.py:84-90) for T0 = (tp + c) + s on an nlat x nlon grid: out2[0] = sum of
 * max(-T0, 0) C0 area, out2[1] = sum of (I0 g0 - Ip gp) area, with g0 = grounded(i0, T0)
 * (i0 > 0 and (T0 > 0 or rhoi i0 > rhow |T0|)), C0 = T0 < 0 and not g0, area = wrow[row]; gp the
 * present grounded mask (bytes).  Deterministic sums (fixed partition, fixed order).  scratch:
 * sle_topo_scratch_bytes() device bytes, zero before the first call and left so by each call.
 * Synchronises the stream (the host reads out2). */
int sle_topo_residual(const double* tp, const double* s, double c, const double* i0, const double* ip,
                      const unsigned char* gp, const double* wrow, int nlat, int nlon, double rhoi, double rhow,
                      void* scratch, double* out2, void* stream);
long long sle_topo_scratch_bytes(void);

/* ------------------------------------------------------- measurement */
/* Kernel classes timed by sle_prof_*: 0 row FFT + fold, 1 Legendre analysis, 2 Legendre
 * synthesis, 3 inverse FFT + unfold, 4 modal-state advance, 5 the Legendre analysis of the inner
 * iteration's rO field (every stepping slot's field active; class 1 has the other analyses),
 * then the inner loop's elementwise passes, their units being the slots still iterating:
 * 6 eq. B18, 7 conservation / load update / xi, 8 deltasl + ocean function + grounded test,
 * 9 C* refresh, 10 dI after a grounded-mask change.
 * Timing is off by default; when on, each launch of these classes is bracketed by CUDA events on
 * its own stream. */
int sle_prof_enable(int on);
int sle_prof_collect(void);        /* wait for recorded events and accumulate */
int sle_prof_reset(void);          /* also resets the launch counter */
/* accumulated device milliseconds, launch count and fields processed ("units") of a class */
int sle_prof_read(int cls, double* ms, long long* count, double* units);
/* kernels launched by this library since the last sle_prof_reset() */
long long sle_launch_count(void);
/* Launch mode of the inner loop's elementwise kernels, the row-FFT fold and the unfold: 1 launches
 * each as a programmatic dependent of the kernel before it in its stream (scheduled while that
 * kernel drains; it waits for that kernel's completion before touching memory, so results do not
 * change), 0 as plain launches.  The initial mode is 1 unless the environment variable
 * SLEVOLVE_B200_NO_PDL is set to a non-empty value other than "0".  Applies to work enqueued or
 * captured afterwards: a batch keeps the mode its loop graph was captured with.  *previous (may
 * be NULL) receives the mode before the call.  No counterpart in the reference. */
int sle_set_programmatic_launch(int on, int* previous);
/* FP64 FMA throughput of the current device (TFLOP/s), from a timed dependent-free FMA kernel */
int sle_probe_fp64_tflops(double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* SLEVOLVE_B200_H */
