/*
 * larmor_b200 — C ABI of the B200-native voxelwise fitting hot path of Larmor (larmor-dmri).
 *
 * Every entry point returns an int status (LAR_OK = 0) and never throws; lar_last_error()
 * gives the message of the last failure on the calling host thread. Per-voxel numerical
 * failure never fails a call: it is encoded in the outputs (fallback parameters, flags), as in
 * the reference. Array arguments are plain pointers with explicit sizes, row-major, one voxel
 * per row. "device" arrays live in the current CUDA device's memory; "host" arrays in host
 * memory. `stream` is a cudaStream_t (NULL for the legacy default stream); the calls are
 * asynchronous on it unless stated otherwise.
 *
 * Design handles copy their matrices at creation (to host and device memory) and are
 * immutable afterwards, as the reference's design objects are (cpp/src/python/sd.cpp:42-62).
 *
 * Reference interfaces replaced (paths within the larmor-dmri project):
 *   lar_log_design_*, lar_fit_log_signal     larmor._core.fit_log_signal
 *                                            (cpp/src/python/dwi.cpp:42, src/larmor/_core.pyi:223)
 *   lar_fit_dti_maps                         DTIModel.fit's chunk loop + compute_dti_metrics
 *                                            (src/larmor/dwi/dti.py:156-163, :170-235)
 *   lar_fit_dki_maps, lar_dki_maps           DKIModel.fit's chunk loop + compute_kurtosis_metrics
 *                                            (src/larmor/dwi/dki.py:243-282, :285-540)
 *   lar_lsi_design_*, lar_fit_lsi            larmor._core.LsiDesign, larmor._core.fit_lsi
 *                                            (cpp/src/python/sd.cpp:361-392, cpp/src/sd/lsi.cpp)
 *   lar_l2nnls_create, lar_fod_solver_*      larmor._core.FodSolver.l2nnls (cpp/src/python/sd.cpp:89)
 *   lar_deconv_kernel_*                      larmor._core.DeconvKernel (cpp/src/python/sd.cpp:260)
 *   lar_fit_multi_tissue                     larmor._core.fit_multi_tissue (cpp/src/python/sd.cpp:310,
 *                                            cpp/src/sd/multi_tissue.cpp:76-148)
 *   lar_fit_single_tissue                    larmor._core.fit_single_tissue (cpp/src/sd/solver.cpp:422)
 */
#ifndef LARMOR_B200_H
#define LARMOR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LAR_OK 0
#define LAR_ERR_INVALID 1 /* bad shape, size or argument: ValueError in the Python layer */
#define LAR_ERR_CUDA 2    /* a CUDA runtime call failed */
#define LAR_ERR_MEMORY 3  /* out of host or device memory */

/* Arithmetic of a fit: FP64 follows the reference's double precision; FP32 is the plain
 * single-precision variant of the same kernels, kept as the comparison baseline. */
#define LAR_FP64 0
#define LAR_FP32 1
#define LAR_TF32X3 2 /* dRL only: products on the tensor cores as three TF32 products, FP32 state */

/* Sample types of a raw volume for lar_stage_dwi. */
#define LAR_DTYPE_F32 0
#define LAR_DTYPE_F64 1
#define LAR_DTYPE_I16 2
#define LAR_DTYPE_U16 3
#define LAR_DTYPE_I8 4
#define LAR_DTYPE_U8 5
#define LAR_DTYPE_I32 6
#define LAR_DTYPE_U32 7

/* Message of the last failed call on this host thread ("" if none). */
const char* lar_last_error(void);

/* Library version string. */
const char* lar_version(void);

/* ---- Launch accounting ----------------------------------------------------------------
 * No counterpart in the reference (its fits run on host threads). Every kernel launch of the
 * library is counted; with timing on, each is bracketed by CUDA events on its stream so that a
 * benchmark can time one kernel of a multi-kernel call. */

/* Kernels the library has launched since it was loaded. */
int64_t lar_launch_count(void);

/* Launch settings a tuner may set (no counterpart in the reference): "dti.voxels_per_cta"
 * (16, 32 or 64; used when the table fits), "log.warp.waves" (resident-CTA waves of the
 * warp-per-voxel log fit's grid, default 4), and the resident CTAs per SM of the persistent
 * grids, "dki.refit.ctas_per_sm", "lsi.ctas_per_sm", "sd.nnls.ctas_per_sm" and
 * "sd.fractions.ctas_per_sm" (at most the occupancy limit). 0 restores the library's choice.
 * Results do not depend on them; an unknown name or a value out of range is LAR_ERR_INVALID. */
int lar_set_launch_setting(const char* name, int64_t value);
int lar_get_launch_setting(const char* name, int64_t* value);

/* Turns per-kernel event timing on (enable != 0) or off; either way clears the records. */
int lar_kernel_timing(int enable);

/* Total device time (ms) and number of the timed launches of kernel `name` (as the library
 * names it, e.g. "lsi_kernel", "ridge_nnls_kernel<2,2>"); waits for their events. */
int lar_kernel_time(const char* name, double* total_ms, int64_t* launches);

/* ---- Log-signal fits (DTI, DKI) ------------------------------------------------------- */

typedef struct lar_log_design_s* lar_log_design;

/* Prepares the design x (n, p), n >= p, of full column rank, and constraints g (m, p), m >= 0
 * (host arrays): unit-norm columns, the pseudo-inverse, the constraints with the same column
 * scales. Replaces make_log_signal_design (cpp/src/dwi/log_fit.cpp:220). */
int lar_log_design_create(const double* x, int64_t n, int64_t p, const double* g, int64_t m,
                          lar_log_design* out);
void lar_log_design_destroy(lar_log_design design);

/* The number of voxels of the last constrained fit on this design whose fit broke a
 * constraint and took the constrained re-fit (0 without constraints). Read it after that
 * call's stream has finished. A diagnostic with no counterpart in the reference. */
int lar_log_design_violators(lar_log_design design, int64_t* count);

/* Fits each row of log_s (v, n) (device) by least squares on the design: ordinary, or
 * weighted by the predicted signal iterated until no predicted log signal changes by more than
 * tol or for max_iter weighted fits; a voxel whose weighted normal equations are singular or
 * whose fit is not finite keeps the ordinary fit. With constraints, a voxel with g p < 0 in
 * some row is fitted again subject to g p >= 0 (least distance by NNLS) and flagged in broke.
 * Writes params (v, p) (device, double) and broke (v,) (device, uint8). iterations (v,)
 * (device, int32, may be NULL) receives each voxel's number of weighted fits.
 * Replaces larmor._core.fit_log_signal (cpp/src/python/dwi.cpp:42-82). */
int lar_fit_log_signal(lar_log_design design, const double* log_s, int64_t v, int weighted,
                       int64_t max_iter, double tol, int precision, double* params,
                       uint8_t* broke, int32_t* iterations, void* stream);

/* The fused DTI path of DTIModel.fit: float32 signals (v, n) (device) are floored (a sample
 * that is not finite and positive becomes floor[voxel], device double (v,)), logged, fitted as
 * lar_fit_log_signal does (design columns [1, -b_matrix]), and turned into the maps of
 * compute_dti_metrics. maps (16, v) (device float32, one row per map) holds dt (6: xx, xy, xz,
 * yy, yz, zz), fa, md, ad, rd, pe (3), eigen_vals (3, descending); npd (v,) (device uint8) is
 * l3 <= 0. params (v, 7) (device double) may be NULL. */
int lar_fit_dti_maps(lar_log_design design, const float* signals, const double* floor,
                     int64_t v, int weighted, int64_t max_iter, double tol, int precision,
                     float* maps, uint8_t* npd, double* params, void* stream);

/* The DKI maps of 22-parameter fits params (v, 22) (device double): maps (36, v) (device
 * float32) holds rows 0-15 as lar_fit_dti_maps, rows 16-30 kt (W1111 ... W3312), row 31 s0,
 * rows 32-35 mk, ak, rk, ka; npd (v,) is l3 <= 0. Replaces compute_kurtosis_metrics and the
 * map assembly of DKIModel.fit (src/larmor/dwi/dki.py:261-282, :285-342). */
int lar_dki_maps(const double* params, int64_t v, float* maps, uint8_t* npd, void* stream);

/* The fused DKI path of DKIModel.fit: float32 signals (v, n) (device) are prepared as the
 * reference does (src/larmor/dwi/dki.py:243-250): with s0 (v,) (device double, or NULL for a
 * table without b0) the b0 samples of a voxel whose own b0 mean differs from s0 become s0 and
 * the diffusion-weighted samples are capped at s0; samples that are not finite and positive
 * become floor[voxel]. is_b0 (n,) (device uint8) marks the b0 measurements. The log signals
 * are fitted (constrained when the design has constraints; the re-fit of violators runs in
 * FP64), params (v, 22) (device double, required) receives the parameters, broke (v,) the
 * constraint flags, and maps/npd the maps of lar_dki_maps. */
int lar_fit_dki_maps(lar_log_design design, const float* signals, const double* s0, const double* floor,
                     const uint8_t* is_b0, int64_t v, int weighted, int64_t max_iter, double tol,
                     int precision, float* maps, uint8_t* npd, uint8_t* broke, double* params,
                     void* stream);

/* ---- Least squares with inequality constraints (MSMT-CSD) ----------------------------- */

typedef struct lar_lsi_design_s* lar_lsi_design;

/* Prepares min ||a x - s||^2 + ridge^2 ||x||^2 subject to g x >= 0 for a (m, n) and g (k, n)
 * (host arrays), n <= 63: the column-pivoted QR of [a; ridge I], q_t, P R^-1, the unit-row
 * E = G P R^-1, its Gram and absolute row sums, in FP64, copied to the device. Fails with
 * LAR_ERR_INVALID when [a; ridge I] does not have full column rank or ridge < 0.
 * Replaces larmor._core.LsiDesign (cpp/src/python/sd.cpp:361, cpp/src/sd/lsi.cpp:75). */
int lar_lsi_design_create(const double* a, int64_t m, int64_t n, const double* g, int64_t k, double ridge,
                          lar_lsi_design* out);
void lar_lsi_design_destroy(lar_lsi_design design);

/* Copies the prepared matrices to host arrays (any may be NULL): q_t (n, m), back (n, n),
 * e (k, n), gram (k, k), abs_sums (k,). */
int lar_lsi_design_matrices(lar_lsi_design design, double* q_t, double* back, double* e, double* gram,
                            double* abs_sums);

/* Solves the problem for every row of signals (v, m) (device double): x (v, n) (device double)
 * and converged (v,) (device uint8), 0 where the NNLS stopped at its limit of inner steps.
 * Optional (NULL to skip): status (v,) 0 Cholesky path, 1 QR fallback, 2 no bound active;
 * outer (v,) int32 outer steps; active (v, k) uint8 the constraints with a non-zero
 * multiplier. only_qr forces the fallback (cpp/src/sd/lsi.cpp:346). Calls on one design handle
 * must not overlap on the GPU (they share its scratch).
 * Replaces larmor._core.fit_lsi (cpp/src/python/sd.cpp:370-392). */
int lar_fit_lsi(lar_lsi_design design, const double* signals, int64_t v, int only_qr, double* x,
                uint8_t* converged, uint8_t* status, int32_t* outer, uint8_t* active, void* stream);

/* The plain single-precision LSI fit, the comparison baseline of lar_fit_lsi (no counterpart in
 * the reference): float32 signals (v, m) (device) in, float32 solutions x (v, n) (device) out;
 * one warp per voxel runs the reference's steps in FP32 with the Cholesky factor of the active
 * constraints formed anew for every fit and no QR fallback. status (v,) (device uint8, may be
 * NULL): 0 converged, 1 the factor failed or more than 64 constraints became active, 2 f = 0
 * (the unconstrained solution), 3 a step limit. */
int lar_fit_lsi_plain_fp32(lar_lsi_design design, const float* signals, int64_t v, float* x, uint8_t* status,
                           void* stream);

/* ---- Multi-tissue spherical deconvolution (SDModel, method mFOD) ---------------------- */

typedef struct lar_fod_solver_s* lar_fod_solver;
typedef struct lar_deconv_kernel_s* lar_deconv_kernel;

/* Prepares the ridge-penalised NNLS min ||k f - s||^2 + reg^2 ||f||^2 over f >= 0 for the
 * weighted anisotropic kernel k (m, c) (host): its Gram k^T k + reg^2 I and whether the fits
 * use the normal equations (reg = 0, or a condition bound (||k||_F^2 + reg^2) / reg^2 <= 1e8;
 * otherwise QR). A coefficient enters only when its gradient exceeds tol_x. Fails with
 * LAR_ERR_INVALID for reg < 0 or tol_x <= 0. Replaces FodSolver.l2nnls
 * (cpp/src/python/sd.cpp:89-102, cpp/src/sd/nnls.cpp:348-360). */
/* FodSolver.drl (cpp/src/python/sd.cpp:127-145): a damped Richardson-Lucy solver
 * (cpp/src/sd/drl.cpp:39-100) of K^T (c, m) and K^T K (c, c), host arrays copied: damping
 * threshold nu, at most n_iter (>= 0) iterations per voxel, every amplitude started at init.
 * c <= 640, m > 1. lar_fit_single_tissue runs it; lar_fit_multi_tissue takes it for either
 * resolution (GRL: each round's and the final FODs by dRL on the anisotropic signal,
 * cpp/src/sd/multi_tissue.cpp:40-95). */
int lar_drl_create(const double* k_t, const double* k_t_k, int64_t c, int64_t m, double nu, int64_t n_iter,
                   double init, lar_fod_solver* out);

int lar_l2nnls_create(const double* k, int64_t m, int64_t c, double reg, double tol_x, lar_fod_solver* out);

/* The arithmetic of a dRL solver's fits (no reference counterpart: the reference computes in
 * double). LAR_FP64 (the default): the FP64 kernels, the reference's arithmetic. LAR_TF32X3:
 * for 65 to 320 directions, each iteration's product K^T K f on the tcgen05 tensor cores as
 * three TF32 products with FP32 accumulation (the operands split into TF32 heads and FP32
 * remainders), the amplitudes and their update in FP32: FODs within 1e-4 of the voxel's
 * largest amplitude of the FP64 fit. Fails with LAR_ERR_INVALID for another solver, precision
 * or size. */
int lar_drl_set_precision(lar_fod_solver solver, int precision);

/* 1 in *out when a tensor-core dRL fit of this solver stopped at a bounded wait (its FODs are
 * then not valid), else 0. Waits for the device. */
int lar_drl_errors(lar_fod_solver solver, int* out);
void lar_fod_solver_destroy(lar_fod_solver solver);

/* One resolution of a multi-tissue kernel (host arrays): k_aniso (m, ca), k_iso and w_k_iso
 * (m, ci), and the (start, stop) columns of each anisotropic response, blocks (nb, 2). Fails
 * with LAR_ERR_INVALID for an empty block or one outside 0..ca. Replaces DeconvKernel
 * (cpp/src/python/sd.cpp:260-292). */
int lar_deconv_kernel_create(const double* k_aniso, int64_t m, int64_t ca, const double* k_iso,
                             const double* w_k_iso, int64_t ci, const int64_t* blocks, int64_t nb,
                             lar_deconv_kernel* out);
void lar_deconv_kernel_destroy(lar_deconv_kernel kernel);

/* Fits the FODs and tissue fractions of every row of signals (v, m) (device double, normalised
 * by S0): up to max_outer rounds of a low-resolution FOD fit and a fraction fit, until no
 * fraction changes by fraction_tol, then the high-resolution FOD and the final fractions (NNLS
 * tolerance final_tol_x), normalised to sum to 1. weights (m,) (host) are the shell weights of
 * the FOD fits. Writes fods (v, ca_hr) and fractions (v, nb_hr + ci) (device double); rounds
 * (v,) int32 and status (v,) uint8 (1 where an active set outgrew the QR workspace) may be
 * NULL. Without stream capture it reads each round's voxel count back on the host (waiting for
 * its stream once per round); under capture it enqueues max_outer rounds that read their counts
 * on the device (an earlier uncaptured call on these solvers must have used the same weights
 * and no fewer voxels). Calls sharing hr_solver must not overlap on the GPU.
 * Replaces larmor._core.fit_multi_tissue (cpp/src/python/sd.cpp:310-358). */
int lar_fit_multi_tissue(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                         lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                         int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                         double* fractions, int32_t* rounds, uint8_t* status, void* stream);

/* lar_fit_multi_tissue without host waits (no counterpart in the reference, whose rounds run on
 * host threads): every one of max_outer rounds is enqueued and reads its voxel count on the
 * device, exiting at once when it is 0, so the call returns as soon as the work is enqueued and
 * concurrent fits on other streams are not held up by host round trips. Results are those of
 * lar_fit_multi_tissue. The weights are copied at the call (the host buffer may be reused after
 * it returns). */
int lar_fit_multi_tissue_async(const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                               lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                               int64_t max_outer, double fraction_tol, double final_tol_x, double* fods,
                               double* fractions, int32_t* rounds, uint8_t* status, void* stream);

/* The plain single-precision multi-tissue fit, the comparison baseline of lar_fit_multi_tissue
 * (no reference counterpart: the reference computes in double only). The same model and
 * arguments in FP32: signals (v, m), FODs (v, ca_hr) and fractions (v, nb + ci) are device
 * floats, weights (m,) a host double array. One warp per voxel runs all its rounds in one kernel
 * with the textbook Lawson-Hanson steps (a Cholesky factor formed anew for every fit, at most 64
 * active columns, no QR fallback). Takes L2NNLS solvers, at most 512 measurements, 320
 * directions and 4 fraction columns. status (v,) gets 0, 1 (the factor failed) or 2 (a step
 * limit); rounds and status may be NULL. */
int lar_fit_multi_tissue_plain_fp32(const float* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                                    lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver,
                                    int64_t max_outer, double fraction_tol, double final_tol_x, float* fods,
                                    float* fractions, int32_t* rounds, uint8_t* status, void* stream);

/* Solves one non-negative least-squares problem, min ||c x - d|| over x >= 0, for c (m, n)
 * row-major and d (m,), device doubles, by Lawson-Hanson with QR fits and at most 3 n inner
 * steps (the fraction fits' solver). A column enters only when its gradient exceeds tol_x; with
 * default_tol != 0, tol_x = 10 eps norm1(c) max(m, n) instead. Writes x (n,) (device double).
 * m >= 1, 1 <= n <= 16. Replaces larmor._core.lsqnonneg (cpp/src/python/sd.cpp:208-228,
 * cpp/src/sd/nnls.cpp:187-258). */
int lar_lsqnonneg(const double* c, int64_t m, int64_t n, const double* d, int default_tol, double tol_x, double* x,
                  void* stream);

/* The FOD (v, c) of every row of signals (v, m) (device double) with one L2NNLS solver.
 * Replaces larmor._core.fit_single_tissue (cpp/src/python/sd.cpp, cpp/src/sd/solver.cpp:422). */
int lar_fit_single_tissue(const double* signals, int64_t v, lar_fod_solver solver, double* fods,
                          uint8_t* status, void* stream);

/* ---- FOD amplitudes to spherical harmonics ----------------------------------------------
 * The SD fit's _to_sh (src/larmor/sd/model.py:412-440, fit_sh src/larmor/sd/sh.py:134): the
 * least-squares SH fit of amplitudes on a sphere grid, as the product with a projector
 * P = density pinv(B) (ncoef, ca) that the caller forms once per (grid, lmax, basis). */
typedef struct lar_sh_projector_s* lar_sh_projector;

/* Copies the projector (ncoef, ca) (host, row-major) to the device. */
int lar_sh_projector_create(const double* projector, int64_t ncoef, int64_t ca, lar_sh_projector* out);

void lar_sh_projector_destroy(lar_sh_projector projector);

/* out (v, ncoef; row stride ldo) = amplitudes (v, ca; row stride lda) P^T, all device double;
 * with exact_integral the l = 0 coefficient is the amplitudes' sum / sqrt(4 pi) instead. */
int lar_project_sh(lar_sh_projector projector, const double* amplitudes, int64_t v, int64_t lda,
                   int exact_integral, double* out, int64_t ldo, void* stream);

/* ---- Single-shell CSD ----------------------------------------------------------------- */

/* The matrices of one shell's constrained spherical deconvolution, copied to the device
 * (_core.fit_csd's problem, cpp/src/sd/csd.cpp:11-22): initial (c0, m) maps a signal to the
 * first c0 <= c coefficients of the starting FOD, forward M (m, c), constraint C (k, c) the
 * weighted SH basis on the constraint directions; the Gram matrix M^T M + norm_weight I is formed
 * here. c <= 255, k <= 65535, max_iter >= 0; LAR_ERR_INVALID otherwise or when the packed
 * system does not fit a warp's shared memory. */
typedef struct lar_csd_s* lar_csd;

int lar_csd_create(const double* initial, int64_t c0, int64_t m, const double* forward, int64_t c,
                   const double* constraint, int64_t k, double norm_weight, double threshold, int64_t max_iter,
                   lar_csd* out);

void lar_csd_destroy(lar_csd csd);

/* _core.fit_csd (cpp/src/python/sd.cpp:171-209, cpp/src/sd/csd.cpp:24-65) for v signals (v, m),
 * device: fods (v, c) and converged (v,) (1 where the set of constrained directions repeated, or
 * max_iter is 0), device. Signals are fitted as given (the Python layer clamps them at 0). */
int lar_fit_csd(lar_csd csd, const double* signals, int64_t v, double* fods, uint8_t* converged, void* stream);

/* ---- Device input staging ------------------------------------------------------------- */

/* The inputs of a voxelwise fit from a raw DWI volume on the device, replacing the host steps of
 * src/larmor/dwi/inputs.py. volume is (nx, ny, nz, n) C-ordered samples of type dtype
 * (LAR_DTYPE_*), the stored values of Volume.data; voxels (v) the flat grid indices
 * ((x ny + y) nz + z) of the mask voxels, increasing (np.nonzero order); is_b0 (n) host flags of
 * the table's b0s. Writes, all device arrays:
 *   signals (v, n) float32: the samples converted to float32, then scaled by slope and intercept
 *       in float32 unless that is the identity (Volume.as_float / signal_rows,
 *       src/larmor/types/volume.py:116-123, src/larmor/dwi/inputs.py:137-172);
 *   s0 (v): estimate_s0 (src/larmor/dwi/inputs.py:78-134): the mean b0, and for a mask voxel whose
 *       mean b0 is at or below its mean diffusion-weighted sample, the mean S0 of the plausible mask
 *       voxels within 3x3x3, else 5x5x5, NaN when there is none. Required with b0s; untouched
 *       without;
 *   finite (v): 1 where every sample of the row is finite;
 *   floor (v) (may be NULL): floor_bad_samples' value for the row (src/larmor/dwi/inputs.py:
 *       227-252): 1e-3 S0 where S0 is finite and positive, else 1e-3 times largest;
 *   largest (1) (may be NULL): largest_finite_signal (src/larmor/dwi/inputs.py:212-224).
 * Allocates a stream-ordered workspace of 17 bytes per mask voxel and 4 per grid voxel. */
int lar_stage_dwi(const void* volume, int dtype, int64_t nx, int64_t ny, int64_t nz, int64_t n, double slope,
                  double intercept, const int64_t* voxels, int64_t v, const uint8_t* is_b0, float* signals, double* s0,
                  uint8_t* finite, double* floor, double* largest, void* stream);

/* The SD models' S0-normalised signals (src/larmor/sd/model.py:184-200): normalised (v, n) =
 * min(signals / s0, 1) in FP64, finite (v) = 1 where every quotient is finite. Device arrays. */
/* Puts map-major values (rows, v) (device floats) of the mask voxels back on the grid:
 * out(voxels[i], r) = values(r, i) with out (grid, rows) voxel-major, device floats; out's other
 * entries are left as they are (the caller fills them). Replaces the host unmask of the model
 * results (src/larmor/dwi/mask.py:139), so one copy of the grid maps leaves the device. */
int lar_unmask_rows(const float* values, int64_t rows, int64_t v, const int64_t* voxels, int64_t grid, float* out,
                    void* stream);

int lar_normalise_signals(const float* signals, const double* s0, int64_t v, int64_t n, double* normalised,
                          uint8_t* finite, void* stream);

/* ---- FOD peaks ------------------------------------------------------------------------ */

/* Series in the tournier basis: n_coeffs(lmax, full) = (lmax + 1)(lmax + 2) / 2 even degrees, or
 * (lmax + 1)^2 all degrees when full; lmax <= 20, even unless full. Each entry point returns
 * LAR_ERR_INVALID for another lmax, a row stride below the coefficient count or a negative
 * count, before any device work. */

/* A sphere for the peak search: nv unit vertices (nv, 3) and the indices of the 6 neighbours of
 * each (nv, 6; a vertex with 5 lists itself), host arrays copied to the device. Replaces the
 * sphere the reference builds per call in _core.peaks_chunk (cpp/src/python/sh.cpp:130-147):
 * LAR_ERR_INVALID when a neighbour index is outside [0, nv). */
typedef struct lar_peak_sphere_s* lar_peak_sphere;

int lar_peak_sphere_create(const double* vertices, const int64_t* neighbours, int64_t nv, lar_peak_sphere* out);

void lar_peak_sphere_destroy(lar_peak_sphere sphere);

/* _core.sh_derivatives (cpp/src/python/sh.cpp:69-82, cpp/src/sh/harmonics.cpp:139-196) for n
 * points: out (n, 6) = f, df/dtheta, df/dphi / sin theta, d2f/dtheta2, d2f/dtheta dphi / sin theta,
 * d2f/dphi2 / sin^2 theta of series i (row i of coeffs, stride ldc) at (theta[i], phi[i]). All
 * device arrays. */
int lar_sh_derivatives(const double* coeffs, int64_t n, int64_t ldc, int lmax, int full, const double* theta,
                       const double* phi, double* out, void* stream);

/* _core.climb (cpp/src/python/sh.cpp:84-108, cpp/src/sh/peaks.cpp:31-78) for n climbs: series i
 * from the unit vector starts[i] (n, 3) to directions (n, 3) and amplitudes (n), NaN where the
 * climb has not stopped within max_iters (>= 0) steps. All device arrays. */
int lar_climb(const double* coeffs, int64_t n, int64_t ldc, int lmax, int full, const double* starts, int max_iters,
              double tol, double max_step, double* directions, double* amplitudes, void* stream);

/* _core.peaks_chunk (cpp/src/python/sh.cpp:112-176, cpp/src/sh/peaks.cpp:80-133): the peaks of
 * n voxels' series (row stride ldc) from their amplitudes on the sphere's vertices (on_sphere,
 * row stride lds >= nv), largest first, into directions (n, n_peaks, 3) and amplitudes
 * (n, n_peaks), NaN where a voxel has fewer; symmetric series' peaks turned to z >= 0. n_peaks
 * >= 1, n < 2^31. All device arrays except the sphere. Waits for its stream once, to size the
 * list of the chunk's climbs; allocates stream-ordered workspaces of 20 bytes per voxel and 40
 * bytes per climb (one per local maximum of a voxel's amplitudes). */
int lar_find_peaks(lar_peak_sphere sphere, const double* coeffs, int64_t n, int64_t ldc, int lmax, int full,
                   const double* on_sphere, int64_t lds, int n_peaks, double relative_threshold, double threshold,
                   double* directions, double* amplitudes, void* stream);

/* ---- Batches: many volumes, one work queue per model family ---------------------------- */

/* A batch of volumes ("jobs") of the DTI, DKI and multi-tissue (mFOD) models, of different
 * sizes and gradient tables. Each family's stages run as single launches over all of the
 * family's volumes, whose CTAs or warps take (volume, voxel-block) tickets from one device
 * counter, as the reference's block queue does within a volume
 * (cpp/src/common/parallel.hpp:26-84); a volume's results equal those of its own fit
 * (lar_fit_dti_maps, lar_fit_dki_maps with LAR_FP64, lar_fit_multi_tissue). No reference
 * function takes several volumes at once: the batched-uneven workload is a driver loop over
 * volumes there. */
typedef struct lar_batch_s* lar_batch;

#define LAR_BATCH_DTI 1
#define LAR_BATCH_DKI 2
#define LAR_BATCH_MFOD 4

int lar_batch_create(lar_batch* out);
void lar_batch_destroy(lar_batch batch);

/* Adds a DTI volume: the arguments of lar_fit_dti_maps (device pointers, FP64, no params).
 * Every DTI job of a batch takes the same weighted, max_iter and tol. */
int lar_batch_add_dti(lar_batch batch, lar_log_design design, const float* signals, const double* floor, int64_t v,
                      int weighted, int64_t max_iter, double tol, float* maps, uint8_t* npd);

/* Adds a DKI volume: the arguments of lar_fit_dki_maps (device pointers, FP64). Every DKI job
 * of a batch takes the same weighted, max_iter and tol. */
int lar_batch_add_dki(lar_batch batch, lar_log_design design, const float* signals, const double* s0,
                      const double* floor, const uint8_t* is_b0, int64_t v, int weighted, int64_t max_iter, double tol,
                      float* maps, uint8_t* npd, uint8_t* broke, double* params);

/* Adds a multi-tissue volume: the arguments of lar_fit_multi_tissue (signals and outputs on the
 * device, weights (m,) on the host). The solvers must be ridge NNLS (L2NNLS) solvers with normal
 * equations, the low-resolution kernel of at most 48 directions and the high-resolution one of
 * 65 to 320; every mFOD job of a batch takes the same max_outer, fraction_tol and final_tol_x. */
int lar_batch_add_mfod(lar_batch batch, const double* signals, int64_t v, const double* weights, lar_deconv_kernel lr,
                       lar_fod_solver lr_solver, lar_deconv_kernel hr, lar_fod_solver hr_solver, int64_t max_outer,
                       double fraction_tol, double final_tol_x, double* fods, double* fractions, int32_t* rounds,
                       uint8_t* status);

/* Uploads the job tables and allocates the batch's scratch; no job can be added afterwards.
 * The jobs' designs, kernels, solvers, inputs and outputs must outlive the batch. */
int lar_batch_finalize(lar_batch batch);

/* Enqueues the stages of the families in `families` (LAR_BATCH_* bits) on `stream`. A
 * family's runs must not overlap one another on the GPU; different families may run on
 * different streams at once. Allocates nothing and does not wait on the host. */
int lar_batch_run(lar_batch batch, int families, void* stream);

/* ---- A fit that allocates no device memory ------------------------------------------- */

/* No counterpart in the reference: an entry point for callers that cannot allocate device
 * memory (an application that owns all device memory through its own allocator or budget, a
 * plugin host that hands out only its own buffers, code where an allocation is not allowed).
 * It fits each row of log_s (v, n) (device) like lar_fit_log_signal at FP64, with the design
 * x (n, p) and constraints g (m, p) given as host arrays and prepared on the host, and writes
 * params (v, p) and broke (v,) (device). Everything else it needs on the device -- the
 * prepared design, the violator list and the constrained re-fit's workspace -- lives in one
 * static device array of 32 MiB that every GPU loading this library holds until exit; the
 * call returns LAR_ERR_INVALID, with the largest voxel count that fits, when the design and v
 * need more. It calls no cudaMalloc or cudaFree. Its first call on a device looks up the
 * array's address there (cudaGetSymbolAddress): make that first call before any stream
 * capture. Calls share the array: calls whose work overlaps on the GPU race and must be
 * serialised by the caller. The call waits for its stream once, after copying the design. */
int lar_fit_log_signal_noalloc(const double* x, int64_t n, int64_t p, const double* g, int64_t m,
                               const double* log_s, int64_t v, int weighted, int64_t max_iter,
                               double tol, double* params, uint8_t* broke, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LARMOR_B200_H */
