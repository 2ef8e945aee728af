/*
 * mgkmc B200 C-ABI: the drop-in boundary for mgkmc's mechanical-equilibrium
 * hot path.  Plain C types only (pointers, sizes, scalars); every device
 * pointer is a CUDA device address owned by the caller (for example a
 * torch.Tensor's data_ptr()), every function returns an mgk_status and takes
 * the CUDA stream the work is ordered on.  No call blocks indefinitely or
 * traps; device-side loops are bounded by iteration caps.
 *
 * Array layouts are the reference's (C order, float64 unless noted):
 *   small strain 2D   E, nu (nx,ny);  eps, sig, eps_plastic (nx,ny,2,2)
 *   small strain 3D   E, nu (nx,ny,nz); eps, sig, eps_plastic (nx,ny,nz,3,3)
 *   KMC 2D            Q, Q0 (nx,ny,M); catalog (nx,ny,M,2,2); soft_prop (nx,ny,2)
 *   KMC 3D            Q, Q0 (nx,ny,nz,M); catalog (nx,ny,nz,M,3,3); soft_prop (nx,ny,nz,4)
 *
 * Reference interfaces each entry point replaces are cited as file:line within
 * the mgkmc project.
 */
#ifndef MGKMC_B200_H
#define MGKMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MGK_API __attribute__((visibility("default")))
#else
#define MGK_API
#endif

typedef struct CUstream_st* mgk_stream_t; /* == cudaStream_t */

typedef enum {
  MGK_OK = 0,
  MGK_NOT_CONVERGED = 1, /* iteration cap reached (the reference returns silently) */
  MGK_NONFINITE = 2,     /* NaN/Inf in a field or a norm */
  MGK_BAD_ARG = 3,
  MGK_OOM = 4,
  MGK_TIMEOUT = 5,
  MGK_CUDA_ERROR = 6
} mgk_status;

enum { MGK_PLANE_STRAIN = 0, MGK_PLANE_STRESS = 1 };
/* precision forms: FP64 throughout (the reference's arithmetic), or mixed:
 * FP32 storage/FFT/Green operator until the update norm is below
 * max(tol, 2e-6), then FP64 iterations to tol; norms are FP64 in both */
enum { MGK_FP64 = 0, MGK_MIXED = 1 };

/* ------------------------------------------------------------- library --- */
MGK_API int mgk_version(void);
MGK_API const char* mgk_status_string(int status);
/* Text of the last error raised on the calling host thread. */
MGK_API const char* mgk_last_error(void);
/* 1 if n = 2^a 3^b with 1 <= n <= 4096 (grid sides the FFT supports; the
 * 2D solvers also need nx even, the 3D solver nx*ny even). */
MGK_API int mgk_fft_supported(int n);

/* ------------------------------------------- 2D small-strain LS solver --- */
/* Replaces mgkmc/linear_elastic_simulator.py:12-88 spectral_solver_2d (and the
 * Green operator build of mgkmc/elasticity.py:20-53, applied on the fly). */
typedef struct mgk_ls2d_plan* mgk_ls2d_t;

typedef struct {
  int iterations;       /* LS iterations performed */
  int status;           /* MGK_OK or MGK_NOT_CONVERGED */
  double final_diff;    /* ||eps_new - eps|| / (||eps|| + 1e-20) of the last iteration */
  double eps_mean[4];   /* eps.mean(axis=(0,1)) as (xx, xy, yx, yy) */
  double sig_mean[4];   /* sig_out.mean(axis=(0,1)) */
} mgk_ls_info;

/* A plan holds nrep independent replicas ("slots"); mgk_ls2d_create makes a
 * plan of one.  The voxel size only enters the wave vectors, where it
 * cancels, so it is not an argument. */
MGK_API int mgk_ls2d_create(int nx, int ny, int plane_mode, int precision, mgk_ls2d_t* out);
/* Batched plan: replica r has grid nx[r] x ny[r] (sizes may differ). */
MGK_API int mgk_ls2d_create_batch(int nrep, const int* nx, const int* ny, int plane_mode, int precision,
                                  mgk_ls2d_t* out);
MGK_API int mgk_ls2d_destroy(mgk_ls2d_t plan);
/* Moduli fields E, nu (nx,ny) and the eigenstrain eps_plastic (nx,ny,2,2) or
 * NULL (= zero).  Computes mu, lambda per voxel and the reference medium
 * C0 = (mean E, mean nu) on the device (linear_elastic_simulator.py:22-23). */
MGK_API int mgk_ls2d_set_material(mgk_ls2d_t plan, const double* E, const double* nu,
                          const double* eps_plastic, mgk_stream_t stream);
MGK_API int mgk_ls2d_set_material_rep(mgk_ls2d_t plan, int rep, const double* E, const double* nu,
                                      const double* eps_plastic, mgk_stream_t stream);
/* Lame fields lam, mu (nx,ny) given directly, as spectral_solver_secant_2d
 * takes them (mgkmc/linear_elastic_simulator.py:614-619), with the reference
 * medium C0 = (mean lam, mean mu) (:679-681). */
MGK_API int mgk_ls2d_set_lame_rep(mgk_ls2d_t plan, int rep, const double* lam, const double* mu,
                                  const double* eps_plastic, mgk_stream_t stream);
/* Constitutive law of every replica: d = 0 linear elastic; otherwise the
 * secant degradation law of spectral_solver_secant_2d
 * (linear_elastic_simulator.py:614-765; elasticity.py:112-150, :189-260):
 * sigma = lam tr(e) I + 2 mu (1 - d (1 - exp(-k eq(e)))) e, e = eps - eps_p,
 * eq the plane-strain von Mises equivalent strain.  0 <= d <= 1, k >= 0;
 * FP64 plans only.  Takes effect at the next solve. */
MGK_API int mgk_ls2d_set_secant(mgk_ls2d_t plan, double d, double k);
/* The Rose secant-modulus law of spectral_solver_rose_2d
 * (linear_elastic_simulator.py:852-950; elasticity.py:868-944) for every
 * replica: G = max(mu exp(-eta eq), floor_fraction mu), bulk modulus kept,
 * sigma_yx copied from sigma_xy; plane_stress != 0 solves eps_zz per voxel by
 * the reference's five fixed-point steps.  Reference medium (mean lam,
 * (mean mu + floor_fraction mean mu) / 2): call before mgk_ls2d_set_lame_rep.
 * Macro strain, eigenstrain and warm start must be symmetric; FP64 plans. */
MGK_API int mgk_ls2d_set_rose(mgk_ls2d_t plan, double eta, double floor_fraction, int plane_stress);
/* The Landau small-strain law of spectral_solver_landau_2d
 * (linear_elastic_simulator.py:952-1228; elasticity.py:487-639) for every
 * replica: v = (v1, v2, v3, g1, g2, g3, g4); capping 0 none, 1 piecewise,
 * 2 smooth (tanh of power smooth_power) at the equivalent strain e_cap with
 * tangent 2 tangent_ratio mu.  plane_stress = 0: e33 = 0; != 0: e33 per voxel
 * from Newton steps on sigma33 = 0 (elasticity.py:571-616) until the step is
 * below 1e-9, the stress evaluated at the stepped e33 (the reference evaluates
 * before the last step and carries a warm start between calls; both fixed
 * points solve sigma33 = 0).  Medium (mean lam, mean mu), lam the 3D lambda:
 * give the material with mgk_ls2d_set_lame_rep.  Symmetric strains; FP64
 * plans only.  A solve runs the basic scheme; mgk_ls2d_set_anderson adds the
 * reference's Anderson mixing of the iterates inside the device loop. */
MGK_API int mgk_ls2d_set_landau(mgk_ls2d_t plan, const double* v, int capping, double e_cap, double tangent_ratio,
                                double smooth_power, int plane_stress);
/* Where the output pass of later solves writes replica rep's out-of-plane
 * strain e33 under the plane-stress Landau law (device, N doubles; NULL: not
 * written), the field the reference returns in its e33_state
 * (elasticity.py:614-615). */
MGK_API int mgk_ls2d_set_e33_out(mgk_ls2d_t plan, int rep, double* e33);
/* Type-II Anderson mixing of depth m (0 <= m <= 8; 0 turns it off) inside
 * the device loop of every later solve of this FP64 plan, as
 * spectral_solver_landau_2d mixes its iterates
 * (linear_elastic_simulator.py:1185-1209): after each iteration that neither
 * converged nor went non-finite, x = g - dG gamma with gamma the
 * least-squares fit of the last residual by the last m residual differences
 * (strain inner products over the four tensor entries; eigenvalues of the
 * Gram matrix below 1e-14 of the largest are dropped); a mix with
 * non-finite coefficients takes the plain step and restarts the history
 * from the last pair.  When the iteration cap ends the loop the outputs are
 * those of the last mixed iterate; when it converges, of the image g.  A
 * solve with m > 0 selects one replica and needs a nonlinear law
 * (mgk_ls2d_set_secant, _set_rose or _set_landau).  Allocates a ring of
 * (3 + 2m) strain fields (3 N doubles each) at the first call that needs
 * it. */
MGK_API int mgk_ls2d_set_anderson(mgk_ls2d_t plan, int m);
/* Type-II Anderson mixing (linear_elastic_simulator.py:1185-1209) of
 * fixed-point iterates x -> g = G(x), fields of n doubles, history depth
 * 1 <= m <= 8.  hist: (2m + 2) n doubles (dF columns, dG columns, f_prev,
 * g_prev).  mgk_aa_update forms f = g - x; with have_prev, column `slot`
 * becomes dF = f - f_prev, dG = g - g_prev; f, g become the previous pair;
 * dots (16 doubles, device) receive <dF_j, dF_slot> at j and <dF_j, f> at
 * 8 + j for j < ncols.  The caller solves the ncols x ncols least-squares
 * system; mgk_aa_mix writes x = g - sum_j gamma_j dG_j (gamma on the host).
 * work: mgk_aa_work_bytes bytes of device memory. */
MGK_API int64_t mgk_aa_work_bytes(int64_t n);
MGK_API int mgk_aa_update(int64_t n, const double* x, const double* g, double* hist, int m, int slot, int have_prev,
                          int ncols, double* dots, void* work, mgk_stream_t stream);
MGK_API int mgk_aa_mix(int64_t n, const double* g, const double* hist, int m, int ncols, const double* gamma,
                       double* x, mgk_stream_t stream);
/* Update only the eigenstrain field (KMC flips). */
MGK_API int mgk_ls2d_set_eigenstrain(mgk_ls2d_t plan, const double* eps_plastic, mgk_stream_t stream);
MGK_API int mgk_ls2d_set_eigenstrain_rep(mgk_ls2d_t plan, int rep, const double* eps_plastic,
                                         mgk_stream_t stream);
/* One LS solve.  eps_bar: host (2,2).  eps_init: device (nx,ny,2,2) warm start
 * or NULL (uniform eps_bar start, :32-41).  eps_out, sig_out: device
 * (nx,ny,2,2).  info: host, may be NULL; when given the call synchronises the
 * stream to fill it.  Convergence is tested on the device after every
 * iteration; the loop runs as one CUDA graph with a device-driven while node. */
MGK_API int mgk_ls2d_solve(mgk_ls2d_t plan, const double* eps_bar, const double* eps_init,
                   double* eps_out, double* sig_out, int max_iter, double tol,
                   mgk_ls_info* info, mgk_stream_t stream);
/* Batched solve of nsel replicas sel[0..nsel) (sel NULL = 0..nsel-1), one
 * launch per stage for all of them, each replica converging on its own.
 * eps_bar: host nsel x 4.  eps_init, eps_out, sig_out: host arrays of nsel
 * device pointers (entries may be NULL; eps_init itself may be NULL).
 * infos: host nsel entries or NULL (NULL = no synchronisation). */
MGK_API int mgk_ls2d_solve_batch(mgk_ls2d_t plan, int nsel, const int* sel, const double* eps_bar,
                                 const double* const* eps_init, double* const* eps_out,
                                 double* const* sig_out, int max_iter, double tol, mgk_ls_info* infos,
                                 mgk_stream_t stream);

/* Autotuner: times one iteration of every kernel family that can serve the
 * plan (warp-line kernels for sides up to 256 / 512 / 1024 with their column
 * tiles, and the CTA-wide passes with theirs) on the selection, `reps` times
 * each, and keeps the fastest (FP64 plus FP32 kernels for mixed plans).
 * *chosen: 0 CTA-wide, or 256/512/1024; *best_ms: its iteration time.  Leaves
 * the replicas' iterates unspecified (call before solving).  No counterpart in
 * the reference. */
MGK_API int mgk_ls2d_autotune(mgk_ls2d_t plan, int nsel, const int* sel, const double* eps_bar, int reps,
                              int* chosen, float* best_ms, mgk_stream_t stream);

/* Sets the kernel family directly (0 CTA-wide, 256/512/1024 warp-line; at
 * least the plan's largest side), e.g. one the autotuner chose for an equal
 * plan.  Synchronises the device.  No counterpart in the reference. */
MGK_API int mgk_ls2d_set_family(mgk_ls2d_t plan, int family);

/* Results of the last solve of replicas sel[0..nsel) (iterations, status,
 * final diff, mean strain and stress) after a solve_batch call that passed
 * infos = NULL: synchronises `stream` once.  Lets a scheduler launch the
 * solves of several plans on their own streams before waiting on any.  No
 * counterpart in the reference (its solves are synchronous). */
MGK_API int mgk_ls2d_collect(mgk_ls2d_t plan, int nsel, const int* sel, mgk_ls_info* infos, mgk_stream_t stream);

/* Timing hook: runs `reps` LS iterations (tolerance 0) and returns the mean
 * duration of the row kernel (C2R+update+tau+R2C along y) and of the column
 * kernel (FFT+Gamma+IFFT along x), timed with CUDA events on `stream`.
 * Leaves the plan's iterate in an unspecified state. */
MGK_API int mgk_ls2d_profile(mgk_ls2d_t plan, const double* eps_bar, int reps, float* row_ms, float* col_ms,
                             mgk_stream_t stream);
/* Same over a batch selection; fp32 = 1 times the FP32 kernels of a mixed plan. */
MGK_API int mgk_ls2d_profile_batch(mgk_ls2d_t plan, int nsel, const int* sel, const double* eps_bar, int fp32,
                                   int reps, float* row_ms, float* col_ms, mgk_stream_t stream);

/* Allocation-free 2D LS solve.  No counterpart in the reference: an addition
 * for callers that cannot allocate device memory -- code inside a host
 * application or framework whose caching allocator already holds the GPU's
 * memory, serving processes with a fixed memory budget that must not allocate
 * after start-up, and code that must avoid the device-wide synchronisation
 * cudaFree implies.  Same arguments and results as
 * mgk_ls2d_create + mgk_ls2d_set_material + mgk_ls2d_solve (FP64), but every
 * buffer beyond the caller's inputs and outputs lives in one file-scope
 * device array sized for grids up to MGK_NOALLOC_MAX_SIDE per side (about
 * 7 MB, held by every GPU that loads the library until the process exits).
 * Larger grids are rejected with MGK_BAD_ARG.  The call calls no cudaMalloc
 * or cudaFree and synchronises `stream` before returning.
 *   - The first call on a device resolves the array's device address
 *     (cudaGetSymbolAddress, which may load the module); make that first
 *     call before any stream capture.
 *   - All calls on a device share the one array and each call resets what
 *     must start at zero; calls that overlap on the GPU (other streams, other
 *     host threads) race on it and must be serialised by the caller.
 *   - The resolved address belongs to the device's primary context: after a
 *     cudaDeviceReset (or any destruction of that context) the entry point
 *     must not be called again in the same process. */
#define MGK_NOALLOC_MAX_SIDE 256
MGK_API int mgk_ls2d_solve_noalloc(int nx, int ny, int plane_mode, const double* E, const double* nu,
                                   const double* eps_plastic, const double* eps_bar, const double* eps_init,
                                   double* eps_out, double* sig_out, int max_iter, double tol,
                                   mgk_ls_info* info, mgk_stream_t stream);

/* ------------------------------------------- 3D small-strain LS solver --- */
/* Replaces mgkmc/linear_elastic_simulator.py:274-376 spectral_solver_3d (and
 * mgkmc/stz/update_fft.py:4-22 update_stress_fft_full, which wraps it), with
 * the Green operator of mgkmc/elasticity.py:70-105 applied on the fly.  FP64.
 * Batched plans as for 2D; eps_bar is 9 doubles per replica (3x3, C order);
 * fields are (nx,ny,nz,3,3). */
typedef struct mgk_ls3d_plan* mgk_ls3d_t;
typedef struct {
  int iterations;
  int status;
  double final_diff;
  double eps_mean[9];
  double sig_mean[9];
} mgk_ls_info3;
MGK_API int mgk_ls3d_create(int nx, int ny, int nz, mgk_ls3d_t* out);
MGK_API int mgk_ls3d_create_batch(int nrep, const int* nx, const int* ny, const int* nz, mgk_ls3d_t* out);
MGK_API int mgk_ls3d_destroy(mgk_ls3d_t plan);
/* Precision form (plans whose sides are all 64, 96 or 128): MGK_MIXED runs
 * FP32 iterations (fields, spectra, Gamma0) until the update norm is below
 * max(tol, 2e-6), then FP64 iterations from that field to tol; norms and
 * partial sums stay FP64.  Call before set_material.  No counterpart in the
 * reference (FP64 only). */
MGK_API int mgk_ls3d_set_precision(mgk_ls3d_t plan, int precision);
MGK_API int mgk_ls3d_set_material_rep(mgk_ls3d_t plan, int rep, const double* E, const double* nu,
                                      const double* eps_plastic, mgk_stream_t stream);
MGK_API int mgk_ls3d_set_eigenstrain_rep(mgk_ls3d_t plan, int rep, const double* eps_plastic,
                                         mgk_stream_t stream);
/* Lame fields lam, mu (nx,ny,nz) given directly, as spectral_solver_secant_3d
 * takes them (mgkmc/linear_elastic_simulator.py:768-771), with the reference
 * medium C0 = (mean lam, mean mu) (:783-784). */
MGK_API int mgk_ls3d_set_lame_rep(mgk_ls3d_t plan, int rep, const double* lam, const double* mu,
                                  const double* eps_plastic, mgk_stream_t stream);
/* Constitutive law of every replica: d = 0 linear elastic; otherwise the
 * secant degradation law of spectral_solver_secant_3d
 * (linear_elastic_simulator.py:768-850; elasticity.py:261-295, :665-728):
 * sigma = lam tr(e) I + 2 mu (1 - d (1 - exp(-k eq(e)))) e, e = eps - eps_p,
 * eq the von Mises equivalent strain.  0 <= d <= 1, k >= 0; FP64 plans
 * only.  Takes effect at the next solve. */
MGK_API int mgk_ls3d_set_secant(mgk_ls3d_t plan, double d, double k);
/* The Landau small-strain law of spectral_solver_landau_3d
 * (linear_elastic_simulator.py:1231-1350; elasticity.py:811-857 with the
 * capping of :297-334) for every replica: v = (v1, v2, v3, g1, g2, g3, g4);
 * capping 0 none, 1 piecewise, 2 smooth (tanh of power smooth_power) at the
 * equivalent strain e_cap with tangent 2 tangent_ratio mu.  Medium (mean lam,
 * mean mu): give the material with mgk_ls3d_set_lame_rep.  The basic scheme
 * (no mixing, as the reference's 3D solver); symmetric strains; FP64 plans. */
MGK_API int mgk_ls3d_set_landau(mgk_ls3d_t plan, const double* v, int capping, double e_cap, double tangent_ratio,
                                double smooth_power);
MGK_API int mgk_ls3d_solve_batch(mgk_ls3d_t plan, int nsel, const int* sel, const double* eps_bar,
                                 const double* const* eps_init, double* const* eps_out,
                                 double* const* sig_out, int max_iter, double tol, mgk_ls_info3* infos,
                                 mgk_stream_t stream);

/* After a KMC flip changed voxel (x, y) = d_xy[0..1] (device int64, e.g.
 * from mgk_kmc2d_event) of the caller's eigenstrain field, copy that voxel
 * into replica `rep`'s planes instead of re-reading the whole field.  The
 * replica's material must have been set with an eigenstrain field. */
MGK_API int mgk_ls2d_sync_voxel(mgk_ls2d_t plan, int rep, const double* eps_plastic, const int64_t* d_xy,
                                mgk_stream_t stream);

/* ------------------------------------ 3D finite strain (de Geus Newton) --- */
/* Replaces mgkmc/finite_strain_simulator.py:2967-3168
 * finite_strain_solver_step_3d with solver="newton_cg" (the Ghat4 projection
 * of :1121-1188 and the SVK / F_p constitutive law of :1647-1885 applied
 * matrix-free; CG Krylov solver with FP64 inner products).  model: 0 SVK,
 * 1 Neo-Hookean (the reference's 2D plane-strain law restated in 3D).
 * Fields are tensor-first (3,3,nx,ny,nz) like the reference API. */
typedef struct mgk_fs3d_plan* mgk_fs3d_t;
typedef struct {
  int newton_iterations;   /* summed over the macro iterations */
  int krylov_iterations;   /* CG iterations (one matvec each) */
  int macro_iterations;
  int status;
  double max_stress_error; /* Pa, last macro iteration */
  double sig_mean[9];      /* mean Cauchy stress of the returned field */
} mgk_fs_info;
MGK_API int mgk_fs3d_create(int nx, int ny, int nz, int model, mgk_fs3d_t* out);
MGK_API int mgk_fs3d_destroy(mgk_fs3d_t plan);
/* lam, mu: device (nx,ny,nz) Lame fields (C4[0,0,1,1], C4[0,1,0,1] of the
 * reference's C4); Fp: device (3,3,nx,ny,nz) plastic deformation gradient or
 * NULL (no F_p: the reference's tangent branch without F_p). */
/* Precision form of the Krylov matvecs: MGK_FP64 (default), or MGK_MIXED:
 * the tangent product K:dF, the FFTs and the projection of the CG matvecs in
 * FP32, while the Newton right-hand side (-G:P, -G:K:DbarF), the CG vectors x
 * and r, every inner product and norm, the line search and the macro loop
 * stay FP64.  No counterpart in the reference (FP64 only). */
MGK_API int mgk_fs3d_set_precision(mgk_fs3d_t plan, int precision);
MGK_API int mgk_fs3d_set_material(mgk_fs3d_t plan, const double* lam, const double* mu, const double* Fp,
                                  mgk_stream_t stream);
/* Current deformation gradient (device, tensor-first); the plan keeps it. */
MGK_API int mgk_fs3d_set_F(mgk_fs3d_t plan, const double* F, mgk_stream_t stream);
/* One load step from the plan's F: F_bar_in (host 3x3), the driving
 * component, P_target (host 3x3, Pa, may be NULL) and P_mask (host 3x3 int,
 * may be NULL), E_avg/nu_avg for the compliance correction, the tolerances
 * and caps of the reference.  F_bar_out (host 3x3) receives the macro
 * deformation.  Returns MGK_NOT_CONVERGED where the reference raises
 * ValueError (line search, Newton or macro loop). */
MGK_API int mgk_fs3d_step(mgk_fs3d_t plan, const double* F_bar_in, int driving_i, int driving_j,
                          const double* P_target, const int* P_mask, double E_avg, double nu_avg, double tol_NW,
                          double tol_CG, int max_NW, double tol_macro, int max_iter_macro, double* F_bar_out,
                          mgk_fs_info* info, mgk_stream_t stream);
/* Copy out F and P (device, tensor-first) and compute the Cauchy stress
 * (cauchy_from_P_3d :1892-1904); any pointer may be NULL. */
MGK_API int mgk_fs3d_get(mgk_fs3d_t plan, double* F_out, double* P_out, double* sig_out, mgk_stream_t stream);
/* 2D plane-strain finite strain (mgkmc/finite_strain_simulator.py:2356-2572
 * finite_strain_solver_step_2d, solver="newton_cg"; laws :591-1087 with
 * plane_mode="plane_strain") on a plan created as (nx, 1, ny): the plane's
 * axes are the plan's x and z, the out-of-plane axis is y (one voxel, no
 * wave vector) with F_yy = 1, tensor index 1 of the 2D fields is index 2 of
 * the plan's.  The 3D SVK and Neo-Hookean laws at F_yy = 1 are the
 * reference's plane-strain laws, and the projection keeps every out-of-plane
 * component of dF at zero, so the plan solves the 2D problem; on != 0 makes
 * the Newton test use the 2D field's norm (||F|| without the N unit F_yy
 * entries, :2521).  No counterpart in the reference as an entry point. */
MGK_API int mgk_fs3d_set_plane_strain(mgk_fs3d_t plan, int on);
/* 2D plane-stress finite strain (finite_strain_simulator.py:631-684
 * Neo-Hookean, :1038-1049 SVK, cauchy_from_P :1094-1115 with F33) on an
 * (nx, 1, ny) plan: the plane-strain embedding and Newton norm of
 * mgk_fs3d_set_plane_strain, the material's lam being the plane-stress
 * lambda E nu / (1 - nu^2) of build_C4_2d (:233-259).  SVK: the in-plane
 * stress and tangent are the reference's, F33 = sqrt(max(1e-12,
 * 1 - (lam / mu) tr E)), E the in-plane Green-Lagrange strain of F Fp^-1.
 * Neo-Hookean: per voxel x = F33^2 from the reference's Newton solve of
 * mu x + lam_3d/2 ln x = mu - lam_3d ln Je, S = mu I - mu x C^-1 and the
 * condensed tangent (lam*, mu x).  The Cauchy stress divides by
 * J = det(F) F33. */
MGK_API int mgk_fs3d_set_plane_stress(mgk_fs3d_t plan, int on);
/* Autotuner: times one Krylov iteration of each kernel family that can serve
 * the plan (warp-line passes, sides 64/96/128; CTA-wide passes) on the current
 * state and keeps the faster; *chosen 1 warp-line, 0 CTA-wide.  Call after a
 * step (the state must be valid); leaves the Krylov vectors unspecified.  No
 * counterpart in the reference. */
MGK_API int mgk_fs3d_autotune(mgk_fs3d_t plan, int reps, int* chosen, float* best_ms, mgk_stream_t stream);
/* Timing hook: mean duration (ms, CUDA events on `stream`) of the six kernels
 * of one Krylov iteration (z forward with K:p, y pass, x pass with G, inverse
 * y pass, z inverse with p.q, CG update), ms_out[6]; fp32 = 1 times the mixed
 * form's FP32 kernels.  Leaves the Krylov vectors in an unspecified state.
 * No counterpart in the reference. */
MGK_API int mgk_fs3d_profile(mgk_fs3d_t plan, int fp32, int reps, float* ms_out, mgk_stream_t stream);

/* ------------------------------------------------------ 2D STZ / KMC --- */
/* mgkmc/kmc_simulator_functions.py:100-160 compute_barrier_2d (in place on Q).
 * scheme: 0 isotropic, 1 directional.  tau: +inf for no decay. */
MGK_API int mgk_kmc2d_barrier(int nx, int ny, int M, double* Q, const double* Q0, const double* sig,
                      const double* catalog, double volume, const double* soft_prop,
                      const double* last_event_time, double current_time,
                      const double* prev_strain_dir, double softening_cap, int scheme, double tau,
                      mgk_stream_t stream);

/* mgkmc/kmc_simulator_functions.py:5-56 compute_rates_2d / _compute_rates_2d_jit.
 * temperature: device (nx,ny) field or NULL to use temperature_scalar.
 * Writes rates[count], indices[count] (int64) and the prefix array
 * prefix[count] of the sequential left-to-right FP64 running sum (prefix[count-1]
 * is the reference's total_rate, bit for bit).  count and total land in the
 * device scalars *d_count (int64) and *d_total.  rates/indices/prefix need
 * nx*ny*M entries.  work: device scratch of mgk_kmc_rates_work_bytes(). */
MGK_API int64_t mgk_kmc_rates_work_bytes(int64_t n_modes);
MGK_API int mgk_kmc2d_rates(int nx, int ny, int M, const double* Q, double volume,
                    const double* temperature, double temperature_scalar, double nu0,
                    int cascade_mode, double* rates, int64_t* indices, double* prefix,
                    int64_t* d_count, double* d_total, void* work, mgk_stream_t stream);

/* Sequential left-to-right running sum of n given rates into prefix[n]; the
 * total (prefix[n-1], 0 if n == 0) lands in *d_total and n in *d_count.  This
 * is the total_rate chain of kmc_simulator_functions.py:36-55, for callers
 * that hold a rates array of their own (select_event_2d(rates, total)). */
MGK_API int mgk_kmc_prefix(const double* rates, int64_t n, double* prefix, int64_t* d_count,
                           double* d_total, mgk_stream_t stream);

/* mgkmc/kmc_simulator_functions.py:58-67 select_event_2d with an explicit
 * uniform draw u in [0,1): r = u * total, result = first i with prefix[i] >= r
 * (count-1 if none, -1 if total <= 0).  Bit-exact with the reference given the
 * same rates and draw.  Result in *d_index (device int64). */
MGK_API int mgk_kmc_select(const double* prefix, const int64_t* d_count, const double* d_total, double u,
                   int64_t* d_index, mgk_stream_t stream);

/* Fast selection mode, the rate step of a KMC/AQS step in one pass:
 * mgk_kmc2d_barrier (Q written as there; volume is the barrier's), then each
 * mode's KMC-mode rate from its new barrier (same per-mode arithmetic as
 * mgk_kmc2d_rates, rate_volume * nu0 as its prefactor) and the FP64 sum of
 * all rates into *d_total, summed per CTA in a fixed order (it can differ
 * from the reference's sequential total in the last bits).  No rate array is
 * written: a caller computes rates and running sums only when an event is
 * drawn.  No counterpart in the reference (its compute_barrier_2d and
 * compute_rates_2d are two passes).  work: mgk_kmc_scan_work_bytes(nx*ny*M). */
MGK_API int mgk_kmc2d_barrier_total(int nx, int ny, int M, double* Q, const double* Q0, const double* sig,
                                    const double* catalog, double volume, const double* soft_prop,
                                    const double* last_event_time, double current_time,
                                    const double* prev_strain_dir, double softening_cap, int scheme,
                                    double tau, double rate_volume, const double* temperature,
                                    double temperature_scalar, double nu0, double* d_total, void* work,
                                    mgk_stream_t stream);

/* KMC-mode rates only (every mode an event; no running sum), for the fast
 * selection mode below.  Same per-mode arithmetic as mgk_kmc2d_rates. */
MGK_API int mgk_kmc2d_rates_only(int nx, int ny, int M, const double* Q, double volume,
                                 const double* temperature, double temperature_scalar, double nu0,
                                 double* rates, mgk_stream_t stream);

/* Fast selection mode: parallel inclusive FP64 scan of n rates into prefix
 * (total in *d_total, n in *d_count).  Its running sums differ from the
 * reference's sequential chain by rounding, so the selected index can differ
 * from the reference's only when u*total falls within that rounding of a
 * running sum.  work: mgk_kmc_scan_work_bytes(n) bytes. */
MGK_API int64_t mgk_kmc_scan_work_bytes(int64_t n);
MGK_API int mgk_kmc_prefix_fast(const double* rates, int64_t n, double* prefix, int64_t* d_count,
                                double* d_total, void* work, mgk_stream_t stream);

/* One KMC event on the device: mgkmc/kmc_simulator.py:899-900 (index ->
 * x, y, m via indices[*d_sel], decode_index_2d), :1025 apply_flip_soa_2d,
 * :1030 prev_strain_dir[x,y] = catalog[x,y,m], and :1035-1042 the redraw of
 * the voxel's catalog (new_catalog, M x 2 x 2) and barriers (new_q0, M),
 * both drawn by the host (NULL: keep).  indices NULL means identity (KMC
 * mode).  Writes (x, y, m) to d_xym (device int64[3], may be NULL); a
 * negative *d_sel (no event) leaves everything unchanged. */
MGK_API int mgk_kmc2d_event(int nx, int ny, int M, const int64_t* d_sel, const int64_t* indices,
                            double* eps_plastic, double* soft_prop, double* last_event_time, double* catalog,
                            double* Q0, double* prev_strain_dir, const double* new_catalog, const double* new_q0,
                            double current_time, double jp, double jt, double g_max, double jn_frac,
                            int64_t* d_xym, mgk_stream_t stream);

/* Fast-patching stress patches: replaces KmcSimulation2D._precompute_patch_kernels
 * (mgkmc/kmc_simulator.py:229-261) after its two LS solves.  r0, r1 (nx,ny,2,2)
 * are the stress responses to the unit eigenstrains [[1,0],[0,-1]] and
 * [[0,1],[1,0]] at voxel (nx/2, ny/2) under zero macro strain.  Writes
 * kernels (2, 2R+1, 2R+1, 2, 2): each response in the window centred on that
 * voxel (periodic), and missing_mean (2, 2, 2): mean(r_b) - sum(window_b) /
 * (nx*ny).  0 <= R <= 4096. */
MGK_API int mgk_kmc2d_patch_setup(int nx, int ny, int R, const double* r0, const double* r1, double* kernels,
                                  double* missing_mean, mgk_stream_t stream);

/* One fast-patching stress update of sig (nx,ny,2,2) in place: replaces
 * mgkmc/kmc_simulator.py:1052-1069 (KMC event) and :764-774 (cascade flip).
 * The mode is the device selection d_sel (through `indices` when non-null,
 * as in mgk_kmc2d_event); gxx, gxy are its catalog entries (0,0) and (0,1)
 * when the call runs: enqueue it before mgk_kmc2d_event for the pre-flip
 * direction (KMC events), after it for the redrawn one (cascade flips).
 * sig += sig_unit * unit_scale when sig_unit is non-null, then
 * gxx*K0 + gxy*K1 added in the window around the mode's voxel, then
 * gxx*m0 + gxy*m1 added to every voxel.  A negative selection leaves the
 * patch out; a null d_sel applies only the sig_unit term (the macro-strain
 * increment of :1094-1096).  sig and sig_unit 16-byte aligned. */
MGK_API int mgk_kmc2d_patch(int nx, int ny, int M, double* sig, const double* sig_unit, double unit_scale,
                            const double* kernels, const double* missing_mean, int R, const double* catalog,
                            const int64_t* d_sel, const int64_t* indices, mgk_stream_t stream);

/* mgkmc/kmc_simulator_functions.py:183-218 apply_flip_soa_2d (in place). */
MGK_API int mgk_kmc2d_flip(int nx, int ny, int M, double* eps_plastic, double* soft_prop,
                   double* last_event_time, const double* catalog, int x, int y, int m,
                   double current_time, double jp, double jt, double g_max, double jn_frac,
                   mgk_stream_t stream);

/* ------------------------------------------------------ 3D STZ / KMC --- */
/* mgkmc/stz/barriers.py:4-100 compute_barrier (in place on Q; soft_prop has 4
 * slots per voxel, of which 0 and 1 are used). */
MGK_API int mgk_kmc3d_barrier(int nx, int ny, int nz, int M, double* Q, const double* Q0, const double* sig,
                              const double* catalog, double volume, const double* soft_prop,
                              const double* last_event_time, double current_time,
                              const double* prev_strain_dir, double softening_cap, int scheme, double tau,
                              mgk_stream_t stream);
/* mgkmc/stz/kmc.py:4-74 compute_rates / _compute_rates_jit (index encoding
 * ((x*ny + y)*nz + z)*M + m); outputs as mgk_kmc2d_rates. */
MGK_API int mgk_kmc3d_rates(int nx, int ny, int nz, int M, const double* Q, double volume,
                            const double* temperature, double temperature_scalar, double nu0, int cascade_mode,
                            double* rates, int64_t* indices, double* prefix, int64_t* d_count, double* d_total,
                            void* work, mgk_stream_t stream);
/* mgkmc/stz/cascade.py:43-111 apply_flip_soa (in place; 26-neighbour softening). */
MGK_API int mgk_kmc3d_flip(int nx, int ny, int nz, int M, double* eps_plastic, double* soft_prop,
                           double* last_event_time, const double* catalog, int x, int y, int z, int m,
                           double current_time, double jp, double jt, double g_max, double jn_frac,
                           mgk_stream_t stream);

/* One 3D KMC event on the device: mgkmc/aqs.py:889-892 (position *d_sel ->
 * mode index via indices (NULL: identity, KMC mode) -> x, y, z, m by
 * decode_index, stz/kmc.py:94-103), :996 apply_flip_soa, :997
 * prev_strain_dir[x,y,z] = catalog[x,y,z,m], and :1006-1013 the redraw of
 * the voxel's catalog (new_catalog, M x 3 x 3) and barriers (new_q0, M), both
 * drawn by the host (NULL: keep).  Writes (x, y, z, m) to d_xyzm (device
 * int64[4], may be NULL); a negative *d_sel leaves everything unchanged. */
MGK_API int mgk_kmc3d_event(int nx, int ny, int nz, int M, const int64_t* d_sel, const int64_t* indices,
                            double* eps_plastic, double* soft_prop, double* last_event_time, double* catalog,
                            double* Q0, double* prev_strain_dir, const double* new_catalog, const double* new_q0,
                            double current_time, double jp, double jt, double g_max, double jn_frac,
                            int64_t* d_xyzm, mgk_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MGKMC_B200_H */
