/*
 * rism3d_b200 -- B200-native 3D-RISM solver, C ABI.
 *
 * Drop-in for the solve path of rismical-dev/3D-RISM-CUDA (src-cuda/).  The
 * reference has no library API: its public surface is the C++ class
 * RISM3D with initialize / iterate / output (rism3d.h:25-27), driven by
 * main (main.cu:6-64), plus its file formats.  This header gives
 *   (1) rism3d_initialize / rism3d_iterate / rism3d_output: the same three
 *       steps with the same arguments, reading and writing the same files;
 *   (2) an array-level API (create / set_solvent / set_solute / solve /
 *       forces / grad / get_grid / solve_batch / destroy) so that callers
 *       can drive a solve from memory without files.
 * Plain C types only: pointers, sizes, POD structs.  Every call returns a
 * status code; no call exits the process (the reference calls exit(1) on
 * bad input, e.g. read_input.cu:31-32, solvent_read.cc:16-19).
 *
 * Units follow the reference: lengths in Angstrom, solute/solvent epsilon
 * in J/mol, charges in e, solvent densities in molecules/A^3, energies
 * reported in J/mol, PMV in L/mol, pressure in J/m^3.
 */
#ifndef RISM3D_B200_H
#define RISM3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define RISM3D_MAX_SITES 8

/* status codes */
enum {
  RISM3D_OK = 0,
  RISM3D_BAD_INPUT = 1,          /* malformed file / argument */
  RISM3D_UNSUPPORTED_SHAPE = 2,  /* grid not a multiple of 4, too many sites */
  RISM3D_CUDA_ERROR = 3,
  RISM3D_CUFFT_ERROR = 4,
  RISM3D_DIVERGED = 5,           /* non-finite residual (iterate.cu:54-57) */
  RISM3D_NOT_CONVERGED = 6,      /* maxstep reached (iterate.cu:76-79) */
  RISM3D_NO_DEVICE = 7,
  RISM3D_BAD_STATE = 8           /* call out of order */
};

enum { RISM3D_KH = 0, RISM3D_HNC = 1 };          /* read_input.cu:37-44 */
enum { RISM3D_FP64 = 0, RISM3D_MIXED = 1 };      /* arithmetic of the iteration */

/* grids returned by rism3d_get_grid, each natv * N doubles (site-major,
 * x fastest: ip = ix + nx*(iy + ny*iz)) unless noted */
enum {
  RISM3D_GRID_G = 0,    /* g_uv(r) (the .guv payload, output_guv.cu)       */
  RISM3D_GRID_H = 1,    /* h_uv(r) from the OZ step (output_huv.cu)        */
  RISM3D_GRID_C = 2,    /* c_uv(r) = h - t (output_cuv.cu)                  */
  RISM3D_GRID_T = 3,    /* t_uv(r) (the .tuv payload, write_tuv.cu)        */
  RISM3D_GRID_U = 4,    /* beta u_LJ per site (cal_LJ.cu)                   */
  RISM3D_GRID_E = 5,    /* beta sum q/r, N doubles (cal_Coulomb.cu)         */
  RISM3D_GRID_FR = 6,   /* beta long-range part, N doubles                  */
  RISM3D_GRID_QV = 7    /* sum_v rho_v q_v g_v, N doubles (cal_qv.cu)       */
};

typedef struct {
  int grid[3];            /* nx ny nz, each a multiple of 4 (fft3d.cu:71-94) */
  double box[3];          /* Angstrom */
  int closure;            /* RISM3D_KH / RISM3D_HNC */
  double convergence;     /* rms residual target (iterate.cu:58) */
  int maxstep;
  int an2_count;          /* Picard steps before AN2 (anderson.cu:43-49) */
  double an2_m;           /* AN2 mixing factor */
  double an2_mp;          /* AN2 bias on the newer slot */
  int precision;          /* RISM3D_FP64 or RISM3D_MIXED */
  double mixed_switch;    /* MIXED: plain FP32 -> FP32 refinement once rms <= this (0 = 100 x convergence) */
  int device;             /* CUDA ordinal (main.cu:57) */
  int verbose;            /* 1: print " Step = n Reside = r" like iterate.cu:63 */
  void *stream;           /* caller-owned cudaStream_t for all work; NULL: the
                             context creates its own (the reference uses the
                             legacy default stream) */
  long long batch_chunk_points; /* rism3d_solve_batch: solutes of one cell run
                             in sub-batches of about this many grid points in
                             all, which converge, finish and overlap on their
                             own.  0 = autotuned: the first batch with a given
                             set of cells is solved once per candidate size
                             (2^18 .. 2^22 points) and the fastest is kept for
                             later batches with that set */
} rism3d_params;

typedef struct {
  int natv;
  int natom;
  double sfe_sc;          /* SFE_SC, J/mol (KH functional for KH, HNC for HNC) */
  double sfe_sc_hnc;      /* SFE_SC_HNC (reported for KH only) */
  double sfe_gf;          /* SFE_GF */
  double sfec_sc[RISM3D_MAX_SITES];
  double sfec_sc_hnc[RISM3D_MAX_SITES];
  double sfec_gf[RISM3D_MAX_SITES];
  double pmv;             /* L/mol */
  double pressure;        /* J/m^3 */
  double correction;      /* J/mol, -P * PMV */
  double se, se_lj, se_es;/* solute-solvent energy, J/mol */
  double rms;             /* final residual */
  int iterations;         /* all iterations (all stages, both precisions) */
  int iterations_fp32;    /* of which in FP32 (MIXED) */
  int status;             /* RISM3D_OK / DIVERGED / NOT_CONVERGED */
  double ms_setup;        /* potential grids + chi table (device time) */
  double ms_iterate;
  double ms_observe;
  double sfe_rmdft;       /* SFE_RMDFT, J/mol (output_xmu.cu:25-28); 0 unless
                             rism3d_set_rmdft tables are set */
} rism3d_result;

typedef struct rism3d_ctx rism3d_ctx;

/* ---- array-level API ---------------------------------------------------
 * Replaces: RISM3D::initialize's file readers + cal_potential
 * (initialize.cu:4-13), RISM3D::iterate (iterate.cu:6-90) and the
 * observables of RISM3D::output (output.cu:6-62). */

/* Allocate a context on params->device.  Replaces the implicit RISM3D
 * constructor + Cell::setup (cell.cc:8-22) + FFT3D::initialize
 * (fft3d.cu:4-19).  Besides its grids, the context owns a stream-ordered
 * memory pool for per-solve scratch (potential phase rows, partial sums,
 * the RMDFT buffer, the adjoint's history).  The pool keeps what it has
 * allocated until rism3d_destroy; the device's default pool is not
 * touched. */
int rism3d_create(const rism3d_params *params, rism3d_ctx **ctx);

/* Solvent sites after merging equivalent sites (solvent_read.cc:68-80):
 * rho in molecules/A^3, chi table xvv[natv][natv][ntab] at
 * k_i = (i+1) pi / (dr ntab), row b fastest (solvent_read.cc:51-58).
 * Replaces Solvent::read + Solvent::spline (solvent_spline.cu:8-91). */
int rism3d_set_solvent(rism3d_ctx *ctx, int natv, const double *rho,
                       const double *q, const double *sig, const double *eps,
                       double temperature, double xt, int ntab, double dr,
                       const double *xvv);

/* Solute atoms, coordinates already placed in the cell (the reference
 * centres them in read_input.cu:80-82; rism3d_initialize does the same).
 * Replaces Solute::init/setup_cuda (solute.cu:5-56) and computes the
 * potential grids of cal_potential (cal_potential.cu:3-14). */
int rism3d_set_solute(rism3d_ctx *ctx, int natom, const double *sig,
                      const double *eps, const double *q, const double *xyz);

/* Optional restart guess t_uv[natv][N] (read_tuv.cu:6-34).  NULL clears. */
int rism3d_set_tuv(rism3d_ctx *ctx, const double *tuv);

/* Solve with `chargeup` charge-up stages (main.cu -c; iterate.cu:34-47)
 * and evaluate mu_ex (cal_exchem.cu), PMV (cal_pmv.cu), pressure
 * (cal_pressure.cu) and SE (cal_euv.cu). */
int rism3d_solve(rism3d_ctx *ctx, int chargeup, rism3d_result *result);

/* Per (site, atom) solute-solvent energies euv[2][natv][natom] (LJ then
 * ES, J/mol, already times dv; cal_euv.cu:7-33 + output_euv.cu). */
int rism3d_euv(rism3d_ctx *ctx, double *euv);

/* cal_grad forces (cal_grad.cu:8-48 + output_grad.cu): dulj[natom][3],
 * due[natom][3] in J/mol/A, already times dv. */
int rism3d_forces(rism3d_ctx *ctx, double *dulj, double *due);

/* Adjoint: d(SFE_SC)/d(parameter) in J/mol per unit, by back-propagating
 * rho_v g_v(r) through the potential-grid kernel with per-atom potentials
 * recomputed.  Any output pointer may be NULL.  dmu_dR is [natom][3]. */
int rism3d_grad(rism3d_ctx *ctx, double *dmu_dq, double *dmu_dsig,
                double *dmu_deps, double *dmu_dR);

/* The same gradients in a chosen arithmetic.  RISM3D_FP64 is rism3d_grad
 * (transposed-Jacobian solve to 1e-10 relative).  RISM3D_MIXED solves the
 * transposed system in FP32 (FP32 operator and storage, FP64 dot products,
 * mixing coefficients and sums) to 2e-6 relative and evaluates the LJ pair
 * factors of the back-projection in FP32; the Coulomb and long-range terms
 * and every accumulation stay FP64.  Works on FP64 and MIXED contexts (an
 * FP64 context makes its FP32 transform plan on the first call).  No
 * counterpart in the reference, which has only the cal_grad forces. */
int rism3d_grad_precision(rism3d_ctx *ctx, int precision, double *dmu_dq,
                          double *dmu_dsig, double *dmu_deps, double *dmu_dR);

/* ESP cube potential (cal_Coulomb.cu:41-96, the reference's -e input):
 * esp[N] in Hartree/e on the cell grid, x fastest, replaces the point-charge
 * Coulomb potential e that enters the closure (e = esp hartree / (kB T));
 * the long-range fr / fk stay the point-charge forms, as in the reference.
 * NULL removes it.  Applies to the current solute at once and to every
 * later one; rism3d_grad refuses while it is set.  Single-solute contexts. */
int rism3d_set_esp(rism3d_ctx *ctx, const double *esp);

/* RMDFT free-energy correction (the reference's -r option,
 * cal_rmdft.cu:5-115, tables of solvent_read.cc:88-140 and
 * solvent_spline2.cu:7-103).  cvk[natv][natv][ntab]: the solvent direct
 * correlation c(k) on the knots of the chi table (the .cvk file beside the
 * .xvk; same layout as xvv).  Site 0's hard-sphere table (the -r file):
 * ntab2 rows of k[i] (ascending), chs[i] (hard-sphere chi(k)) and w[i]
 * (weight function), its packing fraction pfhs and w(k = 0) w0.  Every
 * later solve reports SFE_RMDFT in rism3d_result.sfe_rmdft and the .xmu.
 * cvk NULL switches it off, and so does any failed call.  Call after
 * rism3d_set_solvent (which also switches it off); BAD_INPUT when the
 * hard-sphere table ends below the grid's largest |k| or its knots do not
 * increase.  Single-solute contexts. */
int rism3d_set_rmdft(rism3d_ctx *ctx, const double *cvk, int ntab2, const double *k,
                     const double *chs, const double *w, double pfhs, double w0);

/* Recompute the potential grids from the solute already on the device
 * (no host->device traffic); the next rism3d_solve starts from them. */
int rism3d_refresh_potentials(rism3d_ctx *ctx);

/* Kernels of this library launched by ctx so far (cuFFT's own kernels are
 * not counted). */
long long rism3d_kernel_launches(const rism3d_ctx *ctx);

/* Measurement hook: launch one kernel `reps` times back to back on the
 * context stream and report the mean device time per launch (CUDA events).
 * which: 0/1/2 = FP64 pass A / pass K / pass R, 10/11/12 = the FP32
 * versions (MIXED contexts), 13/15 = FP32 pass A / pass R of the
 * refinement form (MIXED, after a solve), 20 = real-space potential kernel.  The
 * iteration kernels run on the current state with an AN2 update armed, so
 * the stored solution is invalid afterwards (solve again to restore it). */
int rism3d_time_kernel(rism3d_ctx *ctx, int which, int reps, double *ms_per_launch);

/* Copy a result grid to host memory (see RISM3D_GRID_*). */
int rism3d_get_grid(rism3d_ctx *ctx, int which, double *host);

/* The same grid formed on the device into caller-owned device memory (a
 * torch tensor's data pointer, a DLPack buffer, ...) on the context's GPU:
 * no host traffic.  With a caller stream (rism3d_params.stream) the work is
 * ordered on that stream and the call returns without waiting; with the
 * context's own stream it waits for the copy.  BAD_INPUT for a pointer that
 * is not device memory of the context's GPU. */
int rism3d_get_grid_device(rism3d_ctx *ctx, int which, double *dev);

/* Batched small solutes (no reference counterpart; the reference solves
 * one solute per process).  Solute m has natoms[m] atoms starting at
 * atom offset off[m] in the concatenated arrays, a cubic grid
 * grids[m]^3 and cubic box boxes[m].  results[m] receives its result. */
int rism3d_solve_batch(rism3d_ctx *ctx, int nmol, const int *natoms,
                       const int *grids, const double *boxes,
                       const double *sig, const double *eps, const double *q,
                       const double *xyz, rism3d_result *results);

/* Free the context: its grids, plans, stream (unless caller-owned), batch
 * children and memory pool. */
void rism3d_destroy(rism3d_ctx *ctx);

/* Allocation-free mu_ex / PMV integrals.  No counterpart in the reference
 * (it has no library API).  For callers that cannot call cudaMalloc where
 * they need these integrals: a host application whose own pool allocator
 * has already reserved the free device memory (cudaMalloc would fail or
 * fragment that pool), or a latency-critical loop that cannot afford
 * cudaMalloc's implicit device synchronisation.  Inputs are the caller's
 * device grids h[natv][n] (Re h of the OZ step) and t[natv][n] (absolute
 * t), rho[natv] on the host; out (host) receives 3*natv+1 doubles:
 * SFEC_SC[v], SFEC_SC_HNC[v], SFEC_GF[v] in J/mol (output_xmu.cu) and
 * sum_v rho_v dv int c_v (cal_pmv.cu; PMV = xt (1 - that) N_A kB T).
 * Work runs on `stream` (NULL: legacy default) and the call returns after
 * it.  The reduction scratch is one static device array of 148 KiB
 * (592 blocks x 32 sums), held by every GPU that loads the library until
 * exit; limit: natv <= 8, n < 2^31 (larger sizes return
 * RISM3D_UNSUPPORTED_SHAPE).  The first call on a device looks up the
 * array's device address with that device current -- make that first call
 * before any stream capture.  All calls share the array and every value a
 * call reads is written by that same call (nothing needs clearing), so
 * calls that overlap on the GPU race.  Errors: rism3d_last_error(NULL). */
int rism3d_exchem_noalloc(int closure, int natv, long long n, double dv,
                          double temperature, const double *rho,
                          const double *d_h, const double *d_t, void *stream,
                          double *out);

/* Last error message of ctx, or, when ctx is NULL, of the last failed call
 * without a context (create, initialize, exchem_noalloc) made by the calling
 * host thread: that message is kept per thread, so threads that drive
 * different GPUs do not overwrite each other's.  The pointer stays valid
 * until the next such call on the same thread. */
const char *rism3d_last_error(const rism3d_ctx *ctx);

/* ---- file-driven API: the three public RISM3D methods -------------------
 * rism3d_initialize == RISM3D::initialize(control, structure, esp, hs,
 * centering, q0) (initialize.cu:4-13): reads the .inp (and optional
 * structure file), the .xvk named in it, centres the solute, zeroes the
 * charges when q0, and computes the potential grids.  esp names an ESP
 * cube (NULL or "" for none; its grid must equal the control file's, else
 * BAD_INPUT with the reference's message); hs names the RMDFT hard-sphere
 * file (NULL or "" for none), which also reads the .cvk beside the .xvk. 
 * `device` selects the GPU (main.cu -d) and `precision` the arithmetic. */
int rism3d_initialize(rism3d_ctx **ctx, const char *control,
                      const char *structure, const char *esp, const char *hs,
                      int centering, int q0, int device, int precision);

/* RISM3D::iterate(cu) (iterate.cu:6-90), including the .tuv restart read
 * when <basename>.tuv exists and the ksave writes. */
int rism3d_iterate(rism3d_ctx *ctx, int chargeup);

/* RISM3D::output() (output.cu:6-62): writes .xmu/.xmu0, .gra, .guv, .huv,
 * .cuv, .euv, .qv according to the control file's outlist letters. */
int rism3d_output(rism3d_ctx *ctx);

/* ---- 1D XRISM / DRISM solvent tables ----------------------------------
 * No counterpart in the reference: it reads X_ab(k) from .xvk files
 * (solvent_read.cc:31-60) made by a separate program that it does not
 * ship.  rism1d_solve computes them for a molecular solvent (any mixture of
 * rigid molecules and ions) with the 1D extended RISM equations and the KH
 * (or HNC) closure on the grid r_i = i dr, k_j = j pi / (ntab dr), and
 * rism1d_write_xvk writes them in the .xvk layout the 3D solver reads.
 * With dielectric > 0 the equations are the dielectrically consistent
 * DRISM ones (Perkyns and Pettitt): every molecule with a dipole moment
 * must have it along +z or -z in its site coordinates. */
typedef struct {
  double temperature;   /* K */
  int ntab;             /* radial / k points (power of two) */
  double dr;            /* A */
  int closure;          /* RISM3D_KH or RISM3D_HNC */
  double convergence;   /* rms of the t update (0 = 1e-12) */
  int maxstep;          /* 0 = 10000 */
  double mixing;        /* DIIS mixing (0 = 0.3; with DRISM 0.1) */
  int verbose;
  double dielectric;    /* > 0: DRISM with this dielectric constant; 0: XRISM */
  double smear;         /* DRISM bridge damping length a, A (0 = 2.0) */
} rism1d_params;

typedef struct {
  char name[8];
  int spc;              /* molecule (species) index, 1-based */
  int sym;              /* site type, 1-based; negative: same type as |sym| */
  double sigma;         /* A */
  double epsilon;       /* J/mol */
  double charge;        /* e */
  double x, y, z;       /* A, in the molecule frame */
  double density;       /* mol/L of the species */
} rism1d_site;

/* xvv (may be NULL): [ntype][ntype][ntab], X_ab(k_j) = sum over the sites
 * of type b of (w_ab + rho_b h_ab), a the first site of its type (the
 * layout of Solvent::xvv); xt: isothermal compressibility (1/Pa). */
int rism1d_solve(const rism1d_params *p, int nsite, const rism1d_site *sites,
                 double *xvv, double *xt, int *iterations);
int rism1d_write_xvk(const char *path, const rism1d_params *p, int nsite,
                     const rism1d_site *sites, const double *xvv, double xt);
const char *rism1d_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* RISM3D_B200_H */
