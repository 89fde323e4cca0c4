// Internal declarations of the B200 3D-RISM solver (not part of the ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <map>
#include <string>
#include <vector>

#include "rism3d_b200.h"

namespace rism3d {

constexpr int kMaxSites = RISM3D_MAX_SITES;

// Physical constants, the same values as the reference (physical.h:4-17).
constexpr double kAvogadro = 6.02214076e23;
constexpr double kBohr = 0.5291771500001;         // Angstrom
constexpr double kBoltzmann = 1.380649e-23;       // J/K
constexpr double kHartree = 4.359744722207185e-18;
constexpr double kPi = 3.14159265358979323846;

// Device-resident iteration control.  Written only by k_finalize (one
// thread); read by every pass of the next iteration, so the loop runs with
// no host round trip.  Mirrors the host-side state of AN2
// (anderson.h:16-37) and RISM3D::iterate (iterate.cu:49-73).
struct DevState {
  int done;        // 0 running, 1 converged, 2 diverged, 3 maxstep reached,
                   // 4 stalled (no 10% rms gain in 30 steps while watched)
  int after_done;  // finalize calls since `done` was set
  int iter;        // iterations completed in this run
  int mode;        // update the next pass A applies: 0 none, 1 Picard, 2 AN2
  int upd_slot;    // history slot written by that update
  int binary;      // AN2 ping-pong bit for the following update
  int count;       // Picard warm-up steps left
  int maxstep;
  int measure;     // 1: the finalize only records the sums (kernel timing)
  int watch;       // 1: stop as stalled (done = 4) when progress stops
  int since;       // steps since the best rms last improved by 10 %
  int loops;       // device-side loop: bodies run in this launch (solute 0)
  int bodies;      // device-side loop bodies of the whole solve (solute 0)
  int stage_iter;  // steps of this charge-up stage, all phases
  int total_iter;  // steps of the solve, all stages and phases
  int total32;     // of which FP32
  int fallback;    // (solute 0) the FP32 bulk diverged: stage restarts in FP64
  int restart_next;  // (solute 0) FP64 phase starts a fresh AN2 history
  int fault;       // a device-side wait gave up (a bulk or tile copy never
                   // arrived): the loop was stopped and the solve reports it
  double best;     // best rms of this run (stagnation watch)
  double conv;
  double m, mp;    // AN2 mixing factor and bias
  double s1, s2;   // AN2 coefficients for the next update
  double rms;
  double sums[6];  // sum R^2, c0, c1, a00, a01, a11 of the last pass R
  int dm_fill;     // depth-M Anderson (opt-in): history slots filled,
  int dm_last;     // the slot written last (-1: none yet),
  int dm_use;      // and the slots the next update mixes
  double sdm[8];   // its coefficients per slot (bias included)
};

// 1/sqrt(x) for x > 0: the FP64 hardware approximation (rsqrt.approx.f64,
// ~2^-22 relative error e) refined by STEPS Newton-Raphson steps
// y <- y (3 - x y^2) / 2, each of which squares the error (1.5 e^2 after
// one step, ~1e-13; FP64 rounding after two).  x below 1e-300 is treated as
// 1e-300 (callers handle r = 0 separately).
#ifdef __CUDACC__
template <int STEPS>
__device__ __forceinline__ double rsqrt_nr(double x) {
  x = fmax(x, 1.0e-300);
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
#pragma unroll
  for (int s = 0; s < STEPS; ++s) y = y * (1.5 - 0.5 * x * y * y);
  return y;
}
#endif

// Per charge-up stage constants, read by the kernels through a pointer so
// that one captured iteration graph serves every stage.
struct StageParams {
  double qcf[kMaxSites];   // q_v * cf
  double irho[kMaxSites];  // 1 / rho_v (AN2 weights, anderson.cu:28-31)
};

// Natural-spline coefficients of chi_ab(k) on the uniform knots
// k_i = dk (i+1): for knot i and pair ab, {y, c0, c1, c2}
// (spline.cc:36-42, splint.cc:18-19).
struct ChiTable {
  int ntab = 0;
  double dk = 0.0;
  double *d_coef = nullptr;  // [ntab][natv*natv][4]
};

// Division by a runtime constant d >= 1 for dividends x < 2^31 by
// multiply-high and shift (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994, round-up variant):
// s = ceil(log2 d), m = floor(2^32 (2^s - d) / d) + 1, q = (mulhi(x,m) + x) >> s.
struct FastDiv {
  unsigned d = 1, m = 1, s = 0;
  FastDiv() = default;
  explicit FastDiv(unsigned dd) : d(dd) {
    s = 0;
    while ((1ull << s) < dd) ++s;
    m = (unsigned)(((1ull << 32) * ((1ull << s) - dd)) / dd + 1);
  }
#ifdef __CUDACC__
  __device__ __forceinline__ unsigned div(unsigned x) const {
    return (__umulhi(x, m) + x) >> s;
  }
#endif
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
};

struct Context {
  rism3d_params prm{};
  std::string err;
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  // Stream-ordered scratch comes from this pool, which keeps its memory until
  // the context is destroyed: the device's default pool returns freed memory
  // at every synchronisation, and mapping it again while the next solve's
  // kernels ran slowed whole 256^3 solves 3-7x on B200 (about one in three).
  cudaMemPool_t pool = nullptr;
  long long launches = 0;      // kernels of this library launched so far

  // solutes solved together on this context (same cell; rism3d_solve_batch)
  int nb = 1;
  // cell (cell.cc:8-22)
  int nx = 0, ny = 0, nz = 0;
  long long n = 0;
  double vol = 0, dv = 0, dr[3] = {0, 0, 0};

  // solvent
  int natv = 0;
  double rho[kMaxSites], qv[kMaxSites], sigv[kMaxSites], epsv[kMaxSites];
  double temper = 0, xt = 0;
  bool have_solvent = false;
  ChiTable chi;
  // cubic cells: chi_ab tabulated per s = ox^2 + oy^2 + oz^2 (odd o_d), so
  // |k| = (pi/L) sqrt(s) and the table index is (s - 3) / 8
  double *d_xs = nullptr;    // [nidx][V*V] or null (general cells: spline)
  float *d_xs32 = nullptr;   // the same in FP32 for the FP32 passes
  int nxs = 0;
  std::vector<double> xvv_host;
  int ntab = 0;
  double xdr = 0;

  // solute
  int natom = 0;
  std::vector<double> sig, eps, q, xyz;
  bool have_solute = false;

  // device grids
  double *d_u = nullptr;     // [V][N] beta u_LJ
  double *d_e = nullptr;     // [N]   beta sum q e^-r / r (short-range Coulomb)
  double *d_fr = nullptr;    // [N]   beta long-range part
  double *d_esp = nullptr;   // [N]   ESP cube (Hartree/e) replacing the point-charge e, or null
  // RMDFT correction (cal_rmdft.cu): solvent c(k) and site 0's hard-sphere table
  bool rmdft = false;
  double rm_pfhs = 0.0, rm_w0 = 0.0;
  int rm_ntab2 = 0;
  double *d_rm_ccoef = nullptr;  // [ntab][V*V][4] spline of c(k) on the chi knots
  double *d_rm_k2 = nullptr;     // [ntab2] hard-sphere table knots
  double *d_rm_hcoef = nullptr;  // [ntab2][2][4] splines of chi_hs(k) and w(k)
  double2 *d_fkh = nullptr;  // [N/2] beta fk on the owner half of k space
  double *d_atoms = nullptr; // [A][8] x y z q sig eps pad (all solutes)
  int *d_atom_off = nullptr; // [nb] first atom of each solute
  int *d_atom_cnt = nullptr; // [nb] atoms of each solute
  std::vector<int> atom_off, atom_cnt;
  double2 *d_tw = nullptr;   // twiddle rows: [nx] [ny] [nz] exp(-i pi x/n)
  float2 *d_twf = nullptr;

  // FP64 iteration state
  double *d_U = nullptr;     // [V][N] short-range potential of the stage
  double *d_t = nullptr;     // [V][N] t_SR = t - q cf fr
  double *d_Y = nullptr;     // [2][V][N] history t + m R
  double *d_RP = nullptr;    // [2][V][N] history R
  double2 *d_buf = nullptr;  // [P][N] packed site pairs (FFT in place)
  double *d_h = nullptr;     // [V][N] final h (snapshot)
  double *d_g = nullptr;     // [V][N] final g
  // FP32 iteration state (MIXED)
  float *f_U = nullptr, *f_t = nullptr, *f_Y = nullptr, *f_RP = nullptr;
  float2 *f_buf = nullptr;
  // FP32 refinement: base residual R0 and closure argument x0 = t0 - U_SR
  float *f_R0 = nullptr, *f_x0 = nullptr;

  double *d_part = nullptr;  // reduction partials
  int nred_blocks = 0;
  DevState *d_state = nullptr;
  DevState *h_state = nullptr;  // pinned mirror
  StageParams *d_stage = nullptr;
  StageParams *d_stage_ref = nullptr;  // refinement passes: qcf = 0
  double *d_obs = nullptr;      // observables scratch
  double *d_atom_part = nullptr;
  int natom_part_cap = 0;

  cufftHandle plan64 = 0, plan32 = 0;
  // FP32 passes with the x and y axes of the transforms folded in (single
  // solutes, natv <= 2, nx = ny = 64 or 256): cuFFT then transforms along z
  // only (plan32z), with the x-line roots of unity in d_xroots
  // depth-M Anderson for the plain FP32 bulk (opt-in RISM3D_MDIIS=M):
  // history [M][V][N] of Y = t + m R and of R
  int dm_depth = 0;
  float *f_Ydm = nullptr, *f_RPdm = nullptr;
  bool pipe_r = false;       // pass R as the cp.async pipeline (natv <= 2)
  bool bulk_r = false;       // pass R as the bulk-copy (cp.async.bulk) stream
  bool xfused = false;
  cufftHandle plan32z = 0;
  float2 *d_xroots = nullptr;
  // TMA form of the fused pass K (nx = ny = 256): tensor map over f_buf and
  // beta fk in FP32 laid out [nz/2][nx][ny]
  CUtensorMap *ky_map = nullptr;
  float2 *d_fkt = nullptr;
  cufftHandle plan1 = 0;     // one Z2Z transform of the cell (RMDFT), made on first use
  bool plans_ok = false;
  // one captured iteration per precision, reused by every solve
  cudaGraphExec_t graph64 = nullptr, graph32 = nullptr, graph32r = nullptr;
  // the same iterations inside a device-side while loop (conditional graph
  // node): one launch runs a whole phase; null when the driver refuses it
  cudaGraphExec_t loop64 = nullptr, loop32 = nullptr, loop32r = nullptr;
  bool no_device_loop = false;
  double *d_hist = nullptr;     // per-iteration rms (verbose single solves)
  int hist_cap = 0;
  unsigned *d_count = nullptr;  // pass-R block counter (last block finalizes)

  // restart guess
  std::vector<double> t_init;

  // results
  bool solved = false;
  double cf_final = 1.0;
  rism3d_result res{};
  std::vector<rism3d_result> bres;   // per solute when nb > 1
  std::vector<double> euv;       // [2][V][A] (x dv)
  std::vector<double> dulj, due; // [A][3] (x dv)
  bool have_forces = false;
  int adj_steps = 0;             // Anderson steps of the last adjoint solve
  bool adj_stalled = false;      // FP32 adjoint stopped at its rounding floor

  // file-driven mode (rism3d_initialize)
  std::string outlist, fname, fsolvent, control_dir;
  int ksave = 0;
  bool zero = false;
  double shift[3] = {0, 0, 0};
  std::vector<double> sig_in, eps_in, q_in, xyz_in;  // as read (pre-shift)

  Timer tm_setup, tm_iter, tm_obs;

  // batched solves: one child context per (grid, box, count) group, kept for
  // reuse by later batches (buffers, plans and captured graphs)
  struct Child {
    int grid = 0, nb = 0;
    double box = 0;
    Context *ctx = nullptr;
    long long last_call = 0;   // batch call that last used it
    size_t bytes = 0;          // device memory it holds (measured at creation)
  };
  std::vector<Child> children;
  long long batch_calls = 0;
  // autotuned sub-batch size (grid points) per set of cells in a batch
  std::map<std::string, long long> batch_tuned;
};

// ---- kernels/launchers (implemented in the .cu files) ----
int build_twiddles(Context &c);
int compute_potentials(Context &c);               // potential.cu
int launch_potential_r(Context &c);               // potential.cu (timing hook)
int upload_chi(Context &c);                       // solver.cu
// decide on and set up the fused-axis FP32 passes (plan, roots, limits)
int setup_fused_axes(Context &c);                 // solver.cu
int setup_kspace_tma(Context &c);                 // solver.cu: TMA fused pass K
int fused_fk_columns(Context &c);                 // solver.cu: fk copy for it
int setup_pipe_r(Context &c);                     // solver.cu: pipelined pass R
// spline.cc:4-43: natural cubic spline through (xp[k], yp[k]), k < np; writes
// {y_k, b_k, c_k, d_k} (y + b t + c t^2 + d t^3 on interval k; zero
// coefficients on the last knot) to out[k * stride + 0..3]
void spline_coefficients(const double *xp, const double *yp, int np, double *out,
                         size_t stride);            // solver.cu
int compute_rmdft(Context &c);                     // rmdft.cu
int run_solve(Context &c, int chargeup);          // solver.cu
int compute_observables(Context &c);              // observe.cu
int compute_atom_integrals(Context &c, bool forces);  // observe.cu
int compute_se_from_grids(Context &c);            // observe.cu: SE totals, one solute
int device_grid(Context &c, int which, double *out);  // observe.cu: rism3d_get_grid_device
// precision RISM3D_FP64: FP64 throughout; RISM3D_MIXED: FP32 transposed
// solve and FP32 LJ pair factors of the back-projection, FP64 accumulation
int compute_adjoint(Context &c, int precision, double *dq, double *dsig, double *deps,
                    double *dR);                  // adjoint.cu
// FP64 OZ k-space pass on a packed buffer (adjoint solve)
int launch_oz_kspace(Context &c, double2 *buf, const StageParams *sp, DevState *st);
// the same pass in FP32 (the adjoint's FP32 variant)
int launch_oz_kspace32(Context &c, float2 *buf, const StageParams *sp, DevState *st);
int fetch_grid(Context &c, int which, double *host);
int time_kernel(Context &c, int which, int reps, double *ms);   // solver.cu
void free_device(Context &c);
int context_init(Context &c, const rism3d_params *p, int nb, std::string &err);
int context_set_solvent(Context &c, int natv, const double *rho, const double *q,
                        const double *sig, const double *eps, double temperature, double xt,
                        int ntab, double dr, const double *xvv);
int context_set_atoms(Context &c, const std::vector<int> &cnt, const double *sig,
                      const double *eps, const double *q, const double *xyz);
void context_release(Context &c);

bool cuda_ok(Context &c, cudaError_t e, const char *what);
// stream-ordered allocation of `bytes` from the context's pool on its stream
inline cudaError_t pool_alloc(Context &c, void **p, size_t bytes) {
  return cudaMallocFromPoolAsync(p, bytes, c.pool, c.stream);
}
// message returned by rism3d_last_error(NULL) (context-free entry points)
void set_create_error(const std::string &msg);
bool cufft_ok(Context &c, cufftResult r, const char *what);

}  // namespace rism3d
