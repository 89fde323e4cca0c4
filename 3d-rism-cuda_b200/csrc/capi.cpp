// C ABI of the solver (include/rism3d_b200.h).  Host code: validation,
// device buffers, cuFFT plans, and the file-driven RISM3D-style entry
// points.  No compute happens on the host: every grid operation is a CUDA
// kernel or cuFFT, and a missing or failing device is an error, never a
// fallback.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <string>

#include "rism3d_impl.h"
#include "rism3d_io.h"

using namespace rism3d;

struct rism3d_ctx {
  Context c;
};

// Errors of calls that have no context (create, initialize, the
// allocation-free integrals): one message per host thread, so that threads
// driving different GPUs never share the string.
static thread_local std::string g_create_err;

namespace rism3d {

void set_create_error(const std::string &msg) { g_create_err = msg; }

// Free everything a context owns, its batch children included.
void context_release(Context &c) {
  cudaSetDevice(c.dev);
  if (c.stream) cudaStreamSynchronize(c.stream);
  for (Context::Child &ch : c.children) {
    context_release(*ch.ctx);
    delete ch.ctx;
  }
  c.children.clear();
  free_device(c);
  for (Timer *t : {&c.tm_setup, &c.tm_iter, &c.tm_obs}) {
    if (t->a) cudaEventDestroy(t->a);
    if (t->b) cudaEventDestroy(t->b);
    t->a = t->b = nullptr;
  }
  if (c.stream && c.own_stream) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
  if (c.pool) cudaMemPoolDestroy(c.pool);
  c.pool = nullptr;
}

bool cuda_ok(Context &c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  c.err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

bool cufft_ok(Context &c, cufftResult r, const char *what) {
  if (r == CUFFT_SUCCESS) return true;
  c.err = std::string(what) + ": cuFFT error " + std::to_string((int)r);
  return false;
}

void free_device(Context &c) {
  void *ptrs[] = {c.d_u, c.d_e, c.d_fr, c.d_fkh, c.d_atoms, c.d_tw, c.d_twf,
                  c.d_U, c.d_t, c.d_Y, c.d_RP, c.d_buf, c.d_h, c.d_g,
                  c.f_U, c.f_t, c.f_Y, c.f_RP, c.f_buf, c.f_R0, c.f_x0, c.d_part, c.d_state,
                  c.d_stage, c.d_stage_ref, c.d_obs, c.d_atom_part, c.chi.d_coef, c.d_xs,
                  c.d_atom_off, c.d_atom_cnt, c.d_esp, c.d_rm_ccoef, c.d_rm_k2, c.d_rm_hcoef};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  c.d_u = c.d_e = c.d_fr = nullptr; c.d_fkh = nullptr; c.d_atoms = nullptr; c.d_esp = nullptr;
  c.d_rm_ccoef = c.d_rm_k2 = c.d_rm_hcoef = nullptr; c.rmdft = false;
  c.d_tw = nullptr; c.d_twf = nullptr; c.d_U = c.d_t = c.d_Y = c.d_RP = nullptr;
  c.d_buf = nullptr; c.d_h = c.d_g = nullptr;
  c.f_U = c.f_t = c.f_Y = c.f_RP = nullptr; c.f_buf = nullptr; c.f_R0 = c.f_x0 = nullptr;
  c.d_part = nullptr; c.d_state = nullptr; c.d_stage = nullptr; c.d_stage_ref = nullptr;
  c.d_obs = nullptr;
  c.d_atom_part = nullptr; c.chi.d_coef = nullptr; c.natom_part_cap = 0;
  c.d_xs = nullptr; c.nxs = 0;
  if (c.d_xs32) cudaFree(c.d_xs32);
  c.d_xs32 = nullptr;
  c.d_atom_off = c.d_atom_cnt = nullptr;
  if (c.h_state) cudaFreeHost(c.h_state);
  c.h_state = nullptr;
  if (c.graph64) cudaGraphExecDestroy(c.graph64);
  if (c.graph32) cudaGraphExecDestroy(c.graph32);
  if (c.graph32r) cudaGraphExecDestroy(c.graph32r);
  c.graph64 = c.graph32 = c.graph32r = nullptr;
  for (cudaGraphExec_t *g : {&c.loop64, &c.loop32, &c.loop32r}) {
    if (*g) cudaGraphExecDestroy(*g);
    *g = nullptr;
  }
  if (c.d_hist) cudaFree(c.d_hist);
  c.d_hist = nullptr;
  c.hist_cap = 0;
  if (c.d_count) cudaFree(c.d_count);
  c.d_count = nullptr;
  if (c.plan32z) cufftDestroy(c.plan32z);
  c.plan32z = 0;
  c.xfused = false;
  if (c.d_xroots) cudaFree(c.d_xroots);
  c.d_xroots = nullptr;
  if (c.f_Ydm) cudaFree(c.f_Ydm);
  if (c.f_RPdm) cudaFree(c.f_RPdm);
  c.f_Ydm = c.f_RPdm = nullptr;
  c.dm_depth = 0;
  if (c.d_fkt) cudaFree(c.d_fkt);
  c.d_fkt = nullptr;
  delete c.ky_map;
  c.ky_map = nullptr;
  if (c.plan64) cufftDestroy(c.plan64);
  if (c.plan32) cufftDestroy(c.plan32);
  if (c.plan1) cufftDestroy(c.plan1);
  c.plan64 = c.plan32 = c.plan1 = 0;
  c.plans_ok = false;
}

int fetch_grid(Context &c, int which, double *host) {
  const size_t n = (size_t)c.n, V = (size_t)c.natv;
  auto get = [&](const double *d, double *h, size_t cnt) {
    return cuda_ok(c, cudaMemcpyAsync(h, d, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c.stream),
                   "get_grid") &&
           cuda_ok(c, cudaStreamSynchronize(c.stream), "get_grid");
  };
  switch (which) {
    case RISM3D_GRID_U: return get(c.d_u, host, V * n) ? RISM3D_OK : RISM3D_CUDA_ERROR;
    case RISM3D_GRID_FR: return get(c.d_fr, host, n) ? RISM3D_OK : RISM3D_CUDA_ERROR;
    case RISM3D_GRID_E: {
      std::vector<double> fr(n);
      if (!get(c.d_e, host, n) || !get(c.d_fr, fr.data(), n)) return RISM3D_CUDA_ERROR;
      for (size_t j = 0; j < n; ++j) host[j] += fr[j];   // e = esr + fr
      return RISM3D_OK;
    }
    default: break;
  }
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  switch (which) {
    case RISM3D_GRID_G: return get(c.d_g, host, V * n) ? RISM3D_OK : RISM3D_CUDA_ERROR;
    case RISM3D_GRID_H: return get(c.d_h, host, V * n) ? RISM3D_OK : RISM3D_CUDA_ERROR;
    case RISM3D_GRID_T:
    case RISM3D_GRID_C: {
      std::vector<double> fr(n), h;
      if (!get(c.d_t, host, V * n) || !get(c.d_fr, fr.data(), n)) return RISM3D_CUDA_ERROR;
      for (size_t v = 0; v < V; ++v)
        for (size_t j = 0; j < n; ++j) host[v * n + j] += c.qv[v] * c.cf_final * fr[j];
      if (which == RISM3D_GRID_C) {
        h.resize(V * n);
        if (!get(c.d_h, h.data(), V * n)) return RISM3D_CUDA_ERROR;
        for (size_t i = 0; i < V * n; ++i) host[i] = h[i] - host[i];
      }
      return RISM3D_OK;
    }
    case RISM3D_GRID_QV: {                                  // cal_qv.cu:20-27
      std::vector<double> g(V * n);
      if (!get(c.d_g, g.data(), V * n)) return RISM3D_CUDA_ERROR;
      for (size_t j = 0; j < n; ++j) host[j] = 0.0;
      for (size_t v = 0; v < V; ++v)
        for (size_t j = 0; j < n; ++j) host[j] += g[v * n + j] * (c.rho[v] * c.qv[v]);
      return RISM3D_OK;
    }
  }
  c.err = "unknown grid id";
  return RISM3D_BAD_INPUT;
}

}  // namespace rism3d

static int alloc_state(Context &c) {
  // every per-solute grid is [nb][...]
  const size_t n = (size_t)c.n * c.nb, V = (size_t)c.natv, P = (V + 1) / 2;
  const bool mixed = c.prm.precision == RISM3D_MIXED;
  auto A = [&](void **p, size_t bytes, const char *w) {
    return cuda_ok(c, cudaMalloc(p, bytes), w);
  };
  bool ok = A((void **)&c.d_u, sizeof(double) * V * n, "alloc u") &&
            A((void **)&c.d_U, sizeof(double) * V * n, "alloc U") &&
            A((void **)&c.d_t, sizeof(double) * V * n, "alloc t") &&
            A((void **)&c.d_Y, sizeof(double) * 2 * V * n, "alloc Y") &&
            A((void **)&c.d_RP, sizeof(double) * 2 * V * n, "alloc RP") &&
            A((void **)&c.d_buf, sizeof(double2) * P * n, "alloc buf") &&
            A((void **)&c.d_h, sizeof(double) * V * n, "alloc h") &&
            A((void **)&c.d_g, sizeof(double) * V * n, "alloc g") &&
            A((void **)&c.d_obs, sizeof(double) * 64 * c.nb, "alloc obs");
  if (ok && mixed)
    ok = A((void **)&c.f_U, sizeof(float) * V * n, "alloc U32") &&
         A((void **)&c.f_t, sizeof(float) * V * n, "alloc t32") &&
         A((void **)&c.f_Y, sizeof(float) * 2 * V * n, "alloc Y32") &&
         A((void **)&c.f_RP, sizeof(float) * 2 * V * n, "alloc RP32") &&
         A((void **)&c.f_buf, sizeof(float2) * P * n, "alloc buf32") &&
         A((void **)&c.f_R0, sizeof(float) * V * n, "alloc R0 32") &&
         A((void **)&c.f_x0, sizeof(float) * V * n, "alloc x0 32");
  if (!ok) return RISM3D_CUDA_ERROR;
  // batched 3D plans over the site pairs; x is the fastest axis
  // one batched plan over all site pairs of all solutes
  int dims[3] = {c.nz, c.ny, c.nx};
  const int np = (int)c.n, nbat = (int)(P * c.nb);
  if (!cufft_ok(c, cufftPlanMany(&c.plan64, 3, dims, nullptr, 1, np, nullptr, 1, np,
                                 CUFFT_Z2Z, nbat), "cufftPlanMany Z2Z"))
    return RISM3D_CUFFT_ERROR;
  if (mixed && !cufft_ok(c, cufftPlanMany(&c.plan32, 3, dims, nullptr, 1, np, nullptr, 1,
                                          np, CUFFT_C2C, nbat), "cufftPlanMany C2C"))
    return RISM3D_CUFFT_ERROR;
  if (mixed) {
    const int rc = setup_fused_axes(c);
    if (rc != RISM3D_OK) return rc;
  }
  // depth-M Anderson for the plain FP32 bulk (opt-in, single solutes)
  c.dm_depth = 0;
  if (const char *e = getenv("RISM3D_MDIIS")) {
    const int M = atoi(e);
    if (mixed && c.nb == 1 && M >= 2 && M <= 6) {
      const size_t b = sizeof(float) * (size_t)M * V * n;
      if (!A((void **)&c.f_Ydm, b, "alloc MDIIS history") ||
          !A((void **)&c.f_RPdm, b, "alloc MDIIS history"))
        return RISM3D_CUDA_ERROR;
      c.dm_depth = M;
    }
  }
  {
    const int rc = setup_pipe_r(c);
    if (rc != RISM3D_OK) return rc;
  }
  c.plans_ok = true;
  return RISM3D_OK;
}

extern "C" {

}  // extern "C"

namespace rism3d {

// Validate params and set up a context for nb solutes sharing one cell
// (nb = 1 for rism3d_create; rism3d_solve_batch uses nb > 1).
int context_init(Context &c, const rism3d_params *p, int nb, std::string &err) {
  for (int d = 0; d < 3; ++d) {
    if (p->grid[d] < 4 || p->grid[d] % 4 != 0 || p->grid[d] > 2048) {
      err = "grid sizes must be multiples of 4 in [4, 2048] (half-shifted transform, fft3d.cu)";
      return RISM3D_UNSUPPORTED_SHAPE;
    }
    if (!(p->box[d] > 0)) { err = "box must be positive"; return RISM3D_BAD_INPUT; }
  }
  if ((long long)p->grid[0] * p->grid[1] * p->grid[2] >= (1LL << 31)) {
    err = "grid has 2^31 points or more";
    return RISM3D_UNSUPPORTED_SHAPE;
  }
  if (p->closure != RISM3D_KH && p->closure != RISM3D_HNC) {
    err = "Unexpected closure switch";
    return RISM3D_BAD_INPUT;
  }
  if (p->maxstep < 1 || !(p->convergence > 0) || p->an2_count < 0 || nb < 1) {
    err = "bad iteration control";
    return RISM3D_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    err = "no CUDA device";
    return RISM3D_NO_DEVICE;
  }
  if (p->device < 0 || p->device >= ndev) { err = "bad device ordinal"; return RISM3D_NO_DEVICE; }
  c.prm = *p;
  c.dev = p->device;
  c.nb = nb;
  if (cudaSetDevice(c.dev) != cudaSuccess) {
    err = "cannot initialise the CUDA device";
    return RISM3D_CUDA_ERROR;
  }
  if (p->stream) {
    c.stream = (cudaStream_t)p->stream;
    c.own_stream = false;
  } else if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    err = "cannot create a CUDA stream";
    return RISM3D_CUDA_ERROR;
  }
  {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c.dev;
    uint64_t keep = ~0ull;
    if (cudaMemPoolCreate(&c.pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
      err = "cannot create a CUDA memory pool";
      if (c.pool) cudaMemPoolDestroy(c.pool);
      c.pool = nullptr;
      if (c.own_stream) cudaStreamDestroy(c.stream);
      c.stream = nullptr;
      return RISM3D_CUDA_ERROR;
    }
  }
  c.nx = p->grid[0]; c.ny = p->grid[1]; c.nz = p->grid[2];
  c.n = (long long)c.nx * c.ny * c.nz;
  c.vol = p->box[0] * p->box[1] * p->box[2];             // cell.cc:9-14
  c.dv = c.vol / (double)c.n;
  for (int d = 0; d < 3; ++d) c.dr[d] = p->box[d] / p->grid[d];
  const long long nn = c.n * nb;
  bool ok = cuda_ok(c, cudaMalloc(&c.d_e, sizeof(double) * nn), "alloc esr") &&
            cuda_ok(c, cudaMalloc(&c.d_fr, sizeof(double) * nn), "alloc fr") &&
            cuda_ok(c, cudaMalloc(&c.d_fkh, sizeof(double2) * (nn / 2)), "alloc fk") &&
            cuda_ok(c, cudaMalloc(&c.d_tw, sizeof(double2) * (c.nx + c.ny + c.nz)), "alloc tw") &&
            cuda_ok(c, cudaMalloc(&c.d_twf, sizeof(float2) * (c.nx + c.ny + c.nz)), "alloc tw") &&
            cuda_ok(c, cudaMalloc(&c.d_state, sizeof(DevState) * nb), "alloc state") &&
            cuda_ok(c, cudaMalloc(&c.d_stage, sizeof(StageParams)), "alloc stage") &&
            cuda_ok(c, cudaMalloc(&c.d_stage_ref, sizeof(StageParams)), "alloc stage") &&
            (!(p->verbose && nb == 1) ||
             cuda_ok(c, cudaMalloc(&c.d_hist, sizeof(double) * ((size_t)std::max(p->maxstep, 1) + 8)),
                     "alloc history")) &&
            cuda_ok(c, cudaHostAlloc(&c.h_state, sizeof(DevState) * 4 * nb, cudaHostAllocDefault), "alloc pinned");
  if (c.d_hist) c.hist_cap = std::max(p->maxstep, 1) + 8;
  // RISM3D_HOST_LOOP=1: drive iterations from the host (one graph launch per
  // iteration) instead of the device-side loop, e.g. for per-launch profiling
  if (const char *e = getenv("RISM3D_HOST_LOOP")) c.no_device_loop = e[0] == '1';
  long long nbk = (c.n + 255) / 256;
  c.nred_blocks = (int)(nbk < 148 * 8 ? nbk : 148 * 8);
  ok = ok && cuda_ok(c, cudaMalloc(&c.d_part, sizeof(double) * 64 * c.nred_blocks * nb), "alloc partials") &&
       cuda_ok(c, cudaMalloc(&c.d_count, sizeof(unsigned) * nb), "alloc counter") &&
       cuda_ok(c, cudaMemset(c.d_count, 0, sizeof(unsigned) * nb), "zero counter");
  for (Timer *t : {&c.tm_setup, &c.tm_iter, &c.tm_obs}) {
    cudaEventCreate(&t->a);
    cudaEventCreate(&t->b);
  }
  if (!ok || build_twiddles(c) != RISM3D_OK) {
    err = c.err;
    free_device(c);
    if (c.own_stream) cudaStreamDestroy(c.stream);
    c.stream = nullptr;
    cudaMemPoolDestroy(c.pool);
    c.pool = nullptr;
    return RISM3D_CUDA_ERROR;
  }
  return RISM3D_OK;
}

int context_set_solvent(Context &c, int natv, const double *rho, const double *q,
                        const double *sig, const double *eps, double temperature, double xt,
                        int ntab, double dr, const double *xvv);
int context_set_atoms(Context &c, const std::vector<int> &cnt, const double *sig,
                      const double *eps, const double *q, const double *xyz);

}  // namespace rism3d

extern "C" {

int rism3d_create(const rism3d_params *p, rism3d_ctx **out) {
  if (!p || !out) { g_create_err = "null argument"; return RISM3D_BAD_INPUT; }
  *out = nullptr;
  rism3d_ctx *x = new (std::nothrow) rism3d_ctx;
  if (!x) return RISM3D_BAD_INPUT;
  std::string err;
  int rc = context_init(x->c, p, 1, err);
  if (rc != RISM3D_OK) {
    g_create_err = err;
    delete x;
    return rc;
  }
  *out = x;
  return RISM3D_OK;
}

}  // extern "C"

namespace rism3d {

int context_set_solvent(Context &c, int natv, const double *rho, const double *q,
                        const double *sig, const double *eps, double temperature, double xt,
                        int ntab, double dr, const double *xvv) {
  cudaSetDevice(c.dev);
  if (natv < 1 || natv > kMaxSites) { c.err = "natv must be 1..8"; return RISM3D_UNSUPPORTED_SHAPE; }
  if (!rho || !q || !sig || !eps || !xvv || ntab < 4 || !(dr > 0) || !(temperature > 0) || !(xt > 0)) {
    c.err = "bad solvent arguments";
    return RISM3D_BAD_INPUT;
  }
  for (int v = 0; v < natv; ++v)
    if (!(rho[v] > 0)) { c.err = "solvent densities must be positive"; return RISM3D_BAD_INPUT; }
  if (c.have_solvent && natv != c.natv) {
    c.err = "solvent site count cannot change on a context";
    return RISM3D_BAD_STATE;
  }
  c.natv = natv;
  for (int v = 0; v < natv; ++v) { c.rho[v] = rho[v]; c.qv[v] = q[v]; c.sigv[v] = sig[v]; c.epsv[v] = eps[v]; }
  c.temper = temperature; c.xt = xt; c.ntab = ntab; c.xdr = dr;
  c.xvv_host.assign(xvv, xvv + (size_t)natv * natv * ntab);
  if (!c.have_solvent) {
    int rc = alloc_state(c);
    if (rc != RISM3D_OK) return rc;
  }
  int rc = upload_chi(c);
  if (rc != RISM3D_OK) return rc;
  c.have_solvent = true;
  c.have_solute = false;
  c.solved = false;
  return RISM3D_OK;
}

// Atoms of the nb solutes, concatenated (cnt[b] atoms each), then the
// potential grids of every solute.
int context_set_atoms(Context &c, const std::vector<int> &cnt, const double *sig,
                      const double *eps, const double *q, const double *xyz) {
  cudaSetDevice(c.dev);
  if (!c.have_solvent) { c.err = "set the solvent first"; return RISM3D_BAD_STATE; }
  if ((int)cnt.size() != c.nb || !sig || !eps || !q || !xyz) {
    c.err = "bad solute arguments";
    return RISM3D_BAD_INPUT;
  }
  int natom = 0;
  c.atom_off.assign(c.nb, 0);
  c.atom_cnt = cnt;
  for (int b = 0; b < c.nb; ++b) {
    if (cnt[b] < 1) { c.err = "every solute needs at least one atom"; return RISM3D_BAD_INPUT; }
    c.atom_off[b] = natom;
    natom += cnt[b];
  }
  c.natom = natom;
  c.sig.assign(sig, sig + natom);
  c.eps.assign(eps, eps + natom);
  c.q.assign(q, q + natom);
  c.xyz.assign(xyz, xyz + 3 * (size_t)natom);
  std::vector<double> pack((size_t)natom * 8, 0.0);
  for (int i = 0; i < natom; ++i) {
    double *a = &pack[(size_t)i * 8];
    a[0] = xyz[3 * i]; a[1] = xyz[3 * i + 1]; a[2] = xyz[3 * i + 2];
    a[3] = q[i]; a[4] = sig[i]; a[5] = eps[i];
    if (!std::isfinite(a[0] + a[1] + a[2] + a[3] + a[4] + a[5]) || eps[i] < 0) {
      c.err = "non-finite or negative solute parameter";
      return RISM3D_BAD_INPUT;
    }
  }
  if (c.d_atoms) cudaFree(c.d_atoms);
  c.d_atoms = nullptr;
  if (!c.d_atom_off &&
      (!cuda_ok(c, cudaMalloc(&c.d_atom_off, sizeof(int) * c.nb), "alloc atom offsets") ||
       !cuda_ok(c, cudaMalloc(&c.d_atom_cnt, sizeof(int) * c.nb), "alloc atom counts")))
    return RISM3D_CUDA_ERROR;
  if (!cuda_ok(c, cudaMalloc(&c.d_atoms, sizeof(double) * pack.size()), "alloc atoms") ||
      !cuda_ok(c, cudaMemcpyAsync(c.d_atoms, pack.data(), sizeof(double) * pack.size(),
                                  cudaMemcpyHostToDevice, c.stream), "copy atoms") ||
      !cuda_ok(c, cudaMemcpyAsync(c.d_atom_off, c.atom_off.data(), sizeof(int) * c.nb,
                                  cudaMemcpyHostToDevice, c.stream), "copy atoms") ||
      !cuda_ok(c, cudaMemcpyAsync(c.d_atom_cnt, c.atom_cnt.data(), sizeof(int) * c.nb,
                                  cudaMemcpyHostToDevice, c.stream), "copy atoms"))
    return RISM3D_CUDA_ERROR;
  cudaEventRecord(c.tm_setup.a, c.stream);
  int rc = compute_potentials(c);
  cudaEventRecord(c.tm_setup.b, c.stream);
  if (rc != RISM3D_OK) return rc;
  if (!cuda_ok(c, cudaStreamSynchronize(c.stream), "potentials")) return RISM3D_CUDA_ERROR;
  c.have_solute = true;
  c.solved = false;
  c.have_forces = false;
  return RISM3D_OK;
}

}  // namespace rism3d

extern "C" {

int rism3d_set_solvent(rism3d_ctx *x, int natv, const double *rho, const double *q,
                       const double *sig, const double *eps, double temperature, double xt,
                       int ntab, double dr, const double *xvv) {
  if (!x) return RISM3D_BAD_INPUT;
  rism3d_set_rmdft(x, nullptr, 0, nullptr, nullptr, nullptr, 0.0, 0.0);  // tables follow the solvent
  return context_set_solvent(x->c, natv, rho, q, sig, eps, temperature, xt, ntab, dr, xvv);
}

int rism3d_set_rmdft(rism3d_ctx *x, const double *cvk, int ntab2, const double *k,
                     const double *chs, const double *w, double pfhs, double w0) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  for (double **p : {&c.d_rm_ccoef, &c.d_rm_k2, &c.d_rm_hcoef}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  c.rmdft = false;
  if (!cvk) return RISM3D_OK;
  if (c.nb != 1) { c.err = "RMDFT is for single-solute contexts"; return RISM3D_BAD_STATE; }
  if (!c.have_solvent) { c.err = "set the solvent first"; return RISM3D_BAD_STATE; }
  if (ntab2 < 4 || !k || !chs || !w || !std::isfinite(w0) || !(pfhs >= 0.0 && pfhs < 1.0)) {
    c.err = "bad RMDFT hard-sphere table";
    return RISM3D_BAD_INPUT;
  }
  for (int i = 1; i < ntab2; ++i)
    if (!(k[i] > k[i - 1])) { c.err = "RMDFT hard-sphere knots must increase"; return RISM3D_BAD_INPUT; }
  // the table must reach the grid's largest |k| (solvent_spline2.cu:16-19)
  const double kx = 2.0 * kPi * (c.nx / 2.0 - 0.5) / c.prm.box[0];
  const double ky = 2.0 * kPi * (c.ny / 2.0 - 0.5) / c.prm.box[1];
  const double kz = 2.0 * kPi * (c.nz / 2.0 - 0.5) / c.prm.box[2];
  if (sqrt(kx * kx + ky * ky + kz * kz) > k[ntab2 - 1]) {
    c.err = "insufficient maximal T tabulated";
    return RISM3D_BAD_INPUT;
  }
  const int V = c.natv, nt = c.chi.ntab;
  std::vector<double> xp(nt), cc((size_t)nt * V * V * 4), hc((size_t)ntab2 * 8);
  for (int i = 0; i < nt; ++i) xp[i] = c.chi.dk * (i + 1);      // solvent_spline.cu:50-62
  for (int ab = 0; ab < V * V; ++ab)
    spline_coefficients(xp.data(), cvk + (size_t)ab * nt, nt, &cc[(size_t)ab * 4],
                        (size_t)V * V * 4);
  spline_coefficients(k, chs, ntab2, &hc[0], 8);                 // solvent_spline2.cu:33-56
  spline_coefficients(k, w, ntab2, &hc[4], 8);
  if (!cuda_ok(c, cudaMalloc(&c.d_rm_ccoef, sizeof(double) * cc.size()), "alloc RMDFT") ||
      !cuda_ok(c, cudaMalloc(&c.d_rm_k2, sizeof(double) * ntab2), "alloc RMDFT") ||
      !cuda_ok(c, cudaMalloc(&c.d_rm_hcoef, sizeof(double) * hc.size()), "alloc RMDFT") ||
      !cuda_ok(c, cudaMemcpy(c.d_rm_ccoef, cc.data(), sizeof(double) * cc.size(),
                             cudaMemcpyHostToDevice), "copy RMDFT") ||
      !cuda_ok(c, cudaMemcpy(c.d_rm_k2, k, sizeof(double) * ntab2, cudaMemcpyHostToDevice),
               "copy RMDFT") ||
      !cuda_ok(c, cudaMemcpy(c.d_rm_hcoef, hc.data(), sizeof(double) * hc.size(),
                             cudaMemcpyHostToDevice), "copy RMDFT"))
    return RISM3D_CUDA_ERROR;
  c.rm_ntab2 = ntab2;
  c.rm_pfhs = pfhs;
  c.rm_w0 = w0;
  c.rmdft = true;
  return RISM3D_OK;
}

int rism3d_set_solute(rism3d_ctx *x, int natom, const double *sig, const double *eps,
                      const double *q, const double *xyz) {
  if (!x) return RISM3D_BAD_INPUT;
  if (natom < 1) { x->c.err = "bad solute arguments"; return RISM3D_BAD_INPUT; }
  return context_set_atoms(x->c, std::vector<int>(1, natom), sig, eps, q, xyz);
}

int rism3d_set_tuv(rism3d_ctx *x, const double *t) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  if (!c.have_solvent) { c.err = "set the solvent first"; return RISM3D_BAD_STATE; }
  if (!t) c.t_init.clear();
  else c.t_init.assign(t, t + (size_t)c.natv * c.n);
  return RISM3D_OK;
}

int rism3d_solve(rism3d_ctx *x, int chargeup, rism3d_result *res) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.have_solvent || !c.have_solute) { c.err = "solvent and solute must be set"; return RISM3D_BAD_STATE; }
  if (chargeup < 0) { c.err = "chargeup must be >= 0"; return RISM3D_BAD_INPUT; }
  c.res = rism3d_result{};
  c.have_forces = false;
  cudaEventRecord(c.tm_iter.a, c.stream);
  int rc = run_solve(c, chargeup);
  cudaEventRecord(c.tm_iter.b, c.stream);
  if (rc != RISM3D_OK) return rc;
  cudaEventRecord(c.tm_obs.a, c.stream);
  rc = compute_observables(c);
  // SE: from the grids for one solute with the point-charge potential; per
  // (site, atom) pairs otherwise (an ESP cube is not the atoms' potential)
  if (rc == RISM3D_OK)
    rc = (c.nb == 1 && !c.d_esp) ? compute_se_from_grids(c) : compute_atom_integrals(c, false);
  if (rc == RISM3D_OK) rc = compute_rmdft(c);                // output.cu:25
  cudaEventRecord(c.tm_obs.b, c.stream);
  if (rc != RISM3D_OK) return rc;
  if (!cuda_ok(c, cudaStreamSynchronize(c.stream), "solve")) return RISM3D_CUDA_ERROR;
  float ms = 0;
  cudaEventElapsedTime(&ms, c.tm_setup.a, c.tm_setup.b); c.res.ms_setup = ms;
  cudaEventElapsedTime(&ms, c.tm_iter.a, c.tm_iter.b); c.res.ms_iterate = ms;
  cudaEventElapsedTime(&ms, c.tm_obs.a, c.tm_obs.b); c.res.ms_observe = ms;
  c.solved = true;
  if (res) *res = c.res;
  if (c.res.status != RISM3D_OK) return c.res.status;
  return RISM3D_OK;
}

// the per-(site, atom) pair integrals (and forces) after a solve whose SE
// came from the grids; the reported SE totals stay those of the solve
static int atom_integrals_keep_se(Context &c, bool forces) {
  const double se = c.res.se, lj = c.res.se_lj, es = c.res.se_es;
  int rc = compute_atom_integrals(c, forces);
  c.res.se = se; c.res.se_lj = lj; c.res.se_es = es;
  return rc;
}

int rism3d_euv(rism3d_ctx *x, double *euv) {
  if (!x || !euv) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  if (c.euv.empty()) {
    int rc = atom_integrals_keep_se(c, false);
    if (rc != RISM3D_OK) return rc;
  }
  std::copy(c.euv.begin(), c.euv.end(), euv);
  return RISM3D_OK;
}

int rism3d_forces(rism3d_ctx *x, double *dulj, double *due) {
  if (!x || !dulj || !due) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  if (!c.have_forces) {
    int rc = atom_integrals_keep_se(c, true);
    if (rc != RISM3D_OK) return rc;
  }
  std::copy(c.dulj.begin(), c.dulj.end(), dulj);
  std::copy(c.due.begin(), c.due.end(), due);
  return RISM3D_OK;
}

int rism3d_grad(rism3d_ctx *x, double *dq, double *dsig, double *deps, double *dR) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  if (c.d_esp) {
    c.err = "gradients are not defined with an ESP cube potential (it does not follow the solute)";
    return RISM3D_BAD_STATE;
  }
  return compute_adjoint(c, RISM3D_FP64, dq, dsig, deps, dR);
}

int rism3d_grad_precision(rism3d_ctx *x, int precision, double *dq, double *dsig, double *deps,
                          double *dR) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (precision != RISM3D_FP64 && precision != RISM3D_MIXED) {
    c.err = "precision must be RISM3D_FP64 or RISM3D_MIXED";
    return RISM3D_BAD_INPUT;
  }
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  if (c.d_esp) {
    c.err = "gradients are not defined with an ESP cube potential (it does not follow the solute)";
    return RISM3D_BAD_STATE;
  }
  return compute_adjoint(c, precision, dq, dsig, deps, dR);
}

int rism3d_set_esp(rism3d_ctx *x, const double *esp) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (c.nb != 1) { c.err = "an ESP cube is for single-solute contexts"; return RISM3D_BAD_STATE; }
  if (!esp) {
    if (c.d_esp) cudaFree(c.d_esp);
    c.d_esp = nullptr;
  } else {
    if (!c.d_esp && !cuda_ok(c, cudaMalloc(&c.d_esp, sizeof(double) * c.n), "alloc esp"))
      return RISM3D_CUDA_ERROR;
    if (!cuda_ok(c, cudaMemcpyAsync(c.d_esp, esp, sizeof(double) * c.n, cudaMemcpyHostToDevice,
                                    c.stream), "copy esp"))
      return RISM3D_CUDA_ERROR;
  }
  if (!c.have_solute)
    return cuda_ok(c, cudaStreamSynchronize(c.stream), "copy esp") ? RISM3D_OK : RISM3D_CUDA_ERROR;
  int rc = compute_potentials(c);                 // the solute's grids follow at once
  if (rc != RISM3D_OK) return rc;
  if (!cuda_ok(c, cudaStreamSynchronize(c.stream), "potentials")) return RISM3D_CUDA_ERROR;
  c.solved = false;
  c.have_forces = false;
  return RISM3D_OK;
}

int rism3d_get_grid(rism3d_ctx *x, int which, double *host) {
  if (!x || !host) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.have_solute) { c.err = "no solute"; return RISM3D_BAD_STATE; }
  return fetch_grid(c, which, host);
}

int rism3d_get_grid_device(rism3d_ctx *x, int which, double *dev) {
  if (!x || !dev) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.have_solute) { c.err = "no solute"; return RISM3D_BAD_STATE; }
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, dev) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
      at.device != c.dev) {
    cudaGetLastError();
    c.err = "get_grid_device: not a device pointer on the context's GPU";
    return RISM3D_BAD_INPUT;
  }
  int rc = device_grid(c, which, dev);
  if (rc == RISM3D_OK && c.own_stream && !cuda_ok(c, cudaStreamSynchronize(c.stream), "get_grid_device"))
    return RISM3D_CUDA_ERROR;
  return rc;
}

void rism3d_destroy(rism3d_ctx *x) {
  if (!x) return;
  context_release(x->c);
  delete x;
}

int rism3d_refresh_potentials(rism3d_ctx *x) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.have_solute) { c.err = "no solute"; return RISM3D_BAD_STATE; }
  cudaEventRecord(c.tm_setup.a, c.stream);
  int rc = compute_potentials(c);
  cudaEventRecord(c.tm_setup.b, c.stream);
  c.solved = false;
  c.have_forces = false;
  return rc;
}

long long rism3d_kernel_launches(const rism3d_ctx *x) { return x ? x->c.launches : 0; }

int rism3d_time_kernel(rism3d_ctx *x, int which, int reps, double *ms) {
  if (!x || !ms || reps < 1) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.have_solute) { c.err = "no solute"; return RISM3D_BAD_STATE; }
  return time_kernel(c, which, reps, ms);
}

const char *rism3d_last_error(const rism3d_ctx *x) {
  if (!x) return g_create_err.c_str();
  return x->c.err.c_str();
}

// ------------------------------------------------------------ file driven
static std::string dir_of(const std::string &p) {
  size_t s = p.rfind('/');
  return s == std::string::npos ? std::string() : p.substr(0, s + 1);
}

int rism3d_initialize(rism3d_ctx **out, const char *control, const char *structure,
                      const char *esp, const char *hs, int centering, int q0, int device,
                      int precision) {
  if (!out || !control) { g_create_err = "null argument"; return RISM3D_BAD_INPUT; }
  *out = nullptr;
  io::ControlFile cf;
  std::string err;
  std::string st = structure ? structure : "";
  if (!io::read_control(control, st, cf, err)) { g_create_err = err; return RISM3D_BAD_INPUT; }
  std::string ctl = control;
  std::string svpath = cf.fsolvent;
  if (!svpath.empty() && svpath[0] != '/') {
    // the reference opens the solvent path relative to the working directory
    std::ifstream probe(svpath.c_str());
    if (!probe) svpath = dir_of(ctl) + cf.fsolvent;
  }
  io::SolventFile sf;
  if (!io::read_xvk(svpath, sf, err)) { g_create_err = err; return RISM3D_BAD_INPUT; }
  rism3d_params p{};
  for (int d = 0; d < 3; ++d) { p.grid[d] = cf.grid[d]; p.box[d] = cf.box[d]; }
  p.closure = cf.closure; p.convergence = cf.conv; p.maxstep = cf.maxstep;
  p.an2_count = cf.count; p.an2_m = cf.m; p.an2_mp = cf.mp;
  p.precision = precision; p.device = device; p.verbose = 1;
  rism3d_ctx *x = nullptr;
  int rc = rism3d_create(&p, &x);
  if (rc != RISM3D_OK) return rc;
  Context &c = x->c;
  c.outlist = cf.outlist; c.ksave = cf.ksave; c.zero = q0 != 0;
  c.sig_in = cf.sig; c.eps_in = cf.eps; c.q_in = cf.q; c.xyz_in = cf.xyz;
  std::string base = st.empty() ? ctl : st;                    // set_fname.cu:5-12
  size_t dot = base.rfind('.');
  c.fname = dot == std::string::npos ? base : base.substr(0, dot);
  std::vector<double> xyz = cf.xyz, q = cf.q;
  if (centering) io::centre(xyz, c.shift);                    // read_input.cu:80-82
  if (q0) for (double &v : q) v = 0.0;                        // solute.cu:45-49
  rc = rism3d_set_solvent(x, sf.natv, sf.rho.data(), sf.q.data(), sf.sig.data(), sf.eps.data(),
                          sf.temper, sf.xt, sf.ntab, sf.dr, sf.xvv.data());
  if (rc == RISM3D_OK && hs && *hs) {                         // solvent_read.cc:88-140
    io::SolventFile cv;
    io::HardSphereFile hf;
    const size_t dot = svpath.rfind('.');
    const std::string cvk = (dot == std::string::npos ? svpath : svpath.substr(0, dot)) + ".cvk";
    if (!io::read_xvk(cvk, cv, err)) {
      c.err = "cvk file could not be opened! (" + err + ")";
      rc = RISM3D_BAD_INPUT;
    } else if (cv.natv != sf.natv || cv.ntab != sf.ntab) {
      c.err = "the .cvk table does not match the .xvk (sites or rows)";
      rc = RISM3D_BAD_INPUT;
    } else if (!io::read_hard_sphere(hs, hf, err)) {
      c.err = err;
      rc = RISM3D_BAD_INPUT;
    } else {
      rc = rism3d_set_rmdft(x, cv.xvv.data(), hf.ntab2, hf.k.data(), hf.chs.data(), hf.w.data(),
                            hf.pfhs, hf.w0);
    }
  }
  if (rc == RISM3D_OK && esp && *esp) {                       // cal_Coulomb.cu:41-96
    std::vector<double> cube;
    if (!io::read_esp_cube(esp, p.grid, cube, err)) {
      c.err = err;
      rc = RISM3D_BAD_INPUT;
    } else {
      rc = rism3d_set_esp(x, cube.data());
    }
  }
  if (rc == RISM3D_OK)
    rc = rism3d_set_solute(x, (int)q.size(), cf.sig.data(), cf.eps.data(), q.data(), xyz.data());
  if (rc != RISM3D_OK) {
    g_create_err = c.err;
    rism3d_destroy(x);
    return rc;
  }
  *out = x;
  return RISM3D_OK;
}

int rism3d_iterate(rism3d_ctx *x, int chargeup) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  std::string tuv = c.fname + ".tuv";                          // iterate.cu:25-33
  std::vector<double> t;
  std::string warn;
  if (io::read_tuv(tuv, c.prm.grid, c.natv, t, warn)) {
    if (!warn.empty()) fprintf(stderr, "%s\n", warn.c_str());
    if (t.size() == (size_t)c.natv * c.n) c.t_init = t;
    chargeup = 0;
  }
  if (chargeup > 0) printf("Charge up %d\n", chargeup);
  int rc = rism3d_solve(x, chargeup, nullptr);
  c.t_init.clear();
  if (rc == RISM3D_CUDA_ERROR || rc == RISM3D_CUFFT_ERROR || rc == RISM3D_BAD_STATE) return rc;
  if (c.ksave != 0 && c.res.status == RISM3D_OK) {             // iterate.cu:64-71
    std::vector<double> tt((size_t)c.natv * c.n);
    if (fetch_grid(c, RISM3D_GRID_T, tt.data()) == RISM3D_OK)
      io::write_tuv(tuv, c.prm.grid, c.natv, tt.data(), c.n);
  }
  return rc;
}

int rism3d_output(rism3d_ctx *x) {
  if (!x) return RISM3D_BAD_INPUT;
  Context &c = x->c;
  cudaSetDevice(c.dev);
  if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
  std::string ol = c.outlist;
  for (char &ch : ol) ch = (char)tolower(ch);                   // output.cu:8
  auto has = [&](char k) { return ol.find(k) != std::string::npos; };
  const size_t n = (size_t)c.n, V = (size_t)c.natv;
  if (has('m')) {
    io::XmuValues xv{};
    xv.natv = c.natv; xv.closure = c.prm.closure;
    for (int v = 0; v < c.natv; ++v) {
      xv.sfec_sc[v] = c.res.sfec_sc[v];
      xv.sfec_sc_hnc[v] = c.res.sfec_sc_hnc[v];
      xv.sfec_gf[v] = c.res.sfec_gf[v];
    }
    xv.se = c.res.se; xv.se_lj = c.res.se_lj; xv.se_es = c.res.se_es;
    xv.pmv_l = c.res.pmv; xv.pressure = c.res.pressure; xv.correction = c.res.correction;
    xv.rmdft = c.rmdft; xv.sfe_rmdft = c.res.sfe_rmdft;
    if (!io::write_xmu(c.fname + (c.zero ? ".xmu0" : ".xmu"), xv)) { c.err = "cannot write .xmu"; return RISM3D_BAD_INPUT; }
  }
  if (has('d')) {
    std::vector<double> a((size_t)c.natom * 3), b((size_t)c.natom * 3);
    int rc = rism3d_forces(x, a.data(), b.data());
    if (rc != RISM3D_OK) return rc;
    io::write_gra(c.fname + ".gra", c.natom, a.data(), b.data());
  }
  std::vector<double> buf;
  if (has('c')) {
    buf.resize(V * n);
    fetch_grid(c, RISM3D_GRID_C, buf.data());
    io::write_grid_text(c.fname + ".cuv", c.prm.box, c.prm.grid, c.natom, c.q.data(), c.sig.data(),
                        c.eps.data(), c.xyz.data(), c.natv, buf.data(), c.n);
  }
  if (has('g')) {
    buf.resize(V * n);
    fetch_grid(c, RISM3D_GRID_G, buf.data());
    io::write_guv(c.fname + ".guv", c.natv, c.prm.grid, c.prm.box, c.shift, buf.data(), c.n);
  }
  if (has('h')) {
    buf.resize(V * n);
    fetch_grid(c, RISM3D_GRID_H, buf.data());
    io::write_grid_text(c.fname + ".huv", c.prm.box, c.prm.grid, c.natom, c.q.data(), c.sig.data(),
                        c.eps.data(), c.xyz.data(), c.natv, buf.data(), c.n);
  }
  if (has('e')) {
    if (c.euv.empty()) {
      int rc = atom_integrals_keep_se(c, false);
      if (rc != RISM3D_OK) return rc;
    }
    io::write_euv(c.fname + ".euv", c.natom, c.natv, c.euv.data());
  }
  if (has('q')) {
    buf.resize(n);
    fetch_grid(c, RISM3D_GRID_QV, buf.data());
    for (double &v : buf) v *= c.dv;
    io::write_qv(c.fname + ".qv", c.prm.grid, c.dr, buf.data(), c.n);
  }
  return RISM3D_OK;
}

}  // extern "C"
