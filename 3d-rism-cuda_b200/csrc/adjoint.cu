// Adjoint gradients of the solvation free energy SFE_SC with respect to the
// solute parameters (charges, LJ sigma and epsilon, positions): the exact
// derivative of the reference's discrete mu_ex (cal_exchem.cu:55-122) at
// the converged solution.
//
// With t the state, x = -beta u - q e + t the closure argument, g = C(x),
// h the OZ result and c = h - t, the discrete equations of the reference
// (calculate_cuda.cu, fft3d.cu) are h = L(c + delta), where L is the OZ
// operator (L v)_a = F^-1[sum_b X_ab F[v_b]] -- symmetric in the inner
// product weighted by rho, since rho_a X_ab = rho_b X_ba -- and
// delta_a = q_a (fr - F^-1[fk]) is the mismatch between the real-space
// long-range grid and its analytic transform (cal_Coulomb.cu:109-140: fk is
// not the discrete transform of fr).  Differentiating the KH/HNC functional
// at the solution and eliminating dc/dp with one adjoint solve gives
//
//   dSFE/dp / (N_A kB T) = <rho (g - zeta/2), d(beta u)/dp>
//                          + 1/2 <sum_a rho_a q_a (zeta_a - h_a), d(fr - F^-1 fk)/dp>
//
// with zeta = L xi + w, w = L delta and xi the solution of the linear system
//   G xi - (G - 1) L xi = (G - 1) w,      G = C'(x)
// (the transpose of the solve's own Jacobian; no division by g, which is 0
// in the solute core).  Without the mismatch (delta = 0) zeta vanishes and
// the first term is the familiar <rho g d(beta u)/dp>.
//
// Inside the solute core G underflows and the system pins zeta to
// G xi / (G - 1), i.e. to zero with g.  The iterative solve leaves a residual
// of order its tolerance in L xi + w there, which the steep repulsive
// potential (d(beta u)/dp ~ r^-14 near an atom) would amplify; zeta is
// therefore taken from the pointwise form wherever G < 1/2, where both forms
// agree at the solution.
//
// Kernels: the linear solve reuses the k-space OZ pass of the iteration
// around cuFFT and is accelerated by Anderson mixing (depth 6; per step one
// fused pass forms the residual, the mixing vector and the Gram dots, and one
// pass combines the stored mixing vectors); the gradient
// back-propagates the weights through the potential-grid computation, one
// atom per thread with grid points streamed through shared memory and every
// pair term recomputed (cal_LJ.cu:57-71, cal_Coulomb.cu:109-121), and through
// the k-space fk kernel with per-axis phase rows.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "rism3d_impl.h"
#include "halfshift.cuh"

namespace rism3d {
namespace {

constexpr int kThreads = 256;
constexpr int kAtomsPerBlock = 128;
constexpr int kPtsTile = 128;
constexpr int NOUT = 6;   // dq, dsigma, deps, dRx, dRy, dRz
constexpr int kDepth = 6; // Anderson history of the adjoint solve
constexpr int kDotBlocks = 2368;

struct SiteW {
  double sig[kMaxSites], eps[kMaxSites], q[kMaxSites], rho[kMaxSites];
};

// inverse-transform input for the real function with transform fk (owner
// half stored): dir fk at k and -dir conj(fk) at the mirror -k
__global__ void k_fk_to_buf(long long n, int nx, int ny, const double2 *fkh, double2 *buf) {
  const long long nh = n / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nh;
       j += (long long)gridDim.x * blockDim.x) {
    const long long r = j / nx;
    const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
    const int dir = ((ix + iy + iz) & 1) ? -1 : 1;
    const double2 f = fkh[j];
    buf[j] = make_double2(dir * f.x, dir * f.y);
    buf[n - 1 - j] = make_double2(-dir * f.x, dir * f.y);
  }
}

// delta_a = q_a (fr - F^-1 fk)
__global__ void k_delta(long long n, int nv, const double *fr, const double *finv,
                        const StageParams *sp, double *delta) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const double d = fr[j] - finv[j];
    for (int v = 0; v < nv; ++v) delta[(size_t)v * n + j] = sp->qcf[v] * d;
  }
}

// closure derivative G = C'(x), x = t_SR - U_SR (KH: 1 for x >= 0, else e^x),
// stored in the solve's precision T
template <typename T>
__global__ void k_gprime(long long tot, int closure, const double *t, const double *U, T *G) {
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < tot;
       f += (long long)gridDim.x * blockDim.x) {
    const double x = t[f] - U[f];
    G[f] = (T)((closure == 0 && x >= 0.0) ? 1.0 : exp(x));
  }
}

template <typename A, typename B>
__global__ void k_cast(long long n, const A *src, B *dst) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x)
    dst[j] = (B)src[j];
}

// One Anderson step's bookkeeping in one pass:
//   r = (G - 1)(w + L xi) - G xi          into residual slot `slot`
//   y = xi + eta r                        into mixing slot `slot`
// and the partial dots of r with the first ns residual slots (the slot
// itself contributes |r|^2) and |r|^2 (last row), summed in a fixed order by
// k_sum_rows.  The other slots are read before the slot is written.
// T is the storage precision of the solve (double or float); the residual
// is formed and the dots are accumulated in FP64.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_residual_dots(long long tot, const T *__restrict__ G, const T *__restrict__ w,
                const T *__restrict__ Lxi, const T *__restrict__ xi, double eta,
                T *const *rs, int slot, int ns, T *__restrict__ ys, double *part) {
  __shared__ double red[kThreads / 32][kDepth + 1];
  double acc[kDepth + 1];
#pragma unroll
  for (int i = 0; i <= kDepth; ++i) acc[i] = 0.0;
  T *__restrict__ rslot = rs[slot];
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < tot;
       f += (long long)gridDim.x * blockDim.x) {
    const double g = G[f], x = xi[f];
    const double rd = (g - 1.0) * ((double)w[f] + (double)Lxi[f]) - g * x;
    const T rt = (T)rd;
    const double r = (double)rt;             // the stored value enters the dots
#pragma unroll
    for (int i = 0; i < kDepth; ++i)
      if (i < ns) acc[i] += r * (i == slot ? r : (double)rs[i][f]);
    acc[kDepth] += r * r;
    rslot[f] = rt;
    ys[f] = (T)(x + eta * r);
  }
#pragma unroll
  for (int i = 0; i <= kDepth; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[i] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int i = 0; i <= kDepth; ++i) red[wid][i] = acc[i];
  __syncthreads();
  if (threadIdx.x <= kDepth) {
    double t = 0.0;
    for (int v = 0; v < kThreads / 32; ++v) t += red[v][threadIdx.x];
    part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

__global__ void k_sum_rows(const double *part, int ncols, double *out) {
  __shared__ double red[kThreads];
  const int k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < ncols; b += blockDim.x) s += part[(size_t)k * ncols + b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = red[0];
}

template <typename T>
struct Mix {
  const T *ys[kDepth];        // xi_i + eta r_i of the stored steps
  double c[kDepth];
  int ns;
};

// xi = sum_i c_i y_i, y_i = xi_i + eta r_i (summed in FP64)
template <typename T>
__global__ void k_combine(long long tot, Mix<T> mx, T *xi) {
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < tot;
       f += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kDepth; ++i)
      if (i < mx.ns) s += mx.c[i] * (double)mx.ys[i][f];
    xi[f] = (T)s;
  }
}

// zeta (L xi + w, or G xi / (G - 1) where G < 1/2), then the weights
//   W_a = rho_a (g_a - zeta_a / 2),  Omega = sum_a rho_a q_a (zeta_a - h_a)
template <typename T>
__global__ void k_weights(long long n, int nv, const double *g, const double *h,
                          const T *G, const T *xi, const T *Lxi,
                          const double *w, SiteW sv, double *W, double *Om) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    double om = 0.0;
    for (int v = 0; v < nv; ++v) {
      const size_t i = (size_t)v * n + j;
      const double gp = G[i], x = xi[i];
      const double zeta = gp < 0.5 ? gp * x / (gp - 1.0) : (double)Lxi[i] + w[i];
      W[i] = sv.rho[v] * (g[i] - 0.5 * zeta);
      om += sv.rho[v] * sv.q[v] * (zeta - h[i]);
    }
    Om[j] = om;
  }
}

// Real-space back-propagation, one atom per thread:
//   W-weighted derivatives of beta u_LJ (N_A kB T units cancel) and of
//   q_v e (x cc), plus the Omega-weighted derivative of fr (x cc / 2).
// 1/r comes from the refined reciprocal square root (1/r^2 as its square),
// and e^-r is dropped beyond 40 A (below 4.3e-18, as in the potential
// kernel).  MIX evaluates the LJ pair factors in FP32 (the FP32 variant);
// the Coulomb and long-range terms and every sum stay FP64.
template <int V, bool MIX>
__global__ void __launch_bounds__(kAtomsPerBlock)
k_adjoint_r(int nx, int ny, int nz, double drx, double dry, double drz,
            const double *__restrict__ W, const double *__restrict__ Om,
            const double *__restrict__ atoms, int natom, SiteW sv, double cc,
            long long chunk, double *part) {
  __shared__ double4 pp[kPtsTile];          // x y z Omega
  __shared__ double pw[V][kPtsTile];
  const long long n = (long long)nx * ny * nz;
  const int ia = blockIdx.x * kAtomsPerBlock + threadIdx.x;
  const bool live = ia < natom;
  double X = 0, Y = 0, Z = 0, qu = 0, su = 0, eu = 0;
  if (live) {
    const double *a = atoms + 8 * (size_t)ia;
    X = a[0]; Y = a[1]; Z = a[2]; qu = a[3]; su = a[4]; eu = a[5];
  }
  // per site: sigma_uv^2 and the prefactors of d/d sigma_u, d/d eps_u and
  // the radial force of the LJ term
  double sg2[V], fs[V], fe[V], ff[V], qc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const double sg = (su + sv.sig[v]) * 0.5;    // cal_LJ.cu:28
    const double euv = sqrt(eu * sv.eps[v]);     // cal_LJ.cu:29
    sg2[v] = sg * sg;
    fs[v] = 12.0 * euv / sg;
    fe[v] = eu > 0.0 ? 2.0 * euv / eu : 0.0;
    ff[v] = 24.0 * euv;
    qc[v] = sv.q[v] * cc;
  }
  double acc[NOUT] = {0, 0, 0, 0, 0, 0};
  const long long j0 = (long long)blockIdx.y * chunk;
  const long long j1 = min(n, j0 + chunk);
  for (long long base = j0; base < j1; base += kPtsTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kPtsTile; i += blockDim.x) {
      const long long j = base + i;
      if (j < j1) {
        const long long r = j / nx;
        const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
        pp[i] = make_double4((ix - nx / 2) * drx, (iy - ny / 2) * dry, (iz - nz / 2) * drz, Om[j]);
#pragma unroll
        for (int v = 0; v < V; ++v) pw[v][i] = W[(size_t)v * n + j];
      } else {
        pp[i] = make_double4(1.0e30, 1.0e30, 1.0e30, 0.0);
#pragma unroll
        for (int v = 0; v < V; ++v) pw[v][i] = 0.0;
      }
    }
    __syncthreads();
    if (!live) continue;
    const int m = (int)min((long long)kPtsTile, j1 - base);
    for (int i = 0; i < m; ++i) {
      const double4 p = pp[i];
      const double dx = p.x - X, dy = p.y - Y, dz = p.z - Z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const bool clamped = r2 < 1.0e-4;            // cal_LJ.cu:64
      const double ri = r2 > 0.0 ? rsqrt_nr<2>(r2) : 0.0;
      const double ir2 = clamped ? 1.0e4 : ri * ri;
      const double ra = r2 * ri;
      const bool coul = ra >= 1.0e-5;              // cal_Coulomb.cu:114
      double wq = 0.0, fr = 0.0;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double w = pw[v][i];
        // w = 0 in the solute core, where g and zeta underflow
        if (w != 0.0) {
          double b12, b6;                          // 2 s^12 - s^6 and s^12 - s^6
          if (MIX) {
            const float s2 = (float)sg2[v] * (float)ir2;
            const float s6 = s2 * s2 * s2, s12 = s6 * s6;
            b12 = (double)(2.0f * s12 - s6);
            b6 = (double)(s12 - s6);
          } else {
            const double s2 = sg2[v] * ir2;
            const double s6 = s2 * s2 * s2, s12 = s6 * s6;
            b12 = 2.0 * s12 - s6;
            b6 = s12 - s6;
          }
          acc[1] += w * fs[v] * b12;               // d/d sigma_u
          acc[2] += w * fe[v] * b6;                // d/d eps_u
          if (!clamped) fr += w * ff[v] * b12 * ir2;
        }
        if (coul) wq += w * qc[v];
      }
      // half-weighted long-range term: phi(r) = (1 - e^-r)/r, phi = 1 below 1e-5
      const double om = 0.5 * cc * p.w;
      if (coul) {
        acc[0] += wq * ri;
        fr += wq * qu * ri * ri * ri;
        const double em = ra < 40.0 ? exp(-ra) : 0.0;
        const double phi = (1.0 - em) * ri;
        const double dphi = (ra * em - (1.0 - em)) * ri * ri;      // d phi / d r
        acc[0] += om * phi;
        fr -= om * qu * dphi * ri;                 // d phi(|p - R|)/dR = -phi' (p - R)/r
      } else {
        acc[0] += om;                              // fr gets q below 1e-5
      }
      acc[3] += fr * dx;
      acc[4] += fr * dy;
      acc[5] += fr * dz;
    }
  }
  if (live) {
    double *o = part + ((size_t)blockIdx.y * natom + ia) * NOUT;
#pragma unroll
    for (int k = 0; k < NOUT; ++k) o[k] = acc[k];
  }
}

// k-space back-propagation of the fk term: per atom
//   scale * sum over the owner half of e^{-ik.R} 4 pi conj(Omega^) / (k^2 (k^2+1))
// (the mirror half contributes the complex conjugate, folded into scale)
__global__ void __launch_bounds__(kAtomsPerBlock)
k_adjoint_k(int nx, int ny, int nz, double bx, double by, double bz, const double2 *omh,
            const double2 *ph, const double *atoms, int natom, double scale, long long chunk,
            double *part) {
  __shared__ double2 sw[kPtsTile];            // 4 pi conj(Omega^) / (k^2 (k^2 + 1))
  __shared__ double4 sk[kPtsTile];            // kx ky kz
  __shared__ int4 si[kPtsTile];               // ix iy iz
  const long long nh = (long long)nx * ny * nz / 2;
  const int L = nx + ny + nz;
  const int ia = blockIdx.x * kAtomsPerBlock + threadIdx.x;
  const bool live = ia < natom;
  const double qu = live ? atoms[8 * (size_t)ia + 3] : 0.0;
  const double2 *row = ph + (size_t)(live ? ia : 0) * L;
  double aq = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
  const long long j0 = (long long)blockIdx.y * chunk;
  const long long j1 = min(nh, j0 + chunk);
  for (long long base = j0; base < j1; base += kPtsTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kPtsTile; i += blockDim.x) {
      const long long j = base + i;
      if (j < j1) {
        const long long r = j / nx;
        const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
        const double kx = 2.0 * kPi * (ix - nx / 2.0 + 0.5) / bx;   // set_g
        const double ky = 2.0 * kPi * (iy - ny / 2.0 + 0.5) / by;
        const double kz = 2.0 * kPi * (iz - nz / 2.0 + 0.5) / bz;
        const double k2 = kx * kx + ky * ky + kz * kz;
        const double f = 4.0 * kPi / (k2 * (k2 + 1.0));
        const double2 o = omh[j];
        sw[i] = make_double2(o.x * f, -o.y * f);
        sk[i] = make_double4(kx, ky, kz, 0.0);
        si[i] = make_int4(ix, iy, iz, 0);
      } else {
        sw[i] = make_double2(0.0, 0.0);
        sk[i] = make_double4(0.0, 0.0, 0.0, 0.0);
        si[i] = make_int4(0, 0, 0, 0);
      }
    }
    __syncthreads();
    if (!live) continue;
    const int m = (int)min((long long)kPtsTile, j1 - base);
    for (int i = 0; i < m; ++i) {
      const int4 id = si[i];
      const double2 px = row[id.x], py = row[nx + id.y], pz = row[nx + ny + id.z];
      const double yzr = py.x * pz.x - py.y * pz.y, yzi = py.x * pz.y + py.y * pz.x;
      const double er = px.x * yzr - px.y * yzi, ei = px.x * yzi + px.y * yzr;  // e^{-ik.R}
      const double2 w = sw[i];
      const double pr = er * w.x - ei * w.y, pim = er * w.y + ei * w.x;
      aq += pr;                                     // d/dq_u: Re(e^{-ik.R} w)
      ax += sk[i].x * pim;                          // d/dR_u: Re(-i k q e^{-ik.R} w)
      ay += sk[i].y * pim;
      az += sk[i].z * pim;
    }
  }
  if (live) {
    double *o = part + ((size_t)blockIdx.y * natom + ia) * 4;
    o[0] = scale * aq;
    o[1] = scale * qu * ax;
    o[2] = scale * qu * ay;
    o[3] = scale * qu * az;
  }
}

// Omega^ = F[Omega] on the owner half: dv dir Y (Y = FFT of dir dkf Omega;
// the packed imaginary part is zero, so no unpacking is needed)
__global__ void k_forward_post(long long n, int nx, int ny, double dv, const double2 *buf,
                               double2 *out) {
  const long long nh = n / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nh;
       j += (long long)gridDim.x * blockDim.x) {
    const long long r = j / nx;
    const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
    const double s = dv * (((ix + iy + iz) & 1) ? -1.0 : 1.0);
    const double2 y = buf[j];
    out[j] = make_double2(s * y.x, s * y.y);
  }
}

__global__ void k_sum_chunks(const double *part, int nchunk, int natom, int na, double *out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= natom * na) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += part[(size_t)c * natom * na + idx];
  out[idx] = s;
}

// per-atom phase rows e^{-i k_x X}, e^{-i k_y Y}, e^{-i k_z Z}
__global__ void k_phase_rows_adj(int nx, int ny, int nz, double bx, double by, double bz,
                                 const double *__restrict__ atoms, int natom,
                                 double2 *__restrict__ ph) {
  const int L = nx + ny + nz;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)natom * L) return;
  const int u = (int)(idx / L), i = (int)(idx % L);
  double k, R;
  if (i < nx) { k = 2.0 * kPi * (i - nx / 2.0 + 0.5) / bx; R = atoms[8 * (size_t)u + 0]; }
  else if (i < nx + ny) { k = 2.0 * kPi * (i - nx - ny / 2.0 + 0.5) / by; R = atoms[8 * (size_t)u + 1]; }
  else { k = 2.0 * kPi * (i - nx - ny - nz / 2.0 + 0.5) / bz; R = atoms[8 * (size_t)u + 2]; }
  double s, c;
  sincos(k * R, &s, &c);
  ph[idx] = make_double2(c, -s);
}

int blocks_for(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

// Device scratch of one adjoint evaluation (stream-ordered, freed at the end).
struct Scratch {
  std::vector<void *> ptrs;
  Context &c;
  explicit Scratch(Context &cc) : c(cc) {}
  template <typename T> T *get(size_t count) {
    void *p = nullptr;
    if (pool_alloc(c, &p, sizeof(T) * count) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T *)p;
  }
  ~Scratch() {
    for (void *p : ptrs) cudaFreeAsync(p, c.stream);
    cudaStreamSynchronize(c.stream);
  }
};

// Solve min |sum c_i r_i| subject to sum c_i = 1 over m stored residuals
// (Gram matrix gram[a][b] = <r_a, r_b>) by the bordered normal equations.
void anderson_coefficients(const std::vector<double> &gram, int m, std::vector<double> &c) {
  const int dd = m + 1;
  std::vector<double> M((size_t)dd * dd, 0.0), rhs(dd, 0.0), x(dd, 0.0);
  double sc = 0.0;
  for (int a = 0; a < m; ++a) sc = std::max(sc, gram[(size_t)a * kDepth + a]);
  if (!(sc > 0)) sc = 1.0;
  for (int a = 0; a < m; ++a) {
    for (int b = 0; b < m; ++b) M[(size_t)a * dd + b] = gram[(size_t)a * kDepth + b] / sc;
    M[(size_t)a * dd + m] = 1.0;
    M[(size_t)m * dd + a] = 1.0;
  }
  rhs[m] = 1.0;
  for (int col = 0; col < dd; ++col) {                 // partial pivoting
    int pv = col;
    for (int rr = col + 1; rr < dd; ++rr)
      if (fabs(M[(size_t)rr * dd + col]) > fabs(M[(size_t)pv * dd + col])) pv = rr;
    for (int k = 0; k < dd; ++k) std::swap(M[(size_t)col * dd + k], M[(size_t)pv * dd + k]);
    std::swap(rhs[col], rhs[pv]);
    const double piv = M[(size_t)col * dd + col];
    if (fabs(piv) < 1e-300) continue;
    for (int rr = col + 1; rr < dd; ++rr) {
      const double f = M[(size_t)rr * dd + col] / piv;
      for (int k = col; k < dd; ++k) M[(size_t)rr * dd + k] -= f * M[(size_t)col * dd + k];
      rhs[rr] -= f * rhs[col];
    }
  }
  for (int rr = dd - 1; rr >= 0; --rr) {
    double s = rhs[rr];
    for (int k = rr + 1; k < dd; ++k) s -= M[(size_t)rr * dd + k] * x[k];
    const double piv = M[(size_t)rr * dd + rr];
    x[rr] = fabs(piv) < 1e-300 ? 0.0 : s / piv;
  }
  c.assign(x.begin(), x.begin() + m);
}

// The transposed solve's operator in precision T: (L v)_a = F^-1[sum_b
// X_ab F[v_b]] with the iteration's own k-space pass between the transforms.
template <typename T> struct OzOp;

template <> struct OzOp<double> {
  Context &c;
  double2 *buf;
  explicit OzOp(Context &cc, double2 *b) : c(cc), buf(b) {}
  int apply(int V, const double *v, double *out, const StageParams *sp, DevState *st) {
    const int gb = blocks_for(c.n);
    k_pack<<<gb, kThreads, 0, c.stream>>>(c.n, V, c.nx, c.ny, c.d_tw, v, buf);
    if (cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)buf, (cufftDoubleComplex *)buf,
                     CUFFT_FORWARD) != CUFFT_SUCCESS) return RISM3D_CUFFT_ERROR;
    int rc = launch_oz_kspace(c, buf, sp, st);
    if (rc != RISM3D_OK) return rc;
    if (cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)buf, (cufftDoubleComplex *)buf,
                     CUFFT_INVERSE) != CUFFT_SUCCESS) return RISM3D_CUFFT_ERROR;
    k_unpack<<<gb, kThreads, 0, c.stream>>>(c.n, V, c.nx, c.ny, c.d_tw, 1.0 / c.vol, buf, out);
    c.launches += 2;
    return RISM3D_OK;
  }
};

template <> struct OzOp<float> {
  Context &c;
  float2 *buf;
  explicit OzOp(Context &cc, float2 *b) : c(cc), buf(b) {}
  int apply(int V, const float *v, float *out, const StageParams *sp, DevState *st) {
    const int gb = blocks_for(c.n);
    k_pack32<<<gb, kThreads, 0, c.stream>>>(c.n, V, c.nx, c.ny, c.d_twf, v, buf);
    if (cufftExecC2C(c.plan32, (cufftComplex *)buf, (cufftComplex *)buf, CUFFT_FORWARD) !=
        CUFFT_SUCCESS)
      return RISM3D_CUFFT_ERROR;
    int rc = launch_oz_kspace32(c, buf, sp, st);
    if (rc != RISM3D_OK) return rc;
    if (cufftExecC2C(c.plan32, (cufftComplex *)buf, (cufftComplex *)buf, CUFFT_INVERSE) !=
        CUFFT_SUCCESS)
      return RISM3D_CUFFT_ERROR;
    k_unpack32<<<gb, kThreads, 0, c.stream>>>(c.n, V, c.nx, c.ny, c.d_twf, (float)(1.0 / c.vol),
                                              buf, out);
    c.launches += 2;
    return RISM3D_OK;
  }
};

// Solve tolerance (relative residual) per precision: FP64 solves to 1e-10;
// FP32 stores its residuals in FP32, whose rounding leaves a floor near
// 1e-7 of |b|, so it stops at 2e-6 (or, stalled at its floor, within 10x
// of that).
template <typename T> struct SolveTol;
template <> struct SolveTol<double> { static constexpr double tol = 1.0e-10; };
template <> struct SolveTol<float> { static constexpr double tol = 2.0e-6; };

// T: arithmetic and storage of the transposed-Jacobian solve (double: the
// FP64 adjoint; float: the FP32 variant, with FP64 dot products, mixing
// coefficients and sums).  The right-hand side w = L delta and the mismatch
// delta are formed in FP64 in both.
template <int V, typename T>
int adjoint_v(Context &c, double *dq, double *dsig, double *deps, double *dR) {
  const long long n = c.n, tot = (long long)V * n;
  const int P = (V + 1) / 2, gb = blocks_for(n), gt = blocks_for(tot);
  const int A = c.natom;
  constexpr bool F32 = sizeof(T) == 4;
  Scratch S(c);
  double *w64 = S.get<double>(tot), *tmp = S.get<double>(tot), *Om = S.get<double>(n);
  T *G = S.get<T>(tot), *xi = S.get<T>(tot), *Lxi = S.get<T>(tot);
  T *w = F32 ? S.get<T>(tot) : (T *)w64;
  T *ys = S.get<T>((size_t)kDepth * tot), *rs = S.get<T>((size_t)kDepth * tot);
  double *dpart = S.get<double>((size_t)(kDepth + 1) * kDotBlocks);
  double *dsum = S.get<double>(kDepth + 1);
  T **hist = S.get<T *>(kDepth);
  StageParams *sp0 = S.get<StageParams>(1), *spq = S.get<StageParams>(1);
  DevState *st0 = S.get<DevState>(1);
  double2 *buf = c.d_buf;                       // the solve is finished: reuse
  typedef typename std::conditional<F32, float2, double2>::type CT;
  CT *bufT = F32 ? (CT *)c.f_buf : (CT *)buf;
  if (F32 && !bufT) bufT = (CT *)S.get<float2>((size_t)P * n);
  if (!G || !w || !w64 || !xi || !Lxi || !tmp || !Om || !ys || !rs || !dpart || !dsum ||
      !hist || !sp0 || !spq || !st0 || !bufT) {
    c.err = "adjoint: out of device memory";
    return RISM3D_CUDA_ERROR;
  }
  if (F32 && !c.plan32) {                       // FP64 context: the FP32 plan, made once
    int dims[3] = {c.nz, c.ny, c.nx};
    if (!cufft_ok(c, cufftPlanMany(&c.plan32, 3, dims, nullptr, 1, (int)n, nullptr, 1, (int)n,
                                   CUFFT_C2C, P), "cufftPlanMany C2C"))
      return RISM3D_CUFFT_ERROR;
  }
  StageParams zero{}, q{};
  for (int v = 0; v < V; ++v) q.qcf[v] = c.qv[v] * c.cf_final;
  DevState run{};
  std::vector<T *> hp(kDepth);
  for (int i = 0; i < kDepth; ++i) hp[i] = rs + (size_t)i * tot;
  if (!cuda_ok(c, cudaMemcpyAsync(sp0, &zero, sizeof(zero), cudaMemcpyHostToDevice, c.stream), "adjoint") ||
      !cuda_ok(c, cudaMemcpyAsync(spq, &q, sizeof(q), cudaMemcpyHostToDevice, c.stream), "adjoint") ||
      !cuda_ok(c, cudaMemcpyAsync(st0, &run, sizeof(run), cudaMemcpyHostToDevice, c.stream), "adjoint") ||
      !cuda_ok(c, cudaMemcpyAsync(hist, hp.data(), sizeof(T *) * kDepth,
                                  cudaMemcpyHostToDevice, c.stream), "adjoint") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "adjoint"))
    return RISM3D_CUDA_ERROR;
  if (!cufft_ok(c, cufftSetStream(c.plan64, c.stream), "cufftSetStream")) return RISM3D_CUFFT_ERROR;
  if (F32 && !cufft_ok(c, cufftSetStream(c.plan32, c.stream), "cufftSetStream"))
    return RISM3D_CUFFT_ERROR;
  OzOp<double> L64(c, buf);
  OzOp<T> LT(c, bufT);
  // delta = q (fr - F^-1 fk) (into tmp), w = L delta (FP64)
  cudaMemsetAsync(buf, 0, sizeof(double2) * P * n, c.stream);
  k_fk_to_buf<<<gb, kThreads, 0, c.stream>>>(n, c.nx, c.ny, c.d_fkh, buf);
  if (cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)buf, (cufftDoubleComplex *)buf,
                   CUFFT_INVERSE) != CUFFT_SUCCESS)
    return RISM3D_CUFFT_ERROR;
  k_unpack<<<gb, kThreads, 0, c.stream>>>(n, 1, c.nx, c.ny, c.d_tw, 1.0 / c.vol, buf, Om);
  k_delta<<<gb, kThreads, 0, c.stream>>>(n, V, c.d_fr, Om, spq, tmp);
  c.launches += 3;
  int rc = L64.apply(V, tmp, w64, sp0, st0);
  if (rc != RISM3D_OK) return rc;
  if (F32) {
    k_cast<double, T><<<gt, kThreads, 0, c.stream>>>(tot, w64, w);
    c.launches += 1;
  }
  k_gprime<T><<<gt, kThreads, 0, c.stream>>>(tot, c.prm.closure, c.d_t, c.d_U, G);
  c.launches += 1;
  static const bool trace = getenv("RISM3D_TRACE") && getenv("RISM3D_TRACE")[0] == '1';
  const auto w0 = std::chrono::steady_clock::now();
  // Anderson-accelerated solve of G xi - (G - 1) L xi = (G - 1) w from xi = 0
  cudaMemsetAsync(xi, 0, sizeof(T) * tot, c.stream);
  cudaMemsetAsync(ys, 0, sizeof(T) * kDepth * tot, c.stream);
  cudaMemsetAsync(rs, 0, sizeof(T) * kDepth * tot, c.stream);
  std::vector<double> gram((size_t)kDepth * kDepth, 0.0), coef;
  double bnorm = -1.0, best = 1e300;
  int ns = 0, slot = 0, it = 0, since_best = 0;
  const double eta = 0.5, tol = SolveTol<T>::tol;
  const int maxit = 3000;
  bool stalled = false;
  for (; it < maxit; ++it) {
    rc = LT.apply(V, xi, Lxi, sp0, st0);
    if (rc != RISM3D_OK) return rc;
    const int nd = ns < kDepth ? ns + 1 : kDepth;      // filled slots incl. this one
    k_residual_dots<T><<<kDotBlocks, kThreads, 0, c.stream>>>(
        tot, G, w, Lxi, xi, eta, hist, slot, nd, ys + (size_t)slot * tot, dpart);
    k_sum_rows<<<kDepth + 1, kThreads, 0, c.stream>>>(dpart, kDotBlocks, dsum);
    c.launches += 2;
    double d[kDepth + 1];
    if (!cuda_ok(c, cudaMemcpyAsync(d, dsum, sizeof(d), cudaMemcpyDeviceToHost, c.stream), "adjoint") ||
        !cuda_ok(c, cudaStreamSynchronize(c.stream), "adjoint"))
      return RISM3D_CUDA_ERROR;
    if (!std::isfinite(d[kDepth])) { c.err = "adjoint solve diverged"; return RISM3D_DIVERGED; }
    const double rn = sqrt(d[kDepth]);
    if (bnorm < 0) bnorm = rn;                         // xi = 0: r = (G - 1) w
    if (rn <= tol * bnorm) break;
    // FP32: 200 steps without a 1 % gain end the solve at its rounding
    // floor when that is within 10x of the target
    if (rn < 0.99 * best) { best = rn; since_best = 0; }
    else if (F32 && ++since_best > 200 && rn <= 10.0 * tol * bnorm) { stalled = true; break; }
    for (int i = 0; i < kDepth; ++i)
      gram[(size_t)slot * kDepth + i] = gram[(size_t)i * kDepth + slot] = d[i];
    gram[(size_t)slot * kDepth + slot] = d[kDepth];
    ns = nd;
    anderson_coefficients(gram, ns, coef);
    Mix<T> mx{};
    mx.ns = ns;
    for (int a = 0; a < ns; ++a) {
      mx.ys[a] = ys + (size_t)a * tot;
      mx.c[a] = coef[a];
    }
    k_combine<T><<<gt, kThreads, 0, c.stream>>>(tot, mx, xi);
    c.launches += 1;
    slot = (slot + 1) % kDepth;
  }
  if (it == maxit) { c.err = "adjoint solve did not converge"; return RISM3D_NOT_CONVERGED; }
  const auto w1 = std::chrono::steady_clock::now();
  // weights from zeta; L xi is current (the loop leaves right after applyL)
  double *W = tmp;                              // delta no longer needed
  SiteW sv{};
  for (int v = 0; v < V; ++v) {
    sv.sig[v] = c.sigv[v]; sv.eps[v] = c.epsv[v]; sv.q[v] = c.qv[v] * c.cf_final; sv.rho[v] = c.rho[v];
  }
  k_weights<T><<<gb, kThreads, 0, c.stream>>>(n, V, c.d_g, c.d_h, G, xi, Lxi, w64, sv, W, Om);
  c.launches += 1;
  const double cc = kHartree * kBohr * kAvogadro;      // N_A kB T x ubeta
  // real-space part: atoms in tiles of 128, grid points split in chunks
  const int tiles = (A + kAtomsPerBlock - 1) / kAtomsPerBlock;
  const int want = std::max(1, 148 * 8 / tiles);
  long long chunk = (n + want - 1) / want;
  chunk = ((chunk + kPtsTile - 1) / kPtsTile) * kPtsTile;
  const int nchunk = (int)((n + chunk - 1) / chunk);
  long long chunk_k = (n / 2 + want - 1) / want;
  chunk_k = ((chunk_k + kPtsTile - 1) / kPtsTile) * kPtsTile;
  const int nchunk_k = (int)((n / 2 + chunk_k - 1) / chunk_k);
  double *part_r = S.get<double>((size_t)(nchunk + 1) * A * NOUT);
  double *part_k = S.get<double>((size_t)(nchunk_k + 1) * A * 4);
  double2 *ph = S.get<double2>((size_t)A * (c.nx + c.ny + c.nz));
  double2 *omh = S.get<double2>(n / 2);
  if (!part_r || !part_k || !ph || !omh) { c.err = "adjoint: out of device memory"; return RISM3D_CUDA_ERROR; }
  k_adjoint_r<V, F32><<<dim3(tiles, nchunk), kAtomsPerBlock, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], W, Om, c.d_atoms, A, sv, cc, chunk, part_r);
  double *sum_r = part_r + (size_t)nchunk * A * NOUT;
  k_sum_chunks<<<(A * NOUT + 255) / 256, 256, 0, c.stream>>>(part_r, nchunk, A, NOUT, sum_r);
  // k-space part: Omega^ = F[Omega]; -cc/2 (1/V) sum over all k = -cc/V Re over the owner half
  k_pack<<<gb, kThreads, 0, c.stream>>>(n, 1, c.nx, c.ny, c.d_tw, Om, buf);
  if (cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)buf, (cufftDoubleComplex *)buf,
                   CUFFT_FORWARD) != CUFFT_SUCCESS)
    return RISM3D_CUFFT_ERROR;
  k_forward_post<<<gb, kThreads, 0, c.stream>>>(n, c.nx, c.ny, c.dv, buf, omh);
  const long long L3 = (long long)A * (c.nx + c.ny + c.nz);
  k_phase_rows_adj<<<(unsigned)((L3 + 255) / 256), 256, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.prm.box[0], c.prm.box[1], c.prm.box[2], c.d_atoms, A, ph);
  k_adjoint_k<<<dim3(tiles, nchunk_k), kAtomsPerBlock, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.prm.box[0], c.prm.box[1], c.prm.box[2], omh, ph, c.d_atoms, A,
      -cc / c.vol, chunk_k, part_k);
  double *sum_k = part_k + (size_t)nchunk_k * A * 4;
  k_sum_chunks<<<(A * 4 + 255) / 256, 256, 0, c.stream>>>(part_k, nchunk_k, A, 4, sum_k);
  c.launches += 7;
  std::vector<double> hr((size_t)A * NOUT), hk((size_t)A * 4);
  if (!cuda_ok(c, cudaGetLastError(), "adjoint") ||
      !cuda_ok(c, cudaMemcpyAsync(hr.data(), sum_r, sizeof(double) * hr.size(), cudaMemcpyDeviceToHost, c.stream), "adjoint") ||
      !cuda_ok(c, cudaMemcpyAsync(hk.data(), sum_k, sizeof(double) * hk.size(), cudaMemcpyDeviceToHost, c.stream), "adjoint") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "adjoint"))
    return RISM3D_CUDA_ERROR;
  c.adj_steps = it;
  c.adj_stalled = stalled;
  if (trace) {
    const auto w2 = std::chrono::steady_clock::now();
    fprintf(stderr, "[rism3d] adjoint (%s): %d Anderson steps %.1f ms, back-projection %.1f ms%s\n",
            F32 ? "fp32" : "fp64", it,
            std::chrono::duration<double, std::milli>(w1 - w0).count(),
            std::chrono::duration<double, std::milli>(w2 - w1).count(),
            stalled ? " (stopped at the FP32 floor)" : "");
  }
  // the charge-up factor of the last stage is already in the site charges
  for (int u = 0; u < A; ++u) {
    const double *o = &hr[(size_t)u * NOUT], *kk = &hk[(size_t)u * 4];
    if (dq) dq[u] = o[0] * c.dv + kk[0];
    if (dsig) dsig[u] = o[1] * c.dv;
    if (deps) deps[u] = o[2] * c.dv;
    if (dR)
      for (int k = 0; k < 3; ++k) dR[3 * u + k] = o[3 + k] * c.dv + kk[1 + k];
  }
  return RISM3D_OK;
}

template <int V>
int adjoint_p(Context &c, int precision, double *dq, double *dsig, double *deps, double *dR) {
  return precision == RISM3D_MIXED ? adjoint_v<V, float>(c, dq, dsig, deps, dR)
                                   : adjoint_v<V, double>(c, dq, dsig, deps, dR);
}

}  // namespace

int compute_adjoint(Context &c, int precision, double *dq, double *dsig, double *deps,
                    double *dR) {
  if (c.nb != 1) { c.err = "gradients are for single-solute contexts"; return RISM3D_BAD_STATE; }
  switch (c.natv) {
    case 1: return adjoint_p<1>(c, precision, dq, dsig, deps, dR);
    case 2: return adjoint_p<2>(c, precision, dq, dsig, deps, dR);
    case 3: return adjoint_p<3>(c, precision, dq, dsig, deps, dR);
    case 4: return adjoint_p<4>(c, precision, dq, dsig, deps, dR);
    case 5: return adjoint_p<5>(c, precision, dq, dsig, deps, dR);
    case 6: return adjoint_p<6>(c, precision, dq, dsig, deps, dR);
    case 7: return adjoint_p<7>(c, precision, dq, dsig, deps, dR);
    case 8: return adjoint_p<8>(c, precision, dq, dsig, deps, dR);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

}  // namespace rism3d
