// RMDFT free-energy correction of the reference's -r option
// (cal_rmdft.cu:5-115): a functional of the converged OZ h with the solvent
// direct correlation c(k) (.cvk) and a hard-sphere reference fluid on site 0
// (the -r table: packing fraction, hard-sphere chi(k), weight w(k);
// solvent_read.cc:88-140, solvent_spline2.cu:7-103, excp_fd.cc:1-6):
//
//   xmu1 = -sum_v rho_v sum_r h_v
//   w_v  = F^-1[sum_v' (c_vv' - [v = v' = 0] chs rho_0 / rho_0) rho_v' H_v']
//   xmu2 = sum_v rho_v sum_r w_v,  xmu3 = sum_v rho_v sum_r w_v h_v
//   n    = rho_0 + F^-1[rho_0 w H_0]                     (weighted density)
//   f    = rho_0 ((h_0 + 1) fd(a n, n) - fd(pf, rho_0)),  a = pf / rho_0,
//          fd(p, d) = (4 - 2p) / (1 - p)^3 p / d
//   eda  = rho_0 sum_r ((F^-1[w F f] + e)(h_0 + 1) - e),  e = rho_0 fd(pf, rho_0) w(0)
//   SFE_RMDFT = N_A kB T (xmu1 + xmu2 + xmu3 / 2 - eda) dv
//
// The table file carries site 0 only; the other sites' hard-sphere tables
// are zero, so they add nothing to the density terms (the reference reads
// them from uninitialised arrays).  All transforms are the half-shifted FP64
// transform of the iteration, two sites per complex cuFFT; the splines are
// evaluated per k point with the bisection of splint.cc:4-20.  It runs once
// per solve, after the observables.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rism3d_impl.h"
#include "halfshift.cuh"

namespace rism3d {
namespace {

constexpr int kThr = 256;
constexpr int kRedBlocks = 148 * 8;

struct RmArgs {
  long long n;
  int nx, ny, nz;
  FastDiv fdx, fdy;
  double bx, by, bz;
  const double2 *tw;
  double dv, invvol;
  const double *ccoef;      // [ntab][V*V][4], knots dk (i + 1)
  int ntab;
  double dk;
  const double *k2;         // [ntab2] hard-sphere knots
  const double *hcoef;      // [ntab2][2][4]: chi_hs, w
  int ntab2;
  double rho[kMaxSites];
  double rho0, a, bex, ex;
};

__device__ __forceinline__ double spline_at(const double *o, double t) {
  return ((o[3] * t + o[2]) * t + o[1]) * t + o[0];
}

// |k| of grid point (ix, iy, iz) (set_g, initialize_g.cu:53-63)
__device__ __forceinline__ double kmag(const RmArgs &r, int ix, int iy, int iz) {
  const double kx = 2.0 * kPi * (ix - r.nx / 2.0 + 0.5) / r.bx;
  const double ky = 2.0 * kPi * (iy - r.ny / 2.0 + 0.5) / r.by;
  const double kz = 2.0 * kPi * (iz - r.nz / 2.0 + 0.5) / r.bz;
  return sqrt(kx * kx + ky * ky + kz * kz);
}

// splint.cc:9-16: bisection for the interval klo with knot(klo) <= x
template <typename Knot>
__device__ __forceinline__ int bisect(int np, double x, Knot knot) {
  int klo = 0, khi = np - 1;
  while (khi - klo > 1) {
    const int k = (khi + klo) >> 1;
    if (knot(k) > x) khi = k; else klo = k;
  }
  return klo;
}

__device__ __forceinline__ void owner_index(const RmArgs &r, long long j, int &ix, int &iy,
                                            int &iz) {
  const unsigned q = r.fdx.div((unsigned)j);
  ix = (int)(j - (long long)q * r.nx);
  iz = (int)r.fdy.div(q);
  iy = (int)(q - (unsigned)iz * r.ny);
}

__device__ __forceinline__ void hard_sphere_at(const RmArgs &r, double kk, double &chs,
                                               double &w) {
  const int h0 = bisect(r.ntab2, kk, [&](int k) { return r.k2[k]; });
  const double th = kk - r.k2[h0];
  chs = spline_at(r.hcoef + (size_t)h0 * 8, th);
  w = spline_at(r.hcoef + (size_t)h0 * 8 + 4, th);
}

// k space, first pass (cal_dwork and rho0wfkhk on one mirror pair): the
// forward-transformed site pairs H in buf become W = (c - chs) rho H (pairs,
// in place) and D = rho_0 w H_0 (one packed real function, in buf2), both
// repacked for the inverse transform
template <int V>
__global__ void __launch_bounds__(kThr) k_rm_k1(RmArgs r, double2 *buf, double2 *buf2) {
  constexpr int P = (V + 1) / 2;
  const long long n = r.n, nh = n / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nh;
       j += (long long)gridDim.x * blockDim.x) {
    const long long jm = n - 1 - j;
    int ix, iy, iz;
    owner_index(r, j, ix, iy, iz);
    const int dir = ((ix + iy + iz) & 1) ? -1 : 1;
    const double sc = r.dv * 0.5 * dir;
    double2 F[V];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const double2 y = buf[(size_t)p * n + j], ym = buf[(size_t)p * n + jm];
      F[2 * p] = make_double2(sc * (y.x - ym.x), sc * (y.y + ym.y));
      if (2 * p + 1 < V) F[2 * p + 1] = make_double2(sc * (y.y - ym.y), -sc * (y.x + ym.x));
    }
    const double kk = kmag(r, ix, iy, iz);
    const int k0 = bisect(r.ntab, kk, [&](int k) { return r.dk * (k + 1); });
    const double t = kk - r.dk * (k0 + 1);
    double chs, w;
    hard_sphere_at(r, kk, chs, w);
    double2 W[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double wr = 0.0, wi = 0.0;
#pragma unroll
      for (int u = 0; u < V; ++u) {
        double cvu = spline_at(r.ccoef + ((size_t)k0 * V * V + v * V + u) * 4, t);
        if (v == 0 && u == 0) cvu -= chs * (r.rho0 / r.rho[0]);
        wr += F[u].x * cvu * r.rho[u];
        wi += F[u].y * cvu * r.rho[u];
      }
      W[v] = make_double2(wr, wi);
    }
    const double d = dir;
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const double2 ha = W[2 * p];
      const double2 hb = (2 * p + 1 < V) ? W[2 * p + 1] : make_double2(0.0, 0.0);
      buf[(size_t)p * n + j] = make_double2(d * (ha.x - hb.y), d * (ha.y + hb.x));
      buf[(size_t)p * n + jm] = make_double2(-d * (ha.x + hb.y), -d * (hb.x - ha.y));
    }
    const double rw = r.rho0 * w;
    const double2 D = make_double2(rw * F[0].x, rw * F[0].y);
    buf2[j] = make_double2(d * D.x, d * D.y);
    buf2[jm] = make_double2(-d * D.x, d * D.y);
  }
}

// k space, second pass (wfka): F[f] times w(|k|) on one packed real function
__global__ void __launch_bounds__(kThr) k_rm_k2(RmArgs r, double2 *buf2) {
  const long long n = r.n, nh = n / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nh;
       j += (long long)gridDim.x * blockDim.x) {
    const long long jm = n - 1 - j;
    int ix, iy, iz;
    owner_index(r, j, ix, iy, iz);
    const int dir = ((ix + iy + iz) & 1) ? -1 : 1;
    const double sc = r.dv * 0.5 * dir;
    const double2 y = buf2[j], ym = buf2[jm];
    const double2 F = make_double2(sc * (y.x - ym.x), sc * (y.y + ym.y));
    double chs, w;
    hard_sphere_at(r, kmag(r, ix, iy, iz), chs, w);
    const double d = dir;
    buf2[j] = make_double2(d * w * F.x, d * w * F.y);
    buf2[jm] = make_double2(-d * w * F.x, d * w * F.y);
  }
}

template <int NS>
__device__ __forceinline__ void block_sums(double (&acc)[NS], double *part) {
  __shared__ double red[kThr / 32][NS];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][i] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < NS) {
    double s = 0.0;
    for (int w = 0; w < kThr / 32; ++w) s += red[w][threadIdx.x];
    part[(size_t)blockIdx.x * NS + threadIdx.x] = s;
  }
}

// real space after the first inverse: the xmu1..3 sums, the weighted
// density n, and f (rho0guvfmbex) packed into buf2 for the forward transform
template <int V>
__global__ void __launch_bounds__(kThr)
k_rm_r1(RmArgs r, const double2 *buf, double2 *buf2, const double *h, double *part) {
  constexpr int P = (V + 1) / 2;
  const long long n = r.n;
  double acc[3] = {0.0, 0.0, 0.0};
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    double2 tw;
    point_dir_dkf(j, r.nx, r.ny, r.tw, dir, tw);
    const double s = r.invvol * dir;
    double wv[2 * P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const double2 z = buf[(size_t)p * n + j];
      wv[2 * p] = s * (z.x * tw.x + z.y * tw.y);
      wv[2 * p + 1] = s * (z.y * tw.x - z.x * tw.y);
    }
    double h0 = 0.0;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double hv = h[(size_t)v * n + j];
      if (v == 0) h0 = hv;
      acc[0] += r.rho[v] * hv;
      acc[1] += r.rho[v] * wv[v];
      acc[2] += r.rho[v] * wv[v] * hv;
    }
    const double2 z = buf2[j];
    const double dens = s * (z.x * tw.x + z.y * tw.y) + r.rho0;
    const double pf = r.a * dens;
    const double fd = (4.0 - 2.0 * pf) / ((1.0 - pf) * (1.0 - pf) * (1.0 - pf)) * (pf / dens);
    const double f = r.rho0 * ((h0 + 1.0) * fd - r.bex);
    buf2[j] = make_double2(dir * (f * tw.x), dir * (f * tw.y));
  }
  block_sums<3>(acc, part);
}

// real space after the last inverse: the eda sum of site 0
__global__ void __launch_bounds__(kThr)
k_rm_r2(RmArgs r, const double2 *buf2, const double *h, double *part) {
  const long long n = r.n;
  double acc[1] = {0.0};
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    double2 tw;
    point_dir_dkf(j, r.nx, r.ny, r.tw, dir, tw);
    const double2 z = buf2[j];
    const double g = r.invvol * dir * (z.x * tw.x + z.y * tw.y);
    acc[0] += (g + r.ex) * (h[j] + 1.0) - r.ex;
  }
  block_sums<1>(acc, part);
}

double fd_bulk(double pf, double dens) {            // excp_fd.cc:1-6
  return (4.0 - 2.0 * pf) / ((1.0 - pf) * (1.0 - pf) * (1.0 - pf)) * (pf / dens);
}

template <int V>
int rmdft_v(Context &c) {
  const long long n = c.n;
  if (!c.plan1) {
    int dims[3] = {c.nz, c.ny, c.nx};
    const int np = (int)n;
    if (!cufft_ok(c, cufftPlanMany(&c.plan1, 3, dims, nullptr, 1, np, nullptr, 1, np,
                                   CUFFT_Z2Z, 1), "cufftPlanMany RMDFT"))
      return RISM3D_CUFFT_ERROR;
  }
  if (!cufft_ok(c, cufftSetStream(c.plan1, c.stream), "cufftSetStream") ||
      !cufft_ok(c, cufftSetStream(c.plan64, c.stream), "cufftSetStream"))
    return RISM3D_CUFFT_ERROR;
  double2 *buf = c.d_buf, *buf2 = nullptr;      // the solve is finished: buf is free
  double *part = nullptr;
  if (!cuda_ok(c, pool_alloc(c, (void **)&buf2, sizeof(double2) * n), "RMDFT buffer") ||
      !cuda_ok(c, pool_alloc(c, (void **)&part, sizeof(double) * kRedBlocks * 4), "RMDFT sums"))
    return RISM3D_CUDA_ERROR;
  RmArgs r{};
  r.n = n; r.nx = c.nx; r.ny = c.ny; r.nz = c.nz;
  r.fdx = FastDiv((unsigned)c.nx); r.fdy = FastDiv((unsigned)c.ny);
  r.bx = c.prm.box[0]; r.by = c.prm.box[1]; r.bz = c.prm.box[2];
  r.tw = c.d_tw; r.dv = c.dv; r.invvol = 1.0 / c.vol;
  r.ccoef = c.d_rm_ccoef; r.ntab = c.chi.ntab; r.dk = c.chi.dk;
  r.k2 = c.d_rm_k2; r.hcoef = c.d_rm_hcoef; r.ntab2 = c.rm_ntab2;
  for (int v = 0; v < V; ++v) r.rho[v] = c.rho[v];
  r.rho0 = c.rho[0];
  r.a = c.rm_pfhs / r.rho0;
  r.bex = fd_bulk(c.rm_pfhs, r.rho0);
  r.ex = r.rho0 * r.bex * c.rm_w0;
  const int gk = (int)std::min<long long>((n / 2 + kThr - 1) / kThr, 148 * 16);
  bool fft_failed = false;
  auto fft = [&](cufftHandle pl, double2 *a, int d) {
    const bool good = cufft_ok(
        c, cufftExecZ2Z(pl, (cufftDoubleComplex *)a, (cufftDoubleComplex *)a, d), "RMDFT transform");
    fft_failed = fft_failed || !good;
    return good;
  };
  k_pack<<<kRedBlocks, kThr, 0, c.stream>>>(n, V, c.nx, c.ny, c.d_tw, c.d_h, buf);
  bool ok = fft(c.plan64, buf, CUFFT_FORWARD);
  if (ok) {
    k_rm_k1<V><<<gk, kThr, 0, c.stream>>>(r, buf, buf2);
    ok = fft(c.plan64, buf, CUFFT_INVERSE) && fft(c.plan1, buf2, CUFFT_INVERSE);
  }
  if (ok) {
    k_rm_r1<V><<<kRedBlocks, kThr, 0, c.stream>>>(r, buf, buf2, c.d_h, part);
    ok = fft(c.plan1, buf2, CUFFT_FORWARD);
  }
  if (ok) {
    k_rm_k2<<<gk, kThr, 0, c.stream>>>(r, buf2);
    ok = fft(c.plan1, buf2, CUFFT_INVERSE);
  }
  if (ok) k_rm_r2<<<kRedBlocks, kThr, 0, c.stream>>>(r, buf2, c.d_h, part + kRedBlocks * 3);
  c.launches += 5;
  std::vector<double> hp((size_t)kRedBlocks * 4);
  ok = ok && cuda_ok(c, cudaGetLastError(), "RMDFT") &&
       cuda_ok(c, cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(),
                                  cudaMemcpyDeviceToHost, c.stream), "RMDFT sums");
  cudaFreeAsync(buf2, c.stream);
  cudaFreeAsync(part, c.stream);
  if (!ok || !cuda_ok(c, cudaStreamSynchronize(c.stream), "RMDFT"))
    return fft_failed ? RISM3D_CUFFT_ERROR : RISM3D_CUDA_ERROR;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = 0; b < kRedBlocks; ++b)
    for (int k = 0; k < 3; ++k) s[k] += hp[(size_t)b * 3 + k];
  for (int b = 0; b < kRedBlocks; ++b) s[3] += hp[(size_t)kRedBlocks * 3 + b];
  const double dft = (-s[0] + s[1] + 0.5 * s[2] - r.rho[0] * s[3]) * c.dv;
  c.res.sfe_rmdft = kAvogadro * kBoltzmann * c.temper * dft;
  return RISM3D_OK;
}

}  // namespace

int compute_rmdft(Context &c) {
  c.res.sfe_rmdft = 0.0;
  if (!c.rmdft || c.nb != 1) return RISM3D_OK;
  switch (c.natv) {
    case 1: return rmdft_v<1>(c);
    case 2: return rmdft_v<2>(c);
    case 3: return rmdft_v<3>(c);
    case 4: return rmdft_v<4>(c);
    case 5: return rmdft_v<5>(c);
    case 6: return rmdft_v<6>(c);
    case 7: return rmdft_v<7>(c);
    case 8: return rmdft_v<8>(c);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

}  // namespace rism3d
