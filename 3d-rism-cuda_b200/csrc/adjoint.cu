// Adjoint gradients of the solvation free energy SFE_SC with respect to the
// solute parameters (charges, LJ sigma and epsilon, positions).
//
// For the KH and HNC closures the reference's free-energy expression
// (cal_exchem.cu:55-122) is stationary with respect to the correlation
// functions at the solution, so the derivative with respect to any solute
// parameter p only sees the explicit potential:
//
//   dSFE/dp = N_A kB T sum_v rho_v dv sum_r g_v(r) d(beta u_v(r))/dp
//
// with beta u_v = beta u_LJ,v + q_v beta e (cal_LJ.cu:57-71,
// cal_Coulomb.cu:109-121).  The kernel back-propagates w_v(r) = rho_v g_v(r)
// through the potential-grid computation: one atom per thread, grid points
// streamed through shared memory, and every pair term recomputed from the
// atom parameters instead of being stored.  Per pair it uses the same
// rules as the forward kernel: r^2 clamped at 1e-4 for LJ (no positional
// derivative inside the clamp) and no Coulomb term below r = 1e-5.
#include <cmath>
#include <vector>

#include "rism3d_impl.h"

namespace rism3d {
namespace {

constexpr int kAtomsPerBlock = 128;
constexpr int kPtsTile = 128;
constexpr int NOUT = 6;   // dq, dsigma, deps, dRx, dRy, dRz

struct SiteW {
  double sig[kMaxSites], eps[kMaxSites], q[kMaxSites], rho[kMaxSites];
};

template <int V>
__global__ void __launch_bounds__(kAtomsPerBlock)
k_adjoint(int nx, int ny, int nz, double drx, double dry, double drz,
          const double *__restrict__ g, const double *__restrict__ atoms, int natom,
          SiteW sv, double cc, long long chunk, double *part) {
  __shared__ double4 pp[kPtsTile];
  __shared__ double pw[V][kPtsTile];       // rho_v g_v at the point
  const long long n = (long long)nx * ny * nz;
  const int ia = blockIdx.x * kAtomsPerBlock + threadIdx.x;
  const bool live = ia < natom;
  double X = 0, Y = 0, Z = 0, qu = 0, su = 0, eu = 0;
  if (live) {
    const double *a = atoms + 8 * (size_t)ia;
    X = a[0]; Y = a[1]; Z = a[2]; qu = a[3]; su = a[4]; eu = a[5];
  }
  double sg[V], sg2[V], euv[V], deps_fac[V], qc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    sg[v] = (su + sv.sig[v]) * 0.5;               // cal_LJ.cu:28
    sg2[v] = sg[v] * sg[v];
    euv[v] = sqrt(eu * sv.eps[v]);               // cal_LJ.cu:29
    deps_fac[v] = eu > 0.0 ? 0.5 * euv[v] / eu : 0.0;   // d eps_uv / d eps_u
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
        pp[i] = make_double4((ix - nx / 2) * drx, (iy - ny / 2) * dry, (iz - nz / 2) * drz, 0.0);
#pragma unroll
        for (int v = 0; v < V; ++v) pw[v][i] = sv.rho[v] * g[(size_t)v * n + j];
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
      const bool clamped = r2 < 1.0e-4;
      const double ir2 = clamped ? 1.0e4 : 1.0 / r2;
      const double ri = r2 > 0.0 ? rsqrt(r2) : 0.0;
      const bool coul = r2 * ri >= 1.0e-5;
      double wsum_q = 0.0, fr = 0.0;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double w = pw[v][i];
        const double s2 = sg2[v] * ir2;
        const double s6 = s2 * s2 * s2, s12 = s6 * s6;
        // d/d sigma_u of 4 eps (s^12 - s^6): (24 eps/sigma_uv)(2 s^12 - s^6) / 2
        acc[1] += w * 12.0 * euv[v] / sg[v] * (2.0 * s12 - s6);
        // d/d eps_u: 4 (s^12 - s^6) d eps_uv / d eps_u
        acc[2] += w * 4.0 * (s12 - s6) * deps_fac[v];
        // d/d R_u: 24 eps (2 s^12 - s^6) / r^2 (r - R_u)  (cal_grad.cu:73)
        if (!clamped) fr += w * 24.0 * euv[v] * (2.0 * s12 - s6) * ir2;
        if (coul) wsum_q += w * qc[v];
      }
      if (coul) {
        acc[0] += wsum_q * ri;                     // d/d q_u of q_u q_v cc / r
        fr += wsum_q * qu * ri * ri * ri;          // q_u q_v cc (r - R_u) / r^3
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

__global__ void k_adjoint_sum(const double *part, int nchunk, int natom, double *out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= natom * NOUT) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += part[(size_t)c * natom * NOUT + idx];
  out[idx] = s;
}

template <int V>
int adjoint_v(Context &c, double *dq, double *dsig, double *deps, double *dR) {
  const int A = c.natom;
  const int tiles = (A + kAtomsPerBlock - 1) / kAtomsPerBlock;
  int nchunk = (148 * 8 + tiles - 1) / tiles;
  long long chunk = (c.n + nchunk - 1) / nchunk;
  chunk = ((chunk + kPtsTile - 1) / kPtsTile) * kPtsTile;
  nchunk = (int)((c.n + chunk - 1) / chunk);
  double *part = nullptr;
  const size_t need = (size_t)nchunk * A * NOUT + (size_t)A * NOUT;
  if (!cuda_ok(c, cudaMallocAsync(&part, sizeof(double) * need, c.stream), "adjoint scratch"))
    return RISM3D_CUDA_ERROR;
  SiteW sv{};
  for (int v = 0; v < V; ++v) {
    sv.sig[v] = c.sigv[v]; sv.eps[v] = c.epsv[v]; sv.q[v] = c.qv[v]; sv.rho[v] = c.rho[v];
  }
  const double cc = kHartree * kBohr * kAvogadro;      // N_A kB T * ubeta
  k_adjoint<V><<<dim3(tiles, nchunk), kAtomsPerBlock, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_g, c.d_atoms, A, sv, cc, chunk, part);
  double *sum = part + (size_t)nchunk * A * NOUT;
  k_adjoint_sum<<<(A * NOUT + 255) / 256, 256, 0, c.stream>>>(part, nchunk, A, sum);
  c.launches += 2;
  std::vector<double> h((size_t)A * NOUT);
  bool ok = cuda_ok(c, cudaGetLastError(), "adjoint") &&
            cuda_ok(c, cudaMemcpyAsync(h.data(), sum, sizeof(double) * h.size(),
                                       cudaMemcpyDeviceToHost, c.stream), "adjoint") &&
            cuda_ok(c, cudaFreeAsync(part, c.stream), "adjoint") &&
            cuda_ok(c, cudaStreamSynchronize(c.stream), "adjoint");
  if (!ok) return RISM3D_CUDA_ERROR;
  // charges enter the closure as q cf; gradients are for the final stage
  for (int u = 0; u < A; ++u) {
    const double *o = &h[(size_t)u * NOUT];
    if (dq) dq[u] = o[0] * c.dv * c.cf_final;
    if (dsig) dsig[u] = o[1] * c.dv;
    if (deps) deps[u] = o[2] * c.dv;
    if (dR)
      for (int k = 0; k < 3; ++k) dR[3 * u + k] = o[3 + k] * c.dv;
  }
  return RISM3D_OK;
}

}  // namespace

int compute_adjoint(Context &c, double *dq, double *dsig, double *deps, double *dR) {
  switch (c.natv) {
    case 1: return adjoint_v<1>(c, dq, dsig, deps, dR);
    case 2: return adjoint_v<2>(c, dq, dsig, deps, dR);
    case 3: return adjoint_v<3>(c, dq, dsig, deps, dR);
    case 4: return adjoint_v<4>(c, dq, dsig, deps, dR);
    case 5: return adjoint_v<5>(c, dq, dsig, deps, dR);
    case 6: return adjoint_v<6>(c, dq, dsig, deps, dR);
    case 7: return adjoint_v<7>(c, dq, dsig, deps, dR);
    case 8: return adjoint_v<8>(c, dq, dsig, deps, dR);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

}  // namespace rism3d
