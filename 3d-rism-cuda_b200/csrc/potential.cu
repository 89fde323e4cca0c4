// Potential grids for one solute (reference: cal_potential.cu:3-14,
// cal_LJ.cu:4-72, cal_Coulomb.cu:8-155), one fused pass over the real-space
// grid and one over the owner half of k space.
//
// Real space, per grid point r and solvent site v (beta = 1/(N_A kB T) for
// LJ, ubeta = hartree*bohr/(kB T) for Coulomb):
//   u_v(r)  = beta  sum_u 4 eps_uv [(s/r)^12 - (s/r)^6], r^2 clamped >= 1e-4
//   fr(r)   = ubeta sum_u q_u (1 - e^-r)/r   (r < 1e-5: + q_u)
//   esr(r)  = ubeta sum_u q_u e^-r / r       (r < 1e-5: - q_u)
// esr = e - fr is the short-range Coulomb part: the closure only ever sees
// -q_v cf e + t = -q_v cf esr + t_SR with t_SR = t - q_v cf fr, so e is not
// stored (e = esr + fr when a caller asks for it).
// k space, on the owner half (iz < nz/2; the other half is its conjugate):
//   fk(k)   = ubeta sum_u 4 pi q_u e^{-ik.R_u} / (k^2 (k^2 + 1))
//
// Atoms are staged through shared memory in tiles (every thread of a block
// reads the same atom: broadcast); all sites are produced in one pass.
#include "rism3d_impl.h"

namespace rism3d {
namespace {

constexpr int kTile = 128;
constexpr int kThreads = 256;

struct SiteLJ {
  double sig[kMaxSites];
  double eps[kMaxSites];
};

template <int V>
__global__ void __launch_bounds__(kThreads)
k_potential_r(int nx, int ny, int nz, double drx, double dry, double drz,
              const double *__restrict__ atoms, int natom, SiteLJ sites,
              double ikbt, double ubeta, double *__restrict__ u,
              double *__restrict__ esr, double *__restrict__ fr) {
  __shared__ double sx[kTile], sy[kTile], sz[kTile], sq[kTile];
  __shared__ double ss2[V][kTile], se4[V][kTile];
  const long long n = (long long)nx * ny * nz;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double rx = 0, ry = 0, rz = 0;
  if (j < n) {
    int ix = (int)(j % nx);
    long long r = j / nx;
    int iy = (int)(r % ny), iz = (int)(r / ny);
    rx = (ix - nx / 2) * drx;   // cal_LJ.cu:54-56 (integer n/2)
    ry = (iy - ny / 2) * dry;
    rz = (iz - nz / 2) * drz;
  }
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  double afr = 0.0, aes = 0.0;
  const double cut2 = 1.0e-4;   // (1e-2)^2, cal_LJ.cu:11-12
  for (int t0 = 0; t0 < natom; t0 += kTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
      int ia = t0 + i;
      if (ia < natom) {
        const double *a = atoms + 8 * (size_t)ia;
        sx[i] = a[0]; sy[i] = a[1]; sz[i] = a[2]; sq[i] = a[3];
#pragma unroll
        for (int v = 0; v < V; ++v) {
          double s = (a[4] + sites.sig[v]) * 0.5;      // cal_LJ.cu:28
          ss2[v][i] = s * s;
          se4[v][i] = 4.0 * sqrt(a[5] * sites.eps[v]) * ikbt;  // :29, :38
        }
      } else {
        sx[i] = sy[i] = sz[i] = 1.0e30; sq[i] = 0.0;
#pragma unroll
        for (int v = 0; v < V; ++v) { ss2[v][i] = 0.0; se4[v][i] = 0.0; }
      }
    }
    __syncthreads();
    const int m = min(kTile, natom - t0);
    for (int i = 0; i < m; ++i) {
      double dx = rx - sx[i], dy = ry - sy[i], dz = rz - sz[i];
      double r2 = dx * dx + dy * dy + dz * dz;
      double r2c = r2 < cut2 ? cut2 : r2;
      double ir2 = 1.0 / r2c;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        double s2 = ss2[v][i] * ir2;
        double s6 = s2 * s2 * s2;
        acc[v] += se4[v][i] * s6 * (s6 - 1.0);
      }
      double ra = sqrt(r2);
      if (ra >= 1.0e-5) {                 // cal_Coulomb.cu:114-120
        double qr = sq[i] / ra;
        double em1 = expm1(-ra);          // e^-r - 1
        afr -= qr * em1;                  // q (1 - e^-r) / r
        aes += qr * (em1 + 1.0);          // q e^-r / r
      } else {
        afr += sq[i];
        aes -= sq[i];
      }
    }
  }
  if (j < n) {
#pragma unroll
    for (int v = 0; v < V; ++v) u[(size_t)v * n + j] = acc[v];
    fr[j] = afr * ubeta;
    esr[j] = aes * ubeta;
  }
}

// fk on the owner half j < N/2 (cal_Coulomb.cu:125-149; k from set_g,
// initialize_g.cu:58-60).
__global__ void __launch_bounds__(kThreads)
k_potential_k(int nx, int ny, int nz, double bx, double by, double bz,
              const double *__restrict__ atoms, int natom, double ubeta,
              double2 *__restrict__ fkh) {
  __shared__ double sx[kTile], sy[kTile], sz[kTile], sq[kTile];
  const long long nh = (long long)nx * ny * nz / 2;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double kx = 0, ky = 0, kz = 0;
  if (j < nh) {
    int ix = (int)(j % nx);
    long long r = j / nx;
    int iy = (int)(r % ny), iz = (int)(r / ny);
    kx = 2.0 * kPi * (ix - nx / 2.0 + 0.5) / bx;
    ky = 2.0 * kPi * (iy - ny / 2.0 + 0.5) / by;
    kz = 2.0 * kPi * (iz - nz / 2.0 + 0.5) / bz;
  }
  double rk2 = kx * kx + ky * ky + kz * kz;
  double rk4i = 1.0 / (rk2 * (rk2 + 1.0));
  double re = 0.0, im = 0.0;
  for (int t0 = 0; t0 < natom; t0 += kTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
      int ia = t0 + i;
      if (ia < natom) {
        const double *a = atoms + 8 * (size_t)ia;
        sx[i] = a[0]; sy[i] = a[1]; sz[i] = a[2]; sq[i] = a[3];
      } else {
        sx[i] = sy[i] = sz[i] = 0.0; sq[i] = 0.0;
      }
    }
    __syncthreads();
    const int m = min(kTile, natom - t0);
    for (int i = 0; i < m; ++i) {
      double ruk = kx * sx[i] + ky * sy[i] + kz * sz[i];
      double s, c;
      sincos(ruk, &s, &c);
      double tmp = 4.0 * kPi * sq[i];
      re += tmp * c;
      im -= tmp * s;
    }
  }
  if (j < nh) fkh[j] = make_double2(re * rk4i * ubeta, im * rk4i * ubeta);
}

template <int V>
void launch_r(Context &c, const SiteLJ &sl, double ikbt, double ubeta) {
  long long blocks = (c.n + kThreads - 1) / kThreads;
  k_potential_r<V><<<(unsigned)blocks, kThreads, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_atoms, c.natom, sl,
      ikbt, ubeta, c.d_u, c.d_e, c.d_fr);
}

}  // namespace

int launch_potential_r(Context &c) {
  SiteLJ sl{};
  for (int v = 0; v < c.natv; ++v) { sl.sig[v] = c.sigv[v]; sl.eps[v] = c.epsv[v]; }
  const double ikbt = 1.0 / (kAvogadro * kBoltzmann * c.temper);
  const double ubeta = kHartree * kBohr / (kBoltzmann * c.temper);
  switch (c.natv) {
    case 1: launch_r<1>(c, sl, ikbt, ubeta); break;
    case 2: launch_r<2>(c, sl, ikbt, ubeta); break;
    case 3: launch_r<3>(c, sl, ikbt, ubeta); break;
    case 4: launch_r<4>(c, sl, ikbt, ubeta); break;
    case 5: launch_r<5>(c, sl, ikbt, ubeta); break;
    case 6: launch_r<6>(c, sl, ikbt, ubeta); break;
    case 7: launch_r<7>(c, sl, ikbt, ubeta); break;
    case 8: launch_r<8>(c, sl, ikbt, ubeta); break;
    default: return RISM3D_UNSUPPORTED_SHAPE;
  }
  c.launches += 1;
  return RISM3D_OK;
}

int compute_potentials(Context &c) {
  SiteLJ sl{};
  for (int v = 0; v < c.natv; ++v) { sl.sig[v] = c.sigv[v]; sl.eps[v] = c.epsv[v]; }
  const double ikbt = 1.0 / (kAvogadro * kBoltzmann * c.temper);  // cal_LJ.cu:38
  const double ubeta = kHartree * kBohr / (kBoltzmann * c.temper); // cal_Coulomb.cu:34
  switch (c.natv) {
    case 1: launch_r<1>(c, sl, ikbt, ubeta); break;
    case 2: launch_r<2>(c, sl, ikbt, ubeta); break;
    case 3: launch_r<3>(c, sl, ikbt, ubeta); break;
    case 4: launch_r<4>(c, sl, ikbt, ubeta); break;
    case 5: launch_r<5>(c, sl, ikbt, ubeta); break;
    case 6: launch_r<6>(c, sl, ikbt, ubeta); break;
    case 7: launch_r<7>(c, sl, ikbt, ubeta); break;
    case 8: launch_r<8>(c, sl, ikbt, ubeta); break;
    default: c.err = "unsupported number of solvent sites"; return RISM3D_UNSUPPORTED_SHAPE;
  }
  if (!cuda_ok(c, cudaGetLastError(), "k_potential_r")) return RISM3D_CUDA_ERROR;
  long long blocks = (c.n / 2 + kThreads - 1) / kThreads;
  k_potential_k<<<(unsigned)blocks, kThreads, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.prm.box[0], c.prm.box[1], c.prm.box[2], c.d_atoms,
      c.natom, ubeta, c.d_fkh);
  if (!cuda_ok(c, cudaGetLastError(), "k_potential_k")) return RISM3D_CUDA_ERROR;
  c.launches += 2;
  return RISM3D_OK;
}

}  // namespace rism3d
