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
//
// Mixed-precision contexts (MIX) evaluate the LJ pair terms in FP32 with
// per-tile FP64 accumulation and the e^-r factor beyond 20 A in FP32 (there
// it is below 2e-9, so fr keeps FP64 accuracy); fr itself, 1/r and the
// sums stay FP64.
#include <algorithm>

#include "rism3d_impl.h"

namespace rism3d {
namespace {

constexpr int kTile = 128;
constexpr int kThreads = 256;

struct SiteLJ {
  double sig[kMaxSites];
  double eps[kMaxSites];
};

// e^-x in FP64 for 0 <= x <= 40 (the e^-r factor of the split Coulomb
// terms), branch-free: Cody-Waite range reduction x = k ln2 + f with k the
// integer nearest x / ln2, so |f| <= ln2 / 2 (ln2 split into a 39-bit head,
// exact in k ln2 for |k| < 2^13, and the rest), then e^-f from its Taylor
// series to degree 13 (truncation below 5e-18 relative for |f| <= ln2 / 2),
// and the factor 2^-k written into the exponent field.
__device__ __forceinline__ double exp_neg(double x) {
  constexpr double kLn2Hi = 0.6931471805592082, kLn2Lo = 7.371002565167799e-13;
  constexpr double kInvLn2 = 1.4426950408889634;
  const double k = rint(x * kInvLn2);
  const double g = -fma(-k, kLn2Lo, fma(-k, kLn2Hi, x));      // -f
  double p = 1.0 / 6227020800.0;                                // 1/13!
  p = fma(p, g, 1.0 / 479001600.0);
  p = fma(p, g, 1.0 / 39916800.0);
  p = fma(p, g, 1.0 / 3628800.0);
  p = fma(p, g, 1.0 / 362880.0);
  p = fma(p, g, 1.0 / 40320.0);
  p = fma(p, g, 1.0 / 5040.0);
  p = fma(p, g, 1.0 / 720.0);
  p = fma(p, g, 1.0 / 120.0);
  p = fma(p, g, 1.0 / 24.0);
  p = fma(p, g, 1.0 / 6.0);
  p = fma(p, g, 0.5);
  p = fma(p, g, 1.0);
  p = fma(p, g, 1.0);
  return p * __longlong_as_double((long long)(1023 - (int)k) << 52);
}

// Real-space grids.  A block covers a brick of 8 x 8 x 8 grid points and
// each warp a compact 8 x 4 x 2 sub-brick (4 x 2 x 1 A at 0.5 A spacing);
// each thread owns two neighbouring points along x (the atom tile read once
// for both).  With compact warps the distance tests below (the e^-r branch,
// the 40 A bound, the r^2 clamp) take the same side for nearly every lane,
// where a warp along one x row (64 points, 32 A) diverged on every atom
// within about 40 A.  Per (point, atom) one refined reciprocal square root
// gives 1/r, r and 1/r^2.  Beyond 40 A the factor e^-r (< 4.3e-18) is
// dropped: there the reference's q (1 - e^-r) / r already rounds to q / r.
constexpr int kPts = 2;
constexpr int kBrick = 8;        // brick edge (points); x: 4 threads x kPts

template <int V, bool MIX>
__global__ void __launch_bounds__(kThreads)
k_potential_r(int nx, int ny, int nz, int bricks_x, int bricks_y, double drx, double dry,
              double drz, const double *__restrict__ atoms_all, const int *__restrict__ aoff,
              const int *__restrict__ acnt, SiteLJ sites, double ikbt, double ubeta,
              double *__restrict__ u, double *__restrict__ esr, double *__restrict__ fr) {
  __shared__ double4 sa[kTile];           // x y z q
  __shared__ double2 sl[V][kTile];        // sigma_uv^2, 4 eps_uv / kBT
  __shared__ float2 slf[V][kTile];        // the same in FP32 (MIX)
  const long long n = (long long)nx * ny * nz;
  // solute blockIdx.y: its atoms and its [V][N] / [N] grids
  const int sb = blockIdx.y;
  const double *__restrict__ atoms = atoms_all + 8 * (size_t)aoff[sb];
  const int natom = acnt[sb];
  u += (size_t)sb * V * n;
  esr += (size_t)sb * n;
  fr += (size_t)sb * n;
  // brick of this block, sub-brick of this warp, points of this thread
  const int b = blockIdx.x;
  const int bxi = b % bricks_x, byz = b / bricks_x;
  const int byi = byz % bricks_y, bzi = byz / bricks_y;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ix = bxi * kBrick + (lane & 3) * kPts;
  const int iy = byi * kBrick + (w & 1) * 4 + ((lane >> 2) & 3);
  const int iz = bzi * kBrick + (w >> 1) * 2 + (lane >> 4);
  // grid sizes are even, so ix < nx covers both points of the thread
  const bool live = ix < nx && iy < ny && iz < nz;
  double rx[kPts];
  for (int k = 0; k < kPts; ++k) rx[k] = (ix + k - nx / 2) * drx;   // cal_LJ.cu:54-56
  const double ry = (iy - ny / 2) * dry, rz = (iz - nz / 2) * drz;
  double acc[kPts][V], afr[kPts], aes[kPts];
#pragma unroll
  for (int k = 0; k < kPts; ++k) {
    afr[k] = aes[k] = 0.0;
#pragma unroll
    for (int v = 0; v < V; ++v) acc[k][v] = 0.0;
  }
  const double cut2 = 1.0e-4;   // (1e-2)^2, cal_LJ.cu:11-12
  for (int t0 = 0; t0 < natom; t0 += kTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
      const int ia = t0 + i;
      if (ia < natom) {
        const double *a = atoms + 8 * (size_t)ia;
        sa[i] = make_double4(a[0], a[1], a[2], a[3]);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double sg = (a[4] + sites.sig[v]) * 0.5;                 // cal_LJ.cu:28
          sl[v][i] = make_double2(sg * sg, 4.0 * sqrt(a[5] * sites.eps[v]) * ikbt);  // :29, :38
          slf[v][i] = make_float2((float)sl[v][i].x, (float)sl[v][i].y);
        }
      }
    }
    __syncthreads();
    if (!live) continue;
    const int m = min(kTile, natom - t0);
    float accf[kPts][V];
#pragma unroll
    for (int k = 0; k < kPts; ++k)
#pragma unroll
      for (int v = 0; v < V; ++v) accf[k][v] = 0.0f;
    for (int i = 0; i < m; ++i) {
      const double4 at = sa[i];
      const double dy = ry - at.y, dz = rz - at.z;
      const double dyz = dy * dy + dz * dz;
#pragma unroll
      for (int k = 0; k < kPts; ++k) {
        const double dx = rx[k] - at.x;
        const double r2 = dx * dx + dyz;
        const double ri = rsqrt_nr<MIX ? 1 : 2>(r2);
        if (MIX) {
          const float ir2 = r2 < cut2 ? (float)(1.0 / cut2) : (float)(ri * ri);
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const float2 p = slf[v][i];
            const float s2 = p.x * ir2;
            const float s6 = s2 * s2 * s2;
            accf[k][v] += p.y * s6 * (s6 - 1.0f);
          }
        } else {
          const double ir2 = r2 < cut2 ? 1.0 / cut2 : ri * ri;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const double2 p = sl[v][i];
            const double s2 = p.x * ir2;
            const double s6 = s2 * s2 * s2;
            acc[k][v] += p.y * s6 * (s6 - 1.0);
          }
        }
        if (r2 >= 1600.0) {                 // r >= 40 A: e^-r is below FP64 resolution
          afr[k] += at.w * ri;
          continue;
        }
        const double ra = r2 > 0.0 ? r2 * ri : 0.0;
        if (ra >= 1.0e-5) {                 // cal_Coulomb.cu:114-120
          const double qr = at.w * ri;
          if (ra < (MIX ? 20.0 : 40.0)) {
            const double er = exp_neg(ra);  // e^-r
            afr[k] += qr * (1.0 - er);      // q (1 - e^-r) / r
            aes[k] += qr * er;              // q e^-r / r
          } else if (MIX && ra < 40.0) {
            const double es = qr * (double)expf(-(float)ra);
            afr[k] += qr - es;
            aes[k] += es;
          } else {
            afr[k] += qr;
          }
        } else {
          afr[k] += at.w;
          aes[k] -= at.w;
        }
      }
    }
    if (MIX) {
#pragma unroll
      for (int k = 0; k < kPts; ++k)
#pragma unroll
        for (int v = 0; v < V; ++v) acc[k][v] += (double)accf[k][v];
    }
  }
  if (!live) return;
  const size_t j = (size_t)ix + (size_t)nx * ((size_t)iy + (size_t)ny * iz);
#pragma unroll
  for (int k = 0; k < kPts; ++k) {
#pragma unroll
    for (int v = 0; v < V; ++v) u[(size_t)v * n + j + k] = acc[k][v];
    fr[j + k] = afr[k] * ubeta;
    esr[j + k] = aes[k] * ubeta;
  }
}

// Per-atom phase rows e^{-i k_d R_d} for the three axes (k from set_g,
// initialize_g.cu:58-60): ph[u][0..nx+ny+nz).
__global__ void k_phase_rows(int nx, int ny, int nz, double bx, double by, double bz,
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

// fk on the owner half j < N/2 (cal_Coulomb.cu:125-149): the phase
// e^{-ik.R} is the product of the three per-axis rows.  A block covers whole
// x rows (or one row segment when nx > blockDim): per atom tile, the y-z
// phase product of each of the block's rows is formed once in shared memory,
// and each thread adds q e^{-i kx X} (yz) with one coalesced row load.
constexpr int kRowsMax = 10;    // rows a block of min(256, 8 nx) points can touch

__global__ void __launch_bounds__(kThreads)
k_potential_k(int nx, int ny, int nz, double bx, double by, double bz,
              const double *__restrict__ atoms_all, const int *__restrict__ aoff,
              const int *__restrict__ acnt, double ubeta,
              const double2 *__restrict__ ph_all, double2 *__restrict__ fkh) {
  __shared__ double sq[kTile];
  __shared__ double2 syz[kRowsMax][kTile];
  const long long nh = (long long)nx * ny * nz / 2;
  const int sb = blockIdx.y;
  const double *__restrict__ atoms = atoms_all + 8 * (size_t)aoff[sb];
  const int natom = acnt[sb];
  const double2 *__restrict__ ph = ph_all + (size_t)aoff[sb] * (nx + ny + nz);
  fkh += (size_t)sb * nh;
  const long long jb = (long long)blockIdx.x * blockDim.x;      // first point of the block
  const long long j = jb + threadIdx.x;
  const long long jj = j < nh ? j : nh - 1;
  const int ix = (int)(jj % nx);
  const long long row = jj / nx, row0 = jb / nx;
  const int lrow = (int)(row - row0);                           // row within the block
  const int nrows = (int)(min(nh - 1, jb + (long long)blockDim.x - 1) / nx - row0) + 1;
  const int iy = (int)(row % ny), iz = (int)(row / ny);
  const double kx = 2.0 * kPi * (ix - nx / 2.0 + 0.5) / bx;
  const double ky = 2.0 * kPi * (iy - ny / 2.0 + 0.5) / by;
  const double kz = 2.0 * kPi * (iz - nz / 2.0 + 0.5) / bz;
  const double rk2 = kx * kx + ky * ky + kz * kz;
  const double rk4i = 1.0 / (rk2 * (rk2 + 1.0));
  const int L = nx + ny + nz;
  double re = 0.0, im = 0.0;
  for (int t0 = 0; t0 < natom; t0 += kTile) {
    const int m = min(kTile, natom - t0);
    __syncthreads();
    for (int i = threadIdx.x; i < kTile; i += blockDim.x)
      sq[i] = i < m ? 4.0 * kPi * atoms[8 * (size_t)(t0 + i) + 3] : 0.0;
    for (int e = threadIdx.x; e < nrows * m; e += blockDim.x) {
      const int r = e / m, i = e - r * m;
      const long long rw = row0 + r;
      const int y = (int)(rw % ny), z = (int)(rw / ny);
      const double2 *rowp = ph + (size_t)(t0 + i) * L;
      const double2 py = rowp[nx + y], pz = rowp[nx + ny + z];
      syz[r][i] = make_double2(py.x * pz.x - py.y * pz.y, py.x * pz.y + py.y * pz.x);
    }
    __syncthreads();
    for (int i = 0; i < m; ++i) {
      const double2 px = ph[(size_t)(t0 + i) * L + ix];
      const double2 yz = syz[lrow][i];
      const double cr = px.x * yz.x - px.y * yz.y, ci = px.x * yz.y + px.y * yz.x;
      re += sq[i] * cr;      // + 4 pi q cos(k.R)
      im += sq[i] * ci;      // - 4 pi q sin(k.R)
    }
  }
  if (j < nh) fkh[j] = make_double2(re * rk4i * ubeta, im * rk4i * ubeta);
}

template <int V>
void launch_r(Context &c, const SiteLJ &sl, double ikbt, double ubeta) {
  const int bx = (c.nx + kBrick - 1) / kBrick, by = (c.ny + kBrick - 1) / kBrick,
            bz = (c.nz + kBrick - 1) / kBrick;
  const dim3 grid((unsigned)((long long)bx * by * bz), c.nb);
  if (c.prm.precision == RISM3D_MIXED)
    k_potential_r<V, true><<<grid, kThreads, 0, c.stream>>>(
        c.nx, c.ny, c.nz, bx, by, c.dr[0], c.dr[1], c.dr[2], c.d_atoms, c.d_atom_off,
        c.d_atom_cnt, sl, ikbt, ubeta, c.d_u, c.d_e, c.d_fr);
  else
    k_potential_r<V, false><<<grid, kThreads, 0, c.stream>>>(
        c.nx, c.ny, c.nz, bx, by, c.dr[0], c.dr[1], c.dr[2], c.d_atoms, c.d_atom_off,
        c.d_atom_cnt, sl, ikbt, ubeta, c.d_u, c.d_e, c.d_fr);
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

// ESP cube in place of the point-charge potential (cal_Coulomb.cu:88-90):
// e = esp hartree / (kB T), so the stored short-range part is esr = e - fr;
// fr and fk keep the point-charge forms.
__global__ void k_esp_esr(long long n, const double *__restrict__ esp, double ubeta,
                          const double *__restrict__ fr, double *__restrict__ esr) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x)
    esr[j] = esp[j] * ubeta - fr[j];
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
  const long long L = c.nx + c.ny + c.nz;
  double2 *ph = nullptr;
  if (!cuda_ok(c, pool_alloc(c, (void **)&ph, sizeof(double2) * L * c.natom), "phase rows"))
    return RISM3D_CUDA_ERROR;
  k_phase_rows<<<(unsigned)((L * c.natom + 255) / 256), 256, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.prm.box[0], c.prm.box[1], c.prm.box[2], c.d_atoms, c.natom, ph);
  const int thr = c.nx >= 32 ? kThreads : 8 * c.nx;        // at most kRowsMax rows per block
  long long blocks = (c.n / 2 + thr - 1) / thr;
  k_potential_k<<<dim3((unsigned)blocks, c.nb), thr, 0, c.stream>>>(
      c.nx, c.ny, c.nz, c.prm.box[0], c.prm.box[1], c.prm.box[2], c.d_atoms,
      c.d_atom_off, c.d_atom_cnt, ubeta, ph, c.d_fkh);
  cudaFreeAsync(ph, c.stream);
  if (!cuda_ok(c, cudaGetLastError(), "k_potential_k")) return RISM3D_CUDA_ERROR;
  c.launches += 3;
  if (c.d_fkt) {                                  // the TMA fused pass K reads fk by columns
    const int rc = fused_fk_columns(c);
    if (rc != RISM3D_OK) return rc;
  }
  if (c.d_esp && c.nb == 1) {
    const long long eb = std::min<long long>((c.n + kThreads - 1) / kThreads, 148 * 16);
    k_esp_esr<<<(unsigned)eb, kThreads, 0, c.stream>>>(
        c.n, c.d_esp, kHartree / (kBoltzmann * c.temper), c.d_fr, c.d_e);
    if (!cuda_ok(c, cudaGetLastError(), "k_esp_esr")) return RISM3D_CUDA_ERROR;
    c.launches += 1;
  }
  return RISM3D_OK;
}

}  // namespace rism3d
