// Observables at convergence (reference: output.cu:6-62).
//
// k_observe: one FP64 pass over the grid gives, per site v, the KH, HNC and
// GF excess-chemical-potential integrands and the PMV integral
// (cal_exchem.cu:55-154, cal_pmv.cu:25-55) with h = Re h_OZ and
// t = t_SR + q_v cf fr, c = h - t.  Block partials are reduced in a fixed
// order, so the sums do not depend on scheduling.
//
// k_atom_integrals: SE per (site, atom) (cal_euv.cu:35-76) and the
// cal_grad gradients (cal_grad.cu:51-145) for ALL atoms in one launch: one
// atom per thread, grid points streamed through shared memory (the
// reference launches one full-grid kernel + Thrust reductions per pair).
// Mixed-precision contexts evaluate the SE pair terms in FP32 (coordinates
// as FP32 hi/lo pairs) and add each tile's FP32 sums into FP64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rism3d_impl.h"

namespace rism3d {
namespace {

constexpr int kThreads = 256;

template <int V, int CLOS>
__global__ void __launch_bounds__(kThreads)
k_observe(long long n, const double *__restrict__ h, const double *__restrict__ t,
          const double *__restrict__ fr, const StageParams *sp, double *part,
          int nblocks) {
  constexpr int NS = 4 * V;
  // solute blockIdx.y
  h += (size_t)blockIdx.y * V * n;
  t += (size_t)blockIdx.y * V * n;
  fr += (size_t)blockIdx.y * n;
  part += (size_t)blockIdx.y * NS * nblocks;
  __shared__ double red[kThreads / 32][NS];
  double acc[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) acc[k] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const double f = fr[j];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double hh = h[(size_t)v * n + j];
      const double tt = t[(size_t)v * n + j] + sp->qcf[v] * f;
      const double c = hh - tt;
      const double hnc = hh * 0.5 * tt - c;                     // ehnc
      const double gf = -(hh * 0.5 + 1.0) * c;                  // egf
      const double kh = hh > 0.0 ? gf : hnc;                    // ekh
      acc[4 * v + 0] += CLOS == 0 ? kh : hnc;
      acc[4 * v + 1] += hnc;
      acc[4 * v + 2] += gf;
      acc[4 * v + 3] += c;                                      // pmv_cuv
    }
  }
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < NS; ++k) red[wid][k] = acc[k];
  __syncthreads();
  for (int k = threadIdx.x; k < NS; k += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += red[w][k];
    part[(size_t)k * nblocks + blockIdx.x] = s;
  }
}

// out[k] = sum_b part[k][b], fixed order, one block per k.
__global__ void k_reduce_rows(const double *part, int ncols, double *out) {
  __shared__ double red[256];
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

struct SiteAll {
  double sig[kMaxSites], eps[kMaxSites], q[kMaxSites], rho[kMaxSites];
};

constexpr int kAtomsPerBlock = 128;
constexpr int kPtsTile = 128;

// part layout: [chunk][atom][2V + 6]: SE_LJ[v], SE_ES[v] (rho_v applied),
// grad LJ xyz, grad ES xyz (sum over v of rho_v * ...).  One FP64 rsqrt per
// (point, atom) gives 1/r, r and 1/r^2; the cutoff r < sigma_uv/2 of the
// reference is tested on r, with the correctly rounded sqrt only for points
// within 1e-12 of the cutoff radius.
template <int V, int GRAD>
__global__ void __launch_bounds__(kAtomsPerBlock)
k_atom_integrals(int nx, int ny, int nz, double drx, double dry, double drz,
                 const double *__restrict__ g, const double *__restrict__ atoms_all,
                 const int *__restrict__ aoff, const int *__restrict__ acnt, int natom_tot,
                 SiteAll sv, double cc, long long chunk, double *part) {
  constexpr int NA = 2 * V + 6;
  // solute blockIdx.z: its atoms against its own g; partials indexed by the
  // global atom number
  const int sb = blockIdx.z;
  const double *__restrict__ atoms = atoms_all + 8 * (size_t)aoff[sb];
  const int natom = acnt[sb];
  g += (size_t)sb * V * (size_t)nx * ny * nz;
  __shared__ double4 pp[kPtsTile];          // x y z
  __shared__ double pg[V][kPtsTile];
  const long long n = (long long)nx * ny * nz;
  const int ia = blockIdx.x * kAtomsPerBlock + threadIdx.x;
  const bool live = ia < natom;
  double X = 0, Y = 0, Z = 0, qu = 0, su = 0, eu = 0;
  if (live) {
    const double *a = atoms + 8 * (size_t)ia;
    X = a[0]; Y = a[1]; Z = a[2]; qu = a[3]; su = a[4]; eu = a[5];
  }
  double s6v[V], e4[V], qq[V], hs[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const double sg = (su + sv.sig[v]) * 0.5;  // cal_LJ.cu:28
    const double sg2 = sg * sg;
    s6v[v] = sg2 * sg2 * sg2;
    e4[v] = 4.0 * sqrt(eu * sv.eps[v]);        // cal_LJ.cu:29
    qq[v] = qu * sv.q[v] * cc;
    hs[v] = sg * 0.5;
  }
  double acc[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) acc[k] = 0.0;
  const long long j0 = (long long)blockIdx.y * chunk;
  const long long j1 = min(n, j0 + chunk);
  for (long long base = j0; base < j1; base += kPtsTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kPtsTile; i += blockDim.x) {
      const long long j = base + i;
      if (j < j1) {
        const long long r = j / nx;
        const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
        pp[i] = make_double4((ix - nx / 2) * drx, (iy - ny / 2) * dry,   // cal_euv.cu:45-47
                             (iz - nz / 2) * drz, 0.0);
#pragma unroll
        for (int v = 0; v < V; ++v) pg[v][i] = g[(size_t)v * n + j];
      } else {
        pp[i] = make_double4(1.0e30, 1.0e30, 1.0e30, 0.0);
#pragma unroll
        for (int v = 0; v < V; ++v) pg[v][i] = 0.0;
      }
    }
    __syncthreads();
    if (!live) continue;
    const int m = (int)min((long long)kPtsTile, j1 - base);
    for (int i = 0; i < m; ++i) {
      const double4 p = pp[i];
      const double dx = p.x - X, dy = p.y - Y, dz = p.z - Z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double ri = rsqrt_nr<2>(r2);
      const double r1 = r2 * ri;
      const double ir2 = ri * ri;
      const double ir6 = ir2 * ir2 * ir2;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        bool inside = !(r1 >= hs[v]);           // r = 0 gives NaN: inside
        if (fabs(r1 - hs[v]) < 1.0e-12 * hs[v]) inside = sqrt(r2) < hs[v];
        if (inside) continue;                 // cutoff r < sigma/2
        const double gv = pg[v][i];
        const double rs6i = s6v[v] * ir6;
        acc[v] += e4[v] * rs6i * (rs6i - 1.0) * gv;
        acc[V + v] += qq[v] * ri * gv;
        if (GRAD) {
          const double ulj = 6.0 * e4[v] * rs6i * ir2 * (2.0 * rs6i - 1.0) * gv * sv.rho[v];
          const double uco = qq[v] * ri * ir2 * gv * sv.rho[v];
          acc[2 * V + 0] += ulj * dx; acc[2 * V + 1] += ulj * dy; acc[2 * V + 2] += ulj * dz;
          acc[2 * V + 3] += uco * dx; acc[2 * V + 4] += uco * dy; acc[2 * V + 5] += uco * dz;
        }
      }
    }
  }
  if (live) {
    double *o = part + ((size_t)blockIdx.y * natom_tot + aoff[sb] + ia) * NA;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      o[v] = acc[v] * sv.rho[v];
      o[V + v] = acc[V + v] * sv.rho[v];
    }
#pragma unroll
    for (int k = 2 * V; k < NA; ++k) o[k] = acc[k];
  }
}

// SE only, pair terms in FP32 (mixed-precision contexts); same partial
// layout as k_atom_integrals with GRAD = 0.  Coordinates are carried as FP32
// (hi, lo) pairs, so dx = (x_hi - X_hi) + (x_lo - X_lo) is accurate to FP32
// relative precision of dx itself without any FP64 work in the pair loop.
// Per site the loop accumulates g (s/r)^6 ((s/r)^6 - 1) and g / r; the
// factors 4 eps_uv and q_u q_v cc are applied per tile in FP64.  The cutoff
// r < sigma/2 zeroes g (r^2 is clamped at 1e-4 so the masked terms stay
// finite; every unmasked point lies beyond the smallest cutoff, 0.1 A);
// points within 2e-5 of a cutoff re-test it in FP64.  Each thread carries
// NA_T atoms; grid points come through shared memory in tiles of kSeTile.
constexpr int kSeTile = 512;

template <int V, int NA_T>
__global__ void __launch_bounds__(kAtomsPerBlock, V <= 5 ? 4 : 2)
k_atom_se32(int nx, int ny, int nz, double drx, double dry, double drz,
            const double *__restrict__ g, const double *__restrict__ atoms_all,
            const int *__restrict__ aoff, const int *__restrict__ acnt, int natom_tot,
            SiteAll sv, double cc, long long chunk, double *part) {
  constexpr int NA = 2 * V + 6;
  const int sb = blockIdx.z;
  const double *__restrict__ atoms = atoms_all + 8 * (size_t)aoff[sb];
  const int natom = acnt[sb];
  g += (size_t)sb * V * (size_t)nx * ny * nz;
  __shared__ float4 ph[kSeTile];            // x_hi y_hi z_hi
  __shared__ float4 pl[kSeTile];            // x_lo y_lo z_lo
  __shared__ float pg[V][kSeTile];
  const long long n = (long long)nx * ny * nz;
  int ia[NA_T];
  bool live[NA_T], any = false;
  float Xh[NA_T], Yh[NA_T], Zh[NA_T], Xl[NA_T], Yl[NA_T], Zl[NA_T];
  float s6v[NA_T][V], hs2[NA_T][V], blo[NA_T][V], bhi[NA_T][V];
  double e4[NA_T][V], qq[NA_T][V];
#pragma unroll
  for (int a = 0; a < NA_T; ++a) {
    ia[a] = blockIdx.x * kAtomsPerBlock * NA_T + a * kAtomsPerBlock + threadIdx.x;
    live[a] = ia[a] < natom;
    any = any || live[a];
    double X = 0, Y = 0, Z = 0, qu = 0, su = 0, eu = 0;
    if (live[a]) {
      const double *p = atoms + 8 * (size_t)ia[a];
      X = p[0]; Y = p[1]; Z = p[2]; qu = p[3]; su = p[4]; eu = p[5];
    }
    Xh[a] = (float)X; Yh[a] = (float)Y; Zh[a] = (float)Z;
    Xl[a] = (float)(X - Xh[a]); Yl[a] = (float)(Y - Yh[a]); Zl[a] = (float)(Z - Zh[a]);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double sg = (su + sv.sig[v]) * 0.5;  // cal_LJ.cu:28
      const double sg2 = sg * sg;
      s6v[a][v] = (float)(sg2 * sg2 * sg2);
      e4[a][v] = 4.0 * sqrt(eu * sv.eps[v]);
      qq[a][v] = qu * sv.q[v] * cc;
      hs2[a][v] = (float)(0.25 * sg2);
      blo[a][v] = (float)(0.25 * sg2 * (1.0 - 2.0e-5));
      bhi[a][v] = (float)(0.25 * sg2 * (1.0 + 2.0e-5));
    }
  }
  double acc[NA_T][2 * V];
#pragma unroll
  for (int a = 0; a < NA_T; ++a)
#pragma unroll
    for (int k = 0; k < 2 * V; ++k) acc[a][k] = 0.0;
  const long long j0 = (long long)blockIdx.y * chunk;
  const long long j1 = min(n, j0 + chunk);
  for (long long base = j0; base < j1; base += kSeTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kSeTile; i += blockDim.x) {
      const long long j = base + i;
      if (j < j1) {
        const long long r = j / nx;
        const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
        const double px = (ix - nx / 2) * drx, py = (iy - ny / 2) * dry,   // cal_euv.cu:45-47
                     pz = (iz - nz / 2) * drz;
        const float hx = (float)px, hy = (float)py, hz = (float)pz;
        ph[i] = make_float4(hx, hy, hz, 0.0f);
        pl[i] = make_float4((float)(px - hx), (float)(py - hy), (float)(pz - hz), 0.0f);
#pragma unroll
        for (int v = 0; v < V; ++v) pg[v][i] = (float)g[(size_t)v * n + j];
      } else {
        ph[i] = make_float4(1.0e30f, 1.0e30f, 1.0e30f, 0.0f);
        pl[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
        for (int v = 0; v < V; ++v) pg[v][i] = 0.0f;
      }
    }
    __syncthreads();
    if (!any) continue;
    const int m = (int)min((long long)kSeTile, j1 - base);
    float tl[NA_T][2 * V];
#pragma unroll
    for (int a = 0; a < NA_T; ++a)
#pragma unroll
      for (int k = 0; k < 2 * V; ++k) tl[a][k] = 0.0f;
    for (int i = 0; i < m; ++i) {
      const float4 h = ph[i], l = pl[i];
      float gv[V];
#pragma unroll
      for (int v = 0; v < V; ++v) gv[v] = pg[v][i];
#pragma unroll
      for (int a = 0; a < NA_T; ++a) {
        const float dx = (h.x - Xh[a]) + (l.x - Xl[a]);
        const float dy = (h.y - Yh[a]) + (l.y - Yl[a]);
        const float dz = (h.z - Zh[a]) + (l.z - Zl[a]);
        const float r2 = dx * dx + dy * dy + dz * dz;
        const float ri = rsqrtf(fmaxf(r2, 1.0e-4f));
        const float ir2 = ri * ri;
        const float ir6 = ir2 * ir2 * ir2;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          bool inside = r2 < hs2[a][v];
          if (r2 > blo[a][v] && r2 < bhi[a][v]) {   // rare: exact test
            const double *p = atoms + 8 * (size_t)ia[a];
            const double ex = ((double)h.x + l.x) - p[0], ey = ((double)h.y + l.y) - p[1],
                         ez = ((double)h.z + l.z) - p[2];
            inside = sqrt(ex * ex + ey * ey + ez * ez) < (p[4] + sv.sig[v]) * 0.25;
          }
          const float w = inside ? 0.0f : gv[v];
          const float rs6i = s6v[a][v] * ir6;
          tl[a][v] = fmaf(w, rs6i * (rs6i - 1.0f), tl[a][v]);
          tl[a][V + v] = fmaf(w, ri, tl[a][V + v]);
        }
      }
    }
#pragma unroll
    for (int a = 0; a < NA_T; ++a)
#pragma unroll
      for (int v = 0; v < V; ++v) {
        acc[a][v] += e4[a][v] * (double)tl[a][v];
        acc[a][V + v] += qq[a][v] * (double)tl[a][V + v];
      }
  }
#pragma unroll
  for (int a = 0; a < NA_T; ++a) {
    if (!live[a]) continue;
    double *o = part + ((size_t)blockIdx.y * natom_tot + aoff[sb] + ia[a]) * NA;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      o[v] = acc[a][v] * sv.rho[v];
      o[V + v] = acc[a][V + v] * sv.rho[v];
    }
#pragma unroll
    for (int k = 2 * V; k < NA; ++k) o[k] = 0.0;
  }
}

// sum over chunks, fixed order: out[atom][k]
__global__ void k_sum_chunks(const double *part, int nchunk, int natom, int na,
                             double *out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= natom * na) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; ++c) s += part[(size_t)c * natom * na + idx];
  out[idx] = s;
}

template <int V>
int observe_v(Context &c) {
  const int nb = c.nred_blocks, B = c.nb;
  StageParams sp{};
  for (int v = 0; v < V; ++v) sp.qcf[v] = c.qv[v] * c.cf_final;
  cudaMemcpyAsync(c.d_stage, &sp, sizeof(sp), cudaMemcpyHostToDevice, c.stream);
  if (c.prm.closure == RISM3D_KH)
    k_observe<V, 0><<<dim3(nb, B), kThreads, 0, c.stream>>>(c.n, c.d_h, c.d_t, c.d_fr, c.d_stage, c.d_part, nb);
  else
    k_observe<V, 1><<<dim3(nb, B), kThreads, 0, c.stream>>>(c.n, c.d_h, c.d_t, c.d_fr, c.d_stage, c.d_part, nb);
  k_reduce_rows<<<4 * V * B, 256, 0, c.stream>>>(c.d_part, nb, c.d_obs);
  c.launches += 2;
  std::vector<double> s((size_t)4 * V * B);
  if (!cuda_ok(c, cudaMemcpyAsync(s.data(), c.d_obs, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, c.stream), "observe") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "observe"))
    return RISM3D_CUDA_ERROR;
  const double ibeta = kAvogadro * kBoltzmann * c.temper;   // output_xmu.cu:19
  double pres = 0.0;                                         // cal_pressure.cu
  for (int v = 0; v < V; ++v) pres += c.rho[v];
  pres *= 1.0e30 / kAvogadro;
  pres = 0.5 * (pres + 1.0 / (c.xt * ibeta));
  for (int b = 0; b < B; ++b) {
    rism3d_result &r = (B == 1) ? c.res : c.bres[b];
    const double *sb = &s[(size_t)b * 4 * V];
    r.natv = V;
    r.natom = (B == 1) ? c.natom : c.atom_cnt[b];
    r.sfe_sc = r.sfe_sc_hnc = r.sfe_gf = 0.0;
    double cuv = 0.0;
    for (int v = 0; v < V; ++v) {
      r.sfec_sc[v] = ibeta * sb[4 * v + 0] * c.rho[v] * c.dv;
      r.sfec_sc_hnc[v] = ibeta * sb[4 * v + 1] * c.rho[v] * c.dv;
      r.sfec_gf[v] = ibeta * sb[4 * v + 2] * c.rho[v] * c.dv;
      r.sfe_sc += r.sfec_sc[v];
      r.sfe_sc_hnc += r.sfec_sc_hnc[v];
      r.sfe_gf += r.sfec_gf[v];
      cuv += sb[4 * v + 3] * c.rho[v];
    }
    cuv *= c.dv;
    const double pmv = c.xt * (1.0 - cuv) * ibeta;           // cal_pmv.cu:18-19
    r.pmv = pmv * 1000.0;
    r.pressure = ibeta * pres;
    r.correction = -pres * pmv * ibeta;                      // output_xmu.cu:21
  }
  return RISM3D_OK;
}

template <int V>
int atoms_v(Context &c, bool forces) {
  constexpr int NA = 2 * V + 6;
  const int A = c.natom;            // all solutes
  int amax = 0;
  for (int x : c.atom_cnt) amax = std::max(amax, x);
  // FP32 SE (mixed contexts, no forces): kSeAtoms atoms per thread (two for
  // up to 2 sites: more would spill under the 4-blocks-per-SM bound)
  constexpr int kSeAtoms = V <= 2 ? 2 : 1;
  const bool se32 = !forces && c.prm.precision == RISM3D_MIXED;
  const int per_block = kAtomsPerBlock * (se32 ? kSeAtoms : 1);
  const int tiles = (amax + per_block - 1) / per_block;
  // enough chunks to fill the GPU a few times over
  int nchunk = (148 * 8 + tiles * c.nb - 1) / (tiles * c.nb);
  if (nchunk < 1) nchunk = 1;
  long long chunk = (c.n + nchunk - 1) / nchunk;
  const int tile = se32 ? kSeTile : kPtsTile;
  chunk = ((chunk + tile - 1) / tile) * tile;
  nchunk = (int)((c.n + chunk - 1) / chunk);
  size_t need = (size_t)nchunk * A * NA + (size_t)A * NA;
  if ((int)need > c.natom_part_cap) {
    if (c.d_atom_part) cudaFree(c.d_atom_part);
    if (!cuda_ok(c, cudaMalloc(&c.d_atom_part, sizeof(double) * need), "atom partials"))
      return RISM3D_CUDA_ERROR;
    c.natom_part_cap = (int)need;
  }
  SiteAll sv{};
  for (int v = 0; v < V; ++v) {
    sv.sig[v] = c.sigv[v]; sv.eps[v] = c.epsv[v]; sv.q[v] = c.qv[v]; sv.rho[v] = c.rho[v];
  }
  const double cc = kHartree * kBohr * kAvogadro;            // cal_euv.cu:39
  dim3 grid(tiles, nchunk, c.nb);
  if (forces)
    k_atom_integrals<V, 1><<<grid, kAtomsPerBlock, 0, c.stream>>>(
        c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_g, c.d_atoms, c.d_atom_off,
        c.d_atom_cnt, A, sv, cc, chunk, c.d_atom_part);
  else if (se32)
    k_atom_se32<V, kSeAtoms><<<grid, kAtomsPerBlock, 0, c.stream>>>(
        c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_g, c.d_atoms, c.d_atom_off,
        c.d_atom_cnt, A, sv, cc, chunk, c.d_atom_part);
  else
    k_atom_integrals<V, 0><<<grid, kAtomsPerBlock, 0, c.stream>>>(
        c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_g, c.d_atoms, c.d_atom_off,
        c.d_atom_cnt, A, sv, cc, chunk, c.d_atom_part);
  double *sum = c.d_atom_part + (size_t)nchunk * A * NA;
  k_sum_chunks<<<(A * NA + 255) / 256, 256, 0, c.stream>>>(c.d_atom_part, nchunk, A, NA, sum);
  c.launches += 2;
  std::vector<double> h((size_t)A * NA);
  if (!cuda_ok(c, cudaGetLastError(), "atom integrals") ||
      !cuda_ok(c, cudaMemcpyAsync(h.data(), sum, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream), "atom integrals") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "atom integrals"))
    return RISM3D_CUDA_ERROR;
  if (c.nb > 1) {                   // per-solute SE totals (batched solves)
    for (int b = 0; b < c.nb; ++b) {
      double slj = 0.0, ses = 0.0;
      for (int u = c.atom_off[b]; u < c.atom_off[b] + c.atom_cnt[b]; ++u)
        for (int v = 0; v < V; ++v) {
          slj += h[(size_t)u * NA + v] * c.dv;
          ses += h[(size_t)u * NA + V + v] * c.dv;
        }
      c.bres[b].se_lj = slj;
      c.bres[b].se_es = ses;
      c.bres[b].se = slj + ses;
    }
    return RISM3D_OK;
  }
  c.euv.assign((size_t)2 * V * A, 0.0);
  double slj = 0.0, ses = 0.0;
  for (int u = 0; u < A; ++u)
    for (int v = 0; v < V; ++v) {
      double lj = h[(size_t)u * NA + v] * c.dv, es = h[(size_t)u * NA + V + v] * c.dv;
      c.euv[(size_t)A * v + u] = lj;                         // cal_euv.cu:28-29
      c.euv[(size_t)V * A + (size_t)A * v + u] = es;
    }
  for (size_t i = 0; i < (size_t)V * A; ++i) slj += c.euv[i];
  for (size_t i = (size_t)V * A; i < (size_t)2 * V * A; ++i) ses += c.euv[i];
  c.res.se_lj = slj;
  c.res.se_es = ses;
  c.res.se = slj + ses;
  if (forces) {
    c.dulj.assign((size_t)A * 3, 0.0);
    c.due.assign((size_t)A * 3, 0.0);
    for (int u = 0; u < A; ++u)
      for (int k = 0; k < 3; ++k) {
        c.dulj[(size_t)u * 3 + k] = h[(size_t)u * NA + 2 * V + k] * c.dv;
        c.due[(size_t)u * 3 + k] = h[(size_t)u * NA + 2 * V + 3 + k] * c.dv;
      }
    c.have_forces = true;
  }
  return RISM3D_OK;
}

}  // namespace

// SE totals from the grids (single solute, point-charge potential).  The
// reference's per-(site, atom) sums over r >= sigma_uv / 2 (cal_euv.cu:7-76)
// add up, over the atoms, to one sum over the grid of g times the potential
// grids the solve already holds -- u_v = sum_u beta u_LJ,uv with r^2 clamped
// at 1e-4 (cal_LJ.cu:57-71) and e = esr + fr = beta sum_u q_u / r over
// r >= 1e-5 (cal_Coulomb.cu:109-121) -- minus each atom's own terms at the
// grid points inside its exclusion sphere r < sigma_uv / 2, where g is
// essentially zero.  That is one streaming pass plus a few thousand points
// per atom, in place of every (point, atom) pair.
template <int V>
__global__ void __launch_bounds__(kThreads)
k_se_grid(long long n, const double *__restrict__ g, const double *__restrict__ u,
          const double *__restrict__ esr, const double *__restrict__ fr, double *part) {
  double acc[2 * V];
#pragma unroll
  for (int i = 0; i < 2 * V; ++i) acc[i] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    const double e = esr[j] + fr[j];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double gv = g[(size_t)v * n + j];
      acc[v] += gv * u[(size_t)v * n + j];
      acc[V + v] += gv * e;
    }
  }
  __shared__ double red[kThreads / 32][2 * V];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < 2 * V; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][i] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < 2 * V) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w][threadIdx.x];
    part[(size_t)blockIdx.x * 2 * V + threadIdx.x] = t;
  }
}

// One atom per block: its LJ (beta units, clamped as in the grid) and q / r
// (r >= 1e-5) terms times g at the grid points with r < sigma_uv / 2,
// per site; part[atom][2V]
template <int V>
__global__ void __launch_bounds__(kThreads)
k_se_core(int nx, int ny, int nz, double drx, double dry, double drz,
          const double *__restrict__ g, const double *__restrict__ atoms, SiteAll sv,
          double ikbt, double *part) {
  const double *a = atoms + 8 * (size_t)blockIdx.x;
  const double X = a[0], Y = a[1], Z = a[2], q = a[3];
  double half[V], s2uv[V], e4[V], rmax = 0.0;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const double sg = (a[4] + sv.sig[v]) * 0.5;                     // cal_euv.cu:31-32
    half[v] = sg * 0.5;
    s2uv[v] = sg * sg;
    e4[v] = 4.0 * sqrt(a[5] * sv.eps[v]) * ikbt;
    rmax = fmax(rmax, half[v]);
  }
  const long long n = (long long)nx * ny * nz;
  // grid coordinates (i - n/2) d (cal_LJ.cu:54-56): the index box of the sphere
  const int x0 = max(0, (int)floor((X - rmax) / drx) + nx / 2 - 1);
  const int x1 = min(nx - 1, (int)ceil((X + rmax) / drx) + nx / 2 + 1);
  const int y0 = max(0, (int)floor((Y - rmax) / dry) + ny / 2 - 1);
  const int y1 = min(ny - 1, (int)ceil((Y + rmax) / dry) + ny / 2 + 1);
  const int z0 = max(0, (int)floor((Z - rmax) / drz) + nz / 2 - 1);
  const int z1 = min(nz - 1, (int)ceil((Z + rmax) / drz) + nz / 2 + 1);
  const long long wx = x1 - x0 + 1, wy = y1 - y0 + 1, wz = z1 - z0 + 1;
  const long long pts = (wx > 0 && wy > 0 && wz > 0) ? wx * wy * wz : 0;
  double acc[2 * V];
#pragma unroll
  for (int i = 0; i < 2 * V; ++i) acc[i] = 0.0;
  for (long long p = threadIdx.x; p < pts; p += blockDim.x) {
    const int ix = x0 + (int)(p % wx);
    const int iy = y0 + (int)((p / wx) % wy);
    const int iz = z0 + (int)(p / (wx * wy));
    const double dx = (ix - nx / 2) * drx - X, dy = (iy - ny / 2) * dry - Y,
                 dz = (iz - nz / 2) * drz - Z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = sqrt(r2);
    const double ir2 = r2 < 1.0e-4 ? 1.0e4 : 1.0 / r2;
    const long long j = ix + (long long)nx * (iy + (long long)ny * iz);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (r < half[v]) {
        const double gv = g[(size_t)v * n + j];
        const double s2 = s2uv[v] * ir2, s6 = s2 * s2 * s2;
        acc[v] += gv * e4[v] * s6 * (s6 - 1.0);
        if (r >= 1.0e-5) acc[V + v] += gv * q / r;
      }
    }
  }
  __shared__ double red[kThreads / 32][2 * V];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < 2 * V; ++i) {
    double v = acc[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][i] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < 2 * V) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w][threadIdx.x];
    part[(size_t)blockIdx.x * 2 * V + threadIdx.x] = t;
  }
}

constexpr int kSeGridBlocks = 148 * 8;

template <int V>
int se_grid_v(Context &c) {
  const int A = c.natom;
  double *part = nullptr;
  const size_t np = (size_t)(kSeGridBlocks + A) * 2 * V;
  if (!cuda_ok(c, pool_alloc(c, (void **)&part, sizeof(double) * np), "SE partials"))
    return RISM3D_CUDA_ERROR;
  SiteAll sv{};
  for (int v = 0; v < V; ++v) {
    sv.sig[v] = c.sigv[v]; sv.eps[v] = c.epsv[v]; sv.q[v] = c.qv[v]; sv.rho[v] = c.rho[v];
  }
  const double ikbt = 1.0 / (kAvogadro * kBoltzmann * c.temper);
  k_se_grid<V><<<kSeGridBlocks, kThreads, 0, c.stream>>>(c.n, c.d_g, c.d_u, c.d_e, c.d_fr, part);
  k_se_core<V><<<A, kThreads, 0, c.stream>>>(c.nx, c.ny, c.nz, c.dr[0], c.dr[1], c.dr[2], c.d_g,
                                             c.d_atoms, sv, ikbt,
                                             part + (size_t)kSeGridBlocks * 2 * V);
  c.launches += 2;
  std::vector<double> h(np);
  bool ok = cuda_ok(c, cudaGetLastError(), "SE grid") &&
            cuda_ok(c, cudaMemcpyAsync(h.data(), part, sizeof(double) * np, cudaMemcpyDeviceToHost,
                                       c.stream), "SE grid");
  cudaFreeAsync(part, c.stream);
  if (!ok || !cuda_ok(c, cudaStreamSynchronize(c.stream), "SE grid")) return RISM3D_CUDA_ERROR;
  double sg[2 * V] = {}, sc[2 * V] = {};
  for (int b = 0; b < kSeGridBlocks; ++b)
    for (int i = 0; i < 2 * V; ++i) sg[i] += h[(size_t)b * 2 * V + i];
  for (int u = 0; u < A; ++u)
    for (int i = 0; i < 2 * V; ++i) sc[i] += h[(size_t)(kSeGridBlocks + u) * 2 * V + i];
  const double ibeta = kAvogadro * kBoltzmann * c.temper;               // J/mol per beta unit
  const double ubeta = kHartree * kBohr / (kBoltzmann * c.temper);      // e grid per q / r
  const double cc = kHartree * kBohr * kAvogadro;                       // cal_euv.cu:39
  double slj = 0.0, ses = 0.0;
  for (int v = 0; v < V; ++v) {
    slj += c.rho[v] * ibeta * (sg[v] - sc[v]) * c.dv;
    ses += c.rho[v] * c.qv[v] * cc * (sg[V + v] / ubeta - sc[V + v]) * c.dv;
  }
  c.res.se_lj = slj;
  c.res.se_es = ses;
  c.res.se = slj + ses;
  c.euv.clear();                    // per-atom values on request (rism3d_euv)
  return RISM3D_OK;
}

int compute_observables(Context &c) {
  switch (c.natv) {
    case 1: return observe_v<1>(c);
    case 2: return observe_v<2>(c);
    case 3: return observe_v<3>(c);
    case 4: return observe_v<4>(c);
    case 5: return observe_v<5>(c);
    case 6: return observe_v<6>(c);
    case 7: return observe_v<7>(c);
    case 8: return observe_v<8>(c);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

// Result grids formed on the device into caller memory (rism3d_get_grid_device):
// mode 0: out = a + b (e = esr + fr); 1: out_v = a_v + qcf_v b (t = t_SR + q cf fr);
// 2: out_v = h_v - (a_v + qcf_v b) (c = h - t); 3: out = sum_v w_v g_v (cal_qv.cu:20-27)
struct GridArgs {
  double coef[kMaxSites];
  int nv, mode;
};

__global__ void k_grid_out(long long n, GridArgs ga, const double *__restrict__ a,
                           const double *__restrict__ b, const double *__restrict__ h,
                           double *__restrict__ out) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    if (ga.mode == 0) {
      out[j] = a[j] + b[j];
    } else if (ga.mode == 3) {
      double s = 0.0;
      for (int v = 0; v < ga.nv; ++v) s += a[(size_t)v * n + j] * ga.coef[v];
      out[j] = s;
    } else {
      const double fr = b[j];
      for (int v = 0; v < ga.nv; ++v) {
        const double t = a[(size_t)v * n + j] + ga.coef[v] * fr;
        out[(size_t)v * n + j] = ga.mode == 1 ? t : h[(size_t)v * n + j] - t;
      }
    }
  }
}

int device_grid(Context &c, int which, double *out) {
  const long long n = c.n;
  const size_t V = (size_t)c.natv;
  auto copy = [&](const double *src, size_t cnt) {
    return cuda_ok(c, cudaMemcpyAsync(out, src, sizeof(double) * cnt, cudaMemcpyDeviceToDevice,
                                      c.stream), "get_grid_device") ? RISM3D_OK : RISM3D_CUDA_ERROR;
  };
  GridArgs ga{};
  ga.nv = c.natv;
  const double *a = nullptr, *b = nullptr, *h = nullptr;
  switch (which) {
    case RISM3D_GRID_U: return copy(c.d_u, V * n);
    case RISM3D_GRID_FR: return copy(c.d_fr, n);
    case RISM3D_GRID_E: ga.mode = 0; a = c.d_e; b = c.d_fr; break;
    case RISM3D_GRID_G: case RISM3D_GRID_H: case RISM3D_GRID_T: case RISM3D_GRID_C:
    case RISM3D_GRID_QV:
      if (!c.solved) { c.err = "no solution yet"; return RISM3D_BAD_STATE; }
      if (which == RISM3D_GRID_G) return copy(c.d_g, V * n);
      if (which == RISM3D_GRID_H) return copy(c.d_h, V * n);
      if (which == RISM3D_GRID_QV) {
        ga.mode = 3; a = c.d_g;
        for (int v = 0; v < c.natv; ++v) ga.coef[v] = c.rho[v] * c.qv[v];
      } else {
        ga.mode = which == RISM3D_GRID_T ? 1 : 2; a = c.d_t; b = c.d_fr; h = c.d_h;
        for (int v = 0; v < c.natv; ++v) ga.coef[v] = c.qv[v] * c.cf_final;
      }
      break;
    default:
      c.err = "unknown grid id";
      return RISM3D_BAD_INPUT;
  }
  const long long blocks = std::min<long long>((n + kThreads - 1) / kThreads, 148 * 16);
  k_grid_out<<<(unsigned)blocks, kThreads, 0, c.stream>>>(n, ga, a, b, h, out);
  c.launches += 1;
  return cuda_ok(c, cudaGetLastError(), "get_grid_device") ? RISM3D_OK : RISM3D_CUDA_ERROR;
}

int compute_se_from_grids(Context &c) {
  switch (c.natv) {
    case 1: return se_grid_v<1>(c);
    case 2: return se_grid_v<2>(c);
    case 3: return se_grid_v<3>(c);
    case 4: return se_grid_v<4>(c);
    case 5: return se_grid_v<5>(c);
    case 6: return se_grid_v<6>(c);
    case 7: return se_grid_v<7>(c);
    case 8: return se_grid_v<8>(c);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

int compute_atom_integrals(Context &c, bool forces) {
  switch (c.natv) {
    case 1: return atoms_v<1>(c, forces);
    case 2: return atoms_v<2>(c, forces);
    case 3: return atoms_v<3>(c, forces);
    case 4: return atoms_v<4>(c, forces);
    case 5: return atoms_v<5>(c, forces);
    case 6: return atoms_v<6>(c, forces);
    case 7: return atoms_v<7>(c, forces);
    case 8: return atoms_v<8>(c, forces);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

}  // namespace rism3d
