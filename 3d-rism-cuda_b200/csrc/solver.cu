// The 3D-RISM fixed-point iteration (reference: iterate.cu:6-90,
// calculate.cu:4-58, calculate_cuda.cu:1-66, fft3d.cu:4-94, cal_rms.cu,
// anderson.cu:13-112, anderson_cuda.cu:1-66), re-designed around three
// streaming passes and two cuFFT transforms per iteration:
//
//   pass A  (k_pass_a)   residual of the previous cycle + AN2/Picard update
//                        + closure + c_SR + forward pre-twiddle; two real
//                        sites are packed into one complex grid
//   FFT forward          cuFFT C2C/Z2Z, in place, one transform per site pair
//   pass K  (k_kspace)   unpack the pair (F(-k) = conj F(k)), post-twiddle,
//                        minus the long-range fk, OZ site product with chi
//                        spline-evaluated at |k|, repack for the inverse
//   FFT inverse
//   pass R  (k_pass_r)   post-twiddle, closure, residual R = h + 1 - g,
//                        FP64 block sums of R^2 and the five AN2 Gram terms
//   finalize             (last block of pass R) fixed-order reduction of the
//                        block sums, rms, convergence / divergence / maxstep
//                        decision, 2x2 AN2 solve -- on the device, no host
//                        sync, no extra launch.
//
// The state variable is the short-range indirect correlation
// t_SR = t - q_v cf fr.  The closure exponent -u - q cf e + t equals
// -U_SR + t_SR with U_SR = u + q cf (e - fr), and c_SR = g - 1 - t + q cf fr
// = g - 1 - t_SR, so the long-range Coulomb terms never enter the passes.
// The AN2 history stores Y_i = tp_i + m rp_i and RP_i = rp_i: the reference
// update u + m(v - u) (anderson_cuda.cu:16-22) is algebraically
// y + s1 (Y_0 - y) + s2 (Y_1 - y) with y = t + m R.
//
// Mixed precision iterates in FP32 in two forms.  The plain form carries t
// itself; its rounding floor (eps32 times the size of g and h near the
// solute, ~1e-5 in rms) ends it.  The refinement form (REF) carries the
// correction d = t - t0 to a fixed FP64 base t0 whose residual R0 = R(t0)
// was computed once in FP64.  Because the OZ operator L is linear,
//   R(t0 + d) = R0 + L[dc] - dg,   dg = C(x0 + d) - C(x0),  dc = dg - d,
// with x0 = t0 - U_SR, and the long-range fk term cancels.  Every FP32
// quantity is then of the size of the correction, so the residual is exact
// to eps32 |d| and AN2 (which is affine, so it acts on d unchanged)
// converges to the FP64 tolerance in FP32 passes.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "rism3d_impl.h"
#include "tma.cuh"
#include "xfft.cuh"

namespace rism3d {

template <typename T> struct Cx;
template <> struct Cx<double> { typedef double2 t; };
template <> struct Cx<float> { typedef float2 t; };

namespace {

constexpr int kThreads = 256;

template <typename T>
struct IterArgs {
  long long n;
  int nx, ny, nz;
  FastDiv fdx, fdy;         // division by nx and ny
  const double *xs;         // chi table per odd-square sum (cubic cells) or null
  const float *xs32;        // the same table in FP32 (read by the FP32 passes)
  typename Cx<T>::t *buf;   // [P][N]
  T *t, *U, *Y, *RP;        // t, U: [V][N]; Y, RP: [2][V][N]
  const T *R0;              // refinement: base residual [V][N] (t = d, U = x0)
  double *hout, *gout;      // final snapshot, [V][N] (may be null)
  const typename Cx<T>::t *tw;  // px[nx] py[ny] pz[nz]
  double invvol, dv;
  const double2 *fkh;       // [N/2]
  const double *chi;        // [ntab][V*V][4]
  int ntab;
  double dk;
  double bx, by, bz;
  DevState *st;
  const StageParams *sp;
  double *part;
  int nblocks;
  unsigned *count;          // blocks of pass R done (reset by the last one)
  double *hist;             // per-iteration rms (single solves, verbose) or null
  int hist_cap;
  int nofk;                 // refinement: q cf fk cancels, fk is not read
  const float2 *xroots;     // fused-axis passes: W_nx^m, m < nx (nx == ny)
  const float2 *fkt;        // fused-axis pass K (nx = 256): beta fk as [nz/2][nx][ny]
};

// Batched solves: blockIdx.y selects the solute; every per-solute array is
// laid out solute-major ([B][...]) and this view offsets the pointers, so
// the kernel bodies below are the single-solute code unchanged.
template <typename T, int V>
__device__ __forceinline__ IterArgs<T> solute_view(const IterArgs<T> &a) {
  constexpr int P = (V + 1) / 2;
  IterArgs<T> s = a;
  const size_t b = blockIdx.y, n = (size_t)a.n;
  if (b == 0) return s;
  s.buf = a.buf + b * P * n;
  s.t = a.t + b * V * n;
  s.U = a.U + b * V * n;
  s.Y = a.Y + b * 2 * V * n;
  s.RP = a.RP + b * 2 * V * n;
  if (a.hout) { s.hout = a.hout + b * V * n; s.gout = a.gout + b * V * n; }
  if (a.R0) s.R0 = a.R0 + b * V * n;
  s.fkh = a.fkh + b * (n / 2);
  s.st = a.st + b;
  s.part = a.part + b * 6 * (size_t)a.nblocks;
  s.count = a.count + b;
  return s;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C mk(double x, double y);
template <> __device__ __forceinline__ double2 mk<double2>(double x, double y) {
  return make_double2(x, y);
}
template <> __device__ __forceinline__ float2 mk<float2>(double x, double y) {
  return make_float2((float)x, (float)y);
}

// Vector access to PTS (1 or 2) consecutive points of a real or complex
// array; point pairs start at even indices, so 2-wide accesses are aligned.
template <typename T> struct V2;
template <> struct V2<float> { typedef float2 t; typedef float4 c; };
template <> struct V2<double> { typedef double2 t; typedef double4 c; };

template <int PTS, typename T>
__device__ __forceinline__ void ldr(const T *__restrict__ p, T (&o)[PTS]) {
  if (PTS == 1) {
    o[0] = p[0];
  } else {
    const typename V2<T>::t w = *reinterpret_cast<const typename V2<T>::t *>(p);
    o[0] = w.x;
    o[PTS - 1] = w.y;
  }
}
template <int PTS, typename T>
__device__ __forceinline__ void str(T *__restrict__ p, const T (&o)[PTS]) {
  if (PTS == 1) {
    p[0] = o[0];
  } else {
    typename V2<T>::t w;
    w.x = o[0];
    w.y = o[PTS - 1];
    *reinterpret_cast<typename V2<T>::t *>(p) = w;
  }
}
template <int PTS, typename C>
__device__ __forceinline__ void ldc(const C *__restrict__ p, C (&o)[PTS]) {
#pragma unroll
  for (int k = 0; k < PTS; ++k) o[k] = p[k];
}
template <int PTS, typename C>
__device__ __forceinline__ void stc(C *__restrict__ p, const C (&o)[PTS]) {
#pragma unroll
  for (int k = 0; k < PTS; ++k) p[k] = o[k];
}
// FP32 complex pairs move as one 16-byte access
template <>
__device__ __forceinline__ void ldc<2, float2>(const float2 *__restrict__ p, float2 (&o)[2]) {
  const float4 w = *reinterpret_cast<const float4 *>(p);
  o[0] = make_float2(w.x, w.y);
  o[1] = make_float2(w.z, w.w);
}
template <>
__device__ __forceinline__ void stc<2, float2>(float2 *__restrict__ p, const float2 (&o)[2]) {
  *reinterpret_cast<float4 *>(p) = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
}

__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float fexp(float x) { return expf(x); }

// calculate_cuda.cu:1-20: KH g = 1 + x (x >= 0) or e^x; HNC g = e^x.
template <int CLOS, typename T>
__device__ __forceinline__ T closure(T x) {
  if (CLOS == 0) return x >= T(0) ? T(1) + x : fexp(x);
  return fexp(x);
}

__device__ __forceinline__ double fexpm1(double x) { return expm1(x); }
__device__ __forceinline__ float fexpm1(float x) { return expm1f(x); }

// C(x0 + d) - C(x0) to the relative precision of the difference itself
// (refinement form).  KH: C(x) - 1 = max(x, 0) + expm1(min(x, 0)), so with
// a = min(x0 + d, 0), b = min(x0, 0)
//   C(x0 + d) - C(x0) = [max(x0 + d, 0) - max(x0, 0)] + e^b expm1(a - b),
// where the linear bracket is d itself when both arguments are >= 0 and
// a - b is d itself when both are < 0: e^x0 expm1(d) on the exponential
// branch, d on the linear one, and in the two mixed cases (|x0| <= |d|)
// x - expm1(x0) and expm1(x) - x0.  One exp and one expm1 per call and no
// branches, so the lanes of a warp never split over the four cases.
template <int CLOS, typename T>
__device__ __forceinline__ T closure_diff(T x0, T d) {
  if (CLOS == 1) return fexp(x0) * fexpm1(d);
  const T x = x0 + d;
  const bool pos = x >= T(0), pos0 = x0 >= T(0);
  const T zero = T(0);
  const T lin = (pos && pos0) ? d : (fmax(x, zero) - fmax(x0, zero));
  const T b = fmin(x0, zero);
  const T da = (!pos && !pos0) ? d : (fmin(x, zero) - b);
  return lin + fexp(b) * fexpm1(da);
}

// Residual of the cycle at the current state: plain h + 1 - C(t - U);
// refinement R0 + h - [C(x0 + d) - C(x0)] (t = d, U = x0, h = L[dc]).
template <int CLOS, bool REF, typename T>
__device__ __forceinline__ T residual(T h, T t, T U, T r0) {
  if (REF) return r0 + h - closure_diff<CLOS>(U, t);
  return h + T(1) - closure<CLOS>(t - U);
}

// Packed FFT input: plain c_SR = C(t - U) - 1 - t; refinement dc = dg - d.
template <int CLOS, bool REF, typename T>
__device__ __forceinline__ T cfun(T t, T U) {
  if (REF) return closure_diff<CLOS>(U, t) - t;
  return closure<CLOS>(t - U) - T(1) - t;
}

// Point index -> (ix, iy, iz), +-1 checkerboard dir = (-1)^(ix+iy+iz)
// (set_ir, fft3d.cu:86-94) and dkf = exp(-i pi sum x_d/n_d)
// (set_kf, fft3d.cu:71-83) as a product of three per-axis phases.
__device__ __forceinline__ void split_index(long long j, const FastDiv &fdx,
                                            const FastDiv &fdy, int &ix, int &iy,
                                            int &iz) {
  const unsigned u = (unsigned)j;                 // N < 2^31
  const unsigned r = fdx.div(u);
  ix = (int)(u - r * fdx.d);
  iz = (int)fdy.div(r);
  iy = (int)(r - (unsigned)iz * fdy.d);
}

template <typename C>
__device__ __forceinline__ void point_phase(long long j, const FastDiv &fdx,
                                            const FastDiv &fdy, const C *tw,
                                            int &ix, int &iy, int &iz, int &dir,
                                            C &dkf) {
  split_index(j, fdx, fdy, ix, iy, iz);
  dir = ((ix + iy + iz) & 1) ? -1 : 1;
  const int nx = (int)fdx.d, ny = (int)fdy.d;
  dkf = cmul(cmul(tw[ix], tw[nx + iy]), tw[nx + ny + iz]);
}

// ---------------------------------------------------------------- pass A
// One straight-line body per update mode (the mode is device state, read
// once per thread): every load of a point is issued before any store.  Each
// thread handles PTS adjacent points (2 for FP32, so each thread keeps as
// many bytes in flight as the FP64 version).
template <typename T, int V, int CLOS, int MODE, int PTS, bool REF>
__device__ __forceinline__ void pass_a_body(const IterArgs<T> &a, int slot, T s1, T s2, T m) {
  typedef typename Cx<T>::t C;
  constexpr int P = (V + 1) / 2;
  const long long n = a.n;
  C *__restrict__ buf = a.buf;
  T *__restrict__ tt = a.t;
  const T *__restrict__ UU = a.U;
  T *__restrict__ Y = a.Y;
  T *__restrict__ RP = a.RP;
  const C *__restrict__ tw = a.tw;
  for (long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * PTS; j < n;
       j += (long long)gridDim.x * blockDim.x * PTS) {
    C zb[P][PTS];
    T tv[V][PTS], Uv[V][PTS], y0[V][PTS], y1[V][PTS], r0[V][PTS];
    if (MODE != 0) {
#pragma unroll
      for (int p = 0; p < P; ++p) ldc<PTS>(buf + (size_t)p * n + j, zb[p]);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      ldr<PTS>(tt + (size_t)v * n + j, tv[v]);
      ldr<PTS>(UU + (size_t)v * n + j, Uv[v]);
      if (REF && MODE != 0) ldr<PTS>(a.R0 + (size_t)v * n + j, r0[v]);
      else {
#pragma unroll
        for (int k = 0; k < PTS; ++k) r0[v][k] = T(0);
      }
      if (MODE == 2) {
        ldr<PTS>(Y + (size_t)v * n + j, y0[v]);
        ldr<PTS>(Y + (size_t)(V + v) * n + j, y1[v]);
      }
    }
    int ix, iy, iz, dir0;
    C dkf[PTS];
    point_phase(j, a.fdx, a.fdy, tw, ix, iy, iz, dir0, dkf[0]);
    if (PTS == 2) dkf[PTS - 1] = cmul(cmul(tw[ix + 1], tw[a.nx + iy]), tw[a.nx + a.ny + iz]);
    T tn[V][PTS];
    if (MODE != 0) {
      T yw[V][PTS], rw[V][PTS];
#pragma unroll
      for (int k = 0; k < PTS; ++k) {
        const int dir = (k & 1) ? -dir0 : dir0;
        // inverse post-twiddle (timekb, fft3d.cu:52-60): (1/V) dir conj(dkf)
        const T sc = (T)a.invvol * (T)dir;
        const C w = mk<C>(dkf[k].x * sc, -dkf[k].y * sc);
        T h[V];
#pragma unroll
        for (int p = 0; p < P; ++p) {
          C z = cmul(zb[p][k], w);
          h[2 * p] = z.x;
          if (2 * p + 1 < V) h[2 * p + 1] = z.y;
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const T R = residual<CLOS, REF>(h[v], tv[v][k], Uv[v][k], r0[v][k]);   // tr
          rw[v][k] = R;
          if (MODE == 1) {                       // newdt0 (Picard)
            yw[v][k] = tv[v][k] + m * R;
            tn[v][k] = tv[v][k] + R;
          } else {                               // newdt (AN2)
            const T y = tv[v][k] + m * R;
            yw[v][k] = y;
            tn[v][k] = y + s1 * (y0[v][k] - y) + s2 * (y1[v][k] - y);
          }
        }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const size_t iv = (size_t)v * n + j;
        str<PTS>(Y + (size_t)slot * V * n + iv, yw[v]);
        str<PTS>(RP + (size_t)slot * V * n + iv, rw[v]);
        str<PTS>(tt + iv, tn[v]);
      }
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v)
#pragma unroll
        for (int k = 0; k < PTS; ++k) tn[v][k] = tv[v][k];
    }
    // closure + c_SR (kh/hnc + trm1mt, calculate_cuda.cu:1-29) and the
    // forward pre-twiddle (timekf, fft3d.cu:41-49): dir * dkf * (c_a + i c_b)
#pragma unroll
    for (int p = 0; p < P; ++p) {
      C out[PTS];
#pragma unroll
      for (int k = 0; k < PTS; ++k) {
        const int dir = (k & 1) ? -dir0 : dir0;
        const C wf = mk<C>(dkf[k].x * dir, dkf[k].y * dir);
        C z;
        z.x = cfun<CLOS, REF>(tn[2 * p][k], Uv[2 * p][k]);
        z.y = (2 * p + 1 < V) ? cfun<CLOS, REF>(tn[2 * p + 1][k], Uv[2 * p + 1][k]) : T(0);
        out[k] = cmul(z, wf);
      }
      stc<PTS>(buf + (size_t)p * n + j, out);
    }
  }
}

// First pass after the loop stopped: snapshot h (Re of the last OZ) and g
// (closure of the t used in that cycle), and when maxstep ended the loop
// apply the pending update as the reference does (iterate.cu:61 runs
// ma->calculate before the step bound is tested).
template <typename T, int V, int CLOS, bool REF>
__device__ void pass_a_final(const IterArgs<T> &a, int mode, int done, int slot, T s1,
                             T s2, T m) {
  typedef typename Cx<T>::t C;
  constexpr int P = (V + 1) / 2;
  const long long n = a.n;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int ix, iy, iz, dir;
    C dkf;
    point_phase(j, a.fdx, a.fdy, a.tw, ix, iy, iz, dir, dkf);
    const T sc = (T)a.invvol * (T)dir;
    const C w = mk<C>(dkf.x * sc, -dkf.y * sc);
    T h[V];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      C z = cmul(a.buf[(size_t)p * n + j], w);
      h[2 * p] = z.x;
      if (2 * p + 1 < V) h[2 * p + 1] = z.y;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const size_t iv = (size_t)v * n + j;
      const T t = a.t[iv];
      if (!REF && a.hout) {
        a.hout[iv] = (double)h[v];
        a.gout[iv] = (double)closure<CLOS>(t - a.U[iv]);
      }
      if (done == 3 && mode != 0) {
        const T R = residual<CLOS, REF>(h[v], t, a.U[iv], REF ? a.R0[iv] : T(0));
        const T y = t + m * R;
        T tn = t + R;
        if (mode == 2) tn = y + s1 * (a.Y[iv] - y) + s2 * (a.Y[(size_t)V * n + iv] - y);
        a.Y[(size_t)slot * V * n + iv] = y;
        a.RP[(size_t)slot * V * n + iv] = R;
        a.t[iv] = tn;
      }
    }
  }
}

// Resident blocks per SM that pass A's register bound asks for: with one
// packed site pair the FP32 plain form fits 64 registers (4 blocks) and the
// FP64 KH plain form 80 (3 blocks) without spills.  Every other form keeps
// the compiler's choice: a bound spills there, or (the FP32 refinement form,
// used when its pipelined pass is off) runs slower at 64 registers.
template <typename T, int V, int CLOS, bool REF> struct PassAOccupancy {
  static constexpr int blocks =
      V > 2 ? 1 : sizeof(T) == 4 ? (REF ? 1 : 4) : (V == 1 || (CLOS == 0 && !REF)) ? 3 : 1;
};

template <typename T, int V, int CLOS, bool REF>
__global__ void __launch_bounds__(kThreads, (PassAOccupancy<T, V, CLOS, REF>::blocks))
    k_pass_a(IterArgs<T> a0) {
  const IterArgs<T> a = solute_view<T, V>(a0);
  const DevState *st = a.st;
  const int done = st->done;
  const int mode = st->mode;
  const int slot = st->upd_slot;
  const T s1 = (T)st->s1, s2 = (T)st->s2, m = (T)st->m;
  if (done) {
    if (st->after_done == 0) pass_a_final<T, V, CLOS, REF>(a, mode, done, slot, s1, s2, m);
    return;                                     // past the snapshot: idle
  }
  constexpr int PTS = (sizeof(T) == 4 && V <= 2) ? 2 : 1;
  if (mode == 2) pass_a_body<T, V, CLOS, 2, PTS, REF>(a, slot, s1, s2, m);
  else if (mode == 1) pass_a_body<T, V, CLOS, 1, PTS, REF>(a, slot, s1, s2, m);
  else pass_a_body<T, V, CLOS, 0, PTS, REF>(a, slot, s1, s2, m);
}

// ---------------------------------------------------------------- pass K
// One mirror pair of k points: j (the owner, j < N/2, grid indices ix iy iz)
// and jm = N-1-j with k(jm) = -k(j).  y/ym are the forward-transformed
// packed site pairs at j and jm; out/outm receive the OZ result repacked
// for the inverse transform.
// fk is beta fk at the owner point (zero when a.nofk).
template <typename T, int V>
__device__ __forceinline__ void kspace_pair_fk(const IterArgs<T> &a, double2 fk, int ix, int iy,
                                               int iz, const typename Cx<T>::t *y,
                                               const typename Cx<T>::t *ym,
                                               typename Cx<T>::t *out, typename Cx<T>::t *outm) {
  typedef typename Cx<T>::t C;
  constexpr int P = (V + 1) / 2;
  const StageParams *sp = a.sp;
  const int dir = ((ix + iy + iz) & 1) ? -1 : 1;
  // unpack the site pairs and finish the forward transform
  // (timeirvol * dv, fft3d.cu:32) and subtract q cf fk (mqvfk)
  // (in the working precision T: the FP32 passes round F to FP32 anyway)
  C F[V];
  const T sc = (T)(a.dv * 0.5 * dir);
  const T fx = (T)fk.x, fy = (T)fk.y;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const T qa = (T)sp->qcf[2 * p];
    F[2 * p] = mk<C>(sc * (y[p].x - ym[p].x) - qa * fx, sc * (y[p].y + ym[p].y) - qa * fy);
    if (2 * p + 1 < V) {
      const T qb = (T)sp->qcf[2 * p + 1];
      F[2 * p + 1] = mk<C>(sc * (y[p].y - ym[p].y) - qb * fx, -sc * (y[p].x + ym[p].x) - qb * fy);
    }
  }
  // chi_ab(|k|) (solvent_spline.cu:36-47, applied per point by oz), in T
  T X[V * V];
  if (a.xs) {
    // cubic cell: |k| = (pi/L) sqrt(s), s = sum of three odd squares
    const int ox = 2 * ix - a.nx + 1, oy = 2 * iy - a.ny + 1, oz = 2 * iz - a.nz + 1;
    const unsigned sq = (unsigned)(ox * ox + oy * oy + oz * oz);
    const size_t row = (size_t)((sq - 3u) >> 3) * V * V;
    if constexpr (sizeof(T) == 4 && V * V % 4 == 0) {
      const float4 *xr = reinterpret_cast<const float4 *>(a.xs32 + row);   // 16-byte rows
#pragma unroll
      for (int ab = 0; ab < V * V / 4; ++ab) {
        const float4 q = xr[ab];
        X[4 * ab] = q.x;
        X[4 * ab + 1] = q.y;
        X[4 * ab + 2] = q.z;
        X[4 * ab + 3] = q.w;
      }
    } else if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int ab = 0; ab < V * V; ++ab) X[ab] = a.xs32[row + ab];
    } else {
      const double2 *xr = reinterpret_cast<const double2 *>(a.xs + row);
#pragma unroll
      for (int ab = 0; ab < V * V / 2; ++ab) {
        const double2 q = xr[ab];
        X[2 * ab] = (T)q.x;
        X[2 * ab + 1] = (T)q.y;
      }
      if (V * V % 2) X[V * V - 1] = (T)a.xs[row + V * V - 1];
    }
  } else {
    // general cell: natural spline on knots k_i = dk (i+1) with the
    // bisection semantics of splint.cc:9-16 on uniform knots
    const double kx = 2.0 * kPi * (ix - a.nx / 2.0 + 0.5) / a.bx;   // set_g
    const double ky = 2.0 * kPi * (iy - a.ny / 2.0 + 0.5) / a.by;
    const double kz = 2.0 * kPi * (iz - a.nz / 2.0 + 0.5) / a.bz;
    const double kk = sqrt(kx * kx + ky * ky + kz * kz);
    int k0 = (int)(kk / a.dk) - 1;
    k0 = k0 < 0 ? 0 : (k0 > a.ntab - 2 ? a.ntab - 2 : k0);
    while (k0 < a.ntab - 2 && a.dk * (k0 + 2) <= kk) ++k0;
    while (k0 > 0 && a.dk * (k0 + 1) > kk) --k0;
    const double tt = kk - a.dk * (k0 + 1);
    const double2 *cf = reinterpret_cast<const double2 *>(a.chi + (size_t)k0 * V * V * 4);
#pragma unroll
    for (int ab = 0; ab < V * V; ++ab) {
      const double2 lo = cf[2 * ab], hi2 = cf[2 * ab + 1];
      X[ab] = (T)(((hi2.y * tt + hi2.x) * tt + lo.y) * tt + lo.x);
    }
  }
  C H[V];
#pragma unroll
  for (int va = 0; va < V; ++va) {
    T hr = 0, hi = 0;
#pragma unroll
    for (int vb = 0; vb < V; ++vb) {
      const T x = X[va * V + vb];
      hr += F[vb].x * x;                       // oz, calculate_cuda.cu:44-58
      hi += F[vb].y * x;
    }
    H[va] = mk<C>(hr, hi);
  }
  // repack for the inverse: dir (h_a + i h_b) at k and its mirror
  // (timeirvol before the inverse, fft3d.cu:34)
  const T d = (T)dir;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const C ha = H[2 * p];
    const C hb = (2 * p + 1 < V) ? H[2 * p + 1] : mk<C>(0.0, 0.0);
    out[p] = mk<C>(d * (ha.x - hb.y), d * (ha.y + hb.x));
    outm[p] = mk<C>(-d * (ha.x + hb.y), -d * (hb.x - ha.y));
  }
}

template <typename T, int V>
__device__ __forceinline__ void kspace_pair(const IterArgs<T> &a, long long j, int ix, int iy,
                                            int iz, const typename Cx<T>::t *y,
                                            const typename Cx<T>::t *ym,
                                            typename Cx<T>::t *out, typename Cx<T>::t *outm) {
  const double2 fk = a.nofk ? make_double2(0.0, 0.0) : a.fkh[j];
  kspace_pair_fk<T, V>(a, fk, ix, iy, iz, y, ym, out, outm);
}

template <typename T, int V>
__global__ void __launch_bounds__(kThreads) k_kspace(IterArgs<T> a0) {
  const IterArgs<T> a = solute_view<T, V>(a0);
  typedef typename Cx<T>::t C;
  constexpr int P = (V + 1) / 2;
  if (a.st->done) return;
  const long long n = a.n, nh = n / 2;
  C *__restrict__ buf = a.buf;
  if constexpr (sizeof(T) == 4 && P == 1) {
    // FP32, one site pair: two neighbouring owner points j, j + 1 (j even,
    // same x row) and their mirrors jm - 1, jm per thread, each pair of
    // complex values one 16-byte access, so twice the bytes are in flight
    for (long long j = 2 * ((long long)blockIdx.x * blockDim.x + threadIdx.x); j < nh;
         j += 2 * (long long)gridDim.x * blockDim.x) {
      const long long jm = n - 1 - j;           // k(jm) = -k(j); jm - 1 mirrors j + 1
      const float4 w = *reinterpret_cast<const float4 *>(buf + j);
      const float4 wm = *reinterpret_cast<const float4 *>(buf + jm - 1);
      int ix, iy, iz;
      split_index(j, a.fdx, a.fdy, ix, iy, iz);
      C y0[1] = {make_float2(w.x, w.y)}, y1[1] = {make_float2(w.z, w.w)};
      C ym0[1] = {make_float2(wm.z, wm.w)}, ym1[1] = {make_float2(wm.x, wm.y)};
      C o0[1], om0[1], o1[1], om1[1];
      kspace_pair<T, V>(a, j, ix, iy, iz, y0, ym0, o0, om0);
      kspace_pair<T, V>(a, j + 1, ix + 1, iy, iz, y1, ym1, o1, om1);
      *reinterpret_cast<float4 *>(buf + j) = make_float4(o0[0].x, o0[0].y, o1[0].x, o1[0].y);
      *reinterpret_cast<float4 *>(buf + jm - 1) =
          make_float4(om1[0].x, om1[0].y, om0[0].x, om0[0].y);
    }
    return;
  }
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nh;
       j += (long long)gridDim.x * blockDim.x) {
    const long long jm = n - 1 - j;             // k(jm) = -k(j)
    int ix, iy, iz;
    split_index(j, a.fdx, a.fdy, ix, iy, iz);
    C y[P], ym[P], o[P], om[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      y[p] = buf[(size_t)p * n + j];
      ym[p] = buf[(size_t)p * n + jm];
    }
    kspace_pair<T, V>(a, j, ix, iy, iz, y, ym, o, om);
#pragma unroll
    for (int p = 0; p < P; ++p) {
      buf[(size_t)p * n + j] = o[p];
      buf[(size_t)p * n + jm] = om[p];
    }
  }
}


// ---------------------------------------------------------------- pass R
__device__ void finalize_block(DevState *st, const double *part, int nblocks,
                               double nv_points, double *hist, int hist_cap);

template <typename T, int V, int CLOS, bool REF>
__global__ void __launch_bounds__(kThreads) k_pass_r(IterArgs<T> a0) {
  const IterArgs<T> a = solute_view<T, V>(a0);
  typedef typename Cx<T>::t C;
  constexpr int P = (V + 1) / 2;
  constexpr int PTS = sizeof(T) == 4 ? 2 : 1;
  __shared__ double red[kThreads / 32][6];
  __shared__ bool last;
  DevState *st = a.st;
  if (st->done) {                                // loop stopped: count idle cycles
    if (blockIdx.x == 0 && threadIdx.x == 0) st->after_done += 1;
    return;
  }
  const bool gram = st->count <= 0;
  const long long n = a.n;
  const StageParams *sp = a.sp;
  const C *__restrict__ buf = a.buf;
  const T *__restrict__ tt = a.t;
  const T *__restrict__ UU = a.U;
  const T *__restrict__ RP = a.RP;
  const C *__restrict__ tw = a.tw;
  double w8[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w8[v] = sp->irho[v];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * PTS; j < n;
       j += (long long)gridDim.x * blockDim.x * PTS) {
    C zb[P][PTS];
    T tv[V][PTS], Uv[V][PTS], r0[V][PTS], r1[V][PTS], rb[V][PTS];
#pragma unroll
    for (int p = 0; p < P; ++p) ldc<PTS>(buf + (size_t)p * n + j, zb[p]);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      ldr<PTS>(tt + (size_t)v * n + j, tv[v]);
      ldr<PTS>(UU + (size_t)v * n + j, Uv[v]);
      if (REF) ldr<PTS>(a.R0 + (size_t)v * n + j, rb[v]);
      else {
#pragma unroll
        for (int k = 0; k < PTS; ++k) rb[v][k] = T(0);
      }
      if (gram) {
        ldr<PTS>(RP + (size_t)v * n + j, r0[v]);
        ldr<PTS>(RP + (size_t)(V + v) * n + j, r1[v]);
      }
    }
    int ix, iy, iz, dir0;
    C dkf[PTS];
    point_phase(j, a.fdx, a.fdy, tw, ix, iy, iz, dir0, dkf[0]);
    if (PTS == 2) dkf[PTS - 1] = cmul(cmul(tw[ix + 1], tw[a.nx + iy]), tw[a.nx + a.ny + iz]);
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
      const int dir = (k & 1) ? -dir0 : dir0;
      const T sc = (T)a.invvol * (T)dir;
      const C w = mk<C>(dkf[k].x * sc, -dkf[k].y * sc);
      T h[V];
#pragma unroll
      for (int p = 0; p < P; ++p) {
        C z = cmul(zb[p][k], w);
        h[2 * p] = z.x;
        if (2 * p + 1 < V) h[2 * p + 1] = z.y;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double R = (double)residual<CLOS, REF>(h[v], tv[v][k], Uv[v][k], rb[v][k]);
        acc[0] += R * R;                          // cal_rms.cu:18
        if (gram) {                               // theta30, anderson_cuda.cu:33-39
          const double d0 = R - (double)r0[v][k];
          const double d1 = R - (double)r1[v][k];
          acc[1] += w8[v] * R * d0;
          acc[2] += w8[v] * R * d1;
          acc[3] += w8[v] * d0 * d0;
          acc[4] += w8[v] * d0 * d1;
          acc[5] += w8[v] * d1 * d1;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 6; ++k) red[wid][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
    a.part[(size_t)threadIdx.x * a.nblocks + blockIdx.x] = s;
  }
  // the last block to finish reduces all block sums and steers the loop
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_block(st, a.part, a.nblocks, (double)n * V, a.hist, a.hist_cap);
  if (threadIdx.x == 0) *a.count = 0u;
}

// --------------------------------------------- passes with a fused axis
// FP32 single-solute solves on grids with nx = ny = E^2 (E = 8 or 16) fold
// two axes of each 3D transform into the streaming passes, so that cuFFT
// only transforms along z (one strided pass per direction, c.plan32z):
//   k_pass_ax  inverse x-DFT of the last OZ result + pass A + forward x-DFT
//   cuFFT z    forward
//   k_kspace_y forward y-DFT + pass K + inverse y-DFT (owner/mirror tiles)
//   cuFFT z    inverse
//   k_pass_rx  inverse x-DFT + pass R (residual sums, finalize)
// DFTs along different axes commute, so passes K and R see the same values
// as on the 3D cuFFT path.  An x line of E^2 points is held by a group of E
// consecutive lanes, E points each (xfft.cuh); the half-shift twiddles are
// applied per point as in the unfused passes.
constexpr int kXThreads = 256;

template <int V, int CLOS, bool REF, int E>
__global__ void __launch_bounds__(kXThreads, 4) k_pass_ax(IterArgs<float> a) {
  constexpr int NX = E * E, LPB = kXThreads / E, P = (V + 1) / 2;
  __shared__ float2 scr[LPB][(E + 1) * E];
  const DevState *st = a.st;
  const int done = st->done, mode = st->mode, slot = st->upd_slot;
  if (done && st->after_done != 0) return;      // past the snapshot: idle
  const float s1 = (float)st->s1, s2 = (float)st->s2, m = (float)st->m;
  const long long n = a.n;
  const int g = threadIdx.x / E, t = threadIdx.x % E;
  const unsigned mask = (E == 16) ? (0xffffu << (threadIdx.x & 16)) : (0xffu << (threadIdx.x & 24));
  const int lines = a.ny * a.nz;
  const float2 *tw = a.tw;
  const float iv = (float)a.invvol;
  const bool need_h = done || mode != 0;
  for (int line = blockIdx.x * LPB + g; line < lines; line += gridDim.x * LPB) {
    const int iy = line % a.ny, iz = line / a.ny;
    const size_t base = (size_t)line * NX;
    const float2 twyz = cmul(tw[NX + iy], tw[NX + a.ny + iz]);
    const int dyz = (iy + iz) & 1;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
      float2 z[E];
      float2 *zs = scr[g];                    // the line, point ix = t + E k at zs[k E + t]
      if (need_h) {
#pragma unroll
        for (int j = 0; j < E; ++j) z[j] = a.buf[(size_t)p * n + base + t + E * j];
        xfft::line_dft<E, true>(z, t, scr[g], a.xroots, mask);   // z[k] at ix = t + E k
      }
      __syncwarp(mask);                       // the transpose's reads are done
      if (need_h)
#pragma unroll
        for (int k = 0; k < E; ++k) zs[k * E + t] = z[k];
      // per point: one copy of the body (the refinement closure inlined for
      // every point of an unrolled loop overflowed the instruction cache)
#pragma unroll 1
      for (int k = 0; k < E; ++k) {
        const int ix = t + E * k;
        const size_t j = base + ix;
        const float dir = ((ix & 1) ^ dyz) ? -1.0f : 1.0f;
        const float2 dkf = cmul(tw[ix], twyz);
        float h[2] = {0.0f, 0.0f};
        if (need_h) {
          // inverse post-twiddle (timekb, fft3d.cu:52-60): (1/V) dir conj(dkf)
          const float sc = iv * dir;
          const float2 zz = cmul(zs[k * E + t], make_float2(dkf.x * sc, -dkf.y * sc));
          h[0] = zz.x;
          h[1] = zz.y;
        }
        float cv[2] = {0.0f, 0.0f};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int v = 2 * p + q;
          if (v >= V) break;
          const size_t i2 = (size_t)v * n + j;
          const float tv = a.t[i2], Uv = a.U[i2];
          if (done) {                           // pass_a_final, fused form
            if (!REF && a.hout) {
              a.hout[i2] = (double)h[q];
              a.gout[i2] = (double)closure<CLOS>(tv - Uv);
            }
            if (done == 3 && mode != 0) {
              const float r0 = REF ? a.R0[i2] : 0.0f;
              const float R = residual<CLOS, REF>(h[q], tv, Uv, r0);
              const float y = tv + m * R;
              float tn = tv + R;
              if (mode == 2) tn = y + s1 * (a.Y[i2] - y) + s2 * (a.Y[(size_t)V * n + i2] - y);
              a.Y[(size_t)slot * V * n + i2] = y;
              a.RP[(size_t)slot * V * n + i2] = R;
              a.t[i2] = tn;
            }
            continue;
          }
          float tn = tv;
          if (mode != 0) {
            const float r0 = REF ? a.R0[i2] : 0.0f;
            const float R = residual<CLOS, REF>(h[q], tv, Uv, r0);   // tr
            const float y = tv + m * R;
            if (mode == 1) tn = tv + R;                              // newdt0 (Picard)
            else tn = y + s1 * (a.Y[i2] - y) + s2 * (a.Y[(size_t)V * n + i2] - y);  // newdt (AN2)
            a.Y[(size_t)slot * V * n + i2] = y;
            a.RP[(size_t)slot * V * n + i2] = R;
            a.t[i2] = tn;
          }
          cv[q] = cfun<CLOS, REF>(tn, Uv);
        }
        // forward pre-twiddle (timekf, fft3d.cu:41-49): dir dkf (c_a + i c_b)
        zs[k * E + t] = cmul(make_float2(cv[0], cv[1]), make_float2(dkf.x * dir, dkf.y * dir));
      }
#pragma unroll
      for (int k = 0; k < E; ++k) z[k] = zs[k * E + t];
      if (done) continue;
      xfft::line_dft<E, false>(z, t, scr[g], a.xroots, mask);    // z[k] at kx = t + E k
#pragma unroll
      for (int k = 0; k < E; ++k) a.buf[(size_t)p * n + base + t + E * k] = z[k];
    }
  }
}

template <int V, int CLOS, bool REF, int E>
__global__ void __launch_bounds__(kXThreads, 3) k_pass_rx(IterArgs<float> a) {
  constexpr int NX = E * E, LPB = kXThreads / E, P = (V + 1) / 2;
  __shared__ float2 scr[LPB][(E + 1) * E];
  __shared__ double red[kXThreads / 32][6];
  __shared__ bool last;
  DevState *st = a.st;
  if (st->done) {                                // loop stopped: count idle cycles
    if (blockIdx.x == 0 && threadIdx.x == 0) st->after_done += 1;
    return;
  }
  const bool gram = st->count <= 0;
  const long long n = a.n;
  const int g = threadIdx.x / E, t = threadIdx.x % E;
  const unsigned mask = (E == 16) ? (0xffffu << (threadIdx.x & 16)) : (0xffu << (threadIdx.x & 24));
  const int lines = a.ny * a.nz;
  const float2 *tw = a.tw;
  const float iv = (float)a.invvol;
  double w8[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w8[v] = a.sp->irho[v];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int line = blockIdx.x * LPB + g; line < lines; line += gridDim.x * LPB) {
    const int iy = line % a.ny, iz = line / a.ny;
    const size_t base = (size_t)line * NX;
    const float2 twyz = cmul(tw[NX + iy], tw[NX + a.ny + iz]);
    const int dyz = (iy + iz) & 1;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
      float2 z[E];
      float2 *zs = scr[g];
#pragma unroll
      for (int j = 0; j < E; ++j) z[j] = a.buf[(size_t)p * n + base + t + E * j];
      xfft::line_dft<E, true>(z, t, scr[g], a.xroots, mask);
      __syncwarp(mask);
#pragma unroll
      for (int k = 0; k < E; ++k) zs[k * E + t] = z[k];
#pragma unroll 2
      for (int k = 0; k < E; ++k) {
        const int ix = t + E * k;
        const size_t j = base + ix;
        const float dir = ((ix & 1) ^ dyz) ? -1.0f : 1.0f;
        const float2 dkf = cmul(tw[ix], twyz);
        const float sc = iv * dir;
        const float2 zz = cmul(zs[k * E + t], make_float2(dkf.x * sc, -dkf.y * sc));
        const float h[2] = {zz.x, zz.y};
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int v = 2 * p + q;
          if (v >= V) break;
          const size_t i2 = (size_t)v * n + j;
          const float rb = REF ? a.R0[i2] : 0.0f;
          const double R = (double)residual<CLOS, REF>(h[q], a.t[i2], a.U[i2], rb);
          acc[0] += R * R;                          // cal_rms.cu:18
          if (gram) {                               // theta30, anderson_cuda.cu:33-39
            const double d0 = R - (double)a.RP[i2];
            const double d1 = R - (double)a.RP[(size_t)V * n + i2];
            acc[1] += w8[v] * R * d0;
            acc[2] += w8[v] * R * d1;
            acc[3] += w8[v] * d0 * d0;
            acc[4] += w8[v] * d0 * d1;
            acc[5] += w8[v] * d1 * d1;
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 6; ++k) red[wid][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kXThreads / 32; ++w) s += red[w][threadIdx.x];
    a.part[(size_t)threadIdx.x * a.nblocks + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_block(st, a.part, a.nblocks, (double)n * V, a.hist, a.hist_cap);
  if (threadIdx.x == 0) *a.count = 0u;
}

// Pass K with the y-axis DFTs folded in (one site pair, P = 1).  A block
// owns the tile of kW consecutive kx columns at one kz < nz/2 and the mirror
// tile (columns nx - c0 - kW .. nx - c0 - 1 at nz - 1 - kz), so that every
// owner point k and its mirror -k meet in the block: forward y-DFT of both
// tiles into shared memory, the OZ pair product of kspace_pair on every
// owner point, inverse y-DFT, with the buffer read and written once.  Thread
// (col, t) moves the points y = t + E j of column col of each tile; a
// column's E threads sit kW apart in the block, so the transposes of the
// y-DFT go through shared memory behind block-wide barriers.
constexpr int kW = 16;

template <int E>
struct KYLayout {
  static constexpr int NY = E * E;
  static constexpr int SCOL = (E + 1) * E + 1;   // transpose scratch per column
  static constexpr int MROW = NY + 1;            // one tile column of ky values
  static constexpr size_t bytes() {
    return sizeof(float2) * ((size_t)kW * SCOL + (size_t)kW * MROW);
  }
};

// y-DFT of one tile column group: v in (points y = t + E j) and out
// (ky = t + E k), optionally also to the tile array T[col][ky].
template <int E, bool INV>
__device__ __forceinline__ void col_dft_to(float2 (&v)[E], int col, int t, float2 *scr,
                                          float2 *T, const float2 *__restrict__ roots) {
  using L = KYLayout<E>;
  xfft::stage1<E, INV>(v, t, roots);
  __syncthreads();                               // scratch free
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) scr[col * L::SCOL + k1 * (E + 1) + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int s = 0; s < E; ++s) v[s] = scr[col * L::SCOL + t * (E + 1) + s];
  xfft::dft_small<E, INV>(v);
  if (T)
#pragma unroll
    for (int k = 0; k < E; ++k) T[col * L::MROW + t + E * k] = v[k];
}

template <int V, int E>
__global__ void __launch_bounds__(kW * E, 2) k_kspace_y(IterArgs<float> a) {
  using L = KYLayout<E>;
  constexpr int NY = L::NY;
  extern __shared__ float2 ksm[];
  float2 *scr = ksm;                             // [kW][SCOL]
  float2 *M = ksm + (size_t)kW * L::SCOL;        // mirror tile [kW][MROW]
  if (a.st->done) return;
  const int nx = a.nx, nz = a.nz;
  const int col = threadIdx.x % kW, t = threadIdx.x / kW;
  const int cblocks = nx / kW, tiles = cblocks * (nz / 2);
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int cb = tile % cblocks, kz = tile / cblocks, kzm = nz - 1 - kz;
    const int kx = cb * kW + col, kxm = nx - cb * kW - kW + col;
    float2 v[E], vm[E];
#pragma unroll
    for (int j = 0; j < E; ++j) vm[j] = a.buf[((size_t)kzm * NY + t + E * j) * nx + kxm];
    col_dft_to<E, false>(vm, col, t, scr, M, a.xroots);
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = a.buf[((size_t)kz * NY + t + E * j) * nx + kx];
    col_dft_to<E, false>(v, col, t, scr, nullptr, a.xroots);   // owner stays in registers
    __syncthreads();                             // M complete
    // owner point (kx, ky, kz), ky = t + E k, and its mirror (nx-1-kx,
    // ny-1-ky, nz-1-kz): column kW-1-col, row NY-1-ky of the mirror tile
#pragma unroll 2
    for (int k = 0; k < E; ++k) {
      const int ky = t + E * k;
      const long long j = (long long)kx + (long long)nx * (ky + (long long)NY * kz);
      float2 *mp = M + (kW - 1 - col) * L::MROW + (NY - 1 - ky);
      float2 y[1] = {v[k]}, ym[1] = {*mp}, o[1], om[1];
      kspace_pair<float, V>(a, j, kx, ky, kz, y, ym, o, om);
      v[k] = o[0];
      *mp = om[0];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < E; ++j) vm[j] = M[col * L::MROW + t + E * j];
    col_dft_to<E, true>(v, col, t, scr, nullptr, a.xroots);
    col_dft_to<E, true>(vm, col, t, scr, nullptr, a.xroots);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int y = t + E * j;
      a.buf[((size_t)kz * NY + y) * nx + kx] = v[j];
      a.buf[((size_t)kzm * NY + y) * nx + kxm] = vm[j];
    }
  }
}



// Pass K with the y-axis DFTs folded in, TMA form (nx = ny = 256, one site
// pair).  A tile is 16 consecutive kx columns x 256 ky rows at one kz < nz/2
// (32 KB of FP32 complex values) together with its mirror tile (columns
// nx - c0 - 16 .. nx - c0 - 1 at nz - 1 - kz).  The TMA unit fetches both
// into one of three shared-memory stages (128-byte rows, 128B swizzle) two
// tiles ahead of the one being transformed, and tile stores write the
// results back from the same stage, so the block's threads never issue a
// global load or store of the grid themselves.
//
// Warp w transforms owner column w (lanes 0-15) and mirror column 15 - w
// (lanes 16-31).  Lane t holds the points y = t + 16 j of its column; the
// transpose of each 256-point DFT runs in place in the column's own
// shared-memory slots (skewed so that both of its sides are free of bank
// conflicts) behind __syncwarp only.  After the forward DFT the mirror of
// owner point ky = t + 16 k (-k: nx-1-kx, ny-1-ky, nz-1-kz) sits in lane
// t ^ 31 at register 15 - k, so a lane takes half of its column's
// owner/mirror pairs with one shuffle each way.  beta fk comes from an FP32
// copy laid out [kz][kx][ky] (ky fastest): the pairs of one step of a warp
// read two runs of 16 consecutive values.  (Only the plain FP32 bulk reads
// fk: the refinement form cancels it and the FP64 cycles use the FP64 grid,
// so its FP32 rounding stays below the bulk's own rounding floor.)
constexpr int kKyThreads = 512;
constexpr int kKyStages = 3;
constexpr unsigned kKyTileBytes = 16u * 256u * (unsigned)sizeof(float2);
constexpr size_t kKySmem = (size_t)kKyStages * 2 * kKyTileBytes + 1024;   // + alignment
constexpr long long kKyWaitPolls = 1LL << 24;

// byte offset of float2 (row r, column c) in a tile of 16-column rows
// stored with the 128B swizzle (16-byte chunk index XOR row mod 8)
__device__ __forceinline__ unsigned ky_swz(int r, int c) {
  return (unsigned)r * 128u + ((((unsigned)c >> 1) ^ ((unsigned)r & 7u)) << 4) +
         (((unsigned)c & 1u) << 3);
}

// 256-point DFT of one tile column held by 16 lanes (v[j] = x[t + 16 j] in,
// v[k] = X[t + 16 k] out); the transpose goes through the column's slots:
// A_t[k1] is stored at row 16 k1 + ((t + k1) mod 16).
template <bool INV>
__device__ __forceinline__ void ky_col_dft(float2 (&v)[16], int t, unsigned char *tile, int c,
                                           const float2 *__restrict__ roots) {
  xfft::stage1<16, INV>(v, t, roots);
  __syncwarp();                                  // the column's inputs are all read
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1)
    *reinterpret_cast<float2 *>(tile + ky_swz(16 * k1 + ((t + k1) & 15), c)) = v[k1];
  __syncwarp();
#pragma unroll
  for (int s = 0; s < 16; ++s)
    v[s] = *reinterpret_cast<const float2 *>(tile + ky_swz(16 * t + ((s + t) & 15), c));
  xfft::dft_small<16, INV>(v);
}

template <int V>
__global__ void __launch_bounds__(kKyThreads, 1)
    k_kspace_yt(IterArgs<float> a, const __grid_constant__ CUtensorMap map) {
  constexpr int NY = 256;
  extern __shared__ unsigned char ky_raw[];
  __shared__ __align__(8) uint64_t full[kKyStages];
  DevState *st = a.st;
  if (st->done) return;
  unsigned char *sm =
      reinterpret_cast<unsigned char *>(((uintptr_t)ky_raw + 1023) & ~(uintptr_t)1023);
  const int nx = a.nx, nz = a.nz;
  const int cblocks = nx / 16, tiles = cblocks * (nz / 2);
  const int mine = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, t = lane & 15;
  const bool own = lane < 16;
  const int c = own ? w : 15 - w;                // this half-warp's column in its tile
  const unsigned half = own ? 0u : kKyTileBytes;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kKyStages; ++s) tma::mbar_init(&full[s], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  // thread 0: fetch this block's tile i (owner and mirror) into stage i mod 3
  auto fetch = [&](int i) {
    const int tile = (int)blockIdx.x + i * (int)gridDim.x;
    const int cb = tile % cblocks, kz = tile / cblocks;
    unsigned char *dst = sm + (size_t)(i % kKyStages) * 2 * kKyTileBytes;
    uint64_t *bar = &full[i % kKyStages];
    tma::mbar_arrive_expect_tx(bar, 2 * kKyTileBytes);
    tma::load_2d(dst, &map, bar, 2 * 16 * cb, kz * NY);
    tma::load_2d(dst + kKyTileBytes, &map, bar, 2 * (nx - 16 * cb - 16), (nz - 1 - kz) * NY);
  };
  int fetched = 0;
  if (threadIdx.x == 0)
    for (; fetched < 2 && fetched < mine; ++fetched) fetch(fetched);
  int fault = 0, i = 0;
  for (; i < mine; ++i) {
    const int tile = (int)blockIdx.x + i * (int)gridDim.x;
    const int cb = tile % cblocks, kz = tile / cblocks;
    const int kx = 16 * cb + w;                  // the warp's owner column
    // beta fk at the owner points of this lane's eight pairs, before the wait
    float2 fk[8];
    if (a.nofk) {
#pragma unroll
      for (int k = 0; k < 8; ++k) fk[k] = make_float2(0.0f, 0.0f);
    } else {
      const float2 *fc = a.fkt + ((size_t)kz * nx + kx) * NY;
#pragma unroll
      for (int k = 0; k < 8; ++k) fk[k] = fc[own ? t + 16 * k : (15 - t) + 16 * (15 - k)];
    }
    // (warp-uniform, so that the shuffles below always run on full warps)
    const bool ready = __all_sync(0xffffffffu, tma::mbar_wait_bounded(&full[i % kKyStages],
                                                                      (unsigned)(i / kKyStages) & 1u,
                                                                      kKyWaitPolls));
    unsigned char *col = sm + (size_t)(i % kKyStages) * 2 * kKyTileBytes + half;
    if (ready) {
      float2 v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = *reinterpret_cast<const float2 *>(col + ky_swz(t + 16 * j, c));
      ky_col_dft<false>(v, t, col, c, a.xroots);
      // owner lane t: pairs k = 0..7 of its column; mirror lane t ^ 31:
      // the owner registers 15..8 of lane t
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float2 p;
        p.x = __shfl_xor_sync(0xffffffffu, v[15 - k].x, 31);
        p.y = __shfl_xor_sync(0xffffffffu, v[15 - k].y, 31);
        const int ky = own ? t + 16 * k : (15 - t) + 16 * (15 - k);
        float2 y[1] = {own ? v[k] : p}, ym[1] = {own ? p : v[k]}, o[1], om[1];
        kspace_pair_fk<float, V>(a, make_double2(fk[k].x, fk[k].y), kx, ky, kz, y, ym, o, om);
        v[k] = own ? o[0] : om[0];
        const float2 back = own ? om[0] : o[0];
        v[15 - k].x = __shfl_xor_sync(0xffffffffu, back.x, 31);
        v[15 - k].y = __shfl_xor_sync(0xffffffffu, back.y, 31);
      }
      ky_col_dft<true>(v, t, col, c, a.xroots);
      __syncwarp();                              // the transpose's reads are done
#pragma unroll
      for (int j = 0; j < 16; ++j) *reinterpret_cast<float2 *>(col + ky_swz(t + 16 * j, c)) = v[j];
    }
    tma::fence_proxy_async();                    // the stage's writes, before the TMA reads them
    fault = __syncthreads_or(!ready);
    if (fault) break;
    if (threadIdx.x == 0) {
      const unsigned char *src = sm + (size_t)(i % kKyStages) * 2 * kKyTileBytes;
      tma::store_2d(&map, src, 2 * 16 * cb, kz * NY);
      tma::store_2d(&map, src + kKyTileBytes, 2 * (nx - 16 * cb - 16), (nz - 1 - kz) * NY);
      tma::bulk_commit();
      if (fetched < mine) {
        tma::bulk_wait_read<1>();                // that stage's previous tile is stored
        fetch(fetched++);
      }
    }
  }
  if (threadIdx.x == 0) {
    if (fault) {
      // a tile never arrived: wait (bounded) for every fetch still in flight
      // before the block's shared memory goes away, then stop the loop
      for (int f = i; f < fetched; ++f)
        tma::mbar_wait_bounded(&full[f % kKyStages], (unsigned)(f / kKyStages) & 1u, kKyWaitPolls);
      st->fault = 1;
      st->done = 2;
    }
    tma::bulk_wait<0>();
  }
}

// beta fk re-laid out for k_kspace_yt: each kz plane of the owner half
// transposed from [ky][kx] to [kx][ky] and rounded to FP32, 32 x 32 tiles
// through shared memory.
__global__ void k_fk_columns(int nx, int ny, const double2 *__restrict__ fkh,
                             float2 *__restrict__ fkt) {
  __shared__ double2 tile[32][33];
  const size_t plane = (size_t)blockIdx.z * nx * ny;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int x = x0 + threadIdx.x, y = y0 + r;
    if (x < nx && y < ny) tile[r][threadIdx.x] = fkh[plane + (size_t)y * nx + x];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int x = x0 + r, y = y0 + threadIdx.x;
    if (x < nx && y < ny)
      fkt[plane + (size_t)x * ny + y] =
          make_float2((float)tile[threadIdx.x][r].x, (float)tile[threadIdx.x][r].y);
  }
}

// Pass R as a software pipeline (V <= 2, one packed site pair): a block
// walks chunks of kThreads * PTS consecutive points (PTS = 16 bytes of T),
// and each thread copies its own 16-byte slice of every input of the NEXT
// chunk into its private shared-memory slots with cp.async while it works
// on the current one, two stages deep.  A thread reads back only what it
// copied, so no block barrier is needed; the loads in flight per SM are
// those of a whole chunk per resident block (the plain pass R holds only
// what its registers can).
constexpr int kPipeStages = 2;

__device__ __forceinline__ void cp16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// slots of one thread in one stage (16-byte units): buf (2: PTS complex
// points), t[V], U[V], RP0[V], RP1[V], R0[V]
template <int V> struct PipeSlots {
  static constexpr int BUF = 0, T = 2, U = 2 + V, RP0 = 2 + 2 * V, RP1 = 2 + 3 * V,
                       R0 = 2 + 4 * V, N = 2 + 5 * V;
};

template <typename T, int V>
constexpr size_t pass_r_pipe_smem() {
  return (size_t)16 * PipeSlots<V>::N * kPipeStages * kThreads;
}

template <typename T, int V, int CLOS, bool REF>
__global__ void __launch_bounds__(kThreads) k_pass_r_pipe(IterArgs<T> a0) {
  static_assert(V <= 2, "one packed site pair");
  const IterArgs<T> a = solute_view<T, V>(a0);
  typedef typename Cx<T>::t C;
  constexpr int PTS = 16 / sizeof(T);            // points per 16-byte slice
  constexpr int CP = kThreads * PTS;             // points per chunk
  using S = PipeSlots<V>;
  extern __shared__ float4 pipe_sm[];
  __shared__ double red[kThreads / 32][6];
  __shared__ bool last;
  DevState *st = a.st;
  if (st->done) {                                // loop stopped: count idle cycles
    if (blockIdx.x == 0 && threadIdx.x == 0) st->after_done += 1;
    return;
  }
  const bool gram = st->count <= 0;
  const long long n = a.n;
  const StageParams *sp = a.sp;
  const C *tw = a.tw;
  double w8[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w8[v] = sp->irho[v];
  // this thread's slots: [stage][slot], 16 bytes each, interleaved by thread
  auto slot = [&](int stage, int k) -> float4 * {
    return pipe_sm + ((size_t)(stage * S::N + k) * kThreads + threadIdx.x);
  };
  const long long nchunks = (n + CP - 1) / CP;
  auto issue = [&](long long c, int stage) {
    const long long j = c * CP + (long long)threadIdx.x * PTS;
    if (c < nchunks && j < n) {
      cp16(slot(stage, S::BUF), a.buf + j);
      cp16(slot(stage, S::BUF + 1), a.buf + j + PTS / 2);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        cp16(slot(stage, S::T + v), a.t + (size_t)v * n + j);
        cp16(slot(stage, S::U + v), a.U + (size_t)v * n + j);
        if (gram) {
          cp16(slot(stage, S::RP0 + v), a.RP + (size_t)v * n + j);
          cp16(slot(stage, S::RP1 + v), a.RP + (size_t)(V + v) * n + j);
        }
        if (REF) cp16(slot(stage, S::R0 + v), a.R0 + (size_t)v * n + j);
      }
    }
    cp_commit();                                 // an empty group keeps the count
  };
  double acc[6] = {0, 0, 0, 0, 0, 0};
  long long c = blockIdx.x;
  issue(c, 0);
  for (int stage = 0; c < nchunks; c += gridDim.x, stage ^= 1) {
    issue(c + gridDim.x, stage ^ 1);             // the next chunk, in flight meanwhile
    cp_wait<1>();                                // this chunk's slices have landed
    const long long j = c * CP + (long long)threadIdx.x * PTS;
    if (j >= n) continue;
    // PTS complex points over two 16-byte slots (PTS / 2 in each)
    const T *bz0 = reinterpret_cast<const T *>(slot(stage, S::BUF));
    const T *bz1 = reinterpret_cast<const T *>(slot(stage, S::BUF + 1));
    int ix, iy, iz, dir0;
    C dkf[PTS];
    point_phase(j, a.fdx, a.fdy, tw, ix, iy, iz, dir0, dkf[0]);
    {
      const C tyz = cmul(tw[a.nx + iy], tw[a.nx + a.ny + iz]);
#pragma unroll
      for (int k = 1; k < PTS; ++k) dkf[k] = cmul(tw[ix + k], tyz);
    }
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
      const int dir = (k & 1) ? -dir0 : dir0;
      const T sc = (T)a.invvol * (T)dir;
      const C w = mk<C>(dkf[k].x * sc, -dkf[k].y * sc);
      const T *bz = k < PTS / 2 ? bz0 + 2 * k : bz1 + 2 * (k - PTS / 2);
      C zz;
      zz.x = bz[0];
      zz.y = bz[1];
      const C z = cmul(zz, w);
      const T h[2] = {z.x, z.y};
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T tv = reinterpret_cast<const T *>(slot(stage, S::T + v))[k];
        const T Uv = reinterpret_cast<const T *>(slot(stage, S::U + v))[k];
        const T rb = REF ? reinterpret_cast<const T *>(slot(stage, S::R0 + v))[k] : T(0);
        const double R = (double)residual<CLOS, REF>(h[v], tv, Uv, rb);
        acc[0] += R * R;                          // cal_rms.cu:18
        if (gram) {                               // theta30, anderson_cuda.cu:33-39
          const double d0 = R - (double)reinterpret_cast<const T *>(slot(stage, S::RP0 + v))[k];
          const double d1 = R - (double)reinterpret_cast<const T *>(slot(stage, S::RP1 + v))[k];
          acc[1] += w8[v] * R * d0;
          acc[2] += w8[v] * R * d1;
          acc[3] += w8[v] * d0 * d0;
          acc[4] += w8[v] * d0 * d1;
          acc[5] += w8[v] * d1 * d1;
        }
      }
    }
  }
  cp_wait<0>();
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 6; ++k) red[wid][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
    a.part[(size_t)threadIdx.x * a.nblocks + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_block(st, a.part, a.nblocks, (double)n * V, a.hist, a.hist_cap);
  if (threadIdx.x == 0) *a.count = 0u;
}

// Pass R as a bulk-copy stream (V <= 2, one packed site pair).  A chunk is
// bulk_pts<T>() consecutive points; thread 0 copies every input stream of a
// chunk (buf, t and U per site, the two RP history slots when the Gram sums
// are due, R0 in the refinement form) into one of kBulkStages shared-memory
// stages with cp.async.bulk, kBulkStages - 1 chunks ahead of the one being
// reduced, the bytes counted on the stage's mbarrier.  The other threads
// issue no global loads at all: they read their points from the stage.  One
// block per SM keeps ~3 x 48 KB of reads in flight.
constexpr int kBulkThreads = 512;
constexpr int kBulkStages = 4;
constexpr long long kBulkWaitPolls = 1LL << 24;
template <typename T> __host__ __device__ constexpr int bulk_pts() {
  return sizeof(T) == 4 ? 1024 : 512;
}
template <typename T, int V> __host__ __device__ constexpr size_t bulk_stage_bytes() {
  return (size_t)bulk_pts<T>() * (2 * sizeof(T) + 5 * V * sizeof(T));   // buf; t U RP0 RP1 R0
}
template <typename T, int V> __host__ __device__ constexpr size_t bulk_smem() {
  return (size_t)kBulkStages * bulk_stage_bytes<T, V>();
}

template <typename T, int V, int CLOS, bool REF>
__global__ void __launch_bounds__(kBulkThreads, 1) k_pass_r_bulk(IterArgs<T> a0) {
  static_assert(V <= 2, "one packed site pair");
  static_assert(kBulkThreads % kThreads == 0, "finalize_block folds groups of kThreads");
  const IterArgs<T> a = solute_view<T, V>(a0);
  typedef typename Cx<T>::t C;
  constexpr int CP = bulk_pts<T>(), PT = CP / kBulkThreads;
  constexpr size_t SB = bulk_stage_bytes<T, V>();
  extern __shared__ __align__(16) unsigned char bulk_sm[];
  __shared__ __align__(8) uint64_t full[kBulkStages];
  __shared__ double red[kBulkThreads / 32][6];
  __shared__ bool last;
  DevState *st = a.st;
  if (st->done) {                                // loop stopped: count idle cycles
    if (blockIdx.x == 0 && threadIdx.x == 0) st->after_done += 1;
    return;
  }
  const bool gram = st->count <= 0;
  const long long n = a.n;
  const C *tw = a.tw;
  double w8[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w8[v] = a.sp->irho[v];
  const long long nchunks = (n + CP - 1) / CP;
  const int mine = (long long)blockIdx.x < nchunks
                       ? (int)((nchunks - 1 - blockIdx.x) / gridDim.x) + 1 : 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kBulkStages; ++s) tma::mbar_init(&full[s], 1);
    tma::mbar_init_fence();
  }
  __syncthreads();
  // thread 0: copy chunk i of this block into stage i mod kBulkStages; stage
  // layout [CP] C buf, then [CP] T each: t[V], U[V], RP0[V], RP1[V], R0[V]
  auto fetch = [&](int i) {
    const long long j0 = ((long long)blockIdx.x + (long long)i * gridDim.x) * CP;
    const unsigned np = (unsigned)min((long long)CP, n - j0);
    unsigned char *sg = bulk_sm + (size_t)(i % kBulkStages) * SB;
    T *sT = reinterpret_cast<T *>(sg + CP * sizeof(C));
    uint64_t *bar = &full[i % kBulkStages];
    const unsigned bt = np * (unsigned)sizeof(T);
    const unsigned streams = 2 * V + (gram ? 2 * V : 0) + (REF ? V : 0);
    tma::mbar_arrive_expect_tx(bar, np * (unsigned)sizeof(C) + streams * bt);
    tma::bulk_load(sg, a.buf + j0, np * (unsigned)sizeof(C), bar);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      tma::bulk_load(sT + (size_t)v * CP, a.t + (size_t)v * n + j0, bt, bar);
      tma::bulk_load(sT + (size_t)(V + v) * CP, a.U + (size_t)v * n + j0, bt, bar);
      if (gram) {
        tma::bulk_load(sT + (size_t)(2 * V + v) * CP, a.RP + (size_t)v * n + j0, bt, bar);
        tma::bulk_load(sT + (size_t)(3 * V + v) * CP, a.RP + (size_t)(V + v) * n + j0, bt, bar);
      }
      if (REF) tma::bulk_load(sT + (size_t)(4 * V + v) * CP, a.R0 + (size_t)v * n + j0, bt, bar);
    }
  };
  int fetched = 0;
  if (threadIdx.x == 0)
    for (; fetched < kBulkStages - 1 && fetched < mine; ++fetched) fetch(fetched);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  int fault = 0, i = 0;
  for (; i < mine; ++i) {
    // every thread is past chunk i - 1: its stage takes chunk i + kBulkStages - 1
    if (__syncthreads_or(fault)) break;
    if (threadIdx.x == 0 && fetched < mine) fetch(fetched++);
    if (!tma::mbar_wait_bounded(&full[i % kBulkStages], (unsigned)(i / kBulkStages) & 1u,
                                kBulkWaitPolls)) {
      fault = 1;
      continue;
    }
    const long long j0 = ((long long)blockIdx.x + (long long)i * gridDim.x) * CP;
    const unsigned char *sg = bulk_sm + (size_t)(i % kBulkStages) * SB;
    const C *sb = reinterpret_cast<const C *>(sg);
    const T *sT = reinterpret_cast<const T *>(sg + CP * sizeof(C));
    // PT consecutive points along x (j0 and PT are even, so they share a
    // row and their twiddles differ only in the x factor)
    const int q0 = threadIdx.x * PT;
    if (j0 + q0 >= n) continue;
    int ix, iy, iz, dir0;
    C dkf0;
    point_phase(j0 + q0, a.fdx, a.fdy, tw, ix, iy, iz, dir0, dkf0);
    const C tyz = PT > 1 ? cmul(tw[a.nx + iy], tw[a.nx + a.ny + iz]) : dkf0;
#pragma unroll
    for (int k = 0; k < PT; ++k) {
      const int q = q0 + k;
      const C dkf = k == 0 ? dkf0 : cmul(tw[ix + k], tyz);
      const T sc = (T)a.invvol * (T)((k & 1) ? -dir0 : dir0);
      const C z = cmul(sb[q], mk<C>(dkf.x * sc, -dkf.y * sc));
      const T h[2] = {z.x, z.y};
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T rb = REF ? sT[(size_t)(4 * V + v) * CP + q] : T(0);
        const double R = (double)residual<CLOS, REF>(h[v], sT[(size_t)v * CP + q],
                                                     sT[(size_t)(V + v) * CP + q], rb);
        acc[0] += R * R;                          // cal_rms.cu:18
        if (gram) {                               // theta30, anderson_cuda.cu:33-39
          const double d0 = R - (double)sT[(size_t)(2 * V + v) * CP + q];
          const double d1 = R - (double)sT[(size_t)(3 * V + v) * CP + q];
          acc[1] += w8[v] * R * d0;
          acc[2] += w8[v] * R * d1;
          acc[3] += w8[v] * d0 * d0;
          acc[4] += w8[v] * d0 * d1;
          acc[5] += w8[v] * d1 * d1;
        }
      }
    }
  }
  fault = __syncthreads_or(fault);
  if (fault) {
    // a chunk never arrived: wait (bounded) for the copies still in flight
    // before the block's shared memory goes away (a chunk already consumed
    // passes at once); the NaN sums make the finalize stop the loop as
    // diverged, and the flag makes it an error
    if (threadIdx.x == 0) {
      for (int f = i > 0 ? i - 1 : 0; f < fetched; ++f)
        tma::mbar_wait_bounded(&full[f % kBulkStages], (unsigned)(f / kBulkStages) & 1u,
                               kBulkWaitPolls);
      st->fault = 1;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = __longlong_as_double(0x7ff8000000000000LL);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 6; ++k) red[wid][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < kBulkThreads / 32; ++w) s += red[w][threadIdx.x];
    a.part[(size_t)threadIdx.x * a.nblocks + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_block(st, a.part, a.nblocks, (double)n * V, a.hist, a.hist_cap);
  if (threadIdx.x == 0) *a.count = 0u;
}

// Pass A as the same software pipeline (V <= 2), used for the refinement
// form (which reads R0 as well): each thread prefetches its 16-byte slices
// of the next chunk's inputs (the packed OZ result, t, U, the two history
// slots Y, R0) while it updates the current chunk; outputs go straight to
// global memory.
template <typename T, int V, int CLOS, bool REF>
__global__ void __launch_bounds__(kThreads) k_pass_a_pipe(IterArgs<T> a0) {
  static_assert(V <= 2, "one packed site pair");
  const IterArgs<T> a = solute_view<T, V>(a0);
  typedef typename Cx<T>::t C;
  typedef typename V2<T>::t T2;
  constexpr int PTS = 16 / sizeof(T);
  constexpr int CP = kThreads * PTS;
  using S = PipeSlots<V>;                        // RP0 / RP1 slots carry Y0 / Y1 here
  extern __shared__ float4 pipe_sm[];
  const DevState *st = a.st;
  const int done = st->done, mode = st->mode, slot_w = st->upd_slot;
  const T s1 = (T)st->s1, s2 = (T)st->s2, m = (T)st->m;
  if (done) {
    if (st->after_done == 0) pass_a_final<T, V, CLOS, REF>(a, mode, done, slot_w, s1, s2, m);
    return;                                     // past the snapshot: idle
  }
  const long long n = a.n;
  const C *tw = a.tw;
  auto slot = [&](int stage, int k) -> float4 * {
    return pipe_sm + ((size_t)(stage * S::N + k) * kThreads + threadIdx.x);
  };
  const long long nchunks = (n + CP - 1) / CP;
  auto issue = [&](long long c, int stage) {
    const long long j = c * CP + (long long)threadIdx.x * PTS;
    if (c < nchunks && j < n) {
      if (mode != 0) {
        cp16(slot(stage, S::BUF), a.buf + j);
        cp16(slot(stage, S::BUF + 1), a.buf + j + PTS / 2);
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        cp16(slot(stage, S::T + v), a.t + (size_t)v * n + j);
        cp16(slot(stage, S::U + v), a.U + (size_t)v * n + j);
        if (mode == 2) {
          cp16(slot(stage, S::RP0 + v), a.Y + (size_t)v * n + j);
          cp16(slot(stage, S::RP1 + v), a.Y + (size_t)(V + v) * n + j);
        }
        if (REF && mode != 0) cp16(slot(stage, S::R0 + v), a.R0 + (size_t)v * n + j);
      }
    }
    cp_commit();
  };
  long long c = blockIdx.x;
  issue(c, 0);
  for (int stage = 0; c < nchunks; c += gridDim.x, stage ^= 1) {
    issue(c + gridDim.x, stage ^ 1);
    cp_wait<1>();
    const long long j = c * CP + (long long)threadIdx.x * PTS;
    if (j >= n) continue;
    const T *bz0 = reinterpret_cast<const T *>(slot(stage, S::BUF));
    const T *bz1 = reinterpret_cast<const T *>(slot(stage, S::BUF + 1));
    int ix, iy, iz, dir0;
    C dkf[PTS];
    point_phase(j, a.fdx, a.fdy, tw, ix, iy, iz, dir0, dkf[0]);
    {
      const C tyz = cmul(tw[a.nx + iy], tw[a.nx + a.ny + iz]);
#pragma unroll
      for (int k = 1; k < PTS; ++k) dkf[k] = cmul(tw[ix + k], tyz);
    }
    T tn[V][PTS], yw[V][PTS], rw[V][PTS];
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
      const int dir = (k & 1) ? -dir0 : dir0;
      T h[2] = {T(0), T(0)};
      if (mode != 0) {
        // inverse post-twiddle (timekb, fft3d.cu:52-60): (1/V) dir conj(dkf)
        const T sc = (T)a.invvol * (T)dir;
        const C w = mk<C>(dkf[k].x * sc, -dkf[k].y * sc);
        const T *bz = k < PTS / 2 ? bz0 + 2 * k : bz1 + 2 * (k - PTS / 2);
        C zz;
        zz.x = bz[0];
        zz.y = bz[1];
        const C z = cmul(zz, w);
        h[0] = z.x;
        h[1] = z.y;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T tv = reinterpret_cast<const T *>(slot(stage, S::T + v))[k];
        tn[v][k] = tv;
        if (mode != 0) {
          const T Uv = reinterpret_cast<const T *>(slot(stage, S::U + v))[k];
          const T r0 = REF ? reinterpret_cast<const T *>(slot(stage, S::R0 + v))[k] : T(0);
          const T R = residual<CLOS, REF>(h[v], tv, Uv, r0);   // tr
          const T y = tv + m * R;
          rw[v][k] = R;
          yw[v][k] = y;
          if (mode == 1) {
            tn[v][k] = tv + R;                                   // newdt0 (Picard)
          } else {                                               // newdt (AN2)
            const T y0 = reinterpret_cast<const T *>(slot(stage, S::RP0 + v))[k];
            const T y1 = reinterpret_cast<const T *>(slot(stage, S::RP1 + v))[k];
            tn[v][k] = y + s1 * (y0 - y) + s2 * (y1 - y);
          }
        }
      }
    }
    if (mode != 0) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const size_t iv = (size_t)v * n + j;
        T *py = a.Y + (size_t)slot_w * V * n + iv, *pr = a.RP + (size_t)slot_w * V * n + iv,
          *pt = a.t + iv;
#pragma unroll
        for (int h2 = 0; h2 < PTS / 2; ++h2) {
          T2 wy, wr, wt;
          wy.x = yw[v][2 * h2]; wy.y = yw[v][2 * h2 + 1];
          wr.x = rw[v][2 * h2]; wr.y = rw[v][2 * h2 + 1];
          wt.x = tn[v][2 * h2]; wt.y = tn[v][2 * h2 + 1];
          reinterpret_cast<T2 *>(py)[h2] = wy;
          reinterpret_cast<T2 *>(pr)[h2] = wr;
          reinterpret_cast<T2 *>(pt)[h2] = wt;
        }
      }
    }
    // closure + c_SR (kh/hnc + trm1mt, calculate_cuda.cu:1-29) and the
    // forward pre-twiddle (timekf, fft3d.cu:41-49): dir * dkf * (c_a + i c_b)
    C out[PTS];
#pragma unroll
    for (int k = 0; k < PTS; ++k) {
      const int dir = (k & 1) ? -dir0 : dir0;
      const C wf = mk<C>(dkf[k].x * dir, dkf[k].y * dir);
      C z;
      z.x = cfun<CLOS, REF>(tn[0][k], reinterpret_cast<const T *>(slot(stage, S::U))[k]);
      z.y = (V > 1) ? cfun<CLOS, REF>(tn[V - 1][k],
                                      reinterpret_cast<const T *>(slot(stage, S::U + V - 1))[k])
                    : T(0);
      out[k] = cmul(z, wf);
    }
#pragma unroll
    for (int k = 0; k < PTS; ++k) a.buf[j + k] = out[k];
  }
  cp_wait<0>();
}

// ------------------------------------------------------------- finalize
// Run by the last block of pass R to finish: fixed-order reduction of the
// block sums, then the host logic of iterate.cu:52-62 and AN2::calculate
// (anderson.cu:35-63) on one thread -- no separate launch, no host sync.
__device__ void finalize_block(DevState *st, const double *part, int nblocks,
                               double nv_points, double *hist, int hist_cap) {
  // blocks of any multiple of kThreads threads: threads past the first
  // kThreads fold their sums into those slots, one group at a time
  __shared__ double red[6][kThreads];
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < 6; ++k) s[k] += __ldcg(part + (size_t)k * nblocks + b);
  if (threadIdx.x < kThreads)
#pragma unroll
    for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int g = kThreads; g < (int)blockDim.x; g += kThreads) {
    if ((int)threadIdx.x >= g && (int)threadIdx.x < g + kThreads)
#pragma unroll
      for (int k = 0; k < 6; ++k) red[k][threadIdx.x - g] += s[k];
    __syncthreads();
  }
  for (int w = min((int)blockDim.x, kThreads) / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < 6; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  for (int k = 0; k < 6; ++k) st->sums[k] = red[k][0];
  const double rms = sqrt(red[0][0] / nv_points);
  st->rms = rms;
  if (st->measure) return;
  st->iter += 1;
  if (hist && st->iter <= hist_cap) hist[st->iter - 1] = rms;  // iterate.cu:63 output
  if (!isfinite(rms)) { st->done = 2; st->mode = 0; return; }  // iterate.cu:54-57
  if (rms <= st->conv) { st->done = 1; st->mode = 0; return; } // :58-59
  if (st->watch) {                       // a phase that may hand over early
    if (rms < 0.9 * st->best) { st->best = rms; st->since = 0; }
    else if (++st->since > 30) { st->done = 4; st->mode = 0; return; }
  }
  if (st->count > 0) {                                         // anderson.cu:43-49
    st->count -= 1;
    st->mode = 1;
  } else {                                                     // anderson.cu:50-61
    // [[a00 a01][a01 a11]] x = [c0 c1], eliminated as leg() does (:87-112)
    double a00 = red[3][0], a01 = red[4][0], a11 = red[5][0];
    double c0 = red[1][0], c1 = red[2][0];
    double p = a00;
    double a01n = a01 / p;
    double r = c0 / p;
    double a11n = a11 - a01 * a01n;
    double c1n = c1 - a01 * r;
    double x1 = c1n / a11n;
    double x0 = r - a01n * x1;
    st->s1 = x0 + st->mp * ((st->binary == 0) ? 0.0 : 1.0);
    st->s2 = x1 + st->mp * ((st->binary == 0) ? 1.0 : 0.0);
    st->mode = 2;
  }
  st->upd_slot = st->binary;
  st->binary = (st->binary == 0) ? 1 : 0;
  if (st->iter >= st->maxstep) st->done = 3;   // iterate.cu:51 loop bound
}

// -------------------------------------------- depth-M Anderson (opt-in)
// RISM3D_MDIIS=M (2..kDmMax): the plain FP32 bulk of a mixed single-solute
// solve mixes the last M history entries instead of AN2's two.  Slot i holds
// Y_i = t_i + m R_i and R_i, written round-robin.  Pass R forms R^2,
// c_i = <R, d_i> and a_ij = <d_i, d_j> (d_i = R - R_i, weights 1/rho_v) over
// the filled slots; the finalize solves a s = c in FP64 and adds the AN2
// bias mp to the newest slot; pass A applies t = y + sum_i s_i (Y_i - y),
// y = t + m R.  With M = 2 this is AN2's update (anderson.cu:35-63), and the
// elimination below runs in the order of the reference's 2 x 2 solve
// (leg, anderson.cu:87-112).  Sums: [0] R^2, [1 + i] c_i, [1 + kDmMax + tri]
// a_ij (packed upper triangle).
constexpr int kDmMax = 6;
constexpr int kDmSums = 1 + kDmMax + kDmMax * (kDmMax + 1) / 2;
__host__ __device__ constexpr int dm_tri(int i, int j) {   // i <= j
  return i * kDmMax - i * (i - 1) / 2 + (j - i);
}

template <int V, int CLOS>
__global__ void __launch_bounds__(kThreads) k_pass_a_dm(IterArgs<float> a) {
  constexpr int P = (V + 1) / 2;
  const DevState *st = a.st;
  const int done = st->done, mode = st->mode, slot = st->upd_slot, use = st->dm_use;
  if (done && (st->after_done != 0 || done != 3 || mode == 0)) return;
  const float m = (float)st->m;
  float s[kDmMax];
#pragma unroll
  for (int i = 0; i < kDmMax; ++i) s[i] = i < use ? (float)st->sdm[i] : 0.0f;
  const long long n = a.n;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int ix, iy, iz, dir;
    float2 dkf;
    point_phase(j, a.fdx, a.fdy, a.tw, ix, iy, iz, dir, dkf);
    float h[2 * P];
    if (mode != 0) {
      const float sc = (float)a.invvol * (float)dir;          // timekb, fft3d.cu:52-60
      const float2 w = make_float2(dkf.x * sc, -dkf.y * sc);
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const float2 z = cmul(a.buf[(size_t)p * n + j], w);
        h[2 * p] = z.x;
        h[2 * p + 1] = z.y;
      }
    }
    float c[2 * P];
#pragma unroll
    for (int v = 0; v < 2 * P; ++v) c[v] = 0.0f;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const size_t iv = (size_t)v * n + j;
      const float tv = a.t[iv], Uv = a.U[iv];
      float tn = tv;
      if (mode != 0) {
        const float R = residual<CLOS, false>(h[v], tv, Uv, 0.0f);
        const float y = tv + m * R;
        if (mode == 1) {
          tn = tv + R;                                          // newdt0 (Picard)
        } else {
          tn = y;
#pragma unroll
          for (int i = 0; i < kDmMax; ++i)
            if (i < use) tn += s[i] * (a.Y[(size_t)i * V * n + iv] - y);
        }
        a.Y[(size_t)slot * V * n + iv] = y;
        a.RP[(size_t)slot * V * n + iv] = R;
        a.t[iv] = tn;
      }
      c[v] = cfun<CLOS, false>(tn, Uv);
    }
    if (done) continue;                          // the pending update only
    const float2 wf = make_float2(dkf.x * dir, dkf.y * dir);   // timekf, fft3d.cu:41-49
#pragma unroll
    for (int p = 0; p < P; ++p) a.buf[(size_t)p * n + j] = cmul(make_float2(c[2 * p], c[2 * p + 1]), wf);
  }
}

// The last block of k_pass_r_dm: fixed-order reduction of the block sums,
// the stopping tests of finalize_block, then the Picard step or the depth-M
// solve, and the slot the next pass A writes.
__device__ void finalize_dm(DevState *st, const double *part, int nblocks, double nv_points,
                            double *hist, int hist_cap, int M) {
  __shared__ double tot[kDmSums];
  __shared__ double wsum[32];
  for (int k = 0; k < kDmSums; ++k) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
      s += __ldcg(part + (size_t)k * nblocks + b);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
      tot[k] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  st->sums[0] = tot[0];
  const double rms = sqrt(tot[0] / nv_points);
  st->rms = rms;
  if (st->measure) return;
  st->iter += 1;
  if (hist && st->iter <= hist_cap) hist[st->iter - 1] = rms;  // iterate.cu:63 output
  if (!isfinite(rms)) { st->done = 2; st->mode = 0; return; }  // iterate.cu:54-57
  if (rms <= st->conv) { st->done = 1; st->mode = 0; return; } // :58-59
  if (st->watch) {
    if (rms < 0.9 * st->best) { st->best = rms; st->since = 0; }
    else if (++st->since > 30) { st->done = 4; st->mode = 0; return; }
  }
  const int fill = st->dm_fill;
  if (st->count > 0 || fill < 1) {                             // anderson.cu:43-49
    if (st->count > 0) st->count -= 1;
    st->mode = 1;
    st->dm_use = 0;
  } else {
    // a s = c over the filled slots: each pivot row normalised, then
    // eliminated from the rows below, then back substitution
    double A[kDmMax][kDmMax], b[kDmMax];
    for (int i = 0; i < fill; ++i) {
      b[i] = tot[1 + i];
      for (int j = 0; j < fill; ++j)
        A[i][j] = tot[1 + kDmMax + (i <= j ? dm_tri(i, j) : dm_tri(j, i))];
    }
    for (int i = 0; i < fill; ++i) {
      const double p = A[i][i];
      for (int j = i + 1; j < fill; ++j) A[i][j] /= p;
      b[i] /= p;
      for (int k = i + 1; k < fill; ++k) {
        const double f = A[k][i];
        for (int j = i + 1; j < fill; ++j) A[k][j] -= f * A[i][j];
        b[k] -= f * b[i];
      }
    }
    for (int i = fill - 1; i >= 0; --i)
      for (int j = i + 1; j < fill; ++j) b[i] -= A[i][j] * b[j];
    for (int i = 0; i < kDmMax; ++i)
      st->sdm[i] = i < fill ? b[i] + (i == st->dm_last ? st->mp : 0.0) : 0.0;
    st->dm_use = fill;
    st->mode = 2;
  }
  const int next = (st->dm_last + 1) % M;                      // round-robin slots
  st->upd_slot = next;
  st->dm_last = next;
  st->dm_fill = fill < M ? fill + 1 : M;
  if (st->iter >= st->maxstep) st->done = 3;   // iterate.cu:51 loop bound
}

template <int V, int CLOS>
__global__ void __launch_bounds__(kThreads) k_pass_r_dm(IterArgs<float> a, int M) {
  constexpr int P = (V + 1) / 2;
  __shared__ double red[kThreads / 32][kDmSums];
  __shared__ bool last;
  DevState *st = a.st;
  if (st->done) {                                // loop stopped: count idle cycles
    if (blockIdx.x == 0 && threadIdx.x == 0) st->after_done += 1;
    return;
  }
  const bool gram = st->count <= 0;
  const int fill = st->dm_fill;
  const long long n = a.n;
  double w8[V];
#pragma unroll
  for (int v = 0; v < V; ++v) w8[v] = a.sp->irho[v];
  double acc[kDmSums];
#pragma unroll
  for (int k = 0; k < kDmSums; ++k) acc[k] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int ix, iy, iz, dir;
    float2 dkf;
    point_phase(j, a.fdx, a.fdy, a.tw, ix, iy, iz, dir, dkf);
    const float sc = (float)a.invvol * (float)dir;
    const float2 w = make_float2(dkf.x * sc, -dkf.y * sc);
    float h[2 * P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float2 z = cmul(a.buf[(size_t)p * n + j], w);
      h[2 * p] = z.x;
      h[2 * p + 1] = z.y;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const size_t iv = (size_t)v * n + j;
      const double R = (double)residual<CLOS, false>(h[v], a.t[iv], a.U[iv], 0.0f);
      acc[0] += R * R;                            // cal_rms.cu:18
      if (gram) {
        double d[kDmMax];
#pragma unroll
        for (int i = 0; i < kDmMax; ++i)
          d[i] = i < fill ? R - (double)a.RP[(size_t)i * V * n + iv] : 0.0;
#pragma unroll
        for (int i = 0; i < kDmMax; ++i) {
          if (i >= fill) break;
          acc[1 + i] += w8[v] * R * d[i];
#pragma unroll
          for (int k = i; k < kDmMax; ++k)
            if (k < fill) acc[1 + kDmMax + dm_tri(i, k)] += w8[v] * d[i] * d[k];
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kDmSums; ++k) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[k] = v;
  }
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < kDmSums; ++k) red[wid][k] = acc[k];
  __syncthreads();
  for (int k = threadIdx.x; k < kDmSums; k += blockDim.x) {
    double s = 0.0;
    for (int w2 = 0; w2 < kThreads / 32; ++w2) s += red[w2][k];
    a.part[(size_t)k * a.nblocks + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_dm(st, a.part, a.nblocks, (double)n * V, a.hist, a.hist_cap, M);
  if (threadIdx.x == 0) *a.count = 0u;
}

// After a depth-M bulk: its two newest history entries become AN2's two
// slots (the newest in slot 1, the other in slot 0, the next write to slot
// 0), so that the refinement continues the history as after an AN2 bulk.
__global__ void k_dm_handover(long long vn, int M, const float *Ydm, const float *RPdm,
                              DevState *st, float *Y, float *RP) {
  const int last = st->dm_last, fill = st->dm_fill;
  if (last < 0 || fill < 1) return;
  const int prev = fill >= 2 ? (last + M - 1) % M : last;
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < vn;
       f += (long long)gridDim.x * blockDim.x) {
    Y[vn + f] = Ydm[(size_t)last * vn + f];
    RP[vn + f] = RPdm[(size_t)last * vn + f];
    Y[f] = Ydm[(size_t)prev * vn + f];
    RP[f] = RPdm[(size_t)prev * vn + f];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->binary = 0;
}

// U_SR = u_v + q_v cf esr for a charge-up stage (FP64 and FP32 copies);
// arrays [B][V][N], esr [B][N].
__global__ void k_stage_u(long long n, int nv, long long total, const double *u,
                          const double *esr, const StageParams *sp, double *U,
                          float *Uf) {
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const long long b = f / (nv * n), r = f - b * nv * n;
    const int v = (int)(r / n);
    const long long j = r - (long long)v * n;
    const double x = u[f] + sp->qcf[v] * esr[b * n + j];
    U[f] = x;
    if (Uf) Uf[f] = (float)x;
  }
}

// t_SR from an absolute restart t (read_tuv.cu) or zero (initialize_tuv.cu:
// t = q fr  <=>  t_SR = 0; charge-up start t = 0 with cf = 0 <=> t_SR = 0).
__global__ void k_init_t(long long n, int nv, long long total, const double *tabs,
                         const double *fr, const StageParams *sp, double *t) {
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    if (!tabs) { t[f] = 0.0; continue; }
    const long long b = f / (nv * n), r = f - b * nv * n;
    const int v = (int)(r / n);
    const long long j = r - (long long)v * n;
    t[f] = tabs[f] - sp->qcf[v] * fr[b * n + j];
  }
}

// Charge-up step (add_tuv.cu): the absolute t gains q cuf fr, so t_SR is
// unchanged while the stored history tp_i (absolute in the reference) must
// be re-expressed in the new stage's short-range frame: Y_i -= q cuf fr.
// Y is [B][2][V][N].
template <typename T>
__global__ void k_shift_history(long long n, int nv, long long total, const double *fr,
                                const StageParams *sp_step, T *Y) {
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const long long b = f / (2 * nv * n), r = f - b * 2 * nv * n;
    const int v = (int)((r / n) % nv);
    const long long j = r % n;
    Y[f] = (T)((double)Y[f] - sp_step->qcf[v] * fr[b * n + j]);
  }
}

// Refinement base, after one FP64 cycle at t0 (buf holds its inverse
// transform): R0 = h + 1 - C(t0 - U), x0 = t0 - U, d = 0, and the FP32 AN2
// history re-expressed as corrections to t0 (Y_i - t0; RP_i unchanged).
template <int V, int CLOS>
__global__ void __launch_bounds__(kThreads)
k_refine_base(IterArgs<double> a0, float *R0, float *x0, float *d, float *Yf) {
  const IterArgs<double> a = solute_view<double, V>(a0);
  constexpr int P = (V + 1) / 2;
  const long long n = a.n;
  const size_t b = blockIdx.y;
  R0 += b * V * n; x0 += b * V * n; d += b * V * n; Yf += b * 2 * V * n;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int ix, iy, iz, dir;
    double2 dkf;
    point_phase(j, a.fdx, a.fdy, a.tw, ix, iy, iz, dir, dkf);
    const double sc = a.invvol * dir;
    const double2 w = make_double2(dkf.x * sc, -dkf.y * sc);
    double h[V];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const double2 z = cmul(a.buf[(size_t)p * n + j], w);
      h[2 * p] = z.x;
      if (2 * p + 1 < V) h[2 * p + 1] = z.y;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const size_t iv = (size_t)v * n + j;
      const double t0 = a.t[iv], x = t0 - a.U[iv];
      R0[iv] = (float)(h[v] + 1.0 - closure<CLOS>(x));
      x0[iv] = (float)x;
      d[iv] = 0.0f;
      Yf[iv] = (float)((double)Yf[iv] - t0);
      Yf[(size_t)V * n + iv] = (float)((double)Yf[(size_t)V * n + iv] - t0);
    }
  }
}

// Refinement end: t = t0 + d and the AN2 history back to absolute FP64
// values; arrays [B][V][N] (t, d) and [B][2][V][N] (history).  After a
// bulk divergence (fallback) nothing changes; after a refinement that blew
// up, t stays t0 and the FP64 phase rebuilds the history (restart_next).
__global__ void k_refine_finish(long long n, int nv, long long total, const float *d,
                                const float *Yf, const float *RPf, const DevState *st,
                                double *t, double *Y, double *RP) {
  if (st[0].fallback) return;
  const bool keep = st[0].restart_next != 0;
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x) {
    const long long b = f / (nv * n), r = f - b * nv * n;
    const size_t h0 = (size_t)b * 2 * nv * n + r, h1 = h0 + (size_t)nv * n;
    const double t0 = t[f];
    if (keep) continue;
    Y[h0] = (double)Yf[h0] + t0;
    Y[h1] = (double)Yf[h1] + t0;
    RP[h0] = (double)RPf[h0];
    RP[h1] = (double)RPf[h1];
    t[f] = t0 + (double)d[f];
  }
}

template <typename A, typename B>
__global__ void k_convert(long long n, const A *src, B *dst) {
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x)
    dst[j] = (B)src[j];
}

int grid_blocks(long long work) {
  long long b = (work + kThreads - 1) / kThreads;
  const long long cap = 148LL * 16;   // 148 SMs x 16 resident 256-thread blocks
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// Blocks along x for a grid-stride pass of one solute: one full wave of the
// kernel's resident blocks (SMs x blocks per SM at kThreads threads, from
// its register and shared-memory use), so that no partial last wave leaves
// most SMs idle.  With 2368 blocks, a kernel holding 5 blocks per SM ran 3.2
// waves and one holding 3 ran 5.3.  Batched launches (solutes on y) keep
// grid_blocks: their many waves make the tail small.
template <typename K>
int wave_blocks(K kernel, long long work, int nb) {
  if (nb > 1) return grid_blocks(work);
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess ||
      sms < 1 || per_sm < 1) {
    cudaGetLastError();
    return grid_blocks(work);
  }
  const long long need = (work + kThreads - 1) / kThreads, wave = (long long)sms * per_sm;
  return (int)std::max(1LL, std::min(need, wave));
}

// Blocks for a grid-stride launch of `kernel` with `threads` threads and
// `smem` dynamic shared memory: the work's blocks, at most one full wave.
template <typename K>
int wave_blocks_smem(K kernel, int threads, size_t smem, long long need) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
      sms < 1 || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
    sms = 148;
  }
  return (int)std::max(1LL, std::min(need, (long long)sms * per_sm));
}

template <int V, int CLOS, bool REF, int E>
int grid_ax(const Context &c) {
  const long long lines = (long long)c.ny * c.nz;
  return wave_blocks_smem(k_pass_ax<V, CLOS, REF, E>, kXThreads, 0,
                          (lines * E + kXThreads - 1) / kXThreads);
}

template <int V, int E>
int grid_ky(const Context &c) {
  return wave_blocks_smem(k_kspace_y<V, E>, kW * E, KYLayout<E>::bytes(),
                          (long long)(c.nx / kW) * (c.nz / 2));
}

// The fused pass K: the TMA form on 256-point lines when its tensor map
// (bound to the context's FP32 transform buffer) exists, else the
// register/shared-memory form.
template <int V, int E>
void launch_kspace_y(Context &c, const IterArgs<float> &a) {
  if constexpr (E == 16) {
    if (c.ky_map && (const void *)a.buf == (const void *)c.f_buf) {
      const int tiles = (c.nx / 16) * (c.nz / 2);
      const int g = wave_blocks_smem(k_kspace_yt<V>, kKyThreads, kKySmem, tiles);
      k_kspace_yt<V><<<g, kKyThreads, kKySmem, c.stream>>>(a, *c.ky_map);
      return;
    }
  }
  k_kspace_y<V, E><<<grid_ky<V, E>(c), kW * E, KYLayout<E>::bytes(), c.stream>>>(a);
}

// One FP32 iteration with the x and y axes of the transforms folded into the
// passes (single solute, V <= 2, nx = ny = E^2): cuFFT transforms along z.
template <int V, int CLOS, bool REF, int E>
void launch_iteration_x(Context &c, const IterArgs<float> &a) {
  k_pass_ax<V, CLOS, REF, E><<<grid_ax<V, CLOS, REF, E>(c), kXThreads, 0, c.stream>>>(a);
  cufftExecC2C(c.plan32z, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_FORWARD);
  launch_kspace_y<V, E>(c, a);
  cufftExecC2C(c.plan32z, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_INVERSE);
  k_pass_rx<V, CLOS, REF, E><<<a.nblocks, kXThreads, 0, c.stream>>>(a);
}

// Blocks of the pipelined pass R: one full wave (it walks the grid), at most
// the partial-sum slots the context has.
template <typename T, int V, int CLOS, bool REF>
int pipe_r_blocks(const Context &c) {
  const int w = wave_blocks_smem(k_pass_r_pipe<T, V, CLOS, REF>, kThreads,
                                 pass_r_pipe_smem<T, V>(), c.nred_blocks);
  return std::min(w, c.nred_blocks);
}

template <typename T, int V, int CLOS, bool REF>
int pipe_a_blocks(const Context &c) {
  constexpr int CP = kThreads * (16 / (int)sizeof(T));
  return wave_blocks_smem(k_pass_a_pipe<T, V, CLOS, REF>, kThreads, pass_r_pipe_smem<T, V>(),
                          (c.n + CP - 1) / CP);
}

// Blocks of the bulk-copy pass R: one per SM (its stages fill the shared
// memory), at most the partial-sum slots the context has.
template <typename T, int V, int CLOS, bool REF>
int bulk_r_blocks(const Context &c) {
  const int w = wave_blocks_smem(k_pass_r_bulk<T, V, CLOS, REF>, kBulkThreads, bulk_smem<T, V>(),
                                 c.nred_blocks);
  return std::min(w, c.nred_blocks);
}

// Pass R in the form the context chose: bulk-copy stream, cp.async
// pipeline, or plain grid-stride.
template <typename T, int V, int CLOS, bool REF>
void launch_pass_r(Context &c, const IterArgs<T> &a) {
  if constexpr (V <= 2) {
    if (c.bulk_r) {
      IterArgs<T> ar = a;
      ar.nblocks = bulk_r_blocks<T, V, CLOS, REF>(c);
      k_pass_r_bulk<T, V, CLOS, REF><<<dim3(ar.nblocks, c.nb), kBulkThreads, bulk_smem<T, V>(),
                                       c.stream>>>(ar);
      return;
    }
    if (c.pipe_r) {
      IterArgs<T> ar = a;
      ar.nblocks = pipe_r_blocks<T, V, CLOS, REF>(c);
      k_pass_r_pipe<T, V, CLOS, REF><<<dim3(ar.nblocks, c.nb), kThreads, pass_r_pipe_smem<T, V>(),
                                       c.stream>>>(ar);
      return;
    }
  }
  k_pass_r<T, V, CLOS, REF><<<dim3(a.nblocks, c.nb), kThreads, 0, c.stream>>>(a);
}

// One FP32 bulk iteration with the depth-M Anderson passes (3D cuFFT path).
template <int V, int CLOS>
void launch_iteration_dm(Context &c, const IterArgs<float> &a, cufftHandle plan) {
  k_pass_a_dm<V, CLOS><<<wave_blocks(k_pass_a_dm<V, CLOS>, a.n, 1), kThreads, 0, c.stream>>>(a);
  cufftExecC2C(plan, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_FORWARD);
  k_kspace<float, V><<<wave_blocks(k_kspace<float, V>, a.n / 2, 1), kThreads, 0, c.stream>>>(a);
  cufftExecC2C(plan, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_INVERSE);
  k_pass_r_dm<V, CLOS><<<a.nblocks, kThreads, 0, c.stream>>>(a, c.dm_depth);
}

template <typename T, int V, int CLOS, bool REF>
void launch_iteration(Context &c, const IterArgs<T> &a, cufftHandle plan) {
  if constexpr (sizeof(T) == 4 && !REF) {
    if (c.dm_depth && (const void *)a.Y == (const void *)c.f_Ydm) {
      launch_iteration_dm<V, CLOS>(c, a, plan);
      return;
    }
  }
  // the fused-axis passes run the plain FP32 bulk; the refinement form
  // (which also streams R0) stays on the 3D transforms, where its pipelined
  // passes are faster.  Every phase starts without a pending update (its
  // first pass A reads no transform), so the two forms never share a buffer.
  if constexpr (sizeof(T) == 4 && V <= 2 && !REF) {
    if (c.xfused) {
      if (c.nx == 256) launch_iteration_x<V, CLOS, REF, 16>(c, a);
      else launch_iteration_x<V, CLOS, REF, 8>(c, a);
      return;
    }
  }
  const dim3 ba(wave_blocks(k_pass_a<T, V, CLOS, REF>, a.n, c.nb), c.nb),
      bk(wave_blocks(k_kspace<T, V>, a.n / 2, c.nb), c.nb), br(a.nblocks, c.nb);
  // the pipelined pass A pays for the refinement form (it reads R0 too);
  // the plain form already streams near bandwidth from registers
  if constexpr (V <= 2 && REF) {
    if (c.pipe_r)
      k_pass_a_pipe<T, V, CLOS, REF><<<dim3(pipe_a_blocks<T, V, CLOS, REF>(c), c.nb), kThreads,
                                       pass_r_pipe_smem<T, V>(), c.stream>>>(a);
    else
      k_pass_a<T, V, CLOS, REF><<<ba, kThreads, 0, c.stream>>>(a);
  } else {
    k_pass_a<T, V, CLOS, REF><<<ba, kThreads, 0, c.stream>>>(a);
  }
  typedef typename Cx<T>::t C;
  if (sizeof(T) == 8) {
    cufftExecZ2Z(plan, (cufftDoubleComplex *)a.buf, (cufftDoubleComplex *)a.buf, CUFFT_FORWARD);
  } else {
    cufftExecC2C(plan, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_FORWARD);
  }
  k_kspace<T, V><<<bk, kThreads, 0, c.stream>>>(a);
  if (sizeof(T) == 8) {
    cufftExecZ2Z(plan, (cufftDoubleComplex *)a.buf, (cufftDoubleComplex *)a.buf, CUFFT_INVERSE);
  } else {
    cufftExecC2C(plan, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_INVERSE);
  }
  launch_pass_r<T, V, CLOS, REF>(c, a);
  (void)sizeof(C);
  (void)br;
}

template <typename T>
IterArgs<T> make_args(Context &c, bool fp64) {
  IterArgs<T> a{};
  a.n = c.n; a.nx = c.nx; a.ny = c.ny; a.nz = c.nz;
  a.fdx = FastDiv((unsigned)c.nx); a.fdy = FastDiv((unsigned)c.ny);
  a.xs = c.d_xs;
  a.xs32 = c.d_xs32;
  a.invvol = 1.0 / c.vol; a.dv = c.dv;
  a.fkh = c.d_fkh; a.chi = c.chi.d_coef; a.ntab = c.chi.ntab; a.dk = c.chi.dk;
  a.bx = c.prm.box[0]; a.by = c.prm.box[1]; a.bz = c.prm.box[2];
  a.st = c.d_state; a.sp = c.d_stage; a.part = c.d_part; a.nblocks = c.nred_blocks;
  a.count = c.d_count;
  a.hist = c.nb == 1 ? c.d_hist : nullptr;
  a.xroots = c.d_xroots;
  a.fkt = c.d_fkt;
  a.hist_cap = c.hist_cap;
  (void)fp64;
  return a;
}

// Capture one iteration (passes, cuFFT, and the fused finalize) as a CUDA
// graph, once per context and precision; every later solve relaunches it.
// If capture of the cuFFT calls is refused, the loop launches directly.
template <typename T, int V, int CLOS, bool REF>
cudaGraphExec_t capture(Context &c, const IterArgs<T> &a, cufftHandle plan) {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  launch_iteration<T, V, CLOS, REF>(c, a, plan);
  cudaError_t e = cudaStreamEndCapture(c.stream, &g);
  if (e != cudaSuccess || !g) {
    cudaGetLastError();
    return nullptr;
  }
  e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return x;
}

// End of one device-side loop body: keep looping while any solute is still
// running or has not yet had the idle pass after its stop (the snapshot);
// the body count is bounded by the phase's step limit plus a margin.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, DevState *st, int nb) {
  if (threadIdx.x != 0) return;
  bool more = false;
  int cap = 1;                 // the largest step budget left to any solute
  for (int b = 0; b < nb; ++b) {
    if (!(st[b].done && st[b].after_done >= 1)) more = true;
    cap = max(cap, st[b].maxstep);
  }
  const int loops = ++st[0].loops;
  st[0].bodies += 1;
  cap = cap < 1000000 ? cap : 1000000;
  if (loops >= cap + 4) more = false;
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

// One whole phase as a single graph: a while node whose body is one
// iteration (passes, cuFFT, finalize) plus k_loop_cond.  Returns null when
// the driver or cuFFT cannot be captured this way; the caller then drives
// the iterations from the host.
template <typename T, int V, int CLOS, bool REF>
cudaGraphExec_t capture_loop(Context &c, const IterArgs<T> &a, cufftHandle plan) {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t x = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  cudaGraphConditionalHandle h;
  bool ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
  // the parameter union has no default constructor: zeroed storage
  alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)] = {};
  cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(raw);
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  ok = ok && cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess;
  if (ok) {
    cudaGraph_t body = np.conditional.phGraph_out[0];
    ok = cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      launch_iteration<T, V, CLOS, REF>(c, a, plan);
      k_loop_cond<<<1, 32, 0, c.stream>>>(h, a.st, c.nb);
      cudaGraph_t out = nullptr;
      ok = cudaStreamEndCapture(c.stream, &out) == cudaSuccess;
    }
  }
  if (ok) ok = cudaGraphInstantiate(&x, g, 0) == cudaSuccess;
  cudaGraphDestroy(g);
  if (!ok) {
    cudaGetLastError();
    if (x) cudaGraphExecDestroy(x);
    return nullptr;
  }
  return x;
}

// Phase control on the device, so that a solve needs no host round trip
// between its phases.  Kinds: the plain FP32 bulk, the FP32 refinement,
// the final FP64 phase, and the single FP64 base cycle of the refinement.
enum PhaseKind { kPlain32 = 0, kRefine32 = 1, kFinal64 = 2, kBase64 = 3 };

// Start of a phase: reset the per-run words of every solute; the step
// budget is what the stage has left (iterate.cu:51).  A refinement after
// an FP32 divergence (fallback) is skipped: one idle body.  The final FP64
// phase restarts AN2 from Picard steps when the history was discarded.
__global__ void k_phase_begin(DevState *st, int nb, int kind, double conv, int maxstep,
                              int watch, int an2_count) {
  const bool fallback = st[0].fallback != 0;
  const bool fresh = fallback || st[0].restart_next != 0;
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    DevState &s = st[b];
    s.done = 0; s.after_done = 0; s.iter = 0; s.mode = 0;
    if (kind == kBase64) continue;
    s.conv = conv;
    s.maxstep = max(1, maxstep - s.stage_iter);
    s.watch = watch; s.since = 0; s.best = 1e300; s.loops = 0;
    if (kind == kRefine32 && fallback) { s.done = 4; s.after_done = 1; }
    if (kind == kPlain32) { s.dm_fill = 0; s.dm_last = -1; s.dm_use = 0; }
    if (kind == kFinal64 && fresh) { s.count = an2_count; s.binary = 0; }
  }
}

// End of a phase: step counters, and the flags the next phases read.
__global__ void k_phase_end(DevState *st, int nb, int kind, int fp32) {
  __shared__ int any_div;
  if (threadIdx.x == 0) any_div = 0;
  __syncthreads();
  const bool fallback = st[0].fallback != 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    DevState &s = st[b];
    const int steps = kind == kBase64 ? (fallback ? 0 : 1) : s.iter;
    s.stage_iter += steps;
    s.total_iter += steps;
    if (fp32) s.total32 += steps;
    if (s.done == 2) atomicOr(&any_div, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (kind == kPlain32) st[0].fallback = any_div;
    if (kind == kRefine32 && !fallback) st[0].restart_next = any_div;
  }
}

__global__ void k_stage_begin(DevState *st, int nb) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) st[b].stage_iter = 0;
  if (threadIdx.x == 0) { st[0].fallback = 0; st[0].restart_next = 0; }
}

// After the FP32 bulk: the refinement base t0 (exact FP32 -> FP64), or on a
// divergence the stage start t_SR = 0 for the FP64 restart.
__global__ void k_promote_base(long long total, const float *tf, const DevState *st,
                               double *t) {
  const bool fallback = st[0].fallback != 0;
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < total;
       f += (long long)gridDim.x * blockDim.x)
    t[f] = fallback ? 0.0 : (double)tf[f];
}

// One phase: the device-side loop graph when available (no host sync), else
// iterations driven from the host.  Progress lines and the optional trace
// need the host and synchronise.
template <typename T, int V, int CLOS, bool REF>
int run_phase(Context &c, cufftHandle plan, T *t, T *U, T *Y, T *RP,
              typename Cx<T>::t *buf, bool snapshot, int kind, double conv, bool watch,
              const T *R0 = nullptr) {
  IterArgs<T> a = make_args<T>(c, sizeof(T) == 8);
  a.buf = buf; a.t = t; a.U = U; a.Y = Y; a.RP = RP;
  if (REF) { a.R0 = R0; a.sp = c.d_stage_ref; a.nofk = 1; }
  a.hout = snapshot ? c.d_h : nullptr;
  a.gout = snapshot ? c.d_g : nullptr;
  a.tw = (const typename Cx<T>::t *)(sizeof(T) == 8 ? (void *)c.d_tw : (void *)c.d_twf);
  const int nb = c.nb;
  k_phase_begin<<<1, 128, 0, c.stream>>>(c.d_state, nb, kind, conv, c.prm.maxstep,
                                         watch ? 1 : 0, c.prm.an2_count);
  c.launches += 1;
  if (!cufft_ok(c, cufftSetStream(plan, c.stream), "cufftSetStream")) return RISM3D_CUFFT_ERROR;
  if (c.plan32z && !cufft_ok(c, cufftSetStream(c.plan32z, c.stream), "cufftSetStream"))
    return RISM3D_CUFFT_ERROR;
  int status = RISM3D_OK;
  static const bool trace = getenv("RISM3D_TRACE") && getenv("RISM3D_TRACE")[0] == '1';
  cudaGraphExec_t &lx = REF ? c.loop32r : (sizeof(T) == 8) ? c.loop64 : c.loop32;
  if (!lx && !c.no_device_loop) {
    lx = capture_loop<T, V, CLOS, REF>(c, a, plan);
    if (!lx) c.no_device_loop = true;
  }
  if (lx) {
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (trace) {
      cudaEventCreate(&t0);
      cudaEventCreate(&t1);
      cudaEventRecord(t0, c.stream);
    }
    if (!cuda_ok(c, cudaGraphLaunch(lx, c.stream), "phase launch")) return RISM3D_CUDA_ERROR;
    if (trace) {
      cudaEventRecord(t1, c.stream);
      DevState s0;
      cudaMemcpyAsync(&s0, c.d_state, sizeof(DevState), cudaMemcpyDeviceToHost, c.stream);
      cudaStreamSynchronize(c.stream);
      float ms = 0;
      cudaEventElapsedTime(&ms, t0, t1);
      fprintf(stderr, "[rism3d] phase %s%s: %d bodies, %d steps, device %.2f ms\n",
              sizeof(T) == 8 ? "fp64" : "fp32", REF ? "-refine" : "", s0.loops, s0.iter, ms);
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
    }
  } else {
    // host-driven: one captured iteration per launch, the state read two
    // iterations late from pinned memory
    cudaGraphExec_t &gx = REF ? c.graph32r : (sizeof(T) == 8) ? c.graph64 : c.graph32;
    if (!gx) gx = capture<T, V, CLOS, REF>(c, a, plan);
    const int kRing = 4, kLag = 2;
    cudaEvent_t ev[kRing];
    for (int i = 0; i < kRing; ++i) cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    int launched = 0;
    bool stop = false;
    while (!stop) {
      if (gx) cudaGraphLaunch(gx, c.stream);
      else launch_iteration<T, V, CLOS, REF>(c, a, plan);
      c.launches += 3;
      cudaMemcpyAsync(&c.h_state[(size_t)(launched % kRing) * nb], c.d_state, sizeof(DevState) * nb,
                      cudaMemcpyDeviceToHost, c.stream);
      cudaEventRecord(ev[launched % kRing], c.stream);
      ++launched;
      if (launched > kLag) {
        int k = (launched - 1 - kLag) % kRing;
        if (!cuda_ok(c, cudaEventSynchronize(ev[k]), "iteration")) { status = RISM3D_CUDA_ERROR; break; }
        const DevState *ss = &c.h_state[(size_t)k * nb];
        bool all_done = true;
        int cap = 1;
        for (int b = 0; b < nb; ++b) {
          if (!ss[b].done) all_done = false;
          cap = std::max(cap, ss[b].maxstep);
        }
        if (all_done) stop = true;
        if (launched > cap + kLag + 2) stop = true;   // hard bound
      }
      if (launched > c.prm.maxstep + kLag + 2) stop = true;
    }
    // drain: one more iteration guarantees the snapshot pass ran
    if (status == RISM3D_OK) {
      if (gx) cudaGraphLaunch(gx, c.stream);
      else launch_iteration<T, V, CLOS, REF>(c, a, plan);
      c.launches += 3;
    }
    for (int i = 0; i < kRing; ++i) cudaEventDestroy(ev[i]);
  }
  // the loop's bodies (4 launches each: passes A, K, R and the loop test)
  // are counted from the device record at the end of the solve
  k_phase_end<<<1, 128, 0, c.stream>>>(c.d_state, nb, kind, sizeof(T) == 4 ? 1 : 0);
  c.launches += 1;
  // progress lines of the reference (iterate.cu:63), from the device record
  if (status == RISM3D_OK && c.prm.verbose && nb == 1 && c.d_hist) {
    DevState s0;
    if (cuda_ok(c, cudaMemcpyAsync(&s0, c.d_state, sizeof(DevState), cudaMemcpyDeviceToHost, c.stream), "state") &&
        cuda_ok(c, cudaStreamSynchronize(c.stream), "state") && s0.iter > 0) {
      std::vector<double> hr(std::min(s0.iter, c.hist_cap));
      if (cuda_ok(c, cudaMemcpy(hr.data(), c.d_hist, sizeof(double) * hr.size(), cudaMemcpyDeviceToHost), "history"))
        for (size_t i = 0; i < hr.size(); ++i) printf(" Step = %d Reside = %g\n", (int)i + 1, hr[i]);
    }
  }
  return status;
}

// One FP64 cycle at the base t0 = d_t without an update (pass A in mode 0,
// both transforms, the k-space pass with the stage's fk), then the
// refinement base: R0, x0, d = 0 and the FP32 history relative to t0.
template <int V, int CLOS>
int refine_base(Context &c) {
  const int nb = c.nb;
  k_phase_begin<<<1, 128, 0, c.stream>>>(c.d_state, nb, kBase64, 0.0, 0, 0, 0);
  IterArgs<double> a = make_args<double>(c, true);
  a.buf = c.d_buf; a.t = c.d_t; a.U = c.d_U; a.Y = c.d_Y; a.RP = c.d_RP;
  a.tw = c.d_tw;
  const dim3 ba(wave_blocks(k_pass_a<double, V, CLOS, false>, c.n, nb), nb),
      bk(wave_blocks(k_kspace<double, V>, c.n / 2, nb), nb),
      bb(wave_blocks(k_refine_base<V, CLOS>, c.n, nb), nb);
  if (!cufft_ok(c, cufftSetStream(c.plan64, c.stream), "cufftSetStream")) return RISM3D_CUFFT_ERROR;
  k_pass_a<double, V, CLOS, false><<<ba, kThreads, 0, c.stream>>>(a);
  if (!cufft_ok(c, cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)a.buf, (cufftDoubleComplex *)a.buf,
                                CUFFT_FORWARD), "refine base FFT"))
    return RISM3D_CUFFT_ERROR;
  k_kspace<double, V><<<bk, kThreads, 0, c.stream>>>(a);
  if (!cufft_ok(c, cufftExecZ2Z(c.plan64, (cufftDoubleComplex *)a.buf, (cufftDoubleComplex *)a.buf,
                                CUFFT_INVERSE), "refine base FFT"))
    return RISM3D_CUFFT_ERROR;
  k_refine_base<V, CLOS><<<bb, kThreads, 0, c.stream>>>(a, c.f_R0, c.f_x0, c.f_t, c.f_Y);
  k_phase_end<<<1, 128, 0, c.stream>>>(c.d_state, nb, kBase64, 0);
  c.launches += 6;
  return cuda_ok(c, cudaGetLastError(), "refine base") ? RISM3D_OK : RISM3D_CUDA_ERROR;
}

template <int V, int CLOS>
int solve_v(Context &c, int chargeup) {
  const long long n = c.n;
  const int nb = c.nb;
  const long long vnb = (long long)V * n * nb;     // elements of a [B][V][N] grid
  const bool mixed = c.prm.precision == RISM3D_MIXED;
  const int gb = grid_blocks(n);
  StageParams sp{};
  for (int v = 0; v < V; ++v) sp.irho[v] = 1.0 / c.rho[v];
  // stage schedule (iterate.cu:30-47)
  int cu = chargeup;
  double cf, cuf = 0.0;
  const bool restart = !c.t_init.empty() && nb == 1;
  if (restart) { cu = 0; cf = 1.0; }
  else if (cu == 0) cf = 1.0;
  else { cuf = 1.0 / cu; cf = 0.0; }

  // AN2 state (anderson.cu:13-32)
  std::vector<DevState> hs0(nb);
  for (DevState &hs : hs0) {
    hs = DevState{};
    hs.count = c.prm.an2_count; hs.binary = 0; hs.m = c.prm.an2_m; hs.mp = c.prm.an2_mp;
    hs.maxstep = c.prm.maxstep; hs.conv = c.prm.convergence;
  }
  cudaMemcpyAsync(c.d_state, hs0.data(), sizeof(DevState) * nb, cudaMemcpyHostToDevice, c.stream);
  cudaMemsetAsync(c.d_Y, 0, sizeof(double) * 2 * vnb, c.stream);
  cudaMemsetAsync(c.d_RP, 0, sizeof(double) * 2 * vnb, c.stream);
  if (mixed) {
    cudaMemsetAsync(c.f_Y, 0, sizeof(float) * 2 * vnb, c.stream);
    cudaMemsetAsync(c.f_RP, 0, sizeof(float) * 2 * vnb, c.stream);
    StageParams spr{};
    for (int v = 0; v < V; ++v) spr.irho[v] = sp.irho[v];   // qcf = 0: fk cancels
    cudaMemcpyAsync(c.d_stage_ref, &spr, sizeof(spr), cudaMemcpyHostToDevice, c.stream);
  }
  // initial t_SR
  for (int v = 0; v < V; ++v) sp.qcf[v] = c.qv[v] * cf;
  cudaMemcpyAsync(c.d_stage, &sp, sizeof(sp), cudaMemcpyHostToDevice, c.stream);
  double *d_tinit = nullptr;
  if (restart) {
    if (!cuda_ok(c, pool_alloc(c, (void **)&d_tinit, sizeof(double) * V * n), "alloc") ||
        !cuda_ok(c, cudaMemcpyAsync(d_tinit, c.t_init.data(), sizeof(double) * V * n, cudaMemcpyHostToDevice, c.stream), "copy"))
      return RISM3D_CUDA_ERROR;
  }
  k_init_t<<<gb, kThreads, 0, c.stream>>>(n, V, vnb, d_tinit, c.d_fr, c.d_stage, c.d_t);
  c.launches += 1;
  if (d_tinit) cudaFreeAsync(d_tinit, c.stream);

  int status = RISM3D_OK;
  std::vector<DevState> fs(nb);
  StageParams *d_step = nullptr;
  if (cu > 0 && !cuda_ok(c, pool_alloc(c, (void **)&d_step, sizeof(StageParams)), "alloc"))
    return RISM3D_CUDA_ERROR;
  for (int s = 0; s <= cu; ++s) {
    if (s > 0) {                                  // add_tuv (iterate.cu:43-47)
      double cfn = cf + cuf;
      if (cfn > 1.0) cfn = 1.0;
      StageParams step{};
      for (int v = 0; v < V; ++v) step.qcf[v] = c.qv[v] * (cfn - cf);
      cudaMemcpyAsync(d_step, &step, sizeof(step), cudaMemcpyHostToDevice, c.stream);
      k_shift_history<double><<<gb, kThreads, 0, c.stream>>>(n, V, 2 * vnb, c.d_fr, d_step, c.d_Y);
      c.launches += 1;
      if (mixed) {
        k_shift_history<float><<<gb, kThreads, 0, c.stream>>>(n, V, 2 * vnb, c.d_fr, d_step, c.f_Y);
        c.launches += 1;
      }
      cf = cfn;
    }
    for (int v = 0; v < V; ++v) sp.qcf[v] = c.qv[v] * cf;
    cudaMemcpyAsync(c.d_stage, &sp, sizeof(sp), cudaMemcpyHostToDevice, c.stream);
    k_stage_u<<<gb, kThreads, 0, c.stream>>>(n, V, vnb, c.d_u, c.d_e, c.d_stage, c.d_U, mixed ? c.f_U : nullptr);
    k_stage_begin<<<1, 128, 0, c.stream>>>(c.d_state, nb);
    c.launches += 2;
    if (c.prm.verbose) printf("relaxing 3D UV RISM: Charge Up Factor = %g\n", cf);
    int st = RISM3D_OK;
    if (mixed) {
      // FP32 bulk (plain form) down to the switch residual, then one FP64
      // cycle fixes the base t0 and FP32 refinement passes carry the
      // correction to the FP64 tolerance; the FP64 phase below then only
      // confirms convergence and snapshots h and g.  A divergence of the
      // bulk restarts the stage in FP64 (decided on the device).
      const long long vn = vnb;
      k_convert<double, float><<<gb, kThreads, 0, c.stream>>>(vn, c.d_t, c.f_t);
      k_convert<double, float><<<gb, kThreads, 0, c.stream>>>(2 * vn, c.d_Y, c.f_Y);
      k_convert<double, float><<<gb, kThreads, 0, c.stream>>>(2 * vn, c.d_RP, c.f_RP);
      c.launches += 3;
      double sw = c.prm.mixed_switch > 0 ? c.prm.mixed_switch : 100.0 * c.prm.convergence;
      if (sw < c.prm.convergence) sw = c.prm.convergence;
      st = run_phase<float, V, CLOS, false>(c, c.plan32, c.f_t, c.f_U,
                                           c.dm_depth ? c.f_Ydm : c.f_Y,
                                           c.dm_depth ? c.f_RPdm : c.f_RP, c.f_buf,
                                           false, kPlain32, sw, true);
      if (st != RISM3D_OK) { status = st; break; }
      if (c.dm_depth) {
        k_dm_handover<<<gb, kThreads, 0, c.stream>>>(vn, c.dm_depth, c.f_Ydm, c.f_RPdm, c.d_state,
                                                      c.f_Y, c.f_RP);
        c.launches += 1;
      }
      k_promote_base<<<gb, kThreads, 0, c.stream>>>(vn, c.f_t, c.d_state, c.d_t);
      c.launches += 1;
      st = refine_base<V, CLOS>(c);
      if (st != RISM3D_OK) { status = st; break; }
      st = run_phase<float, V, CLOS, true>(c, c.plan32, c.f_t, c.f_x0, c.f_Y, c.f_RP, c.f_buf,
                                          false, kRefine32, c.prm.convergence, true, c.f_R0);
      if (st != RISM3D_OK) { status = st; break; }
      k_refine_finish<<<gb, kThreads, 0, c.stream>>>(n, V, vnb, c.f_t, c.f_Y, c.f_RP, c.d_state,
                                                    c.d_t, c.d_Y, c.d_RP);
      c.launches += 1;
    }
    st = run_phase<double, V, CLOS, false>(c, c.plan64, c.d_t, c.d_U, c.d_Y, c.d_RP, c.d_buf,
                                          true, kFinal64, c.prm.convergence, false);
    if (st != RISM3D_OK) { status = st; break; }
    // the stage's outcome: one read of the device state
    if (!cuda_ok(c, cudaMemcpyAsync(fs.data(), c.d_state, sizeof(DevState) * nb, cudaMemcpyDeviceToHost, c.stream), "state read") ||
        !cuda_ok(c, cudaStreamSynchronize(c.stream), "solve"))
      return RISM3D_CUDA_ERROR;
    bool div = false, lim = false;
    for (const DevState &x : fs) { div = div || x.done == 2; lim = lim || (x.done != 1 && x.done != 2); }
    if (div) {                             // iterate.cu:74-75: report, go on
      if (c.prm.verbose) printf("Calculation diverged.\n");
      status = RISM3D_DIVERGED;
    } else if (lim) {                      // iterate.cu:76-79: stop charging
      if (c.prm.verbose) printf("3D UV RISM: reached limit # of relaxation steps: %d\n", c.prm.maxstep);
      status = RISM3D_NOT_CONVERGED;
      break;
    }
  }
  if (d_step) cudaFreeAsync(d_step, c.stream);
  if (!cuda_ok(c, cudaMemcpyAsync(fs.data(), c.d_state, sizeof(DevState) * nb, cudaMemcpyDeviceToHost, c.stream), "state read") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "solve"))
    return RISM3D_CUDA_ERROR;
  int total = 0, total32 = 0;
  long long bodies = 0;
  for (const DevState &x : fs) {
    total = std::max(total, x.total_iter);
    total32 = std::max(total32, x.total32);
  }
  bodies = fs[0].bodies;
  for (const DevState &x : fs)
    if (x.fault) {
      c.err = "a device-side wait gave up: a bulk or tile copy never arrived";
      status = RISM3D_CUDA_ERROR;
    }
  c.launches += 4 * bodies;
  c.res.rms = fs[0].rms;
  if (nb > 1) {
    c.bres.assign(nb, rism3d_result{});
    for (int b = 0; b < nb; ++b) {
      c.bres[b].rms = fs[b].rms;
      c.bres[b].iterations = fs[b].total_iter;
      c.bres[b].iterations_fp32 = fs[b].total32;
      c.bres[b].status = fs[b].done == 1 ? RISM3D_OK
                       : fs[b].done == 2 ? RISM3D_DIVERGED : RISM3D_NOT_CONVERGED;
    }
  }
  c.cf_final = cf;
  c.res.iterations = total;
  c.res.iterations_fp32 = total32;
  c.res.status = status;
  return (status == RISM3D_CUDA_ERROR || status == RISM3D_CUFFT_ERROR) ? status : RISM3D_OK;
}

template <int V, int CLOS, int E>
void time_fused(Context &c, const IterArgs<float> &a, int which, int reps) {
  for (int r = 0; r < reps; ++r) {
    switch (which) {
      case 10: k_pass_ax<V, CLOS, false, E><<<grid_ax<V, CLOS, false, E>(c), kXThreads, 0,
                                                c.stream>>>(a); break;
      case 13: k_pass_ax<V, CLOS, true, E><<<grid_ax<V, CLOS, true, E>(c), kXThreads, 0,
                                               c.stream>>>(a); break;
      case 11: launch_kspace_y<V, E>(c, a); break;
      case 15: k_pass_rx<V, CLOS, true, E><<<a.nblocks, kXThreads, 0, c.stream>>>(a); break;
      default: k_pass_rx<V, CLOS, false, E><<<a.nblocks, kXThreads, 0, c.stream>>>(a); break;
    }
  }
}

template <typename T, int V, int CLOS>
int time_kernel_t(Context &c, int which, int reps, double *ms) {
  const bool fp64 = sizeof(T) == 8;
  IterArgs<T> a = make_args<T>(c, fp64);
  if (fp64) {
    a.buf = (typename Cx<T>::t *)c.d_buf; a.t = (T *)c.d_t; a.U = (T *)c.d_U;
    a.Y = (T *)c.d_Y; a.RP = (T *)c.d_RP;
  } else {
    if (!c.f_buf) { c.err = "FP32 kernels need a MIXED context"; return RISM3D_BAD_STATE; }
    a.buf = (typename Cx<T>::t *)c.f_buf; a.t = (T *)c.f_t; a.U = (T *)c.f_U;
    a.Y = (T *)c.f_Y; a.RP = (T *)c.f_RP;
    if (which == 13 || which == 15) { a.U = (T *)c.f_x0; a.R0 = (const T *)c.f_R0; }
  }
  a.tw = (const typename Cx<T>::t *)(fp64 ? (void *)c.d_tw : (void *)c.d_twf);
  DevState saved, run;
  if (!cuda_ok(c, cudaStreamSynchronize(c.stream), "time_kernel")) return RISM3D_CUDA_ERROR;
  cudaMemcpy(&saved, c.d_state, sizeof(DevState), cudaMemcpyDeviceToHost);
  run = saved;
  run.done = 0; run.after_done = 0; run.mode = 2; run.count = 0; run.upd_slot = 0;
  run.measure = 1;
  run.s1 = 0.25; run.s2 = 0.25;
  cudaMemcpy(c.d_state, &run, sizeof(DevState), cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // the launch shapes of the solve (launch_iteration)
  const int ba = wave_blocks(k_pass_a<T, V, CLOS, false>, a.n, 1),
            bar = wave_blocks(k_pass_a<T, V, CLOS, true>, a.n, 1),
            bk = wave_blocks(k_kspace<T, V>, a.n / 2, 1);
  cudaEventRecord(e0, c.stream);
  bool fused_done = false;
  if constexpr (sizeof(T) == 4 && V <= 2) {
    // the fused-axis passes the FP32 solve runs (ids as below; 14: one
    // cuFFT transform along z)
    if (c.xfused && which != 14) {
      if (c.nx == 256) time_fused<V, CLOS, 16>(c, a, which, reps);
      else time_fused<V, CLOS, 8>(c, a, which, reps);
      fused_done = true;
    }
  }
  if (which == 14) {
    if (!c.plan32z) { c.err = "no z-axis plan (fused-axis passes are off)"; return RISM3D_BAD_STATE; }
    cufftSetStream(c.plan32z, c.stream);
    for (int r = 0; r < reps; ++r) {
      if constexpr (sizeof(T) == 4)
        cufftExecC2C(c.plan32z, (cufftComplex *)a.buf, (cufftComplex *)a.buf, CUFFT_FORWARD);
    }
    fused_done = true;
  }
  for (int r = 0; r < reps && !fused_done; ++r) {
    switch (which) {
      case 0: case 10: k_pass_a<T, V, CLOS, false><<<ba, kThreads, 0, c.stream>>>(a); break;
      case 13:
        if constexpr (V <= 2) {
          if (c.pipe_r) {
            k_pass_a_pipe<T, V, CLOS, true><<<pipe_a_blocks<T, V, CLOS, true>(c), kThreads,
                                              pass_r_pipe_smem<T, V>(), c.stream>>>(a);
            break;
          }
        }
        k_pass_a<T, V, CLOS, true><<<bar, kThreads, 0, c.stream>>>(a);
        break;
      case 1: case 11: k_kspace<T, V><<<bk, kThreads, 0, c.stream>>>(a); break;
      case 15: launch_pass_r<T, V, CLOS, true>(c, a); break;
      default: launch_pass_r<T, V, CLOS, false>(c, a); break;
    }
  }
  cudaEventRecord(e1, c.stream);
  c.launches += reps;
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaMemcpy(c.d_state, &saved, sizeof(DevState), cudaMemcpyHostToDevice);
  c.solved = false;
  c.have_forces = false;
  if (!cuda_ok(c, e, "time_kernel")) return RISM3D_CUDA_ERROR;
  *ms = t / reps;
  return RISM3D_OK;
}

template <int V>
int time_c(Context &c, int which, int reps, double *ms) {
  const bool kh = c.prm.closure == RISM3D_KH;
  if (which < 10) return kh ? time_kernel_t<double, V, 0>(c, which, reps, ms)
                            : time_kernel_t<double, V, 1>(c, which, reps, ms);
  return kh ? time_kernel_t<float, V, 0>(c, which, reps, ms)
            : time_kernel_t<float, V, 1>(c, which, reps, ms);
}

template <int V>
int solve_c(Context &c, int cu) {
  return c.prm.closure == RISM3D_KH ? solve_v<V, 0>(c, cu) : solve_v<V, 1>(c, cu);
}

}  // namespace

template <typename T, int V>
cudaError_t pipe_r_attrs() {
  const int b = (int)pass_r_pipe_smem<T, V>();
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_pass_r_pipe<T, V, 0, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_pipe<T, V, 1, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_pipe<T, V, 0, true>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_pipe<T, V, 1, true>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_a_pipe<T, V, 0, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_a_pipe<T, V, 1, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_a_pipe<T, V, 0, true>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_a_pipe<T, V, 1, true>, at, b);
  return e;
}

template <typename T, int V>
cudaError_t bulk_r_attrs() {
  const int b = (int)bulk_smem<T, V>();
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_pass_r_bulk<T, V, 0, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_bulk<T, V, 1, false>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_bulk<T, V, 0, true>, at, b);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_pass_r_bulk<T, V, 1, true>, at, b);
  return e;
}

// Pass R for natv <= 2: the cp.async pipeline, or with RISM3D_BULK_R=1 the
// bulk-copy stream (every stream's chunk offset must be 16-byte aligned: N
// a multiple of 4).  RISM3D_NO_PIPE_R=1 keeps the plain grid-stride pass.
int setup_pipe_r(Context &c) {
  c.pipe_r = false;
  c.bulk_r = false;
  const char *off = getenv("RISM3D_NO_PIPE_R");
  if ((off && off[0] == '1') || c.natv > 2) return RISM3D_OK;
  cudaError_t e = c.natv == 1 ? pipe_r_attrs<double, 1>() : pipe_r_attrs<double, 2>();
  if (e == cudaSuccess) e = c.natv == 1 ? pipe_r_attrs<float, 1>() : pipe_r_attrs<float, 2>();
  if (!cuda_ok(c, e, "pass R attributes")) return RISM3D_CUDA_ERROR;
  c.pipe_r = true;
  const char *bulk = getenv("RISM3D_BULK_R");
  if (!bulk || bulk[0] != '1' || c.n % 4 != 0) return RISM3D_OK;
  e = c.natv == 1 ? bulk_r_attrs<double, 1>() : bulk_r_attrs<double, 2>();
  if (e == cudaSuccess) e = c.natv == 1 ? bulk_r_attrs<float, 1>() : bulk_r_attrs<float, 2>();
  if (!cuda_ok(c, e, "bulk pass R attributes")) return RISM3D_CUDA_ERROR;
  c.bulk_r = true;
  return RISM3D_OK;
}

// TMA form of the fused pass K (nx = ny = 256): a tensor map over the FP32
// transform buffer seen as (2 nx floats) x (ny nz rows), boxes of 16
// complex columns x 256 rows with the 128B swizzle, and the [kz][kx][ky]
// FP32 copy of beta fk.  RISM3D_KY_TMA=0 keeps the register/shared-memory form.
int setup_kspace_tma(Context &c) {
  const char *off = getenv("RISM3D_KY_TMA");
  if (off && off[0] == '0') return RISM3D_OK;
  typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault,
                                       &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return RISM3D_OK;                            // no TMA entry point: the other form
  }
  cudaError_t e = cudaFuncSetAttribute(k_kspace_yt<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kKySmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_kspace_yt<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kKySmem);
  if (!cuda_ok(c, e, "TMA pass K attributes")) return RISM3D_CUDA_ERROR;
  CUtensorMap *map = new CUtensorMap;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * c.nx, (cuuint64_t)c.ny * c.nz};
  const cuuint64_t strides[1] = {(cuuint64_t)2 * c.nx * sizeof(float)};
  const cuuint32_t box[2] = {32, 256}, estr[2] = {1, 1};
  const CUresult r = ((EncodeTiled)fn)(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, c.f_buf, dims,
                                       strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                       CU_TENSOR_MAP_SWIZZLE_128B,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    delete map;
    c.err = "cuTensorMapEncodeTiled failed: " + std::to_string((int)r);
    return RISM3D_CUDA_ERROR;
  }
  if (!cuda_ok(c, cudaMalloc(&c.d_fkt, sizeof(float2) * (size_t)(c.n / 2)), "alloc fk columns")) {
    delete map;
    return RISM3D_CUDA_ERROR;
  }
  c.ky_map = map;
  return RISM3D_OK;
}

int fused_fk_columns(Context &c) {
  if (!c.d_fkt) return RISM3D_OK;
  k_fk_columns<<<dim3((unsigned)(c.nx + 31) / 32, (unsigned)(c.ny + 31) / 32, (unsigned)c.nz / 2),
                 dim3(32, 8), 0, c.stream>>>(c.nx, c.ny, c.d_fkh, c.d_fkt);
  if (!cuda_ok(c, cudaGetLastError(), "k_fk_columns")) return RISM3D_CUDA_ERROR;
  c.launches += 1;
  return RISM3D_OK;
}

int setup_fused_axes(Context &c) {
  c.xfused = false;
  // opt-in (RISM3D_XFFT=1) until the fused passes beat the 3D cuFFT path
  const char *on = getenv("RISM3D_XFFT");
  if (!on || on[0] != '1') return RISM3D_OK;
  if (c.prm.precision != RISM3D_MIXED || c.nb != 1 || c.natv < 1 || c.natv > 2 ||
      c.nx != c.ny || (c.nx != 256 && c.nx != 64) || c.nz % 2 != 0)
    return RISM3D_OK;
  cudaError_t e = cudaSuccess;
  if (c.nx == 256) {
    const int ks = (int)KYLayout<16>::bytes();
    e = cudaFuncSetAttribute(k_kspace_y<1, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ks);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_kspace_y<2, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ks);
  } else {
    const int ks = (int)KYLayout<8>::bytes();
    e = cudaFuncSetAttribute(k_kspace_y<1, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ks);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_kspace_y<2, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ks);
  }
  if (!cuda_ok(c, e, "fused-axis kernel attributes")) return RISM3D_CUDA_ERROR;
  if (c.nx == 256) {
    const int rc = setup_kspace_tma(c);
    if (rc != RISM3D_OK) return rc;
  }
  std::vector<float2> roots(c.nx);
  for (int m = 0; m < c.nx; ++m) {
    const double ang = 2.0 * kPi * m / c.nx;
    roots[m] = make_float2((float)cos(ang), (float)-sin(ang));
  }
  if (!cuda_ok(c, cudaMalloc(&c.d_xroots, sizeof(float2) * c.nx), "alloc roots") ||
      !cuda_ok(c, cudaMemcpy(c.d_xroots, roots.data(), sizeof(float2) * c.nx, cudaMemcpyHostToDevice),
               "copy roots"))
    return RISM3D_CUDA_ERROR;
  // transforms along z: one per (x, y) column, stride nx ny, columns adjacent
  int nz = c.nz, emb = c.nz;
  const int nxy = c.nx * c.ny;
  if (!cufft_ok(c, cufftPlanMany(&c.plan32z, 1, &nz, &emb, nxy, 1, &emb, nxy, 1, CUFFT_C2C, nxy),
                "cufftPlanMany z"))
    return RISM3D_CUFFT_ERROR;
  c.xfused = true;
  return RISM3D_OK;
}

int build_twiddles(Context &c) {
  std::vector<double2> tw(c.nx + c.ny + c.nz);
  std::vector<float2> twf(tw.size());
  int off = 0;
  for (int d = 0; d < 3; ++d) {
    int nd = d == 0 ? c.nx : (d == 1 ? c.ny : c.nz);
    for (int i = 0; i < nd; ++i) {
      double a = kPi / nd * (i - nd / 2);
      tw[off + i] = make_double2(cos(a), -sin(a));
      twf[off + i] = make_float2((float)cos(a), (float)-sin(a));
    }
    off += nd;
  }
  if (!cuda_ok(c, cudaMemcpyAsync(c.d_tw, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice, c.stream), "twiddles") ||
      !cuda_ok(c, cudaMemcpyAsync(c.d_twf, twf.data(), sizeof(float2) * twf.size(), cudaMemcpyHostToDevice, c.stream), "twiddles") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "twiddles"))
    return RISM3D_CUDA_ERROR;
  return RISM3D_OK;
}

// Natural cubic spline of every chi_ab table (same tridiagonal sweep as
// spline.cc:4-43), uploaded as [knot][ab][y c0 c1 c2].
void spline_coefficients(const double *xp, const double *yp, int np, double *out,
                         size_t stride) {
  std::vector<double> a(np), b(np), cc(np), d(np), s(np);
  const int m = np - 2;
  for (int k = 1; k <= m; ++k) {
    double hl = xp[k] - xp[k - 1], hr = xp[k + 1] - xp[k];
    a[k] = hl / (hl + hr);
    b[k] = 1 - a[k];
    double q1 = (yp[k + 1] - yp[k]) / hr, q2 = (yp[k] - yp[k - 1]) / hl;
    cc[k] = 6.0 * ((q1 - q2) / (hl + hr));
    d[k] = 2.0;
  }
  for (int k = 1; k < m; ++k) {
    b[k] = b[k] / d[k];
    cc[k] = cc[k] / d[k];
    d[k + 1] = d[k + 1] - a[k + 1] * b[k];
    cc[k + 1] = cc[k + 1] - a[k + 1] * cc[k];
  }
  s[m] = cc[m] / d[m];
  for (int k = m - 1; k >= 1; --k) s[k] = cc[k] - b[k] * s[k + 1];
  s[0] = s[m + 1] = 0.0;
  for (int k = 0; k < np; ++k) {
    double *o = out + (size_t)k * stride;
    o[0] = yp[k];
    o[1] = o[2] = o[3] = 0.0;
    if (k <= m) {
      double h = xp[k + 1] - xp[k];
      double c1 = s[k] / 2.0;
      double c2 = (s[k + 1] - s[k]) / (6.0 * h);
      o[1] = (yp[k + 1] - yp[k]) / h - c1 * h - c2 * h * h;
      o[2] = c1;
      o[3] = c2;
    }
  }
}

int upload_chi(Context &c) {
  const int V = c.natv, nt = c.ntab;
  c.chi.ntab = nt;
  c.chi.dk = kPi / (c.xdr * nt);                 // solvent_read.cc:82
  // largest |k| on the grid must be inside the table (solvent_spline.cu:18-21)
  double kx = 2.0 * kPi * (c.nx / 2.0 - 0.5) / c.prm.box[0];
  double ky = 2.0 * kPi * (c.ny / 2.0 - 0.5) / c.prm.box[1];
  double kz = 2.0 * kPi * (c.nz / 2.0 - 0.5) / c.prm.box[2];
  double kmax = sqrt(kx * kx + ky * ky + kz * kz);
  if (kmax > c.chi.dk * nt) {
    c.err = "insufficient maximal T tabulated";
    return RISM3D_BAD_INPUT;
  }
  std::vector<double> xp(nt);
  for (int i = 0; i < nt; ++i) xp[i] = c.chi.dk * (i + 1);
  std::vector<double> tab((size_t)nt * V * V * 4, 0.0);
  for (int va = 0; va < V; ++va)
    for (int vb = 0; vb < V; ++vb)
      spline_coefficients(xp.data(), &c.xvv_host[((size_t)va * V + vb) * nt], nt,
                          &tab[(size_t)(va * V + vb) * 4], (size_t)V * V * 4);
  // the captured iteration graphs embed the table pointers
  if (c.graph64) { cudaGraphExecDestroy(c.graph64); c.graph64 = nullptr; }
  if (c.graph32) { cudaGraphExecDestroy(c.graph32); c.graph32 = nullptr; }
  if (c.graph32r) { cudaGraphExecDestroy(c.graph32r); c.graph32r = nullptr; }
  for (cudaGraphExec_t *g : {&c.loop64, &c.loop32, &c.loop32r}) {
    if (*g) cudaGraphExecDestroy(*g);
    *g = nullptr;
  }
  // Cubic cells: evaluate the spline once per distinct |k|^2 (the sorted
  // unique-|k| table of initialize_g.cu:31-43, indexed directly).
  if (c.d_xs) { cudaFree(c.d_xs); c.d_xs = nullptr; c.nxs = 0; }
  if (c.d_xs32) { cudaFree(c.d_xs32); c.d_xs32 = nullptr; }
  if (c.nx == c.ny && c.nx == c.nz && c.prm.box[0] == c.prm.box[1] &&
      c.prm.box[0] == c.prm.box[2]) {
    const long long nm = c.nx - 1;
    const int nidx = (int)((3 * nm * nm - 3) / 8 + 1);
    std::vector<double> xs((size_t)nidx * V * V);
    for (int idx = 0; idx < nidx; ++idx) {
      const double kk = kPi / c.prm.box[0] * sqrt((double)(8LL * idx + 3));
      int klo = 0, khi = nt - 1;                               // splint.cc:9-16
      while (khi - klo > 1) {
        int k = (khi + klo) >> 1;
        if (xp[k] > kk) khi = k; else klo = k;
      }
      const double t = kk - xp[klo];
      for (int ab = 0; ab < V * V; ++ab) {
        const double *o = &tab[((size_t)klo * V * V + ab) * 4];
        xs[(size_t)idx * V * V + ab] = ((o[3] * t + o[2]) * t + o[1]) * t + o[0];
      }
    }
    std::vector<float> xs32(xs.begin(), xs.end());     // the FP32 passes' copy
    if (!cuda_ok(c, cudaMalloc(&c.d_xs, sizeof(double) * xs.size()), "chi table alloc") ||
        !cuda_ok(c, cudaMemcpy(c.d_xs, xs.data(), sizeof(double) * xs.size(), cudaMemcpyHostToDevice), "chi table copy") ||
        !cuda_ok(c, cudaMalloc(&c.d_xs32, sizeof(float) * xs32.size()), "chi table alloc") ||
        !cuda_ok(c, cudaMemcpy(c.d_xs32, xs32.data(), sizeof(float) * xs32.size(), cudaMemcpyHostToDevice), "chi table copy"))
      return RISM3D_CUDA_ERROR;
    c.nxs = nidx;
  }
  if (c.chi.d_coef) cudaFree(c.chi.d_coef);
  if (!cuda_ok(c, cudaMalloc(&c.chi.d_coef, sizeof(double) * tab.size()), "chi alloc") ||
      !cuda_ok(c, cudaMemcpyAsync(c.chi.d_coef, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c.stream), "chi copy") ||
      !cuda_ok(c, cudaStreamSynchronize(c.stream), "chi"))
    return RISM3D_CUDA_ERROR;
  return RISM3D_OK;
}

int time_kernel(Context &c, int which, int reps, double *ms) {
  if (which == 20) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    for (int r = 0; r < reps; ++r) launch_potential_r(c);
    cudaEventRecord(e1, c.stream);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!cuda_ok(c, e, "time_kernel")) return RISM3D_CUDA_ERROR;
    *ms = t / reps;
    return RISM3D_OK;
  }
  if (!(which >= 0 && which <= 2) && !(which >= 10 && which <= 15)) {
    c.err = "unknown kernel id";
    return RISM3D_BAD_INPUT;
  }
  switch (c.natv) {
    case 1: return time_c<1>(c, which, reps, ms);
    case 2: return time_c<2>(c, which, reps, ms);
    case 3: return time_c<3>(c, which, reps, ms);
    case 4: return time_c<4>(c, which, reps, ms);
    case 5: return time_c<5>(c, which, reps, ms);
    case 6: return time_c<6>(c, which, reps, ms);
    case 7: return time_c<7>(c, which, reps, ms);
    case 8: return time_c<8>(c, which, reps, ms);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

// The FP64 k-space pass alone on a caller-packed buffer (one solute): the
// OZ product h(k) = chi(k) (c(k) - q cf fk) between the two transforms, used
// by the adjoint solve to apply the same discrete operator as the iteration.
template <int V>
int oz_kspace_v(Context &c, double2 *buf, const StageParams *sp, DevState *st) {
  IterArgs<double> a = make_args<double>(c, true);
  a.buf = buf; a.sp = sp; a.st = st;
  k_kspace<double, V><<<dim3(wave_blocks(k_kspace<double, V>, c.n / 2, 1), 1), kThreads, 0,
                        c.stream>>>(a);
  c.launches += 1;
  return cuda_ok(c, cudaGetLastError(), "oz k-space") ? RISM3D_OK : RISM3D_CUDA_ERROR;
}

// The same OZ pass in FP32 (the adjoint's FP32 operator)
template <int V>
int oz_kspace32_v(Context &c, float2 *buf, const StageParams *sp, DevState *st) {
  IterArgs<float> a = make_args<float>(c, false);
  a.buf = buf; a.sp = sp; a.st = st;
  k_kspace<float, V><<<dim3(wave_blocks(k_kspace<float, V>, c.n / 2, 1), 1), kThreads, 0,
                       c.stream>>>(a);
  c.launches += 1;
  return cuda_ok(c, cudaGetLastError(), "oz k-space") ? RISM3D_OK : RISM3D_CUDA_ERROR;
}

int launch_oz_kspace32(Context &c, float2 *buf, const StageParams *sp, DevState *st) {
  switch (c.natv) {
    case 1: return oz_kspace32_v<1>(c, buf, sp, st);
    case 2: return oz_kspace32_v<2>(c, buf, sp, st);
    case 3: return oz_kspace32_v<3>(c, buf, sp, st);
    case 4: return oz_kspace32_v<4>(c, buf, sp, st);
    case 5: return oz_kspace32_v<5>(c, buf, sp, st);
    case 6: return oz_kspace32_v<6>(c, buf, sp, st);
    case 7: return oz_kspace32_v<7>(c, buf, sp, st);
    case 8: return oz_kspace32_v<8>(c, buf, sp, st);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

int launch_oz_kspace(Context &c, double2 *buf, const StageParams *sp, DevState *st) {
  switch (c.natv) {
    case 1: return oz_kspace_v<1>(c, buf, sp, st);
    case 2: return oz_kspace_v<2>(c, buf, sp, st);
    case 3: return oz_kspace_v<3>(c, buf, sp, st);
    case 4: return oz_kspace_v<4>(c, buf, sp, st);
    case 5: return oz_kspace_v<5>(c, buf, sp, st);
    case 6: return oz_kspace_v<6>(c, buf, sp, st);
    case 7: return oz_kspace_v<7>(c, buf, sp, st);
    case 8: return oz_kspace_v<8>(c, buf, sp, st);
  }
  return RISM3D_UNSUPPORTED_SHAPE;
}

int run_solve(Context &c, int chargeup) {
  switch (c.natv) {
    case 1: return solve_c<1>(c, chargeup);
    case 2: return solve_c<2>(c, chargeup);
    case 3: return solve_c<3>(c, chargeup);
    case 4: return solve_c<4>(c, chargeup);
    case 5: return solve_c<5>(c, chargeup);
    case 6: return solve_c<6>(c, chargeup);
    case 7: return solve_c<7>(c, chargeup);
    case 8: return solve_c<8>(c, chargeup);
  }
  c.err = "unsupported number of solvent sites";
  return RISM3D_UNSUPPORTED_SHAPE;
}

}  // namespace rism3d
