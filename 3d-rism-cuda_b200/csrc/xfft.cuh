// Register-resident DFTs of one grid line (256 or 64 complex FP32 points)
// held by a group of E threads, E points each (n = E * E), used to fold one
// axis of the 3D transform into a streaming pass.
//
// Layout: thread t of the group holds the points x = t + E j (j < E), so that
// the E threads of a group read and write E consecutive points at a time
// (coalesced).  The transform is the two-stage Cooley-Tukey split n = E x E:
//   A_t[k1] = sum_j a[t + E j] W_E^(j k1)             (E-point DFT, in registers)
//   A_t[k1] *= W_n^(t k1)                             (twiddle)
//   X[k1 + E k2] = sum_t A_t[k1] W_E^(t k2)           (E-point DFT across the
//                                                      group, after a transpose
//                                                      through shared memory)
// so thread t' ends up holding X[t' + E k2], k2 < E: the same layout as the
// input, and a forward and an inverse transform compose without any
// reordering.  INV selects the unnormalised inverse (conjugate roots).
//
// The 16- and 8-point DFTs are radix-4 / radix-2 splits written out with
// their exact twiddles (cos and sin of multiples of pi/8).
#pragma once

#include <cuda_runtime.h>

namespace rism3d {
namespace xfft {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i (forward) or +i (inverse)
template <bool INV> __device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// 4-point DFT in place
template <bool INV>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
  const float2 s13 = cadd(a1, a3), d13 = mul_mi<INV>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

// 16-point DFT in registers, natural order in and out.  n = n1 + 4 n2,
// k = k2 + 4 k1: 4-point DFTs over n2, twiddles W16^(n1 k2), 4-point DFTs
// over n1, then the 4 x 4 index transpose.
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
  constexpr float c1 = 0.92387953251128674f;   // cos(pi/8)
  constexpr float s1 = 0.38268343236508977f;   // sin(pi/8)
  constexpr float h = 0.70710678118654752f;    // cos(pi/4)
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4<INV>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
  // v[n1 + 4 k2] holds A[n1][k2]; twiddle W16^(n1 k2) = e^(-2 pi i n1 k2 / 16)
  // (conjugated for the inverse)
  const float sg = INV ? 1.0f : -1.0f;
  const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h),
               w3 = make_float2(s1, sg * c1), w4 = make_float2(0.0f, sg),
               w6 = make_float2(-h, sg * h), w9 = make_float2(-c1, -sg * s1);
  v[5] = cmulf(v[5], w1);    // n1 1, k2 1
  v[9] = cmulf(v[9], w2);    // n1 1, k2 2
  v[13] = cmulf(v[13], w3);  // n1 1, k2 3
  v[6] = cmulf(v[6], w2);    // n1 2, k2 1
  v[10] = cmulf(v[10], w4);  // n1 2, k2 2
  v[14] = cmulf(v[14], w6);  // n1 2, k2 3
  v[7] = cmulf(v[7], w3);    // n1 3, k2 1
  v[11] = cmulf(v[11], w6);  // n1 3, k2 2
  v[15] = cmulf(v[15], w9);  // n1 3, k2 3
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) dft4<INV>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
  // v[4 k2 + k1] holds X[k2 + 4 k1]
  float2 t[16];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) t[k2 + 4 * k1] = v[4 * k2 + k1];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// 8-point DFT in registers, natural order: n = n1 + 2 n2 (n1 < 2, n2 < 4),
// k = k2 + 4 k1: 4-point DFTs over n2, twiddles W8^(n1 k2), 2-point DFTs.
template <bool INV>
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
  constexpr float h = 0.70710678118654752f;
  dft4<INV>(v[0], v[2], v[4], v[6]);
  dft4<INV>(v[1], v[3], v[5], v[7]);
  // v[2 k2 + n1] = A[n1][k2]; twiddle for n1 = 1: W8^k2
  const float sg = INV ? 1.0f : -1.0f;
  v[3] = cmulf(v[3], make_float2(h, sg * h));
  v[5] = mul_mi<INV>(v[5]);
  v[7] = cmulf(v[7], make_float2(-h, sg * h));
  float2 t[8];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    t[k2] = cadd(v[2 * k2], v[2 * k2 + 1]);
    t[k2 + 4] = csub(v[2 * k2], v[2 * k2 + 1]);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = t[i];
}

template <int E, bool INV> __device__ __forceinline__ void dft_small(float2 (&v)[E]);
template <> __device__ __forceinline__ void dft_small<16, false>(float2 (&v)[16]) { dft16<false>(v); }
template <> __device__ __forceinline__ void dft_small<16, true>(float2 (&v)[16]) { dft16<true>(v); }
template <> __device__ __forceinline__ void dft_small<8, false>(float2 (&v)[8]) { dft8<false>(v); }
template <> __device__ __forceinline__ void dft_small<8, true>(float2 (&v)[8]) { dft8<true>(v); }

// First stage and twiddle: v[j] = x[t + E j] -> v[k1] = A_t[k1] W_n^(t k1)
// (roots: W_n^m = e^(-2 pi i m / n), m < n, conjugated for the inverse)
template <int E, bool INV>
__device__ __forceinline__ void stage1(float2 (&v)[E], int t, const float2 *__restrict__ roots) {
  constexpr int n = E * E;
  dft_small<E, INV>(v);
#pragma unroll
  for (int k1 = 1; k1 < E; ++k1) {
    float2 w = __ldg(roots + ((t * k1) & (n - 1)));
    if (INV) w.y = -w.y;
    v[k1] = cmulf(v[k1], w);
  }
}

// One line of n = E * E points held by a group of E consecutive lanes of
// one warp (mask): v holds x[t + E j]; on return v holds X[t + E k2].
// scratch: (E + 1) * E float2 of shared memory private to the group (rows
// padded by one so that the transpose is free of bank conflicts).
template <int E, bool INV>
__device__ __forceinline__ void line_dft(float2 (&v)[E], int t, float2 *scratch,
                                         const float2 *__restrict__ roots, unsigned mask) {
  stage1<E, INV>(v, t, roots);
  __syncwarp(mask);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) scratch[k1 * (E + 1) + t] = v[k1];
  __syncwarp(mask);
#pragma unroll
  for (int s = 0; s < E; ++s) v[s] = scratch[t * (E + 1) + s];
  dft_small<E, INV>(v);
}

}  // namespace xfft
}  // namespace rism3d
