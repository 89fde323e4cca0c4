// Half-shifted 3D transform of real site grids, packed two sites per
// complex transform (fft3d.cu:4-94): the pre-twiddle before the forward
// cuFFT and the post-twiddle after the inverse, as kernels over x-fastest
// grids of n points.  Shared by the adjoint solve and the RMDFT correction;
// device code only.
#pragma once

#include "rism3d_impl.h"

namespace rism3d {
namespace {

// dir = (-1)^(ix+iy+iz) and dkf = exp(-i pi (x/nx + y/ny + z/nz)) at point j,
// from the per-axis twiddle rows tw = [nx][ny][nz]
__device__ __forceinline__ void point_dir_dkf(long long j, int nx, int ny, const double2 *tw,
                                              int &dir, double2 &dkf) {
  const long long r = j / nx;
  const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
  dir = ((ix + iy + iz) & 1) ? -1 : 1;
  const double2 a = tw[ix], b = tw[nx + iy], c = tw[nx + ny + iz];
  const double2 ab = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  dkf = make_double2(ab.x * c.x - ab.y * c.y, ab.x * c.y + ab.y * c.x);
}

// real grids v[V][N] -> packed pairs buf[P][N] with the forward pre-twiddle
// dir dkf (timekf, fft3d.cu:41-49)
__global__ void k_pack(long long n, int nv, int nx, int ny, const double2 *tw,
                       const double *v, double2 *buf) {
  const int P = (nv + 1) / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    double2 w;
    point_dir_dkf(j, nx, ny, tw, dir, w);
    for (int p = 0; p < P; ++p) {
      const double a = v[(size_t)(2 * p) * n + j];
      const double b = (2 * p + 1 < nv) ? v[(size_t)(2 * p + 1) * n + j] : 0.0;
      buf[(size_t)p * n + j] = make_double2(dir * (a * w.x - b * w.y), dir * (a * w.y + b * w.x));
    }
  }
}

// packed pairs after the inverse FFT -> real grids, post-twiddle
// (1/V) dir conj(dkf) (timekb, fft3d.cu:52-60)
__global__ void k_unpack(long long n, int nv, int nx, int ny, const double2 *tw, double invvol,
                         const double2 *buf, double *out) {
  const int P = (nv + 1) / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    double2 w;
    point_dir_dkf(j, nx, ny, tw, dir, w);
    const double s = invvol * dir;
    for (int p = 0; p < P; ++p) {
      const double2 z = buf[(size_t)p * n + j];
      const double re = s * (z.x * w.x + z.y * w.y), im = s * (z.y * w.x - z.x * w.y);
      out[(size_t)(2 * p) * n + j] = re;
      if (2 * p + 1 < nv) out[(size_t)(2 * p + 1) * n + j] = im;
    }
  }
}

// FP32 forms of the two passes above (the adjoint's FP32 operator): the
// same pre- and post-twiddles from the FP32 twiddle rows
__device__ __forceinline__ void point_dir_dkf32(long long j, int nx, int ny, const float2 *tw,
                                                int &dir, float2 &dkf) {
  const long long r = j / nx;
  const int ix = (int)(j - r * nx), iy = (int)(r % ny), iz = (int)(r / ny);
  dir = ((ix + iy + iz) & 1) ? -1 : 1;
  const float2 a = tw[ix], b = tw[nx + iy], c = tw[nx + ny + iz];
  const float2 ab = make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  dkf = make_float2(ab.x * c.x - ab.y * c.y, ab.x * c.y + ab.y * c.x);
}

__global__ void k_pack32(long long n, int nv, int nx, int ny, const float2 *tw,
                         const float *v, float2 *buf) {
  const int P = (nv + 1) / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    float2 w;
    point_dir_dkf32(j, nx, ny, tw, dir, w);
    const float d = (float)dir;
    for (int p = 0; p < P; ++p) {
      const float a = v[(size_t)(2 * p) * n + j];
      const float b = (2 * p + 1 < nv) ? v[(size_t)(2 * p + 1) * n + j] : 0.0f;
      buf[(size_t)p * n + j] = make_float2(d * (a * w.x - b * w.y), d * (a * w.y + b * w.x));
    }
  }
}

__global__ void k_unpack32(long long n, int nv, int nx, int ny, const float2 *tw, float invvol,
                           const float2 *buf, float *out) {
  const int P = (nv + 1) / 2;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
    int dir;
    float2 w;
    point_dir_dkf32(j, nx, ny, tw, dir, w);
    const float s = invvol * (float)dir;
    for (int p = 0; p < P; ++p) {
      const float2 z = buf[(size_t)p * n + j];
      const float re = s * (z.x * w.x + z.y * w.y), im = s * (z.y * w.x - z.x * w.y);
      out[(size_t)(2 * p) * n + j] = re;
      if (2 * p + 1 < nv) out[(size_t)(2 * p + 1) * n + j] = im;
    }
  }
}

}  // namespace
}  // namespace rism3d
