// rism3d_exchem_noalloc: the excess-chemical-potential and PMV integrals of
// a converged solution, for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they want these
// integrals: a host application whose own pool allocator has already
// reserved the free device memory (a cudaMalloc then fails or fragments its
// pool), or code running in a latency-critical loop where cudaMalloc's
// implicit device synchronisation is not acceptable.  This entry point takes
// the grids in the caller's device memory, writes the sums to the caller's
// host array, and allocates nothing: the block partial sums of the
// reduction live in one file-scope static device array of fixed size, which
// every GPU that loads this library keeps until the process exits.
//
// The kernel is the per-point integrand pass of the context-based
// observables (k_observe in observe.cu), taking the absolute t directly.
#include <mutex>

#include "rism3d_impl.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 592;                        // 148 SMs x 4 blocks
constexpr int kSums = 4 * RISM3D_MAX_SITES;            // KH, HNC, GF, c per site
constexpr int kMaxDevices = 64;

// Scratch: [kSums][kMaxBlocks] block partials, then [kSums] final sums.
// 32 x 593 doubles = 148 KiB.
static __device__ __align__(256) double g_scratch[kSums * (kMaxBlocks + 1)];

std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices] = {};

template <int V, int CLOS>
__global__ void __launch_bounds__(kThreads)
k_exchem_partials(long long n, const double *__restrict__ h,
                  const double *__restrict__ t, double *part) {
  constexpr int NS = 4 * V;
  __shared__ double red[kThreads / 32][NS];
  double acc[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) acc[k] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double hh = h[(size_t)v * n + j];
      const double tt = t[(size_t)v * n + j];
      const double c = hh - tt;
      const double hnc = hh * 0.5 * tt - c;                     // cal_exchem.cu:98
      const double gf = -(hh * 0.5 + 1.0) * c;                  // cal_exchem.cu:130
      acc[4 * v + 0] += CLOS == 0 ? (hh > 0.0 ? gf : hnc) : hnc; // :61-65
      acc[4 * v + 1] += hnc;
      acc[4 * v + 2] += gf;
      acc[4 * v + 3] += c;                                      // cal_pmv.cu:31
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
    part[(size_t)k * kMaxBlocks + blockIdx.x] = s;
  }
}

// out[k] = sum over the nblocks partials of sum k, in a fixed order
__global__ void k_exchem_sum(const double *part, int nblocks, double *out) {
  __shared__ double red[kThreads];
  const int k = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += part[(size_t)k * kMaxBlocks + b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = red[0];
}

template <int V, int CLOS>
void launch(long long n, int nb, const double *h, const double *t, double *part,
            cudaStream_t st) {
  k_exchem_partials<V, CLOS><<<nb, kThreads, 0, st>>>(n, h, t, part);
}

template <int V>
void launch_c(int closure, long long n, int nb, const double *h, const double *t,
              double *part, cudaStream_t st) {
  if (closure == RISM3D_KH) launch<V, 0>(n, nb, h, t, part, st);
  else launch<V, 1>(n, nb, h, t, part, st);
}

}  // namespace

extern "C" int rism3d_exchem_noalloc(int closure, int natv, long long n, double dv,
                                     double temperature, const double *rho,
                                     const double *d_h, const double *d_t, void *stream,
                                     double *out) {
  using namespace rism3d;
  if (natv < 1 || natv > RISM3D_MAX_SITES) {
    set_create_error("rism3d_exchem_noalloc: natv must be 1..8 (the static scratch holds "
                     "4 sums per site for at most 8 sites)");
    return RISM3D_UNSUPPORTED_SHAPE;
  }
  if (n < 1 || n >= (1LL << 31)) {
    set_create_error("rism3d_exchem_noalloc: the grid must have 1 .. 2^31-1 points");
    return RISM3D_UNSUPPORTED_SHAPE;
  }
  if (!rho || !d_h || !d_t || !out || !(dv > 0) || !(temperature > 0) ||
      (closure != RISM3D_KH && closure != RISM3D_HNC)) {
    set_create_error("rism3d_exchem_noalloc: bad argument");
    return RISM3D_BAD_INPUT;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    set_create_error("rism3d_exchem_noalloc: no usable current device");
    return RISM3D_NO_DEVICE;
  }
  double *scratch = nullptr;
  {
    // once per device, with that device current: the device address of the
    // static array (its host-side name is only a stand-in)
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        set_create_error(std::string("rism3d_exchem_noalloc: cudaGetSymbolAddress: ") +
                         cudaGetErrorString(e));
        return RISM3D_CUDA_ERROR;
      }
      g_scratch_ptr[dev] = (double *)p;
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  long long want = (n + kThreads - 1) / kThreads;
  const int nb = (int)(want < kMaxBlocks ? want : kMaxBlocks);
  double *sums = scratch + (size_t)kSums * kMaxBlocks;
  // every partial slot read below is written by this call, so nothing in the
  // scratch needs clearing first
  switch (natv) {
    case 1: launch_c<1>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 2: launch_c<2>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 3: launch_c<3>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 4: launch_c<4>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 5: launch_c<5>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 6: launch_c<6>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 7: launch_c<7>(closure, n, nb, d_h, d_t, scratch, st); break;
    case 8: launch_c<8>(closure, n, nb, d_h, d_t, scratch, st); break;
  }
  // a launch that failed (no kernel image, bad configuration) must not let
  // the copy below return the previous call's sums from the shared array
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_exchem_sum<<<4 * natv, kThreads, 0, st>>>(scratch, nb, sums);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_create_error(std::string("rism3d_exchem_noalloc: launch: ") + cudaGetErrorString(e));
    return RISM3D_CUDA_ERROR;
  }
  double raw[kSums];
  e = cudaMemcpyAsync(raw, sums, sizeof(double) * 4 * natv, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_create_error(std::string("rism3d_exchem_noalloc: ") + cudaGetErrorString(e));
    return RISM3D_CUDA_ERROR;
  }
  // output_xmu.cu:19-73 (J/mol) and cal_pmv.cu:16 (sum rho dv int c)
  const double ibeta = kAvogadro * kBoltzmann * temperature;
  double cuv = 0.0;
  for (int v = 0; v < natv; ++v) {
    out[v] = ibeta * raw[4 * v + 0] * rho[v] * dv;
    out[natv + v] = ibeta * raw[4 * v + 1] * rho[v] * dv;
    out[2 * natv + v] = ibeta * raw[4 * v + 2] * rho[v] * dv;
    cuv += raw[4 * v + 3] * rho[v];
  }
  out[3 * natv] = cuv * dv;
  return RISM3D_OK;
}
