// gh_noalloc.cu -- plaquette reduction that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a
// measurement: a host driver that is recording its own work into a CUDA graph
// (allocation is not allowed inside stream capture, and cudaMalloc / cudaFree
// synchronise the whole device), or a program whose device memory is owned by
// a fixed arena of another framework.  gh_plaquette_noalloc serves them: the
// caller passes the links (device memory, the reference's array-of-structures
// layout) and a device output, and the per-block partial sums go to a
// file-scope __device__ scratch array instead of an allocation.
//
// Limits and sharing rules (also in include/gauge_higgs_b200.h):
//  - at most GH_NOALLOC_MAX_SITES sites (8192 blocks of 128 sites, 64 KiB of
//    scratch held by every device that loads the library until the process ends);
//  - every call on a device shares the one scratch array and leaves its partial
//    sums there; each call overwrites every slot it reads, so nothing has to be
//    cleared between calls, but calls that overlap on the GPU (different
//    streams, or different host threads) race on it;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it; make that
//    first call before any stream capture.  The cached address belongs to the
//    device's primary context: it does not survive cudaDeviceReset (or any other
//    teardown of that context) — a process that resets a device must not call
//    this entry point on it afterwards;
//  - U_dev must be 16-byte aligned (it is read as complex FP64 pairs) and out_dev
//    8-byte aligned; other pointers are refused with GH_ERR_ARG before any launch.
#include <cuda_runtime.h>
#include <stdint.h>
#include <mutex>
#include <string>
#include "gh_math.cuh"
#include "../../include/gauge_higgs_b200.h"

namespace {

constexpr int NA_BLOCK = 128;
constexpr int NA_MAX_BLOCKS = 8192;
static_assert(GH_NOALLOC_MAX_SITES == NA_BLOCK * NA_MAX_BLOCKS, "scratch size and the documented limit agree");

static __device__ __align__(256) double g_noalloc_scratch[NA_MAX_BLOCKS];

struct Geo { int L[4]; int stride[4]; int V; };

template <int D, int N>
__device__ __forceinline__ ghm::Mat<N, double> ld_aos(const double* __restrict__ U, int s, int mu) {
  ghm::Mat<N, double> M;
  const double2* p = reinterpret_cast<const double2*>(U) + ((size_t)s * D + mu) * N * N;
#pragma unroll
  for (int c = 0; c < N * N; ++c) { const double2 v = __ldg(p + c); M.e[c] = ghm::mk<double>(v.x, v.y); }
  return M;
}

// Sum over the plaquettes of each block's sites: Re Tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag)
// (src/action/gauge_wilson.hpp:50-65), one partial per block into the scratch array.
template <int D, int N>
__global__ void __launch_bounds__(NA_BLOCK) k_plaq_partials(const Geo g, const double* __restrict__ U, double* partials) {
  const int s = blockIdx.x * NA_BLOCK + threadIdx.x;
  double v = 0.0;
  if (s < g.V) {
    int x[D];
    int r = s;
#pragma unroll
    for (int mu = 0; mu < D; ++mu) { x[mu] = r % g.L[mu]; r /= g.L[mu]; }
#pragma unroll
    for (int mu = 0; mu < D; ++mu) {
      const int spm = (x[mu] + 1 < g.L[mu]) ? s + g.stride[mu] : s - x[mu] * g.stride[mu];
      const ghm::Mat<N, double> Umu = ld_aos<D, N>(U, s, mu);
#pragma unroll
      for (int nu = mu + 1; nu < D; ++nu) {
        const int spn = (x[nu] + 1 < g.L[nu]) ? s + g.stride[nu] : s - x[nu] * g.stride[nu];
        const ghm::Mat<N, double> A = ghm::mm(Umu, ld_aos<D, N>(U, spm, nu));
        const ghm::Mat<N, double> B = ghm::mm(ld_aos<D, N>(U, s, nu), ld_aos<D, N>(U, spn, mu));
        v += ghm::retr_nd(A, B);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __shared__ double red[NA_BLOCK / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < NA_BLOCK / 32; ++q) t += red[q];
    partials[blockIdx.x] = t;
  }
}

// out[0] = sum Re Tr U_pl, out[1] = average plaquette (1/N) Re Tr U_pl.
__global__ void k_plaq_total(const double* partials, int nblocks, double nplaq_times_N, double* out) {
  __shared__ double sh[256];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += 256) v += partials[b];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) { out[0] = sh[0]; out[1] = sh[0] / nplaq_times_N; }
}

std::mutex g_mu;
double* g_scratch_ptr[64] = {};
thread_local std::string g_na_err;

int na_fail(int code, const std::string& m) { g_na_err = m; return code; }

}  // namespace

extern "C" {

const char* gh_noalloc_last_error(void) { return g_na_err.c_str(); }

int gh_plaquette_noalloc(int D, int N, const int* L, const double* U_dev, double* out_dev, void* stream) {
  if (D < 2 || D > 4 || N < 2 || N > 3) return na_fail(GH_ERR_UNSUPPORTED, "D must be 2..4 and N 2..3");
  if (!L || !U_dev || !out_dev) return na_fail(GH_ERR_ARG, "null argument");
  // the links are read as 16-byte complex pairs and the outputs written as doubles: a
  // misaligned pointer would raise a sticky misaligned-address error that ends the
  // caller's CUDA context, so it is refused here instead
  if ((reinterpret_cast<uintptr_t>(U_dev) & 15u) != 0)
    return na_fail(GH_ERR_ARG, "U_dev must be 16-byte aligned (complex FP64 pairs)");
  if ((reinterpret_cast<uintptr_t>(out_dev) & 7u) != 0) return na_fail(GH_ERR_ARG, "out_dev must be 8-byte aligned");
  Geo g{};
  long long V = 1;
  for (int mu = 0; mu < 4; ++mu) { g.L[mu] = 1; g.stride[mu] = 0; }
  for (int mu = 0; mu < D; ++mu) {
    if (L[mu] < 1) return na_fail(GH_ERR_ARG, "lattice extents must be >= 1");
    // compared before multiplying, so that no product of extents can overflow
    if (V > GH_NOALLOC_MAX_SITES / L[mu])
      return na_fail(GH_ERR_ARG, "lattice has more sites than gh_plaquette_noalloc handles: at most " +
                                     std::to_string(GH_NOALLOC_MAX_SITES) + " (its fixed scratch array)");
    g.L[mu] = L[mu]; g.stride[mu] = (int)V; V *= L[mu];
  }
  g.V = (int)V;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { cudaGetLastError(); return na_fail(GH_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e)); }
  if (dev < 0 || dev >= 64) return na_fail(GH_ERR_UNSUPPORTED, "device index >= 64");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      // the array's name is a host-side stand-in: its device address comes from
      // the runtime, once per device, with that device current
      e = cudaGetSymbolAddress((void**)&g_scratch_ptr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        cudaGetLastError();
        return na_fail(GH_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (g.V + NA_BLOCK - 1) / NA_BLOCK;
  switch (D * 10 + N) {
    case 22: k_plaq_partials<2, 2><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
    case 32: k_plaq_partials<3, 2><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
    case 42: k_plaq_partials<4, 2><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
    case 23: k_plaq_partials<2, 3><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
    case 33: k_plaq_partials<3, 3><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
    default: k_plaq_partials<4, 3><<<nb, NA_BLOCK, 0, st>>>(g, U_dev, scratch); break;
  }
  const double nplaq = (double)V * (D * (D - 1) / 2);
  k_plaq_total<<<1, 256, 0, st>>>(scratch, nb, nplaq * N, out_dev);
  e = cudaPeekAtLastError();
  if (e != cudaSuccess) { cudaGetLastError(); return na_fail(GH_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e)); }
  return GH_OK;
}

}  // extern "C"
