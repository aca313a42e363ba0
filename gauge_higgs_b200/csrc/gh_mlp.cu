// gh_mlp.cu -- the coupling-scan surrogate: an ensemble of small MLPs trained and
// evaluated by the kernels below (no library GEMMs).
//
// Network (per member): n_in -> H -> ... -> H -> n_out, SiLU between layers,
// FP32 weights and optimiser state, BF16 storage of hidden activations (the
// pre-activations z are kept in FP32 for the SiLU derivative), FP32 accumulation.
// Loss: mean squared error over the batch and the outputs.  Optimiser: Adam with
// bias correction.  All members train on the same minibatches from their own
// initialisation; prediction returns the ensemble mean and variance.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "gh_rng.cuh"
#include "../../include/gauge_higgs_b200.h"

namespace {

constexpr int MAXL = 8;      // layers (weight matrices)
constexpr int BT = 16;       // batch rows per block in the dense kernels

struct Net {
  int M = 0, nl = 0;
  int width[MAXL + 1] = {};
  long woff[MAXL] = {}, boff[MAXL] = {};
  long P = 0;                 // parameters per member
  float* p = nullptr;         // [M][P]
  float* g = nullptr;         // [M][P] gradients
  float* m1 = nullptr;        // Adam first moment
  float* m2 = nullptr;        // Adam second moment
  long t = 0;                 // Adam step
  int cap = 0;                // batch capacity of the activation buffers
  float* x = nullptr;         // [cap][n_in] input
  float* y = nullptr;         // [cap][n_out] target
  float* z[MAXL] = {};        // [M][cap][width[l+1]] pre-activations (FP32)
  __nv_bfloat16* a[MAXL] = {};  // [M][cap][width[l+1]] activations (BF16), last layer unused
  float* out = nullptr;       // [M][cap][n_out]
  float* gz = nullptr;        // [M][cap][maxw] gradient w.r.t. pre-activations
  float* loss = nullptr;      // [M]
  int maxw = 0;
  std::string err;
};

thread_local std::string g_mlp_err;
int mfail(Net* n, int code, const std::string& m) { if (n) n->err = m; g_mlp_err = m; return code; }

__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) { const float s = 1.f / (1.f + __expf(-z)); return s * (1.f + z * (1.f - s)); }

// z[b][j] = sum_i W[j][i] in[b][i] + bias[j]; act: 1 -> a = silu(z) as BF16
// grid (members, ceil(B/BT)), block = out width (rounded to 32).
__global__ void k_dense_fwd(const float* __restrict__ P, long P_stride, long woff, long boff, int nin, int nout,
                            const float* __restrict__ in_f32, long in_mstride, const __nv_bfloat16* __restrict__ in_bf16,
                            int B, float* z, __nv_bfloat16* a, long out_mstride, int act) {
  extern __shared__ float s_in[];   // [BT][nin]
  const int m = blockIdx.x, b0 = blockIdx.y * BT, j = threadIdx.x;
  const float* W = P + m * P_stride + woff;
  const float* bias = P + m * P_stride + boff;
  for (int e = threadIdx.x; e < BT * nin; e += blockDim.x) {
    const int bb = e / nin, i = e % nin, b = b0 + bb;
    float v = 0.f;
    if (b < B) v = in_f32 ? in_f32[(long)b * nin + i] : __bfloat162float(in_bf16[m * in_mstride + (long)b * nin + i]);
    s_in[e] = v;
  }
  __syncthreads();
  if (j >= nout) return;
  float acc[BT];
#pragma unroll
  for (int bb = 0; bb < BT; ++bb) acc[bb] = bias[j];
  for (int i = 0; i < nin; ++i) {
    const float w = W[(long)j * nin + i];
#pragma unroll
    for (int bb = 0; bb < BT; ++bb) acc[bb] = fmaf(w, s_in[bb * nin + i], acc[bb]);
  }
#pragma unroll
  for (int bb = 0; bb < BT; ++bb) {
    const int b = b0 + bb;
    if (b >= B) break;
    const long o = m * out_mstride + (long)b * nout + j;
    z[o] = acc[bb];
    if (act) a[o] = __float2bfloat16(silu(acc[bb]));
  }
}

// loss and output gradient: gz = 2 (out - y) / (B n_out), loss[m] = mean (out - y)^2
__global__ void k_mse(const float* out, long mstride, const float* y, int B, int nout, float* gz, long gstride, float* loss) {
  const int m = blockIdx.x;
  float s = 0.f;
  for (int e = threadIdx.x; e < B * nout; e += blockDim.x) {
    const float d = out[m * mstride + e] - y[e];
    s += d * d;
    gz[m * gstride + e] = 2.f * d / (float)(B * nout);
  }
  __shared__ float sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[m] = sh[0] / (float)(B * nout);
}

// weight / bias gradients: dW[j][i] = sum_b gz[b][j] in[b][i], db[j] = sum_b gz[b][j]
// grid (members, nout), block over i.
__global__ void k_dense_wgrad(const float* gz, long gstride, int nout, const float* in_f32, const __nv_bfloat16* in_bf16,
                              long in_mstride, int nin, int B, float* G, long P_stride, long woff, long boff) {
  const int m = blockIdx.x, j = blockIdx.y;
  float* dW = G + m * P_stride + woff;
  float* db = G + m * P_stride + boff;
  for (int i = threadIdx.x; i <= nin; i += blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < B; ++b) {
      const float gv = gz[m * gstride + (long)b * nout + j];
      const float xv = (i == nin) ? 1.f
                       : in_f32 ? in_f32[(long)b * nin + i] : __bfloat162float(in_bf16[m * in_mstride + (long)b * nin + i]);
      s = fmaf(gv, xv, s);
    }
    if (i == nin) db[j] = s; else dW[(long)j * nin + i] = s;
  }
}

// input gradient through the previous SiLU: gz_prev[b][i] = (sum_j W[j][i] gz[b][j]) silu'(z_prev[b][i])
// grid (members, ceil(B/BT)), block over i.
__global__ void k_dense_bgrad(const float* __restrict__ P, long P_stride, long woff, int nin, int nout, const float* gz,
                              long gstride, const float* zprev, long zstride, int B, float* gzprev, long gpstride) {
  const int m = blockIdx.x, b0 = blockIdx.y * BT, i = threadIdx.x;
  if (i >= nin) return;
  const float* W = P + m * P_stride + woff;
  for (int bb = 0; bb < BT; ++bb) {
    const int b = b0 + bb;
    if (b >= B) break;
    float s = 0.f;
    for (int j = 0; j < nout; ++j) s = fmaf(W[(long)j * nin + i], gz[m * gstride + (long)b * nout + j], s);
    gzprev[m * gpstride + (long)b * nin + i] = s * dsilu(zprev[m * zstride + (long)b * nin + i]);
  }
}

__global__ void k_adam(float* p, const float* g, float* m1, float* m2, long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const float gv = g[e];
    const float a = b1 * m1[e] + (1.f - b1) * gv;
    const float v = b2 * m2[e] + (1.f - b2) * gv * gv;
    m1[e] = a;
    m2[e] = v;
    p[e] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
  }
}

int ensure_cap(Net* n, int B) {
  if (B <= n->cap) return GH_OK;
  auto fr = [](void* q) { if (q) cudaFree(q); };
  fr(n->x); fr(n->y); fr(n->out); fr(n->gz);
  for (int l = 0; l < n->nl; ++l) { fr(n->z[l]); fr(n->a[l]); }
  const int cap = std::max(B, 256);
  cudaError_t e = cudaSuccess;
  e = e ? e : cudaMalloc(&n->x, sizeof(float) * cap * n->width[0]);
  e = e ? e : cudaMalloc(&n->y, sizeof(float) * cap * n->width[n->nl]);
  e = e ? e : cudaMalloc(&n->out, sizeof(float) * n->M * cap * n->width[n->nl]);
  e = e ? e : cudaMalloc(&n->gz, sizeof(float) * n->M * cap * n->maxw * 2);
  for (int l = 0; l < n->nl && !e; ++l) {
    e = cudaMalloc(&n->z[l], sizeof(float) * n->M * cap * n->width[l + 1]);
    if (!e) e = cudaMalloc(&n->a[l], sizeof(__nv_bfloat16) * n->M * cap * n->width[l + 1]);
  }
  if (e) { cudaGetLastError(); return mfail(n, GH_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
  n->cap = cap;
  return GH_OK;
}

void forward(Net* n, int B) {
  for (int l = 0; l < n->nl; ++l) {
    const int nin = n->width[l], nout = n->width[l + 1];
    const int threads = ((std::max(nout, nin) + 31) / 32) * 32;
    dim3 grid(n->M, (B + BT - 1) / BT);
    const bool last = (l == n->nl - 1);
    float* zo = last ? n->out : n->z[l];
    // layer 0 reads the shared FP32 input; layer l > 0 the BF16 activations a[l-1] (member stride cap*nin)
    k_dense_fwd<<<grid, threads, sizeof(float) * BT * nin>>>(
        n->p, n->P, n->woff[l], n->boff[l], nin, nout, l == 0 ? n->x : nullptr, (long)n->cap * nin,
        l == 0 ? nullptr : n->a[l - 1], B, zo, n->a[l], (long)n->cap * nout, last ? 0 : 1);
  }
}

}  // namespace

struct gh_mlp : Net {};

extern "C" {

const char* gh_mlp_last_error(void) { return g_mlp_err.c_str(); }

int gh_mlp_create(int n_members, const int* widths, int n_layers, uint64_t seed, gh_mlp** out) {
  if (!out || !widths || n_members < 1 || n_layers < 1 || n_layers > MAXL) return mfail(nullptr, GH_ERR_ARG, "bad MLP shape");
  for (int l = 0; l <= n_layers; ++l)
    if (widths[l] < 1 || widths[l] > 1024) return mfail(nullptr, GH_ERR_ARG, "layer widths must be 1..1024");
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) { cudaGetLastError(); return mfail(nullptr, GH_ERR_CUDA, "no CUDA device"); }
  gh_mlp* n = new gh_mlp();
  n->M = n_members;
  n->nl = n_layers;
  long off = 0;
  for (int l = 0; l <= n_layers; ++l) { n->width[l] = widths[l]; n->maxw = std::max(n->maxw, widths[l]); }
  for (int l = 0; l < n_layers; ++l) {
    n->woff[l] = off; off += (long)widths[l + 1] * widths[l];
    n->boff[l] = off; off += widths[l + 1];
  }
  n->P = off;
  const long tot = n->P * n->M;
  // initialisation: W ~ U(-1/sqrt(fan_in), 1/sqrt(fan_in)), b = 0, from the project's counter RNG
  std::vector<float> h(tot, 0.f);
  for (int m = 0; m < n->M; ++m)
    for (int l = 0; l < n_layers; ++l) {
      const float a = 1.f / std::sqrt((float)widths[l]);
      for (long e = 0; e < (long)widths[l + 1] * widths[l]; ++e)
        h[m * n->P + n->woff[l] + e] = a * (float)(2.0 * ghrng::uniform(seed, ghrng::key(0x4D4C50, m, l, e)) - 1.0);
    }
  cudaError_t e = cudaSuccess;
  e = e ? e : cudaMalloc(&n->p, sizeof(float) * tot);
  e = e ? e : cudaMalloc(&n->g, sizeof(float) * tot);
  e = e ? e : cudaMalloc(&n->m1, sizeof(float) * tot);
  e = e ? e : cudaMalloc(&n->m2, sizeof(float) * tot);
  e = e ? e : cudaMalloc(&n->loss, sizeof(float) * n->M);
  if (!e) e = cudaMemcpy(n->p, h.data(), sizeof(float) * tot, cudaMemcpyHostToDevice);
  if (!e) e = cudaMemset(n->m1, 0, sizeof(float) * tot);
  if (!e) e = cudaMemset(n->m2, 0, sizeof(float) * tot);
  if (e) { cudaGetLastError(); delete n; return mfail(nullptr, GH_ERR_CUDA, std::string("MLP allocation: ") + cudaGetErrorString(e)); }
  if (ensure_cap(n, 256)) { delete n; return GH_ERR_CUDA; }
  *out = n;
  return GH_OK;
}

int gh_mlp_destroy(gh_mlp* n) {
  if (!n) return GH_OK;
  cudaDeviceSynchronize();
  void* ps[] = {n->p, n->g, n->m1, n->m2, n->loss, n->x, n->y, n->out, n->gz};
  for (void* q : ps) if (q) cudaFree(q);
  for (int l = 0; l < n->nl; ++l) { if (n->z[l]) cudaFree(n->z[l]); if (n->a[l]) cudaFree(n->a[l]); }
  delete n;
  return GH_OK;
}

int gh_mlp_num_params(const gh_mlp* n, long* per_member) {
  if (!n || !per_member) return mfail(nullptr, GH_ERR_ARG, "null argument");
  *per_member = n->P;
  return GH_OK;
}

int gh_mlp_get_params(gh_mlp* n, float* params) {
  if (!n || !params) return mfail(nullptr, GH_ERR_ARG, "null argument");
  if (cudaMemcpy(params, n->p, sizeof(float) * n->P * n->M, cudaMemcpyDeviceToHost)) return mfail(n, GH_ERR_CUDA, "copy");
  return GH_OK;
}

int gh_mlp_set_params(gh_mlp* n, const float* params) {
  if (!n || !params) return mfail(nullptr, GH_ERR_ARG, "null argument");
  if (cudaMemcpy(n->p, params, sizeof(float) * n->P * n->M, cudaMemcpyHostToDevice)) return mfail(n, GH_ERR_CUDA, "copy");
  return GH_OK;
}

// forward + loss + backward on one batch; gradients stay on the device (and are
// copied to grads if non-null: [M][P]); loss: [M].
static int grad_batch(gh_mlp* n, const float* xh, const float* yh, int B, float* grads, float* loss) {
  int rc = ensure_cap(n, B);
  if (rc) return rc;
  const int nin = n->width[0], nout = n->width[n->nl];
  if (cudaMemcpy(n->x, xh, sizeof(float) * B * nin, cudaMemcpyHostToDevice) ||
      cudaMemcpy(n->y, yh, sizeof(float) * B * nout, cudaMemcpyHostToDevice))
    return mfail(n, GH_ERR_CUDA, "copy");
  forward(n, B);
  const long gstride = (long)n->cap * n->maxw;
  float* gcur = n->gz;
  float* gprev = n->gz + (long)n->M * n->cap * n->maxw;
  k_mse<<<n->M, 256>>>(n->out, (long)n->cap * nout, n->y, B, nout, gcur, gstride, n->loss);
  for (int l = n->nl - 1; l >= 0; --l) {
    const int lin = n->width[l], lout = n->width[l + 1];
    dim3 gw(n->M, lout);
    k_dense_wgrad<<<gw, 128>>>(gcur, gstride, lout, l == 0 ? n->x : nullptr, l == 0 ? nullptr : n->a[l - 1],
                               (long)n->cap * lin, lin, B, n->g, n->P, n->woff[l], n->boff[l]);
    if (l > 0) {
      dim3 gb(n->M, (B + BT - 1) / BT);
      const int threads = ((lin + 31) / 32) * 32;
      k_dense_bgrad<<<gb, threads>>>(n->p, n->P, n->woff[l], lin, lout, gcur, gstride, n->z[l - 1], (long)n->cap * lin, B,
                                     gprev, gstride);
      std::swap(gcur, gprev);
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e) return mfail(n, GH_ERR_CUDA, std::string("MLP kernels: ") + cudaGetErrorString(e));
  if (grads && cudaMemcpy(grads, n->g, sizeof(float) * n->P * n->M, cudaMemcpyDeviceToHost)) return mfail(n, GH_ERR_CUDA, "copy");
  if (loss && cudaMemcpy(loss, n->loss, sizeof(float) * n->M, cudaMemcpyDeviceToHost)) return mfail(n, GH_ERR_CUDA, "copy");
  return GH_OK;
}

int gh_mlp_grad(gh_mlp* n, const float* x, const float* y, int B, float* grads, float* loss) {
  if (!n || !x || !y || B < 1) return mfail(n, GH_ERR_ARG, "bad arguments");
  return grad_batch(n, x, y, B, grads, loss);
}

int gh_mlp_adam_step(gh_mlp* n, float lr) {
  if (!n) return mfail(nullptr, GH_ERR_ARG, "null network");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  n->t += 1;
  const float c1 = 1.f - std::pow(b1, (float)n->t), c2 = 1.f - std::pow(b2, (float)n->t);
  k_adam<<<296, 256>>>(n->p, n->g, n->m1, n->m2, n->P * n->M, lr, b1, b2, eps, c1, c2);
  cudaError_t e = cudaGetLastError();
  if (e) return mfail(n, GH_ERR_CUDA, std::string("adam: ") + cudaGetErrorString(e));
  return GH_OK;
}

// epochs over (x, y) in shuffled minibatches of `batch`; loss: mean loss of the last epoch per member
int gh_mlp_train(gh_mlp* n, const float* x, const float* y, int n_samples, int epochs, int batch, float lr, uint64_t seed,
                 float* loss) {
  if (!n || !x || !y || n_samples < 1 || epochs < 1 || batch < 1) return mfail(n, GH_ERR_ARG, "bad arguments");
  const int nin = n->width[0], nout = n->width[n->nl];
  std::vector<int> idx(n_samples);
  std::vector<float> xb((size_t)batch * nin), yb((size_t)batch * nout), lb(n->M), lsum(n->M);
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = 0; i < n_samples; ++i) idx[i] = i;
    for (int i = n_samples - 1; i > 0; --i) {   // Fisher-Yates with the counter RNG
      const int j = (int)(ghrng::uniform(seed, ghrng::key(0x5348, ep, i)) * (i + 1));
      std::swap(idx[i], idx[std::min(j, i)]);
    }
    std::fill(lsum.begin(), lsum.end(), 0.f);
    int nb = 0;
    for (int s0 = 0; s0 < n_samples; s0 += batch, ++nb) {
      const int B = std::min(batch, n_samples - s0);
      for (int b = 0; b < B; ++b) {
        std::memcpy(&xb[(size_t)b * nin], x + (size_t)idx[s0 + b] * nin, sizeof(float) * nin);
        std::memcpy(&yb[(size_t)b * nout], y + (size_t)idx[s0 + b] * nout, sizeof(float) * nout);
      }
      int rc = grad_batch(n, xb.data(), yb.data(), B, nullptr, ep == epochs - 1 ? lb.data() : nullptr);
      if (rc) return rc;
      if ((rc = gh_mlp_adam_step(n, lr))) return rc;
      if (ep == epochs - 1) for (int m = 0; m < n->M; ++m) lsum[m] += lb[m];
    }
    if (ep == epochs - 1 && loss) for (int m = 0; m < n->M; ++m) loss[m] = lsum[m] / nb;
  }
  if (cudaDeviceSynchronize()) return mfail(n, GH_ERR_CUDA, "train sync");
  return GH_OK;
}

// predictions of every member: out [M][n][n_out] (may be null), and the ensemble
// mean / variance [n][n_out] (population variance over members)
int gh_mlp_predict(gh_mlp* n, const float* x, int B, float* per_member, float* mean, float* var) {
  if (!n || !x || B < 1) return mfail(n, GH_ERR_ARG, "bad arguments");
  int rc = ensure_cap(n, B);
  if (rc) return rc;
  const int nin = n->width[0], nout = n->width[n->nl];
  if (cudaMemcpy(n->x, x, sizeof(float) * B * nin, cudaMemcpyHostToDevice)) return mfail(n, GH_ERR_CUDA, "copy");
  forward(n, B);
  std::vector<float> o((size_t)n->M * n->cap * nout);
  if (cudaMemcpy(o.data(), n->out, sizeof(float) * o.size(), cudaMemcpyDeviceToHost)) return mfail(n, GH_ERR_CUDA, "copy");
  for (int b = 0; b < B; ++b)
    for (int k = 0; k < nout; ++k) {
      double s = 0.0, s2 = 0.0;
      for (int m = 0; m < n->M; ++m) {
        const double v = o[(size_t)m * n->cap * nout + (size_t)b * nout + k];
        if (per_member) per_member[((size_t)m * B + b) * nout + k] = (float)v;
        s += v;
        s2 += v * v;
      }
      if (mean) mean[(size_t)b * nout + k] = (float)(s / n->M);
      if (var) var[(size_t)b * nout + k] = (float)std::max(0.0, s2 / n->M - (s / n->M) * (s / n->M));
    }
  return GH_OK;
}

}  // extern "C"
