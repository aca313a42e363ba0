// gh_ctx.cu -- context, device memory, trajectory graph and the C ABI of
// include/gauge_higgs_b200.h.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include "gh_engine.cuh"
#include "gh_potential.h"
#include "gh_sympow.h"
#include "gh_adjprod.h"
#include "../../include/gauge_higgs_b200.h"

using namespace ghk;

namespace {
thread_local std::string g_err;
}
namespace ghpot {
void set_host_error(const std::string& m) { g_err = m; }
}

struct gh_ctx {
  int D = 0, N = 0, ng = 0, nlat = 0, prec = 0, rep = 0, d = 0, real = 0, scalar = 0;
  size_t rs = 8;                      // bytes per real of the field storage
  std::vector<LatDev> lat_h;          // host copy (extents, offsets; counters live on the device)
  long long nU = 0, nP = 0, nF = 0, nG = 0;   // total complex / real / complex / complex elements
  Bufs b{};
  std::unique_ptr<EngineBase> eng;
  cudaStream_t own = nullptr, st = nullptr;
  int integ = 1, nmd = 20;
  double tau = 1.0;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  int use_graph = 1;
  double* staging = nullptr;
  size_t staging_elems = 0;
  double* fbuf = nullptr;             // FP64 SoA force output (links)
  double* fphibuf = nullptr;          // FP64 SoA force output (vectors)
  std::vector<void*> allocs;
  std::string err;
  uint64_t bytes = 0;
  // tempering
  int temper = 0;
  int temper_every = 1;
  uint64_t swap_seed = 0;
  int* t_order = nullptr;             // [nlat] lattice currently holding the k-th kappa (grouped)
  int* t_groups = nullptr;            // [ngroups+1] group boundaries into t_order
  int t_ngroups = 0;
  unsigned long long* t_stats = nullptr;   // [2*nlat + 1] attempts, accepts, counter
  int* t_pairmap = nullptr;
  // tiled kick work table (rebuilt when tile shapes change)
  Work* wk_dev = nullptr;
  size_t wk_cap = 0;
  // general irreps: host copy of the generators T^a_R (multi-invariant potential set-up)
  std::vector<double> T_host;
  // general irreps: closed-form D(U) term lists (single-row irreps, when cheaper than
  // the tensor path or when the tensor buffer does not fit in shared memory)
  ghsym::Terms sp;
  bool use_sp = false;
  // general irreps inside the adjoint product (gh_adjprod.h): the intertwiner Q, and
  // whether the link kernel goes that way (gh_set_rep_path switches it)
  ghadj::Product prod;
  bool has_prod = false;
  // two-slot irreps (n = 2) outside the adjoint product: the register path (k_gen_pair)
  bool has_pair = false;
  size_t gen_warp_bytes = 0, gen_px_off = 0;
  // multi-invariant potential: device copies of the channel superoperator (sparse rows)
  int* sa_ptr = nullptr;
  unsigned short* sa_ij = nullptr;
  double2* sa_v64 = nullptr;
  float2* sa_v32 = nullptr;
  void free_potential() {
    if (sa_ptr) cudaFree(sa_ptr);
    if (sa_ij) cudaFree(sa_ij);
    if (sa_v64) cudaFree(sa_v64);
    if (sa_v32) cudaFree(sa_v32);
    sa_ptr = nullptr; sa_ij = nullptr; sa_v64 = nullptr; sa_v32 = nullptr;
  }
  ~gh_ctx() {
    if (st) cudaStreamSynchronize(st);
    if (wk_dev) cudaFree(wk_dev);
    free_potential();
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : allocs) cudaFree(p);
    if (own) cudaStreamDestroy(own);
  }
};

namespace {

int fail(gh_ctx* c, int code, const std::string& m) {
  if (c) c->err = m; else g_err = m;
  return code;
}
// Copies and fills outside the trajectory run on the context's stream (cudaMemcpyAsync /
// cudaMemsetAsync, a synchronise after every read back): that stream is non-blocking, so
// a plain cudaMemcpy on the legacy default stream is not ordered with its kernels, and
// one from pageable memory may return before its transfer has landed.
#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(ctx, GH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
int dalloc(gh_ctx* ctx, T** p, size_t n) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return fail(ctx, GH_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemsetAsync(q, 0, bytes, ctx->st);
  ctx->allocs.push_back(q);
  ctx->bytes += bytes;
  *p = (T*)q;
  return GH_OK;
}

int launch_check(gh_ctx* ctx, const char* what) {
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, GH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)); }
  return GH_OK;
}

void invalidate_graph(gh_ctx* ctx) {
  if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
}

// ---- integrator building blocks (enqueue only) ----
void enq_kick(gh_ctx* ctx, double eps) {
  if (ctx->rep == REP_GEN) ctx->eng->gen_links(ctx->b, eps, 0, nullptr);
  ctx->eng->kick(ctx->b, eps, M_UPDATE, F_GAUGE | F_MATTER, nullptr, true, true);
  if (ctx->b.frozen) ctx->eng->sphere(ctx->b, 0);   // drop the radial force (src/hmc/gauge_higgs_hmc.hpp:133)
}
void enq_drift(gh_ctx* ctx, double eps) {
  ctx->eng->drift(ctx->b, eps, ctx->prec == GH_PREC_FP32_MD ? 1 : ctx->prec == GH_PREC_FP32_ALL ? 2 : 0);
}

// md_evolve: src/hmc/gauge_higgs_hmc.hpp:149-165 (identical in src/hmc/hmc.hpp:54-70)
void enq_md(gh_ctx* ctx) {
  const double eps = ctx->tau / ctx->nmd;
  if (ctx->integ == GH_LEAPFROG) {
    enq_kick(ctx, 0.5 * eps);
    for (int i = 0; i < ctx->nmd; ++i) { enq_drift(ctx, eps); if (i != ctx->nmd - 1) enq_kick(ctx, eps); }
    enq_kick(ctx, 0.5 * eps);
  } else {
    const double lam = 0.1931833275037836;   // src/core/config.hpp:25
    enq_kick(ctx, lam * eps);
    for (int i = 0; i < ctx->nmd; ++i) {
      enq_drift(ctx, 0.5 * eps);
      enq_kick(ctx, (1.0 - 2.0 * lam) * eps);
      enq_drift(ctx, 0.5 * eps);
      enq_kick(ctx, (i != ctx->nmd - 1 ? 2.0 * lam : lam) * eps);
    }
  }
}

void enq_measure(gh_ctx* ctx, int slot) {
  ctx->eng->measure(ctx->b);
  FinArgs f;
  f.lats = ctx->b.lats; f.blk_first = ctx->b.blk_first; f.partials = ctx->b.partials; f.res = ctx->b.res;
  f.slot = slot; f.D = ctx->D; f.N = ctx->N; f.scalar = ctx->scalar;
  launch(k_finalize, ctx->nlat, 32, 0, ctx->st, f);
}

// Replica-tempering pass in kappa (src/hmc/replica_tempering.hpp:157-205 mechanism).
// coupling 1: kappa (B = 2 V D L_link, the hopping term S_H = ... - kappa B);
// coupling 2: beta  (B = P = n_plaq (plaquette - 1), S_g = -beta P + const,
//                    src/hmc/replica_tempering.hpp:16-42).  Both: Delta = (c_i - c_j)(B_i - B_j).
struct TemperArgs {
  LatDev* lats; const double* res; int* order; const int* groups; int ngroups; int D;
  unsigned long long* stats; const int* pairmap; int nlat; unsigned long long seed; int coupling;
  int every;   // one swap pass after every `every` trajectories (ReplicaTempering::n_sweep)
};
__global__ void k_temper(const TemperArgs a) {
  pdl_enter();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (a.every > 1 && a.lats[0].traj % (unsigned long long)a.every != 0) return;
  unsigned long long& counter = a.stats[2 * a.nlat];
  for (int g = 0; g < a.ngroups; ++g) {
    const int b0 = a.groups[g], b1 = a.groups[g + 1];
    for (int start = 0; start < 2; ++start)
      for (int k = b0 + start; k + 1 < b1; k += 2) {
        const int li = a.order[k], lj = a.order[k + 1];
        LatDev& Li = a.lats[li];
        LatDev& Lj = a.lats[lj];
        const double* ri = a.res + ((size_t)li * 2 + (Li.last_acc ? 1 : 0)) * NRES;
        const double* rj = a.res + ((size_t)lj * 2 + (Lj.last_acc ? 1 : 0)) * NRES;
        const bool beta = a.coupling == 2;
        const double nplaq_i = (double)Li.V * (a.D * (a.D - 1) / 2), nplaq_j = (double)Lj.V * (a.D * (a.D - 1) / 2);
        const double Bi = beta ? nplaq_i * (ri[5] - 1.0) : 2.0 * ri[6] * (double)Li.V * a.D;
        const double Bj = beta ? nplaq_j * (rj[5] - 1.0) : 2.0 * rj[6] * (double)Lj.V * a.D;
        const double delta = beta ? (Li.beta - Lj.beta) * (Bi - Bj) : (Li.kappa - Lj.kappa) * (Bi - Bj);
        const int pid = a.pairmap[k];
        a.stats[pid] += 1;
        bool acc = (delta <= 0.0);
        counter += 1;
        if (!acc) acc = ghrng::uniform(a.seed, ghrng::key(0x57A9, counter)) < exp(-delta);
        if (acc && beta) {
          const double tb = Li.beta; Li.beta = Lj.beta; Lj.beta = tb;
        }
        if (acc && !beta) {
          const double tk = Li.kappa; Li.kappa = Lj.kappa; Lj.kappa = tk;
        }
        if (acc) {
          const int tc = Li.cidx; Li.cidx = Lj.cidx; Lj.cidx = tc;
          a.order[k] = lj; a.order[k + 1] = li;
          a.stats[a.nlat + pid] += 1;
        }
      }
  }
}

void enq_trajectory(gh_ctx* ctx) {
  Bufs& b = ctx->b;
  InitArgs ia{};
  ia.what = 1; ia.pure = ctx->scalar ? 0 : 1; ia.real = ctx->real; ia.d = ctx->d; ia.vec = b.pi;
  ctx->eng->init(b, ia, true, ctx->scalar != 0);
  if (b.frozen) ctx->eng->sphere(b, 0);   // tangent-space momenta (src/hmc/gauge_higgs_hmc.hpp:172)
  cudaMemcpyAsync(b.Us, b.U, (size_t)ctx->nU * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st);
  if (ctx->scalar) cudaMemcpyAsync(b.phis, b.phi, (size_t)ctx->nF * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st);
  enq_measure(ctx, 0);
  enq_md(ctx);
  if (ctx->prec == GH_PREC_FP64) ctx->eng->reunit(b);
  enq_measure(ctx, 1);
  MetroArgs m;
  m.lats = b.lats; m.res = b.res; m.hist = b.hist; m.hist_cap = b.hist_cap; m.nlat = ctx->nlat; m.pure = ctx->scalar ? 0 : 1;
  launch(k_metropolis, (ctx->nlat + 63) / 64, 64, 0, ctx->st, m);
  ctx->eng->restore(b);
  if (ctx->temper && (ctx->scalar || ctx->temper == 2)) {
    TemperArgs t;
    t.lats = b.lats; t.res = b.res; t.order = ctx->t_order; t.groups = ctx->t_groups; t.ngroups = ctx->t_ngroups;
    t.D = ctx->D; t.stats = ctx->t_stats; t.pairmap = ctx->t_pairmap; t.nlat = ctx->nlat; t.seed = ctx->swap_seed; t.coupling = ctx->temper; t.every = ctx->temper_every;
    launch(k_temper, 1, 32, 0, ctx->st, t);
  }
}

bool any_decomposed(const gh_ctx* ctx) {
  for (const LatDev& L : ctx->lat_h)
    if (L.dec) return true;
  return false;
}

int run_traj(gh_ctx* ctx) {
  if (any_decomposed(ctx))
    return fail(ctx, GH_ERR_STATE, "a subdomain of a decomposed lattice: its trajectory is driven by the domain "
                                   "layer (global dH and accept), not by the device Metropolis");
  if (ctx->use_graph) {
    if (!ctx->gexec) {
      CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
      enq_trajectory(ctx);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(ctx->st, &g);
      if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, GH_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)); }
      ctx->graph = g;
      CK(cudaGraphInstantiate(&ctx->gexec, g, 0));
    }
    CK(cudaGraphLaunch(ctx->gexec, ctx->st));
  } else {
    enq_trajectory(ctx);
  }
  return launch_check(ctx, "trajectory");
}

int check_lat(gh_ctx* ctx, int lat, bool allow_all) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (lat == -1 && allow_all) return GH_OK;
  if (lat < 0 || lat >= ctx->nlat) return fail(ctx, GH_ERR_ARG, "lattice index out of range");
  return GH_OK;
}

// AoS host <-> SoA device for one lattice. kind 0 links, 1 momenta, 2 vectors.
int xfer_one(gh_ctx* ctx, int lat, int kind, void* dev, double* host, bool to_dev, bool dev_is_fp64 = false) {
  const LatDev& L = ctx->lat_h[lat];
  const int ncomp = kind == 0 ? ctx->N * ctx->N : kind == 1 ? ctx->ng : ctx->d;
  const size_t nd = (size_t)L.V * (kind == 2 ? ncomp : ctx->D * ncomp) * (kind == 1 ? 1 : 2);
  if (to_dev) CK(cudaMemcpyAsync(ctx->staging, host, nd * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  XferArgs a;
  a.lat = lat; a.kind = kind; a.D = ctx->D; a.ncomp = ncomp; a.host_aos = ctx->staging; a.dev = dev; a.to_dev = to_dev ? 1 : 0;
  if (dev_is_fp64) {
    a.lats = ctx->b.lats;
    k_xfer<double><<<296, 256, 0, ctx->st>>>(a);
  } else {
    ctx->eng->xfer(ctx->b, a);
  }
  int rc = launch_check(ctx, "xfer");
  if (rc) return rc;
  if (!to_dev) {
    CK(cudaMemcpyAsync(host, ctx->staging, nd * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  return GH_OK;
}

size_t lat_elems(const gh_ctx* ctx, int lat, int kind) {
  const LatDev& L = ctx->lat_h[lat];
  return (size_t)L.V * (kind == 0 ? ctx->D * ctx->N * ctx->N * 2 : kind == 1 ? ctx->D * ctx->ng : ctx->d * 2);
}

int xfer_field(gh_ctx* ctx, int lat, int kind, void* dev, const double* host, bool to_dev) {
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (kind == 2 && !ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  if (!host) return fail(ctx, GH_ERR_ARG, "null host pointer");
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  size_t off = 0;
  for (int l = l0; l < l1; ++l) {
    rc = xfer_one(ctx, l, kind, dev, const_cast<double*>(host) + off, to_dev);
    if (rc) return rc;
    if (to_dev) { CK(cudaStreamSynchronize(ctx->st)); }
    off += lat_elems(ctx, l, kind);
  }
  return GH_OK;
}

int ceil_log2(int x) { int k = 0; while ((1 << k) < x) ++k; return k; }

// Default kick tile: fill the KICK_LOG2 bits of a kick block direction by direction
// (direction 0 first), never wider than the lattice -- the shape of consecutive sites.
void default_tile(const int* L, int D, int* lt) {
  int left = KICK_LOG2;
  for (int mu = 0; mu < 4; ++mu) lt[mu] = 0;
  for (int mu = 0; mu < D && left > 0; ++mu) { lt[mu] = std::min(left, ceil_log2(L[mu])); left -= lt[mu]; }
}

// Kick items of the lattices in `lats`: link items direction by direction (all
// tiles of direction 0, then direction 1, ...), then one site item per tile.
// Direction-major order keeps the blocks resident at one time on distinct sites.
void kick_items(const gh_ctx* ctx, const std::vector<int>& lats, std::vector<Work>& out, int& nlinks, int& nsites) {
  std::vector<Work> links, sites, links_mu[4];
  const int D = ctx->D;
  for (int l : lats) {
    const LatDev& Ld = ctx->lat_h[l];
    int t[4], nt[4];
    long long ntiles = 1;
    for (int mu = 0; mu < 4; ++mu) { t[mu] = 1 << Ld.lt[mu]; nt[mu] = mu < D ? (Ld.L[mu] + t[mu] - 1) / t[mu] : 1; ntiles *= nt[mu]; }
    for (long long q = 0; q < ntiles; ++q) {
      long long r = q;
      int s0 = 0, packed = 0;
      for (int mu = 0; mu < D; ++mu) {
        const int o = (int)(r % nt[mu]) * t[mu];
        r /= nt[mu];
        s0 += o * Ld.stride[mu];
        packed |= o << (8 * mu);
      }
      for (int mu = 0; mu < D; ++mu) links_mu[mu].push_back(Work{l, mu, s0, packed});
      sites.push_back(Work{l, -1, s0, packed});
    }
  }
  for (int mu = 0; mu < D; ++mu) links.insert(links.end(), links_mu[mu].begin(), links_mu[mu].end());
  nlinks = (int)links.size();
  nsites = (int)sites.size();
  out = links;
  out.insert(out.end(), sites.begin(), sites.end());
}

int upload_kick_items(gh_ctx* ctx, const std::vector<Work>& items, int nlinks, int nsites) {
  if (items.size() > ctx->wk_cap) {
    if (ctx->wk_dev) cudaFree(ctx->wk_dev);
    ctx->wk_dev = nullptr;
    ctx->wk_cap = 0;
    CK(cudaMalloc(&ctx->wk_dev, sizeof(Work) * items.size()));
    ctx->wk_cap = items.size();
  }
  CK(cudaMemcpyAsync(ctx->wk_dev, items.data(), sizeof(Work) * items.size(), cudaMemcpyHostToDevice, ctx->st));
  ctx->b.w_kick = ctx->wk_dev;
  ctx->b.nwk_links = nlinks;
  ctx->b.nwk_sites = nsites;
  return GH_OK;
}

int push_tiles(gh_ctx* ctx) {
  for (int l = 0; l < ctx->nlat; ++l)
    CK(cudaMemcpyAsync((char*)(ctx->b.lats + l) + offsetof(LatDev, lt), ctx->lat_h[l].lt, sizeof(int) * 4, cudaMemcpyHostToDevice, ctx->st));
  return GH_OK;
}

int rebuild_kick_table(gh_ctx* ctx) {
  CK(cudaStreamSynchronize(ctx->st));
  int rc = push_tiles(ctx);
  if (rc) return rc;
  std::vector<int> all(ctx->nlat);
  for (int l = 0; l < ctx->nlat; ++l) all[l] = l;
  std::vector<Work> items;
  int nl, ns;
  kick_items(ctx, all, items, nl, ns);
  invalidate_graph(ctx);
  return upload_kick_items(ctx, items, nl, ns);
}

int build_general(gh_ctx* ctx, const gh_rep_desc* r) {
  const int d = r->d, N = ctx->N, ng = ctx->ng;
  const long dimT = r->dimT;
  if (d <= 0 || r->n_boxes <= 0 || r->n_boxes > 17 || dimT <= 0 || !r->T || !r->W)
    return fail(ctx, GH_ERR_REP, "general representation needs d, n_boxes, dimT, T and W");
  long pw = 1;
  for (int k = 0; k < r->n_boxes; ++k) pw *= N;
  if (pw != dimT) return fail(ctx, GH_ERR_REP, "dimT must equal N^n_boxes");
  if (dimT > 200000) return fail(ctx, GH_ERR_REP, "N^n exceeds the 200000 cap of the reference (src/rep/rep_general.hpp:34)");
  const double* W = r->W;
  const double* T = r->T;
  ctx->T_host.assign(T, T + 2 * (size_t)ng * d * d);
  std::vector<int> wt_ptr(dimT + 1, 0), wt_l, w_ptr(d + 1, 0), w_i, t_ptr(ng * d + 1, 0), t_j;
  std::vector<double2> wt_v, w_v, t_v;
  for (long i = 0; i < dimT; ++i) {
    for (int l = 0; l < d; ++l) {
      const double re = W[2 * ((size_t)l * dimT + i)], im = W[2 * ((size_t)l * dimT + i) + 1];
      if (re != 0.0 || im != 0.0) { wt_l.push_back(l); wt_v.push_back(make_double2(re, im)); }
    }
    wt_ptr[i + 1] = (int)wt_l.size();
  }
  for (int l = 0; l < d; ++l) {
    for (long i = 0; i < dimT; ++i) {
      const double re = W[2 * ((size_t)l * dimT + i)], im = W[2 * ((size_t)l * dimT + i) + 1];
      if (re != 0.0 || im != 0.0) { w_i.push_back((int)i); w_v.push_back(make_double2(re, im)); }
    }
    w_ptr[l + 1] = (int)w_i.size();
  }
  for (int a = 0; a < ng; ++a)
    for (int i = 0; i < d; ++i) {
      for (int j = 0; j < d; ++j) {
        const size_t o = 2 * (((size_t)a * d + i) * d + j);
        if (T[o] != 0.0 || T[o + 1] != 0.0) { t_j.push_back(j); t_v.push_back(make_double2(T[o], T[o + 1])); }
      }
      t_ptr[a * d + i + 1] = (int)t_j.size();
    }
  GenTables& t = ctx->b.gen;
  t.d = d; t.n = r->n_boxes; t.dimT = (int)dimT; t.ng = ng;
  t.powN[0] = 1;
  for (int k = 1; k < 18; ++k) t.powN[k] = (k <= r->n_boxes) ? t.powN[k - 1] * N : 0;
  for (int k = 0; k < 18; ++k)
    t.pmag[k] = (k >= 1 && t.powN[k] > 0) ? (unsigned)(((1ULL << 32) + (unsigned long long)t.powN[k] - 1) / t.powN[k]) : 0u;
  int *p1, *p2, *p3, *p4, *p5, *p6;
  double2 *v1, *v2, *v3;
  int rc;
  if ((rc = dalloc(ctx, &p1, wt_ptr.size())) || (rc = dalloc(ctx, &p2, wt_l.size())) || (rc = dalloc(ctx, &v1, wt_v.size())) ||
      (rc = dalloc(ctx, &p3, w_ptr.size())) || (rc = dalloc(ctx, &p4, w_i.size())) || (rc = dalloc(ctx, &v2, w_v.size())) ||
      (rc = dalloc(ctx, &p5, t_ptr.size())) || (rc = dalloc(ctx, &p6, t_j.size())) || (rc = dalloc(ctx, &v3, t_v.size())))
    return rc;
  CK(cudaMemcpyAsync(p1, wt_ptr.data(), wt_ptr.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!wt_l.empty()) CK(cudaMemcpyAsync(p2, wt_l.data(), wt_l.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!wt_v.empty()) CK(cudaMemcpyAsync(v1, wt_v.data(), wt_v.size() * 16, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(p3, w_ptr.data(), w_ptr.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!w_i.empty()) CK(cudaMemcpyAsync(p4, w_i.data(), w_i.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!w_v.empty()) CK(cudaMemcpyAsync(v2, w_v.data(), w_v.size() * 16, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(p5, t_ptr.data(), t_ptr.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!t_j.empty()) CK(cudaMemcpyAsync(p6, t_j.data(), t_j.size() * 4, cudaMemcpyHostToDevice, ctx->st));
  if (!t_v.empty()) CK(cudaMemcpyAsync(v3, t_v.data(), t_v.size() * 16, cudaMemcpyHostToDevice, ctx->st));
  t.wt_ptr = p1; t.wt_l = p2; t.wt_v = v1; t.w_ptr = p3; t.w_i = p4; t.w_v = v2; t.t_ptr = p5; t.t_j = p6; t.t_v = v3;
  t.sp_ptr = nullptr; t.sp_c = nullptr; t.sp_e = nullptr;
  t.pq64 = nullptr; t.pq32 = nullptr; t.prow = nullptr; t.pK = 0; t.pnrows = 0; t.pndiag = 0; t.psym = 0;
  if (ctx->has_prod) {
    const std::vector<std::complex<double>>& Q = ctx->prod.Qr;
    std::vector<double2> q64(Q.size());
    std::vector<float2> q32(Q.size());
    for (size_t i = 0; i < Q.size(); ++i) {
      q64[i] = make_double2(Q[i].real(), Q[i].imag());
      q32[i] = make_float2((float)Q[i].real(), (float)Q[i].imag());
    }
    double2* d64;
    float2* d32;
    if ((rc = dalloc(ctx, &d64, q64.size())) || (rc = dalloc(ctx, &d32, q32.size()))) return rc;
    CK(cudaMemcpyAsync(d64, q64.data(), q64.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(d32, q32.data(), q32.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->st));
    int* rows;
    if ((rc = dalloc(ctx, &rows, ctx->prod.rows.size()))) return rc;
    CK(cudaMemcpyAsync(rows, ctx->prod.rows.data(), ctx->prod.rows.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));     // the host vectors go out of scope
    t.pq64 = d64; t.pq32 = d32; t.prow = rows; t.pK = ctx->prod.K;
    t.pnrows = (int)ctx->prod.rows.size(); t.pndiag = ctx->prod.ndiag; t.psym = ctx->prod.sym;
  }
  t.w2_64 = nullptr; t.w2_32 = nullptr;
  if (ctx->has_pair) {
    const size_t nw = (size_t)r->d * r->dimT;
    std::vector<double2> w64(nw);
    std::vector<float2> w32(nw);
    for (size_t i = 0; i < nw; ++i) {
      w64[i] = make_double2(r->W[2 * i], r->W[2 * i + 1]);
      w32[i] = make_float2((float)r->W[2 * i], (float)r->W[2 * i + 1]);
    }
    double2* d64;
    float2* d32;
    if ((rc = dalloc(ctx, &d64, nw)) || (rc = dalloc(ctx, &d32, nw))) return rc;
    CK(cudaMemcpyAsync(d64, w64.data(), nw * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(d32, w32.data(), nw * sizeof(float2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));     // the host vectors go out of scope
    t.w2_64 = d64; t.w2_32 = d32;
  }
  t.warp_bytes = (int)ctx->gen_warp_bytes;
  t.px_off = (int)ctx->gen_px_off;
  if (ctx->use_sp) {
    const ghsym::Terms& q = ctx->sp;
    int* sptr;
    double2* sc;
    unsigned char* se;
    if ((rc = dalloc(ctx, &sptr, q.ptr.size())) || (rc = dalloc(ctx, &sc, q.c.size() / 2)) || (rc = dalloc(ctx, &se, q.off.size())))
      return rc;
    CK(cudaMemcpyAsync(sptr, q.ptr.data(), q.ptr.size() * 4, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(sc, q.c.data(), q.c.size() * 8, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(se, q.off.data(), q.off.size(), cudaMemcpyHostToDevice, ctx->st));   // power-table offsets, word-padded
    t.sp_ptr = sptr; t.sp_c = sc; t.sp_e = se;
  }
  return GH_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* gh_last_error(const gh_ctx* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

int gh_rep_path(const gh_ctx* ctx, int* path) {
  if (!ctx || !path) return fail(nullptr, GH_ERR_ARG, "null argument");
  *path = ctx->rep != REP_GEN ? GH_PATH_REGISTER
          : ctx->b.gen_prod    ? GH_PATH_PRODUCT
          : ctx->b.gen_pair    ? GH_PATH_PAIR
          : (ctx->use_sp ? GH_PATH_CLOSED_FORM : GH_PATH_TENSOR);
  return GH_OK;
}

int gh_set_rep_path(gh_ctx* ctx, int path) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (ctx->rep != REP_GEN) return path == GH_PATH_REGISTER ? GH_OK : fail(ctx, GH_ERR_ARG, "not a general irrep");
  const int base = ctx->use_sp ? GH_PATH_CLOSED_FORM : GH_PATH_TENSOR;
  if (path == GH_PATH_PRODUCT) {
    if (!ctx->has_prod) return fail(ctx, GH_ERR_ARG, "this irrep has no product-of-adjoints form");
    ctx->b.gen_prod = 1;
  } else if (path == GH_PATH_PAIR) {
    if (!ctx->has_pair) return fail(ctx, GH_ERR_ARG, "this irrep is not a two-slot irrep outside the adjoint product");
    ctx->b.gen_pair = 1;
  } else if (path == base) {
    ctx->b.gen_prod = 0;
    ctx->b.gen_pair = 0;
  } else {
    return fail(ctx, GH_ERR_ARG, "path not available for this context");
  }
  invalidate_graph(ctx);
  return GH_OK;
}

// ---- domain decomposition (src/mpi/gauge_mpi.hpp, src/mpi/higgs_mpi.hpp) ----
int gh_set_domain(gh_ctx* ctx, int lat, const int* G, const int* lo, const int* hi, const int* goff) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!G || !lo || !hi || !goff) return fail(ctx, GH_ERR_ARG, "null argument");
  LatDev& L = ctx->lat_h[lat];
  long long Vi = 1, gs = 1;
  int dec = 0;
  for (int mu = 0; mu < ctx->D; ++mu) {
    const int Lm = L.L[mu];
    if (G[mu] < 1 || goff[mu] < 0) return fail(ctx, GH_ERR_ARG, "global extents must be >= 1 and offsets >= 0");
    if (lo[mu] == 0) {
      // a direction that is not split: the whole periodic extent, no halo
      if (hi[mu] != Lm || G[mu] != Lm || goff[mu] != 0)
        return fail(ctx, GH_ERR_ARG, "a direction without halo must hold the whole global extent");
    } else if (lo[mu] == 1) {
      // a split direction: interior [1, L-1) between one halo layer on each side
      if (hi[mu] != Lm - 1 || Lm < 3) return fail(ctx, GH_ERR_ARG, "a split direction needs hi = L - 1 and L >= 3");
      if (goff[mu] + (hi[mu] - lo[mu]) > G[mu]) return fail(ctx, GH_ERR_ARG, "subdomain reaches past the global extent");
      dec = 1;
    } else {
      return fail(ctx, GH_ERR_ARG, "lo must be 0 (whole direction) or 1 (one halo layer)");
    }
    Vi *= hi[mu] - lo[mu];
  }
  for (int mu = 0; mu < 4; ++mu) {
    L.lo[mu] = mu < ctx->D ? lo[mu] : 0;
    L.hi[mu] = mu < ctx->D ? hi[mu] : 1;
    L.goff[mu] = mu < ctx->D ? goff[mu] : 0;
    L.gstr[mu] = gs;
    gs *= mu < ctx->D ? G[mu] : 1;
  }
  L.Vi = (int)Vi;
  L.dec = dec;
  // the domain fields close the descriptor: one copy from lo to the end
  const size_t off = offsetof(LatDev, lo);
  CK(cudaMemcpyAsync((char*)(ctx->b.lats + lat) + off, (const char*)&L + off, sizeof(LatDev) - off,
                     cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_halo_count(gh_ctx* ctx, int lat, int field, int nu, long long* n_complex) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!n_complex) return fail(ctx, GH_ERR_ARG, "null output");
  if (nu < 0 || nu >= ctx->D) return fail(ctx, GH_ERR_ARG, "direction out of range");
  if (field != 0 && !(field == 1 && ctx->scalar)) return fail(ctx, GH_ERR_ARG, "field must be 0 (links) or 1 (phi)");
  const LatDev& L = ctx->lat_h[lat];
  const long long nplane = (long long)L.V / L.L[nu];
  *n_complex = nplane * (field == 0 ? (long long)ctx->D * ctx->N * ctx->N : ctx->d);
  return GH_OK;
}

static int halo_op(gh_ctx* ctx, int lat, int field, int nu, int layer, void* buf, int unpack) {
  long long n = 0;
  int rc = gh_halo_count(ctx, lat, field, nu, &n);
  if (rc) return rc;
  const LatDev& L = ctx->lat_h[lat];
  if (!buf) return fail(ctx, GH_ERR_ARG, "null buffer");
  if (layer < 0 || layer >= L.L[nu]) return fail(ctx, GH_ERR_ARG, "layer out of range");
  if ((reinterpret_cast<uintptr_t>(buf) & 15u) != 0) return fail(ctx, GH_ERR_ARG, "halo buffer must be 16-byte aligned");
  HaloArgs a{};
  a.lat = lat; a.f = field == 0 ? ctx->b.U : ctx->b.phi; a.buf = buf; a.kind = field; a.nu = nu; a.layer = layer;
  a.unpack = unpack; a.D = ctx->D; a.nn = ctx->N * ctx->N; a.d = ctx->d;
  a.nplane = (long long)L.V / L.L[nu];
  a.ncomp = field == 0 ? ctx->D * ctx->N * ctx->N : ctx->d;
  ctx->eng->halo(ctx->b, a);
  return launch_check(ctx, unpack ? "halo unpack" : "halo pack");
}
int gh_halo_pack(gh_ctx* ctx, int lat, int field, int nu, int layer, void* buf) {
  return halo_op(ctx, lat, field, nu, layer, buf, 0);
}
int gh_halo_unpack(gh_ctx* ctx, int lat, int field, int nu, int layer, const void* buf) {
  return halo_op(ctx, lat, field, nu, layer, const_cast<void*>(buf), 1);
}

int gh_save_fields(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaMemcpyAsync(ctx->b.Us, ctx->b.U, (size_t)ctx->nU * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st));
  if (ctx->scalar) CK(cudaMemcpyAsync(ctx->b.phis, ctx->b.phi, (size_t)ctx->nF * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st));
  return GH_OK;
}
int gh_restore_fields(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaMemcpyAsync(ctx->b.U, ctx->b.Us, (size_t)ctx->nU * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st));
  if (ctx->scalar) CK(cudaMemcpyAsync(ctx->b.phi, ctx->b.phis, (size_t)ctx->nF * 2 * ctx->rs, cudaMemcpyDeviceToDevice, ctx->st));
  return GH_OK;
}

uint64_t gh_rng_key(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e) { return ghrng::key(a, b, c, d, e); }
double gh_rng_uniform(uint64_t seed, uint64_t key) { return ghrng::uniform(seed, key); }
double gh_rng_gauss(uint64_t seed, uint64_t key) { return ghrng::gauss(seed, key); }

int gh_ctx_create(int D, int N, int n_lat, const int* L, const gh_rep_desc* rep, int precision,
                  const uint64_t* seeds, gh_ctx** out) {
  gh_ctx* ctx = nullptr;
  if (!out) return fail(nullptr, GH_ERR_ARG, "null output pointer");
  *out = nullptr;
  if (D < 2 || D > 4) return fail(nullptr, GH_ERR_UNSUPPORTED, "D must be 2, 3 or 4");
  if (N < 2 || N > 3) return fail(nullptr, GH_ERR_UNSUPPORTED, "N must be 2 or 3");
  if (n_lat < 1 || !L || !seeds) return fail(nullptr, GH_ERR_ARG, "need n_lat >= 1, extents and seeds");
  if (precision != GH_PREC_FP64 && precision != GH_PREC_FP32_MD && precision != GH_PREC_FP32_ALL)
    return fail(nullptr, GH_ERR_ARG, "unknown precision");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    cudaGetLastError();
    return fail(nullptr, GH_ERR_CUDA, "no CUDA device: the gauge_higgs_b200 engine has no CPU path");
  }
  std::unique_ptr<gh_ctx> c(new gh_ctx());
  ctx = c.get();
  ctx->D = D; ctx->N = N; ctx->ng = N * N - 1; ctx->nlat = n_lat; ctx->prec = precision;
  ctx->rs = precision == GH_PREC_FP64 ? sizeof(double) : sizeof(float);
  const int kind = rep ? rep->kind : GH_REP_NONE;
  switch (kind) {
    case GH_REP_NONE: ctx->rep = REP_NONE; ctx->d = 0; break;
    case GH_REP_FUND: ctx->rep = REP_FUND; ctx->d = N; ctx->real = 0; break;
    case GH_REP_ADJ: ctx->rep = REP_ADJ; ctx->d = N * N - 1; ctx->real = 1; break;
    case GH_REP_GENERAL: ctx->rep = REP_GEN; ctx->d = rep->d; ctx->real = rep->real ? 1 : 0; break;
    default: return fail(nullptr, GH_ERR_REP, "unknown representation kind");
  }
  if (kind == GH_REP_FUND && rep->d && rep->d != N) return fail(nullptr, GH_ERR_REP, "fundamental rep must have d = N");
  if (kind == GH_REP_ADJ && rep->d && rep->d != N * N - 1) return fail(nullptr, GH_ERR_REP, "adjoint rep must have d = N^2-1");
  ctx->scalar = ctx->rep != REP_NONE;
  // lattices, offsets and work tables
  long long u = 0, p = 0, f = 0, g = 0;
  std::vector<Work> wl, ws;
  std::vector<int> blk_first(1, 0);
  size_t stage = 1;
  for (int l = 0; l < n_lat; ++l) {
    LatDev Ld{};
    long long V = 1;
    for (int mu = 0; mu < 4; ++mu) { Ld.L[mu] = 1; Ld.stride[mu] = 0; }
    for (int mu = 0; mu < D; ++mu) {
      if (L[l * D + mu] < 1) return fail(nullptr, GH_ERR_ARG, "lattice extents must be >= 1");
      Ld.L[mu] = L[l * D + mu]; Ld.stride[mu] = (int)V; V *= L[l * D + mu];
    }
    if ((V + ULANE) * D * N * N > (1LL << 31) - 1) return fail(nullptr, GH_ERR_ARG, "lattice too large for 32-bit site indexing");
    Ld.V = (int)V; Ld.Vp = (int)((V + ULANE - 1) / ULANE * ULANE); Ld.cidx = l;
    // the whole lattice is active: no halo, global site = local site
    for (int mu = 0; mu < 4; ++mu) { Ld.lo[mu] = 0; Ld.hi[mu] = Ld.L[mu]; Ld.goff[mu] = 0; Ld.gstr[mu] = Ld.stride[mu]; }
    Ld.Vi = (int)V; Ld.dec = 0;
    Ld.u_off = u; Ld.p_off = p; Ld.f_off = f; Ld.g_off = g;
    Ld.beta = 2.3; Ld.kappa = 0.1; Ld.lambda = 0.5; Ld.seed = seeds[l];
    for (int mu = 0; mu < D; ++mu)
      if (L[l * D + mu] > 256) return fail(nullptr, GH_ERR_UNSUPPORTED, "lattice extents above 256 are not supported");
    default_tile(L + l * D, D, Ld.lt);
    u += (long long)Ld.Vp * D * N * N; p += (long long)Ld.Vp * D * ctx->ng; f += (long long)Ld.Vp * ctx->d;
    g += (ctx->rep == REP_GEN) ? (long long)Ld.Vp * D * ctx->d : 0;
    ctx->lat_h.push_back(Ld);
    for (int mu = 0; mu < D; ++mu)
      for (int s0 = 0; s0 < V; s0 += KBLOCK) wl.push_back(Work{l, mu, s0, (int)std::min<long long>(KBLOCK, V - s0)});
    for (int s0 = 0; s0 < V; s0 += KBLOCK) ws.push_back(Work{l, -1, s0, (int)std::min<long long>(KBLOCK, V - s0)});
    blk_first.push_back((int)ws.size());
    stage = std::max<size_t>(stage, (size_t)V * std::max<size_t>(std::max<size_t>((size_t)D * N * N * 2, (size_t)D * ctx->ng), (size_t)ctx->d * 2));
  }
  ctx->nU = u; ctx->nP = p; ctx->nF = f; ctx->nG = g;
  std::vector<Work> wg, wgp;
  int gw = GEN_WARPS;
  if (ctx->rep == REP_GEN) {
    // one warp per link.  Tensor path: a buffer of N^n complex numbers in shared memory.
    // Single-row irreps: D(U) in closed form (d*d + N*N*(n+1) FP64 complex) when that
    // costs fewer operations than the two slot sweeps of the tensor path, or when the
    // tensor buffer does not fit.
    const size_t cs = 2 * ctx->rs;
    const size_t tensor_warp = ((size_t)rep->dimT + 4 * (size_t)rep->d) * cs;
    if (rep->W && rep->d > 0 && rep->n_boxes >= 1 && rep->n_boxes <= 17 && rep->dimT > 0 && rep->dimT <= 200000) {
      std::string why;
      if (ghsym::build(N, rep->n_boxes, rep->d, rep->dimT, rep->W, 1L << 22, ctx->sp, &why)) {
        const double term_ops = (double)(ctx->sp.c.size() / 2) * N * N + 2.0 * rep->d * rep->d;
        const double tensor_ops = 2.0 * rep->n_boxes * (double)rep->dimT * N;
        ctx->use_sp = term_ops < tensor_ops || tensor_warp > 227 * 1024;
      }
    }
    // a warp's region: [tensor buffer, or D(U) and the powers of U's entries][px py pf pb];
    // the first part also holds the matter force's (a, row) partial sums (ng*d
    // doubles) after it is used, and A(M) of the potential before, where that fits
    size_t region = ctx->use_sp ? ((size_t)rep->d * rep->d + (size_t)N * N * (rep->n_boxes + 1)) * 16
                                : (size_t)rep->dimT * cs;
    region = std::max(region, (size_t)(N * N - 1) * rep->d * 8);
    region = (region + 15) / 16 * 16;
    size_t per_warp = region + 4 * (size_t)rep->d * cs;
    per_warp = (per_warp + 15) / 16 * 16;
    ctx->gen_warp_bytes = per_warp;
    ctx->gen_px_off = region;
    while (gw > 1 && gw * per_warp > 227 * 1024) gw /= 2;
    if (per_warp > 227 * 1024) return fail(nullptr, GH_ERR_REP, "general irrep too large for the shared-memory tensor buffer");
    for (int l = 0; l < n_lat; ++l)
      for (int mu = 0; mu < D; ++mu)
        for (int s0 = 0; s0 < ctx->lat_h[l].V; s0 += gw)
          wg.push_back(Work{l, mu, s0, std::min(gw, ctx->lat_h[l].V - s0)});
    // irreps inside the adjoint product: the product kernel, one item per 32-site block
    // and direction (taken over the tensor and closed-form paths when available)
    std::string pwhy;
    if (rep->W && ghadj::build(N, rep->n_boxes, rep->d, rep->dimT, rep->W, ctx->prod, &pwhy)) {
      ctx->has_prod = true;
      for (int l = 0; l < n_lat; ++l)
        for (int mu = 0; mu < D; ++mu)
          for (int s0 = 0; s0 < ctx->lat_h[l].V; s0 += GP_LINKS)
            wgp.push_back(Work{l, mu, s0, std::min(GP_LINKS, ctx->lat_h[l].V - s0)});
    }
    // two-slot irreps the product does not reach: every basis vector, as an N x N
    // matrix, symmetric (or every one antisymmetric), which the register path needs
    if (!ctx->has_prod && rep->W && rep->n_boxes == 2 && rep->dimT == (long)N * N) {
      int sign = 0;
      bool ok = true;
      for (int b = 0; b < rep->d && ok; ++b)
        for (int i = 0; i < N && ok; ++i)
          for (int j = 0; j < N && ok; ++j) {
            const double* wij = rep->W + 2 * ((size_t)b * N * N + i * N + j);
            const double* wji = rep->W + 2 * ((size_t)b * N * N + j * N + i);
            const double sym = std::fabs(wij[0] - wji[0]) + std::fabs(wij[1] - wji[1]);
            const double anti = std::fabs(wij[0] + wji[0]) + std::fabs(wij[1] + wji[1]);
            const int sg = sym < 1e-12 ? (anti < 1e-12 ? 0 : 1) : (anti < 1e-12 ? -1 : 2);
            if (sg == 2 || (sg != 0 && sign != 0 && sg != sign)) ok = false;
            else if (sg != 0) sign = sg;
          }
      ctx->has_pair = ok;
    }
  }
  std::vector<Work> wall = wl;
  wall.insert(wall.end(), ws.begin(), ws.end());

  ctx->eng.reset(N == 2 ? (precision == GH_PREC_FP64 ? make_engine_n2_f64(D, ctx->rep) : make_engine_n2_f32(D, ctx->rep))
                        : (precision == GH_PREC_FP64 ? make_engine_n3_f64(D, ctx->rep) : make_engine_n3_f32(D, ctx->rep)));
  if (!ctx->eng) return fail(nullptr, GH_ERR_UNSUPPORTED, "no kernel instance for this configuration");
  CK(cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking));
  ctx->st = ctx->own;
  Bufs& b = ctx->b;
  const size_t rs = ctx->rs;
  int rc;
  unsigned char *U, *Us, *P, *phi = nullptr, *phis = nullptr, *pi = nullptr, *psif = nullptr, *psib = nullptr;
  if ((rc = dalloc(ctx, &U, (size_t)u * 2 * rs)) || (rc = dalloc(ctx, &Us, (size_t)u * 2 * rs)) ||
      (rc = dalloc(ctx, &P, (size_t)p * rs)))
    { g_err = ctx->err; return rc; }
  if (ctx->scalar) {
    if ((rc = dalloc(ctx, &phi, (size_t)f * 2 * rs)) || (rc = dalloc(ctx, &phis, (size_t)f * 2 * rs)) ||
        (rc = dalloc(ctx, &pi, (size_t)f * 2 * rs)))
      { g_err = ctx->err; return rc; }
  }
  if (ctx->rep == REP_GEN) {
    if ((rc = dalloc(ctx, &psif, (size_t)g * 2 * rs)) || (rc = dalloc(ctx, &psib, (size_t)g * 2 * rs)) ||
        (rc = dalloc(ctx, &ctx->b.wpot, (size_t)std::max<long long>(f, 1))))
      { g_err = ctx->err; return rc; }
    if ((rc = build_general(ctx, rep))) { g_err = ctx->err; return rc; }
  }
  b.U = U; b.Us = Us; b.P = P; b.phi = phi; b.phis = phis; b.pi = pi; b.psif = psif; b.psib = psib;
  b.nw_links = (int)wl.size(); b.nw_sites = (int)ws.size(); b.nw_gen = (int)wg.size(); b.gen_warps = gw;
  b.nw_gprod = (int)wgp.size(); b.gen_prod = ctx->has_prod ? 1 : 0; b.gen_pair = ctx->has_pair ? 1 : 0;
  b.hist_cap = 1024;
  b.nlat = n_lat; b.D = D; b.N = N; b.d = ctx->d; b.rep = ctx->rep; b.scalar = ctx->scalar; b.st = ctx->st;
  if ((rc = dalloc(ctx, &b.lats, n_lat)) || (rc = dalloc(ctx, &b.w_all, wall.size())) ||
      (rc = dalloc(ctx, &b.w_gen, std::max<size_t>(wg.size(), 1))) ||
      (rc = dalloc(ctx, &b.w_gprod, std::max<size_t>(wgp.size(), 1))) || (rc = dalloc(ctx, &b.blk_first, blk_first.size())) ||
      (rc = dalloc(ctx, &b.partials, (size_t)ws.size() * NRED)) || (rc = dalloc(ctx, &b.res, (size_t)n_lat * 2 * NRES)) ||
      (rc = dalloc(ctx, &b.hist, (size_t)n_lat * b.hist_cap)) || (rc = dalloc(ctx, &ctx->staging, stage)) ||
      (rc = dalloc(ctx, &ctx->fbuf, (size_t)std::max<long long>(p, 1))) ||
      (rc = dalloc(ctx, &ctx->fphibuf, (size_t)std::max<long long>(f, 1) * 2)))
    { g_err = ctx->err; return rc; }
  ctx->staging_elems = stage;
  CK(cudaMemcpyAsync(b.lats, ctx->lat_h.data(), sizeof(LatDev) * n_lat, cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(b.w_all, wall.data(), sizeof(Work) * wall.size(), cudaMemcpyHostToDevice, ctx->st));
  if (!wg.empty()) CK(cudaMemcpyAsync(b.w_gen, wg.data(), sizeof(Work) * wg.size(), cudaMemcpyHostToDevice, ctx->st));
  if (!wgp.empty()) CK(cudaMemcpyAsync(b.w_gprod, wgp.data(), sizeof(Work) * wgp.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(b.blk_first, blk_first.data(), sizeof(int) * blk_first.size(), cudaMemcpyHostToDevice, ctx->st));
  if ((rc = rebuild_kick_table(ctx))) { g_err = ctx->err; return rc; }
  if (ctx->rep == REP_GEN) {
    const size_t sm = ctx->eng->gen_smem(b);
    if (sm > 227 * 1024) { g_err = "general irrep too large for the shared-memory tensor buffer"; return GH_ERR_REP; }
  }
  if ((rc = ctx->eng->prepare(b))) { g_err = "cudaFuncSetAttribute failed for a kernel of this context"; return GH_ERR_CUDA; }
  // identity links and zero fields as the starting state (GaugeField default is zero
  // matrices; a cold start is the useful default for a device engine)
  InitArgs ia{};
  ia.what = 4;
  ctx->eng->init(b, ia, true, false);
  CK(cudaStreamSynchronize(ctx->st));
  if ((rc = launch_check(ctx, "init"))) { g_err = ctx->err; return rc; }
  *out = c.release();
  return GH_OK;
}

int gh_ctx_destroy(gh_ctx* ctx) {
  delete ctx;
  return GH_OK;
}

int gh_set_stream(gh_ctx* ctx, void* stream) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaStreamSynchronize(ctx->st));
  ctx->st = stream ? (cudaStream_t)stream : ctx->own;
  ctx->b.st = ctx->st;
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_sync(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaStreamSynchronize(ctx->st));
  return launch_check(ctx, "sync");
}

int gh_info(const gh_ctx* ctx, int* D, int* N, int* n_lat, int* d, int* rep_kind, int* precision) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (D) *D = ctx->D;
  if (N) *N = ctx->N;
  if (n_lat) *n_lat = ctx->nlat;
  if (d) *d = ctx->d;
  if (rep_kind) *rep_kind = ctx->rep;
  if (precision) *precision = ctx->prec;
  return GH_OK;
}

int gh_device_bytes(const gh_ctx* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return fail(nullptr, GH_ERR_ARG, "null argument");
  *bytes = ctx->bytes;
  return GH_OK;
}

int gh_set_couplings(gh_ctx* ctx, int lat, double beta, double kappa, double lambda) {
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = l0; l < l1; ++l) {
    double v[3] = {beta, kappa, lambda};
    ctx->lat_h[l].beta = beta; ctx->lat_h[l].kappa = kappa; ctx->lat_h[l].lambda = lambda;
    CK(cudaMemcpyAsync((char*)(ctx->b.lats + l) + offsetof(LatDev, beta), v, sizeof(v), cudaMemcpyHostToDevice, ctx->st));
  }
  return GH_OK;
}

int gh_get_couplings(gh_ctx* ctx, int lat, double* beta, double* kappa, double* lambda) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  LatDev L;
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaMemcpyAsync(&L, ctx->b.lats + lat, sizeof(L), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (beta) *beta = L.beta;
  if (kappa) *kappa = L.kappa;
  if (lambda) *lambda = L.lambda;
  return GH_OK;
}

int gh_set_integrator(gh_ctx* ctx, int integ, int nmd, double tau) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if ((integ != GH_LEAPFROG && integ != GH_OMELYAN) || nmd < 1 || !(tau > 0.0))
    return fail(ctx, GH_ERR_ARG, "integrator must be leapfrog/omelyan with nmd >= 1 and tau > 0");
  ctx->integ = integ; ctx->nmd = nmd; ctx->tau = tau;
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_set_traj_count(gh_ctx* ctx, int lat, uint64_t traj_count, uint64_t accept_count) {
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->st));
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = l0; l < l1; ++l) {
    unsigned long long v[2] = {traj_count, accept_count};
    CK(cudaMemcpyAsync((char*)(ctx->b.lats + l) + offsetof(LatDev, traj), v, sizeof(v), cudaMemcpyHostToDevice, ctx->st));
  }
  return GH_OK;
}

int gh_get_traj_count(gh_ctx* ctx, int lat, uint64_t* traj_count, uint64_t* accept_count, uint64_t* nonfinite_count) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  LatDev L;
  CK(cudaStreamSynchronize(ctx->st));
  CK(cudaMemcpyAsync(&L, ctx->b.lats + lat, sizeof(L), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (traj_count) *traj_count = L.traj;
  if (accept_count) *accept_count = L.accepted;
  if (nonfinite_count) *nonfinite_count = L.nonfinite;
  return GH_OK;
}

int gh_set_links(gh_ctx* ctx, int lat, const double* U) { return xfer_field(ctx, lat, 0, ctx ? ctx->b.U : nullptr, U, true); }
int gh_get_links(gh_ctx* ctx, int lat, double* U) { return xfer_field(ctx, lat, 0, ctx ? ctx->b.U : nullptr, U, false); }
int gh_set_mom(gh_ctx* ctx, int lat, const double* P) { return xfer_field(ctx, lat, 1, ctx ? ctx->b.P : nullptr, P, true); }
int gh_get_mom(gh_ctx* ctx, int lat, double* P) { return xfer_field(ctx, lat, 1, ctx ? ctx->b.P : nullptr, P, false); }
int gh_set_phi(gh_ctx* ctx, int lat, const double* phi) { return xfer_field(ctx, lat, 2, ctx ? ctx->b.phi : nullptr, phi, true); }
int gh_get_phi(gh_ctx* ctx, int lat, double* phi) { return xfer_field(ctx, lat, 2, ctx ? ctx->b.phi : nullptr, phi, false); }
int gh_set_pi(gh_ctx* ctx, int lat, const double* pi) { return xfer_field(ctx, lat, 2, ctx ? ctx->b.pi : nullptr, pi, true); }
int gh_get_pi(gh_ctx* ctx, int lat, double* pi) { return xfer_field(ctx, lat, 2, ctx ? ctx->b.pi : nullptr, pi, false); }

int gh_hot_start(gh_ctx* ctx, double sigma) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  InitArgs a{};
  a.what = 0; a.sigma = sigma;
  ctx->eng->init(ctx->b, a, true, false);
  return launch_check(ctx, "hot_start");
}
int gh_cold_start(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  InitArgs a{};
  a.what = 4;
  ctx->eng->init(ctx->b, a, true, false);
  return launch_check(ctx, "cold_start");
}
int gh_phi_gaussian(gh_ctx* ctx, uint64_t stream, double sigma) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  InitArgs a{};
  a.what = 2; a.stream = stream; a.sigma = sigma; a.real = ctx->real; a.d = ctx->d; a.vec = ctx->b.phi;
  ctx->eng->init(ctx->b, a, false, true);
  return launch_check(ctx, "phi_gaussian");
}
int gh_phi_cold(gh_ctx* ctx, double c) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  InitArgs a{};
  a.what = 5; a.sigma = c; a.d = ctx->d; a.vec = ctx->b.phi;
  ctx->eng->init(ctx->b, a, false, true);
  return launch_check(ctx, "phi_cold");
}
int gh_mom_refresh(gh_ctx* ctx, uint64_t stream) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  InitArgs a{};
  a.what = 3; a.stream = stream;
  ctx->eng->init(ctx->b, a, true, false);
  return launch_check(ctx, "mom_refresh");
}
int gh_refresh_momenta(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  InitArgs a{};
  a.what = 1; a.pure = ctx->scalar ? 0 : 1; a.real = ctx->real; a.d = ctx->d; a.vec = ctx->b.pi;
  ctx->eng->init(ctx->b, a, true, ctx->scalar != 0);
  if (ctx->b.frozen) ctx->eng->sphere(ctx->b, 0);
  return launch_check(ctx, "refresh_momenta");
}

// Frozen-length scalar |phi_x| = 1 (GaugeHiggsHMC::frozen_phi, normalize_phi;
// src/hmc/gauge_higgs_hmc.hpp:38-40,61-103).
int gh_set_frozen_phi(gh_ctx* ctx, int on) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (on && !ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  CK(cudaStreamSynchronize(ctx->st));
  ctx->b.frozen = on ? 1 : 0;
  invalidate_graph(ctx);
  return GH_OK;
}
int gh_normalize_phi(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  ctx->eng->sphere(ctx->b, 1);
  return launch_check(ctx, "normalize_phi");
}

int gh_gauge_force(gh_ctx* ctx, int lat, double* F) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!F) return fail(ctx, GH_ERR_ARG, "null output");
  ctx->eng->kick(ctx->b, 0.0, M_WRITE, F_GAUGE, ctx->fbuf, true, false);
  if ((rc = launch_check(ctx, "gauge_force"))) return rc;
  return xfer_one(ctx, lat, 1, ctx->fbuf, F, false, true);
}
int gh_matter_link_force(gh_ctx* ctx, int lat, double* F) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!F) return fail(ctx, GH_ERR_ARG, "null output");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  if (ctx->rep == REP_GEN) ctx->eng->gen_links(ctx->b, 0.0, 2, ctx->fbuf);
  else ctx->eng->kick(ctx->b, 0.0, M_WRITE, F_MATTER, ctx->fbuf, true, false);
  if ((rc = launch_check(ctx, "matter_link_force"))) return rc;
  return xfer_one(ctx, lat, 1, ctx->fbuf, F, false, true);
}
int gh_scalar_force(gh_ctx* ctx, int lat, double* Fphi) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!Fphi) return fail(ctx, GH_ERR_ARG, "null output");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  if (ctx->rep == REP_GEN) ctx->eng->gen_links(ctx->b, 0.0, 2, ctx->fbuf);
  ctx->eng->kick(ctx->b, 0.0, M_WRITE, 0, ctx->fphibuf, false, true);
  if ((rc = launch_check(ctx, "scalar_force"))) return rc;
  return xfer_one(ctx, lat, 2, ctx->fphibuf, Fphi, false, true);
}

int gh_kick(gh_ctx* ctx, double eps) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  enq_kick(ctx, eps);
  return launch_check(ctx, "kick");
}
int gh_drift(gh_ctx* ctx, double eps) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  enq_drift(ctx, eps);
  return launch_check(ctx, "drift");
}
int gh_md_evolve(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  enq_md(ctx);
  return launch_check(ctx, "md_evolve");
}
int gh_reunitarize(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  ctx->eng->reunit(ctx->b);
  return launch_check(ctx, "reunitarize");
}

int gh_measure(gh_ctx* ctx, int lat, gh_obs* out) {
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (!out) return fail(ctx, GH_ERR_ARG, "null output");
  enq_measure(ctx, 0);
  if ((rc = launch_check(ctx, "measure"))) return rc;
  std::vector<double> res((size_t)ctx->nlat * 2 * NRES);
  CK(cudaMemcpyAsync(res.data(), ctx->b.res, res.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = l0; l < l1; ++l) {
    const double* r = &res[(size_t)l * 2 * NRES];
    gh_obs& o = out[l - l0];
    o.H = r[0]; o.S_g = r[1]; o.S_H = r[2]; o.kin_P = r[3]; o.kin_pi = r[4]; o.plaquette = r[5]; o.L_link = r[6]; o.L_phi = r[7];
  }
  return GH_OK;
}

// Per-lattice sums of the per-block partials written by a site-item reduction
// kernel (site items are laid out per lattice in order), divided by norm[l].
int site_partials_to_lattices(gh_ctx* ctx, int lat, const std::vector<double>& norm, double* out) {
  std::vector<double> part(ctx->b.nw_sites);
  CK(cudaMemcpyAsync(part.data(), ctx->b.partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  int first = 0;
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = 0; l < ctx->nlat; ++l) {
    const int nb = (ctx->lat_h[l].V + KBLOCK - 1) / KBLOCK;
    if (l >= l0 && l < l1) {
      double sum = 0.0;
      for (int q = first; q < first + nb; ++q) sum += part[q];
      out[l - l0] = sum / norm[l];
    }
    first += nb;
  }
  return GH_OK;
}

// Probe irrep of a traced loop from its Young rows (NULL: the fundamental); its
// dimension by the hook-content formula d = prod_cells (N + col - row) / hook.
int probe_rep(gh_ctx* ctx, const int* rows, int nrows, LoopArgs& a, double& d) {
  if (!rows || nrows == 0) { a.m = 1; a.lam[0] = 1; d = ctx->N; return GH_OK; }
  if (nrows < 0 || nrows > CHAR_MMAX || nrows > ctx->N) return fail(ctx, GH_ERR_ARG, "probe irrep: 1 to N Young rows");
  for (int i = 0; i < nrows; ++i)
    if (rows[i] < 1 || (i > 0 && rows[i] > rows[i - 1])) return fail(ctx, GH_ERR_ARG, "probe irrep: Young rows must be positive and non-increasing");
  if (rows[0] + nrows - 1 > CHAR_KMAX) return fail(ctx, GH_ERR_UNSUPPORTED, "probe irrep: first row too long");
  a.m = nrows;
  double num = 1.0, den = 1.0;
  for (int i = 0; i < nrows; ++i) {
    a.lam[i] = rows[i];
    for (int j = 0; j < rows[i]; ++j) {
      int below = 0;
      for (int k = i + 1; k < nrows; ++k) below += rows[k] > j;
      num *= (double)(ctx->N + j - i);
      den *= (double)(rows[i] - j - 1 + below + 1);
    }
  }
  d = num / den;
  return GH_OK;
}

// Wilson loops W(Ra, Rb) traced in a probe irrep, averaged over sites and planes
// mu < nu (wilson_loop_fund / wilson_loop_rep, src/measure/observables.hpp:48-79);
// Polyakov loops traced in a probe irrep (polyakov_loop_rep, :81-101).
int gh_wilson_loop(gh_ctx* ctx, int lat, int Ra, int Rb, const int* rows, int nrows, double* out) {
  if (ctx && any_decomposed(ctx)) return fail(ctx, GH_ERR_UNSUPPORTED, "not available on a subdomain of a decomposed lattice");
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (!out) return fail(ctx, GH_ERR_ARG, "null output");
  if (Ra < 1 || Rb < 1) return fail(ctx, GH_ERR_ARG, "loop extents must be >= 1");
  LoopArgs a{};
  double d = 0.0;
  if ((rc = probe_rep(ctx, rows, nrows, a, d))) return rc;
  a.mode = 1; a.Ra = Ra; a.Rb = Rb;
  ctx->eng->loops(ctx->b, a);
  if ((rc = launch_check(ctx, "wilson_loop"))) return rc;
  std::vector<double> norm(ctx->nlat);
  for (int l = 0; l < ctx->nlat; ++l) norm[l] = (double)ctx->lat_h[l].V * (ctx->D * (ctx->D - 1) / 2) * d;
  return site_partials_to_lattices(ctx, lat, norm, out);
}

int gh_polyakov_rep(gh_ctx* ctx, int lat, int tdir, const int* rows, int nrows, double* out) {
  if (ctx && any_decomposed(ctx)) return fail(ctx, GH_ERR_UNSUPPORTED, "not available on a subdomain of a decomposed lattice");
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (!out) return fail(ctx, GH_ERR_ARG, "null output");
  if (tdir < 0) tdir = ctx->D - 1;
  if (tdir >= ctx->D) return fail(ctx, GH_ERR_ARG, "tdir out of range");
  LoopArgs a{};
  double d = 0.0;
  if ((rc = probe_rep(ctx, rows, nrows, a, d))) return rc;
  a.mode = 0; a.tdir = tdir;
  ctx->eng->loops(ctx->b, a);
  if ((rc = launch_check(ctx, "polyakov_rep"))) return rc;
  std::vector<double> norm(ctx->nlat);
  for (int l = 0; l < ctx->nlat; ++l) norm[l] = (double)ctx->lat_h[l].V / ctx->lat_h[l].L[tdir] * d;
  return site_partials_to_lattices(ctx, lat, norm, out);
}

int gh_polyakov(gh_ctx* ctx, int lat, int tdir, double* out) {
  if (ctx && any_decomposed(ctx)) return fail(ctx, GH_ERR_UNSUPPORTED, "not available on a subdomain of a decomposed lattice");
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (!out) return fail(ctx, GH_ERR_ARG, "null output");
  if (tdir < 0) tdir = ctx->D - 1;
  if (tdir >= ctx->D) return fail(ctx, GH_ERR_ARG, "tdir out of range");
  ctx->eng->polyakov(ctx->b, tdir);
  if ((rc = launch_check(ctx, "polyakov"))) return rc;
  std::vector<double> part(ctx->b.nw_sites);
  CK(cudaMemcpyAsync(part.data(), ctx->b.partials, part.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  // blk_first on the host: site items are laid out per lattice in order
  int first = 0;
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = 0; l < ctx->nlat; ++l) {
    const int nb = (ctx->lat_h[l].V + KBLOCK - 1) / KBLOCK;
    if (l >= l0 && l < l1) {
      double s = 0.0;
      for (int q = first; q < first + nb; ++q) s += part[q];
      const double count = (double)ctx->lat_h[l].V / ctx->lat_h[l].L[tdir];
      out[l - l0] = s / (count * ctx->N);
    }
    first += nb;
  }
  return GH_OK;
}

int gh_set_tile(gh_ctx* ctx, int lat, const int* tile) {
  int rc = check_lat(ctx, lat, true);
  if (rc) return rc;
  if (!tile) return fail(ctx, GH_ERR_ARG, "null tile");
  int lt[4] = {0, 0, 0, 0}, sum = 0;
  for (int mu = 0; mu < ctx->D; ++mu) {
    if (tile[mu] < 1 || (tile[mu] & (tile[mu] - 1))) return fail(ctx, GH_ERR_ARG, "tile extents must be powers of two");
    lt[mu] = ceil_log2(tile[mu]);
    sum += lt[mu];
  }
  if (sum > KICK_LOG2) return fail(ctx, GH_ERR_ARG, "a tile holds at most as many sites as a kick block has threads");
  const int l0 = lat < 0 ? 0 : lat, l1 = lat < 0 ? ctx->nlat : lat + 1;
  for (int l = l0; l < l1; ++l) std::memcpy(ctx->lat_h[l].lt, lt, sizeof(lt));
  return rebuild_kick_table(ctx);
}

int gh_get_tile(gh_ctx* ctx, int lat, int* tile) {
  int rc = check_lat(ctx, lat, false);
  if (rc) return rc;
  if (!tile) return fail(ctx, GH_ERR_ARG, "null tile");
  for (int mu = 0; mu < 4; ++mu) tile[mu] = mu < ctx->D ? 1 << ctx->lat_h[lat].lt[mu] : 1;
  return GH_OK;
}

// Choose the kick tile of every group of equal-extent lattices by timing: each
// admissible shape (power-of-two extents, KICK_BLOCK sites, no wider than the lattice)
// runs `reps` zero-step kicks on that group alone; the fastest is kept.
int gh_autotune(gh_ctx* ctx, int reps, double* best_ms) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (reps < 1) reps = 3;
  CK(cudaStreamSynchronize(ctx->st));
  std::map<std::vector<int>, std::vector<int>> groups;
  for (int l = 0; l < ctx->nlat; ++l) groups[std::vector<int>(ctx->lat_h[l].L, ctx->lat_h[l].L + ctx->D)].push_back(l);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double total_best = 0.0;
  int gi = 0;
  for (auto& kv : groups) {
    const std::vector<int>& ext = kv.first;
    const std::vector<int>& lats = kv.second;
    int maxb[4] = {0, 0, 0, 0}, summax = 0;
    for (int mu = 0; mu < ctx->D; ++mu) { maxb[mu] = std::min(KICK_LOG2, ceil_log2(ext[mu])); summax += maxb[mu]; }
    const int target = std::min(KICK_LOG2, summax);
    double best = 1e30;
    int best_lt[4] = {0, 0, 0, 0};
    int lt[4] = {0, 0, 0, 0};
    // enumerate lt in [0, maxb] per direction with sum == target
    for (lt[0] = 0; lt[0] <= maxb[0]; ++lt[0])
      for (lt[1] = 0; lt[1] <= maxb[1]; ++lt[1])
        for (lt[2] = 0; lt[2] <= maxb[2]; ++lt[2])
          for (lt[3] = 0; lt[3] <= maxb[3]; ++lt[3]) {
            if (lt[0] + lt[1] + lt[2] + lt[3] != target) continue;
            for (int l : lats) std::memcpy(ctx->lat_h[l].lt, lt, sizeof(lt));
            int rc = push_tiles(ctx);
            if (rc) return rc;
            std::vector<Work> items;
            int nl, ns;
            kick_items(ctx, lats, items, nl, ns);
            if ((rc = upload_kick_items(ctx, items, nl, ns))) return rc;
            ctx->eng->kick(ctx->b, 0.0, M_UPDATE, F_GAUGE | F_MATTER, nullptr, true, true);
            CK(cudaEventRecord(e0, ctx->st));
            for (int r = 0; r < reps; ++r) ctx->eng->kick(ctx->b, 0.0, M_UPDATE, F_GAUGE | F_MATTER, nullptr, true, true);
            CK(cudaEventRecord(e1, ctx->st));
            CK(cudaEventSynchronize(e1));
            if ((rc = launch_check(ctx, "autotune"))) return rc;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms / reps < best) { best = ms / reps; std::memcpy(best_lt, lt, sizeof(lt)); }
          }
    for (int l : lats) std::memcpy(ctx->lat_h[l].lt, best_lt, sizeof(best_lt));
    total_best += best;
    ++gi;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_ms) *best_ms = total_best;
  return rebuild_kick_table(ctx);
}

// Multi-invariant onsite potential (src/action/scalar_invariants.hpp:190-206): the
// channel superoperator is built on the host (gh_potential.cpp) and its nonzero entries
// are copied to the device (values in both precisions).  The kick's site items and the
// measure kernel apply it for the fundamental and adjoint; for general irreps the link
// kernel computes w = A(M) phi once per site and both read that.
int gh_set_potential_multi(gh_ctx* ctx, int n_channels, const double* f, double mu2) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (!ctx->scalar) return fail(ctx, GH_ERR_STATE, "no scalar field in a pure-gauge context");
  if (n_channels < 0 || (n_channels > 0 && !f)) return fail(ctx, GH_ERR_ARG, "null couplings");
  const int kind = ctx->rep == REP_FUND ? GH_REP_FUND : ctx->rep == REP_ADJ ? GH_REP_ADJ : GH_REP_GENERAL;
  std::vector<double> c2, A;
  std::string err;
  int rc = ghpot::superop(ctx->N, kind, ctx->d, ctx->T_host.empty() ? nullptr : ctx->T_host.data(),
                          std::vector<double>(f, f + n_channels), c2, A, err);
  if (rc) return fail(ctx, rc, err);
  // sparse rows: entries below 1e-15 of the largest are the rounding residue of the
  // projector construction where A vanishes exactly (weight conservation)
  const int d = ctx->d, dd = d * d;
  double amax = 0.0;
  for (size_t k = 0; k < (size_t)dd * dd; ++k) amax = std::max(amax, std::hypot(A[2 * k], A[2 * k + 1]));
  std::vector<int> ptr(dd + 1, 0);
  std::vector<unsigned short> ij;
  std::vector<double2> v64;
  std::vector<float2> v32;
  for (int rq = 0; rq < dd; ++rq) {
    for (int c = 0; c < dd; ++c) {
      const size_t k = (size_t)rq * dd + c;
      if (std::hypot(A[2 * k], A[2 * k + 1]) <= 1e-15 * amax) continue;
      ij.push_back((unsigned short)((c / d) | ((c % d) << 8)));
      v64.push_back(make_double2(A[2 * k], A[2 * k + 1]));
      v32.push_back(make_float2((float)A[2 * k], (float)A[2 * k + 1]));
    }
    ptr[rq + 1] = (int)ij.size();
  }
  const size_t nz = std::max<size_t>(ij.size(), 1);
  CK(cudaStreamSynchronize(ctx->st));
  ctx->free_potential();
  CK(cudaMalloc(&ctx->sa_ptr, ptr.size() * sizeof(int)));
  CK(cudaMalloc(&ctx->sa_ij, nz * sizeof(unsigned short)));
  CK(cudaMalloc(&ctx->sa_v64, nz * sizeof(double2)));
  CK(cudaMalloc(&ctx->sa_v32, nz * sizeof(float2)));
  CK(cudaMemcpyAsync(ctx->sa_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
  if (!ij.empty()) {
    CK(cudaMemcpyAsync(ctx->sa_ij, ij.data(), ij.size() * sizeof(unsigned short), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->sa_v64, v64.data(), v64.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->sa_v32, v32.data(), v32.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->st));
  }
  ctx->b.sa64 = PotA{ctx->sa_ptr, ctx->sa_ij, ctx->sa_v64};
  ctx->b.sa32 = PotA{ctx->sa_ptr, ctx->sa_ij, ctx->sa_v32};
  ctx->b.pot = POT_MULTI;
  ctx->b.mu2 = mu2;
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_set_potential_quartic(gh_ctx* ctx) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaStreamSynchronize(ctx->st));
  ctx->b.pot = POT_QUARTIC;
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_use_graph(gh_ctx* ctx, int enable) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  ctx->use_graph = enable ? 1 : 0;
  return GH_OK;
}

int gh_trajectory(gh_ctx* ctx, double* dH, int* accepted) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  int rc = run_traj(ctx);
  if (rc) return rc;
  std::vector<LatDev> L(ctx->nlat);
  std::vector<double> res((size_t)ctx->nlat * 2 * NRES);
  CK(cudaMemcpyAsync(L.data(), ctx->b.lats, sizeof(LatDev) * ctx->nlat, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(res.data(), ctx->b.res, res.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  for (int l = 0; l < ctx->nlat; ++l) {
    if (dH) dH[l] = res[((size_t)l * 2 + 1) * NRES] - res[(size_t)l * 2 * NRES];
    if (accepted) accepted[l] = L[l].last_acc;
  }
  return GH_OK;
}

int gh_run_trajectories(gh_ctx* ctx, int ntraj, gh_traj_record* records) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (ntraj < 0) return fail(ctx, GH_ERR_ARG, "ntraj < 0");
  const int cap = ctx->b.hist_cap;
  std::vector<TrajRec> h((size_t)ctx->nlat * cap);
  for (int t0 = 0; t0 < ntraj; t0 += cap) {
    const int nt = std::min(cap, ntraj - t0);
    for (int t = 0; t < nt; ++t) { int rc = run_traj(ctx); if (rc) return rc; }
    if (records) {
      std::vector<LatDev> L(ctx->nlat);
      CK(cudaMemcpyAsync(L.data(), ctx->b.lats, sizeof(LatDev) * ctx->nlat, cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaMemcpyAsync(h.data(), ctx->b.hist, sizeof(TrajRec) * h.size(), cudaMemcpyDeviceToHost, ctx->st));
      CK(cudaStreamSynchronize(ctx->st));
      for (int l = 0; l < ctx->nlat; ++l)
        for (int t = 0; t < nt; ++t) {
          const unsigned long long tr = L[l].traj - (unsigned long long)(nt - t);   // traj number - 1 of record t
          const TrajRec& r = h[(size_t)l * cap + (int)(tr % (unsigned long long)cap)];
          gh_traj_record& o = records[(size_t)(t0 + t) * ctx->nlat + l];
          o.dH = r.dH; o.accepted = r.accepted; o.traj = r.traj; o.plaquette = r.plaq; o.L_phi = r.L_phi; o.L_link = r.L_link; o.kappa = r.kappa;
          o.beta = r.beta;
        }
    }
  }
  if (!records) CK(cudaStreamSynchronize(ctx->st));
  return launch_check(ctx, "run_trajectories");
}

int gh_enqueue_trajectories(gh_ctx* ctx, int ntraj) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (ntraj < 0) return fail(ctx, GH_ERR_ARG, "ntraj < 0");
  for (int t = 0; t < ntraj; ++t) { int rc = run_traj(ctx); if (rc) return rc; }
  return GH_OK;
}

int gh_read_records(gh_ctx* ctx, int ntraj, gh_traj_record* records) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  const int cap = ctx->b.hist_cap;
  if (ntraj < 0 || ntraj > cap || !records) return fail(ctx, GH_ERR_ARG, "need 0 <= ntraj <= 1024 and an output array");
  std::vector<TrajRec> h((size_t)ctx->nlat * cap);
  std::vector<LatDev> L(ctx->nlat);
  CK(cudaMemcpyAsync(L.data(), ctx->b.lats, sizeof(LatDev) * ctx->nlat, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaMemcpyAsync(h.data(), ctx->b.hist, sizeof(TrajRec) * h.size(), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  for (int l = 0; l < ctx->nlat; ++l)
    for (int t = 0; t < ntraj; ++t) {
      gh_traj_record& o = records[(size_t)t * ctx->nlat + l];
      if (L[l].traj < (unsigned long long)(ntraj - t)) { std::memset(&o, 0, sizeof(o)); continue; }
      const unsigned long long tr = L[l].traj - (unsigned long long)(ntraj - t);
      const TrajRec& r = h[(size_t)l * cap + (int)(tr % (unsigned long long)cap)];
      o.dH = r.dH; o.accepted = r.accepted; o.traj = r.traj; o.plaquette = r.plaq; o.L_phi = r.L_phi; o.L_link = r.L_link; o.kappa = r.kappa;
          o.beta = r.beta;
    }
  return GH_OK;
}

int gh_trajectory_host(gh_ctx* ctx, double* U, double* phi, gh_traj_record* rec) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (ctx->nlat != 1) return fail(ctx, GH_ERR_ARG, "gh_trajectory_host needs a single-lattice context");
  int rc;
  if (U && (rc = gh_set_links(ctx, 0, U))) return rc;
  if (phi && ctx->scalar && (rc = gh_set_phi(ctx, 0, phi))) return rc;
  if ((rc = run_traj(ctx))) return rc;
  // the record first: a rejected trajectory restores the state that was passed in, so
  // the fields are only copied back when the trajectory was accepted
  LatDev L;
  TrajRec r;
  CK(cudaMemcpyAsync(&L, ctx->b.lats, sizeof(L), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  const int slot = (int)((L.traj - 1) % (unsigned long long)ctx->b.hist_cap);
  CK(cudaMemcpyAsync(&r, ctx->b.hist + slot, sizeof(r), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (r.accepted) {
    if (U && (rc = gh_get_links(ctx, 0, U))) return rc;
    if (phi && ctx->scalar && (rc = gh_get_phi(ctx, 0, phi))) return rc;
  }
  if (rec) {
    rec->dH = r.dH; rec->accepted = r.accepted; rec->traj = r.traj; rec->plaquette = r.plaq; rec->L_phi = r.L_phi; rec->L_link = r.L_link;
    rec->kappa = r.kappa;
    rec->beta = r.beta;
  }
  return GH_OK;
}

int gh_temper_enable(gh_ctx* ctx, int mode, uint64_t swap_seed) {
  if (ctx && any_decomposed(ctx)) return fail(ctx, GH_ERR_UNSUPPORTED, "not available on a subdomain of a decomposed lattice");
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  invalidate_graph(ctx);
  if (mode == 0) { ctx->temper = 0; return GH_OK; }
  if (mode != 1 && mode != 2) return fail(ctx, GH_ERR_ARG, "tempering mode: 1 (kappa) or 2 (beta)");
  if (mode == 1 && !ctx->scalar) return fail(ctx, GH_ERR_STATE, "kappa tempering needs a scalar field");
  CK(cudaStreamSynchronize(ctx->st));
  std::vector<LatDev> L(ctx->nlat);
  CK(cudaMemcpyAsync(L.data(), ctx->b.lats, sizeof(LatDev) * ctx->nlat, cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  // group lattices by extents, order each group by kappa
  std::map<std::vector<int>, std::vector<int>> groups;
  for (int l = 0; l < ctx->nlat; ++l) groups[std::vector<int>(L[l].L, L[l].L + ctx->D)].push_back(l);
  std::vector<int> order, gb(1, 0), pairmap;
  for (auto& kv : groups) {
    auto v = kv.second;
    auto cpl = [&](int l) { return mode == 2 ? L[l].beta : L[l].kappa; };
    std::sort(v.begin(), v.end(), [&](int a, int b) { return cpl(a) < cpl(b); });
    for (size_t k = 0; k + 1 < v.size(); ++k)
      if (!(cpl(v[k + 1]) > cpl(v[k])))
        return fail(ctx, GH_ERR_ARG, "the tempered coupling of equal-extent lattices must be strictly increasing");
    order.insert(order.end(), v.begin(), v.end());
    gb.push_back((int)order.size());
  }
  // pair id of position k (pair (k, k+1) within a group) -> compact index over all groups
  pairmap.assign(order.size(), 0);
  int pid = 0;
  for (size_t g = 0; g + 1 < gb.size(); ++g)
    for (int k = gb[g]; k + 1 < gb[g + 1]; ++k) pairmap[k] = pid++;
  int rc;
  if (!ctx->t_order) {
    if ((rc = dalloc(ctx, &ctx->t_order, ctx->nlat)) || (rc = dalloc(ctx, &ctx->t_groups, ctx->nlat + 1)) ||
        (rc = dalloc(ctx, &ctx->t_stats, 2 * ctx->nlat + 1)) || (rc = dalloc(ctx, &ctx->t_pairmap, ctx->nlat)))
      return rc;
  }
  CK(cudaMemcpyAsync(ctx->t_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->t_groups, gb.data(), sizeof(int) * gb.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->t_pairmap, pairmap.data(), sizeof(int) * pairmap.size(), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaMemsetAsync(ctx->t_stats, 0, sizeof(unsigned long long) * (2 * ctx->nlat + 1), ctx->st));
  ctx->t_ngroups = (int)gb.size() - 1;
  ctx->temper = mode;
  ctx->swap_seed = swap_seed;
  return GH_OK;
}

int gh_temper_interval(gh_ctx* ctx, int n_sweep) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  if (n_sweep < 1) return fail(ctx, GH_ERR_ARG, "n_sweep must be >= 1");
  CK(cudaStreamSynchronize(ctx->st));
  ctx->temper_every = n_sweep;
  invalidate_graph(ctx);
  return GH_OK;
}

int gh_temper_stats(gh_ctx* ctx, uint64_t* attempts, uint64_t* accepts, double* kappa_of_lat) {
  if (!ctx) return fail(nullptr, GH_ERR_ARG, "null context");
  CK(cudaStreamSynchronize(ctx->st));
  if (ctx->t_stats) {
    std::vector<unsigned long long> s(2 * ctx->nlat + 1);
    CK(cudaMemcpyAsync(s.data(), ctx->t_stats, sizeof(unsigned long long) * s.size(), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int k = 0; k < ctx->nlat - 1; ++k) {
      if (attempts) attempts[k] = s[k];
      if (accepts) accepts[k] = s[ctx->nlat + k];
    }
  }
  if (kappa_of_lat) {
    std::vector<LatDev> L(ctx->nlat);
    CK(cudaMemcpyAsync(L.data(), ctx->b.lats, sizeof(LatDev) * ctx->nlat, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int l = 0; l < ctx->nlat; ++l) kappa_of_lat[l] = L[l].kappa;
  }
  return GH_OK;
}

}  // extern "C"
