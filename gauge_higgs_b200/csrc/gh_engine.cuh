// gh_engine.cuh -- launchers of one (D, N, precision, representation) instance.
// The context (gh_ctx.cu) holds one Engine chosen at creation; every launch goes
// to the context's stream, so a whole trajectory can be captured as a graph.
#pragma once
#include <algorithm>
#include "gh_kernels.cuh"

namespace ghk {

// Launch with programmatic stream serialisation (see pdl_enter): the kernel may be
// scheduled while the previous kernel in the stream drains.
template <typename A>
inline void launch(void (*kernel)(A), unsigned grid, unsigned block, size_t smem, cudaStream_t st, const A& args) {
  if (grid == 0) return;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args);
}

struct Bufs {
  void *U, *Us, *P, *phi, *phis, *pi, *psif, *psib;
  LatDev* lats;
  Work* w_all;     // link items (all lattices, all mu) followed by site items
  int nw_links, nw_sites;
  Work* w_gen;     // general irrep: items of gen_warps links (one warp per link)
  int nw_gen;
  Work* w_gprod;   // general irrep, product of adjoints: items of up to 32 links (one 32-site block)
  int nw_gprod;
  int gen_prod;    // 1: general-irrep link work through k_gen_prod (gen.pq64 set)
  int gen_pair;    // 1: general-irrep link work through k_gen_pair (gen.w2_64 set)
  int gen_warps;   // warps per block of k_gen_links (1..GEN_WARPS, from the tensor size)
  int* blk_first;  // [nlat+1] first site item of each lattice (relative to the site items)
  Work* w_kick;    // kick items over 4-D tiles (LatDev::lt): link items then site items
  int nwk_links, nwk_sites;
  double* partials;
  double* res;
  TrajRec* hist;
  int hist_cap;
  GenTables gen;
  int nlat, D, N, d, rep, scalar;
  int frozen;            // frozen-length scalar |phi_x| = 1
  int pot;               // POT_QUARTIC or POT_MULTI
  double mu2;
  PotA sa64, sa32;       // multi-invariant potential superoperator, FP64 and FP32 values
  double2* wpot;         // general irreps: w = A(M) phi per site (FP64, laid out like phi)
  cudaStream_t st;
};

struct EngineBase {
  virtual ~EngineBase() {}
  virtual void kick(const Bufs& b, double eps, int mode, int flags, double* out, bool links, bool sites) = 0;
  virtual void gen_links(const Bufs& b, double eps, int mode, double* out) = 0;
  // reunit: 0 none (FP64 mode), 1 projection in FP64 arithmetic, 2 the all-FP32 update
  virtual void drift(const Bufs& b, double eps, int reunit) = 0;
  virtual void reunit(const Bufs& b) = 0;
  virtual void sphere(const Bufs& b, int what) = 0;
  virtual void measure(const Bufs& b) = 0;
  virtual void init(const Bufs& b, InitArgs a, bool links, bool sites) = 0;
  virtual void restore(const Bufs& b) = 0;
  virtual void polyakov(const Bufs& b, int tdir) = 0;
  virtual void loops(const Bufs& b, LoopArgs a) = 0;
  virtual void xfer(const Bufs& b, XferArgs a) = 0;
  virtual void halo(const Bufs& b, HaloArgs a) = 0;
  virtual size_t gen_smem(const Bufs& b) const = 0;
  virtual int prepare(const Bufs& b) = 0;
};

template <int D, int N, typename R, int REP>
struct Engine : EngineBase {
  typedef typename Cmp<R>::t C;
  Engine() {}
  size_t gen_smem(const Bufs& b) const override {
    return (size_t)b.gen_warps * b.gen.warp_bytes;
  }
  int prepare(const Bufs& b) override {
    if (REP != REP_GEN) return 0;
    cudaError_t e = cudaFuncSetAttribute(k_gen_links<D, N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gen_smem(b));
    if (e == cudaSuccess && b.gen.pq64) {
      e = b.gen.pK == 1 ? cudaFuncSetAttribute(k_gen_prod<D, N, R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)gen_prod_smem<N, 1, C>(b.d, b.gen.pnrows))
                        : cudaFuncSetAttribute(k_gen_prod<D, N, R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)gen_prod_smem<N, 2, C>(b.d, b.gen.pnrows));
    }
    return e == cudaSuccess ? 0 : -1;
  }
  void kick(const Bufs& b, double eps, int mode, int flags, double* out, bool links, bool sites) override {
    KickArgs a;
    a.lats = b.lats; a.U = b.U; a.P = b.P; a.phi = b.phi; a.pi = b.pi; a.psif = b.psif; a.psib = b.psib;
    a.eps = eps; a.mode = mode; a.flags = flags; a.d = b.d; a.out = out;
    a.pot = b.pot; a.mu2 = b.mu2;
    a.sa = sizeof(R) == sizeof(double) ? b.sa64 : b.sa32;
    a.wpot = b.wpot;
    const bool do_sites = sites && b.scalar;
    const int first = links ? 0 : b.nwk_links;
    const int count = (links ? b.nwk_links : 0) + (do_sites ? b.nwk_sites : 0);
    if (count == 0) return;
    a.work = b.w_kick + first;
    launch(k_kick<D, N, R, REP>, count, KICK_BLOCK, 0, b.st, a);
  }
  void gen_links(const Bufs& b, double eps, int mode, double* out) override {
    if (REP != REP_GEN) return;
    GenArgs a;
    a.work = b.w_gen; a.lats = b.lats; a.U = b.U; a.P = b.P; a.phi = b.phi; a.psif = b.psif; a.psib = b.psib;
    a.t = b.gen; a.eps = eps; a.mode = mode; a.out = out;
    a.pot = b.pot; a.sa = b.sa64; a.wpot = b.wpot;
    if (b.gen_pair && b.gen.w2_64 && b.pot != POT_MULTI) {  // two-slot irreps in registers, one thread per link
      a.work = b.w_all;
      launch(k_gen_pair<D, N, R>, b.nw_links, KBLOCK, 0, b.st, a);
      return;
    }
    if (b.gen_prod && b.gen.pq64 && b.pot != POT_MULTI) {   // the potential's w is computed by k_gen_links
      a.work = b.w_gprod;
      if (b.gen.pK == 1) launch(k_gen_prod<D, N, R, 1>, b.nw_gprod, GP_THREADS, gen_prod_smem<N, 1, C>(b.d, b.gen.pnrows), b.st, a);
      else launch(k_gen_prod<D, N, R, 2>, b.nw_gprod, GP_THREADS, gen_prod_smem<N, 2, C>(b.d, b.gen.pnrows), b.st, a);
      return;
    }
    const size_t sm = gen_smem(b);
    launch(k_gen_links<D, N, R>, b.nw_gen, b.gen_warps * 32, sm, b.st, a);
  }
  void drift(const Bufs& b, double eps, int reunit) override {
    DriftArgs a;
    a.work = b.w_all; a.lats = b.lats; a.U = b.U; a.P = b.P; a.phi = b.phi; a.pi = b.pi;
    a.eps = eps; a.d = b.d; a.frozen = b.frozen;
    const unsigned nb = b.nw_links + (b.scalar ? b.nw_sites : 0);
    // reunit 2: the all-FP32 link update (GH_PREC_FP32_ALL); otherwise FP64 arithmetic,
    // projected back to SU(N) (1) or not (0, the FP64 mode)
    if constexpr (sizeof(R) != sizeof(double)) {
      if (reunit == 2) { launch(k_drift<N, R, float, true>, nb, KBLOCK, 0, b.st, a); return; }
    }
    if (reunit) launch(k_drift<N, R, double, true>, nb, KBLOCK, 0, b.st, a);
    else launch(k_drift<N, R, double, false>, nb, KBLOCK, 0, b.st, a);
  }
  void sphere(const Bufs& b, int what) override {
    if (!b.scalar) return;
    SphereArgs a;
    a.work = b.w_all + b.nw_links; a.lats = b.lats; a.phi = b.phi; a.pi = b.pi; a.d = b.d; a.what = what;
    launch(k_sphere<R>, b.nw_sites, KBLOCK, 0, b.st, a);
  }
  void reunit(const Bufs& b) override {
    LinkArgs a;
    a.work = b.w_all; a.lats = b.lats; a.U = b.U; a.Us = b.Us;
    launch(k_reunit<N, R>, b.nw_links, KBLOCK, 0, b.st, a);
  }
  void measure(const Bufs& b) override {
    if (REP == REP_GEN && b.scalar) gen_links(b, 0.0, 1, nullptr);
    MeasArgs a;
    a.work = b.w_all + b.nw_links; a.lats = b.lats; a.U = b.U; a.P = b.P; a.phi = b.phi; a.pi = b.pi;
    a.psif = b.psif; a.d = b.d; a.scalar = b.scalar; a.partials = b.partials;
    a.pot = b.pot; a.mu2 = b.mu2; a.sa = b.sa64; a.wpot = b.wpot;
    launch(k_measure<D, N, R, REP>, b.nw_sites, KBLOCK, 0, b.st, a);
  }
  void init(const Bufs& b, InitArgs a, bool links, bool sites) override {
    a.lats = b.lats; a.U = b.U; a.P = b.P;
    const int first = links ? 0 : b.nw_links;
    const int count = (links ? b.nw_links : 0) + (sites ? b.nw_sites : 0);
    if (count == 0) return;
    a.work = b.w_all + first;
    launch(k_init<N, R>, count, KBLOCK, 0, b.st, a);
  }
  void restore(const Bufs& b) override {
    RestoreArgs a;
    a.work = b.w_all; a.lats = b.lats; a.U = b.U; a.Us = b.Us; a.phi = b.phi; a.phis = b.phis; a.N = N; a.d = b.d;
    launch(k_restore<R>, b.nw_links + (b.scalar ? b.nw_sites : 0), KBLOCK, 0, b.st, a);
  }
  void polyakov(const Bufs& b, int tdir) override {
    PolyArgs a;
    a.work = b.w_all + b.nw_links; a.lats = b.lats; a.U = b.U; a.tdir = tdir; a.partials = b.partials;
    k_polyakov<D, N, R><<<b.nw_sites, KBLOCK, 0, b.st>>>(a);
  }
  void loops(const Bufs& b, LoopArgs a) override {
    a.work = b.w_all + b.nw_links; a.lats = b.lats; a.U = b.U; a.partials = b.partials;
    k_loops<D, N, R><<<b.nw_sites, KBLOCK, 0, b.st>>>(a);
  }
  void xfer(const Bufs& b, XferArgs a) override {
    a.lats = b.lats;
    k_xfer<R><<<296, 256, 0, b.st>>>(a);
  }
  void halo(const Bufs& b, HaloArgs a) override {
    a.lats = b.lats;
    const long long total = a.nplane * a.ncomp;
    const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148 * 8);
    if (grid) k_halo<R><<<grid, 256, 0, b.st>>>(a);
  }
};

// Factories, one per (N, precision) translation unit.
EngineBase* make_engine_n2_f64(int D, int rep);
EngineBase* make_engine_n2_f32(int D, int rep);
EngineBase* make_engine_n3_f64(int D, int rep);
EngineBase* make_engine_n3_f32(int D, int rep);

template <int N, typename R>
EngineBase* make_engine_NR(int D, int rep) {
#define GH_MK(DD) \
  switch (rep) { case REP_NONE: return new Engine<DD, N, R, REP_NONE>(); case REP_FUND: return new Engine<DD, N, R, REP_FUND>(); \
    case REP_ADJ: return new Engine<DD, N, R, REP_ADJ>(); case REP_GEN: return new Engine<DD, N, R, REP_GEN>(); default: return nullptr; }
  switch (D) {
    case 2: GH_MK(2)
    case 3: GH_MK(3)
    case 4: GH_MK(4)
    default: return nullptr;
  }
#undef GH_MK
}

}  // namespace ghk
