/* gauge_higgs_b200.h -- C ABI of the B200 molecular-dynamics engine for SU(N)
 * gauge + arbitrary-irrep Higgs Hybrid Monte Carlo.
 *
 * The reference (hlammiv/gauge_higgs) has no C ABI: its hot path is a C++
 * template / virtual interface.  Each entry point below names the reference
 * interface it replaces (paths relative to that project's root).  A host driver
 * keeps its compile-time NDIM/NCOL and its Representation objects and hands the
 * per-step work to these calls.
 *
 * Conventions
 *  - Host arrays use the reference's layouts (array of structures), FP64:
 *      links    U   [site][mu][i][j] complex   (src/core/fields.hpp:12-20)
 *      momenta  P   [site][mu][a]    double    (src/core/fields.hpp:46-57)
 *      vectors  phi [site][k]        complex   (src/core/scalar_field.hpp:15)
 *    complex = two doubles (re, im); site index mixed radix, direction 0 fastest
 *    (src/core/geometry.hpp:20-38).
 *  - Every call returns GH_OK (0) or a negative GH_ERR_* code; no exception
 *    crosses the ABI.  gh_last_error(ctx) gives the message (ctx may be NULL
 *    for errors of gh_ctx_create).  The reference throws std::runtime_error
 *    (e.g. src/rep/rep_general.hpp:58-69) and its driver exits 1
 *    (src/hmc_higgs.cpp:57-59).
 *  - A context owns all device memory and one CUDA stream; calls on one context
 *    are stream ordered and not thread safe; distinct contexts may be used from
 *    distinct threads.  Host pointers are only borrowed for the duration of a
 *    call; calls that return host data synchronise the stream.
 *  - A context may hold several independent lattices ("batch") of one (D, N,
 *    representation) with their own extents, couplings, seeds and trajectory
 *    counters.  Per-lattice calls take `lat` (0-based); `lat = -1` means all.
 */
#ifndef GAUGE_HIGGS_B200_H
#define GAUGE_HIGGS_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GH_OK 0
#define GH_ERR_ARG -1
#define GH_ERR_CUDA -2
#define GH_ERR_REP -3
#define GH_ERR_STATE -4
#define GH_ERR_NONFINITE -5
#define GH_ERR_UNSUPPORTED -6

enum { GH_REP_NONE = 0, GH_REP_FUND = 1, GH_REP_ADJ = 2, GH_REP_GENERAL = 3 };
/* Precision modes.  FP64: everything FP64 (the reference's arithmetic).  FP32_MD:
 * links, momenta, scalar fields and forces stored and computed in FP32; in every
 * drift exp(i eps P), its product with U and the Gram-Schmidt projection back to
 * SU(N) in FP64 (rounded to FP32 once); Hamiltonian sums and Metropolis in FP64.
 * FP32_ALL: as FP32_MD, with the drift's exponential, product and projection in
 * FP32 as well (a faster, non-default variant). */
enum { GH_PREC_FP64 = 0, GH_PREC_FP32_MD = 1, GH_PREC_FP32_ALL = 2 };
enum { GH_LEAPFROG = 0, GH_OMELYAN = 1 };
/* How D(U) of the scalar's representation is applied on the device (gh_rep_path). */
enum { GH_PATH_REGISTER = 0, GH_PATH_TENSOR = 1, GH_PATH_CLOSED_FORM = 2, GH_PATH_PRODUCT = 3, GH_PATH_PAIR = 4 };

/* Representation R of the scalar.  Replaces the Representation<N> object
 * (src/rep/representation.hpp:12-32).  GENERAL carries the host-built tables of
 * GeneralRep<N> (src/rep/rep_general.hpp:36-42): T^a_R = T[a][i][j] and the
 * irrep basis W[l][t] of V^{x n} (Wflat).  For FUND and ADJ the tables are
 * implied (T, W may be NULL). */
typedef struct {
  int kind;          /* GH_REP_* */
  int d;             /* representation dimension d(R) */
  int real;          /* scalar carries d real dof (heatbath imaginary parts zero) */
  int n_boxes;       /* Young boxes n (GENERAL) */
  long dimT;         /* N^n (GENERAL) */
  const double* T;   /* [N*N-1][d][d] complex (GENERAL, required) */
  const double* W;   /* [d][dimT] complex (GENERAL, required) */
} gh_rep_desc;

/* Per-lattice measurement: H and its parts (src/hmc/gauge_higgs_hmc.hpp:105-110),
 * avg_plaquette (src/action/gauge_wilson.hpp:50-65), link_energy and
 * higgs_length (src/action/scalar_higgs.hpp:132-154). */
typedef struct {
  double H, S_g, S_H, kin_P, kin_pi, plaquette, L_link, L_phi;
} gh_obs;

/* One trajectory of one lattice: dH, accept, and the driver's measurements
 * after accept/reject (src/hmc_higgs.cpp:80-87); kappa and beta are the couplings
 * the trajectory ran at (they move between lattices under tempering). */
typedef struct {
  double dH;
  int accepted;
  int traj;
  double plaquette, L_phi, L_link;
  double kappa, beta;
} gh_traj_record;

typedef struct gh_ctx gh_ctx;

/* ---- context ------------------------------------------------------------
 * Replaces construction of GaugeHiggsHMC<D,N>(extents, rep, seed)
 * (src/hmc/gauge_higgs_hmc.hpp:45-50) and GaugeHMC<D,N>(extents, seed)
 * (src/hmc/hmc.hpp:226-227; rep == NULL or kind GH_REP_NONE selects it).
 * L: n_lat * D extents; seeds: n_lat Rng seeds (src/core/rng.hpp:19-22). */
int gh_ctx_create(int D, int N, int n_lat, const int* L, const gh_rep_desc* rep, int precision,
                  const uint64_t* seeds, gh_ctx** out);
int gh_ctx_destroy(gh_ctx* ctx);
const char* gh_last_error(const gh_ctx* ctx);
/* Launch on an external CUDA stream (cudaStream_t passed as void*); NULL restores the own stream. */
int gh_set_stream(gh_ctx* ctx, void* stream);
int gh_sync(gh_ctx* ctx);
int gh_info(const gh_ctx* ctx, int* D, int* N, int* n_lat, int* d, int* rep_kind, int* precision);
/* Device bytes held by the context (fields, scratch, tables). */
int gh_device_bytes(const gh_ctx* ctx, uint64_t* bytes);

/* ---- couplings / integrator (the public members beta, kappa, lambda, tau,
 * nmd, integ, traj_count of GaugeHiggsHMC, src/hmc/gauge_higgs_hmc.hpp:24-42) */
int gh_set_couplings(gh_ctx* ctx, int lat, double beta, double kappa, double lambda);
int gh_get_couplings(gh_ctx* ctx, int lat, double* beta, double* kappa, double* lambda);
int gh_set_integrator(gh_ctx* ctx, int integ, int nmd, double tau);
int gh_set_traj_count(gh_ctx* ctx, int lat, uint64_t traj_count, uint64_t accept_count);
int gh_get_traj_count(gh_ctx* ctx, int lat, uint64_t* traj_count, uint64_t* accept_count,
                      uint64_t* nonfinite_count);

/* ---- fields: AoS host <-> device (the std::vector members U.u, P.p, phi.data,
 * pi.data of src/hmc/gauge_higgs_hmc.hpp:18-20) ---- */
int gh_set_links(gh_ctx* ctx, int lat, const double* U);
int gh_get_links(gh_ctx* ctx, int lat, double* U);
int gh_set_mom(gh_ctx* ctx, int lat, const double* P);
int gh_get_mom(gh_ctx* ctx, int lat, double* P);
int gh_set_phi(gh_ctx* ctx, int lat, const double* phi);
int gh_get_phi(gh_ctx* ctx, int lat, double* phi);
int gh_set_pi(gh_ctx* ctx, int lat, const double* pi);
int gh_get_pi(gh_ctx* ctx, int lat, double* pi);

/* ---- initialisation with the reference's counter-RNG keys ----
 * gh_hot_start:      GaugeField::hot(rng, sigma)            src/core/fields.hpp:25-34
 * gh_cold_start:     GaugeField::cold()                     src/core/fields.hpp:23
 * gh_phi_gaussian:   CVecField::gaussian(rng, stream, rep.real, sigma)  src/core/scalar_field.hpp:40-50
 * gh_phi_cold:       CVecField::cold(c)                     src/core/scalar_field.hpp:34-37
 * gh_mom_refresh:    LinkMom::refresh(rng, stream)          src/core/fields.hpp:59-66
 * gh_refresh_momenta: GaugeHiggsHMC::refresh_momenta (keys 0xC3 / 0xD4 at traj_count)
 *                    src/hmc/gauge_higgs_hmc.hpp:167-173, GaugeHMC 0xA1 src/hmc/hmc.hpp:271-272
 * All act on every lattice with that lattice's seed. */
int gh_hot_start(gh_ctx* ctx, double sigma);
int gh_cold_start(gh_ctx* ctx);
int gh_phi_gaussian(gh_ctx* ctx, uint64_t stream, double sigma);
int gh_phi_cold(gh_ctx* ctx, double c);
int gh_mom_refresh(gh_ctx* ctx, uint64_t stream);
int gh_refresh_momenta(gh_ctx* ctx);

/* ---- forces (FP64 host output, AoS; one lattice) ----
 * gh_gauge_force:       add_gauge_force onto zero           src/action/gauge_wilson.hpp:70-83
 * gh_matter_link_force: add_matter_link_force onto zero     src/action/scalar_higgs.hpp:113-128
 *                       (uses Representation::hop_link_g, src/rep/representation.hpp:36-46)
 * gh_scalar_force:      scalar_force                        src/action/scalar_higgs.hpp:71-108
 *                       (uses Representation::rotate / rotate_dag, :28-32) */
int gh_gauge_force(gh_ctx* ctx, int lat, double* F);
int gh_matter_link_force(gh_ctx* ctx, int lat, double* F);
int gh_scalar_force(gh_ctx* ctx, int lat, double* Fphi);

/* ---- integrator steps (all lattices) ----
 * gh_kick:      GaugeHiggsHMC::kick(eps) / GaugeHMC::kick   src/hmc/gauge_higgs_hmc.hpp:112-134, src/hmc/hmc.hpp:35-41
 * gh_drift:     ::drift(eps)                                 src/hmc/gauge_higgs_hmc.hpp:136-147, src/hmc/hmc.hpp:44-52
 * gh_md_evolve: ::md_evolve() with the set integrator        src/hmc/gauge_higgs_hmc.hpp:149-165
 * gh_reunitarize: GaugeField::reunitarize_all()             src/core/fields.hpp:36 */
int gh_kick(gh_ctx* ctx, double eps);
int gh_drift(gh_ctx* ctx, double eps);
int gh_md_evolve(gh_ctx* ctx);
int gh_reunitarize(gh_ctx* ctx);

/* ---- measurements (one lattice, or lat = -1 with n_lat entries) ----
 * gh_measure: hamiltonian() and its parts, avg_plaquette, link_energy, higgs_length.
 * gh_polyakov: polyakov_loop(U, tdir)                       src/measure/observables.hpp:17-34 */
int gh_measure(gh_ctx* ctx, int lat, gh_obs* out);
int gh_polyakov(gh_ctx* ctx, int lat, int tdir, double* out);

/* ---- trajectories ----
 * gh_trajectory: GaugeHiggsHMC::trajectory() / GaugeHMC::trajectory() on every
 * lattice (src/hmc/gauge_higgs_hmc.hpp:175-192, src/hmc/hmc.hpp:270-288):
 * refresh, save, H_i, md_evolve, reunitarize (FP64 mode), H_f, Metropolis,
 * restore on reject -- entirely on the device (captured once as a CUDA graph).
 * dH, accepted: n_lat entries each (may be NULL).  NaN/Inf dH is rejected, as
 * in the reference, and counted (gh_get_traj_count). */
int gh_trajectory(gh_ctx* ctx, double* dH, int* accepted);
/* ntraj trajectories back to back without host synchronisation in between;
 * records: ntraj * n_lat entries [t][lat] (may be NULL). */
int gh_run_trajectories(gh_ctx* ctx, int ntraj, gh_traj_record* records);
/* Enqueue ntraj trajectories on the context's stream and return without
 * synchronising (records stay in the device ring of the last 1024 trajectories
 * per lattice; read them with gh_read_records after gh_sync). */
int gh_enqueue_trajectories(gh_ctx* ctx, int ntraj);
/* The records of the last ntraj (<= 1024) trajectories: ntraj * n_lat entries [t][lat]. */
int gh_read_records(gh_ctx* ctx, int ntraj, gh_traj_record* records);
/* Host-resident fields (single lattice): upload U and phi, run one trajectory,
 * download U, phi and the record.  The drop-in for a driver that keeps the
 * fields in host memory like the reference's GaugeField / CVecField.  A rejected
 * trajectory restores the state that was passed in, so U and phi are then left
 * untouched (in FP32-MD mode they keep the caller's FP64 values rather than their
 * FP32 roundings, which the next upload reproduces). */
int gh_trajectory_host(gh_ctx* ctx, double* U, double* phi, gh_traj_record* rec);
/* ---- kick tiles and the autotuner ----
 * The kick kernel gives each 128-thread block a 4-D tile of sites (power-of-two
 * extents per direction); the tile decides how many neighbour links a block
 * reuses from L1.  gh_autotune times every admissible tile on each group of
 * equal-extent lattices (reps zero-step kicks each) and keeps the fastest;
 * best_ms (may be NULL): sum over groups of the best kick time.  Results do not
 * depend on the tile (every link and site is computed the same way). */
int gh_autotune(gh_ctx* ctx, int reps, double* best_ms);
int gh_set_tile(gh_ctx* ctx, int lat, const int* tile);
int gh_get_tile(gh_ctx* ctx, int lat, int* tile);
/* Use (1, default) or bypass (0) the captured trajectory graph. */
int gh_use_graph(gh_ctx* ctx, int enable);

/* ---- replica tempering across the lattices of a batch ----
 * ReplicaTempering::step / attempt_swap (src/hmc/replica_tempering.hpp:157-205):
 * after every trajectory, adjacent pairs of the coupling ladder among lattices
 * with equal extents propose a configuration exchange with
 * Delta = (c_i - c_j)(B_i - B_j), coin uniform(key(0x57A9, ++counter)) on
 * swap_seed; even pass then odd pass.
 *   mode 2: beta, B = n_plaq (plaquette - 1)  -- the reference's tempering;
 *   mode 1: kappa, B = sum_{x,mu} 2 Re phi_x^dag D(U) phi_{x+mu} (no counterpart
 *           in the reference; same mechanism with kappa tempered);
 *   mode 0: off.
 * The exchange swaps the coupling labels on the device (equivalent to swapping
 * U and phi); the couplings each trajectory ran at are in its record. */
int gh_temper_enable(gh_ctx* ctx, int mode, uint64_t swap_seed);
/* One swap pass after every n_sweep trajectories (ReplicaTempering::n_sweep,
 * src/hmc/replica_tempering.hpp:157-167; default 1). */
int gh_temper_interval(gh_ctx* ctx, int n_sweep);
/* attempts/accepts: per adjacent pair in ladder order (n_lat - 1 entries);
 * kappa_of_lat: current kappa of each lattice (see gh_get_couplings for beta). */
int gh_temper_stats(gh_ctx* ctx, uint64_t* attempts, uint64_t* accepts, double* kappa_of_lat);

/* ---- coupling-scan surrogate: an ensemble of MLPs trained on the GPU ----
 * No counterpart in the reference (its coupling scans are uniform grids of
 * independent runs, validate_su2higgs.sh / scripts/).  widths: n_layers + 1
 * layer widths (input first); SiLU between layers; FP32 weights and Adam state,
 * BF16 hidden activations, FP32 accumulation; loss = mean squared error.
 * All members see the same minibatches; they differ by initialisation (seed).
 * Arrays are row-major FP32: x [n][widths[0]], y and outputs [n][widths[n_layers]],
 * params / grads [member][P] with P = gh_mlp_num_params.  Errors:
 * gh_mlp_last_error(). */
typedef struct gh_mlp gh_mlp;
int gh_mlp_create(int n_members, const int* widths, int n_layers, uint64_t seed, gh_mlp** out);
int gh_mlp_destroy(gh_mlp* net);
int gh_mlp_num_params(const gh_mlp* net, long* per_member);
int gh_mlp_get_params(gh_mlp* net, float* params);
int gh_mlp_set_params(gh_mlp* net, const float* params);
/* forward + backward of one batch: grads (may be NULL) and per-member loss (may be NULL) */
int gh_mlp_grad(gh_mlp* net, const float* x, const float* y, int n, float* grads, float* loss);
/* one Adam update (beta1 0.9, beta2 0.999, eps 1e-8) from the last gh_mlp_grad */
int gh_mlp_adam_step(gh_mlp* net, float lr);
/* epochs of shuffled minibatches; loss: per-member mean loss of the last epoch */
int gh_mlp_train(gh_mlp* net, const float* x, const float* y, int n, int epochs, int batch, float lr, uint64_t seed,
                 float* loss);
/* per_member [M][n][n_out], ensemble mean and variance [n][n_out]; any may be NULL */
int gh_mlp_predict(gh_mlp* net, const float* x, int n, float* per_member, float* mean, float* var);
const char* gh_mlp_last_error(void);

/* ---- allocation-free plaquette reduction ----
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory where they measure: a driver recording its own work into a CUDA graph
 * (cudaMalloc is not allowed during stream capture and cudaFree synchronises the
 * device) or a program whose device memory belongs to another framework's arena.
 * U_dev: links in device memory, the reference's AoS layout [site][mu][i][j]
 * complex FP64; out_dev (device): out[0] = sum of Re Tr U_pl, out[1] = average
 * plaquette (as gh_measure's plaquette).  Launches on `stream` (may be NULL) and
 * returns without synchronising.  Allocates nothing: per-block partial sums live
 * in a file-scope __device__ array sized for GH_NOALLOC_MAX_SITES sites (64 KiB,
 * held by every device that loads the library until exit); larger lattices are
 * rejected with GH_ERR_ARG.  All calls on a device share that array: calls that
 * overlap on the GPU race.  The first call on a device looks up the array's
 * device address with that device current: make it before any stream capture.
 * That address is cached for the life of the process and belongs to the device's
 * primary context: after cudaDeviceReset on a device, do not call this entry point
 * on that device again.  U_dev must be 16-byte aligned and out_dev 8-byte aligned
 * (refused with GH_ERR_ARG otherwise, before any launch).
 * Errors: message in gh_noalloc_last_error(). */
#define GH_NOALLOC_MAX_SITES (8192 * 128)
int gh_plaquette_noalloc(int D, int N, const int* L, const double* U_dev, double* out_dev, void* stream);
const char* gh_noalloc_last_error(void);

/* ---- domain decomposition (src/mpi/gauge_mpi.hpp:26-139, src/mpi/higgs_mpi.hpp:150-226) ----
 * A lattice too large for one GPU is split over a process grid; each rank's context
 * holds its subdomain padded by a width-1 halo in every split direction (local
 * extent = interior + 2) and the whole extent in the others.  The reference's
 * DistLattice / DistGaugeHiggsHMC with MPI_Sendrecv halos; here the host moves the
 * halo planes (NCCL or any transport) between these calls:
 * gh_set_domain: G the global extents; per direction lo = 0, hi = L (not split) or
 *   lo = 1, hi = L - 1 (split); goff the global coordinate of the local coordinate lo.
 *   Kernels then act on the interior only, the counter RNG is keyed on the global site
 *   index (hot start, phi init and heatbaths equal the whole lattice's draws), and
 *   gh_measure's sums cover the interior (normalised by its volume: H, S_g, S_H and
 *   the kinetic terms add over ranks, the averages combine weighted by volume).  The
 *   device Metropolis, tempering and loop observables are refused on a subdomain: the
 *   host takes the global dH and the accept decision (the same key on every rank).
 * gh_halo_count: complex elements of one plane x_nu = const of field 0 (links, D N^2
 *   per site) or 1 (phi, d per site), whole padded plane.
 * gh_halo_pack / gh_halo_unpack: gather / scatter that plane at x_nu = layer to / from
 *   a device buffer (16-byte aligned, field precision, [component][plane site] with
 *   the plane's sites in mixed radix over the other directions, direction 0 fastest).
 *   Exchanging the split directions in order with whole planes also fills edges and
 *   corners (the reference's sequential halo_exchange_raw).
 * gh_save_fields / gh_restore_fields: copy U and phi to / from the context's
 *   trajectory save buffers (the reject branch of trajectory()). */
int gh_set_domain(gh_ctx* ctx, int lat, const int* G, const int* lo, const int* hi, const int* goff);
int gh_halo_count(gh_ctx* ctx, int lat, int field, int nu, long long* n_complex);
int gh_halo_pack(gh_ctx* ctx, int lat, int field, int nu, int layer, void* buf);
int gh_halo_unpack(gh_ctx* ctx, int lat, int field, int nu, int layer, const void* buf);
int gh_save_fields(gh_ctx* ctx);
int gh_restore_fields(gh_ctx* ctx);

/* ---- the counter RNG on the host (src/core/rng.hpp:11-46) ----
 * Same bits as the device kernels: key and uniform are integer exact; gauss is the
 * correctly rounded evaluation of sqrt(-2 log u1) cos(2 pi u2).  Pure functions
 * (they return the value, not a status). */
uint64_t gh_rng_key(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e);
double gh_rng_uniform(uint64_t seed, uint64_t key);
double gh_rng_gauss(uint64_t seed, uint64_t key);

/* ---- general irreps: host-side construction of the GeneralRep tables ----
 * The Young-symmetriser basis of src/rep/rep_general.hpp:54-84,338-411, so a
 * driver without the reference headers can still form gh_rep_desc.
 * rows: Young diagram row lengths. */
int gh_rep_general_info(int N, const int* rows, int nrows, int* d, int* n_boxes, long* dimT);
int gh_rep_general_build(int N, const int* rows, int nrows, double* T, double* W);

/* D(U) of a general irrep as a piece of a product of adjoints (host; no GPU).
 * For an irrep of n = K N boxes (K = 1, 2; N = 2, 3) the adjoint's K-fold tensor
 * product holds R: with the fixed isometric intertwiner Q (built from W by the
 * Levi-Civita embedding of the adjoint into V^(x)N, checked by Schur's lemma and
 * against the tensor construction), D_R(U) = Q^dag D_adj(U)^(x)K Q, where
 * D_adj(U)_ab = 2 Re Tr(T^a U T^b U^dag).  The same matrix as the reference's
 * rep_matrix (src/rep/rep_general.hpp:122-131) to rounding.  U: N x N complex;
 * D: d x d complex; K (may be NULL) receives the number of adjoint factors.
 * GH_ERR_REP (message in gh_last_error(NULL)) when the irrep is not reached this way. */
int gh_rep_product_matrix(int N, const gh_rep_desc* rep, const double* U, double* D, int* K);

/* ---- general irreps: how D(U) is applied ----
 * Fundamental and adjoint: in registers (GH_PATH_REGISTER).  A general irrep uses
 * the exact tensor construction <W_k| U^(x)n |W_l> (GH_PATH_TENSOR;
 * src/rep/rep_general.hpp:122-131,184-220), except for a single-row Young diagram
 * {n}, whose basis vectors are symmetrised multisets: there the context builds D(U)
 * per link in closed form, a sum of monomials in the entries of U
 * (GH_PATH_CLOSED_FORM), when that takes fewer operations than the tensor path or
 * when the N^n tensor does not fit in shared memory.  It replaces the reference's
 * GeneralRep fast path exp(i w.T_R) (src/rep/rep_general.hpp:94-112,165-179),
 * which that code enables for the same large single-row irreps (SU(2){12}: d = 13,
 * N^n = 4096); the closed form is the tensor matrix itself, not an approximation
 * of it, and the context checks it against the tensor construction on two test
 * links before using it.
 * Irreps of n = K N boxes inside the K-fold adjoint product (K = 1, 2; SU(3): the
 * octet {2,1}, the 27-plet {4,2}, the 10bar {3,3}) take GH_PATH_PRODUCT instead, when
 * the context finds and checks the intertwiner (gh_rep_product_matrix): a lift by a
 * fixed A x d matrix shared by 32 links per block, the adjoint matrix of each link
 * applied K times, a projection -- the reference's tensor matrix to rounding.  The
 * multi-invariant potential's per-site term is computed on the tensor / closed-form
 * path, so contexts with that potential use it for their link work.
 * Two-slot irreps outside that product (n = 2: SU(3) sextet {2}, antitriplet {1,1})
 * take GH_PATH_PAIR: one thread per link, phi lifted by W to an N x N matrix Phi,
 * D(U) phi the projection of U Phi U^T, the matter force from U Phi_y U^T Phi_x^dag.
 * gh_rep_path: the path a context uses.
 * gh_set_rep_path: switch between GH_PATH_PRODUCT or GH_PATH_PAIR (when available) and
 *   the path the context would use without them; GH_ERR_ARG for any other path.
 * gh_sympow_matrix: host-only evaluation of the closed form D(U) (U: N x N complex
 *   row-major; D: d x d complex) and the number of terms; GH_ERR_REP when the
 *   irrep has no closed form (message through gh_last_error(NULL)). */
int gh_rep_path(const gh_ctx* ctx, int* path);
int gh_set_rep_path(gh_ctx* ctx, int path);
int gh_sympow_matrix(int N, const gh_rep_desc* rep, const double* U, double* D, long* n_terms);

/* ---- multi-invariant onsite potential ----
 * V[phi] = -mu2 phi^dag phi + sum_c f_c Tr(M^dag P_c M), M = phi phi^dag, P_c the
 * projector onto channel c of R (x) Rbar (an eigenspace of the adjoint Casimir
 * superoperator sum_a [T^a_R, [T^a_R, .]]).  Replaces CasimirChannels<N>
 * (src/action/scalar_invariants.hpp:19-27, channel search :152-187) and
 * MultiInvariantPotential<N> plugged into GaugeHiggsHMC::potential
 * (scalar_invariants.hpp:190-206, src/hmc/gauge_higgs_hmc.hpp:25-27).
 * At most 32 components (d <= 32).
 *
 * gh_casimir_channels: the channels' Casimir values C2, ascending -- the order
 *   in which couplings f_c are given (the reference's CasimirChannels::lambda).
 *   rep->kind FUND / ADJ need only d; GENERAL needs rep->T.  Host only.
 * gh_multi_superop: the combined superoperator A = sum_c 2 f_c P_c that the
 *   device applies, [(p*d+q)*d*d + (i*d+j)] complex (re, im), as
 *   MultiInvariantPotential::Asuper (scalar_invariants.hpp:100-118).  Host only.
 *   The two host-only calls report errors through gh_last_error(NULL).
 * gh_set_potential_multi: every lattice of the context uses V from now on (the
 *   quartic coupling lambda is ignored); n_channels must equal the number of
 *   channels.  gh_set_potential_quartic returns to phi^dag phi + lambda
 *   (phi^dag phi - 1)^2 (QuarticPotential, src/action/scalar_higgs.hpp:25-40), the
 *   default.  Both invalidate a captured trajectory graph. */
int gh_casimir_channels(int N, const gh_rep_desc* rep, double* c2, int cap, int* n_channels);
int gh_multi_superop(int N, const gh_rep_desc* rep, int n_channels, const double* f, double* A);
int gh_set_potential_multi(gh_ctx* ctx, int n_channels, const double* f, double mu2);
int gh_set_potential_quartic(gh_ctx* ctx);

/* ---- loops traced in a probe irrep (src/measure/observables.hpp:36-101) ----
 * gh_wilson_loop: <(1/d_R) Re Tr D^(R)(W_loop)> over sites and planes mu < nu of
 *   the Ra x Rb rectangle (wilson_rect :36-46; wilson_loop_fund :48-60 for rows
 *   = NULL, wilson_loop_rep :62-79 otherwise).
 * gh_polyakov_rep: <(1/d_R) Re Tr D^(R)(prod_t U_tdir)> (polyakov_loop_rep :81-101);
 *   tdir < 0 selects D-1.
 * The probe irrep R is given by its Young rows (rows[0] >= rows[1] >= ... >= 1,
 * at most N rows, rows[0] + nrows <= 25; NULL: the fundamental).  The trace is the
 * irrep's character, the same number as the trace of the reference's rep_matrix.
 * FP64 on the device in both precision modes; one value per lattice into out
 * (lat = -1: all lattices). */
int gh_wilson_loop(gh_ctx* ctx, int lat, int Ra, int Rb, const int* rows, int nrows, double* out);
int gh_polyakov_rep(gh_ctx* ctx, int lat, int tdir, const int* rows, int nrows, double* out);

/* ---- frozen-length scalar, |phi_x| = 1 ----
 * Replaces GaugeHiggsHMC::frozen_phi and normalize_phi (src/hmc/gauge_higgs_hmc.hpp:
 * 38-40,61-103): with it on, momenta are projected onto the tangent space of each
 * site's unit sphere after every refresh and kick, and the scalar drift is the exact
 * great-circle flow.  gh_normalize_phi puts every site on the sphere (call once
 * after the initial field, as the reference drivers do).  Both stream-ordered;
 * gh_set_frozen_phi invalidates a captured trajectory graph. */
int gh_set_frozen_phi(gh_ctx* ctx, int on);
int gh_normalize_phi(gh_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
