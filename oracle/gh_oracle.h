/* gh_oracle.h -- CPU restatement of the gauge+Higgs HMC molecular-dynamics path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: a plain-C, FP64,
 * single-threaded restatement of the reference algorithm (hlammiv/gauge_higgs,
 * header-only C++ under src/).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it, and only as the checker.  The
 * product (gauge_higgs_b200) never calls it.
 *
 * Layouts follow the reference exactly (array-of-structures):
 *   U   [site][mu][i][j]  complex  (src/core/fields.hpp:12-20)
 *   P   [site][mu][a]     double   (src/core/fields.hpp:46-57)
 *   phi [site][k]         complex  (src/core/scalar_field.hpp:15)
 * complex = two doubles (re, im).  Site index is mixed-radix with direction 0
 * fastest (src/core/geometry.hpp:20-38).
 *
 * Pinned against: golden vectors produced by the reference itself
 * (tests/golden/make_golden.py drives oracle/_ref, a build of the unmodified
 * reference headers) and live comparison with oracle/_ref where present.
 */
#ifndef GH_ORACLE_H
#define GH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GHO_MAXD 4
#define GHO_MAXN 4

enum { GHO_REP_NONE = 0, GHO_REP_FUND = 1, GHO_REP_ADJ = 2, GHO_REP_GENERAL = 3 };
enum { GHO_LEAPFROG = 0, GHO_OMELYAN = 1 };

typedef struct {
  int D, N;
  int L[GHO_MAXD];
  int64_t vol;
  int64_t stride[GHO_MAXD];
} gho_lattice;

typedef struct {
  int kind;          /* GHO_REP_* */
  int N, d, real;
  int n;             /* Young boxes (general) */
  long dimT;         /* N^n (general) */
  double* T;         /* [N^2-1][d][d] complex, owned */
  double* W;         /* [d][dimT] complex, owned (general only) */
} gho_rep;

/* ---- lattice ---- */
void    gho_lattice_init(gho_lattice* lat, int D, int N, const int* L);
int64_t gho_fwd(const gho_lattice* lat, int64_t s, int mu);
int64_t gho_bwd(const gho_lattice* lat, int64_t s, int mu);

/* ---- RNG (src/core/rng.hpp) ---- */
uint64_t gho_splitmix64(uint64_t x);
uint64_t gho_key(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e);
double   gho_uniform(uint64_t seed, uint64_t k);
double   gho_gauss(uint64_t seed, uint64_t k);

/* ---- group / algebra (src/group/algebra.hpp, src/group/sun.hpp) ---- */
void gho_generators(int N, double* T /* [N^2-1][N][N] complex */);
void gho_structure_constants(int N, double* f /* [ng][ng][ng] */);
void gho_alg_to_mat(int N, const double* v, double* M);
void gho_expi(int N, const double* H, double* U);
void gho_reunitarize(int N, double* U);

/* ---- representations (src/rep/) ---- */
int  gho_rep_init(gho_rep* r, int kind, int N, int d, int real, int n, long dimT,
                  const double* T, const double* W);
void gho_rep_free(gho_rep* r);
void gho_rep_matrix(const gho_rep* r, const double* U, double* Dm /* d x d complex */);
void gho_rep_rotate(const gho_rep* r, const double* U, const double* phi, double* out, int dag);
void gho_rep_hop_link_g(const gho_rep* r, const double* U, const double* phix,
                        const double* phiy, double* g);

/* ---- field initialisation ---- */
void gho_hot_start(const gho_lattice* lat, uint64_t seed, double sigma, double* U);
void gho_cold_start(const gho_lattice* lat, double* U);
void gho_phi_gaussian(const gho_lattice* lat, int d, uint64_t seed, uint64_t stream,
                      int real, double sigma, double* phi);
void gho_mom_refresh(const gho_lattice* lat, uint64_t seed, uint64_t stream, double* P);

/* ---- actions, forces, observables ---- */
double gho_gauge_action(const gho_lattice* lat, const double* U, double beta);
double gho_avg_plaquette(const gho_lattice* lat, const double* U);
void   gho_add_gauge_force(const gho_lattice* lat, const double* U, double beta, double* F);
double gho_scalar_action(const gho_lattice* lat, const gho_rep* r, const double* U,
                         const double* phi, double kappa, double lambda);
void   gho_scalar_force(const gho_lattice* lat, const gho_rep* r, const double* U,
                        const double* phi, double kappa, double lambda, double* Fphi);
void   gho_add_matter_link_force(const gho_lattice* lat, const gho_rep* r, const double* U,
                                 const double* phi, double kappa, double* F);
double gho_link_energy(const gho_lattice* lat, const gho_rep* r, const double* U, const double* phi);
/* multi-invariant onsite potential from its channel superoperator A [(d^2) x (d^2)] complex */
void   gho_multi_potential(int d, const double* A, double mu2, const double* phi, double* value, double* dV);
double gho_scalar_action_multi(const gho_lattice* lat, const gho_rep* r, const double* U,
                               const double* phi, double kappa, const double* A, double mu2);
void   gho_scalar_force_multi(const gho_lattice* lat, const gho_rep* r, const double* U,
                              const double* phi, double kappa, const double* A, double mu2, double* Fphi);
double gho_higgs_length(const gho_lattice* lat, int d, const double* phi);
double gho_polyakov(const gho_lattice* lat, const double* U, int tdir);
double gho_kinetic_mom(const gho_lattice* lat, const double* P);
double gho_kinetic_vec(const gho_lattice* lat, int d, const double* pi);

/* ---- HMC (src/hmc/gauge_higgs_hmc.hpp, src/hmc/hmc.hpp) ----
 * r == NULL (or kind NONE) selects the pure-gauge engine GaugeHMC. */
typedef struct {
  gho_lattice lat;
  const gho_rep* rep;
  uint64_t seed;
  double beta, kappa, lambda, tau;
  int nmd, integ, reunit_each_traj;
  uint64_t traj_count, accept_count;
  double last_dH;
  double *U, *P, *phi, *pi;   /* owned */
} gho_hmc;

int    gho_hmc_init(gho_hmc* h, int D, int N, const int* L, const gho_rep* r, uint64_t seed);
void   gho_hmc_free(gho_hmc* h);
double gho_hmc_hamiltonian(const gho_hmc* h);
void   gho_hmc_kick(gho_hmc* h, double eps);
void   gho_hmc_drift(gho_hmc* h, double eps);
void   gho_hmc_md_evolve(gho_hmc* h);
void   gho_hmc_refresh_momenta(gho_hmc* h);
void   gho_hmc_reunitarize_all(gho_hmc* h);
int    gho_hmc_trajectory(gho_hmc* h);

#ifdef __cplusplus
}
#endif
#endif
