/*
 * lym.h -- C ABI of the B200 (sm_100a) implementation of the TfLeonardYM
 * Wilson-fermion / SU(N) gauge hot path.
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 *  - Device buffers are plain CUDA device pointers in the reference's own
 *    layouts (emanueleusai/TfLeonardYM):
 *        spinor  complex128 (ns, N, V)       dirac.py:458-523
 *        gauge   complex128 (nd, N, N, V)    lattice.py:7 (Configuration)
 *        force / momenta  same as gauge      hmc.py:59-96, gauge_action.py:13-24
 *    with the site index lexicographic, LAST coordinate fastest
 *    (lattice.py:107-114).  complex128 = two interleaved doubles.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *    Work is enqueued on it; calls that return host scalars synchronise it.
 *  - Every function returns an lym_status; lym_last_error() gives the text
 *    of the last failure on the calling thread.
 *  - The boundary condition is the reference's "factor on the last time
 *    slice of the last direction's links" (boundary_conditions.py:10-46),
 *    given as (bc_re, bc_im); (1, 0) is periodic, (-1, 0) antiperiodic.
 *  - Nothing here allocates device memory except the *_create functions and
 *    solver calls, which cache their workspaces in the object they belong to.
 */
#ifndef LYM_H
#define LYM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum lym_status {
  LYM_OK = 0,
  LYM_ERR_BAD_ARG = 1,       /* null pointer, bad size or enum value               */
  LYM_ERR_BAD_SHAPE = 2,     /* mirrors algebra_utils.py:6-7 RuntimeError           */
  LYM_ERR_UNSUPPORTED = 3,   /* mirrors dirac.py:299-300 (nd without fermions), etc */
  LYM_ERR_NOT_CONVERGED = 4, /* solver hit max steps; last iterate returned,
                                as dirac_solver.py:52-53,109-110 do                */
  LYM_ERR_CUDA = 5,          /* CUDA runtime error (text in lym_last_error)         */
  LYM_ERR_OOM = 6,           /* device allocation failed                            */
  LYM_ERR_REJECTED = 7,      /* serving admission refused (HBM budget)              */
  LYM_ERR_TIMEOUT = 8        /* a bounded device wait ran out                       */
} lym_status;

typedef enum lym_precision {
  LYM_PREC_F64 = 0,
  LYM_PREC_F32 = 1,
  LYM_PREC_F16 = 2, /* norm-scaled half spinors, FP32 arithmetic */
  LYM_PREC_BF16 = 3 /* norm-scaled bfloat16 spinors, FP32 arithmetic */
} lym_precision;

/* ------------------------------------------------------------------ */
/* library                                                             */
/* ------------------------------------------------------------------ */
int lym_version(void);
const char* lym_last_error(void);
const char* lym_status_string(int status);

/* ------------------------------------------------------------------ */
/* lattice runtime (host, no GPU needed)                               */
/* ------------------------------------------------------------------ */

/* Neighbour tables sup/sdn and coordinates, each int64 (nd, V), bit-exact
 * with lattice.py:86-120 (mth_lookup_tables). */
int lym_lookup_tables(int nd, const int64_t* dims, int64_t* sup, int64_t* sdn, int64_t* coords);

/* complex128 (V,) field: factor where x_{nd-1} = L_{nd-1}-1, else 1
 * (boundary_conditions.py:10-20, set_antiperiodic_field_in_t_direction). */
int lym_antiperiodic_field(int nd, const int64_t* dims, double factor_re, double factor_im,
                           double* field);

/* ------------------------------------------------------------------ */
/* lattice object on the current device                                */
/* ------------------------------------------------------------------ */
typedef struct lym_lattice lym_lattice;

/* Uploads int32 neighbour tables (lattice.py:86-120) and, when every extent
 * is even, the even-odd maps (builder-defined).  Replaces the per-process
 * translate.set_translate(False, geometry, grid) binding (translate.py:9-36). */
int lym_lattice_create(int nd, const int64_t* dims, lym_lattice** out);
int lym_lattice_destroy(lym_lattice* lat);
/* int64 device copies of sup/sdn (nd, V) for bit-exact checking. */
int lym_lattice_tables_device(const lym_lattice* lat, int64_t* sup_dev, int64_t* sdn_dev, void* stream);

/* ------------------------------------------------------------------ */
/* Wilson Dirac operator, reference layout, FP64                       */
/* ------------------------------------------------------------------ */

/* out = D in, or Q in = gamma_d D in when hermitian != 0, with
 * D psi = psi + kappa sum_mu [U_mu(x)(1-g_mu)psi(x+mu) + U_mu(x-mu)^dag(1+g_mu)psi(x-mu)].
 * Replaces DiracWilsonOperator.multiply_in_fundamental_representation /
 * simple_multiply_in_fundamental_representation + apply_hermiticity
 * (dirac.py:458-523, 649-662).  nd in {2, 4}, the reference's fermion
 * dimensions; any other nd returns LYM_ERR_UNSUPPORTED with the reference's
 * message (dirac.py:299-300).  `in` and `out` must not alias. */
int lym_wilson_apply(const lym_lattice* lat, int nc, double kappa, int hermitian,
                     double bc_re, double bc_im, const void* gauge,
                     const void* in, void* out, void* stream);

/* Batched form: nvec spinors stored back to back (nvec, ns, N, V). */
int lym_wilson_apply_batch(const lym_lattice* lat, int nc, double kappa, int hermitian,
                           double bc_re, double bc_im, const void* gauge, int nvec,
                           const void* in, void* out, void* stream);

/* ------------------------------------------------------------------ */
/* vector algebra on complex128 arrays of n elements                   */
/* ------------------------------------------------------------------ */

/* result[0..1] (host) = sum conj(a) b  (algebra_utils.py:5-11 dot + lattice.py:375 global_sum).
 * Synchronises `stream`. */
int lym_cdot(int64_t n, const void* a, const void* b, double* result, void* stream);
/* y = a*x + b*y with complex a, b (re, im pairs). */
int lym_caxpby(int64_t n, const double* a, const void* x, const double* b, void* y, void* stream);

/* results[2i], results[2i+1] (host) = sum conj(a_i) b_i for nvec vector pairs of n
 * complex128 elements each, stored back to back (nvec, n).  No counterpart in the
 * reference: an entry point for callers that cannot allocate device memory, such as
 * code running under a framework's pooling allocator (which owns the device heap and
 * would not see a cudaMalloc) or under a fixed device-memory budget.  It allocates
 * nothing: its reduction scratch is a static device array of about 263 KB that every
 * GPU loading the library keeps until exit, which limits nvec to 64 (larger nvec
 * returns LYM_ERR_BAD_ARG).  The first call on each device also looks up the array's
 * device address (cudaGetSymbolAddress, once per device, cached for later calls);
 * make that first call before any stream capture.  All calls share the array, so
 * calls that overlap on the GPU (other streams, other host threads) race.
 * Synchronises `stream`. */
int lym_cdot_batch_noalloc(int nvec, int64_t n, const void* a, const void* b, double* results, void* stream);

/* ------------------------------------------------------------------ */
/* gauge objects for the solvers                                       */
/* ------------------------------------------------------------------ */
typedef struct lym_gauge lym_gauge;

/* Converts a reference-layout gauge field (with the boundary factor) into
 * the solver's even-odd layouts: FP64 18-real with the boundary factor
 * folded in, plus the sloppy precisions in `prec_mask` (bit p = lym_precision
 * p) with 12-real SU(3) / 4-real SU(2) reconstruction and the boundary factor
 * applied at load time.  Replaces DiracWilsonOperator.set_gauge_configuration
 * (dirac.py:351-378).  Needs every extent even.  The lattice must outlive it. */
int lym_gauge_create(const lym_lattice* lat, int nc, const void* gauge, double bc_re, double bc_im,
                     unsigned prec_mask, void* stream, lym_gauge** out);
/* Refreshes the internal copies from a new reference-layout field (same lattice). */
int lym_gauge_update(lym_gauge* g, const void* gauge, void* stream);
int lym_gauge_destroy(lym_gauge* g);

typedef struct lym_solver_params {
  double tol;        /* target true relative residual |b - D x| / |b|          */
  int max_iter;      /* iteration cap (counted in operator applications of M^dag M) */
  int precision;     /* lym_precision of the inner (sloppy) iterations          */
  double delta;      /* reliable-update trigger: sloppy |r| fell by this factor  */
  int hermitian;     /* 1: system is Q x = b with Q = gamma_d D                  */
  int chunk;         /* iterations per CUDA graph launch (0 = default)           */
  int rhs_per_thread;/* at most this many right-hand sides per hop-kernel thread
                        (1, 2 or 4; the largest available one is used); 0 = autotune */
  int compressed_links; /* with a forced tile (rhs_per_thread > 0): 1 = the N-1-row
                        links (when the links are SU(N)), 0 = full links */
  int mixed_fma;     /* with a forced tile and FP16 (full links): 0 = FP32 arithmetic on
                        converted values; 1 = half spinor in FP16, U h through f16 x f16 + f32
                        FMAs; 2 = the tensor-core hop (4D SU(3), nrhs a multiple of 16, with
                        rhs_per_thread = 16): projected FP16 half spinors x FP16 links on
                        mma.sync with FP32 accumulation, 8 sites x 16 rhs per CTA; 3 = the
                        colour contraction of each direction in packed FP16 FMAs (half2),
                        accumulated over directions in FP32 (rhs_per_thread = 1; only when
                        asked for: the autotuner does not pick it); 4 = form 1 with the
                        neighbours' indices from coordinate arithmetic instead of the
                        neighbour table; 5 = form 4 with the +-t neighbours' spinors by warp
                        shuffle (when Lt/2 is a power of two <= 32 and V/2 a multiple of 32) */
  double switch_residual; /* lym_multishift_solve_eo with a reduced inner precision: the
                        iterations run in FP64 until the true relative residual of the
                        smallest shift is below this, then in the inner precision
                        (0 = 1e-4 FP32, 1e-6 FP16, 1e-7 BF16; negative = from the start) */
} lym_solver_params;

typedef struct lym_solver_report {
  int status;            /* lym_status of this right-hand side                  */
  int iterations;        /* inner iterations                                     */
  int reliable_updates;  /* FP64 residual recomputations                         */
  double true_residual;  /* FP64 |b - D x| / |b| of the returned x               */
  int64_t kernel_launches; /* lym kernels the whole call launched (graph nodes included) */
  int rhs_per_thread;    /* right-hand sides per thread the autotuner picked for the hop kernels
                            (the tensor-core hop: right-hand sides per CTA, 16) */
  int compressed_links;  /* 1: the hop kernels read the N-1-row sloppy links, 0: full links */
  int mixed_fma;         /* 1: the hop kernels ran the mixed-precision FP16 form; 2: the tensor-core
                            form; 3: the packed-half form; 4: form 1 with arithmetic neighbours;
                            5: form 4 with the t neighbours by warp shuffle */
} lym_solver_report;

/* Solve D x_i = b_i (or Q x_i = b_i) for nrhs right-hand sides stored back to
 * back in reference layout (nrhs, ns, N, V), by even-odd Schur preconditioning
 * (M = 1 - kappa^2 H_eo H_oe, builder-defined: the reference has no even-odd)
 * and CG on M^dag M with FP64 reliable updates.  The reference's own solvers
 * (dirac_solver.py) reach the same x up to tolerance.  `reports` has nrhs
 * entries.  Returns LYM_ERR_NOT_CONVERGED if any rhs missed tol. */
int lym_wilson_solve(lym_gauge* g, double kappa, int nrhs, const void* b, void* x,
                     const lym_solver_params* params, lym_solver_report* reports, void* stream);

/* Several independent lattices at once: gauges[l] (distinct objects of the same nd and N,
 * each with its own geometry and links) with kappas[l], tolerance tols[l] (NULL: params->tol
 * for every lattice) and nrhs[l] right-hand sides b[l] (reference layout), solutions into
 * x[l] -- the systems of lym_wilson_solve, solved
 * together: the sloppy CG iterations of every lattice run in the same five launches per
 * iteration (each lattice owns a range of the blocks), in CUDA graphs; setup, FP64
 * reliable updates and the odd-site reconstruction run per lattice.  One rhs per hop
 * thread (FP32: 12-real links when every lattice's links are SU(N); FP16: the
 * mixed-precision hop).  `reports` has sum(nrhs) entries in lattice order.  No reference
 * counterpart (the reference solves one lattice per process). */
int lym_wilson_solve_multi(int nlat, lym_gauge* const* gauges, const double* kappas, const double* tols,
                           const int* nrhs, const void* const* b, void* const* x,
                           const lym_solver_params* params, lym_solver_report* reports, void* stream);

/* Runs the solver's even-odd hopping kernel s_o = H_oe p_e `repeats` times on
 * the workspace left by the last lym_wilson_solve with this (precision, nrhs):
 * the same kernel the CG iterations launch, for timing and profiling it alone
 * (no reference counterpart; the reference has no separate dslash).  Returns
 * LYM_ERR_BAD_ARG when no such workspace exists. */
int lym_dslash_eo(lym_gauge* g, int precision, int nrhs, int repeats, void* stream);

/* Multishift CG on (Q^2 + sigma_k) x_k = b over the full lattice, FP64
 * (nshift, ns, N, V) solutions.  Replaces multishift_solver.solve on a
 * SquareOperator(DiracWilsonOperator) (dirac_solver.py:19-53) for positive
 * shifts; stops when every shift's residual is below tol * |b|. */
int lym_multishift_solve(lym_gauge* g, double kappa, int nshift, const double* shifts,
                         const void* b, void* xs, double tol, int max_iter,
                         int* iterations, void* stream);

/* Multishift CG on (Q^2 + sigma_k) x_{i,k} = b_i for nrhs right-hand sides b_i
 * (reference layout (nrhs, ns, N, V)) and nshift >= 0 shifts at once, with the
 * inner iterations in params->precision (FP64, FP32, norm-scaled FP16 / BF16)
 * and FP64 reliable updates; every (i, k) is verified by its FP64 true residual
 * and refined by a CG of its own if it is above params->tol |b_i|.  xs receives
 * (nrhs, nshift, ns, N, V); reports has nrhs * nshift entries (i * nshift + k).
 * Replaces multishift_solver.solve on a SquareOperator(DiracWilsonOperator)
 * (dirac_solver.py:19-53) for positive shifts, several sources per call;
 * builder-defined algorithm (even-odd layout, Jegerlehner's recurrences).
 * params->switch_residual sets where a reduced precision takes over from FP64;
 * params->hermitian, compressed_links and mixed_fma are not used;
 * rhs_per_thread = 1 forces one group per hop-kernel thread. */
int lym_multishift_solve_eo(lym_gauge* g, double kappa, int nrhs, int nshift, const double* shifts,
                            const void* b, void* xs, const lym_solver_params* params,
                            lym_solver_report* reports, void* stream);

/* The reference's multishift MMMR itself (dirac_solver.py:19-53): base shift
 * shifts[nshift-1], alpha = omega <p,r>/<p,p>, absolute stop |<r,r>| < precision.
 * *steps receives the step index the reference prints. FP64, full lattice. */
int lym_mmmr_solve(lym_gauge* g, double kappa, int nshift, const double* shifts,
                   const void* b, void* xs, int max_steps, double precision, double omega,
                   int* steps, void* stream);

/* ------------------------------------------------------------------ */
/* gauge side (reference layout, FP64)                                 */
/* ------------------------------------------------------------------ */

/* force = Wilson gauge force -beta/(4N)(W^dag - W), traceless, W = U S^dag with
 * S the staple sum over all planes (gauge_action.py:13-24,42-101).  When
 * `momenta` is not NULL the force is not stored; instead momenta += eps*force
 * (hmc.py:59-61 fused).  `force` may then be NULL. */
int lym_gauge_force(const lym_lattice* lat, int nc, double beta, const void* gauge,
                    void* force, void* momenta, double eps, void* stream);

/* staples (nd, N, N, V) with direction `no_direction` excluded (-1: none)
 * (staples.py:23-58, gauge_action.py:56-101). */
int lym_staples(const lym_lattice* lat, int nc, const void* gauge, int no_direction,
                void* staples, void* stream);

/* The per-plane staple terms of staples.py:23-58 (get_staple_fields), in its list
 * order: terms (nd, 2(nd-1), N, N, V), where for direction mu != no_direction the
 * planes (mu, nu), nu != mu and nu != no_direction in increasing nu, give slot 2k the
 * term U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag (sup_staple_trace, staples.py:13-15) and slot
 * 2k+1 the term U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) (sdn_staple_trace, :18-20).
 * Slots without a plane (all of direction no_direction, and the last two of the
 * others when no_direction is a direction) are not written. */
int lym_staple_terms(const lym_lattice* lat, int nc, const void* gauge, int no_direction,
                     void* terms, void* stream);

/* out[0] (host) = sum_{x, mu<nu} Re Tr P_mu,nu(x); out[1] = Im (gauge_action.py:110-113
 * summed as in measurements.py:22-43 and gauge_action.py:26-39).  Synchronises. */
int lym_plaquette_sum(const lym_lattice* lat, int nc, const void* gauge, double* out, void* stream);

/* momenta (nd, N, N, V) from unit normals (nd, N^2-1, V) (device, float64): the
 * anti-Hermitian traceless matrices random_momenta builds from its draws (hmc.py:69-96):
 * per direction the (re, im) pairs of the entries above the diagonal in row order, then
 * the N-1 Cartan values, each halved; unit variance per generator T^a = lambda^a / 2. */
int lym_momenta_from_normals(int nd, int nc, int64_t volume, const double* normals, void* momenta,
                             void* stream);

/* out (host) = -Re sum Tr P^2 (hmc.py:170-176).  Synchronises. */
int lym_momenta_energy(int nd, int nc, int64_t volume, const void* momenta, double* out, void* stream);

/* momenta += eps * force (hmc.py:59-61); n = nd*N*N*V complex elements. */
int lym_update_momenta(int64_t n, void* momenta, const void* force, double eps, void* stream);

/* gauge <- expm(eps P) gauge per link (hmc.py:40-43), in place.  SU(2)/SU(3)
 * closed forms; reunitarize != 0 projects the result back onto SU(N). */
int lym_update_links(int nd, int nc, int64_t volume, void* gauge, const void* momenta,
                     double eps, int reunitarize, void* stream);

/* The gauge part of an HMC step on nlat independent lattices (each its own lattice
 * object, N, beta, links gauges[l] and momenta momenta[l], reference layout) in two
 * launches whatever their sizes and (nd, N): momenta += eps_p * F_gauge(U) for every
 * link of every lattice (gauge_action.py:13-24 + hmc.py:59-61), then U <- exp(eps_u P) U
 * (hmc.py:40-43).  No reference counterpart (the reference runs one lattice per
 * process); the same arithmetic as lym_gauge_force into the momenta followed by
 * lym_update_links.  nlat <= 256; no buffer may belong to two lattices
 * (LYM_ERR_BAD_ARG). */
int lym_gauge_hmc_step_multi(int nlat, const lym_lattice* const* lats, const int* nc, const double* betas,
                             void* const* gauges, void* const* momenta, double eps_p, double eps_u,
                             void* stream);

/* out = X (X^dag X)^{-1/2} / det^{1/N} per link (smearing.py:17-31). */
int lym_unitary_projection(int nd, int nc, int64_t volume, const void* in, void* out, void* stream);

/* force += scale * sum_i alpha_i [L(X_i, Y_i) + L(Y_i, X_i)] when symmetric != 0,
 * else force += scale * sum_i alpha_i L(X_i, Y_i), with L the Lie derivative of
 * dirac.py:525-565 (fundamental) and X, Y stored (nterms, ns, N, V).
 * The fused form of n_flavor.force (fermion_action.py:64-93). */
int lym_fermion_force(const lym_lattice* lat, int nc, double kappa, int hermitian,
                      double bc_re, double bc_im, const void* gauge, int nterms,
                      const double* alphas, const void* X, const void* Y, int symmetric,
                      double scale, void* force, void* stream);

/* ------------------------------------------------------------------ */
/* adjoint representation (dirac.py:358-370, 380-456, 525-565)         */
/* ------------------------------------------------------------------ */

/* Adjoint Wilson operator on nvec matrix-valued spinors (nvec, ns, N, N, V): out =
 * psi + kappa sum_mu [L_mu(x)(1-g_mu)psi(x+mu)U_mu(x)^dag + L_mu(x-mu)^dag(1+g_mu)
 * psi(x-mu)U_mu(x-mu)], gamma_d applied when hermitian.  L = gauge_left with
 * (bc_re, bc_im) on the last time slice of the last direction (the reference's cfg),
 * U = gauge (its original_cfg); gauge_left may be gauge.  Replaces
 * multiply_in_adjoint_representation / simple_multiply_in_adjoint_representation
 * (same result). */
int lym_wilson_apply_adjoint(const lym_lattice* lat, int nc, double kappa, int hermitian,
                             double bc_re, double bc_im, const void* gauge_left, const void* gauge,
                             int nvec, const void* in, void* out, void* stream);

/* Adjoint links V_mu^{ab} = 2 Tr(T_a U_mu T_b U_mu^dag), (nd, N^2-1, N^2-1, V), times
 * (bc_re, bc_im) on the last time slice of the last direction: the reference's
 * fermion_gauge_field for representation "adjoint" (dirac.py:358-370). */
int lym_adjoint_links(const lym_lattice* lat, int nc, double bc_re, double bc_im,
                      const void* gauge, void* out, void* stream);

/* force += scale * sum_i alpha_i [L(X_i, Y_i) (+ L(Y_i, X_i) if symmetric)] for matrix-valued
 * X, Y (nterms, ns, N, N, V), L the adjoint branch of lie_derivative (dirac.py:525-565) with the
 * adjoint links built in place from gauge and the boundary factor; nterms <= 32. */
int lym_fermion_force_adjoint(const lym_lattice* lat, int nc, double kappa, int hermitian,
                              double bc_re, double bc_im, const void* gauge, int nterms,
                              const double* alphas, const void* X, const void* Y, int symmetric,
                              double scale, void* force, void* stream);

/* ------------------------------------------------------------------ */
/* on-disk gauge format (lattice.py:10-70)                             */
/* ------------------------------------------------------------------ */

/* Decode the link section of the reference's XDR configuration file, already on the
 * device: raw = volume x nd x 3 x 2 x 2 big-endian float32 words (the first two
 * columns of conj(U), re/im, site slowest; 16-byte aligned) -> gauge (nd, 3, 3, V)
 * complex128 with columns 0, 1 Gram-Schmidt normalised and column 2 = conj(col0 x col1),
 * as read_config does.  nc must be 3. */
int lym_decode_xdr_gauge(int nd, int nc, int64_t volume, const void* raw, void* gauge, void* stream);

/* ------------------------------------------------------------------ */
/* gauge observables (measurements.py:46-290)                          */
/* ------------------------------------------------------------------ */

/* Per starting site x, the ordered product of the links along a path of nsteps <= 256
 * steps: +(mu+1) multiplies U_mu(y) and moves y to y + mu, -(mu+1) moves y to y - mu and
 * multiplies U_mu(y)^dag.  trace = 1: out (V) complex128 = Tr of the product (plaquettes,
 * 2x2 squares, Wilson loops, Polyakov loops); trace = 0: out (N, N, V) the product itself
 * (wilson_lines_field). */
int lym_path_product(const lym_lattice* lat, int nc, const void* gauge, int nsteps, const int* steps,
                     int trace, void* out, void* stream);

/* out (device, 2 L doubles, L = the extent of `direction`): out[2z], out[2z+1] = sum of the
 * complex field (V) over the sites with x_direction = z and, when mask_direction >= 0,
 * x_mask_direction = 0 (the zero-momentum projections of measurements.py:160-290). */
int lym_slice_sums(const lym_lattice* lat, int direction, int mask_direction, const void* field,
                   double* out, void* stream);

/* ------------------------------------------------------------------ */
/* fermion measurements (fermion_measurements.py:41-115)               */
/* ------------------------------------------------------------------ */

/* out (device, 2 * L doubles, L = the lattice extent in `direction`): out[2z], out[2z+1] =
 * sum over nvec vectors and the sites with x_direction = z of sum_{spin,colour} conj(S) S
 * (fundamental, vectors (ns, N, V)) or sum_{spin,c,d} conj(S_cd) S_dc (adjoint = 1, vectors
 * (ns, N, N, V)): the slice sums of pion_correlator (fermion_measurements.py:76-90). */
int lym_timeslice_sums(const lym_lattice* lat, int direction, int nvec, int ns, int nc, int adjoint,
                       const void* in, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LYM_H */
