/*
 * energy_level_b200.h -- C ABI of the B200 matrix-free many-body ED library.
 *
 * The library applies and solves the Rydberg Hamiltonian
 *
 *     H = sum_i [ delta_i n_i + (Omega_i/2) sigma^x_i ] + sum_{i<j} V_ij n_i n_j
 *
 * (energies in cyclic MHz, times in ns, phase = 2*pi*1e-3 * E * t) on the full
 * 2^N basis or on a constrained sector (blockade independent sets, fixed
 * excitation number).  Basis identity follows the reference engine: site 0 is
 * the most significant bit of a configuration code, bit = 1 means |r>, sector
 * states are listed in ascending code order.
 *
 * Conventions of every entry point:
 *   - the return value is a status code (EL_OK = 0); el_last_error() gives text;
 *   - no C++ exception crosses the ABI and no kernel traps;
 *   - vectors are caller-owned DEVICE pointers unless a name ends in _host;
 *     a block of `nvec` vectors is stored row-major, [dim][nvec];
 *   - handles and internal workspace are owned by the library;
 *   - all work is queued on the context's stream (el_ctx_set_stream);
 *   - a cancel flag (el_ctx_set_cancel) is polled between launches and turns
 *     into EL_ECANCEL.
 *
 * Each entry point names the reference interface it replaces
 * (paths inside the energy-level project, src/core/manybody/...).
 */
#ifndef ENERGY_LEVEL_B200_H
#define ENERGY_LEVEL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define EL_OK        0
#define EL_EINVAL    1  /* bad argument (maps to ValueError)                    */
#define EL_ENOMEM    2  /* allocation or memory budget (maps to MemoryError)    */
#define EL_ENOTCONV  3  /* iteration cap reached before tolerance               */
#define EL_ECANCEL   4  /* cancel flag observed (maps to RuntimeError 用户取消) */
#define EL_ECUDA     5  /* CUDA runtime error (maps to RuntimeError)            */

/* arithmetic types of state vectors */
#define EL_F32   0
#define EL_F64   1
#define EL_C64   2
#define EL_C128  3

/* basis kinds accepted by el_basis_build */
#define EL_BASIS_FULL      0  /* all 2^N codes                                 */
#define EL_BASIS_BLOCKADE  1  /* independent sets of the edge list             */
#define EL_BASIS_CHARGE    2  /* codes with popcount == k                      */

/* internal layouts reported by el_basis_info */
#define EL_LAYOUT_FULL   0  /* rank(code) = code                                */
#define EL_LAYOUT_CHAIN  1  /* nearest-neighbour path: Zeckendorf ranking       */
#define EL_LAYOUT_RING   2  /* nearest-neighbour cycle: two-branch Zeckendorf   */
#define EL_LAYOUT_TABLE  3  /* general constraint: prefix/suffix class tables   */

/* KPM moment modes */
#define EL_KPM_DIRECT    0  /* mu_n from <z, T_n z>, the reference recurrence   */
#define EL_KPM_DOUBLING  1  /* mu_2n = 2<T_n z,T_n z>-mu_0, mu_2n+1 likewise    */
#define EL_KPM_GENERIC_KERNEL 0x100 /* flag: use the row-parallel kernel even
                                       where the tiled full-basis one applies */

typedef struct el_ctx el_ctx;
typedef struct el_basis el_basis;
typedef struct el_ham el_ham;

/* ---- library and context ------------------------------------------------ */

/* Library version, major*10000 + minor*100 + patch. */
int el_version(void);

/* Create a context bound to CUDA device `device`; `stream` is a cudaStream_t
 * (NULL = legacy default stream).  Replaces the implicit torch device setup of
 * matrix_free.py:177-185 (torch_lanczos_ground_state) and kpm.py:48. */
int el_ctx_create(int device, void *stream, el_ctx **out);
int el_ctx_destroy(el_ctx *ctx);
int el_ctx_set_stream(el_ctx *ctx, void *stream);
/* Host flag polled between launches; nonzero -> EL_ECANCEL.  Mirrors the
 * progress_arr[1] cancel convention of runtime.py:12-14 (check_cancel). */
int el_ctx_set_cancel(el_ctx *ctx, const volatile int32_t *flag);
/* Text of the last error on this context (empty string when none). */
const char *el_last_error(const el_ctx *ctx);
/* Number of kernels this context has launched since creation. */
int64_t el_ctx_launches(const el_ctx *ctx);
/* Host->device and device->host bytes this context has copied since creation
 * (inputs, parameters, scalars and results; device-to-device copies excluded). */
int el_ctx_bytes(const el_ctx *ctx, int64_t *h2d, int64_t *d2h);

/* ---- basis ---------------------------------------------------------------- */

/* Build a basis of `n` sites (1 <= n <= 63).  kind = EL_BASIS_FULL (n <= 34),
 * EL_BASIS_BLOCKADE with `n_edges` pairs in `edges` (host, 2*n_edges int32,
 * validated like basis.py:12-21 validate_edges), or EL_BASIS_CHARGE with
 * excitation number k.  `max_states` <= 0 means no cap; otherwise a larger
 * sector fails with EL_EINVAL like basis.py:38-39.
 * Replaces basis.py:24-47 independent_states, matrix_free.py:12-38
 * number_sector_basis and hamiltonian_plan.py:129-148 build_plan (states). */
int el_basis_build(el_ctx *ctx, int n, const int32_t *edges, int n_edges,
                   int kind, int k, int64_t max_states, el_basis **out);
/* Dimension and internal layout (EL_LAYOUT_*). */
int el_basis_info(const el_basis *basis, int64_t *dim, int *layout);
/* Write the ascending code list (device uint64[dim]).  Bit-exact with the
 * reference's state lists (basis.py:24-47, matrix_free.py:12-38). */
int el_basis_codes(el_ctx *ctx, el_basis *basis, uint64_t *codes);
/* rank[i] = index of codes[i] in the basis or -1 (device arrays).  Replaces
 * the position table / searchsorted of channels.py:177-192. */
int el_basis_rank(el_ctx *ctx, el_basis *basis, const uint64_t *codes,
                  int64_t count, int64_t *ranks);
int el_basis_destroy(el_basis *basis);

/* ---- Hamiltonian ---------------------------------------------------------- */

/* Create H on `basis`.  omega_re/omega_im/delta are per-site host arrays of
 * length n (omega_im may be NULL); pairs (pi[p], pj[p], V[p]) are the I1
 * density-density couplings.  Channel semantics follow channels.py:58-132
 * (diagonal delta n + V n n; sigma^x amplitude Omega/2 for g->r and
 * conj(Omega)/2 for r->g).  Replaces channels.py:91-132 channel_spec and the
 * diagonal of channels.py:58-77. */
int el_ham_create(el_ctx *ctx, el_basis *basis, const double *omega_re,
                  const double *omega_im, const double *delta, int n_pairs,
                  const int32_t *pi, const int32_t *pj, const double *V,
                  el_ham **out);
/* Replace the drive (per-site Omega and delta), keeping basis and V.  Used per
 * piecewise-constant segment, replacing the per-segment CSR rebuild of
 * engine_ed.py:141-144. */
int el_ham_set_drive(el_ctx *ctx, el_ham *ham, const double *omega_re,
                     const double *omega_im, const double *delta);
/* Set (replace) the loss rates gamma[i] (per site, as the reference's
 * gamma_mhz; NULL clears them): the diagonal gains -0.5 i gamma_i 1e-3 / CONV
 * per excited site i (channels.py:69-76).  H is then non-Hermitian and
 * complex: products need complex dtypes, ground states, bounds, KPM, the
 * Chebyshev step and the adjoint refuse it, and evolution uses
 * el_taylor_step. */
int el_ham_set_loss(el_ctx *ctx, el_ham *ham, const double *gamma);
/* Set (replace) the two-site exchange channels of ham: for each pair p the
 * sites (pi[p], pj[p]), J = J_re + i J_im (I2: <g_i r_j|H|r_i g_j> = conj(J),
 * <r_i g_j|H|g_i r_j> = J) and A = A_re + i A_im (I3: <r_i r_j|H|g_i g_j> = A,
 * <g_i g_j|H|r_i r_j> = conj(A)); any of the four amplitude arrays may be
 * NULL (zero).  Targets outside a restricted basis are dropped, as for the
 * sigma^x channels.  A complex J or A makes H complex (complex vector dtypes
 * only).  n_pairs = 0 removes all exchange channels.  With exchange channels
 * every product runs the generic row kernel and KPM the generic recurrence.
 * Replaces the I2/I3 channels of channels.py:119-131 channel_spec. */
int el_ham_set_exchange(el_ctx *ctx, el_ham *ham, int n_pairs, const int32_t *pi,
                        const int32_t *pj, const double *J_re, const double *J_im,
                        const double *A_re, const double *A_im);
/* Full diagonal d(s) = sum delta_i n_i + sum V_ij n_i n_j into a device array
 * of type dtype (EL_F32 or EL_F64).  Replaces channels.py:58-77. */
int el_ham_diag(el_ctx *ctx, el_ham *ham, int dtype, void *out);
int el_ham_destroy(el_ham *ham);

/* ---- apply ------------------------------------------------------------------ */

/* y = H x for a block of nvec vectors (nvec in 1,2,4,8,16,32 or a multiple of
 * 32).  Device pointers.  Replaces channels.py:210-221 ChannelKernel.matvec and
 * the index_select/index_add_ action of matrix_free.py:200-204. */
int el_hv(el_ctx *ctx, el_ham *ham, int dtype, int nvec, const void *x,
          void *y);
/* Same product with HOST buffers: copies in, applies, copies out.  The
 * reference-facing form of matrix_free.py:51-62 hamiltonian_linear_operator. */
int el_hv_host(el_ctx *ctx, el_ham *ham, int dtype, int nvec,
               const void *x_host, void *y_host);

/* ---- spectral bounds and KPM --------------------------------------------- */

/* Extremal eigenvalues by FP64 Lanczos from a seeded start vector.  Replaces
 * kpm.py:82-97 _bounds (ARPACK eigsh SA/LA). */
int el_bounds(el_ctx *ctx, el_ham *ham, int max_iter, double tol,
              uint64_t seed, double *emin, double *emax);
/* Chebyshev moments mu[0..num] of Htil = (H - c)/r from nvec Rademacher
 * probes processed `chunk` at a time (chunk in 1,2,4,8,16,32 or multiple of
 * 32).  probes_host: NULL = counter-based probes from `seed`, else int8
 * [nvec][dim] of +-1.  dtype EL_F32 or EL_F64 (vectors); moments are always
 * accumulated in FP64.  mu[n] = sum_probes <z, T_n z> / (nvec * dim).
 * On the full basis (6 <= N <= 25) EL_KPM_DOUBLING runs the tiled kernel
 * (two reads and two writes per element and step) unless the
 * EL_KPM_GENERIC_KERNEL flag is or-ed into `mode`.
 * Replaces kpm.py:26-75 kpm_moments_gpu and kpm.py:115-151 kpm_moments. */
int el_kpm_moments(el_ctx *ctx, el_ham *ham, int dtype, int num, int nvec,
                   int chunk, uint64_t seed, const int8_t *probes_host,
                   int mode, double c, double r, double *mu_host);

/* ---- Lanczos ground state ------------------------------------------------- */

/* Lowest `nev` (1 or 2) eigenpairs by three-term Lanczos with FP64 alpha/beta,
 * partial (omega-recurrence) or full reorthogonalisation (`reorth` 1 or 2;
 * 0 = none), host tridiagonal eigensolve, explicit restarts.  Vectors in
 * dtype (EL_F32/EL_F64 for real H, EL_C64/EL_C128 for complex Omega).
 * v0: device start vector or NULL (seeded Gaussian).  evals/residuals: host
 * [nev]; residual = ||H x - theta x|| of the returned Ritz vector.
 * vec_out: device [dim] ground Ritz vector or NULL.
 * Replaces matrix_free.py:118-286 torch_lanczos_ground_state and
 * equilibrium.py:35-96 ground_state (eigsh 'SA'). */
int el_lanczos_ground(el_ctx *ctx, el_ham *ham, int dtype, const void *v0,
                      uint64_t seed, int max_iter, int max_restarts,
                      double tol, int nev, int reorth, double *evals,
                      double *residuals, int *iters, int *converged,
                      void *vec_out);
/* Lanczos tridiagonalisation from a source state (device phi, not modified):
 * alphas[n] and betas[n-1] of H in the Krylov basis of phi, with full
 * reorthogonalisation (twice per step) when reorth != 0.  Stops at
 * n_krylov steps, at beta <= 1e-12 or when the Krylov space is the whole
 * basis (converged = 1 then).  norm2 = |phi|^2; ortho_loss = |<q_0, q_last>|
 * (0 without reorth).  Replaces spectrum.py:34-103 (lanczos) for
 * spectrum.py:138-180 (source_spectrum) and eq_route.py:260-337. */
int el_lanczos_tridiag(el_ctx *ctx, el_ham *ham, int dtype, const void *phi, int n_krylov,
                       int reorth, double *alphas, double *betas, int *n, double *norm2,
                       double *ortho_loss, int *converged);

/* ---- batched ground states ---------------------------------------------- */

typedef struct el_batch el_batch;

/* Describe `count` independent Hamiltonians: instance i has n_sites[i] sites
 * (<= 40), basis layout layouts[i] (EL_LAYOUT_CHAIN or EL_LAYOUT_RING
 * blockade sectors, or EL_LAYOUT_FULL up to 24 sites), per-site Omega and
 * delta (host, concatenated over instances) and the I1 pairs
 * pi/pj/V[pair_off[i] .. pair_off[i+1]) (offsets non-decreasing, else
 * EL_EINVAL).  Vectors in dtype (EL_F32/EL_F64),
 * alpha/beta and the tridiagonal solve in FP64; at most max_iter (<= 384)
 * Lanczos steps per instance; convergence when the residual estimates of the
 * two lowest Ritz pairs are <= tol * max(1, |theta|).
 * Replaces the per-instance eigsh calls of eq_route.py:540-728 and the dense
 * batched_ground_state of equilibrium.py:251-311 for sector problems. */
int el_batch_create(el_ctx *ctx, int count, const int32_t *n_sites, const int32_t *layouts,
                    const double *omega, const double *delta, const int32_t *pair_off,
                    const int32_t *pi, const int32_t *pj, const double *V, int dtype,
                    int max_iter, double tol, el_batch **out);
/* As el_batch_create, and layouts[i] may also be EL_LAYOUT_TABLE: the
 * blockade sector of an arbitrary graph, whose edges (site indices) are
 * ei/ej[edge_off[i] .. edge_off[i+1]) (edges of other layouts are ignored).
 * The sector's independent sets are enumerated on the host (at most 2^24
 * rows per instance, else EL_EINVAL) and a flip table of target rows
 * (4 bytes per row and site) is built on the device once.  The batched
 * ground state of the reference for any blockade graph
 * (equilibrium.py:251-311 with the plan of hamiltonian_plan.py:15-50). */
int el_batch_create_graph(el_ctx *ctx, int count, const int32_t *n_sites, const int32_t *layouts,
                          const double *omega, const double *delta, const int32_t *pair_off,
                          const int32_t *pi, const int32_t *pj, const double *V, const int32_t *edge_off,
                          const int32_t *ei, const int32_t *ej, int dtype, int max_iter, double tol,
                          el_batch **out);
/* Queue the whole batch as ONE persistent launch (CTAs pull instances from an
 * atomic queue, largest first).  threads: 256/512/1024 per CTA; ctas_per_sm:
 * 1 or 2.  Asynchronous and capturable in a CUDA graph once a first run has
 * sized the workspace. */
int el_batch_run(el_ctx *ctx, el_batch *batch, int threads, int ctas_per_sm, uint64_t seed);
/* Solve the batch's instances one after another, each with the whole GPU:
 * one cooperative launch per instance splits its rows over up to 64 CTAs
 * (one row per thread) that keep their slices of the Krylov basis in shared
 * memory and reorthogonalise fully every step (classical Gram-Schmidt,
 * reorth_passes = 1 or 2 times), meeting at grid barriers (bounded waits: a timeout returns
 * EL_ECUDA).  For instances too small to fill the GPU with vectors but slow
 * on one SM (a full 2^12 basis: a few thousand rows); EL_EINVAL when an
 * instance's slice does not fit shared memory.  The Ritz values and their
 * residual estimates are evaluated every check_every steps (and at the
 * last).  Same results layout as el_batch_run (read with el_batch_results). */
int el_batch_run_coop(el_ctx *ctx, el_batch *batch, int reorth_passes, int check_every,
                      uint64_t seed);
/* Also form each instance's ground-state site occupations <n_i> in later
 * runs (want != 0; el_batch_run and el_batch_run_coop): the Ritz vector of
 * the lowest Ritz value from the stored Krylov basis, normalised, its
 * weights summed per excited site.  The n_atom output of the reference's
 * batched_ground_state (equilibrium.py:251-311).  Call outside graph
 * capture the first time (it allocates the result buffer). */
int el_batch_want_occupations(el_ctx *ctx, el_batch *batch, int want);
/* Copy the occupations of the last run: n_atom[i * 40 + s] = <n_s> of
 * instance i (caller order, site s as in the calib; zeros beyond n_sites).
 * Synchronises the stream. */
int el_batch_occupations(el_ctx *ctx, el_batch *batch, double *n_atom);
/* Bound of every grid-barrier wait of el_batch_run_coop, in polls of the
 * arrival counter (about 64 ns apart; default 4,194,304).  When a wait runs
 * out, that CTA stops waiting, sets the batch's error flag, every later
 * barrier and step of the launch is skipped, and el_batch_run_coop returns
 * EL_ECUDA ("a grid barrier timed out") with the flag of every instance
 * kept; the context stays usable.  A small bound makes a slow or shared GPU
 * report a stall early.  No counterpart in the reference (its CPU solvers
 * have no device waits). */
int el_batch_set_wait_limit(el_ctx *ctx, el_batch *batch, int32_t polls);
/* Copy results (caller order): ground energy, gap E1 - E0, max residual
 * estimate, Lanczos steps, converged flag.  Synchronises the stream. */
int el_batch_results(el_ctx *ctx, el_batch *batch, double *e0, double *gap, double *residual,
                     int32_t *iters, int32_t *converged);
int el_batch_destroy(el_batch *batch);

/* ---- time evolution ------------------------------------------------------- */

/* psi <- exp(-i 2pi 1e-3 H tau_ns) psi by a Chebyshev expansion truncated at
 * `tol` (dtype EL_C64 or EL_C128).  *n_terms returns the number of terms.
 * Replaces the expm_multiply step of engine_ed.py:125 and engine_ed.py:145. */
int el_cheb_step(el_ctx *ctx, el_ham *ham, int dtype, void *psi,
                 double tau_ns, double tol, int *n_terms);
/* psi <- exp(-i CONV tau H) psi for any H, including a loss diagonal (gamma
 * != 0, non-Hermitian): s substeps of a degree-m Taylor polynomial chosen
 * from the bound ||H|| <= max_r (|d_r| + sum_s |H_rs|) so that the remainder
 * bound is below tol per step; *n_terms = s * m H applications.  Replaces
 * expm_multiply (engine_ed.py:125,145) on the non-Hermitian path. */
int el_taylor_step(el_ctx *ctx, el_ham *ham, int dtype, void *psi, double tau_ns,
                   double tol, int *n_terms);
/* Pulse gradient by the adjoint of the Chebyshev propagator.  K steps; step k
 * lasts tau[k] ns with Omega_i = omega_k[k] * omega_shape[i] and
 * delta_i = -delta_k[k] * delta_shape[i] (shapes NULL = 1), V from `ham`.
 * Objective F = |<target|psi_K>|^2 (target: device state) or, with target
 * NULL, F = sum_r obs_diag[r] |psi_K[r]|^2 (obs_diag: device FP64 [dim]).
 * Returns F and dF/domega_k, dF/ddelta_k (host [K]) of the discretised map
 * (discretise-then-differentiate: reverse recurrence through each
 * Chebyshev expansion, terms recomputed per step from one checkpoint per
 * step).  psi_final (device, may be NULL) receives psi_K.  The reference has
 * no gradient code; it replaces central finite differences of
 * engine_ed.py:130-147 evolutions. */
int el_adjoint_pulse(el_ctx *ctx, el_ham *ham, int dtype, int K, const double *tau,
                     const double *omega_k, const double *delta_k, const double *omega_shape,
                     const double *delta_shape, const void *psi0, const void *target,
                     const double *obs_diag, double tol, double *F, double *grad_omega,
                     double *grad_delta, void *psi_final);
/* How el_adjoint_pulse schedules its sweeps over the basis (per context):
 * EL_ADJ_AUTO (default) and EL_ADJ_COOP run the whole gradient as one
 * cooperative launch with grid barriers between sweeps (bounded waits: a
 * timeout returns EL_ECUDA); EL_ADJ_STREAM launches one kernel per
 * Chebyshev term and reverse term.  Both give the same gradient up to
 * rounding.  No counterpart in the reference (scheduling only). */
#define EL_ADJ_AUTO   0
#define EL_ADJ_STREAM 1
#define EL_ADJ_COOP   2
int el_adjoint_set_mode(el_ctx *ctx, int mode);
/* Site occupations <n_i> (host double[n]) and squared norm of psi.  Replaces
 * the bits @ |psi|^2 reduction of engine_ed.py:259-263 (_reduce). */
int el_observables(el_ctx *ctx, el_ham *ham, int dtype, const void *psi,
                   double *n_site_host, double *norm_host);
/* Spin observables of a device state psi (dtype EL_*): norm, <n_i> and
 * <sigma-_i> (complex, re/im interleaved in sigma_minus[2n]) for every site,
 * and for each of n_pairs site pairs (pi[p], pj[p]), i != j in any order,
 * <n_i n_j> (nn[p]) and <sigma+_i sigma-_j> (complex, xy[2p], xy[2p+1]).  On
 * a restricted basis flip targets outside it drop out.  Any output pointer
 * may be NULL; n_pairs may be 0.  FP64 sums in a fixed order.  Replaces
 * observables.py:117-205 spin_observables / spin_observables_basis and the
 * <n_i n_j> of observables.py:40-47 corr_matrix, evaluated per output time in
 * engine_ed.py:259-281. */
int el_spin_observables(el_ctx *ctx, el_ham *ham, int dtype, const void *psi,
                        int n_pairs, const int32_t *pi, const int32_t *pj,
                        double *n_site, double *norm, double *sigma_minus,
                        double *nn, double *xy);
/* Expectations <psi|P_q|psi> of n_strings Pauli strings (complex, re/im
 * interleaved in out_host[2 n_strings]).  String q is the product over
 * k in [offsets[q], offsets[q+1]) of sigma^{axes[k]} on site sites[k]
 * (axes 'x', 'y', 'z'; distinct sites; standard Pauli matrices in the
 * (|g>, |r>) basis).  On a restricted basis, targets outside it drop out.
 * Replaces observables.py:486-622 PauliPlan.expect (full and basis kinds). */
int el_pauli_expect(el_ctx *ctx, el_ham *ham, int dtype, const void *psi, int n_strings,
                    const int32_t *offsets, const int32_t *sites, const char *axes,
                    double *out_host);
/* el_observables without any allocation.  This entry point has no
 * counterpart in the reference; it exists for callers that must not allocate
 * device memory once they are running, e.g. an evolution driver measuring
 * <n_i> between propagation steps in a process whose own pool already holds
 * the free HBM (a cudaMalloc would fail there, and cudaMalloc / cudaFree can
 * stall the device).  el_observables may grow the context's reduction buffer
 * on first use for a larger basis; this call never allocates: its reduction
 * scratch is one static device array of fixed size (195,200 bytes per
 * device), and the results pass through the context's pinned result area.
 *  - Limit: at most 40 sites; larger systems return EL_EINVAL (message in
 *    el_last_error) and are served by el_observables.
 *  - The scratch's completion counter must be zero when a call starts: it is
 *    zero when the library loads and every call leaves it zero.  Nothing else
 *    in the scratch needs an initial value.
 *  - All callers on one device share the scratch: calls on the same device
 *    must not overlap in time (other host threads, other streams or other
 *    contexts); overlapping calls race and return wrong values.
 *  - The first call on each device looks up the scratch's device address
 *    (cudaGetSymbolAddress); make it before any stream capture starts on that
 *    device.
 * Same arguments, results and dtypes as el_observables. */
int el_observables_noalloc(el_ctx *ctx, el_ham *ham, int dtype, const void *psi,
                           double *n_site_host, double *norm_host);

#ifdef __cplusplus
}
#endif

#endif /* ENERGY_LEVEL_B200_H */
