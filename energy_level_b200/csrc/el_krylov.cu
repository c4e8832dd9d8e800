// Krylov drivers: Lanczos ground state, spectral bounds and KPM moments.
//
// Lanczos (replaces matrix_free.py:118-286 torch_lanczos_ground_state and the
// ARPACK path of equilibrium.py:85): three-term recurrence
//     w = H v_j - beta_j v_{j-1};  alpha_j = <v_j, w>;  w -= alpha_j v_j
// with alpha/beta in FP64 whatever the vector type, partial
// reorthogonalisation driven by Simon's omega recurrence (or full / none),
// a host FP64 tridiagonal eigensolve, Ritz-residual certification as in
// matrix_free.py:258-264 (||H x - theta x|| <= tol * max(1, |theta|)) and
// explicit restarts from the Ritz vectors.
//
// KPM (replaces kpm.py:26-75 and kpm.py:115-151): Hutchinson moments
// mu_n = sum_probes <z, T_n(Htil) z> / (nvec * dim), Htil = (H - c)/r, from
// the fused kernel  t_{n+1} = (2/r) H t_n - (2c/r) t_n - t_{n-1}  with FP64
// dot products.  EL_KPM_DIRECT reproduces the reference recurrence
// (kpm.py:139-149); EL_KPM_DOUBLING uses T_2n = 2 T_n^2 - 1 and
// T_2n+1 = 2 T_n+1 T_n - T_1, halving the number of H applications.
#include "el_internal.cuh"
#include "el_tridiag.h"

#include <algorithm>

namespace {

using el::fail;

bool is_cplx(int dtype) { return dtype == EL_C64 || dtype == EL_C128; }

int sync_read(el_ctx *ctx, const double *dev, int count, double *host) {
  EL_CUDA_TRY(ctx, el::copy(ctx, ctx->h_scalars, dev, count * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < count; ++i) host[i] = ctx->h_scalars[i];
  return EL_OK;
}

struct LanczosOut {
  std::vector<double> alpha, beta;  // beta[j] couples v_j and v_{j+1}
  int steps = 0;
  bool invariant = false;
};

}  // namespace

// ----------------------------------------------------------------- bounds

extern "C" int el_bounds(el_ctx *ctx, el_ham *h, int max_iter, double tol,
                         uint64_t seed, double *emin, double *emax) {
  if (!ctx || !h || !emin || !emax) return EL_EINVAL;
  if (max_iter < 2) return fail(ctx, EL_EINVAL, "max_iter must be >= 2");
  if (h->lossy) return fail(ctx, EL_EINVAL, "spectral bounds need a Hermitian H (gamma = 0)");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t dim = h->basis->dim;
  const int dtype = h->complex_drive ? EL_C128 : EL_F64;
  const size_t vb = (size_t)dim * el::dtype_size(dtype);
  char *buf = (char *)el::workspace(ctx, 0, 3 * vb);
  if (!buf) return EL_ENOMEM;
  void *vp = buf, *v = buf + vb, *w = buf + 2 * vb;
  double *d_sc = ctx->d_scalars;  // [0..3] dots, [8] norm2
  int rc;
  if (dim == 1) {
    double d;
    rc = el::launch_full_diag(ctx, h, EL_F64, v);
    if (rc) return rc;
    rc = sync_read(ctx, (const double *)v, 1, &d);
    if (rc) return rc;
    *emin = *emax = d;
    return EL_OK;
  }
  rc = el::launch_fill_gauss(ctx, dtype, dim, seed, v);
  if (rc) return rc;
  rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, v, d_sc + 8);
  if (rc) return rc;
  rc = el::launch_scale(ctx, dtype, dim, d_sc + 8, 1, v);
  if (rc) return rc;
  EL_CUDA_TRY(ctx, cudaMemsetAsync(vp, 0, vb, ctx->stream));
  // large full bases: the tiled two-pass product (el_kpm_tma.cu) instead of
  // the row kernel, whose high-bit partners come from DRAM again and again
  el_hv_plan *plan = nullptr;
  if (el::hv_tiled_eligible(h, dtype)) {
    void *const bb[3] = {vp, v, w};
    rc = el::hv_tiled_plan(ctx, h, bb, 15, &plan);
    if (rc) return rc;
  }
  struct PlanGuard { el_hv_plan *p; ~PlanGuard() { if (p) el::hv_tiled_free(p); } } guard{plan};
  int ivp = 0, iv = 1, iw = 2;   // buffer indices of vp, v, w in the plan
  std::vector<double> al, be;
  double beta = 0.0, lo_prev = 0, hi_prev = 0;
  // The stored vectors are s_j = kappa_j v_j (v_j the unit Lanczos vectors):
  // one fused update per step forms s_{j+1} = (y - alpha s_j) / (kappa_j
  // beta_pred) with beta_pred from the step's dots, and its norm gives the
  // exact beta and kappa_{j+1}; no separate normalisation pass.
  double kappa = 1.0, kappa_prev = 1.0;
  int stable = 0;
  const int maxit = (int)std::min<int64_t>(max_iter, dim);
  for (int j = 0; j < maxit; ++j) {
    if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
    // y = H s_j - beta_j (kappa_j / kappa_{j-1}) s_{j-1} = kappa_j w_j
    const double cz = j ? -beta * kappa / kappa_prev : 0.0;
    if (plan) {
      rc = el::hv_tiled(ctx, h, plan, iv, iw, ivp, cz, d_sc);
    } else {
      ApplyArgs A;
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = v; A.z = vp; A.y = w;
      A.a = 1.0; A.b = 0.0; A.c = cz; A.dots = d_sc; A.want_dots = 7;
      rc = el::launch_apply(ctx, h, A);
    }
    if (rc) return rc;
    double dots[4];
    rc = sync_read(ctx, d_sc, 4, dots);
    if (rc) return rc;
    const double k2 = kappa * kappa;
    const double alpha = dots[1] / k2;
    const double bp2 = dots[3] / k2 - alpha * alpha;   // |w_j - alpha v_j|^2 from <y,y> (dots[3])
    const double scale_a = std::max(1.0, std::fabs(alpha));
    const bool fused = bp2 > 1e-6 * scale_a * scale_a;  // else: form the norm directly
    const double bpred = fused ? std::sqrt(bp2) : 1.0;
    const double sc = 1.0 / (kappa * bpred);
    rc = el::launch_axpby(ctx, dtype, dim, -alpha * sc, 0, v, sc, 0, w, d_sc + 8);
    if (rc) return rc;
    double n2;
    rc = sync_read(ctx, d_sc + 8, 1, &n2);
    if (rc) return rc;
    al.push_back(alpha);
    // |s_{j+1}|^2 = n2 and s_{j+1} = (beta / bpred) v_{j+1}
    const double kappa_next = std::sqrt(std::max(n2, 0.0));
    beta = kappa_next * bpred;
    const int m = (int)al.size();
    double lo = el::tridiag_eig(al.data(), be.data(), m, 0);
    double hi = el::tridiag_eig_max(al.data(), be.data(), m);
    const double scale = std::max(1.0, std::max(std::fabs(lo), std::fabs(hi)));
    if (m > 2 && std::fabs(lo - lo_prev) <= tol * scale && std::fabs(hi - hi_prev) <= tol * scale) {
      if (++stable >= 3) { lo_prev = lo; hi_prev = hi; break; }
    } else {
      stable = 0;
    }
    lo_prev = lo;
    hi_prev = hi;
    if (beta <= 1e-13 * scale) break;  // invariant subspace: exact extremes
    be.push_back(beta);
    // s_{j-1} <- s_j ; s_j <- s_{j+1}
    std::swap(vp, v);
    std::swap(v, w);
    std::swap(ivp, iv);
    std::swap(iv, iw);
    kappa_prev = kappa;
    kappa = kappa_next;
    if (!fused) {   // bring the vector to unit length before the next step
      rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1.0 / kappa, 0, v, nullptr);
      if (rc) return rc;
      kappa = 1.0;
    }
  }
  if (plan) {
    rc = el::hv_tiled_error(ctx, plan);
    if (rc) return rc;
  }
  *emin = lo_prev;
  *emax = hi_prev;
  return EL_OK;
}

// ------------------------------------------------------------------- KPM

extern "C" int el_kpm_moments(el_ctx *ctx, el_ham *h, int dtype, int num, int nvec,
                              int chunk, uint64_t seed, const int8_t *probes_host,
                              int mode, double c, double r, double *mu_host) {
  if (!ctx || !h || !mu_host) return EL_EINVAL;
  if (dtype != EL_F32 && dtype != EL_F64) return fail(ctx, EL_EINVAL, "KPM vectors must be EL_F32 or EL_F64");
  if (h->complex_drive) return fail(ctx, EL_EINVAL, "KPM needs a real Hamiltonian (real Omega, J and A)");
  if (num < 1 || nvec < 1) return fail(ctx, EL_EINVAL, "num and nvec must be positive integers");
  if (chunk < 1 || chunk > 256 || (chunk & (chunk - 1))) return fail(ctx, EL_EINVAL, "chunk must be a power of two <= 256");
  if (!(r > 0) || !std::isfinite(r) || !std::isfinite(c)) return fail(ctx, EL_EINVAL, "bad scaling c, r");
  const bool force_generic = (mode & EL_KPM_GENERIC_KERNEL) != 0;
  mode &= ~EL_KPM_GENERIC_KERNEL;
  if (mode != EL_KPM_DIRECT && mode != EL_KPM_DOUBLING) return fail(ctx, EL_EINVAL, "unknown KPM mode");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!force_generic && mode == EL_KPM_DOUBLING && el::kpm_tma_eligible(h, dtype, chunk))
    return el::kpm_tma(ctx, h, dtype, num, nvec, chunk, seed, probes_host, c, r, mu_host);
  if (!force_generic && el::kpm_full_eligible(h, dtype, chunk, mode))
    return el::kpm_full(ctx, h, dtype, num, nvec, chunk, seed, probes_host, c, r, mu_host);
  const int64_t dim = h->basis->dim;
  const int es = el::dtype_size(dtype);
  const size_t vb = (size_t)dim * chunk * es;
  const bool direct = (mode == EL_KPM_DIRECT);
  const int nsteps = direct ? num : (num / 2 + 1);   // H applications per chunk
  const size_t dots_per = (size_t)chunk * 4;
  char *buf = (char *)el::workspace(ctx, 0, (direct ? 4 : 3) * vb);
  if (!buf) return EL_ENOMEM;
  double *d_dots = (double *)el::workspace(ctx, 1, (size_t)nsteps * dots_per * sizeof(double));
  if (!d_dots) return EL_ENOMEM;
  int8_t *d_probe8 = nullptr;
  if (probes_host) {
    d_probe8 = (int8_t *)el::workspace(ctx, 2, (size_t)dim * chunk);
    if (!d_probe8) return EL_ENOMEM;
  }
  void *t0 = buf, *t1 = buf + vb, *t2 = buf + 2 * vb;
  void *zp = direct ? (void *)(buf + 3 * vb) : nullptr;
  std::vector<double> acc(num + 1, 0.0);
  std::vector<double> hd((size_t)nsteps * dots_per);
  int rc;
  for (int done = 0; done < nvec; done += chunk) {
    const int b = std::min(chunk, nvec - done);
    // t0 = z (probes beyond b are zero vectors and contribute nothing)
    if (probes_host) {
      EL_CUDA_TRY(ctx, cudaMemsetAsync(d_probe8, 0, (size_t)dim * chunk, ctx->stream));
      EL_CUDA_TRY(ctx, el::copy(ctx, d_probe8, probes_host + (size_t)done * dim, (size_t)dim * b, cudaMemcpyHostToDevice));
      rc = el::launch_probe_copy(ctx, dtype, dim, chunk, d_probe8, t0);
    } else {
      rc = el::launch_fill_rademacher(ctx, dtype, dim, chunk, seed, done, b, t0);
    }
    if (rc) return rc;
    if (direct) EL_CUDA_TRY(ctx, el::copy(ctx, zp, t0, vb, cudaMemcpyDeviceToDevice));
    // first step: t1 = Htil t0 ; dots <t0,t0>, <t0,t1>
    ApplyArgs A;
    memset(&A, 0, sizeof A);
    A.dtype = dtype; A.nvec = chunk;
    A.x = t0; A.y = t1; A.a = 1.0 / r; A.b = -c / r;
    A.dots = d_dots; A.want_dots = 3;
    rc = el::launch_apply(ctx, h, A);
    if (rc) return rc;
    void *xm1 = t0, *x = t1, *y = t2;
    for (int s = 1; s < nsteps; ++s) {
      if ((s & 63) == 0 && el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = chunk;
      A.x = x; A.z = xm1; A.y = y;
      A.a = 2.0 / r; A.b = -2.0 * c / r; A.c = -1.0;
      A.dots = d_dots + (size_t)s * dots_per;
      A.want_dots = direct ? 4 : 3;
      A.probe = direct ? zp : nullptr;
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      void *t = xm1; xm1 = x; x = y; y = t;
    }
    EL_CUDA_TRY(ctx, el::copy(ctx, hd.data(), d_dots, hd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int v = 0; v < b; ++v) {
      const double *d0 = &hd[(size_t)v * 4];
      const double mu0 = d0[0], mu1 = d0[1];  // <z,z>, <z, Htil z>
      acc[0] += mu0;
      if (num >= 1) acc[1] += mu1;
      for (int s = 1; s < nsteps; ++s) {
        const double *ds = &hd[((size_t)s * chunk + v) * 4];
        if (direct) {
          // step s produced t_{s+1}; slot 2 holds <t_{s+1}, z>
          if (s + 1 <= num) acc[s + 1] += ds[2];
        } else {
          // step s has x = t_s, y = t_{s+1}
          if (2 * s <= num) acc[2 * s] += 2.0 * ds[0] - mu0;
          if (2 * s + 1 <= num) acc[2 * s + 1] += 2.0 * ds[1] - mu1;
        }
      }
    }
  }
  const double norm = 1.0 / ((double)nvec * (double)dim);
  for (int n = 0; n <= num; ++n) mu_host[n] = acc[n] * norm;
  return EL_OK;
}

// ---------------------------------------------------------------- Lanczos

extern "C" int el_lanczos_ground(el_ctx *ctx, el_ham *h, int dtype, const void *v0,
                                 uint64_t seed, int max_iter, int max_restarts,
                                 double tol, int nev, int reorth, double *evals,
                                 double *residuals, int *iters, int *converged,
                                 void *vec_out) {
  if (!ctx || !h || !evals || !residuals) return EL_EINVAL;
  if (!el::dtype_size(dtype)) return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  if (h->complex_drive && !is_cplx(dtype)) return fail(ctx, EL_EINVAL, "complex Omega, J or A needs a complex dtype");
  if (nev < 1 || nev > 2) return fail(ctx, EL_EINVAL, "nev must be 1 or 2");
  if (h->lossy) return fail(ctx, EL_EINVAL, "ground states need a Hermitian H (gamma = 0)");
  if (max_iter < 2 || max_restarts < 0) return fail(ctx, EL_EINVAL, "max_iter must be >= 2, max_restarts >= 0");
  if (!(tol > 0) || !std::isfinite(tol)) return fail(ctx, EL_EINVAL, "tol must be positive and finite");
  if (reorth < 0 || reorth > 2) return fail(ctx, EL_EINVAL, "reorth must be 0, 1 or 2");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t dim = h->basis->dim;
  const int es = el::dtype_size(dtype);
  const size_t vb = (size_t)dim * es;
  const int m = (int)std::min<int64_t>(max_iter, dim);
  const bool single = (dtype == EL_F32 || dtype == EL_C64);
  const double eps = single ? 1.19e-7 : 2.22e-16;
  // V: m+1 Krylov vectors (contiguous), w, x (Ritz), r (residual)
  char *Vb = (char *)el::workspace(ctx, 3, (size_t)(m + 1) * vb);
  char *Wb = (char *)el::workspace(ctx, 4, 3 * vb);
  if (!Vb || !Wb) return EL_ENOMEM;
  void *w = Wb, *xr = Wb + vb, *rv = Wb + 2 * vb;
  double *d_sc = ctx->d_scalars;           // [0..3] dots, [8] norm2
  double *d_coef = ctx->d_scalars + 64;    // [2*(m+1)] reorth coefficients
  if (2 * (m + 1) + 64 > EL_SCALARS) return fail(ctx, EL_EINVAL, "max_iter too large (<= %d)", EL_SCALARS / 2 - 40);
  auto Vj = [&](int j) { return (void *)(Vb + (size_t)j * vb); };
  int rc;
  // start vector
  if (v0) {
    EL_CUDA_TRY(ctx, el::copy(ctx, Vj(0), v0, vb, cudaMemcpyDeviceToDevice));
  } else {
    rc = el::launch_fill_gauss(ctx, dtype, dim, seed, Vj(0));
    if (rc) return rc;
  }
  int total_steps = 0;
  bool conv = false;
  std::vector<double> theta(nev, 0.0), resid(nev, 0.0);
  std::vector<std::vector<double>> svec(nev);
  int restart = 0;
  for (restart = 0; restart <= max_restarts; ++restart) {
    // normalise v_0
    rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, Vj(0), d_sc + 8);
    if (rc) return rc;
    double n2;
    rc = sync_read(ctx, d_sc + 8, 1, &n2);
    if (rc) return rc;
    if (!(n2 > 0) || !std::isfinite(n2)) return fail(ctx, EL_EINVAL, "start vector has zero or non-finite norm");
    rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1.0 / std::sqrt(n2), 0, Vj(0), nullptr);
    if (rc) return rc;
    std::vector<double> al, be;
    // omega recurrence state: wprev[k] ~ <v_{j-1}, v_k>, wcur[k] ~ <v_j, v_k>
    std::vector<double> wprev, wcur(1, 1.0), wnext;
    bool force_next = false;
    int j = 0;
    bool invariant = false;
    int last_check = -1;
    for (j = 0; j < m; ++j) {
      if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
      const double bj = j ? be[j - 1] : 0.0;
      ApplyArgs A;
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = Vj(j); A.z = j ? Vj(j - 1) : nullptr; A.y = w;
      A.a = 1.0; A.c = -bj; A.dots = d_sc; A.want_dots = 2;
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      double dots[4];
      rc = sync_read(ctx, d_sc, 4, dots);
      if (rc) return rc;
      const double alpha = dots[1];
      al.push_back(alpha);
      rc = el::launch_axpby(ctx, dtype, dim, -alpha, 0, Vj(j), 1, 0, w, d_sc + 8);
      if (rc) return rc;
      // reorthogonalisation decision
      const bool forced = force_next;
      bool do_reorth = (reorth == 2) || forced;
      double anorm = 0.0;
      for (size_t q = 0; q < al.size(); ++q) anorm = std::max(anorm, std::fabs(al[q]));
      for (size_t q = 0; q < be.size(); ++q) anorm = std::max(anorm, std::fabs(be[q]));
      rc = sync_read(ctx, d_sc + 8, 1, &n2);
      if (rc) return rc;
      double bnext = std::sqrt(std::max(n2, 0.0));
      if (reorth == 1 && j > 0 && bnext > 0) {
        // omega(j+1, k) per Simon (1984), k = 0..j-1
        wnext.assign(j + 2, 0.0);
        for (int k = 0; k < j; ++k) {
          const double bk1 = be[k];                 // couples k, k+1
          const double bk = k ? be[k - 1] : 0.0;    // couples k-1, k
          double t = bk1 * wcur[k + 1] + (al[k] - alpha) * wcur[k] - bj * (k < (int)wprev.size() ? wprev[k] : 0.0);
          if (k > 0) t += bk * wcur[k - 1];
          t /= bnext;
          t += (t >= 0 ? 1.0 : -1.0) * eps * anorm / bnext;
          wnext[k] = t;
        }
        wnext[j] = eps * std::sqrt((double)dim);
        wnext[j + 1] = 1.0;
        double wmax = 0.0;
        for (int k = 0; k < j; ++k) wmax = std::max(wmax, std::fabs(wnext[k]));
        if (wmax > std::sqrt(eps)) do_reorth = true;
      }
      force_next = false;
      if (do_reorth && j > 0) {
        for (int pass = 0; pass < 2; ++pass) {
          rc = el::launch_gemv_t(ctx, dtype, dim, j + 1, Vb, dim, w, d_coef);
          if (rc) return rc;
          rc = el::launch_gemv_n_sub(ctx, dtype, dim, j + 1, Vb, dim, d_coef, w);
          if (rc) return rc;
        }
        rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, w, d_sc + 8);
        if (rc) return rc;
        rc = sync_read(ctx, d_sc + 8, 1, &n2);
        if (rc) return rc;
        bnext = std::sqrt(std::max(n2, 0.0));
        if (reorth == 1) {
          for (int k = 0; k <= j; ++k) wnext[k] = eps;
          wnext[j + 1] = 1.0;
          force_next = !forced;   // Simon: the vector after a triggered step too, once
        }
      }
      if (reorth == 1) {
        if (j == 0) { wnext.assign(2, 0.0); wnext[0] = eps; wnext[1] = 1.0; }
        wprev.swap(wcur);
        wcur.swap(wnext);
      }
      total_steps++;
      const int mm = j + 1;
      const bool last = (j + 1 == m);
      const double scale = std::max(1.0, anorm);
      invariant = !(bnext > 1e-12 * scale);
      // convergence check every few steps
      if (mm >= nev && (invariant || last || mm - last_check >= 4)) {
        last_check = mm;
        bool ok = true;
        for (int q = 0; q < nev && q < mm; ++q) {
          theta[q] = el::tridiag_eig(al.data(), be.data(), mm, q);
          el::tridiag_vec(al.data(), be.data(), mm, theta[q], svec[q]);
          const double est = bnext * std::fabs(svec[q][mm - 1]);
          if (!(est <= 0.1 * tol * std::max(1.0, std::fabs(theta[q])))) ok = false;
        }
        if (ok || invariant || last) { j = mm; break; }
      }
      be.push_back(bnext);
      // v_{j+1} = w / beta
      rc = el::launch_axpby(ctx, dtype, dim, 1.0 / bnext, 0, w, 0, 0, Vj(j + 1), nullptr);
      if (rc) return rc;
    }
    const int mm = (int)al.size();
    // Ritz vectors and true residuals
    const int nq = std::min(nev, mm);
    for (int q = 0; q < nq; ++q) {
      theta[q] = el::tridiag_eig(al.data(), be.data(), mm, q);
      el::tridiag_vec(al.data(), be.data(), mm, theta[q], svec[q]);
      std::vector<double> coef(2 * mm, 0.0);
      for (int k = 0; k < mm; ++k) coef[2 * k] = svec[q][k];
      EL_CUDA_TRY(ctx, el::copy(ctx, d_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice));
      void *dst = (q == 0) ? xr : rv;
      rc = el::launch_gemv_n(ctx, dtype, dim, mm, Vb, dim, d_coef, dst);
      if (rc) return rc;
      // normalise
      rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, dst, d_sc + 8);
      if (rc) return rc;
      rc = sync_read(ctx, d_sc + 8, 1, &n2);
      if (rc) return rc;
      rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1.0 / std::sqrt(n2), 0, dst, nullptr);
      if (rc) return rc;
      // residual ||H x - theta x||
      ApplyArgs A;
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = dst; A.y = w; A.a = 1.0; A.b = -theta[q];
      A.dots = d_sc; A.want_dots = 4;
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      double dots[4];
      rc = sync_read(ctx, d_sc, 4, dots);
      if (rc) return rc;
      resid[q] = std::sqrt(std::max(dots[3], 0.0));
    }
    conv = (nq == nev);
    for (int q = 0; q < nq; ++q)
      if (!(resid[q] <= tol * std::max(1.0, std::fabs(theta[q])))) conv = false;
    if (conv || invariant || mm >= dim) {
      if (invariant || mm >= dim) {
        // exact Krylov space: residuals are rounding-level
        conv = true;
        for (int q = 0; q < nq; ++q)
          if (!(resid[q] <= std::max(tol, 1e3 * eps) * std::max(1.0, std::fabs(theta[q])))) conv = false;
      }
      break;
    }
    if (restart == max_restarts) break;
    // restart from the lowest Ritz vector (plus the second, if wanted)
    if (nev == 2 && nq == 2) {
      rc = el::launch_axpby(ctx, dtype, dim, 0.5, 0, rv, 1, 0, xr, nullptr);
      if (rc) return rc;
    }
    EL_CUDA_TRY(ctx, el::copy(ctx, Vj(0), xr, vb, cudaMemcpyDeviceToDevice));
    if (nev == 2 && nq == 2) {
      // recompute the ground Ritz vector is unnecessary: it is rebuilt next pass
    }
  }
  for (int q = 0; q < nev; ++q) { evals[q] = theta[q]; residuals[q] = resid[q]; }
  if (iters) *iters = total_steps;
  if (converged) *converged = conv ? 1 : 0;
  if (vec_out) {
    EL_CUDA_TRY(ctx, el::copy(ctx, vec_out, xr, vb, cudaMemcpyDeviceToDevice));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return EL_OK;
}

// ------------------------------------------------------- source-state Lanczos
// Lanczos tridiagonalisation of H from a given source state phi, as in
// spectrum.py:34-103 (lanczos): q_0 = phi/|phi|, w = H q_j, alpha_j =
// Re<q_j, w>, w -= alpha_j q_j + beta_{j-1} q_{j-1}; with reorth, w is
// orthogonalised twice against all q_0..q_j (classical Gram-Schmidt: all
// coefficients in one pass, then one update); beta_j = |w|; the run stops
// when beta_j <= 1e-12 or the Krylov space is the whole basis.  beta_j is
// stored only while another step follows (j + 1 < n_krylov), so betas has
// n - 1 entries.  ortho_loss = |<q_0, q_last>| of the last vector formed.
extern "C" int el_lanczos_tridiag(el_ctx *ctx, el_ham *h, int dtype, const void *phi, int n_krylov,
                                  int reorth, double *alphas, double *betas, int *n_out,
                                  double *norm2_out, double *ortho_loss, int *converged) {
  if (!ctx || !h || !phi || !alphas || !betas || !n_out) return EL_EINVAL;
  if (!el::dtype_size(dtype)) return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  if (h->complex_drive && !is_cplx(dtype)) return fail(ctx, EL_EINVAL, "complex Omega, J or A needs a complex dtype");
  if (n_krylov < 1) return fail(ctx, EL_EINVAL, "n_krylov must be positive");
  if (h->lossy) return fail(ctx, EL_EINVAL, "the Lanczos tridiagonalisation needs a Hermitian H (gamma = 0)");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t dim = h->basis->dim;
  const size_t vb = (size_t)dim * el::dtype_size(dtype);
  const int k = (int)std::min<int64_t>(n_krylov, dim);
  if (2 * (k + 1) + 64 > EL_SCALARS) return fail(ctx, EL_EINVAL, "n_krylov too large (<= %d)", EL_SCALARS / 2 - 40);
  char *Vb = (char *)el::workspace(ctx, 3, (size_t)(reorth ? k + 1 : 3) * vb);
  char *Wb = (char *)el::workspace(ctx, 4, vb);
  if (!Vb || !Wb) return EL_ENOMEM;
  void *w = Wb;
  double *d_sc = ctx->d_scalars;
  double *d_coef = ctx->d_scalars + 64;
  // with reorth every q_j is kept; without, three slots rotate
  auto Q = [&](int j) { return (void *)(Vb + (size_t)(reorth ? j : j % 3) * vb); };
  int rc;
  EL_CUDA_TRY(ctx, el::copy(ctx, Q(0), phi, vb, cudaMemcpyDeviceToDevice));
  rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, Q(0), d_sc + 8);
  if (rc) return rc;
  double n2;
  rc = sync_read(ctx, d_sc + 8, 1, &n2);
  if (rc) return rc;
  if (!(n2 > 0) || !std::isfinite(n2)) return fail(ctx, EL_EINVAL, "source state has zero or non-finite norm");
  rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1.0 / std::sqrt(n2), 0, Q(0), nullptr);
  if (rc) return rc;
  double beta = 0.0;
  int n = 0, nb = 0;
  bool conv = false;
  int last = 0;   // index of the last vector formed
  for (int j = 0; j < k; ++j) {
    if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
    ApplyArgs A;
    memset(&A, 0, sizeof A);
    A.dtype = dtype; A.nvec = 1; A.x = Q(j); A.z = j ? Q(j - 1) : nullptr; A.y = w;
    A.a = 1.0; A.c = -beta; A.dots = d_sc; A.want_dots = 2;
    rc = el::launch_apply(ctx, h, A);
    if (rc) return rc;
    double dots[4];
    rc = sync_read(ctx, d_sc, 4, dots);
    if (rc) return rc;
    const double alpha = dots[1];
    rc = el::launch_axpby(ctx, dtype, dim, -alpha, 0, Q(j), 1, 0, w, reorth ? nullptr : d_sc + 8);
    if (rc) return rc;
    if (reorth) {
      for (int pass = 0; pass < 2; ++pass) {
        rc = el::launch_gemv_t(ctx, dtype, dim, j + 1, Vb, dim, w, d_coef);
        if (rc) return rc;
        rc = el::launch_gemv_n_sub(ctx, dtype, dim, j + 1, Vb, dim, d_coef, w);
        if (rc) return rc;
      }
      rc = el::launch_axpby(ctx, dtype, dim, 0, 0, nullptr, 1, 0, w, d_sc + 8);
      if (rc) return rc;
    }
    double w2;
    rc = sync_read(ctx, d_sc + 8, 1, &w2);
    if (rc) return rc;
    beta = std::sqrt(std::max(w2, 0.0));
    alphas[n++] = alpha;
    if (beta <= 1e-12 || n >= dim) { conv = true; break; }
    if (j + 1 < k) betas[nb++] = beta;
    rc = el::launch_axpby(ctx, dtype, dim, 1.0 / beta, 0, w, 0, 0, Q(j + 1), nullptr);
    if (rc) return rc;
    last = j + 1;
    if (j + 1 == k && !reorth) break;
  }
  if (ortho_loss) {
    double ol = 0.0;
    if (reorth) {
      rc = el::launch_gemv_t(ctx, dtype, dim, 1, Q(last), dim, Q(0), d_sc);
      if (rc) return rc;
      double ov[2];
      rc = sync_read(ctx, d_sc, 2, ov);
      if (rc) return rc;
      ol = std::sqrt(ov[0] * ov[0] + (is_cplx(dtype) ? ov[1] * ov[1] : 0.0));
    }
    *ortho_loss = ol;
  }
  *n_out = n;
  if (norm2_out) *norm2_out = n2;
  if (converged) *converged = conv ? 1 : 0;
  return EL_OK;
}
