// Exact piecewise-constant time evolution by a Chebyshev propagator.
//
// One step replaces  psi <- expm_multiply(-i CONV tau H, psi)  of the
// reference (engine_ed.py:125 and engine_ed.py:145, CONV = 2 pi 1e-3 from
// evolve_util.py:12).  With H = a Htil + b and the spectrum of Htil inside
// [-1, 1] (a, b from the Gershgorin interval of H on the basis),
//     exp(-i x Htil) = J_0(x) + 2 sum_{m>=1} (-i)^m J_m(x) T_m(Htil),
//     x = a CONV tau,
// (the Jacobi-Anger expansion), multiplied by the global phase
// exp(-i b CONV tau).  Bessel values J_m(x) come from Miller's backward
// recurrence normalised by J_0 + 2 sum J_2k = 1.  The series is cut when the
// remaining coefficients fall below `tol`.  Each term is one fused kernel:
//     t_{m+1} = (2/a) H t_m - (2b/a) t_m - t_{m-1},  acc += c_{m+1} t_{m+1}.
#include "el_internal.cuh"

#include <algorithm>

namespace {

using el::fail;

constexpr double CONV = 2.0 * 3.14159265358979323846 * 1e-3;

// J_0..J_mmax(x) for x >= 0 by Miller's backward recurrence.
void bessel_j(double x, int mmax, std::vector<double> &J) {
  J.assign(mmax + 1, 0.0);
  if (x < 1e-300) { J[0] = 1.0; return; }
  const int start = 2 * ((std::max(mmax, (int)x) + 16 + (int)std::sqrt(40.0 * std::max(mmax, (int)x + 1))) / 2);
  std::vector<double> t(start + 2, 0.0);
  double jp1 = 0.0, j = 1e-300, norm = 0.0;
  for (int m = start; m >= 0; --m) {
    t[m] = j;
    if (m % 2 == 0) norm += (m == 0 ? 1.0 : 2.0) * j;
    const double jm1 = (m > 0) ? (2.0 * m / x) * j - jp1 : 0.0;
    jp1 = j;
    j = jm1;
    if (std::fabs(j) > 1e250) {
      // rescale everything computed so far
      for (int q = m - 1 < 0 ? 0 : m; q <= start; ++q) t[q] *= 1e-250;
      norm *= 1e-250;
      jp1 *= 1e-250;
      j *= 1e-250;
    }
  }
  for (int m = 0; m <= mmax; ++m) J[m] = t[m] / norm;
}

}  // namespace

namespace el {

int cheb_plan(el_ctx *ctx, el_ham *h, double tau_ns, double tol, ChebPlan *plan) {
  double lo, hi;
  int rc = gershgorin(ctx, h, &lo, &hi);
  if (rc) return rc;
  cheb_plan_bounds(lo, hi, tau_ns, tol, plan);
  return EL_OK;
}

void cheb_plan_bounds(double lo, double hi, double tau_ns, double tol, ChebPlan *plan) {
  plan->b = 0.5 * (hi + lo);
  plan->a = std::max(0.5 * (hi - lo) * (1.0 + 1e-6), 1e-12);
  const double x = plan->a * CONV * tau_ns;
  const double phi = plan->b * CONV * tau_ns;
  int mmax = (int)(x + 30.0 + 6.0 * std::cbrt(x + 1.0));
  std::vector<double> J;
  bessel_j(x, mmax, J);
  int M = 1;
  for (int m = mmax; m >= 1; --m)
    if (std::fabs(J[m]) * 2.0 > tol * 0.25) { M = m + 1; break; }
  M = std::min(M, mmax);
  plan->M = M;
  plan->c_re.assign(M + 1, 0.0);
  plan->c_im.assign(M + 1, 0.0);
  const double cph = std::cos(phi), sph = -std::sin(phi);
  for (int m = 0; m <= M; ++m) {
    const double mag = (m == 0 ? 1.0 : 2.0) * J[m];
    double pr, pi;
    switch (m & 3) {  // (-i)^m
      case 0: pr = 1; pi = 0; break;
      case 1: pr = 0; pi = -1; break;
      case 2: pr = -1; pi = 0; break;
      default: pr = 0; pi = 1; break;
    }
    plan->c_re[m] = mag * (pr * cph - pi * sph);
    plan->c_im[m] = mag * (pr * sph + pi * cph);
  }
}

}  // namespace el

extern "C" int el_cheb_step(el_ctx *ctx, el_ham *h, int dtype, void *psi,
                            double tau_ns, double tol, int *n_terms) {
  if (!ctx || !h || !psi) return EL_EINVAL;
  if (dtype != EL_C64 && dtype != EL_C128) return fail(ctx, EL_EINVAL, "evolution needs EL_C64 or EL_C128");
  if (!std::isfinite(tau_ns) || tau_ns < 0) return fail(ctx, EL_EINVAL, "tau must be finite and >= 0");
  if (!(tol > 0) || tol >= 1) return fail(ctx, EL_EINVAL, "tol must be in (0, 1)");
  if (h->lossy) return fail(ctx, EL_EINVAL, "the Chebyshev step needs a Hermitian H; use el_taylor_step with gamma != 0");
  if (n_terms) *n_terms = 0;
  if (tau_ns == 0.0) return EL_OK;
  if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t dim = h->basis->dim;
  const size_t vb = (size_t)dim * el::dtype_size(dtype);
  el::ChebPlan plan;
  int rc = el::cheb_plan(ctx, h, tau_ns, tol, &plan);
  if (rc) return rc;
  const double a = plan.a, b = plan.b;
  const int M = plan.M;
  auto coef = [&](int m, double *re, double *im) { *re = plan.c_re[m]; *im = plan.c_im[m]; };
  char *buf = (char *)el::workspace(ctx, 5, 4 * vb);
  if (!buf) return EL_ENOMEM;
  void *t0 = buf, *t1 = buf + vb, *t2 = buf + 2 * vb, *acc = buf + 3 * vb;
  EL_CUDA_TRY(ctx, el::copy(ctx, t0, psi, vb, cudaMemcpyDeviceToDevice));
  double cre, cim;
  coef(0, &cre, &cim);
  rc = el::launch_axpby(ctx, dtype, dim, cre, cim, t0, 0, 0, acc, nullptr);
  if (rc) return rc;
  // t1 = Htil t0 ; acc += c1 t1
  ApplyArgs A;
  memset(&A, 0, sizeof A);
  coef(1, &cre, &cim);
  A.dtype = dtype; A.nvec = 1; A.x = t0; A.y = t1; A.acc = acc;
  A.a = 1.0 / a; A.b = -b / a; A.w_re = cre; A.w_im = cim;
  rc = el::launch_apply(ctx, h, A);
  if (rc) return rc;
  void *xm1 = t0, *xc = t1, *y = t2;
  for (int m = 2; m <= M; ++m) {
    coef(m, &cre, &cim);
    memset(&A, 0, sizeof A);
    A.dtype = dtype; A.nvec = 1; A.x = xc; A.z = xm1; A.y = (m < M) ? y : nullptr; A.acc = acc;
    A.a = 2.0 / a; A.b = -2.0 * b / a; A.c = -1.0; A.w_re = cre; A.w_im = cim;
    rc = el::launch_apply(ctx, h, A);
    if (rc) return rc;
    void *t = xm1; xm1 = xc; xc = y; y = t;
  }
  EL_CUDA_TRY(ctx, el::copy(ctx, psi, acc, vb, cudaMemcpyDeviceToDevice));
  if (n_terms) *n_terms = M + 1;
  return EL_OK;
}

// ------------------------------------------------------------------- Taylor
// Non-Hermitian H (loss diagonal -i gamma/2): psi <- exp(A) psi with
// A = -i CONV tau H, the operation of expm_multiply in engine_ed.py:125,145
// for gamma != 0.  H is shifted by the centre c of its real Gershgorin
// interval [lo, hi] (a global phase exp(-i CONV tau c) put back in the term
// weights); then ||H - c|| <= (hi - lo)/2 + sum_k |loss_k| bounds the
// 1- and 2-norm (row and column sums agree: the off-diagonal part is
// Hermitian).  exp(A) is applied as s substeps exp(A/s) with
// ||A/s|| <= theta, each a Taylor polynomial of degree m, the smallest m
// whose remainder bound sum_{j>m} theta_s^j / j! is below tol / s.  With
// u_0 = psi, u_j = (CONV tau / (s j)) (H - c) u_{j-1}, the terms are
// e^{-i phi} (-i)^j u_j (phi = CONV tau c / s): one fused launch per term
// (real scale and shift on H x, complex weight on acc).
extern "C" int el_taylor_step(el_ctx *ctx, el_ham *h, int dtype, void *psi,
                              double tau_ns, double tol, int *n_terms) {
  if (!ctx || !h || !psi) return EL_EINVAL;
  if (dtype != EL_C64 && dtype != EL_C128) return fail(ctx, EL_EINVAL, "evolution needs EL_C64 or EL_C128");
  if (!std::isfinite(tau_ns) || tau_ns < 0) return fail(ctx, EL_EINVAL, "tau must be finite and >= 0");
  if (!(tol > 0) || tol >= 1) return fail(ctx, EL_EINVAL, "tol must be in (0, 1)");
  if (n_terms) *n_terms = 0;
  if (tau_ns == 0.0) return EL_OK;
  if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t dim = h->basis->dim;
  const size_t vb = (size_t)dim * el::dtype_size(dtype);
  double lo, hi, nrm;
  int rc = el::gershgorin(ctx, h, &lo, &hi, &nrm);
  if (rc) return rc;
  const double c = 0.5 * (lo + hi);
  double lsum = 0.0;
  for (int k = 0; k < h->n; ++k) lsum += std::fabs(h->loss[k]);
  const double bound = std::min(nrm + std::fabs(c), 0.5 * (hi - lo) + lsum);
  const double x = CONV * tau_ns * bound;
  const double theta = (dtype == EL_C128) ? 2.0 : 1.0;
  const int s = std::max(1, (int)std::ceil(x / theta));
  const double ths = x / s;
  // smallest m with sum_{j > m} ths^j / j! <= tol / s
  int m = 1;
  for (; m < 120; ++m) {
    double term = 1.0, rem = 0.0;
    for (int j = 1; j <= m + 80; ++j) {
      term *= ths / j;
      if (j > m) rem += term;
    }
    if (rem <= tol / s) break;
  }
  char *buf = (char *)el::workspace(ctx, 13, 3 * vb);
  if (!buf) return EL_ENOMEM;
  void *ta = buf, *tb = buf + vb, *acc = buf + 2 * vb;
  const double scale = CONV * tau_ns / s;
  const double cph = std::cos(scale * c), sph = -std::sin(scale * c);   // e^{-i phi}
  for (int step = 0; step < s; ++step) {
    if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
    rc = el::launch_axpby(ctx, dtype, dim, cph, sph, psi, 0, 0, acc, nullptr);   // acc = e^{-i phi} psi
    if (rc) return rc;
    const void *xc = psi;
    void *y = ta;
    for (int j = 1; j <= m; ++j) {
      ApplyArgs A;
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = xc; A.y = (j < m) ? y : nullptr; A.acc = acc;
      A.a = scale / j;
      A.b = -scale * c / j;
      double wr = 0, wi = 0;
      switch (j & 3) {  // (-i)^j
        case 0: wr = 1; break;
        case 1: wi = -1; break;
        case 2: wr = -1; break;
        default: wi = 1; break;
      }
      A.w_re = wr * cph - wi * sph;   // (-i)^j e^{-i phi}
      A.w_im = wr * sph + wi * cph;
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      xc = y;
      y = (y == ta) ? tb : ta;
    }
    EL_CUDA_TRY(ctx, el::copy(ctx, psi, acc, vb, cudaMemcpyDeviceToDevice));
  }
  if (n_terms) *n_terms = s * m;
  return EL_OK;
}
