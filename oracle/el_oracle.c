/*
 * el_oracle.c -- CPU restatement of the full-basis H-apply and the KPM
 * Chebyshev recurrence.  TEST INFRASTRUCTURE ONLY: used by the tests as a
 * checker and by bench.py as the timed CPU baseline; never linked into the
 * product library.
 *
 * Follows the reference semantics:
 *   diagonal d(s) = sum_i delta_i n_i + sum_{i<j} V_ij n_i n_j
 *       (src/core/manybody/channels.py:58-77)
 *   sigma^x channels with amplitude Omega_i/2 (real Omega here)
 *       (channels.py:114-118, ChannelKernel.matvec channels.py:210-221)
 *   KPM recurrence T0 z = z, T1 z = Htil z, T_n z = 2 Htil T_{n-1} z - T_{n-2} z,
 *   acc[n] += <T_n z, z>, mu = acc / (nvec * D)   (kpm.py:133-151)
 * Site 0 is the most significant bit (basis.py:6-9).
 * Vectors are blocks [dim][nvec] of doubles; rows are split over OpenMP threads.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

/* d[s] for all 2^n codes */
void oracle_diag_full(int n, const double *delta, int npairs, const int *pi,
                      const int *pj, const double *V, double *d) {
  const int64_t dim = (int64_t)1 << n;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < dim; ++s) {
    double acc = 0.0;
    for (int i = 0; i < n; ++i)
      if ((s >> (n - 1 - i)) & 1) acc += delta[i];
    for (int p = 0; p < npairs; ++p)
      if (((s >> (n - 1 - pi[p])) & 1) && ((s >> (n - 1 - pj[p])) & 1)) acc += V[p];
    d[s] = acc;
  }
}

/* y = a * (H x) + b * x + c * z  (z may be NULL); block [dim][nvec] */
void oracle_apply_full(int n, const double *omega, const double *d, int nvec,
                       double a, double b, double c, const double *x,
                       const double *z, double *y) {
  const int64_t dim = (int64_t)1 << n;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < dim; ++s) {
    double hx[256];
    const double *xs = x + s * nvec;
    for (int v = 0; v < nvec; ++v) hx[v] = d[s] * xs[v];
    for (int i = 0; i < n; ++i) {
      const double amp = 0.5 * omega[i];
      if (amp == 0.0) continue;
      const double *xt = x + (s ^ ((int64_t)1 << (n - 1 - i))) * nvec;
      for (int v = 0; v < nvec; ++v) hx[v] += amp * xt[v];
    }
    double *ys = y + s * nvec;
    for (int v = 0; v < nvec; ++v) {
      double r = a * hx[v] + b * xs[v];
      if (z) r += c * z[s * nvec + v];
      ys[v] = r;
    }
  }
}

/* mu[0..num]: probes int8 [nvec][dim]; returns 0 on success */
int oracle_kpm_full(int n, const double *omega, const double *d, double c,
                    double r, int num, int nvec, const int8_t *probes,
                    double *mu) {
  if (nvec < 1 || nvec > 256 || num < 1) return 1;
  const int64_t dim = (int64_t)1 << n;
  const size_t bytes = (size_t)dim * nvec * sizeof(double);
  double *z = (double *)malloc(bytes), *t0 = (double *)malloc(bytes);
  double *t1 = (double *)malloc(bytes), *t2 = (double *)malloc(bytes);
  if (!z || !t0 || !t1 || !t2) { free(z); free(t0); free(t1); free(t2); return 2; }
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < dim; ++s)
    for (int v = 0; v < nvec; ++v) z[s * nvec + v] = (double)probes[(int64_t)v * dim + s];
  memcpy(t0, z, bytes);
  double *acc = (double *)calloc((size_t)num + 1, sizeof(double));
  oracle_apply_full(n, omega, d, nvec, 1.0 / r, -c / r, 0.0, t0, NULL, t1);
  double s0 = 0.0, s1 = 0.0;
#pragma omp parallel for reduction(+ : s0, s1) schedule(static)
  for (int64_t i = 0; i < dim * nvec; ++i) { s0 += t0[i] * z[i]; s1 += t1[i] * z[i]; }
  acc[0] = s0;
  acc[1] = s1;
  for (int k = 2; k <= num; ++k) {
    oracle_apply_full(n, omega, d, nvec, 2.0 / r, -2.0 * c / r, -1.0, t1, t0, t2);
    double sk = 0.0;
#pragma omp parallel for reduction(+ : sk) schedule(static)
    for (int64_t i = 0; i < dim * nvec; ++i) sk += t2[i] * z[i];
    acc[k] = sk;
    double *tmp = t0; t0 = t1; t1 = t2; t2 = tmp;
  }
  for (int k = 0; k <= num; ++k) mu[k] = acc[k] / ((double)nvec * (double)dim);
  free(acc); free(z); free(t0); free(t1); free(t2);
  return 0;
}
