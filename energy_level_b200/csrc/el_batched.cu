// Batched Lanczos ground states: many independent Hamiltonians with uneven
// sector dimensions in ONE persistent launch.
//
// Every CTA pulls instances from an atomic queue (the host orders them by
// decreasing dimension, so the longest solves start first) and runs the whole
// three-term Lanczos recurrence of one instance on its own slice of the
// workspace:
//   w = H v_j - beta_j v_{j-1};  alpha_j = <v_j, w>;  w -= alpha_j v_j
// Vectors are FP32 (or FP64); alpha/beta, the omega recurrence of partial
// reorthogonalisation (Simon 1984) and the tridiagonal eigensolve are FP64.
// The two lowest Ritz values come from a warp-parallel Sturm multisection;
// the residual estimate beta_{j+1} |s_j| of the lowest pair from inverse
// iteration on one thread.  Convergence: residual estimate of both pairs
// <= tol * max(1, |theta|).  H follows channels.py:58-132 (diagonal
// delta n + V n n, sigma^x with Omega/2) on nearest-neighbour chain / ring
// blockade sectors (Zeckendorf ranking), full bases, or the blockade sector
// of any graph (TABLE: the instance's independent sets as an ascending code
// list, and a flip table of target rows built once at set-up); this is the batched
// counterpart of the reference's dense batched_ground_state
// (equilibrium.py:251-311) and of per-instance eigsh calls (eq_route.py:540).
#include "el_internal.cuh"

#include <algorithm>
#include <numeric>

namespace {

using el::fail;

constexpr int MAXIT = 384;      // Krylov steps per instance (workspace rows)
constexpr int MAXN = 40;        // sites per instance

struct Inst {
  int n, layout, pad0, pad1;
  int64_t dim, off;             // rows and offset into the concatenated diagonal
  double om[MAXN];              // Omega/2 per bit position
  // TABLE layout: this instance's ascending codes [dim] and flip table
  // [n][dim] (target row of flipping bit k of row r, -1 where the blockade
  // forbids it); null for the arithmetic layouts
  const uint64_t *codes;
  const int32_t *tgt;
};

struct BatchArgs {
  int count, max_iter, use_fp64, pad;
  double tol, eps;
  const Inst *inst;             // [count], processing order
  const double *diag;           // concatenated diagonal (FP64)
  void *ws;                     // per-CTA workspace: (max_iter + 2) * dim_max values
  int64_t dim_max;
  unsigned int *queue;
  uint64_t seed;
  double *e0, *e1, *res, *gap;  // outputs in processing order
  int *iters, *conv;
  double *nat;                  // [count][MAXN] ground-state <n_k> by bit position, or null
};


template <int NT>
__device__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += red[w];   // same order on every thread
  return s;
}

// Characteristic polynomials chi_k(x) = det(x I - T_k) of the leading k x k
// blocks of T (a[0..m-1], b[0..m-2]):
//   chi_0 = 1, chi_1 = x - a_0, chi_k = (x - a_{k-1}) chi_{k-1} - b_{k-2}^2 chi_{k-2}.
// The recurrence needs no division; the pair (chi_k, chi_{k-1}) is rescaled by
// a power of two whenever it grows large, which keeps signs and ratios exact.
__device__ __forceinline__ void rescale2(double &p, double &q) {
  const double ap = fabs(p);
  if (ap > 0x1p+400 || (ap < 0x1p-400 && ap > 0.0 && fabs(q) < 0x1p-400)) {
    const int e = ilogb(ap);
    p = scalbn(p, -e);
    q = scalbn(q, -e);
  }
}

// Number of eigenvalues of T below x: the number of k in 1..m at which
// chi_k(x) and chi_{k-1}(x) have the same sign (a zero counts as the sign
// opposite to its predecessor).
__device__ int sturm(const double *a, const double *b, int m, double x) {
  int cnt = 0;
  double pm = 1.0, p = x - a[0];
  double sprev = 1.0;
  double sp = (p == 0.0) ? -sprev : p;
  if (sp > 0) ++cnt;
  sprev = sp;
  for (int i = 1; i < m; ++i) {
    const double pn = fma(x - a[i], p, -(b[i - 1] * b[i - 1]) * pm);
    pm = p;
    p = pn;
    rescale2(p, pm);
    const double s = (p == 0.0) ? -sprev : p;
    if ((s > 0) == (sprev > 0)) ++cnt;
    sprev = s;
  }
  return cnt;
}

// k-th smallest eigenvalue by 32-way multisection within one warp.
__device__ double warp_eig(const double *a, const double *b, int m, int k, double lo, double hi) {
  const int lane = threadIdx.x & 31;
  for (int round = 0; round < 14; ++round) {
    const double x = lo + (hi - lo) * (lane + 1) / 33.0;
    const int c = sturm(a, b, m, x);
    const unsigned below = __ballot_sync(0xffffffffu, c > k);   // points above the eigenvalue
    const int first = below ? (__ffs(below) - 1) : 32;
    const double nlo = lo + (hi - lo) * first / 33.0;
    const double nhi = lo + (hi - lo) * (first + 1) / 33.0;
    lo = nlo;
    hi = nhi;
    if (hi - lo <= 1e-15 * fmax(1.0, fabs(hi))) break;
  }
  return 0.5 * (lo + hi);
}

// Last component of the unit eigenvector of T for eigenvalue lam (inverse
// iteration with a pivoted tridiagonal LU, one thread).
__device__ double last_component(const double *a, const double *b, int m, double lam, double *work) {
  if (m == 1) return 1.0;
  double *d = work, *u1 = work + m, *u2 = work + 2 * m, *l = work + 3 * m, *x = work + 4 * m;
  int *piv = (int *)(work + 5 * m);
  double scale = 0.0;
  for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(a[i]) + (i < m - 1 ? fabs(b[i]) : 0.0));
  const double eps = 2.2e-16 * fmax(scale, 1e-300);
  double cd = a[0] - lam, cu1 = b[0], cu2 = 0.0;
  for (int i = 0; i < m - 1; ++i) {
    const double sub = b[i], nd = a[i + 1] - lam, nu1 = (i + 1 < m - 1) ? b[i + 1] : 0.0;
    if (fabs(cd) >= fabs(sub)) {
      piv[i] = 0;
      double dv = fabs(cd) < eps ? (cd < 0 ? -eps : eps) : cd;
      const double f = sub / dv;
      l[i] = f; d[i] = dv; u1[i] = cu1; u2[i] = cu2;
      cd = nd - f * cu1; cu1 = nu1 - f * cu2; cu2 = 0.0;
    } else {
      piv[i] = 1;
      const double f = cd / sub;
      l[i] = f; d[i] = sub; u1[i] = nd; u2[i] = nu1;
      cd = cu1 - f * nd; cu1 = cu2 - f * nu1; cu2 = 0.0;
    }
  }
  d[m - 1] = fabs(cd) < eps ? (cd < 0 ? -eps : eps) : cd;
  for (int i = 0; i < m; ++i) d[i] = 1.0 / d[i];            // reciprocal pivots
  for (int i = 0; i < m; ++i) x[i] = 1.0 + 0.01 * sin(1.0 + i);
  for (int it = 0; it < 3; ++it) {
    for (int i = 0; i < m - 1; ++i) {
      if (piv[i]) { const double t = x[i]; x[i] = x[i + 1]; x[i + 1] = t; }
      x[i + 1] -= l[i] * x[i];
    }
    for (int i = m - 1; i >= 0; --i) {
      double s = x[i];
      if (i + 1 < m) s -= u1[i] * x[i + 1];
      if (i + 2 < m) s -= u2[i] * x[i + 2];
      x[i] = s * d[i];
    }
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) nrm += x[i] * x[i];
    nrm = sqrt(nrm);
    if (!(nrm > 0) || !isfinite(nrm)) return 1.0;
    const double inv = 1.0 / nrm;
    for (int i = 0; i < m; ++i) x[i] *= inv;
  }
  return fabs(x[m - 1]);
}

// Code of a row by the layout's arithmetic (FULL, CHAIN, RING).
__device__ __forceinline__ uint64_t unrank_arith(const Inst &I, const uint64_t *fib, int64_t row) {
  if (I.layout == EL_LAYOUT_FULL) return (uint64_t)row;
  uint64_t r = (uint64_t)row, c = 0;
  const int n = I.n;
  if (I.layout == EL_LAYOUT_CHAIN) {
    for (int k = n - 1; k >= 0; --k) { const uint64_t w = fib[k + 2]; if (r >= w) { c |= 1ULL << k; r -= w; } }
    return c;
  }
  if (r < fib[n + 1]) {
    for (int k = n - 2; k >= 0; --k) { const uint64_t w = fib[k + 2]; if (r >= w) { c |= 1ULL << k; r -= w; } }
    return c;
  }
  r -= fib[n + 1];
  c = 1ULL << (n - 1);
  for (int k = n - 3; k >= 1; --k) { const uint64_t w = fib[k + 1]; if (r >= w) { c |= 1ULL << k; r -= w; } }
  return c;
}

// Code of a row: from the instance's code list where it has one (TABLE
// instances, and chain / ring sectors, whose codes are listed once at
// set-up so that no Lanczos step ranks its rows again), else arithmetic.
__device__ __forceinline__ uint64_t unrank_b(const Inst &I, const uint64_t *fib, int64_t row) {
  if (I.codes) return I.codes[row];
  return unrank_arith(I, fib, row);
}

__device__ __forceinline__ int64_t ring_rank(const uint64_t *fib, int n, uint64_t c) {
  int64_t r = 0;
  if ((c >> (n - 1)) & 1ULL) {
    r = (int64_t)fib[n + 1];
    uint64_t m = c & ~(1ULL << (n - 1));
    while (m) { const int k = __ffsll((long long)m) - 1; r += (int64_t)fib[k + 1]; m &= m - 1; }
  } else {
    uint64_t m = c;
    while (m) { const int k = __ffsll((long long)m) - 1; r += (int64_t)fib[k + 2]; m &= m - 1; }
  }
  return r;
}

__device__ __forceinline__ int64_t flip_b(const Inst &I, const uint64_t *fib, uint64_t code,
                                          int64_t row, int k) {
  const uint64_t bit = 1ULL << k;
  const bool set = (code & bit) != 0;
  if (I.layout == EL_LAYOUT_FULL) return row ^ (int64_t)bit;
  if (I.layout == EL_LAYOUT_TABLE) return (int64_t)I.tgt[(int64_t)k * I.dim + row];
  const int n = I.n;
  uint64_t adj = 0;
  if (k + 1 < n) adj |= bit << 1;
  if (k > 0) adj |= bit >> 1;
  if (I.layout == EL_LAYOUT_RING) {
    if (k == 0) adj |= 1ULL << (n - 1);
    if (k == n - 1) adj |= 1ULL;
  }
  if (!set && (code & adj)) return -1;
  if (I.layout == EL_LAYOUT_CHAIN) {
    const int64_t w = (int64_t)fib[k + 2];
    return set ? row - w : row + w;
  }
  if (k == n - 1) return ring_rank(fib, n, code ^ bit);
  const bool top = (code >> (n - 1)) & 1ULL;
  const int64_t w = (int64_t)(top ? fib[k + 1] : fib[k + 2]);
  return set ? row - w : row + w;
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_lanczos_batch(const BatchArgs A) {
  __shared__ Inst I;
  __shared__ uint64_t fib[MAXN + 3];
  __shared__ double red[NT / 32];
  __shared__ double al[MAXIT], be[MAXIT];
  __shared__ double wcur[MAXIT + 2], wprev[MAXIT + 2];
  __shared__ double work[8 * MAXIT + 8];   // [0, MAXIT): omega row; [2 MAXIT, 8 MAXIT): projection coefficients, then inverse iteration
  __shared__ int s_idx, s_flag, s_done, s_force, s_trig, nsel;
  __shared__ short sel[MAXIT + 2];         // vectors of the current reorthogonalisation
  __shared__ double s_th[2], s_res[2], s_pth[2], s_pdth[2];
  __shared__ int s_have, s_next;
  const int tid = threadIdx.x;
  if (tid == 0) {
    fib[0] = 0; fib[1] = 1;
    for (int i = 2; i < MAXN + 3; ++i) fib[i] = fib[i - 1] + fib[i - 2];
  }
  T *Vb = reinterpret_cast<T *>(A.ws) + (size_t)blockIdx.x * (A.max_iter + 2) * A.dim_max;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_idx = (int)atomicAdd(A.queue, 1u);
    __syncthreads();
    const int idx = s_idx;
    if (idx >= A.count) break;
    if (tid == 0) I = A.inst[idx];
    __syncthreads();
    const int64_t dim = I.dim;
    const double *D = A.diag + I.off;
    const int m = (int)min((int64_t)A.max_iter, dim);
    T *W = Vb + (size_t)(A.max_iter + 1) * A.dim_max;
    // start vector: counter-based Gaussian, normalised
    double nrm = 0.0;
    for (int64_t r = tid; r < dim; r += NT) {
      const uint64_t h1 = el::counter_hash(A.seed + idx, 0x77, (uint64_t)r);
      const uint64_t h2 = el::counter_hash(A.seed + idx, 0x99, (uint64_t)r);
      const double u1 = ((h1 >> 11) + 1.0) * (1.0 / 9007199254740993.0);
      const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
      const T v = (T)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
      Vb[r] = v;
      nrm += (double)v * (double)v;
    }
    nrm = block_sum<NT>(nrm, red);
    {
      const T sc = (T)(1.0 / sqrt(nrm));
      for (int64_t r = tid; r < dim; r += NT) Vb[r] *= sc;
    }
    if (tid == 0) {
      wcur[0] = 1.0; s_force = 0; s_done = 0; s_th[0] = s_th[1] = 0.0; s_res[0] = s_res[1] = 1e300;
      s_have = 0; s_next = 8;
    }
    __syncthreads();
    double beta = 0.0, anorm = 0.0;
    int j = 0, steps = 0;
    for (j = 0; j < m; ++j) {
      const T *v = Vb + (size_t)j * A.dim_max;
      const T *vp = j ? Vb + (size_t)(j - 1) * A.dim_max : nullptr;
      // w = H v - beta v_prev ; alpha = <v, w>
      double pa = 0.0;
      for (int64_t r = tid; r < dim; r += NT) {
        const uint64_t code = unrank_b(I, fib, r);
        double h = D[r] * (double)v[r];
        for (int k = 0; k < I.n; ++k) {
          const double amp = I.om[k];
          if (amp == 0.0) continue;
          const int64_t t = flip_b(I, fib, code, r, k);
          if (t >= 0) h += amp * (double)v[t];
        }
        const T wv = (T)(h - (vp ? beta * (double)vp[r] : 0.0));
        W[r] = wv;
        pa += (double)v[r] * (double)wv;
      }
      const double alpha = block_sum<NT>(pa, red);
      double pn = 0.0;
      for (int64_t r = tid; r < dim; r += NT) {
        const T wv = (T)((double)W[r] - alpha * (double)v[r]);
        W[r] = wv;
        pn += (double)wv * (double)wv;
      }
      double b2 = block_sum<NT>(pn, red);
      anorm = fmax(anorm, fabs(alpha) + beta);
      double bnext = sqrt(fmax(b2, 0.0));
      // partial reorthogonalisation (Simon): one warp advances the omega
      // recurrence over k; when max |omega| exceeds sqrt(eps) the new vector
      // is orthogonalised against the v_k with |omega_k| >= eps^(3/4) (plus
      // v_{j-1}, v_j), and the next vector against the same set
      if (tid < 32) {
        const int forced = s_force;
        double wmax = 0.0;
        if (j > 0 && bnext > 0) {
          for (int k = tid; k < j; k += 32) {
            double t = be[k] * wcur[k + 1] + (al[k] - alpha) * wcur[k] - beta * wprev[k];
            if (k > 0) t += be[k - 1] * wcur[k - 1];
            t /= bnext;
            t += (t >= 0 ? 1.0 : -1.0) * A.eps * anorm / bnext;
            work[k] = t;
            wmax = fmax(wmax, fabs(t));
          }
          for (int o = 16; o > 0; o >>= 1) wmax = fmax(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        }
        const bool trig = (j > 0) && (bnext > 0) && (wmax > sqrt(A.eps)) && !forced;
        __syncwarp();
        if (trig) {
          const double eta = pow(A.eps, 0.75);
          int cnt = 0;
          for (int k0 = 0; k0 <= j; k0 += 32) {
            const int k = k0 + tid;
            const bool pick = (k <= j) && (k >= j - 1 || fabs(work[k]) >= eta);
            const unsigned bal = __ballot_sync(0xffffffffu, pick);
            if (pick) sel[cnt + __popc(bal & ((1u << tid) - 1u))] = (short)k;
            cnt += __popc(bal);
          }
          if (tid == 0) nsel = cnt;
        } else if (forced && tid == 0) {
          sel[nsel++] = (short)j;   // previous set (which holds j-1) plus the new v_j
        }
        if (tid == 0) {
          al[j] = alpha;
          s_force = 0;
          s_flag = (trig || forced) ? 1 : 0;
          s_trig = trig ? 1 : 0;
        }
      }
      __syncthreads();
      if (s_flag && j > 0) {
        // classical Gram-Schmidt, twice: each warp forms the dot products of
        // its share of v_0..v_j with w (FP64, fixed order), then every thread
        // subtracts all projections from its rows
        double *cf = work + 2 * MAXIT;
        for (int pass = 0; pass < 2; ++pass) {
          const int lane = tid & 31, warp = tid >> 5;
          const int ns = nsel;
          for (int q = warp; q < ns; q += NT / 32) {
            const T *vk = Vb + (size_t)sel[q] * A.dim_max;
            double pc0 = 0.0, pc1 = 0.0, pc2 = 0.0, pc3 = 0.0;
            int64_t r = lane;
            for (; r + 96 < dim; r += 128) {
              pc0 += (double)vk[r] * (double)W[r];
              pc1 += (double)vk[r + 32] * (double)W[r + 32];
              pc2 += (double)vk[r + 64] * (double)W[r + 64];
              pc3 += (double)vk[r + 96] * (double)W[r + 96];
            }
            for (; r < dim; r += 32) pc0 += (double)vk[r] * (double)W[r];
            double pc = (pc0 + pc1) + (pc2 + pc3);
            for (int o = 16; o > 0; o >>= 1) pc += __shfl_xor_sync(0xffffffffu, pc, o);
            if (lane == 0) cf[q] = pc;
          }
          __syncthreads();
          for (int64_t r = tid; r < dim; r += NT) {
            const T *col = Vb + r;
            double w0 = (double)W[r], w1 = 0.0, w2 = 0.0, w3 = 0.0;
            int q = 0;
            for (; q + 4 <= ns; q += 4) {
              const double v0 = (double)col[(size_t)sel[q] * A.dim_max];
              const double v1 = (double)col[(size_t)sel[q + 1] * A.dim_max];
              const double v2 = (double)col[(size_t)sel[q + 2] * A.dim_max];
              const double v3 = (double)col[(size_t)sel[q + 3] * A.dim_max];
              w0 -= cf[q] * v0;
              w1 -= cf[q + 1] * v1;
              w2 -= cf[q + 2] * v2;
              w3 -= cf[q + 3] * v3;
            }
            for (; q < ns; ++q) w0 -= cf[q] * (double)col[(size_t)sel[q] * A.dim_max];
            W[r] = (T)((w0 + w1) + (w2 + w3));
          }
          __syncthreads();
        }
        double pn2 = 0.0;
        for (int64_t r = tid; r < dim; r += NT) pn2 += (double)W[r] * (double)W[r];
        b2 = block_sum<NT>(pn2, red);
        bnext = sqrt(fmax(b2, 0.0));
      }
      if (tid == 0) {
        // advance the omega recurrence (reset after a reorthogonalisation)
        if (j == 0) {
          wprev[0] = 1.0;
          wcur[0] = A.eps; wcur[1] = 1.0;
        } else {
          for (int k = 0; k <= j - 1; ++k) wprev[k] = wcur[k];
          wprev[j] = wcur[j];
          for (int k = 0; k < j; ++k) wcur[k] = work[k];
          wcur[j] = A.eps * sqrt((double)dim);
          if (s_flag)
            for (int q = 0; q < nsel; ++q) wcur[sel[q]] = A.eps;
          if (s_trig) s_force = 1;   // the next vector is orthogonalised against the same set
          wcur[j + 1] = 1.0;
        }
        be[j] = bnext;
      }
      __syncthreads();   // al/be/omega rows visible to warp 0 and everyone
      steps = j + 1;
      const bool invariant = !(bnext > 1e-12 * fmax(1.0, anorm));
      // Ritz check every 8 steps (every 32 while the residuals are far from
      // tolerance); the multisection starts from the previous Ritz values,
      // upper bounds by Cauchy interlacing, with a Sturm-confirmed narrow
      // lower bound when one holds
      const bool check = invariant || (j + 1 == m) || ((steps >= 2) && (steps >= s_next));
      if (check && tid < 32) {
        const int mm = steps;
        double glo = 1e300, ghi = -1e300;
        for (int i = 0; i < mm; ++i) {
          const double rr = (i > 0 ? fabs(be[i - 1]) : 0.0) + (i + 1 < mm ? fabs(be[i]) : 0.0);
          glo = fmin(glo, al[i] - rr);
          ghi = fmax(ghi, al[i] + rr);
        }
        const double scale = fmax(1.0, fmax(fabs(glo), fabs(ghi)));
        glo -= 1e-9 * scale;
        ghi += 1e-9 * scale;
        const int ne = mm >= 2 ? 2 : 1;
        double worst = 0.0;
        for (int q = 0; q < ne; ++q) {
          double lo = glo, hi = ghi;
          if (s_have) {
            hi = fmin(ghi, s_pth[q] + 1e-12 * scale);
            const double cand = hi - fmax(16.0 * s_pdth[q], 1e-10 * scale);
            if (cand > glo && sturm(al, be, mm, cand) <= q) lo = cand;
          }
          const double th = warp_eig(al, be, mm, q, lo, hi);
          if (tid == 0) {
            s_pdth[q] = s_have ? fmax(s_pth[q] - th, 0.0) : fabs(ghi - glo);
            s_pth[q] = th;
            s_th[q] = th;
            s_res[q] = bnext * last_component(al, be, mm, th, work + 2 * MAXIT);
            worst = fmax(worst, s_res[q] / (A.tol * fmax(1.0, fabs(th))));
          }
          __syncwarp();
        }
        if (tid == 0) {
          bool ok = (ne == 2);
          for (int q = 0; q < ne; ++q) ok = ok && (s_res[q] <= A.tol * fmax(1.0, fabs(s_th[q])));
          s_done = (ok || invariant || j + 1 == m) ? 1 : 0;
          s_have = (ne == 2) ? 1 : 0;
          s_next = mm + (worst > 1e3 ? 32 : 8);
        }
      }
      __syncthreads();
      if (s_done) break;
      // v_{j+1} = w / beta
      T *vn = Vb + (size_t)(j + 1) * A.dim_max;
      const double inv = 1.0 / bnext;
      for (int64_t r = tid; r < dim; r += NT) vn[r] = (T)((double)W[r] * inv);
      beta = bnext;
      __syncthreads();
    }
    if (tid == 0) {
      A.e0[idx] = s_th[0];
      A.e1[idx] = s_th[1];
      A.gap[idx] = s_th[1] - s_th[0];
      A.res[idx] = fmax(s_res[0], s_res[1]);
      A.iters[idx] = steps;
      A.conv[idx] = (s_res[0] <= A.tol * fmax(1.0, fabs(s_th[0])) &&
                     s_res[1] <= A.tol * fmax(1.0, fabs(s_th[1]))) ? 1 : 0;
    }
    if (A.nat) {
      // site occupations of the ground-state Ritz vector x = sum_j y_j v_j
      // (y: unit eigenvector of T for theta_0, by inverse iteration):
      // <n_k> = sum_r x_r^2 bit_k(r) / sum_r x_r^2, fixed-order block sums
      __syncthreads();
      if (tid == 0) {
        if (steps == 1) work[2 * MAXIT + 4] = 1.0;   // a one-vector Krylov space
        else last_component(al, be, steps, s_th[0], work + 2 * MAXIT);
      }
      __syncthreads();
      const double *y = work + 2 * MAXIT + 4 * steps;
      // lane l of each warp owns bit positions l and l + 32: the warp's rows
      // pass by shuffles, so no thread keeps a per-site array
      const int lane = tid & 31;
      double occ_lo = 0.0, occ_hi = 0.0, tot = 0.0;
      for (int64_t r0 = tid - lane; r0 < dim; r0 += NT) {
        const int64_t r = r0 + lane;
        double p2 = 0.0;
        uint64_t code = 0;
        if (r < dim) {
          double x = 0.0;
          for (int jj = 0; jj < steps; ++jj) x += y[jj] * (double)Vb[(size_t)jj * A.dim_max + r];
          p2 = x * x;
          code = unrank_b(I, fib, r);
        }
        tot += p2;
        for (int src = 0; src < 32; ++src) {
          const double ps = __shfl_sync(0xffffffffu, p2, src);
          const uint64_t cs = __shfl_sync(0xffffffffu, code, src);
          if ((cs >> lane) & 1ULL) occ_lo += ps;
          if (lane + 32 < MAXN && ((cs >> (lane + 32)) & 1ULL)) occ_hi += ps;
        }
      }
      tot = block_sum<NT>(tot, red);
      for (int k = 0; k < I.n; ++k) {
        const double mine = (lane == (k & 31)) ? (k < 32 ? occ_lo : occ_hi) : 0.0;
        const double sk = block_sum<NT>(mine, red);
        if (tid == 0) A.nat[(size_t)idx * MAXN + k] = tot > 0 ? sk / tot : 0.0;
      }
    }
  }
}

// ------------------------------------------------ one instance, whole GPU
// Cooperative Lanczos for one instance that is too small to fill the GPU
// with vectors but too slow on one SM: the rows are split over G CTAs (NT
// rows each, one row per thread) and every CTA keeps its slice of the
// Krylov basis in shared memory, so the full reorthogonalisation (classical
// Gram-Schmidt, twice, every step) touches only shared memory; the
// coefficients are summed across CTAs through small global arrays.  A step
// needs two grid barriers per projection sum (partials, then the sums, each
// formed by one CTA) -- the last one also carries |w|^2 before it, so that
// |w_final|^2 = |w|^2 - |c|^2 costs no further barrier -- and one to publish
// the next vector, whose entries the sigma^x flips of every CTA read: five
// with two Gram-Schmidt passes, three with one.  Every sum is
// formed once, in a fixed order, and read by all CTAs, so every CTA holds
// the same alpha/beta bits and takes the same decisions.  The grid barrier is a
// monotonic arrival counter polled by one thread per CTA with a bounded
// number of polls; a timeout sets the error flag, after which no barrier
// waits again and the kernel runs out its bounded loop.
struct CoopArgs {
  int p, m, nctas, check_every, passes, pad2;
  double tol, eps;
  const Inst *inst;
  const double *diag;
  void *vpub;                   // [dim] the current Lanczos vector, published
  double *part;                 // [2][nctas][MAXIT + 2] per-CTA partial sums
  double *tot;                  // [2][MAXIT + 2] the sums, each formed by one CTA
  unsigned *bar;                // arrival counter, zero at launch
  int *err;
  int poll_limit;               // polls per barrier before giving up
  uint64_t seed;
  double *e0, *e1, *res, *gap;
  int *iters, *conv;
  double *nat;                  // [count][MAXN] ground-state <n_k>, or null
};

__device__ __forceinline__ void grid_barrier(const CoopArgs &G, unsigned &gen) {
  __syncthreads();
  gen += (unsigned)G.nctas;
  if (threadIdx.x == 0) {
    // release this CTA's writes with the arrival, acquire the others' with
    // the poll that sees the count complete
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(G.bar) : "memory");
    if (!*(volatile int *)G.err) {
      int polls = 0;
      unsigned v;
      for (;;) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(G.bar) : "memory");
        if (v >= gen) break;
        if (++polls > G.poll_limit) { atomicExch(G.err, 1); break; }
        if ((polls & 255) == 0 && *(volatile int *)G.err) break;
      }
    }
  }
  __syncthreads();
}

// Dynamic shared memory of the cooperative kernel: the Krylov slice
// [m + 1][NT + 1] then two inverse-iteration buffers.
__host__ __device__ inline size_t coop_slice_bytes(int m, int nt, int es) {
  return (((size_t)(m + 1) * (nt + 1) * es) + 15) / 16 * 16;
}
constexpr size_t COOP_WORK_BYTES = 2 * (6 * MAXIT + 8) * sizeof(double);

// Per-CTA partial sums of the ground-state occupations: x = sum_j y_j v_j on
// this thread's row (v_j in the CTA's Krylov slice), out[k] = sum over the
// CTA's rows of x^2 bit_k, out[n] = sum of x^2 (kept out of line: it runs
// once per solve and must not add to the main loop's registers).
template <typename T, int NT>
__device__ __noinline__ void coop_occupation_partials(const double *y, const T *Vs, int pitch, int steps,
                                                      bool valid, uint64_t code, int n, double *red,
                                                      double *out) {
  double x = 0.0;
  if (valid)
    for (int jj = 0; jj < steps; ++jj) x += y[jj] * (double)Vs[(size_t)jj * pitch + threadIdx.x];
  const double p2 = x * x;
  for (int k = 0; k < n; ++k) {
    const double sk = block_sum<NT>(((code >> k) & 1ULL) ? p2 : 0.0, red);
    if (threadIdx.x == 0) out[k] = sk;
  }
  const double tot = block_sum<NT>(p2, red);
  if (threadIdx.x == 0) out[n] = tot;
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_lanczos_coop(const CoopArgs G) {
  extern __shared__ __align__(16) unsigned char coop_smem[];
  T *Vs = reinterpret_cast<T *>(coop_smem);           // [m + 1][NT + 1]
  constexpr int PITCH = NT + 1;
  __shared__ Inst I;
  __shared__ uint64_t fib[MAXN + 3];
  __shared__ double red[NT / 32 > 0 ? NT / 32 : 1];
  __shared__ double al[MAXIT], be[MAXIT];
  __shared__ double cs[MAXIT + 2];
  __shared__ T wsm[NT];
  __shared__ double s_th[2], s_res[2];
  __shared__ double prev_th[2], prev_dth[2];
  __shared__ int have_prev, s_next;
  __shared__ int s_done, s_err;
  const int tid = threadIdx.x;
  if (tid == 0) {
    fib[0] = 0; fib[1] = 1;
    for (int i = 2; i < MAXN + 3; ++i) fib[i] = fib[i - 1] + fib[i - 2];
    I = G.inst[G.p];
    s_err = 0;
    have_prev = 0;
    s_next = 16;
    s_th[0] = s_th[1] = 0.0; s_res[0] = s_res[1] = 1e300; s_done = 0;
  }
  __syncthreads();
  const int64_t dim = I.dim;
  const int64_t row = (int64_t)blockIdx.x * NT + tid;
  const bool valid = row < dim;
  const double *D = G.diag + I.off;
  T *vpub = reinterpret_cast<T *>(G.vpub);
  const int m = (int)min((int64_t)G.m, dim);
  // inverse-iteration buffers of lanes 0 and 1 follow the slice in dynamic memory
  double *work = reinterpret_cast<double *>(coop_smem + coop_slice_bytes(m, NT, (int)sizeof(T)));
  unsigned gen = 0;
  int slot = 0;
  auto part = [&](int sl, int c, int k) -> double * {
    return G.part + ((size_t)sl * G.nctas + c) * (MAXIT + 2) + k;
  };
  // partials part(slot, *, k), k < nk, written -> cs[k] = their sum in
  // every CTA.  CTA c forms the sums k = c, c + G, ... (one warp per sum,
  // lanes over CTAs, fixed tree) into tot, then every CTA reads tot: two
  // barriers, O(nk) loads per CTA instead of O(nk x G)
  auto reduce_all = [&](int nk) {
    grid_barrier(G, gen);
    const int lane = tid & 31, warp = tid >> 5;
    double *tt = G.tot + (size_t)slot * (MAXIT + 2);
    for (int k = blockIdx.x + warp * G.nctas; k < nk; k += G.nctas * (NT / 32)) {
      double v = 0.0;
      for (int cc = lane; cc < G.nctas; cc += 32) v += __ldcg(part(slot, cc, k));
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) tt[k] = v;
    }
    grid_barrier(G, gen);
    for (int k = tid; k < nk; k += NT) cs[k] = __ldcg(&tt[k]);
    slot ^= 1;
    __syncthreads();
  };
  // sum over CTAs of a block-reduced scalar
  auto grid_scalar = [&](double v) -> double {
    v = block_sum<NT>(v, red);
    if (tid == 0) *part(slot, blockIdx.x, 0) = v;
    reduce_all(1);
    return cs[0];
  };
  // start vector: counter-based Gaussian (same stream as the batched kernel)
  double x0 = 0.0;
  if (valid) {
    const uint64_t h1 = el::counter_hash(G.seed + G.p, 0x77, (uint64_t)row);
    const uint64_t h2 = el::counter_hash(G.seed + G.p, 0x99, (uint64_t)row);
    const double u1 = ((h1 >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    x0 = (double)(T)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
  }
  const double n0 = grid_scalar(x0 * x0);
  {
    const T v = (T)(x0 / sqrt(n0));
    Vs[tid] = valid ? v : (T)0;
    if (valid) vpub[row] = v;
  }
  grid_barrier(G, gen);
  int steps = 0;
  double bnext = 0.0, anorm = 0.0;
  for (int j = 0; j < m; ++j) {
    // a barrier timed out somewhere: stop (the flag is read once per CTA)
    if (tid == 0) s_err = *(volatile int *)G.err;
    __syncthreads();
    if (s_err) break;
    // w = H v_j (flip partners read from the published vector)
    double w = 0.0;
    if (valid) {
      const uint64_t code = unrank_b(I, fib, row);
      w = D[row] * (double)Vs[(size_t)j * PITCH + tid];
      for (int k = 0; k < I.n; ++k) {
        const double amp = I.om[k];
        if (amp == 0.0) continue;
        const int64_t t = flip_b(I, fib, code, row, k);
        if (t >= 0) w += amp * (double)__ldcg(&vpub[t]);
      }
    }
    // classical Gram-Schmidt against v_0..v_j, G.passes times; alpha = sum
    // of the v_j coefficients.  The last pass also sums |w|^2 (slot j + 1).
    double alpha = 0.0, b2 = 0.0;
    for (int pass = 0; pass < G.passes; ++pass) {
      const int last_pass = (pass == G.passes - 1);
      wsm[tid] = (T)w;
      __syncthreads();
      for (int k = tid; k <= j; k += NT) {
        const T *vk = Vs + (size_t)k * PITCH;
        double c0 = 0.0, c1 = 0.0;
        int r = 0;
        for (; r + 1 < NT; r += 2) {
          c0 += (double)vk[r] * (double)wsm[r];
          c1 += (double)vk[r + 1] * (double)wsm[r + 1];
        }
        for (; r < NT; ++r) c0 += (double)vk[r] * (double)wsm[r];
        *part(slot, blockIdx.x, k) = c0 + c1;
      }
      if (last_pass) {
        const double ww = block_sum<NT>(valid ? w * w : 0.0, red);
        if (tid == 0) *part(slot, blockIdx.x, j + 1) = ww;
      }
      reduce_all(j + 1 + last_pass);
      alpha += cs[j];
      if (last_pass) {
        double cc2 = 0.0;
        for (int k = 0; k <= j; ++k) cc2 += cs[k] * cs[k];
        b2 = cs[j + 1] - cc2;
      }
      if (valid) {
        double acc0 = w, acc1 = 0.0;
        int k = 0;
        for (; k + 1 <= j; k += 2) {
          acc0 -= cs[k] * (double)Vs[(size_t)k * PITCH + tid];
          acc1 -= cs[k + 1] * (double)Vs[(size_t)(k + 1) * PITCH + tid];
        }
        for (; k <= j; ++k) acc0 -= cs[k] * (double)Vs[(size_t)k * PITCH + tid];
        w = (double)(T)(acc0 + acc1);
      }
      __syncthreads();
    }
    bnext = sqrt(fmax(b2, 0.0));
    anorm = fmax(anorm, fabs(alpha) + bnext);
    if (tid == 0) { al[j] = alpha; be[j] = bnext; }
    __syncthreads();
    steps = j + 1;
    const int next_check = s_next;
    const bool invariant = !(bnext > 1e-12 * fmax(1.0, anorm));
    // Ritz values and residual estimates at step next_check (and at the
    // end).  By Cauchy interlacing the q-th Ritz value never rises as the
    // tridiagonal grows, so the previous value bounds it from above; a
    // Sturm count confirms a narrow lower bound below it (else the
    // Gershgorin bound is used), which saves most multisection rounds.  The
    // two residual estimates (inverse iteration) run on lanes 0 and 1.
    const bool check = invariant || (j + 1 == m) || (steps >= next_check);
    if (check && tid < 32) {
      const int mm = steps;
      double glo = 1e300, ghi = -1e300;
      for (int i = 0; i < mm; ++i) {
        const double rr = (i > 0 ? fabs(be[i - 1]) : 0.0) + (i + 1 < mm ? fabs(be[i]) : 0.0);
        glo = fmin(glo, al[i] - rr);
        ghi = fmax(ghi, al[i] + rr);
      }
      const double scale = fmax(1.0, fmax(fabs(glo), fabs(ghi)));
      glo -= 1e-9 * scale;
      ghi += 1e-9 * scale;
      const int ne = mm >= 2 ? 2 : 1;
      double th[2] = {0.0, 0.0};
      for (int q = 0; q < ne; ++q) {
        double lo = glo, hi = ghi;
        if (have_prev) {
          hi = fmin(ghi, prev_th[q] + 1e-12 * scale);
          const double d = fmax(16.0 * prev_dth[q], 1e-10 * scale);
          const double cand = hi - d;
          if (cand > glo && sturm(al, be, mm, cand) <= q) lo = cand;
        }
        th[q] = warp_eig(al, be, mm, q, lo, hi);
      }
      if (tid < ne) {
        const double r = bnext * last_component(al, be, mm, th[tid], work + (size_t)tid * (6 * MAXIT + 8));
        s_res[tid] = r;
        s_th[tid] = th[tid];
      }
      __syncwarp();
      if (tid == 0) {
        bool ok = (ne == 2);
        double worst = 0.0;
        for (int q = 0; q < ne; ++q) {
          const double lim = G.tol * fmax(1.0, fabs(s_th[q]));
          ok = ok && (s_res[q] <= lim);
          worst = fmax(worst, s_res[q] / lim);
        }
        s_done = (ok || invariant || j + 1 == m) ? 1 : 0;
        // far from converged: look again later
        s_next = mm + (worst > 1e3 ? 4 : 1) * G.check_every;
      }
      if (tid < ne) {
        prev_dth[tid] = have_prev ? fmax(prev_th[tid] - th[tid], 0.0) : fabs(ghi - glo);
        prev_th[tid] = th[tid];
      }
      if (tid == 0) have_prev = 1;
    }
    __syncthreads();
    if (s_done) break;
    // v_{j+1} = w / beta, into the shared slice and the published vector
    const T vn = (T)(w / bnext);
    Vs[(size_t)(j + 1) * PITCH + tid] = valid ? vn : (T)0;
    if (valid) vpub[row] = vn;
    grid_barrier(G, gen);
  }
  if (G.nat) {
    // site occupations of the ground-state Ritz vector (as in the batched
    // kernel): every CTA forms y from the same alpha/beta, its rows of x from
    // its Krylov slice, and per-site partial sums that reduce_all adds up
    __syncthreads();
    if (tid == 0) {
      if (steps <= 1) work[4] = 1.0;
      else last_component(al, be, steps, s_th[0], work);
    }
    __syncthreads();
    coop_occupation_partials<T, NT>(work + 4 * (steps <= 1 ? 1 : steps), Vs, PITCH, steps, valid,
                                    valid ? unrank_b(I, fib, row) : 0, I.n, red,
                                    part(slot, blockIdx.x, 0));
    reduce_all(I.n + 1);
    if (blockIdx.x == 0 && tid < I.n)
      G.nat[(size_t)G.p * MAXN + tid] = cs[I.n] > 0 ? cs[tid] / cs[I.n] : 0.0;
  }
  if (blockIdx.x == 0 && tid == 0) {
    const int p = G.p;
    G.e0[p] = s_th[0];
    G.e1[p] = s_th[1];
    G.gap[p] = s_th[1] - s_th[0];
    G.res[p] = fmax(s_res[0], s_res[1]);
    G.iters[p] = steps;
    G.conv[p] = (!*(volatile int *)G.err && s_res[0] <= G.tol * fmax(1.0, fabs(s_th[0])) &&
                 s_res[1] <= G.tol * fmax(1.0, fabs(s_th[1]))) ? 1 : 0;
  }
}

// Code lists of the chain and ring instances (the arithmetic unranking, once).
__global__ void k_batch_fill_codes(int count, const Inst *inst) {
  __shared__ uint64_t fib[MAXN + 3];
  if (threadIdx.x == 0) {
    fib[0] = 0; fib[1] = 1;
    for (int i = 2; i < MAXN + 3; ++i) fib[i] = fib[i - 1] + fib[i - 2];
  }
  __syncthreads();
  for (int i = blockIdx.y; i < count; i += gridDim.y) {
    const Inst &I = inst[i];
    if (I.layout != EL_LAYOUT_CHAIN && I.layout != EL_LAYOUT_RING) continue;
    uint64_t *out = const_cast<uint64_t *>(I.codes);
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < I.dim; r += (int64_t)gridDim.x * blockDim.x)
      out[r] = unrank_arith(I, fib, r);
  }
}

// Flip tables of the TABLE instances: target row of flipping bit k of row r,
// found by binary search in the instance's ascending code list; -1 when bit
// k is clear and one of its graph neighbours (adj, by bit position) is set.
__global__ void k_batch_flip_table(int count, const Inst *inst, const uint64_t *adj) {
  for (int i = blockIdx.y; i < count; i += gridDim.y) {
    const Inst &I = inst[i];
    if (I.layout != EL_LAYOUT_TABLE) continue;
    const int64_t cells = I.dim * I.n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cells;
         e += (int64_t)gridDim.x * blockDim.x) {
      const int k = (int)(e / I.dim);
      const int64_t r = e - (int64_t)k * I.dim;
      const uint64_t code = I.codes[r], bit = 1ULL << k;
      int32_t t = -1;
      if ((code & bit) || !(code & adj[(size_t)i * MAXN + k])) {
        const uint64_t want = code ^ bit;
        int64_t lo = 0, hi = I.dim - 1;
        while (lo < hi) {
          const int64_t mid = (lo + hi) >> 1;
          if (I.codes[mid] < want) lo = mid + 1;
          else hi = mid;
        }
        if (I.codes[lo] == want) t = (int32_t)lo;
      }
      const_cast<int32_t *>(I.tgt)[e] = t;
    }
  }
}

// diagonal of every instance: V part + delta part, concatenated
__global__ void k_batch_diag(int count, const Inst *inst, const double *Vmats, const double *deltas,
                             double *diag) {
  __shared__ uint64_t fib[MAXN + 3];
  if (threadIdx.x == 0) {
    fib[0] = 0; fib[1] = 1;
    for (int i = 2; i < MAXN + 3; ++i) fib[i] = fib[i - 1] + fib[i - 2];
  }
  __syncthreads();
  for (int i = blockIdx.y; i < count; i += gridDim.y) {
    const Inst &I = inst[i];
    const double *V = Vmats + (size_t)i * MAXN * MAXN;
    const double *dl = deltas + (size_t)i * MAXN;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < I.dim;
         r += (int64_t)gridDim.x * blockDim.x) {
      const uint64_t code = unrank_b(I, fib, r);
      double s = 0.0;
      uint64_t m = code;
      while (m) {
        const int k = __ffsll((long long)m) - 1;
        m &= m - 1;
        s += dl[k];
        uint64_t m2 = m;
        while (m2) {
          const int k2 = __ffsll((long long)m2) - 1;
          m2 &= m2 - 1;
          s += V[k * MAXN + k2];
        }
      }
      diag[I.off + r] = s;
    }
  }
}

uint64_t fibh(int i) { uint64_t a = 0, b = 1; for (int k = 0; k < i; ++k) { uint64_t t = a + b; a = b; b = t; } return a; }

struct el_batch_impl {
  int count = 0, dtype = 0, max_iter = 0;
  double tol = 0;
  int64_t total_rows = 0, dim_max = 0;
  int wait_polls = 1 << 22;         // grid-barrier polls before a timeout (cooperative solver)
  int want_nat = 0;                 // form the ground-state site occupations
  double *d_nat = nullptr;          // [count][MAXN]
  std::vector<int> order;           // processing position -> caller index
  Inst *d_inst = nullptr;
  double *d_diag = nullptr;
  double *d_out = nullptr;          // 4 doubles per instance
  int *d_iout = nullptr;            // 2 ints per instance
  unsigned *d_queue = nullptr;
  void *ws = nullptr;
  size_t ws_bytes = 0;
  int device = 0;
  std::vector<int64_t> dims;        // per processing position
  std::vector<int> nsites;          // per processing position
  // cooperative solver workspace
  void *c_vpub = nullptr;
  double *c_part = nullptr;
  unsigned *c_sync = nullptr;       // [0] arrival counter, [1] error flag
  int c_nctas = 0;
  // TABLE instances: concatenated ascending codes and flip tables
  uint64_t *d_codes = nullptr;
  int32_t *d_tgt = nullptr;
  uint64_t *d_scodes = nullptr;     // chain / ring instances: codes in rank order
};

// Independent sets of a graph on n bit positions (adjb[k]: the neighbours
// of bit k) in ascending code order: bits are decided from the top down,
// clear before set, and a bit is set only when no decided neighbour is.
// Returns false as soon as there are more than `limit`.
struct IndepSets {
  int n;
  const uint64_t *adjb;
  int64_t limit;
  std::vector<uint64_t> *out;
  bool walk(int k, uint64_t code) {
    if (k < 0) {
      if ((int64_t)out->size() >= limit) return false;
      out->push_back(code);
      return true;
    }
    if (!walk(k - 1, code)) return false;
    if (!(code & adjb[k]) && !walk(k - 1, code | (1ULL << k))) return false;
    return true;
  }
};

constexpr int64_t TABLE_MAX_ROWS = 1LL << 24;   // rows of one TABLE instance

}  // namespace

struct el_batch : el_batch_impl {};

extern "C" {

int el_batch_create(el_ctx *ctx, int count, const int32_t *n_sites, const int32_t *layouts,
                    const double *omega, const double *delta, const int32_t *pair_off,
                    const int32_t *pi, const int32_t *pj, const double *V, int dtype,
                    int max_iter, double tol, el_batch **out) {
  return el_batch_create_graph(ctx, count, n_sites, layouts, omega, delta, pair_off, pi, pj, V, nullptr,
                               nullptr, nullptr, dtype, max_iter, tol, out);
}

int el_batch_create_graph(el_ctx *ctx, int count, const int32_t *n_sites, const int32_t *layouts,
                          const double *omega, const double *delta, const int32_t *pair_off,
                          const int32_t *pi, const int32_t *pj, const double *V, const int32_t *edge_off,
                          const int32_t *ei, const int32_t *ej, int dtype, int max_iter, double tol,
                          el_batch **out) {
  if (!ctx || !out || count < 1 || !n_sites || !layouts || !omega || !delta || !pair_off) return EL_EINVAL;
  *out = nullptr;
  if (dtype != EL_F32 && dtype != EL_F64) return fail(ctx, EL_EINVAL, "batched Lanczos vectors must be EL_F32 or EL_F64");
  if (max_iter < 2 || max_iter > MAXIT) return fail(ctx, EL_EINVAL, "max_iter must be in [2, %d]", MAXIT);
  if (!(tol > 0) || !std::isfinite(tol)) return fail(ctx, EL_EINVAL, "tol must be positive");
  for (int i = 0; i < count; ++i)
    if (pair_off[i] < 0 || pair_off[i + 1] < pair_off[i])
      return fail(ctx, EL_EINVAL, "pair offsets must be non-negative and non-decreasing (instance %d)", i);
  if (pair_off[count] > pair_off[0] && (!pi || !pj || !V))
    return fail(ctx, EL_EINVAL, "pair arrays missing for %d pairs", pair_off[count] - pair_off[0]);
  if (edge_off)
    for (int i = 0; i < count; ++i)
      if (edge_off[i] < 0 || edge_off[i + 1] < edge_off[i])
        return fail(ctx, EL_EINVAL, "edge offsets must be non-negative and non-decreasing (instance %d)", i);
  if (edge_off && edge_off[count] > edge_off[0] && (!ei || !ej))
    return fail(ctx, EL_EINVAL, "edge arrays missing for %d edges", edge_off[count] - edge_off[0]);
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<int64_t> dims(count);
  // TABLE instances: neighbours by bit position and the ascending code list
  std::vector<uint64_t> adjb((size_t)count * MAXN, 0);
  std::vector<std::vector<uint64_t>> tcodes(count);
  for (int i = 0; i < count; ++i) {
    const int n = n_sites[i];
    if (n < 1 || n > MAXN) return fail(ctx, EL_EINVAL, "instance %d: n must be in [1, %d]", i, MAXN);
    if (layouts[i] == EL_LAYOUT_TABLE) {
      if (!edge_off) return fail(ctx, EL_EINVAL, "instance %d: a TABLE (graph blockade) instance needs its edges", i);
      for (int q = edge_off[i]; q < edge_off[i + 1]; ++q) {
        const int a = ei[q], c = ej[q];
        if (a < 0 || c < 0 || a >= n || c >= n || a == c)
          return fail(ctx, EL_EINVAL, "instance %d: bad edge (%d, %d)", i, a, c);
        const int qa = n - 1 - a, qc = n - 1 - c;
        adjb[(size_t)i * MAXN + qa] |= 1ULL << qc;
        adjb[(size_t)i * MAXN + qc] |= 1ULL << qa;
      }
      IndepSets w{n, &adjb[(size_t)i * MAXN], TABLE_MAX_ROWS, &tcodes[i]};
      if (!w.walk(n - 1, 0))
        return fail(ctx, EL_EINVAL, "instance %d: blockade sector larger than %lld rows", i,
                    (long long)TABLE_MAX_ROWS);
      dims[i] = (int64_t)tcodes[i].size();
    } else if (layouts[i] == EL_LAYOUT_CHAIN) dims[i] = (int64_t)fibh(n + 2);
    else if (layouts[i] == EL_LAYOUT_RING) {
      if (n < 3) return fail(ctx, EL_EINVAL, "instance %d: ring needs n >= 3", i);
      dims[i] = (int64_t)(fibh(n + 1) + fibh(n - 1));
    } else if (layouts[i] == EL_LAYOUT_FULL) {
      if (n > 24) return fail(ctx, EL_EINVAL, "instance %d: full basis in a batch limited to n <= 24", i);
      dims[i] = 1LL << n;
    } else {
      return fail(ctx, EL_EINVAL, "instance %d: layout must be chain, ring, full or table", i);
    }
  }
  el_batch *b = new el_batch();
  b->count = count; b->dtype = dtype; b->max_iter = max_iter; b->tol = tol; b->device = ctx->device;
  b->order.resize(count);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return dims[x] > dims[y]; });
  std::vector<int> noff(count + 1, 0);
  for (int i = 0; i < count; ++i) noff[i + 1] = noff[i] + n_sites[i];
  std::vector<Inst> inst(count);
  std::vector<double> Vm((size_t)count * MAXN * MAXN, 0.0), Dl((size_t)count * MAXN, 0.0);
  int64_t off = 0;
  int rc = EL_OK;
  for (int p = 0; p < count && rc == EL_OK; ++p) {
    const int i = b->order[p];
    const int n = n_sites[i];
    Inst &I = inst[p];
    memset(&I, 0, sizeof I);
    I.n = n; I.layout = layouts[i]; I.dim = dims[i]; I.off = off;
    for (int s2 = 0; s2 < n; ++s2) {
      const double o = omega[noff[i] + s2], dd = delta[noff[i] + s2];
      if (!std::isfinite(o) || !std::isfinite(dd)) { rc = fail(ctx, EL_EINVAL, "instance %d: non-finite drive", i); break; }
      I.om[n - 1 - s2] = 0.5 * o;
      Dl[(size_t)p * MAXN + (n - 1 - s2)] = dd;
    }
    for (int q = pair_off[i]; q < pair_off[i + 1] && rc == EL_OK; ++q) {
      const int a = pi[q], c = pj[q];
      if (a < 0 || c < 0 || a >= n || c >= n || a == c || !std::isfinite(V[q])) {
        rc = fail(ctx, EL_EINVAL, "instance %d: bad pair (%d, %d)", i, a, c);
        break;
      }
      const int qa = n - 1 - a, qb = n - 1 - c;
      Vm[(size_t)p * MAXN * MAXN + qa * MAXN + qb] += V[q];
      Vm[(size_t)p * MAXN * MAXN + qb * MAXN + qa] += V[q];
    }
    off += dims[i];
    b->dims.push_back(dims[i]);
    b->nsites.push_back(n);
    b->dim_max = std::max(b->dim_max, dims[i]);
  }
  b->total_rows = off;
  // TABLE instances: codes and flip tables; chain / ring instances: codes;
  // concatenated in processing order
  int64_t tab_rows = 0, tab_cells = 0, seq_rows = 0;
  for (int p = 0; p < count; ++p) {
    const int i = b->order[p];
    if (layouts[i] == EL_LAYOUT_CHAIN || layouts[i] == EL_LAYOUT_RING) seq_rows += dims[i];
    if (layouts[i] != EL_LAYOUT_TABLE) continue;
    tab_rows += dims[i];
    tab_cells += dims[i] * n_sites[i];
  }
  double *d_V = nullptr, *d_D = nullptr;
  uint64_t *d_adj = nullptr;
  cudaError_t e = cudaSuccess;
  if (rc == EL_OK && seq_rows > 0) do {
    if ((e = cudaMalloc(&b->d_scodes, (size_t)seq_rows * 8)) != cudaSuccess) break;
    int64_t so = 0;
    for (int p = 0; p < count; ++p) {
      const int i = b->order[p];
      if (layouts[i] != EL_LAYOUT_CHAIN && layouts[i] != EL_LAYOUT_RING) continue;
      inst[p].codes = b->d_scodes + so;
      so += dims[i];
    }
  } while (0);
  if (rc == EL_OK && e == cudaSuccess && tab_rows > 0) do {
    if ((e = cudaMalloc(&b->d_codes, (size_t)tab_rows * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&b->d_tgt, (size_t)tab_cells * 4)) != cudaSuccess) break;
    std::vector<uint64_t> adjp((size_t)count * MAXN, 0);
    int64_t co = 0, to = 0;
    for (int p = 0; p < count && e == cudaSuccess; ++p) {
      const int i = b->order[p];
      for (int k = 0; k < MAXN; ++k) adjp[(size_t)p * MAXN + k] = adjb[(size_t)i * MAXN + k];
      if (layouts[i] != EL_LAYOUT_TABLE) continue;
      inst[p].codes = b->d_codes + co;
      inst[p].tgt = b->d_tgt + to;
      e = el::copy(ctx, b->d_codes + co, tcodes[i].data(), (size_t)dims[i] * 8, cudaMemcpyHostToDevice);
      co += dims[i];
      to += dims[i] * n_sites[i];
    }
    if (e != cudaSuccess) break;
    if ((e = cudaMalloc(&d_adj, adjp.size() * 8)) != cudaSuccess) break;
    e = el::copy(ctx, d_adj, adjp.data(), adjp.size() * 8, cudaMemcpyHostToDevice);
  } while (0);
  if (rc == EL_OK && e == cudaSuccess) do {
    if ((e = cudaMalloc(&b->d_inst, sizeof(Inst) * count)) != cudaSuccess) break;
    if ((e = cudaMalloc(&b->d_diag, (size_t)off * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&b->d_out, (size_t)count * 4 * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&b->d_iout, (size_t)count * 2 * 4)) != cudaSuccess) break;
    if ((e = cudaMalloc(&b->d_queue, 64)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_V, Vm.size() * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_D, Dl.size() * 8)) != cudaSuccess) break;
    if ((e = el::copy(ctx, b->d_inst, inst.data(), sizeof(Inst) * count, cudaMemcpyHostToDevice)) != cudaSuccess) break;
    if ((e = el::copy(ctx, d_V, Vm.data(), Vm.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess) break;
    if ((e = el::copy(ctx, d_D, Dl.data(), Dl.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess) break;
    if (seq_rows > 0) {
      k_batch_fill_codes<<<dim3(64, std::min(count, 1024)), 256, 0, ctx->stream>>>(count, b->d_inst);
      ctx->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) break;
    }
    if (tab_rows > 0) {
      k_batch_flip_table<<<dim3(256, std::min(count, 1024)), 256, 0, ctx->stream>>>(count, b->d_inst, d_adj);
      ctx->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) break;
    }
    k_batch_diag<<<dim3(64, std::min(count, 1024)), 256, 0, ctx->stream>>>(count, b->d_inst, d_V, d_D, b->d_diag);
    ctx->launches++;
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    e = cudaStreamSynchronize(ctx->stream);
  } while (0);
  if (d_V) cudaFree(d_V);
  if (d_D) cudaFree(d_D);
  if (d_adj) cudaFree(d_adj);
  if (rc == EL_OK && e != cudaSuccess) rc = el::cuda_fail(ctx, e, "el_batch_create");
  if (rc != EL_OK) { el_batch_destroy(b); return rc; }
  *out = b;
  return EL_OK;
}

int el_batch_run(el_ctx *ctx, el_batch *b, int threads, int ctas_per_sm, uint64_t seed) {
  if (!ctx || !b) return EL_EINVAL;
  if (threads != 256 && threads != 512 && threads != 1024) return fail(ctx, EL_EINVAL, "threads must be 256, 512 or 1024");
  if (ctas_per_sm < 1 || ctas_per_sm > 2) return fail(ctx, EL_EINVAL, "ctas_per_sm must be 1 or 2");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int grid = std::min(b->count, sms * ctas_per_sm);
  const size_t es = b->dtype == EL_F32 ? 4 : 8;
  const size_t need = (size_t)grid * (b->max_iter + 2) * b->dim_max * es;
  if (need > b->ws_bytes) {
    // grows only outside graph capture (a first run sizes it)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (cs != cudaStreamCaptureStatusNone) return fail(ctx, EL_EINVAL, "run the batch once before capturing it");
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (b->ws) cudaFree(b->ws);
    b->ws = nullptr;
    b->ws_bytes = 0;
    cudaError_t e = cudaMalloc(&b->ws, need);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, EL_ENOMEM, "batched workspace of %zu bytes", need); }
    b->ws_bytes = need;
  }
  EL_CUDA_TRY(ctx, cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned), ctx->stream));
  BatchArgs A;
  memset(&A, 0, sizeof A);
  A.count = b->count; A.max_iter = b->max_iter; A.tol = b->tol; A.eps = b->dtype == EL_F32 ? 1.19e-7 : 2.22e-16;
  A.inst = b->d_inst; A.diag = b->d_diag; A.ws = b->ws; A.dim_max = b->dim_max; A.queue = b->d_queue;
  A.seed = seed;
  A.e0 = b->d_out; A.e1 = b->d_out + b->count; A.res = b->d_out + 2 * b->count; A.gap = b->d_out + 3 * b->count;
  A.iters = b->d_iout; A.conv = b->d_iout + b->count;
  A.nat = b->want_nat ? b->d_nat : nullptr;
#define EL_BCASE(TT, NTV) k_lanczos_batch<TT, NTV><<<grid, NTV, 0, ctx->stream>>>(A)
  if (b->dtype == EL_F32) {
    if (threads == 256) EL_BCASE(float, 256); else if (threads == 512) EL_BCASE(float, 512); else EL_BCASE(float, 1024);
  } else {
    if (threads == 256) EL_BCASE(double, 256); else if (threads == 512) EL_BCASE(double, 512); else EL_BCASE(double, 1024);
  }
#undef EL_BCASE
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int el_batch_run_coop(el_ctx *ctx, el_batch *b, int reorth_passes, int check_every, uint64_t seed) {
  if (!ctx || !b) return EL_EINVAL;
  if (check_every < 1) return fail(ctx, EL_EINVAL, "check_every must be >= 1");
  if (reorth_passes < 1 || reorth_passes > 2) return fail(ctx, EL_EINVAL, "reorth_passes must be 1 or 2");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const size_t es = b->dtype == EL_F32 ? 4 : 8;
  const int m = b->max_iter;
  // threads (= rows) per CTA: the smallest power of two >= 32 that keeps
  // the grid within 64 CTAs, then the Krylov slice must fit shared memory
  // and the grid must be co-resident (one CTA per SM)
  struct Plan { int nt, nctas; size_t smem; };
  std::vector<Plan> plans(b->count);
  int nctas_max = 0;
  for (int p = 0; p < b->count; ++p) {
    const int64_t dim = b->dims[p];
    int nt = 32;
    while (nt < 1024 && (dim + nt - 1) / nt > 64) nt <<= 1;
    auto slice = [&](int t) { return coop_slice_bytes((int)std::min<int64_t>(m, dim), t, (int)es); };
    // a slice too large for shared memory: more, narrower CTAs (up to one per SM)
    while (slice(nt) > 160 * 1024 && nt > 32 && (dim + nt / 2 - 1) / (nt / 2) <= sms) nt >>= 1;
    const int64_t g = (dim + nt - 1) / nt;
    const size_t smem = slice(nt) + COOP_WORK_BYTES;
    if (g > sms || slice(nt) > 160 * 1024)
      return fail(ctx, EL_EINVAL, "instance of dimension %lld is too large for the cooperative solver "
                  "(use el_batch_run)", (long long)dim);
    plans[p] = {nt, (int)g, smem};
    nctas_max = std::max(nctas_max, (int)g);
  }
  if (!b->c_vpub || nctas_max > b->c_nctas) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (cs != cudaStreamCaptureStatusNone) return fail(ctx, EL_EINVAL, "run the batch once before capturing it");
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(b->c_vpub); cudaFree(b->c_part); cudaFree(b->c_sync);
    b->c_vpub = nullptr; b->c_part = nullptr; b->c_sync = nullptr; b->c_nctas = 0;
    cudaError_t e = cudaMalloc(&b->c_vpub, (size_t)b->dim_max * es);
    if (e == cudaSuccess) e = cudaMalloc(&b->c_part, ((size_t)2 * nctas_max + 2) * (MAXIT + 2) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->c_sync, 2 * sizeof(unsigned));
    if (e != cudaSuccess) { cudaGetLastError(); return fail(ctx, EL_ENOMEM, "cooperative workspace"); }
    b->c_nctas = nctas_max;
  }
  // counter and error flag start at zero; between instances only the
  // counter is reset, so a timeout in any instance stays visible to the host
  EL_CUDA_TRY(ctx, cudaMemsetAsync(b->c_sync, 0, 2 * sizeof(unsigned), ctx->stream));
  for (int p = 0; p < b->count; ++p) {
    const Plan &P = plans[p];
    CoopArgs G;
    memset(&G, 0, sizeof G);
    G.poll_limit = b->wait_polls;
    G.p = p; G.m = m; G.nctas = P.nctas; G.check_every = check_every; G.passes = reorth_passes;
    G.tol = b->tol; G.eps = b->dtype == EL_F32 ? 1.19e-7 : 2.22e-16;
    G.inst = b->d_inst; G.diag = b->d_diag; G.vpub = b->c_vpub; G.part = b->c_part;
    G.tot = b->c_part + (size_t)2 * P.nctas * (MAXIT + 2);
    G.bar = b->c_sync; G.err = (int *)(b->c_sync + 1); G.seed = seed;
    G.e0 = b->d_out; G.e1 = b->d_out + b->count; G.res = b->d_out + 2 * b->count; G.gap = b->d_out + 3 * b->count;
    G.iters = b->d_iout; G.conv = b->d_iout + b->count;
    G.nat = b->want_nat ? b->d_nat : nullptr;
    if (p > 0) EL_CUDA_TRY(ctx, cudaMemsetAsync(b->c_sync, 0, sizeof(unsigned), ctx->stream));
    void *kargs[] = {(void *)&G};
    const void *fn = nullptr;
#define EL_CPICK(TT)                                                                   \
    switch (P.nt) {                                                                    \
      case 32: fn = (const void *)k_lanczos_coop<TT, 32>; break;                       \
      case 64: fn = (const void *)k_lanczos_coop<TT, 64>; break;                       \
      case 128: fn = (const void *)k_lanczos_coop<TT, 128>; break;                     \
      case 256: fn = (const void *)k_lanczos_coop<TT, 256>; break;                     \
      case 512: fn = (const void *)k_lanczos_coop<TT, 512>; break;                     \
      default: fn = (const void *)k_lanczos_coop<TT, 1024>; break;                     \
    }
    if (b->dtype == EL_F32) { EL_CPICK(float) } else { EL_CPICK(double) }
#undef EL_CPICK
    EL_CUDA_TRY(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem));
    int per_sm = 0;
    EL_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, P.nt, P.smem));
    if (per_sm * sms < P.nctas) return fail(ctx, EL_EINVAL, "cooperative grid of %d CTAs is not co-resident", P.nctas);
    EL_CUDA_TRY(ctx, cudaLaunchCooperativeKernel(fn, dim3(P.nctas), dim3(P.nt), kargs, P.smem, ctx->stream));
    ctx->launches++;
  }
  // a barrier that timed out leaves the flag set
  unsigned hs[2] = {0, 0};
  EL_CUDA_TRY(ctx, el::copy(ctx, hs, b->c_sync, sizeof hs, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs[1]) return fail(ctx, EL_ECUDA, "cooperative Lanczos: a grid barrier timed out");
  return EL_OK;
}

int el_batch_want_occupations(el_ctx *ctx, el_batch *b, int want) {
  if (!ctx || !b) return EL_EINVAL;
  if (want && !b->d_nat) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx->stream, &cs);
    if (cs != cudaStreamCaptureStatusNone) return fail(ctx, EL_EINVAL, "request occupations before capturing");
    cudaError_t e = cudaMalloc(&b->d_nat, (size_t)b->count * MAXN * sizeof(double));
    if (e != cudaSuccess) { cudaGetLastError(); b->d_nat = nullptr; return fail(ctx, EL_ENOMEM, "occupation buffer"); }
    EL_CUDA_TRY(ctx, cudaMemsetAsync(b->d_nat, 0, (size_t)b->count * MAXN * sizeof(double), ctx->stream));
  }
  b->want_nat = want ? 1 : 0;
  return EL_OK;
}

int el_batch_occupations(el_ctx *ctx, el_batch *b, double *n_atom) {
  if (!ctx || !b || !n_atom) return EL_EINVAL;
  if (!b->d_nat) return fail(ctx, EL_EINVAL, "occupations were not requested (el_batch_want_occupations)");
  std::vector<double> h((size_t)b->count * MAXN);
  EL_CUDA_TRY(ctx, el::copy(ctx, h.data(), b->d_nat, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  // processing order -> caller order; bit position k is site n-1-k
  for (int p = 0; p < b->count; ++p) {
    const int i = b->order[p];
    const int n = b->nsites[p];
    for (int s2 = 0; s2 < MAXN; ++s2)
      n_atom[(size_t)i * MAXN + s2] = s2 < n ? h[(size_t)p * MAXN + (n - 1 - s2)] : 0.0;
  }
  return EL_OK;
}

int el_batch_set_wait_limit(el_ctx *ctx, el_batch *b, int32_t polls) {
  if (!ctx || !b) return EL_EINVAL;
  if (polls < 0) return fail(ctx, EL_EINVAL, "wait limit must be >= 0 polls");
  b->wait_polls = polls;
  return EL_OK;
}

int el_batch_results(el_ctx *ctx, el_batch *b, double *e0, double *gap, double *residual,
                     int32_t *iters, int32_t *converged) {
  if (!ctx || !b || !e0 || !gap) return EL_EINVAL;
  const int count = b->count;
  std::vector<double> ho((size_t)count * 4);
  std::vector<int> hi((size_t)count * 2);
  EL_CUDA_TRY(ctx, el::copy(ctx, ho.data(), b->d_out, ho.size() * 8, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, el::copy(ctx, hi.data(), b->d_iout, hi.size() * 4, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int p = 0; p < count; ++p) {
    const int i = b->order[p];
    e0[i] = ho[p];
    gap[i] = ho[(size_t)3 * count + p];
    if (residual) residual[i] = ho[(size_t)2 * count + p];
    if (iters) iters[i] = hi[p];
    if (converged) converged[i] = hi[(size_t)count + p];
  }
  return EL_OK;
}

int el_batch_destroy(el_batch *b) {
  if (!b) return EL_OK;
  cudaSetDevice(b->device);
  if (b->d_inst) cudaFree(b->d_inst);
  if (b->d_diag) cudaFree(b->d_diag);
  if (b->d_out) cudaFree(b->d_out);
  if (b->d_iout) cudaFree(b->d_iout);
  if (b->d_queue) cudaFree(b->d_queue);
  if (b->ws) cudaFree(b->ws);
  if (b->c_vpub) cudaFree(b->c_vpub);
  if (b->c_part) cudaFree(b->c_part);
  if (b->c_sync) cudaFree(b->c_sync);
  if (b->d_nat) cudaFree(b->d_nat);
  if (b->d_codes) cudaFree(b->d_codes);
  if (b->d_scodes) cudaFree(b->d_scodes);
  if (b->d_tgt) cudaFree(b->d_tgt);
  delete b;
  return EL_OK;
}

}  // extern "C"
