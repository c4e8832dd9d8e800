// Adjoint pulse gradients through the Chebyshev propagator.
//
// Pulse: K piecewise-constant steps; step k lasts tau_k with
//     H_k = sum_i [ -Delta_k b_i n_i + (Omega_k a_i / 2) sigma^x_i ] + sum V n n
// (a_i, b_i: fixed site shapes, 1 by default; the reference's delta is
// -Delta, channels.py:68-73).  Each step applies the truncated expansion
//     U_k = sum_{m<=M} c_m T_m(Htil_k),  Htil_k = (H_k - b_k)/a_k
// of el_cheb_step.  Objective: F = |<phi|psi_K>|^2 (fidelity with a target)
// or F = <psi_K|O|psi_K> for a diagonal observable O.
//
// Discretise-then-differentiate: with lambda_K = dF/d(conj psi_K) / 2
// (a phi for the fidelity, O psi_K for the observable) the gradient of the
// computed map follows from reverse-mode differentiation of the Chebyshev
// recurrence t_0 = psi, t_1 = Htil t_0, t_{m+1} = 2 Htil t_m - t_{m-1}:
//     u_M = conj(c_M) lambda,  u_m = conj(c_m) lambda + s_{m+1} Htil u_{m+1} - u_{m+2}
//     (s_1 = 1, s_m = 2 otherwise),   lambda_{k-1} = u_0,
//     dF/dtheta_k = 2 sum_{m>=1} s_m Re <G_theta u_m, t_{m-1}> / a_k,
// with G_Omega = sum a_i sigma^x_i / 2 and G_Delta = -sum b_i n_i.  a_k, b_k
// are held fixed (the map depends on them only at the truncation level).
// The forward pass keeps one state per step; the backward pass recomputes the
// Chebyshev terms t_0..t_{M-1} of one step at a time from that checkpoint
// (the recurrence is recomputed, never stored across steps).
#include "el_internal.cuh"

#include <algorithm>

namespace {

using el::fail;

template <typename S>
struct AdjArgs {
  const S *diagV;
  S delta[EL_MAX_SITES];   // current -Delta_k b_i per bit position
  S ahalf[EL_MAX_SITES];   // a_i / 2 per bit position
  S bsh[EL_MAX_SITES];     // b_i per bit position
  S om;                    // Omega_k
  S alpha, beta;           // y = clam lam + alpha H x + beta x - z
  S cl_re, cl_im;
  const S *x, *z, *lam, *t;
  S *y;
  double *partials;
  unsigned int *counter;
  double *out;             // [2]: Re<G_O x, t>, Re<G_D x, t>
};

// One adjoint step over all rows: y = clam lam + alpha H x + beta x - z and
// the two gradient dots.  ADJ_LANES adjacent lanes share a row and take the
// sites k = lane, lane + ADJ_LANES, ...: the small bases that the pulse
// gradient runs on (tens of thousands of rows) would otherwise leave most
// SMs idle while each thread walks all n flips.  The row loop is uniform
// over the block so that every lane reaches the shuffles.  The CTA that
// finishes last sums the per-CTA partials with all its threads in a fixed
// order (the result does not depend on which CTA is last).
constexpr int ADJ_LANES = 4;
constexpr int ADJ_UNROLL = 4;   // gathers in flight per lane

template <typename S>
__global__ void __launch_bounds__(256, 4) k_adjoint_step(BasisDev B, AdjArgs<S> P) {
  constexpr int G = ADJ_LANES;
  typedef typename el::VecT<S, true>::type V2;   // one complex entry, one load
  __shared__ double red[2][256];
  __shared__ bool last;
  const int lane = (int)threadIdx.x & (G - 1);
  const int64_t rpb = blockDim.x / G;
  double gO = 0.0, gD = 0.0;
  for (int64_t base = (int64_t)blockIdx.x * rpb; base < B.dim; base += (int64_t)gridDim.x * rpb) {
    const int64_t mine = base + threadIdx.x / G;
    const bool active = mine < B.dim;           // the same for the G lanes of a row
    const int64_t r = active ? mine : 0;        // lanes past the end work on row 0
    const uint64_t code = el::unrank_row(B, r);
    S sre = 0, sim = 0, dpart = 0, nb = 0;
    // a lane's sites k = (j0 + u) G + lane: all U gathers of a round are
    // issued before any of them is accumulated
    for (int j0 = 0; j0 * G < B.n; j0 += ADJ_UNROLL) {
      S xa[ADJ_UNROLL], xb[ADJ_UNROLL], am[ADJ_UNROLL];
#pragma unroll
      for (int u = 0; u < ADJ_UNROLL; ++u) {
        const int k = (j0 + u) * G + lane;
        am[u] = S(0);
        xa[u] = S(0);
        xb[u] = S(0);
        if (k < B.n) {
          if ((code >> k) & 1ULL) { dpart += P.delta[k]; nb += P.bsh[k]; }
          const S amp = P.ahalf[k];
          const int64_t tg = amp == S(0) ? -1 : el::flip_target(B, code, r, k);
          if (tg >= 0) {
            const V2 v = reinterpret_cast<const V2 *>(P.x)[tg];
            am[u] = amp;
            xa[u] = v.x;
            xb[u] = v.y;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < ADJ_UNROLL; ++u) {   // a skipped flip adds 0 * 0
        sre += am[u] * xa[u];
        sim += am[u] * xb[u];
      }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) {
      sre += __shfl_xor_sync(0xffffffffu, sre, off);
      sim += __shfl_xor_sync(0xffffffffu, sim, off);
      dpart += __shfl_xor_sync(0xffffffffu, dpart, off);
      nb += __shfl_xor_sync(0xffffffffu, nb, off);
    }
    if (lane != 0 || !active) continue;
    const S xr = P.x[2 * r], xi = P.x[2 * r + 1];
    const S dsum = P.diagV[r] + dpart;
    // H x = dsum x + Omega S
    const S hre = dsum * xr + P.om * sre, him = dsum * xi + P.om * sim;
    S yre = P.alpha * hre + P.beta * xr, yim = P.alpha * him + P.beta * xi;
    if (P.z) { yre -= P.z[2 * r]; yim -= P.z[2 * r + 1]; }
    if (P.lam) {
      const S lr = P.lam[2 * r], li = P.lam[2 * r + 1];
      yre += P.cl_re * lr - P.cl_im * li;
      yim += P.cl_re * li + P.cl_im * lr;
    }
    P.y[2 * r] = yre;
    P.y[2 * r + 1] = yim;
    if (P.t) {
      const double tr = P.t[2 * r], ti = P.t[2 * r + 1];
      gO += (double)sre * tr + (double)sim * ti;               // Re(conj(G_O x) t)
      gD += -(double)nb * ((double)xr * tr + (double)xi * ti); // Re(conj(G_D x) t)
    }
  }
  red[0][threadIdx.x] = gO;
  red[1][threadIdx.x] = gD;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    P.partials[2 * blockIdx.x] = red[0][0];
    P.partials[2 * blockIdx.x + 1] = red[1][0];
    __threadfence();
    last = (atomicAdd(P.counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0, b = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    a += __ldcg(&P.partials[2 * i]);
    b += __ldcg(&P.partials[2 * i + 1]);
  }
  red[0][threadIdx.x] = a;
  red[1][threadIdx.x] = b;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[0][threadIdx.x] += red[0][threadIdx.x + s];
      red[1][threadIdx.x] += red[1][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    P.out[0] = red[0][0];
    P.out[1] = red[1][0];
    *P.counter = 0u;
  }
}

// lam = O psi (elementwise, O real per row)
template <typename S>
__global__ void k_diag_mul(int64_t dim, const double *O, const S *psi, S *lam, double *partials,
                           unsigned int *counter, double *out) {
  __shared__ double red[256];
  __shared__ bool last;
  double f = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < dim;
       r += (int64_t)gridDim.x * blockDim.x) {
    const double o = O[r], a = psi[2 * r], b = psi[2 * r + 1];
    lam[2 * r] = (S)(o * a);
    lam[2 * r + 1] = (S)(o * b);
    f += o * (a * a + b * b);
  }
  red[threadIdx.x] = f;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = red[0];
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double s = 0.0;
    for (unsigned i = 0; i < gridDim.x; ++i) s += __ldcg(&partials[i]);
    out[0] = s;
    *counter = 0u;
  }
}

// Gershgorin bounds of every step's H_k in one launch: row r contributes
// d -+ R with d = diagV[r] + sum_{set q} (-Delta_k b_q) and R = sum over its
// allowed flips of |Omega_k a_q / 2|, summed in the order (and with the
// roundings) of k_gershgorin for the drive of that step.  Per block and
// step: the block's min and max, out[(block K + k) 2 + {0, 1}].
struct StepShapes { double a[EL_MAX_SITES], b[EL_MAX_SITES]; };   // by bit position

__global__ void k_step_bounds(BasisDev B, const double *__restrict__ diagV, StepShapes sh, int K,
                              const double *__restrict__ om, const double *__restrict__ dl, double *out) {
  __shared__ double lo_s[256], hi_s[256];
  // with one row per thread (the pulse problems' small bases) the row's
  // code and its allowed flips are found once for all steps
  const bool one = B.dim <= (int64_t)gridDim.x * blockDim.x;
  const int64_t r1 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t code1 = 0, flips1 = 0;
  if (one && r1 < B.dim) {
    code1 = el::unrank_row(B, r1);
    for (int q = 0; q < B.n; ++q)
      if (el::flip_target(B, code1, r1, q) >= 0) flips1 |= 1ULL << q;
  }
  for (int k = 0; k < K; ++k) {
    const double o = om[k], d0 = dl[k];
    double lo = 1e300, hi = -1e300;
    for (int64_t r = r1; r < B.dim; r += (int64_t)gridDim.x * blockDim.x) {
      const uint64_t code = one ? code1 : el::unrank_row(B, r);
      double d = diagV[r], R = 0.0;
      for (int q = 0; q < B.n; ++q) {
        if ((code >> q) & 1ULL) d += d0 * sh.b[q];
        const double amp = fabs(0.5 * (o * sh.a[q]));
        if (amp == 0.0) continue;
        if (one ? ((flips1 >> q) & 1ULL) != 0 : el::flip_target(B, code, r, q) >= 0) R += amp;
      }
      lo = fmin(lo, d - R);
      hi = fmax(hi, d + R);
    }
    lo_s[threadIdx.x] = lo;
    hi_s[threadIdx.x] = hi;
    __syncthreads();
    for (int s2 = 128; s2 > 0; s2 >>= 1) {
      if (threadIdx.x < s2) {
        lo_s[threadIdx.x] = fmin(lo_s[threadIdx.x], lo_s[threadIdx.x + s2]);
        hi_s[threadIdx.x] = fmax(hi_s[threadIdx.x], hi_s[threadIdx.x + s2]);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      out[((size_t)blockIdx.x * K + k) * 2] = lo_s[0];
      out[((size_t)blockIdx.x * K + k) * 2 + 1] = hi_s[0];
    }
    __syncthreads();
  }
}

// lo[k], hi[k] of every step (one launch, one copy back).
int step_bounds(el_ctx *ctx, el_ham *h, int K, const double *omega_k, const double *delta_k,
                const std::vector<double> &ash, const std::vector<double> &bsh, std::vector<double> &lo,
                std::vector<double> &hi) {
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  int sms = 148;
  EL_CUDA_TRY(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const int grid = (int)std::min<int64_t>(el::grid_for(dim, 256), 2 * (int64_t)sms);
  double *d = (double *)el::workspace(ctx, 12, ((size_t)2 * K + (size_t)grid * K * 2) * sizeof(double));
  if (!d) return EL_ENOMEM;
  double *d_om = d, *d_dl = d + K, *d_out = d + 2 * K;
  std::vector<double> hom(K), hdl(K);
  for (int k = 0; k < K; ++k) { hom[k] = omega_k[k]; hdl[k] = -delta_k[k]; }
  EL_CUDA_TRY(ctx, el::copy(ctx, d_om, hom.data(), K * sizeof(double), cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_dl, hdl.data(), K * sizeof(double), cudaMemcpyHostToDevice));
  StepShapes sh;
  memset(&sh, 0, sizeof sh);
  for (int q = 0; q < n; ++q) { sh.a[q] = ash[n - 1 - q]; sh.b[q] = bsh[n - 1 - q]; }
  k_step_bounds<<<grid, 256, 0, ctx->stream>>>(el::basis_dev(h->basis), h->d_diagV64, sh, K, d_om, d_dl, d_out);
  ctx->launches++;
  EL_LAUNCH_CHECK(ctx);
  std::vector<double> part((size_t)grid * K * 2);
  EL_CUDA_TRY(ctx, el::copy(ctx, part.data(), d_out, part.size() * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  lo.assign(K, 1e300);
  hi.assign(K, -1e300);
  for (int b = 0; b < grid; ++b)
    for (int k = 0; k < K; ++k) {
      lo[k] = std::min(lo[k], part[((size_t)b * K + k) * 2]);
      hi[k] = std::max(hi[k], part[((size_t)b * K + k) * 2 + 1]);
    }
  return EL_OK;
}

template <typename S>
int adjoint_impl(el_ctx *ctx, el_ham *h, int dtype, int K, const double *tau, const double *omega_k,
                 const double *delta_k, const double *oshape, const double *dshape, const void *psi0,
                 const void *target, const double *obs_diag, double tol, double *F_out,
                 double *gO_out, double *gD_out, void *psi_final) {
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  const size_t vb = (size_t)dim * 2 * sizeof(S);
  std::vector<double> ash(n, 1.0), bsh(n, 1.0);
  for (int i = 0; i < n; ++i) {
    if (oshape) ash[i] = oshape[i];
    if (dshape) bsh[i] = dshape[i];
  }
  auto set_drive = [&](int k) {
    std::vector<double> ore(n), oim(n, 0.0), de(n);
    for (int i = 0; i < n; ++i) { ore[i] = omega_k[k] * ash[i]; de[i] = -delta_k[k] * bsh[i]; }
    return el_ham_set_drive(ctx, h, ore.data(), oim.data(), de.data());
  };
  // plans of all steps: the Gershgorin bounds of every step in one launch,
  // then the expansions on the host
  std::vector<el::ChebPlan> plans(K);
  int Mmax = 1;
  {
    std::vector<double> lo, hi;
    int rc = step_bounds(ctx, h, K, omega_k, delta_k, ash, bsh, lo, hi);
    if (rc) return rc;
    for (int k = 0; k < K; ++k) {
      el::cheb_plan_bounds(lo[k], hi[k], tau[k], tol, &plans[k]);
      Mmax = std::max(Mmax, plans[k].M);
    }
  }
  // workspace: K+1 checkpoints, Mmax+1 terms, 3 adjoint vectors, lambda
  char *buf = (char *)el::workspace(ctx, 11, (size_t)(K + 1 + Mmax + 1 + 4) * vb);
  if (!buf) return EL_ENOMEM;
  auto ckp = [&](int k) { return (void *)(buf + (size_t)k * vb); };
  char *tb = buf + (size_t)(K + 1) * vb;
  auto term = [&](int m) { return (void *)(tb + (size_t)m * vb); };
  char *ub = tb + (size_t)(Mmax + 1) * vb;
  void *U[3] = {ub, ub + vb, ub + 2 * vb};
  void *lam = ub + 3 * vb;
  if (ctx->adjoint_mode != EL_ADJ_STREAM) {
    // one cooperative launch for the whole gradient
    std::vector<double> hg;
    double F = 0.0;
    int rc = el::adjoint_coop<S>(ctx, h, K, plans, Mmax, omega_k, delta_k, ash, bsh, psi0, target, obs_diag,
                                 buf, hg, F);
    if (rc) return rc;
    if (psi_final) {
      EL_CUDA_TRY(ctx, el::copy(ctx, psi_final, ckp(K), vb, cudaMemcpyDeviceToDevice));
      EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    rc = set_drive(0);   // the drive the stream path leaves behind
    if (rc) return rc;
    for (int k = 0; k < K; ++k) {
      const el::ChebPlan &pl = plans[k];
      double go = 0.0, gd = 0.0;
      for (int m = 1; m <= pl.M; ++m) {
        const double s = (m == 1) ? 1.0 : 2.0;
        go += s * hg[((size_t)k * (Mmax + 1) + m) * 2];
        gd += s * hg[((size_t)k * (Mmax + 1) + m) * 2 + 1];
      }
      gO_out[k] = 2.0 * go / pl.a;
      gD_out[k] = 2.0 * gd / pl.a;
    }
    *F_out = F;
    return EL_OK;
  }
  double *d_g = (double *)el::workspace(ctx, 12, (size_t)K * (Mmax + 1) * 2 * sizeof(double) + 64);
  if (!d_g) return EL_ENOMEM;
  EL_CUDA_TRY(ctx, cudaMemsetAsync(d_g, 0, (size_t)K * (Mmax + 1) * 2 * sizeof(double), ctx->stream));
  EL_CUDA_TRY(ctx, el::copy(ctx, ckp(0), psi0, vb, cudaMemcpyDeviceToDevice));
  int rc;
  // ---- forward: psi_k = U_k psi_{k-1}
  for (int k = 0; k < K; ++k) {
    if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
    rc = set_drive(k);
    if (rc) return rc;
    const el::ChebPlan &pl = plans[k];
    void *out = ckp(k + 1);
    rc = el::launch_axpby(ctx, dtype, dim, pl.c_re[0], pl.c_im[0], ckp(k), 0, 0, out, nullptr);
    if (rc) return rc;
    ApplyArgs A;
    memset(&A, 0, sizeof A);
    A.dtype = dtype; A.nvec = 1; A.x = ckp(k); A.y = term(1); A.acc = out;
    A.a = 1.0 / pl.a; A.b = -pl.b / pl.a; A.w_re = pl.c_re[1]; A.w_im = pl.c_im[1];
    rc = el::launch_apply(ctx, h, A);
    if (rc) return rc;
    void *xm1 = ckp(k), *xc = term(1);
    for (int m = 2; m <= pl.M; ++m) {
      void *y = term(m);
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = xc; A.z = xm1; A.y = y; A.acc = out;
      A.a = 2.0 / pl.a; A.b = -2.0 * pl.b / pl.a; A.c = -1.0; A.w_re = pl.c_re[m]; A.w_im = pl.c_im[m];
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      xm1 = xc;
      xc = y;
    }
  }
  // ---- objective and lambda_K
  double F = 0.0;
  const int grid = el::grid_for(dim, 256);
  const int agrid = el::grid_for(dim * ADJ_LANES, 256);
  rc = el::ensure_partials(ctx, (size_t)std::max(std::max(grid, agrid), 2) * 2);
  if (rc) return rc;
  if (target) {
    rc = el::launch_gemv_t(ctx, dtype, dim, 1, target, dim, ckp(K), ctx->d_scalars);
    if (rc) return rc;
    double ov[2];
    EL_CUDA_TRY(ctx, el::copy(ctx, ov, ctx->d_scalars, 2 * sizeof(double), cudaMemcpyDeviceToHost));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    F = ov[0] * ov[0] + ov[1] * ov[1];
    rc = el::launch_axpby(ctx, dtype, dim, ov[0], ov[1], target, 0, 0, lam, nullptr);
    if (rc) return rc;
  } else {
    k_diag_mul<S><<<grid, 256, 0, ctx->stream>>>(dim, obs_diag, (const S *)ckp(K), (S *)lam,
                                                  ctx->d_partials, ctx->d_counter, ctx->d_scalars);
    EL_LAUNCH_CHECK(ctx);
    double f;
    EL_CUDA_TRY(ctx, el::copy(ctx, &f, ctx->d_scalars, sizeof(double), cudaMemcpyDeviceToHost));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    F = f;
  }
  // ---- backward
  const BasisDev B = el::basis_dev(h->basis);
  if (std::is_same<S, float>::value) { rc = el::ham_diag32(ctx, h); if (rc) return rc; }
  const S *diagV = std::is_same<S, float>::value ? (const S *)(void *)h->d_diagV32
                                                 : (const S *)(void *)h->d_diagV64;
  for (int k = K - 1; k >= 0; --k) {
    if (el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
    rc = set_drive(k);
    if (rc) return rc;
    const el::ChebPlan &pl = plans[k];
    const int M = pl.M;
    // recompute t_0 .. t_{M-1} of this step from its checkpoint
    EL_CUDA_TRY(ctx, el::copy(ctx, term(0), ckp(k), vb, cudaMemcpyDeviceToDevice));
    ApplyArgs A;
    if (M >= 2) {
      memset(&A, 0, sizeof A);
      A.dtype = dtype; A.nvec = 1; A.x = term(0); A.y = term(1); A.a = 1.0 / pl.a; A.b = -pl.b / pl.a;
      rc = el::launch_apply(ctx, h, A);
      if (rc) return rc;
      for (int m = 2; m <= M - 1; ++m) {
        memset(&A, 0, sizeof A);
        A.dtype = dtype; A.nvec = 1; A.x = term(m - 1); A.z = term(m - 2); A.y = term(m);
        A.a = 2.0 / pl.a; A.b = -2.0 * pl.b / pl.a; A.c = -1.0;
        rc = el::launch_apply(ctx, h, A);
        if (rc) return rc;
      }
    }
    // reverse recurrence.  u_M = conj(c_M) lam
    void *uM = U[M % 3];
    rc = el::launch_axpby(ctx, dtype, dim, pl.c_re[M], -pl.c_im[M], lam, 0, 0, uM, nullptr);
    if (rc) return rc;
    AdjArgs<S> P;
    memset(&P, 0, sizeof P);
    P.diagV = diagV;
    for (int q = 0; q < n; ++q) {
      P.delta[q] = (S)h->delta[q];
      P.ahalf[q] = (S)(0.5 * ash[n - 1 - q]);
      P.bsh[q] = (S)bsh[n - 1 - q];
    }
    P.om = (S)omega_k[k];
    P.partials = ctx->d_partials;
    P.counter = ctx->d_counter;
    for (int m = M - 1; m >= 0; --m) {
      // u_m = conj(c_m) lam + s_{m+1} Htil u_{m+1} - u_{m+2}; dots pair u_{m+1} with t_m
      const double s = (m == 0) ? 1.0 : 2.0;
      P.alpha = (S)(s / pl.a);
      P.beta = (S)(-s * pl.b / pl.a);
      P.cl_re = (S)pl.c_re[m];
      P.cl_im = (S)(-pl.c_im[m]);
      P.x = (const S *)U[(m + 1) % 3];
      P.z = (m + 2 <= M) ? (const S *)U[(m + 2) % 3] : nullptr;
      P.lam = (const S *)lam;
      P.t = (const S *)term(m);
      P.y = (S *)U[m % 3];
      P.out = d_g + ((size_t)k * (Mmax + 1) + (m + 1)) * 2;
      k_adjoint_step<S><<<agrid, 256, 0, ctx->stream>>>(B, P);
      EL_LAUNCH_CHECK(ctx);
    }
    // lambda_{k-1} = u_0
    EL_CUDA_TRY(ctx, el::copy(ctx, lam, U[0], vb, cudaMemcpyDeviceToDevice));
  }
  std::vector<double> hg((size_t)K * (Mmax + 1) * 2);
  EL_CUDA_TRY(ctx, el::copy(ctx, hg.data(), d_g, hg.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (psi_final) EL_CUDA_TRY(ctx, el::copy(ctx, psi_final, ckp(K), vb, cudaMemcpyDeviceToDevice));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < K; ++k) {
    const el::ChebPlan &pl = plans[k];
    double go = 0.0, gd = 0.0;
    for (int m = 1; m <= pl.M; ++m) {
      const double s = (m == 1) ? 1.0 : 2.0;
      go += s * hg[((size_t)k * (Mmax + 1) + m) * 2];
      gd += s * hg[((size_t)k * (Mmax + 1) + m) * 2 + 1];
    }
    gO_out[k] = 2.0 * go / pl.a;
    gD_out[k] = 2.0 * gd / pl.a;
  }
  *F_out = F;
  return EL_OK;
}

}  // namespace

extern "C" int el_adjoint_set_mode(el_ctx *ctx, int mode) {
  if (!ctx) return EL_EINVAL;
  if (mode != EL_ADJ_AUTO && mode != EL_ADJ_STREAM && mode != EL_ADJ_COOP)
    return fail(ctx, EL_EINVAL, "adjoint mode must be EL_ADJ_AUTO, EL_ADJ_STREAM or EL_ADJ_COOP");
  ctx->adjoint_mode = mode;
  return EL_OK;
}

extern "C" int el_adjoint_pulse(el_ctx *ctx, el_ham *h, int dtype, int K, const double *tau,
                                const double *omega_k, const double *delta_k,
                                const double *omega_shape, const double *delta_shape,
                                const void *psi0, const void *target, const double *obs_diag,
                                double tol, double *F, double *grad_omega, double *grad_delta,
                                void *psi_final) {
  if (!ctx || !h || !tau || !omega_k || !delta_k || !psi0 || !F || !grad_omega || !grad_delta)
    return EL_EINVAL;
  if (dtype != EL_C64 && dtype != EL_C128) return fail(ctx, EL_EINVAL, "adjoint needs EL_C64 or EL_C128");
  if (K < 1) return fail(ctx, EL_EINVAL, "K must be >= 1");
  if (h->lossy) return fail(ctx, EL_EINVAL, "the adjoint gradient needs a Hermitian H (gamma = 0)");
  if (!h->px.empty())
    return fail(ctx, EL_EINVAL, "the adjoint gradient implements the Omega/delta/V model (no J/A channels)");
  if (!target && !obs_diag) return fail(ctx, EL_EINVAL, "give a target state or a diagonal observable");
  if (!(tol > 0) || tol >= 1) return fail(ctx, EL_EINVAL, "tol must be in (0, 1)");
  for (int k = 0; k < K; ++k)
    if (!std::isfinite(tau[k]) || tau[k] < 0 || !std::isfinite(omega_k[k]) || !std::isfinite(delta_k[k]))
      return fail(ctx, EL_EINVAL, "step %d: tau/Omega/Delta must be finite, tau >= 0", k);
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (dtype == EL_C64)
    return adjoint_impl<float>(ctx, h, dtype, K, tau, omega_k, delta_k, omega_shape, delta_shape, psi0,
                               target, obs_diag, tol, F, grad_omega, grad_delta, psi_final);
  return adjoint_impl<double>(ctx, h, dtype, K, tau, omega_k, delta_k, omega_shape, delta_shape, psi0,
                              target, obs_diag, tol, F, grad_omega, grad_delta, psi_final);
}
