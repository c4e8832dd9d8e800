// The whole adjoint pulse gradient in one cooperative launch.
//
// Same mathematics as el_adjoint.cu (forward Chebyshev steps with one
// checkpoint per step, the objective and lambda_K, then per step the terms
// t_0..t_{M-1} recomputed from the checkpoint and the reverse recurrence
//     u_M = conj(c_M) lambda,
//     u_m = conj(c_m) lambda + (s/a) (H - b) u_{m+1} - u_{m+2}
// with the gradient dots Re<G_Omega u_{m+1}, t_m>, Re<G_Delta u_{m+1}, t_m>),
// but every sweep over the basis is one phase of a single persistent
// kernel, separated by grid barriers, instead of one launch: the bases the
// pulse gradient runs on hold tens of thousands of rows, so the separate
// launches of the stream path (about 3 K M of them) cost more than their
// work.  Four lanes share a row (its flips split between them) as in
// k_adjoint_step, and keep its flip targets in registers across all
// sweeps; every step's Chebyshev plan (a, b, M, c_m) is computed on
// the host first and read from device arrays.  Gradient dots go to per-CTA
// slots [step][m][CTA] that the host adds up in a fixed order, so the
// result does not depend on scheduling.  Grid-barrier waits are bounded: a
// wait that runs out sets an error flag, every later barrier returns at
// once, and the host reports EL_ECUDA.
#include "el_internal.cuh"

#include <algorithm>

namespace el {

namespace {

constexpr int CL = 4;      // lanes per row
constexpr int CNT = 256;   // threads per CTA

template <typename S>
struct CoopAdj {
  BasisDev B;
  int K, Mmax, nctas, poll_limit;
  const double *pa, *pb;   // [K] expansion interval: Htil = (H - b) / a
  const int *pm;           // [K] terms
  const double *pc;        // [K][Mmax + 1][2] coefficients c_m
  const double *om, *dl;   // [K] Omega_k and -Delta_k
  const S *diagV;          // the V part of the diagonal
  S ahalf[EL_MAX_SITES];   // a_i / 2 per bit position
  S bsh[EL_MAX_SITES];     // b_i per bit position
  S *ckp;                  // [K + 1][dim] complex checkpoints
  S *term;                 // [Mmax + 1][dim] complex Chebyshev terms
  S *U;                    // [3][dim] complex adjoint vectors
  S *lam;                  // [dim] complex
  const S *target;         // fidelity target, or null
  const double *obs;       // diagonal observable, or null
  double *part;            // [K][Mmax + 1][nctas][2] gradient dots per CTA
  double *fpart;           // [nctas][2] objective partials
  double *fout;            // [2]: <target, psi_K> (or F, 0)
  unsigned *bar;           // arrival counter, zero at launch
  int *err;                // set when a barrier wait ran out
};

__device__ __forceinline__ void coop_sync(unsigned *bar, int *err, int nctas, int poll_limit, unsigned &gen) {
  __syncthreads();
  gen += (unsigned)nctas;
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    if (!*(volatile int *)err) {
      int polls = 0;
      unsigned v;
      for (;;) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
        if (v >= gen) break;
        if (++polls > poll_limit) { atomicExch(err, 1); break; }
        if ((polls & 255) == 0 && *(volatile int *)err) break;
      }
    }
  }
  __syncthreads();
}

// The flip sum (sum over allowed flips of a_i/2 x[target], complex) and
// nb = sum of b_i over the set sites of a row, reduced over the CL lanes of
// the row (every lane ends with the totals).
template <typename S>
__device__ __forceinline__ void row_flips(const CoopAdj<S> &P, uint64_t code, int64_t r, int lane,
                                          const S *__restrict__ x, S &sre, S &sim, S &nb) {
  sre = S(0); sim = S(0); nb = S(0);
  for (int k = lane; k < P.B.n; k += CL) {
    if ((code >> k) & 1ULL) nb += P.bsh[k];
    const S amp = P.ahalf[k];
    if (amp == S(0)) continue;
    const int64_t tg = el::flip_target(P.B, code, r, k);
    if (tg >= 0) {
      sre += amp * x[2 * tg];
      sim += amp * x[2 * tg + 1];
    }
  }
#pragma unroll
  for (int off = CL / 2; off > 0; off >>= 1) {
    sre += __shfl_xor_sync(0xffffffffu, sre, off);
    sim += __shfl_xor_sync(0xffffffffu, sim, off);
    nb += __shfl_xor_sync(0xffffffffu, nb, off);
  }
}

// Block sum of two doubles into slot[0..1] (thread 0 writes).
__device__ __forceinline__ void block_sum2(double a, double b, double *red, double *slot) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { red[2 * warp] = a; red[2 * warp + 1] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int w = 0; w < CNT / 32; ++w) { sa += red[2 * w]; sb += red[2 * w + 1]; }
    slot[0] = sa;
    slot[1] = sb;
  }
  __syncthreads();
}

// A lane's share of its row when every row fits one pass of the grid (and
// the row has at most 8 flips per lane): the row, the targets and
// amplitudes of the lane's flips and the row's b-weighted occupation,
// formed once for all sweeps and kept in registers -- ranking the row and
// its flip targets again in every sweep cost more than the sweep's loads.
template <typename S>
struct RowCache {
  int64_t r;
  bool active;
  int64_t tg[8];   // slot q: the flip of bit lane + CL q, -1 where blocked or absent
  S amp[8];
  S nb;
};

template <typename S>
__device__ __forceinline__ void row_cache(const CoopAdj<S> &P, RowCache<S> &c) {
  const int lane = threadIdx.x & (CL - 1);
  const int64_t mine = (int64_t)blockIdx.x * (CNT / CL) + threadIdx.x / CL;
  c.active = mine < P.B.dim;
  c.r = c.active ? mine : 0;
  const uint64_t code = el::unrank_row(P.B, c.r);
  S nb = S(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int k = lane + CL * q;
    c.tg[q] = -1;
    c.amp[q] = S(0);
    if (k >= P.B.n) continue;
    if ((code >> k) & 1ULL) nb += P.bsh[k];
    const S amp = P.ahalf[k];
    if (amp == S(0)) continue;
    c.tg[q] = el::flip_target(P.B, code, c.r, k);
    c.amp[q] = amp;
  }
#pragma unroll
  for (int off = CL / 2; off > 0; off >>= 1) nb += __shfl_xor_sync(0xffffffffu, nb, off);
  c.nb = nb;
}

// One sweep over the basis:  y = alpha H_k x + beta x - z + conj-weighted
// lambda (cl = (clr, cli)), with optional accumulation into acc (mode 1:
// acc = w0 x + w y; mode 2: acc += w y) and optional gradient dots against t.
template <typename S>
struct Sweep {
  const S *x, *z, *lam, *t;
  S *y, *acc;
  S alpha, beta, clr, cli, wr, wi, w0r, w0i;
  int acc_mode;
};

template <typename S>
__device__ __forceinline__ void sweep(const CoopAdj<S> &P, S om, S dl, const Sweep<S> &W, double &gO, double &gD,
                                      const RowCache<S> &rc, bool cached) {
  const int64_t dim = P.B.dim;
  const int lane = threadIdx.x & (CL - 1);
  const int64_t rpb = CNT / CL;
  for (int64_t base = (int64_t)blockIdx.x * rpb; base < dim; base += (int64_t)gridDim.x * rpb) {
    int64_t r;
    bool active;
    S sre, sim, nb;
    if (cached) {
      r = rc.r;
      active = rc.active;
      sre = S(0); sim = S(0);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (rc.tg[q] < 0) continue;
        sre += rc.amp[q] * W.x[2 * rc.tg[q]];
        sim += rc.amp[q] * W.x[2 * rc.tg[q] + 1];
      }
#pragma unroll
      for (int off = CL / 2; off > 0; off >>= 1) {
        sre += __shfl_xor_sync(0xffffffffu, sre, off);
        sim += __shfl_xor_sync(0xffffffffu, sim, off);
      }
      nb = rc.nb;
    } else {
      const int64_t mine = base + threadIdx.x / CL;
      active = mine < dim;
      r = active ? mine : 0;
      const uint64_t code = el::unrank_row(P.B, r);
      row_flips<S>(P, code, r, lane, W.x, sre, sim, nb);
    }
    if (lane != 0 || !active) continue;
    const S xr = W.x[2 * r], xi = W.x[2 * r + 1];
    const S dsum = P.diagV[r] + dl * nb;
    const S hre = dsum * xr + om * sre, him = dsum * xi + om * sim;
    S yre = W.alpha * hre + W.beta * xr, yim = W.alpha * him + W.beta * xi;
    if (W.z) { yre -= W.z[2 * r]; yim -= W.z[2 * r + 1]; }
    if (W.lam) {
      const S lr = W.lam[2 * r], li = W.lam[2 * r + 1];
      yre += W.clr * lr - W.cli * li;
      yim += W.clr * li + W.cli * lr;
    }
    W.y[2 * r] = yre;
    W.y[2 * r + 1] = yim;
    if (W.acc_mode == 1) {
      W.acc[2 * r] = W.w0r * xr - W.w0i * xi + W.wr * yre - W.wi * yim;
      W.acc[2 * r + 1] = W.w0r * xi + W.w0i * xr + W.wr * yim + W.wi * yre;
    } else if (W.acc_mode == 2) {
      W.acc[2 * r] += W.wr * yre - W.wi * yim;
      W.acc[2 * r + 1] += W.wr * yim + W.wi * yre;
    }
    if (W.t) {
      const double tr = W.t[2 * r], ti = W.t[2 * r + 1];
      gO += (double)sre * tr + (double)sim * ti;                  // Re(conj(G_O x) t)
      gD += -(double)nb * ((double)xr * tr + (double)xi * ti);    // Re(conj(G_D x) t)
    }
  }
}

template <typename S>
// Two CTAs per SM (at most 128 registers): the pulse problems' bases then
// fit one pass of the grid, which the register cache of the rows needs.
__global__ void __launch_bounds__(CNT, 2) k_adjoint_coop(const CoopAdj<S> P) {
  __shared__ double red[2 * (CNT / 32)];
  __shared__ double s_ov[2];
  const int64_t dim = P.B.dim;
  const size_t vs = (size_t)dim * 2;   // values per complex vector
  unsigned gen = 0;
  auto sync = [&]() { coop_sync(P.bar, P.err, P.nctas, P.poll_limit, gen); };
  double g0 = 0.0, g1 = 0.0;
  // rows cached per lane when one pass of the grid covers the basis (and no
  // lane has more than 8 flips)
  RowCache<S> cache;
  const bool one_pass = dim <= (int64_t)gridDim.x * (CNT / CL) && P.B.n <= 8 * CL;
  if (one_pass) row_cache<S>(P, cache);
  // ---- forward: psi_{k+1} = sum_m c_m T_m(Htil_k) psi_k
  for (int k = 0; k < P.K; ++k) {
    const S a = (S)P.pa[k], b = (S)P.pb[k];
    const int M = P.pm[k];
    const double *c = P.pc + (size_t)k * (P.Mmax + 1) * 2;
    const S om = (S)P.om[k], dl = (S)P.dl[k];
    const S *x0 = P.ckp + (size_t)k * vs;
    S *out = P.ckp + (size_t)(k + 1) * vs;
    Sweep<S> W{};
    W.x = x0; W.y = P.term + vs; W.acc = out; W.acc_mode = 1;
    W.alpha = S(1) / a; W.beta = -b / a;
    W.w0r = (S)c[0]; W.w0i = (S)c[1]; W.wr = (S)c[2]; W.wi = (S)c[3];
    sweep<S>(P, om, dl, W, g0, g1, cache, one_pass);
    sync();
    for (int m = 2; m <= M; ++m) {
      Sweep<S> V{};
      V.x = P.term + (size_t)(m - 1) * vs;
      V.z = (m == 2) ? x0 : P.term + (size_t)(m - 2) * vs;
      V.y = P.term + (size_t)m * vs;
      V.acc = out; V.acc_mode = 2;
      V.alpha = S(2) / a; V.beta = S(-2) * b / a;
      V.wr = (S)c[2 * m]; V.wi = (S)c[2 * m + 1];
      sweep<S>(P, om, dl, V, g0, g1, cache, one_pass);
      sync();
    }
  }
  // ---- objective and lambda_K
  {
    const S *psi = P.ckp + (size_t)P.K * vs;
    double fa = 0.0, fb = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * CNT + threadIdx.x; r < dim; r += (int64_t)gridDim.x * CNT) {
      const double pr = psi[2 * r], pi = psi[2 * r + 1];
      if (P.target) {
        const double tr = P.target[2 * r], ti = P.target[2 * r + 1];
        fa += tr * pr + ti * pi;   // conj(target) psi
        fb += tr * pi - ti * pr;
      } else {
        fa += P.obs[r] * (pr * pr + pi * pi);
      }
    }
    block_sum2(fa, fb, red, P.fpart + 2 * blockIdx.x);
    sync();
    if (threadIdx.x == 0) {
      double sa = 0.0, sb = 0.0;
      for (int i = 0; i < P.nctas; ++i) { sa += __ldcg(&P.fpart[2 * i]); sb += __ldcg(&P.fpart[2 * i + 1]); }
      s_ov[0] = sa;
      s_ov[1] = sb;
      if (blockIdx.x == 0) { P.fout[0] = sa; P.fout[1] = sb; }
    }
    __syncthreads();
    const S ovr = (S)s_ov[0], ovi = (S)s_ov[1];
    for (int64_t r = (int64_t)blockIdx.x * CNT + threadIdx.x; r < dim; r += (int64_t)gridDim.x * CNT) {
      if (P.target) {   // lambda = <target, psi> target
        const S tr = P.target[2 * r], ti = P.target[2 * r + 1];
        P.lam[2 * r] = ovr * tr - ovi * ti;
        P.lam[2 * r + 1] = ovr * ti + ovi * tr;
      } else {          // lambda = O psi
        const S o = (S)P.obs[r];
        P.lam[2 * r] = o * psi[2 * r];
        P.lam[2 * r + 1] = o * psi[2 * r + 1];
      }
    }
    sync();
  }
  // ---- backward, one step at a time from the last
  for (int k = P.K - 1; k >= 0; --k) {
    const S a = (S)P.pa[k], b = (S)P.pb[k];
    const int M = P.pm[k];
    const double *c = P.pc + (size_t)k * (P.Mmax + 1) * 2;
    const S om = (S)P.om[k], dl = (S)P.dl[k];
    const S *x0 = P.ckp + (size_t)k * vs;
    // t_1 .. t_{M-1} of this step again from its checkpoint (t_0 = x0)
    for (int m = 1; m <= M - 1; ++m) {
      Sweep<S> V{};
      V.x = (m == 1) ? x0 : P.term + (size_t)(m - 1) * vs;
      V.z = (m == 1) ? nullptr : ((m == 2) ? x0 : P.term + (size_t)(m - 2) * vs);
      V.y = P.term + (size_t)m * vs;
      V.alpha = (m == 1 ? S(1) : S(2)) / a;
      V.beta = (m == 1 ? -b : S(-2) * b) / a;
      sweep<S>(P, om, dl, V, g0, g1, cache, one_pass);
      sync();
    }
    // u_M = conj(c_M) lambda
    {
      const S cr = (S)c[2 * M], ci = (S)(-c[2 * M + 1]);
      S *uM = P.U + (size_t)(M % 3) * vs;
      for (int64_t r = (int64_t)blockIdx.x * CNT + threadIdx.x; r < dim; r += (int64_t)gridDim.x * CNT) {
        const S lr = P.lam[2 * r], li = P.lam[2 * r + 1];
        uM[2 * r] = cr * lr - ci * li;
        uM[2 * r + 1] = cr * li + ci * lr;
      }
    }
    sync();
    // u_m = conj(c_m) lambda + (s/a)(H - b) u_{m+1} - u_{m+2}, with the dots of u_{m+1} and t_m
    for (int m = M - 1; m >= 0; --m) {
      const S s = (m == 0) ? S(1) : S(2);
      Sweep<S> V{};
      V.x = P.U + (size_t)((m + 1) % 3) * vs;
      V.z = (m + 2 <= M) ? P.U + (size_t)((m + 2) % 3) * vs : nullptr;
      V.y = P.U + (size_t)(m % 3) * vs;
      V.lam = P.lam;
      V.clr = (S)c[2 * m];
      V.cli = (S)(-c[2 * m + 1]);
      V.t = (m == 0) ? x0 : P.term + (size_t)m * vs;
      V.alpha = s / a;
      V.beta = -s * b / a;
      double gO = 0.0, gD = 0.0;
      sweep<S>(P, om, dl, V, gO, gD, cache, one_pass);
      block_sum2(gO, gD, red, P.part + (((size_t)k * (P.Mmax + 1) + (m + 1)) * P.nctas + blockIdx.x) * 2);
      sync();
    }
    // lambda_{k-1} = u_0
    {
      const S *u0 = P.U;
      for (int64_t r = (int64_t)blockIdx.x * CNT + threadIdx.x; r < (int64_t)vs; r += (int64_t)gridDim.x * CNT)
        P.lam[r] = u0[r];
    }
    sync();
  }
}

}  // namespace

// Run the cooperative gradient; plans[k] are the steps' expansions.  Fills
// hg[(k (Mmax + 1) + m) 2 + {0, 1}] (the per-term dots, as the stream path
// does) and F.  EL_ECUDA when a grid-barrier wait ran out.
template <typename S>
int adjoint_coop(el_ctx *ctx, el_ham *h, int K, const std::vector<ChebPlan> &plans, int Mmax,
                 const double *omega_k, const double *delta_k, const std::vector<double> &ash,
                 const std::vector<double> &bsh, const void *psi0, const void *target, const double *obs_diag,
                 void *buf, std::vector<double> &hg, double &F) {
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  const size_t vb = (size_t)dim * 2 * sizeof(S);
  int per_sm = 0, sms = 148;
  EL_CUDA_TRY(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  EL_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint_coop<S>, CNT, 0));
  if (per_sm < 1) return fail(ctx, EL_EINVAL, "cooperative adjoint kernel does not fit an SM");
  const int64_t rpb = CNT / CL;
  const int64_t want = (dim + rpb - 1) / rpb;
  const int nctas = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)per_sm * sms));
  // device tables: plans, drive, dots
  const size_t nplan = (size_t)K * (Mmax + 1) * 2;
  const size_t nparts = (size_t)K * (Mmax + 1) * nctas * 2;
  const size_t tab_doubles = 4 * (size_t)K + nplan + nparts + (size_t)nctas * 2 + 2;
  const size_t tab_bytes = tab_doubles * 8 + (size_t)K * 4 + 64;
  char *tb = (char *)el::workspace(ctx, 12, tab_bytes);
  if (!tb) return EL_ENOMEM;
  double *d_pa = (double *)tb, *d_pb = d_pa + K, *d_om = d_pb + K, *d_dl = d_om + K, *d_pc = d_dl + K;
  double *d_part = d_pc + nplan, *d_fpart = d_part + nparts, *d_fout = d_fpart + (size_t)nctas * 2;
  int *d_pm = (int *)(d_fout + 2);
  unsigned *d_sync = (unsigned *)(((uintptr_t)(d_pm + K) + 15) & ~(uintptr_t)15);   // [0] counter, [1] flag
  std::vector<double> hpa(K), hpb(K), hom(K), hdl(K), hpc(nplan, 0.0);
  std::vector<int> hpm(K);
  for (int k = 0; k < K; ++k) {
    hpa[k] = plans[k].a; hpb[k] = plans[k].b; hpm[k] = plans[k].M;
    hom[k] = omega_k[k]; hdl[k] = -delta_k[k];
    for (int m = 0; m <= plans[k].M; ++m) {
      hpc[((size_t)k * (Mmax + 1) + m) * 2] = plans[k].c_re[m];
      hpc[((size_t)k * (Mmax + 1) + m) * 2 + 1] = plans[k].c_im[m];
    }
  }
  EL_CUDA_TRY(ctx, el::copy(ctx, d_pa, hpa.data(), K * 8, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_pb, hpb.data(), K * 8, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_om, hom.data(), K * 8, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_dl, hdl.data(), K * 8, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_pc, hpc.data(), nplan * 8, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, d_pm, hpm.data(), K * 4, cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, cudaMemsetAsync(d_sync, 0, 2 * sizeof(unsigned), ctx->stream));
  // vectors: the stream path's layout
  char *vbuf = (char *)buf;
  EL_CUDA_TRY(ctx, el::copy(ctx, vbuf, psi0, vb, cudaMemcpyDeviceToDevice));
  CoopAdj<S> P;
  memset(&P, 0, sizeof P);
  P.B = el::basis_dev(h->basis);
  P.K = K; P.Mmax = Mmax; P.nctas = nctas; P.poll_limit = 1 << 22;
  P.pa = d_pa; P.pb = d_pb; P.pm = d_pm; P.pc = d_pc; P.om = d_om; P.dl = d_dl;
  if (std::is_same<S, float>::value) { int rc = el::ham_diag32(ctx, h); if (rc) return rc; }
  P.diagV = std::is_same<S, float>::value ? (const S *)(void *)h->d_diagV32 : (const S *)(void *)h->d_diagV64;
  for (int q = 0; q < n; ++q) {
    P.ahalf[q] = (S)(0.5 * ash[n - 1 - q]);
    P.bsh[q] = (S)bsh[n - 1 - q];
  }
  P.ckp = (S *)vbuf;
  P.term = (S *)(vbuf + (size_t)(K + 1) * vb);
  P.U = (S *)(vbuf + (size_t)(K + 1 + Mmax + 1) * vb);
  P.lam = (S *)(vbuf + (size_t)(K + 1 + Mmax + 1 + 3) * vb);
  P.target = (const S *)target;
  P.obs = obs_diag;
  P.part = d_part; P.fpart = d_fpart; P.fout = d_fout;
  P.bar = d_sync; P.err = (int *)(d_sync + 1);
  void *kargs[] = {(void *)&P};
  EL_CUDA_TRY(ctx, cudaLaunchCooperativeKernel((const void *)k_adjoint_coop<S>, dim3(nctas), dim3(CNT), kargs, 0,
                                               ctx->stream));
  ctx->launches++;
  std::vector<double> parts(nparts);
  double fo[2];
  unsigned hs[2];
  EL_CUDA_TRY(ctx, el::copy(ctx, parts.data(), d_part, nparts * 8, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, el::copy(ctx, fo, d_fout, 16, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, el::copy(ctx, hs, d_sync, 8, cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs[1]) return fail(ctx, EL_ECUDA, "cooperative adjoint: grid barrier timed out");
  hg.assign((size_t)K * (Mmax + 1) * 2, 0.0);
  for (int k = 0; k < K; ++k)
    for (int m = 1; m <= plans[k].M; ++m)
      for (int q = 0; q < 2; ++q) {
        double s = 0.0;
        for (int b = 0; b < nctas; ++b) s += parts[(((size_t)k * (Mmax + 1) + m) * nctas + b) * 2 + q];
        hg[((size_t)k * (Mmax + 1) + m) * 2 + q] = s;
      }
  F = target ? fo[0] * fo[0] + fo[1] * fo[1] : fo[0];
  return EL_OK;
}

template int adjoint_coop<float>(el_ctx *, el_ham *, int, const std::vector<ChebPlan> &, int, const double *,
                                 const double *, const std::vector<double> &, const std::vector<double> &,
                                 const void *, const void *, const double *, void *, std::vector<double> &,
                                 double &);
template int adjoint_coop<double>(el_ctx *, el_ham *, int, const std::vector<ChebPlan> &, int, const double *,
                                  const double *, const std::vector<double> &, const std::vector<double> &,
                                  const void *, const void *, const double *, void *, std::vector<double> &,
                                  double &);

}  // namespace el
