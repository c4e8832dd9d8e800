// Tiled KPM recurrence on the full 2^N basis (N <= 25), FP32 or FP64 vectors.
//
// Probe vectors are stored as 16-byte cells, [probe group][row] with 4 FP32
// (or 2 FP64) probes per cell, so every row access is a 16-byte vector load
// and a pair of adjacent rows fills a 32-byte DRAM sector.
//
// The sigma^x part of H is split by row bit into X = X_A + X_B:
//   group A = row bits [0, a)                 tiles: 2^a consecutive rows
//   group B = row bits [a, N) (+ row bit 0 as  tiles: 2^(N-a+1) rows, pairs of
//             the lowest tile bit, not applied) adjacent rows 2^a apart
// so X_A is local to an A tile and X_B to a B tile (tiles <= 2^13 rows, 128 KB
// of shared memory).  A Chebyshev step t_{m+1} = 2 Htil t_m - t_{m-1} is then
// one pass over the tiles of one group G, alternating A, B, A, ...:
//   P holds p_m = t_m minus its X_G t_{m-1} term, Q holds t_{m-1};
//   t_m     = p_m + s_m X_G t_{m-1}                     (stored over P)
//   p_{m+1} = 2(D-c)/r t_m + (2/r) X_G t_m - t_{m-1}   (stored over Q)
// and p_{m+1} lacks exactly X_{G'} t_m, which the next pass (group G') adds.
// Per element and step this reads 2 and writes 2 vectors.  The pass also
// yields <t_m, t_m> and <t_m, t_{m-1}>, from which the moments follow by
// T_2m = 2 T_m^2 - T_0 and T_2m-1 = 2 T_m T_m-1 - T_1.
#include "el_internal.cuh"

#include <algorithm>

namespace {

using el::fail;

template <typename T> struct CellT;
// V: the 16-byte cell of a row; U: the half cell one CTA works on (8 bytes).
template <> struct CellT<float> { typedef float4 V; typedef float2 U; static constexpr int PG = 4; };
template <> struct CellT<double> { typedef double2 V; typedef double U; static constexpr int PG = 2; };

__device__ __forceinline__ float2 u_zero(float2) { return make_float2(0.f, 0.f); }
__device__ __forceinline__ double u_zero(double) { return 0.0; }
__device__ __forceinline__ float2 u_fma(float s, float2 x, float2 y) {
  return make_float2(fmaf(s, x.x, y.x), fmaf(s, x.y, y.y));
}
__device__ __forceinline__ double u_fma(double s, double x, double y) { return fma(s, x, y); }
__device__ __forceinline__ float2 u_scale(float s, float2 x) { return make_float2(s * x.x, s * x.y); }
__device__ __forceinline__ double u_scale(double s, double x) { return s * x; }
__device__ __forceinline__ float2 u_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double u_sub(double a, double b) { return a - b; }
__device__ __forceinline__ double u_get(float2 v, int i) { return (double)(i ? v.y : v.x); }
__device__ __forceinline__ double u_get(double v, int) { return v; }

enum { PASS_A = 0, PASS_B = 1, PASS_ONE = 2 };
enum { MODE_STEP = 0, MODE_PROLOGUE = 1, MODE_LAST = 2 };

template <typename T>
struct PassArgs {
  int n, a, mode, ng, log_tiles;
  int64_t dim, tiles, items;
  T s_m, two_r, pro_alpha, pro_beta;
  T amp[16];               // per local bit (0 if not applied in this pass)
  const T *d2;             // 2 (D - c) / r per row
  void *P, *Q;             // cells [ng][dim]
  double *partials;        // [gridDim][ng * PG * 2]
  unsigned int *counter;
  double *dots;            // [ng * PG][2]
};

// Row of local cell l = tid + NT*j inside a tile: rbase(tid, tile) + j*jstride.
// Rows fit in 32 bits (dim <= 2^25), so per-cell offsets stay cheap.
template <int KIND, int NT>
__device__ __forceinline__ uint32_t row_base(int a, uint32_t tile, int tid) {
  if (KIND == PASS_A) return (tile << a) + (uint32_t)tid;
  if (KIND == PASS_B) return (uint32_t)(tid & 1) + ((uint32_t)(tid >> 1) << a) + (tile << 1);
  return (uint32_t)tid;
}
template <int KIND, int NT>
__device__ __forceinline__ uint32_t row_jstride(int a) {
  if (KIND == PASS_B) return (uint32_t)(NT / 2) << a;
  return (uint32_t)NT;
}


__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}

// Error-free accumulation of x*y into (s, c) in the working precision:
// TwoProduct by FMA and TwoSum (Ogita, Rump, Oishi, "Accurate sum and dot
// product", SIAM J. Sci. Comput. 26 (2005)); the pair is widened to FP64 once
// per tile.
__device__ __forceinline__ void dot2_acc(float x, float y, float &s, float &c) {
  const float p = x * y;
  const float e = fmaf(x, y, -p);
  const float t = s + p;
  const float z = t - s;
  c += (s - (t - z)) + (p - z) + e;
  s = t;
}
__device__ __forceinline__ void dot2_acc(double x, double y, double &s, double &c) {
  s = fma(x, y, s);
  (void)c;
}

template <typename T> struct Acc2 {
  T s[2][CellT<T>::PG / 2], c[2][CellT<T>::PG / 2];
};

// Gather of the shared-memory tile bits k in [k0, KMAX): sum amp_k * S[l ^ 2^k].
template <typename T, int K0, int KMAX>
__device__ __forceinline__ typename CellT<T>::U gather_s(const typename CellT<T>::U *S, int l,
                                                         const PassArgs<T> &A) {
  typedef typename CellT<T>::U U;
  U h0 = u_zero(U{}), h1 = u_zero(U{});
#pragma unroll
  for (int k = K0; k < KMAX; ++k) {
    const U x = S[l ^ (1 << k)];
    if (k & 1) h1 = u_fma(A.amp[k], x, h1); else h0 = u_fma(A.amp[k], x, h0);
  }
  return u_fma((T)1, h1, h0);
}

// One pass over (probe group, tile, half cell) work items; see the file
// header for the recurrence.  Shared memory holds two half-cell tiles:
//   S  = t_{m-1}            (gathered in phase 2, own cell read in phase 4)
//   S2 = p_m, then t_m      (updated in place in phase 2, gathered in phase 4)
// Each thread owns the R cells l = tid + NT*j; the tile bits above LOG2(NT)
// index j, so their partners are the thread's own cells, loaded once into
// registers per phase.
template <typename T, int TB, int KIND>
__global__ void __launch_bounds__(512, 1) k_kpm_pass(const PassArgs<T> A) {
  typedef typename CellT<T>::U U;
  constexpr int PH = CellT<T>::PG / 2;   // probes per half cell
  constexpr int R = TB >= 9 ? (1 << (TB - 9)) : 1;
  constexpr int NT = (1 << TB) / R;
  constexpr int LOGNT = TB >= 9 ? 9 : TB;
  constexpr int NWARP = NT / 32;
  constexpr int K0 = (KIND == PASS_B) ? 1 : 0;   // bit 0 of a B tile is not applied
  extern __shared__ __align__(16) unsigned char smem_raw[];
  U *S = reinterpret_cast<U *>(smem_raw);
  U *S2 = S + (1 << TB);
  __shared__ double wred[NWARP][2 * PH];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int ndots = A.ng * PH * 4;                   // [ng][2 halves][PH][2]
  double *dacc = A.partials + (size_t)blockIdx.x * ndots;
  for (int i = tid; i < ndots; i += NT) dacc[i] = 0.0;
  const T *__restrict__ d2 = A.d2;
  const T s_m = A.s_m, two_r = A.two_r;
  const uint32_t rs = row_jstride<KIND, NT>(A.a);

  for (int64_t item = blockIdx.x; item < A.items; item += gridDim.x) {
    // order: group, tile, half -- the two halves of a tile run side by side
    const int half = (int)(item & 1);
    const int64_t it2 = item >> 1;
    const int g = (int)(it2 >> A.log_tiles);       // tiles is a power of two
    const uint32_t tile = (uint32_t)(it2 & (A.tiles - 1));
    U *__restrict__ P = reinterpret_cast<U *>(A.P) + ((size_t)g * A.dim) * 2 + half;
    U *__restrict__ Q = reinterpret_cast<U *>(A.Q) + ((size_t)g * A.dim) * 2 + half;
    const uint32_t rb = row_base<KIND, NT>(A.a, tile, tid);
    // phase 1: Q tile -> S, P tile -> S2 (asynchronous copies)
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const uint32_t row = rb + rs * (uint32_t)j;
      cp_async8(&S[tid + NT * j], &Q[2 * (size_t)row]);
      if (A.mode != MODE_PROLOGUE) cp_async8(&S2[tid + NT * j], &P[2 * (size_t)row]);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    Acc2<T> ac;
#pragma unroll
    for (int q = 0; q < PH; ++q) { ac.s[0][q] = ac.c[0][q] = ac.s[1][q] = ac.c[1][q] = (T)0; }
    U own[R];

    if (A.mode == MODE_PROLOGUE) {
      // p_1 = (D-c)/r t_0 + pro_beta X_G t_0, written to P
#pragma unroll
      for (int j = 0; j < R; ++j) own[j] = S[tid + NT * j];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int l = tid + NT * j;
        const uint32_t row = rb + rs * (uint32_t)j;
        U out = u_scale(A.pro_alpha * d2[row], own[j]);
        if (KIND != PASS_ONE) {
          U hx = gather_s<T, K0, LOGNT>(S, l, A);
#pragma unroll
          for (int b = 0; (1 << b) < R; ++b) hx = u_fma(A.amp[LOGNT + b], own[j ^ (1 << b)], hx);
          out = u_fma(A.pro_beta, hx, out);
        }
        P[2 * (size_t)row] = out;
#pragma unroll
        for (int q = 0; q < PH; ++q) {
          const T xv = (T)u_get(own[j], q);
          dot2_acc(xv, xv, ac.s[0][q], ac.c[0][q]);
        }
      }
    } else {
      // phase 2: t_m = p_m + s_m X_G t_{m-1}   (t_m over S2 and into P)
#pragma unroll
      for (int j = 0; j < R; ++j) own[j] = S[tid + NT * j];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int l = tid + NT * j;
        U hx = gather_s<T, K0, LOGNT>(S, l, A);
#pragma unroll
        for (int b = 0; (1 << b) < R; ++b) hx = u_fma(A.amp[LOGNT + b], own[j ^ (1 << b)], hx);
        const U acc = u_fma(s_m, hx, S2[l]);
        if (A.mode != MODE_LAST) {
          S2[l] = acc;
          P[2 * (size_t)(rb + rs * (uint32_t)j)] = acc;
        }
#pragma unroll
        for (int q = 0; q < PH; ++q) {
          const T av = (T)u_get(acc, q);
          dot2_acc(av, av, ac.s[0][q], ac.c[0][q]);
          dot2_acc(av, (T)u_get(own[j], q), ac.s[1][q], ac.c[1][q]);
        }
      }
      if (A.mode != MODE_LAST) {
        __syncthreads();
        // phase 4: p_{m+1} = d2 t_m + (2/r) X_G t_m - t_{m-1}   (into Q).
        // With a single tile group the X term is left to the next pass.
#pragma unroll
        for (int j = 0; j < R; ++j) own[j] = S2[tid + NT * j];
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int l = tid + NT * j;
          const uint32_t row = rb + rs * (uint32_t)j;
          U out = u_scale(d2[row], own[j]);
          if (KIND != PASS_ONE) {
            U hx = gather_s<T, K0, LOGNT>(S2, l, A);
#pragma unroll
            for (int b = 0; (1 << b) < R; ++b) hx = u_fma(A.amp[LOGNT + b], own[j ^ (1 << b)], hx);
            out = u_fma(two_r, hx, out);
          }
          Q[2 * (size_t)row] = u_sub(out, S[l]);
        }
      }
    }
    // per-item dot partials: widen once, warp shuffle, fixed-order warp sum
#pragma unroll
    for (int q = 0; q < PH; ++q) {
      double x = (double)ac.s[0][q] + (double)ac.c[0][q];
      double y = (double)ac.s[1][q] + (double)ac.c[1][q];
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) { wred[warp][2 * q] = x; wred[warp][2 * q + 1] = y; }
    }
    __syncthreads();
    if (tid < 2 * PH) {
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
      dacc[(g * 2 + half) * PH * 2 + tid] += sum;
    }
    // the next item's first shared-memory write happens after this barrier
    __syncthreads();
  }
  // cross-CTA deterministic reduction (own partial row already in place)
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(A.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int i = tid; i < ndots; i += NT) {
    double sum = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) sum += __ldcg(&A.partials[(size_t)b * ndots + i]);
    A.dots[i] = sum;
  }
  if (tid == 0) *A.counter = 0u;
}

// probes -> cells [ng][dim]; probe p = g*PG + lane; probes >= nvalid are zero
template <typename T>
__global__ void k_cells_rademacher(int64_t dim, int ng, uint64_t seed, int64_t probe0,
                                   int nvalid, const int8_t *probes, T *out) {
  constexpr int PG = CellT<T>::PG;
  const int64_t total = dim * ng * PG;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int lane = (int)(t % PG);
    const int64_t cell = t / PG;
    const int64_t row = cell % dim;
    const int g = (int)(cell / dim);
    const int p = g * PG + lane;
    T v = 0;
    if (p < nvalid)
      v = probes ? (T)probes[(int64_t)p * dim + row]
                 : (T)el::rademacher(seed, (uint64_t)(probe0 + p), (uint64_t)row);
    out[t] = v;
  }
}

template <typename T>
__global__ void k_d2(BasisDev B, const double *diagV, const double *delta_bits, double c,
                     double r, T *out) {
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < B.dim;
       row += (int64_t)gridDim.x * blockDim.x) {
    double d = diagV[row];
    for (int k = 0; k < B.n; ++k) if ((row >> k) & 1) d += delta_bits[k];
    out[row] = (T)(2.0 * (d - c) / r);
  }
}

template <typename T>
int run_passes(el_ctx *ctx, el_ham *h, int nvalid_total, int chunk, uint64_t seed,
               const int8_t *probes_host, int num, double c, double r, std::vector<double> &acc) {
  constexpr int PG = CellT<T>::PG;
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  const int ng = chunk / PG;
  const size_t vb = (size_t)dim * chunk * sizeof(T);
  char *buf = (char *)el::workspace(ctx, 6, 2 * vb + (size_t)dim * sizeof(T));
  if (!buf) return EL_ENOMEM;
  void *P = buf, *Q = buf + vb;
  T *d2 = reinterpret_cast<T *>(buf + 2 * vb);
  const int M = (num + 1) / 2;  // passes producing t_1 .. t_M
  double *d_dots = (double *)el::workspace(ctx, 7, (size_t)(M + 1) * chunk * 2 * sizeof(double));
  if (!d_dots) return EL_ENOMEM;
  int8_t *d_probe8 = nullptr;
  if (probes_host) {
    d_probe8 = (int8_t *)el::workspace(ctx, 2, (size_t)dim * chunk);
    if (!d_probe8) return EL_ENOMEM;
  }
  // 2(D - c)/r
  {
    double *d_delta = (double *)el::workspace(ctx, 8, 64 * sizeof(double));
    if (!d_delta) return EL_ENOMEM;
    EL_CUDA_TRY(ctx, el::copy(ctx, d_delta, h->delta, 64 * sizeof(double), cudaMemcpyHostToDevice));
    BasisDev B = el::basis_dev(h->basis);
    k_d2<T><<<el::grid_for(dim, 256), 256, 0, ctx->stream>>>(B, h->d_diagV64, d_delta, c, r, d2);
    EL_LAUNCH_CHECK(ctx);
  }
  // group split
  const bool one = (n <= 13);
  int a = n;
  if (!one) a = std::min(13, std::max((n + 2) / 2, n - 12));
  const int TBA = one ? n : a, TBB = one ? n : n - a + 1;
  int dev_sms = 148;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
  auto make = [&](int kind, int mode, double s_m, int *tb_out) {
    PassArgs<T> A;
    memset(&A, 0, sizeof A);
    A.n = n; A.a = a; A.mode = mode; A.ng = ng; A.dim = dim;
    const int TB = (kind == PASS_B) ? TBB : TBA;
    *tb_out = TB;
    A.tiles = (kind == PASS_A && !one) ? (dim >> a) : (kind == PASS_B ? ((int64_t)1 << (a - 1)) : 1);
    A.items = A.tiles * ng * 2;
    A.log_tiles = 0;
    while (((int64_t)1 << A.log_tiles) < A.tiles) ++A.log_tiles;
    A.s_m = (T)s_m; A.two_r = (T)(2.0 / r);
    for (int k = 0; k < TB; ++k) {
      int rowbit = -1;
      if (kind == PASS_A || kind == PASS_ONE) rowbit = k;
      else if (k >= 1) rowbit = a + k - 1;
      A.amp[k] = (T)((rowbit >= 0) ? 0.5 * h->om_re[rowbit] : 0.0);
    }
    A.d2 = d2; A.P = P; A.Q = Q;
    A.counter = ctx->d_counter;
    return A;
  };
  auto launch = [&](PassArgs<T> &A, int kind, int tb) -> int {
    const int R = tb >= 9 ? (1 << (tb - 9)) : 1;
    const int NT = (1 << tb) / R;
    const size_t smem = ((size_t)1 << tb) * 8 * 2;
    const int per_sm = smem <= 96 * 1024 ? 2 : 1;
    int grid = (int)std::min<int64_t>(A.items, (int64_t)dev_sms * per_sm);
    int rc = el::ensure_partials(ctx, (size_t)grid * ng * PG * 2);
    if (rc) return rc;
    A.partials = ctx->d_partials;
    bool ok = false;
#define EL_CASE(TBV, KV)                                                                   \
  if (tb == TBV && kind == KV) {                                                           \
    cudaFuncSetAttribute(k_kpm_pass<T, TBV, KV>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                         (int)smem);                                                       \
    k_kpm_pass<T, TBV, KV><<<grid, NT, smem, ctx->stream>>>(A);                            \
    ok = true;                                                                             \
  }
#define EL_KINDS(TBV) EL_CASE(TBV, PASS_A) EL_CASE(TBV, PASS_B) EL_CASE(TBV, PASS_ONE)
    EL_KINDS(6) EL_KINDS(7) EL_KINDS(8) EL_KINDS(9) EL_KINDS(10) EL_KINDS(11) EL_KINDS(12) EL_KINDS(13)
#undef EL_KINDS
#undef EL_CASE
    if (!ok) return fail(ctx, EL_EINVAL, "tile of %d bits not instantiated", tb);
    EL_LAUNCH_CHECK(ctx);
    return EL_OK;
  };
  std::vector<double> hd((size_t)(M + 1) * chunk * 2);
  for (int done = 0; done < nvalid_total; done += chunk) {
    const int b = std::min(chunk, nvalid_total - done);
    if (probes_host) {
      EL_CUDA_TRY(ctx, el::copy(ctx, d_probe8, probes_host + (size_t)done * dim, (size_t)dim * b, cudaMemcpyHostToDevice));
    }
    k_cells_rademacher<T><<<el::grid_for(dim * chunk, 256), 256, 0, ctx->stream>>>(
        dim, ng, seed, done, b, d_probe8, reinterpret_cast<T *>(Q));
    EL_LAUNCH_CHECK(ctx);
    // prologue: p_1 from t_0 on the other group's tiles
    int tb = 0;
    const int k0 = one ? PASS_ONE : PASS_B;
    PassArgs<T> A0 = make(k0, MODE_PROLOGUE, 0.0, &tb);
    A0.pro_alpha = (T)0.5;
    A0.pro_beta = (T)(one ? 0.0 : 1.0 / r);
    A0.dots = d_dots;
    int rc = launch(A0, k0, tb);
    if (rc) return rc;
    for (int m = 1; m <= M; ++m) {
      if ((m & 63) == 0 && el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
      const int kind = one ? PASS_ONE : ((m & 1) ? PASS_A : PASS_B);
      PassArgs<T> Am = make(kind, m == M ? MODE_LAST : MODE_STEP, m == 1 ? 1.0 / r : 2.0 / r, &tb);
      Am.dots = d_dots + (size_t)m * chunk * 2;
      rc = launch(Am, kind, tb);
      if (rc) return rc;
      std::swap(P, Q);
    }
    // swap back so the buffers keep their roles for the next chunk
    if (M & 1) std::swap(P, Q);
    EL_CUDA_TRY(ctx, el::copy(ctx, hd.data(), d_dots, hd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int p = 0; p < b; ++p) {
      const double mu0 = hd[(size_t)p * 2];                       // <t0, t0>
      const double mu1 = hd[((size_t)chunk + p) * 2 + 1];         // <t1, t0>
      acc[0] += mu0;
      if (num >= 1) acc[1] += mu1;
      for (int m = 1; m <= M; ++m) {
        const double tt = hd[((size_t)m * chunk + p) * 2];
        const double tq = hd[((size_t)m * chunk + p) * 2 + 1];
        if (2 * m <= num) acc[2 * m] += 2.0 * tt - mu0;
        if (m >= 2 && 2 * m - 1 <= num) acc[2 * m - 1] += 2.0 * tq - mu1;
      }
    }
  }
  return EL_OK;
}

}  // namespace

namespace el {

bool kpm_full_eligible(const el_ham *h, int dtype, int chunk, int mode) {
  if (mode != EL_KPM_DOUBLING) return false;
  if (h->basis->layout != EL_LAYOUT_FULL) return false;
  if (!h->px.empty()) return false;   // sigma^x channels only
  if (h->n < 6 || h->n > 25) return false;
  if (h->complex_drive) return false;
  const int pg = (dtype == EL_F32) ? 4 : 2;
  if (chunk % pg != 0 || chunk / pg > 64) return false;
  return dtype == EL_F32 || dtype == EL_F64;
}

int kpm_full(el_ctx *ctx, el_ham *h, int dtype, int num, int nvec, int chunk, uint64_t seed,
             const int8_t *probes_host, double c, double r, double *mu_host) {
  std::vector<double> acc(num + 1, 0.0);
  int rc = (dtype == EL_F32)
               ? run_passes<float>(ctx, h, nvec, chunk, seed, probes_host, num, c, r, acc)
               : run_passes<double>(ctx, h, nvec, chunk, seed, probes_host, num, c, r, acc);
  if (rc) return rc;
  const double norm = 1.0 / ((double)nvec * (double)h->basis->dim);
  for (int k = 0; k <= num; ++k) mu_host[k] = acc[k] * norm;
  return EL_OK;
}

}  // namespace el
