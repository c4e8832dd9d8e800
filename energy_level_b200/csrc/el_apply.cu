// Generic fused H-apply kernel and the vector helpers used by the drivers.
//
// One thread handles one (row, vector) element of a block [dim][nvec]; the
// nvec lanes of a row are adjacent, so every flip gather of a row block is a
// contiguous nvec-element segment.  For each row the kernel
//   - recovers the configuration code (arithmetic unranking or code table),
//   - accumulates the delta part of the diagonal bit by bit,
//   - gathers x[target] for every sigma^x flip whose target is in the basis
//     (flip targets computed arithmetically or from the class tables),
// and fuses the caller's recurrence  y = a*Hx + b*x + c*z,  acc += w*y  and
// the FP64 dot products the drivers need (moments, alpha, beta, norms).
// Channel semantics: channels.py:58-132 (diagonal delta n + V n n, sigma^x
// amplitude Omega/2 into |r>, conj(Omega)/2 into |g>).
#include "el_internal.cuh"

#include <algorithm>

namespace {

using el::fail;

template <typename S>
struct HamArgs {
  const S *diagV;
  S delta[EL_MAX_SITES];
  S up_re[EL_MAX_SITES];  // amplitude into a row whose bit k is 1: Omega/2
  S up_im[EL_MAX_SITES];  // (into a row whose bit k is 0: conj(Omega)/2)
  const ExPair *px;       // exchange channels (generic kernel only)
  int npx;
  int lossy;              // loss diagonal present (generic kernel only)
  int real_amp;           // every sigma^x amplitude is real (row kernel: cheaper complex FMAs)
  S loss[EL_MAX_SITES];   // imaginary diagonal per set bit: -gamma/2 (evolution units)
};

// Amplitude <row|H|row ^ (bit bi | bit bj)> of exchange pair e for a row whose
// bits at bi, bj are (si, sj): J channel (channels.py:121-125) when the bits
// differ -- J into (r, g), conj(J) into (g, r) -- and A channel
// (channels.py:126-130) when they agree -- A into (r, r), conj(A) into (g, g).
__device__ __forceinline__ void exchange_amp(const ExPair &e, bool si, bool sj,
                                             double &re, double &im) {
  if (si != sj) { re = e.jre; im = si ? e.jim : -e.jim; }
  else { re = e.are; im = si ? e.aim : -e.aim; }
}

struct KArgs {
  int64_t nvec;
  int lognv;
  const void *x;
  const void *z;
  void *y;
  void *acc;
  double a, b, c, w_re, w_im;
  double *dots;
  int want;
  int skip_diag;
  const void *probe;
  double *partials;
  unsigned int *counter;
};

template <typename S, bool C> struct Val;
template <typename S> struct Val<S, false> {
  S v;
  __device__ static Val load(const void *p, int64_t i) { Val r; r.v = ((const S *)p)[i]; return r; }
  __device__ void store(void *p, int64_t i) const { ((S *)p)[i] = v; }
};
template <typename S> struct Val<S, true> {
  S re, im;
  __device__ static Val load(const void *p, int64_t i) {
    Val r; r.re = ((const S *)p)[2 * i]; r.im = ((const S *)p)[2 * i + 1]; return r;
  }
  __device__ void store(void *p, int64_t i) const { ((S *)p)[2 * i] = re; ((S *)p)[2 * i + 1] = im; }
};

// Block reduction of 4 doubles per thread into per-(vector, quantity) sums,
// then a deterministic cross-block sum by the last block to finish.
__device__ void reduce4(const KArgs &K, double q0, double q1, double q2, double q3) {
  __shared__ double red[256][4];
  __shared__ bool last;
  const int tid = threadIdx.x;
  red[tid][0] = q0; red[tid][1] = q1; red[tid][2] = q2; red[tid][3] = q3;
  __syncthreads();
  const int nv = (int)K.nvec;            // nvec divides 256
  const int per = 256 / nv;
  const int nout = nv * 4;
  for (int o = tid; o < nout; o += 256) {
    const int v = o >> 2, q = o & 3;
    double s = 0.0;
    for (int j = 0; j < per; ++j) s += red[v + j * nv][q];
    K.partials[(size_t)blockIdx.x * nout + o] = s;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(K.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int o = tid; o < nout; o += 256) {
    double s = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(&K.partials[(size_t)b * nout + o]);
    K.dots[o] = s;
  }
  if (tid == 0) *K.counter = 0u;
}

template <typename S, bool C>
__global__ void __launch_bounds__(256) k_apply(BasisDev B, HamArgs<S> H, KArgs K) {
  typedef Val<S, C> V;
  const int64_t total = B.dim * K.nvec;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int64_t row = t >> K.lognv;
    const int64_t v = t & (K.nvec - 1);
    const uint64_t code = el::unrank_row(B, row);
    const V xr = V::load(K.x, t);
    S hre = 0, him = 0, dsum = 0, dimg = 0;
    for (int k = 0; k < B.n; ++k) {
      const bool set = (code >> k) & 1ULL;
      if (set) {
        dsum += H.delta[k];
        if constexpr (C) dimg += H.loss[k];
      }
      const S are = H.up_re[k];
      const S aim = C ? (set ? H.up_im[k] : -H.up_im[k]) : S(0);
      if (are == S(0) && aim == S(0)) continue;
      const int64_t tg = el::flip_target(B, code, row, k);
      if (tg < 0) continue;
      const V xs = V::load(K.x, (tg << K.lognv) + v);
      if constexpr (C) {
        hre += are * xs.re - aim * xs.im;
        him += are * xs.im + aim * xs.re;
      } else {
        hre += are * xs.v;
      }
    }
    for (int p = 0; p < H.npx; ++p) {
      const ExPair e = H.px[p];
      double pre, pim;
      exchange_amp(e, (code >> e.bi) & 1ULL, (code >> e.bj) & 1ULL, pre, pim);
      if (pre == 0.0 && pim == 0.0) continue;
      const int64_t tg = el::rank_any(B, code ^ ((1ULL << e.bi) | (1ULL << e.bj)));
      if (tg < 0) continue;
      const V xs = V::load(K.x, (tg << K.lognv) + v);
      const S are = (S)pre, aim = (S)pim;
      if constexpr (C) {
        hre += are * xs.re - aim * xs.im;
        him += are * xs.im + aim * xs.re;
      } else {
        hre += are * xs.v;
      }
    }
    if (!K.skip_diag) {
      dsum += H.diagV[row];
      if constexpr (C) {
        hre += dsum * xr.re - dimg * xr.im;
        him += dsum * xr.im + dimg * xr.re;
      } else {
        hre += dsum * xr.v;
      }
    }
    V yv;
    if constexpr (C) {
      yv.re = (S)K.a * hre + (S)K.b * xr.re;
      yv.im = (S)K.a * him + (S)K.b * xr.im;
      if (K.z) { const V zv = V::load(K.z, t); yv.re += (S)K.c * zv.re; yv.im += (S)K.c * zv.im; }
      if (K.acc) {
        V av = V::load(K.acc, t);
        av.re += (S)K.w_re * yv.re - (S)K.w_im * yv.im;
        av.im += (S)K.w_re * yv.im + (S)K.w_im * yv.re;
        av.store(K.acc, t);
      }
    } else {
      yv.v = (S)K.a * hre + (S)K.b * xr.v;
      if (K.z) { const V zv = V::load(K.z, t); yv.v += (S)K.c * zv.v; }
      if (K.acc) { V av = V::load(K.acc, t); av.v += (S)K.w_re * yv.v; av.store(K.acc, t); }
    }
    if (K.y) yv.store(K.y, t);
    if (K.want) {
      // FP32 values are widened before multiplying: the products are exact in
      // FP64, so only the FP64 summation rounds.
      if constexpr (C) {
        const double xre = xr.re, xim = xr.im, yre = yv.re, yim = yv.im;
        q0 += xre * xre + xim * xim;
        q1 += xre * yre + xim * yim;
        q2 += xre * yim - xim * yre;
        q3 += yre * yre + yim * yim;
      } else {
        const double xd = xr.v, yd = yv.v;
        q0 += xd * xd;
        q1 += xd * yd;
        q3 += yd * yd;
        if (K.probe) q2 += yd * (double)V::load(K.probe, t).v;
      }
    }
  }
  if (K.want) reduce4(K, q0, q1, q2, q3);
}

// --------------------------------------------- hop kernel (exchange channels)
// H with exchange channels on a FULL or TABLE (fixed-excitation, general
// restricted) basis of at most 32 sites: the generic kernel's per-element
// work, but the J channels are visited as hops -- every (set bit a, clear bit
// b) pair of the row, k (n - k) of them, with the amplitude from a table in
// shared memory -- instead of testing every site pair, codes and table ranks
// are 32-bit, and only the pairs with a nonzero A are scanned.
__device__ __forceinline__ int rank32(const BasisDev &B, uint32_t c) {
  if (B.layout == EL_LAYOUT_FULL) return (int)c;
  const uint32_t p = c >> B.L, sfx = c & ((1u << B.L) - 1u);
  const int64_t off = B.pre_off[p];
  if (off < 0) return -1;
  const int32_t rr = B.suf_rank[((uint32_t)B.pre_cls[p] << B.L) + sfx];
  return rr < 0 ? -1 : (int)off + rr;
}

template <typename S, bool C>
__global__ void __launch_bounds__(256) k_apply_hop(BasisDev B, HamArgs<S> H, KArgs K, const double *hop,
                                                   const ExPair *pxA, int npxA) {
  typedef Val<S, C> V;
  extern __shared__ __align__(16) unsigned char hop_smem[];
  const int n = B.n;
  S *hre_t = reinterpret_cast<S *>(hop_smem);
  S *him_t = hre_t + n * n;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
    hre_t[i] = (S)hop[i];
    if constexpr (C) him_t[i] = (S)hop[n * n + i];
  }
  __syncthreads();
  const uint32_t full = (n >= 32) ? 0xffffffffu : ((1u << n) - 1u);
  const int64_t total = B.dim * K.nvec;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
    const int64_t row = t >> K.lognv;
    const int64_t v = t & (K.nvec - 1);
    const uint32_t code = (B.layout == EL_LAYOUT_FULL) ? (uint32_t)row : (uint32_t)B.codes[row];
    const V xr = V::load(K.x, t);
    S hre = 0, him = 0, dsum = 0, dimg = 0;
    for (uint32_t m = code; m; m &= m - 1) {
      const int k = __ffs(m) - 1;
      dsum += H.delta[k];
      if constexpr (C) dimg += H.loss[k];
    }
    // sigma^x channels (bits with a nonzero Omega)
    for (int k = 0; k < n; ++k) {
      const bool set = (code >> k) & 1u;
      const S are = H.up_re[k];
      const S aim = C ? (set ? H.up_im[k] : -H.up_im[k]) : S(0);
      if (are == S(0) && aim == S(0)) continue;
      const int tg = rank32(B, code ^ (1u << k));
      if (tg < 0) continue;
      const V xs = V::load(K.x, ((int64_t)tg << K.lognv) + v);
      if constexpr (C) { hre += are * xs.re - aim * xs.im; him += are * xs.im + aim * xs.re; }
      else { hre += are * xs.v; }
    }
    // J channels: move one excitation from a set bit a to a clear bit b
    for (uint32_t ma = code; ma; ma &= ma - 1) {
      const int a = __ffs(ma) - 1;
      const S *hr = hre_t + a * n;
      const S *hi = him_t + a * n;
      for (uint32_t mb = ~code & full; mb; mb &= mb - 1) {
        const int b = __ffs(mb) - 1;
        const S are = hr[b];
        const S aim = C ? hi[b] : S(0);
        if (are == S(0) && aim == S(0)) continue;
        const int tg = rank32(B, code ^ (1u << a) ^ (1u << b));
        if (tg < 0) continue;
        const V xs = V::load(K.x, ((int64_t)tg << K.lognv) + v);
        if constexpr (C) { hre += are * xs.re - aim * xs.im; him += are * xs.im + aim * xs.re; }
        else { hre += are * xs.v; }
      }
    }
    // A channels: create or remove both excitations
    for (int p = 0; p < npxA; ++p) {
      const ExPair e = pxA[p];
      const bool si = (code >> e.bi) & 1u, sj = (code >> e.bj) & 1u;
      if (si != sj) continue;
      const S are = (S)e.are;
      const S aim = C ? (S)(si ? e.aim : -e.aim) : S(0);
      const int tg = rank32(B, code ^ (1u << e.bi) ^ (1u << e.bj));
      if (tg < 0) continue;
      const V xs = V::load(K.x, ((int64_t)tg << K.lognv) + v);
      if constexpr (C) { hre += are * xs.re - aim * xs.im; him += are * xs.im + aim * xs.re; }
      else { hre += are * xs.v; }
    }
    if (!K.skip_diag) {
      dsum += H.diagV[row];
      if constexpr (C) {
        hre += dsum * xr.re - dimg * xr.im;
        him += dsum * xr.im + dimg * xr.re;
      } else {
        hre += dsum * xr.v;
      }
    }
    V yv;
    if constexpr (C) {
      yv.re = (S)K.a * hre + (S)K.b * xr.re;
      yv.im = (S)K.a * him + (S)K.b * xr.im;
      if (K.z) { const V zv = V::load(K.z, t); yv.re += (S)K.c * zv.re; yv.im += (S)K.c * zv.im; }
      if (K.acc) {
        V av = V::load(K.acc, t);
        av.re += (S)K.w_re * yv.re - (S)K.w_im * yv.im;
        av.im += (S)K.w_re * yv.im + (S)K.w_im * yv.re;
        av.store(K.acc, t);
      }
    } else {
      yv.v = (S)K.a * hre + (S)K.b * xr.v;
      if (K.z) { const V zv = V::load(K.z, t); yv.v += (S)K.c * zv.v; }
      if (K.acc) { V av = V::load(K.acc, t); av.v += (S)K.w_re * yv.v; av.store(K.acc, t); }
    }
    if (K.y) yv.store(K.y, t);
    if (K.want) {
      if constexpr (C) {
        const double xre = xr.re, xim = xr.im, yre = yv.re, yim = yv.im;
        q0 += xre * xre + xim * xim;
        q1 += xre * yre + xim * yim;
        q2 += xre * yim - xim * yre;
        q3 += yre * yre + yim * yim;
      } else {
        const double xd = xr.v, yd = yv.v;
        q0 += xd * xd;
        q1 += xd * yd;
        q3 += yd * yd;
        if (K.probe) q2 += yd * (double)V::load(K.probe, t).v;
      }
    }
  }
  if (K.want) reduce4(K, q0, q1, q2, q3);
}

// ------------------------------------------------- row kernel (FULL/CHAIN/RING)
// One thread per row and all NV vectors of that row (NV <= 8): the code of a
// row is recovered once and every flip gather moves the row's whole NV-vector
// segment with 16-byte loads.  The bit loop runs over k = 0..n-1 in the same
// order in every thread (warp-uniform k), so Fibonacci weights, amplitudes
// and detunings are broadcast kernel-parameter reads; a flip that leaves the
// basis only predicates its load off.  Four bits per round (eight per lane
// when G lanes share a row, below) issue their gathers before any of them
// is accumulated.  CT/RT are 32-bit when the
// code has at most 32 bits and the basis fewer than 2^31 rows, which halves
// the integer work of unranking and target arithmetic.
//
// G > 1 (single vector, small bases): G adjacent lanes of a warp share one
// row and take the bits k = lane, lane + G, ...; their partial flip sums and
// detunings meet in a butterfly of warp shuffles and the row's first lane
// runs the epilogue.  A basis of a few ten thousand rows fills only part of
// the 148 SMs with one thread per row, and each thread then waits for n
// dependent rounds of gathers; G lanes per row cut that chain by G and give
// the grid G times more warps.  The row loop is uniform over the block so
// that every lane reaches the shuffles; lanes past the last row work on
// row 0 and store nothing.

template <typename S, int W>
__device__ __forceinline__ void ld_row(const S *p, S (&v)[W]) {
  constexpr int BYTES = W * (int)sizeof(S);
  if constexpr (BYTES % 16 == 0) {
    union { uint4 u[BYTES / 16]; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) t.u[i] = reinterpret_cast<const uint4 *>(p)[i];
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = t.s[i];
  } else if constexpr (BYTES == 8) {
    union { uint2 u; S s[W]; } t;
    t.u = *reinterpret_cast<const uint2 *>(p);
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = t.s[i];
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = p[i];
  }
}

template <typename S, int W>
__device__ __forceinline__ void st_row(S *p, const S (&v)[W]) {
  constexpr int BYTES = W * (int)sizeof(S);
  if constexpr (BYTES % 16 == 0) {
    union { uint4 u[BYTES / 16]; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < W; ++i) t.s[i] = v[i];
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) reinterpret_cast<uint4 *>(p)[i] = t.u[i];
  } else if constexpr (BYTES == 8) {
    union { uint2 u; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < W; ++i) t.s[i] = v[i];
    *reinterpret_cast<uint2 *>(p) = t.u;
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) p[i] = v[i];
  }
}

// Code of `row` (FULL / CHAIN / RING) in CT arithmetic.
template <int LAY, typename CT, typename RT>
__device__ __forceinline__ CT unrank_fib(const BasisDev &B, RT row) {
  if constexpr (LAY == EL_LAYOUT_FULL) {
    return (CT)row;
  } else {
    const int n = B.n;
    RT r = row;
    CT c = 0;
    if constexpr (LAY == EL_LAYOUT_CHAIN) {
      for (int k = n - 1; k >= 0; --k) {
        const RT w = (RT)B.fib[k + 2];
        if (r >= w) { c |= (CT)1 << k; r -= w; }
      }
      return c;
    } else {
      const RT split = (RT)B.fib[n + 1];
      if (r < split) {
        for (int k = n - 2; k >= 0; --k) {
          const RT w = (RT)B.fib[k + 2];
          if (r >= w) { c |= (CT)1 << k; r -= w; }
        }
        return c;
      }
      r -= split;
      c = (CT)1 << (n - 1);
      for (int k = n - 3; k >= 1; --k) {
        const RT w = (RT)B.fib[k + 1];
        if (r >= w) { c |= (CT)1 << k; r -= w; }
      }
      return c;
    }
  }
}

// Rank of an allowed ring code.
template <typename CT, typename RT>
__device__ __forceinline__ RT ring_rank_t(const BasisDev &B, CT c, int n) {
  RT r = 0;
  if ((c >> (n - 1)) & 1) {
    r = (RT)B.fib[n + 1];
    for (int k = 0; k < n - 1; ++k)
      if ((c >> k) & 1) r += (RT)B.fib[k + 1];
  } else {
    for (int k = 0; k < n; ++k)
      if ((c >> k) & 1) r += (RT)B.fib[k + 2];
  }
  return r;
}

template <typename S, bool C, int NV, int LAY, bool WANT, typename CT, typename RT, int G>
__global__ void __launch_bounds__(256) k_apply_row(BasisDev B, HamArgs<S> H, KArgs K) {
  static_assert(G == 1 || (NV == 1 && 32 % G == 0), "lanes per row: G divides 32, one vector");
  constexpr int W = NV * (C ? 2 : 1);
  constexpr int U = G == 1 ? 4 : 8;   // with lanes, one round covers up to 8 G sites
  const int n = B.n;
  const CT full = (n >= (int)(8 * sizeof(CT))) ? ~(CT)0 : (((CT)1 << n) - 1);
  const S *__restrict__ xp = (const S *)K.x;
  double q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  const RT dim = (RT)B.dim;
  const int lane = (int)threadIdx.x & (G - 1);
  const RT rpb = (RT)(blockDim.x / G);
  const RT stride = (RT)gridDim.x * rpb;
  for (RT base = (RT)blockIdx.x * rpb; base < dim; base += stride) {
    const RT mine = base + (RT)(threadIdx.x / G);
    const bool active = mine < dim;       // the same for the G lanes of a row
    if constexpr (G == 1) {
      if (!active) break;
    }
    const RT row = active ? mine : (RT)0;
    const CT code = unrank_fib<LAY, CT, RT>(B, row);
    CT allowed = full;
    if constexpr (LAY != EL_LAYOUT_FULL) {
      CT occ = (code << 1) | (code >> 1);
      if constexpr (LAY == EL_LAYOUT_RING) occ |= ((code >> (n - 1)) & 1) | ((code & 1) << (n - 1));
      allowed = code | (~occ & full);
    }
    const bool top = (LAY == EL_LAYOUT_RING) && ((code >> (n - 1)) & 1);
    S h[W];
#pragma unroll
    for (int i = 0; i < W; ++i) h[i] = S(0);
    S dsum = S(0);
    for (int j0 = 0; j0 * G < n; j0 += U) {
      S xv[U][W];
      S ar[U], ai[U];
      bool ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = (j0 + u) * G + lane;
        ok[u] = false;
        ar[u] = S(0);
        ai[u] = S(0);
        if (k < n) {
          const bool set = (code >> k) & 1;
          if (set) dsum += H.delta[k];
          ar[u] = H.up_re[k];
          if constexpr (C) ai[u] = set ? H.up_im[k] : -H.up_im[k];
          ok[u] = ((allowed >> k) & 1) && (ar[u] != S(0) || ai[u] != S(0));
          if (ok[u]) {
            RT tg;
            if constexpr (LAY == EL_LAYOUT_FULL) {
              tg = row ^ ((RT)1 << k);
            } else if constexpr (LAY == EL_LAYOUT_CHAIN) {
              const RT w = (RT)B.fib[k + 2];
              tg = set ? row - w : row + w;
            } else {
              if (k == n - 1) {
                tg = ring_rank_t<CT, RT>(B, code ^ ((CT)1 << k), n);
              } else {
                const RT w = (RT)(top ? B.fib[k + 1] : B.fib[k + 2]);
                tg = set ? row - w : row + w;
              }
            }
            ld_row<S, W>(xp + (size_t)tg * W, xv[u]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        if constexpr (C) {
          if (H.real_amp) {   // uniform: a real drive needs two FMAs per complex entry
#pragma unroll
            for (int v = 0; v < 2 * NV; ++v) h[v] += ar[u] * xv[u][v];
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              h[2 * v] += ar[u] * xv[u][2 * v] - ai[u] * xv[u][2 * v + 1];
              h[2 * v + 1] += ar[u] * xv[u][2 * v + 1] + ai[u] * xv[u][2 * v];
            }
          }
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) h[v] += ar[u] * xv[u][v];
        }
      }
    }
    if constexpr (G > 1) {
#pragma unroll
      for (int off = G / 2; off > 0; off >>= 1) {
#pragma unroll
        for (int i = 0; i < W; ++i) h[i] += __shfl_xor_sync(0xffffffffu, h[i], off);
        dsum += __shfl_xor_sync(0xffffffffu, dsum, off);
      }
      if (lane != 0 || !active) continue;
    }
    S xr[W];
    ld_row<S, W>(xp + (size_t)row * W, xr);
    if (!K.skip_diag) {
      dsum += H.diagV[row];
#pragma unroll
      for (int i = 0; i < W; ++i) h[i] += dsum * xr[i];
    }
    S yv[W];
    const S a = (S)K.a, b = (S)K.b;
#pragma unroll
    for (int i = 0; i < W; ++i) yv[i] = a * h[i] + b * xr[i];
    if (K.z) {
      S zv[W];
      ld_row<S, W>((const S *)K.z + (size_t)row * W, zv);
      const S c = (S)K.c;
#pragma unroll
      for (int i = 0; i < W; ++i) yv[i] += c * zv[i];
    }
    if (K.acc) {
      S av[W];
      S *ap = (S *)K.acc + (size_t)row * W;
      ld_row<S, W>(ap, av);
      const S wr = (S)K.w_re, wi = (S)K.w_im;
      if constexpr (C) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          av[2 * v] += wr * yv[2 * v] - wi * yv[2 * v + 1];
          av[2 * v + 1] += wr * yv[2 * v + 1] + wi * yv[2 * v];
        }
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) av[v] += wr * yv[v];
      }
      st_row<S, W>(ap, av);
    }
    if (K.y) st_row<S, W>((S *)K.y + (size_t)row * W, yv);
    if constexpr (WANT) {
      if constexpr (C) {
        const double xre = xr[0], xim = xr[1], yre = yv[0], yim = yv[1];
        q0 += xre * xre + xim * xim;
        q1 += xre * yre + xim * yim;
        q2 += xre * yim - xim * yre;
        q3 += yre * yre + yim * yim;
      } else {
        const double xd = xr[0], yd = yv[0];
        q0 += xd * xd;
        q1 += xd * yd;
        q3 += yd * yd;
        if (K.probe) q2 += yd * (double)((const S *)K.probe)[row];
      }
    }
  }
  if constexpr (WANT) reduce4(K, q0, q1, q2, q3);
}

// ------------------------------------------- chain tile kernel (CHAIN layout)
// Rows of a nearest-neighbour chain sector that share the code bits >= L form
// one contiguous block of F(L+2) rows (F(L+1) when bit L is set), ordered by
// the low L bits exactly like the L-site chain itself.  A CTA takes one such
// block (a tile) at a time:
//   - flips of low bits k < L stay inside the tile: the tile of x is staged
//     in shared memory and the partner is row +- F(k+2) of the same tile;
//   - a flip of a high bit k >= L moves the whole tile by +- F(k+2) rows (the
//     low part is unchanged), and whether it is allowed depends only on the
//     tile's prefix (for k = L and bit L clear: on the tile's first F(L+1)
//     rows), so it is a contiguous, coalesced read of x with one amplitude
//     for the tile.
// Low codes and their detuning sums are tabulated once per CTA in shared
// memory.  Same fused epilogue as the row kernel.

// Streaming (evict-first) row access for vectors that are touched once per
// launch (y, z, acc), so that L2 keeps x, whose rows are re-read as flip
// partners by other tiles.
template <typename S, int W>
__device__ __forceinline__ void ld_row_cs(const S *p, S (&v)[W]) {
  constexpr int BYTES = W * (int)sizeof(S);
  if constexpr (BYTES % 16 == 0) {
    union { uint4 u[BYTES / 16]; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) t.u[i] = __ldcs(reinterpret_cast<const uint4 *>(p) + i);
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = t.s[i];
  } else if constexpr (BYTES == 8) {
    union { uint2 u; S s[W]; } t;
    t.u = __ldcs(reinterpret_cast<const uint2 *>(p));
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = t.s[i];
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = __ldcs(p + i);
  }
}

template <typename S, int W>
__device__ __forceinline__ void st_row_cs(S *p, const S (&v)[W]) {
  constexpr int BYTES = W * (int)sizeof(S);
  if constexpr (BYTES % 16 == 0) {
    union { uint4 u[BYTES / 16]; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < W; ++i) t.s[i] = v[i];
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) __stcs(reinterpret_cast<uint4 *>(p) + i, t.u[i]);
  } else if constexpr (BYTES == 8) {
    union { uint2 u; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < W; ++i) t.s[i] = v[i];
    __stcs(reinterpret_cast<uint2 *>(p), t.u);
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) __stcs(p + i, v[i]);
  }
}

// Shared tile of x: rows of more than 16 bytes are stored chunk-major
// ([16-byte chunk][row]) so that the 16-byte loads of a warp's 32 rows hit
// 32 consecutive chunks instead of a 4- or 8-way bank conflict.
template <typename S, int W>
__device__ __forceinline__ void tile_ld(const S *xt, int ts, int row, S (&v)[W]) {
  constexpr int BYTES = W * (int)sizeof(S);
  if constexpr (BYTES > 16 && BYTES % 16 == 0) {
    union { uint4 u[BYTES / 16]; S s[W]; } t;
#pragma unroll
    for (int i = 0; i < BYTES / 16; ++i) t.u[i] = reinterpret_cast<const uint4 *>(xt)[(size_t)i * ts + row];
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = t.s[i];
  } else {
    ld_row<S, W>(xt + (size_t)row * W, v);
  }
}

struct TileFlip {
  int64_t off;   // row offset of the partner
  int32_t len;   // rows [0, len) of the tile have this flip
  int32_t k;     // bit
};

// RA: the amplitudes are real (real Omega) although the vectors are
// complex: two FMAs per complex entry instead of four.
template <typename S, bool C, int NV, bool RA = false>
__device__ __forceinline__ void acc_flip(S (&h)[NV * (C ? 2 : 1)], S are, S aim,
                                         const S (&xv)[NV * (C ? 2 : 1)]) {
  if constexpr (C && RA) {
#pragma unroll
    for (int v = 0; v < 2 * NV; ++v) h[v] += are * xv[v];
  } else if constexpr (C) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      h[2 * v] += are * xv[2 * v] - aim * xv[2 * v + 1];
      h[2 * v + 1] += are * xv[2 * v + 1] + aim * xv[2 * v];
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) h[v] += are * xv[v];
  }
}

template <typename S, bool C, int NV, bool WANT, bool RA>
__global__ void __launch_bounds__(256) k_apply_chain_tile(BasisDev B, HamArgs<S> H, KArgs K, int L,
                                                          int64_t ntiles) {
  constexpr int W = NV * (C ? 2 : 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = B.n;
  const int TS = (int)B.fib[L + 2];                       // rows of a full tile
  // [TS][W] tile of x, then the S-typed table, then the 4-byte table, so
  // every array starts on a boundary of its element size
  S *xt = reinterpret_cast<S *>(smem_raw);
  S *ld = xt + (size_t)TS * W;                            // low detuning sums
  uint32_t *lc = reinterpret_cast<uint32_t *>(ld + TS);   // low codes
  __shared__ TileFlip hf[EL_MAX_SITES];
  __shared__ S hf_re[EL_MAX_SITES], hf_im[EL_MAX_SITES];
  __shared__ int nhf;
  __shared__ int s_w[EL_MAX_SITES];            // F(k+2) of the low bits
  __shared__ S s_are[EL_MAX_SITES], s_aim[EL_MAX_SITES];
  __shared__ uint32_t s_amp;                    // low bits with a nonzero amplitude
  __shared__ int64_t t_base;
  __shared__ int t_size;
  __shared__ int t_bl;       // bit L of the tile's prefix
  __shared__ S t_delta;      // detuning sum of the prefix bits
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    s_w[k] = (int)B.fib[k + 2];
    s_are[k] = H.up_re[k];
    s_aim[k] = C ? H.up_im[k] : S(0);
  }
  if (threadIdx.x == 0) {
    uint32_t am = 0;
    for (int k = 0; k < L; ++k)
      if (H.up_re[k] != S(0) || (C && H.up_im[k] != S(0))) am |= 1u << k;
    s_amp = am;
  }
  // low codes of the L-site chain in ascending order, and their detunings
  for (int i = threadIdx.x; i < TS; i += blockDim.x) {
    uint32_t c = 0;
    int64_t r = i;
    for (int k = L - 1; k >= 0; --k) {
      const int64_t w = (int64_t)B.fib[k + 2];
      if (r >= w) { c |= 1u << k; r -= w; }
    }
    lc[i] = c;
    S d = S(0);
    for (int k = 0; k < L; ++k)
      if ((c >> k) & 1u) d += H.delta[k];
    ld[i] = d;
  }
  const S *__restrict__ xp = (const S *)K.x;
  double q0 = 0, q1 = 0, q2 = 0, q3 = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    __syncthreads();   // tables ready; previous tile done with xt / hf
    if (threadIdx.x == 0) {
      // prefix of tile t: the (n-L)-site chain code of rank t
      uint64_t p = 0;
      int64_t r = t;
      for (int j = n - L - 1; j >= 0; --j) {
        const int64_t w = (int64_t)B.fib[j + 2];
        if (r >= w) { p |= 1ULL << j; r -= w; }
      }
      int64_t base = 0;
      S dp = S(0);
      for (int j = 0; j < n - L; ++j)
        if ((p >> j) & 1ULL) { base += (int64_t)B.fib[L + j + 2]; dp += H.delta[L + j]; }
      const int bl = (int)(p & 1ULL);
      const int size = bl ? (int)B.fib[L + 1] : TS;
      int cnt = 0;
      for (int j = 0; j < n - L; ++j) {
        const int k = L + j;
        const S are = H.up_re[k];
        const bool set = (p >> j) & 1ULL;
        const S aim = C ? (set ? H.up_im[k] : -H.up_im[k]) : S(0);
        if (are == S(0) && aim == S(0)) continue;
        const int64_t w = (int64_t)B.fib[k + 2];
        TileFlip f;
        f.k = k;
        if (set) {
          f.off = -w;
          f.len = size;
        } else {
          if (j + 1 < n - L && ((p >> (j + 1)) & 1ULL)) continue;
          if (j >= 1 && ((p >> (j - 1)) & 1ULL)) continue;
          f.off = w;
          f.len = (j == 0) ? (int)B.fib[L + 1] : size;   // k = L needs low bit L-1 clear
        }
        hf[cnt] = f;
        hf_re[cnt] = are;
        hf_im[cnt] = aim;
        ++cnt;
      }
      nhf = cnt;
      t_base = base;
      t_size = size;
      t_bl = bl;
      t_delta = dp;
    }
    __syncthreads();
    const int64_t base = t_base;
    const int size = t_size;
    const int bl = t_bl;
    const int nh = nhf;
    // stage the tile of x (16-byte chunks when the row segment allows it)
    {
      constexpr int RB = W * (int)sizeof(S);
      if constexpr (RB > 16 && RB % 16 == 0) {
        constexpr int NC = RB / 16;
        const uint4 *src = reinterpret_cast<const uint4 *>(xp + (size_t)base * W);
        uint4 *dst = reinterpret_cast<uint4 *>(xt);
        const int nch = size * NC;
        for (int g = threadIdx.x; g < nch; g += blockDim.x) dst[(size_t)(g % NC) * TS + g / NC] = src[g];
      } else if constexpr (RB % 16 == 0) {
        const uint4 *src = reinterpret_cast<const uint4 *>(xp + (size_t)base * W);
        uint4 *dst = reinterpret_cast<uint4 *>(xt);
        const int nch = size * (RB / 16);
        for (int i = threadIdx.x; i < nch; i += blockDim.x) dst[i] = src[i];
      } else {
        const S *src = xp + (size_t)base * W;
        for (int i = threadIdx.x; i < size * W; i += blockDim.x) xt[i] = src[i];
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
      const uint32_t c = lc[i];
      S h[W];
#pragma unroll
      for (int q = 0; q < W; ++q) h[q] = S(0);
      // low flips, partners in shared memory: the flippable bits are the set
      // ones and those with both neighbours empty (bit L above the top low
      // bit is the tile's bl); walk the set bits of that mask
      {
        const uint32_t lowmask = (L >= 32) ? ~0u : ((1u << L) - 1u);
        const uint32_t occ = (c << 1) | (c >> 1) | ((uint32_t)bl << (L - 1));
        uint32_t m = (c | (~occ & lowmask)) & s_amp;
        while (m) {
          const int k = __ffs(m) - 1;
          m &= m - 1;
          const bool set = (c >> k) & 1u;
          const int w = s_w[k];
          const int pi = set ? i - w : i + w;
          const S are = s_are[k];
          const S aim = set ? s_aim[k] : -s_aim[k];
          S xv[W];
          tile_ld<S, W>(xt, TS, pi, xv);
          acc_flip<S, C, NV, RA>(h, are, aim, xv);
        }
      }
      // high flips: contiguous partner rows in global memory, two in flight
      for (int f = 0; f < nh; f += 2) {
        S xa[W], xb[W];
        const bool oa = i < hf[f].len;
        const bool ob = (f + 1 < nh) && (i < hf[f + 1].len);
        if (oa) ld_row<S, W>(xp + (size_t)(base + i + hf[f].off) * W, xa);
        if (ob) ld_row<S, W>(xp + (size_t)(base + i + hf[f + 1].off) * W, xb);
        if (oa) acc_flip<S, C, NV, RA>(h, hf_re[f], hf_im[f], xa);
        if (ob) acc_flip<S, C, NV, RA>(h, hf_re[f + 1], hf_im[f + 1], xb);
      }
      const int64_t row = base + i;
      S xr[W];
      tile_ld<S, W>(xt, TS, i, xr);
      if (!K.skip_diag) {
        const S dsum = H.diagV[row] + t_delta + ld[i];
#pragma unroll
        for (int q = 0; q < W; ++q) h[q] += dsum * xr[q];
      }
      S yv[W];
      const S a = (S)K.a, b = (S)K.b;
#pragma unroll
      for (int q = 0; q < W; ++q) yv[q] = a * h[q] + b * xr[q];
      if (K.z) {
        S zv[W];
        ld_row_cs<S, W>((const S *)K.z + (size_t)row * W, zv);
        const S cc = (S)K.c;
#pragma unroll
        for (int q = 0; q < W; ++q) yv[q] += cc * zv[q];
      }
      if (K.acc) {
        S av[W];
        S *ap = (S *)K.acc + (size_t)row * W;
        ld_row_cs<S, W>(ap, av);
        const S wr = (S)K.w_re, wi = (S)K.w_im;
        if constexpr (C) {
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            av[2 * v] += wr * yv[2 * v] - wi * yv[2 * v + 1];
            av[2 * v + 1] += wr * yv[2 * v + 1] + wi * yv[2 * v];
          }
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) av[v] += wr * yv[v];
        }
        st_row_cs<S, W>(ap, av);
      }
      if (K.y) st_row_cs<S, W>((S *)K.y + (size_t)row * W, yv);
      if constexpr (WANT) {
        if constexpr (C) {
          const double xre = xr[0], xim = xr[1], yre = yv[0], yim = yv[1];
          q0 += xre * xre + xim * xim;
          q1 += xre * yre + xim * yim;
          q2 += xre * yim - xim * yre;
          q3 += yre * yre + yim * yim;
        } else {
          const double xd = xr[0], yd = yv[0];
          q0 += xd * xd;
          q1 += xd * yd;
          q3 += yd * yd;
          if (K.probe) q2 += yd * (double)((const S *)K.probe)[row];
        }
      }
    }
  }
  if constexpr (WANT) reduce4(K, q0, q1, q2, q3);
}

template <typename S>
HamArgs<S> ham_args(const el_ham *h, const S *diagV) {
  HamArgs<S> A;
  memset(&A, 0, sizeof A);
  A.diagV = diagV;
  A.px = h->d_px;
  A.npx = (int)h->px.size();
  A.lossy = h->lossy ? 1 : 0;
  A.real_amp = h->drive_complex ? 0 : 1;
  for (int k = 0; k < h->n; ++k) {
    A.delta[k] = (S)h->delta[k];
    A.up_re[k] = (S)(0.5 * h->om_re[k]);
    A.up_im[k] = (S)(0.5 * h->om_im[k]);
    A.loss[k] = (S)h->loss[k];
  }
  return A;
}

int ilog2(int64_t v) {
  int l = 0;
  while ((1LL << l) < v) ++l;
  return l;
}

// ---------------------------------------------------------------- diagonal

__global__ void k_diag_v(BasisDev B, int n, const double *__restrict__ Vg,
                         double *out64, float *out32) {
  extern __shared__ double Vs[];
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) Vs[i] = Vg[i];
  __syncthreads();
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.dim;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t code = el::unrank_row(B, r);
    double s = 0.0;
    uint64_t m = code;
    while (m) {
      const int k = __ffsll((long long)m) - 1;
      m &= m - 1;
      uint64_t m2 = m;
      while (m2) {
        const int k2 = __ffsll((long long)m2) - 1;
        m2 &= m2 - 1;
        s += Vs[k * n + k2];
      }
    }
    if (out64) out64[r] = s;
    if (out32) out32[r] = (float)s;
  }
}

template <typename S>
__global__ void k_full_diag(BasisDev B, HamArgs<double> H, S *out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.dim;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t code = el::unrank_row(B, r);
    double d = H.diagV[r];
    for (int k = 0; k < B.n; ++k) if ((code >> k) & 1ULL) d += H.delta[k];
    out[r] = (S)d;
  }
}

// Gershgorin interval: min_r (d_r - R_r), max_r (d_r + R_r).
__global__ void k_gershgorin(BasisDev B, HamArgs<double> H, double *partials,
                             unsigned int *counter, double *out) {
  __shared__ double lo_s[256], hi_s[256], nm_s[256];
  __shared__ bool last;
  double lo = 1e300, hi = -1e300, nm = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.dim;
       r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t code = el::unrank_row(B, r);
    double d = H.diagV[r], R = 0.0, di = 0.0;
    for (int k = 0; k < B.n; ++k) {
      if ((code >> k) & 1ULL) { d += H.delta[k]; di += H.loss[k]; }
      const double amp = sqrt(H.up_re[k] * H.up_re[k] + H.up_im[k] * H.up_im[k]);
      if (amp == 0.0) continue;
      if (el::flip_target(B, code, r, k) >= 0) R += amp;
    }
    for (int p = 0; p < H.npx; ++p) {
      const ExPair e = H.px[p];
      double pre, pim;
      exchange_amp(e, (code >> e.bi) & 1ULL, (code >> e.bj) & 1ULL, pre, pim);
      if (pre == 0.0 && pim == 0.0) continue;
      if (el::rank_any(B, code ^ ((1ULL << e.bi) | (1ULL << e.bj))) >= 0) R += sqrt(pre * pre + pim * pim);
    }
    lo = fmin(lo, d - R);
    hi = fmax(hi, d + R);
    nm = fmax(nm, sqrt(d * d + di * di) + R);
  }
  lo_s[threadIdx.x] = lo;
  hi_s[threadIdx.x] = hi;
  nm_s[threadIdx.x] = nm;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      lo_s[threadIdx.x] = fmin(lo_s[threadIdx.x], lo_s[threadIdx.x + s]);
      hi_s[threadIdx.x] = fmax(hi_s[threadIdx.x], hi_s[threadIdx.x + s]);
      nm_s[threadIdx.x] = fmax(nm_s[threadIdx.x], nm_s[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = lo_s[0];
    partials[3 * blockIdx.x + 1] = hi_s[0];
    partials[3 * blockIdx.x + 2] = nm_s[0];
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double a = 1e300, b = -1e300, c = 0.0;
    for (unsigned i = 0; i < gridDim.x; ++i) {
      a = fmin(a, __ldcg(&partials[3 * i]));
      b = fmax(b, __ldcg(&partials[3 * i + 1]));
      c = fmax(c, __ldcg(&partials[3 * i + 2]));
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
    *counter = 0u;
  }
}

// ------------------------------------------------------------ BLAS-like ops

template <typename S, bool C>
__global__ void k_axpby(int64_t len, double a_re, double a_im, const S *x,
                        double b_re, double b_im, S *y, double *partials,
                        unsigned int *counter, double *norm2) {
  __shared__ double red[256];
  __shared__ bool last;
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (C) {
      const double xr = x ? (double)x[2 * i] : 0.0, xi = x ? (double)x[2 * i + 1] : 0.0;
      // beta == 0 must not read y: workspace may hold stale bits (NaN)
      const bool ry = (b_re != 0.0 || b_im != 0.0);
      const double yr = ry ? (double)y[2 * i] : 0.0, yi = ry ? (double)y[2 * i + 1] : 0.0;
      const double r = a_re * xr - a_im * xi + b_re * yr - b_im * yi;
      const double im = a_re * xi + a_im * xr + b_re * yi + b_im * yr;
      const S rs = (S)r, is = (S)im;
      y[2 * i] = rs;
      y[2 * i + 1] = is;
      acc += (double)rs * (double)rs + (double)is * (double)is;
    } else {
      const double xv = x ? (double)x[i] : 0.0;
      const double yv = (b_re != 0.0) ? (double)y[i] : 0.0;
      const S r = (S)(a_re * xv + b_re * yv);
      y[i] = r;
      acc += (double)r * (double)r;
    }
  }
  if (!norm2) return;
  red[threadIdx.x] = acc;
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
    *norm2 = s;
    *counter = 0u;
  }
}

// partials[bx][j] (re, im) of <V_j, w> over the block's rows.
constexpr int GJ = 16;
// dots_j = <V_j, w> for a group of GJ columns per blockIdx.y: every thread
// accumulates its rows in FP64 registers, warps reduce by shuffles (fixed
// tree), then the block's warps in order; per-block partials are summed by
// k_sum_partials in block order (deterministic).
template <typename S, bool C>
__global__ void __launch_bounds__(256) k_gemv_t(int64_t len, int k, const S *V, int64_t ld, const S *w,
                                                double *partials) {
  __shared__ double red[8][2 * GJ];
  const int j0 = blockIdx.y * GJ;
  const int nq = min(GJ, k - j0);
  double accr[GJ], acci[GJ];
#pragma unroll
  for (int q = 0; q < GJ; ++q) { accr[q] = 0.0; acci[q] = 0.0; }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (C) {
      const double wr = w[2 * i], wi = w[2 * i + 1];
#pragma unroll
      for (int q = 0; q < GJ; ++q) {
        if (q < nq) {
          const S *vj = V + (size_t)(j0 + q) * ld * 2;
          const double vr = vj[2 * i], vi = vj[2 * i + 1];
          accr[q] += vr * wr + vi * wi;
          acci[q] += vr * wi - vi * wr;
        }
      }
    } else {
      const double wv = w[i];
#pragma unroll
      for (int q = 0; q < GJ; ++q)
        if (q < nq) accr[q] += (double)V[(size_t)(j0 + q) * ld + i] * wv;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < GJ; ++q) {
    double a = accr[q], b = acci[q];
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      if (C) b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) { red[warp][2 * q] = a; red[warp][2 * q + 1] = b; }
  }
  __syncthreads();
  if (threadIdx.x < 2 * GJ) {
    const int q = threadIdx.x >> 1;
    double sum = 0.0;
    for (int wp = 0; wp < (int)(blockDim.x >> 5); ++wp) sum += red[wp][threadIdx.x];
    if (q < nq) partials[((size_t)blockIdx.x * k + j0 + q) * 2 + (threadIdx.x & 1)] = sum;
  }
}

__global__ void k_sum_partials(int nparts, int k, const double *partials, double *out) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < 2 * k; o += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += partials[(size_t)b * 2 * k + o];
    out[o] = s;
  }
}

// w -= sum_j coef_j V_j  (sub = true) or w = sum_j coef_j V_j (sub = false).
// The coefficients are staged in shared memory (k <= GN_MAX, else read from
// global memory); four partial sums per row keep four column loads in flight.
constexpr int GN_MAX = 1024;
template <typename S, bool C>
__global__ void __launch_bounds__(256) k_gemv_n(int64_t len, int k, const S *V, int64_t ld,
                                                const double *coef, S *w, bool sub) {
  __shared__ double cs[2 * GN_MAX];
  const bool staged = k <= GN_MAX;
  if (staged)
    for (int t = threadIdx.x; t < 2 * k; t += blockDim.x) cs[t] = coef[t];
  __syncthreads();
  const double *cf = staged ? cs : coef;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    double sr[4] = {0.0, 0.0, 0.0, 0.0}, si[4] = {0.0, 0.0, 0.0, 0.0};
    int j = 0;
    for (; j + 4 <= k; j += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double cr = cf[2 * (j + u)], ci = cf[2 * (j + u) + 1];
        if constexpr (C) {
          const S *vj = V + (size_t)(j + u) * ld * 2;
          const double vr = vj[2 * i], vi = vj[2 * i + 1];
          sr[u] += cr * vr - ci * vi;
          si[u] += cr * vi + ci * vr;
        } else {
          sr[u] += cr * (double)V[(size_t)(j + u) * ld + i];
        }
      }
    }
    for (; j < k; ++j) {
      const double cr = cf[2 * j], ci = cf[2 * j + 1];
      if constexpr (C) {
        const S *vj = V + (size_t)j * ld * 2;
        const double vr = vj[2 * i], vi = vj[2 * i + 1];
        sr[0] += cr * vr - ci * vi;
        si[0] += cr * vi + ci * vr;
      } else {
        sr[0] += cr * (double)V[(size_t)j * ld + i];
      }
    }
    const double tr = (sr[0] + sr[1]) + (sr[2] + sr[3]);
    const double ti = (si[0] + si[1]) + (si[2] + si[3]);
    if constexpr (C) {
      if (sub) { w[2 * i] = (S)((double)w[2 * i] - tr); w[2 * i + 1] = (S)((double)w[2 * i + 1] - ti); }
      else { w[2 * i] = (S)tr; w[2 * i + 1] = (S)ti; }
    } else {
      w[i] = sub ? (S)((double)w[i] - tr) : (S)tr;
    }
  }
}

// Gaussian start vector from a counter-based hash (Box-Muller).
template <typename S>
__global__ void k_fill_gauss(int64_t len, uint64_t seed, S *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h1 = el::counter_hash(seed, 0x5151, (uint64_t)i);
    const uint64_t h2 = el::counter_hash(seed, 0xA7A7, (uint64_t)i);
    const double u1 = ((h1 >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    out[i] = (S)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
  }
}

// Probe block [dim][nvec]; probes v >= nvalid are zero vectors.
template <typename S>
__global__ void k_fill_rademacher(int64_t dim, int nvec, uint64_t seed,
                                  int64_t probe0, int nvalid, S *out) {
  const int64_t total = dim * nvec;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / nvec, v = t % nvec;
    out[t] = v < nvalid ? (S)el::rademacher(seed, (uint64_t)(probe0 + v), (uint64_t)r) : (S)0;
  }
}

// probes_dev is [nvec][dim] int8; out is [dim][nvec]
template <typename S>
__global__ void k_probe_copy(int64_t dim, int nvec, const int8_t *probes, S *out) {
  const int64_t total = dim * nvec;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / nvec, v = t % nvec;
    out[t] = (S)probes[v * dim + r];
  }
}

template <typename S>
__global__ void k_scale(int64_t len, const double *scale, int invert_sqrt, S *x) {
  const double s = invert_sqrt ? 1.0 / sqrt(*scale) : *scale;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (S)((double)x[i] * s);
}

// out[k] = sum |psi_r|^2 bit_k(r) (k < n), out[n] = sum |psi_r|^2
template <typename S, bool C>
__global__ void k_observables(BasisDev B, const S *psi, double *partials,
                              unsigned int *counter, double *out) {
  __shared__ double ws[8][EL_MAX_SITES + 1];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = B.n;
  for (int k = threadIdx.x; k < 8 * (EL_MAX_SITES + 1); k += blockDim.x) (&ws[0][0])[k] = 0.0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < B.dim; base += stride) {
    const int64_t r = base + threadIdx.x;
    double p = 0.0;
    uint64_t code = 0;
    if (r < B.dim) {
      code = el::unrank_row(B, r);
      if constexpr (C) { const double a = psi[2 * r], b = psi[2 * r + 1]; p = a * a + b * b; }
      else { const double a = psi[r]; p = a * a; }
    }
    for (int k = 0; k <= n; ++k) {
      double v = (k == n) ? p : (((code >> k) & 1ULL) ? p : 0.0);
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) ws[warp][k] += v;
    }
  }
  __syncthreads();
  const int nout = n + 1;
  for (int k = threadIdx.x; k < nout; k += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += ws[w][k];
    partials[(size_t)blockIdx.x * nout + k] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = threadIdx.x; k < nout; k += blockDim.x) {
    double s = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(&partials[(size_t)b * nout + k]);
    out[k] = s;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

bool is_complex(int dtype) { return dtype == EL_C64 || dtype == EL_C128; }

}  // namespace

namespace {

// The row kernel serves FULL/CHAIN/RING bases with 1..8 vectors per row
// (dot products only for one vector) when every vector pointer is aligned for
// its row-segment loads.
bool row_kernel_ok(const el_ham *h, const ApplyArgs &A) {
  if (!h->px.empty() || h->lossy) return false;   // exchange channels or loss: generic kernel
  const int lay = h->basis->layout;
  if (lay != EL_LAYOUT_FULL && lay != EL_LAYOUT_CHAIN && lay != EL_LAYOUT_RING) return false;
  if (A.nvec > 8) return false;
  if (A.dots && A.nvec != 1) return false;
  const size_t row_bytes = (size_t)A.nvec * el::dtype_size(A.dtype);
  const size_t align = row_bytes >= 16 ? 16 : row_bytes;
  for (const void *p : {A.x, (const void *)A.z, (const void *)A.y, (const void *)A.acc, A.probe})
    if (p && ((uintptr_t)p % align) != 0) return false;
  return true;
}

template <typename S, bool C, int NV, bool WANT, typename CT, typename RT, int G>
void launch_row_ct(el_ctx *ctx, int lay, int grid, const BasisDev &B, const HamArgs<S> &H, const KArgs &K) {
  if (lay == EL_LAYOUT_FULL)
    k_apply_row<S, C, NV, EL_LAYOUT_FULL, WANT, CT, RT, G><<<grid, 256, 0, ctx->stream>>>(B, H, K);
  else if (lay == EL_LAYOUT_CHAIN)
    k_apply_row<S, C, NV, EL_LAYOUT_CHAIN, WANT, CT, RT, G><<<grid, 256, 0, ctx->stream>>>(B, H, K);
  else
    k_apply_row<S, C, NV, EL_LAYOUT_RING, WANT, CT, RT, G><<<grid, 256, 0, ctx->stream>>>(B, H, K);
}

// Rows below which a single-vector row kernel gives each row ROW_LANES lanes:
// one thread per row would occupy fewer than two CTAs of 256 per SM.
constexpr int64_t LANE_ROWS = 148 * 512;
constexpr int ROW_LANES = 4;

bool row_lanes(const BasisDev &B, int nvec) {
  return nvec == 1 && B.n <= 32 && B.dim < LANE_ROWS;
}

template <typename S, bool C, int NV, bool WANT>
void launch_row_lay(el_ctx *ctx, int lay, int grid, const BasisDev &B, const HamArgs<S> &H, const KArgs &K) {
  if constexpr (NV == 1) {
    if (row_lanes(B, NV)) {
      launch_row_ct<S, C, NV, WANT, uint32_t, int32_t, ROW_LANES>(ctx, lay, grid, B, H, K);
      return;
    }
  }
  if (B.n <= 32 && B.dim < ((int64_t)1 << 31))
    launch_row_ct<S, C, NV, WANT, uint32_t, int32_t, 1>(ctx, lay, grid, B, H, K);
  else
    launch_row_ct<S, C, NV, WANT, uint64_t, int64_t, 1>(ctx, lay, grid, B, H, K);
}

template <typename S, bool C>
void launch_row_t(el_ctx *ctx, int lay, int nvec, bool want, int grid, const BasisDev &B,
                  const HamArgs<S> &H, const KArgs &K) {
  if (want) { launch_row_lay<S, C, 1, true>(ctx, lay, grid, B, H, K); return; }
  switch (nvec) {
    case 1: launch_row_lay<S, C, 1, false>(ctx, lay, grid, B, H, K); break;
    case 2: launch_row_lay<S, C, 2, false>(ctx, lay, grid, B, H, K); break;
    case 4: launch_row_lay<S, C, 4, false>(ctx, lay, grid, B, H, K); break;
    default: launch_row_lay<S, C, 8, false>(ctx, lay, grid, B, H, K); break;
  }
}

// Tile bits L for the chain tile kernel: the largest L whose tile (rows x
// row bytes, plus 4 + sizeof(S) bytes of tables per row) stays within 40 KB,
// leaving at least 4 prefix bits; 0 if the chain is too short to tile.
int chain_tile_bits(int n, int row_bytes, int scalar_bytes) {
  uint64_t f[70];
  f[0] = 0; f[1] = 1;
  for (int i = 2; i < 70; ++i) f[i] = f[i - 1] + f[i - 2];
  int best = 0;
  for (int L = 4; L + 4 <= n && L + 2 < 70; ++L)
    if (f[L + 2] * (uint64_t)(row_bytes + 4 + scalar_bytes) <= 40960) best = L;
  return best;
}

template <typename S, bool C, int NV, bool WANT, bool RA>
int launch_chain_tile_t(el_ctx *ctx, int L, int64_t ntiles, const BasisDev &B, const HamArgs<S> &H,
                        const KArgs &K) {
  constexpr int W = NV * (C ? 2 : 1);
  const size_t ts = (size_t)B.fib[L + 2];
  const size_t smem = ts * W * sizeof(S) + ts * 4 + ts * sizeof(S) + 16;
  cudaFuncSetAttribute(k_apply_chain_tile<S, C, NV, WANT, RA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)sms * 8);
  k_apply_chain_tile<S, C, NV, WANT, RA><<<grid, 256, smem, ctx->stream>>>(B, H, K, L, ntiles);
  return EL_OK;
}

template <typename S, bool C, bool RA>
int launch_chain_tile_r(el_ctx *ctx, int nvec, bool want, int L, int64_t ntiles, const BasisDev &B,
                        const HamArgs<S> &H, const KArgs &K) {
  if (want) return launch_chain_tile_t<S, C, 1, true, RA>(ctx, L, ntiles, B, H, K);
  switch (nvec) {
    case 1: return launch_chain_tile_t<S, C, 1, false, RA>(ctx, L, ntiles, B, H, K);
    case 2: return launch_chain_tile_t<S, C, 2, false, RA>(ctx, L, ntiles, B, H, K);
    case 4: return launch_chain_tile_t<S, C, 4, false, RA>(ctx, L, ntiles, B, H, K);
    default: return launch_chain_tile_t<S, C, 8, false, RA>(ctx, L, ntiles, B, H, K);
  }
}

// complex vectors with a real drive take the real-amplitude variant, except
// for eight complex64 vectors per row, where it needs 119 registers instead
// of 80 and loses the third CTA per SM
template <typename S, bool C>
int launch_chain_tile_v(el_ctx *ctx, int nvec, bool want, int L, int64_t ntiles, const BasisDev &B,
                        const HamArgs<S> &H, const KArgs &K, bool real_amp) {
  if (C && real_amp && (want || nvec <= 4 || sizeof(S) == 8))
    return launch_chain_tile_r<S, C, true>(ctx, nvec, want, L, ntiles, B, H, K);
  return launch_chain_tile_r<S, C, false>(ctx, nvec, want, L, ntiles, B, H, K);
}

int launch_apply_row(el_ctx *ctx, el_ham *h, const ApplyArgs &A, const BasisDev &B, KArgs K) {
  const int lay = h->basis->layout;
  const int64_t lanes = row_lanes(B, (int)A.nvec) ? ROW_LANES : 1;
  const int grid = el::grid_for(h->basis->dim * lanes, 256);
  const bool want = K.want != 0;
  if (want) {
    K.nvec = 1;
    K.lognv = 0;
    // partial sums for the row grid or the tile grid (at most 8 CTAs per SM)
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    int rc = el::ensure_partials(ctx, (size_t)std::max(grid, 8 * sms) * 4);
    if (rc) return rc;
    K.partials = ctx->d_partials;
  }
  if (lay == EL_LAYOUT_CHAIN) {
    const int ss = (A.dtype == EL_F32 || A.dtype == EL_C64) ? 4 : 8;
    const int L = chain_tile_bits(h->n, (int)A.nvec * el::dtype_size(A.dtype), ss);
    if (L > 0) {
      const int64_t ntiles = (int64_t)B.fib[h->n - L + 2];
      switch (A.dtype) {
        case EL_F32: launch_chain_tile_v<float, false>(ctx, A.nvec, want, L, ntiles, B, ham_args<float>(h, h->d_diagV32), K, false); break;
        case EL_F64: launch_chain_tile_v<double, false>(ctx, A.nvec, want, L, ntiles, B, ham_args<double>(h, h->d_diagV64), K, false); break;
        case EL_C64: launch_chain_tile_v<float, true>(ctx, A.nvec, want, L, ntiles, B, ham_args<float>(h, h->d_diagV32), K, !h->drive_complex); break;
        case EL_C128: launch_chain_tile_v<double, true>(ctx, A.nvec, want, L, ntiles, B, ham_args<double>(h, h->d_diagV64), K, !h->drive_complex); break;
        default: return el::fail(ctx, EL_EINVAL, "unknown dtype %d", A.dtype);
      }
      EL_LAUNCH_CHECK(ctx);
      return EL_OK;
    }
  }
  switch (A.dtype) {
    case EL_F32: launch_row_t<float, false>(ctx, lay, A.nvec, want, grid, B, ham_args<float>(h, h->d_diagV32), K); break;
    case EL_F64: launch_row_t<double, false>(ctx, lay, A.nvec, want, grid, B, ham_args<double>(h, h->d_diagV64), K); break;
    case EL_C64: launch_row_t<float, true>(ctx, lay, A.nvec, want, grid, B, ham_args<float>(h, h->d_diagV32), K); break;
    case EL_C128: launch_row_t<double, true>(ctx, lay, A.nvec, want, grid, B, ham_args<double>(h, h->d_diagV64), K); break;
    default: return el::fail(ctx, EL_EINVAL, "unknown dtype %d", A.dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

}  // namespace

namespace el {

int launch_apply(el_ctx *ctx, el_ham *h, const ApplyArgs &A) {
  const int64_t nvec = A.nvec;
  if (nvec < 1 || nvec > 256 || (nvec & (nvec - 1)))
    return fail(ctx, EL_EINVAL, "nvec must be a power of two in [1, 256], got %lld", (long long)nvec);
  if (!is_complex(A.dtype) && (h->complex_drive))
    return fail(ctx, EL_EINVAL, "complex Omega, J or A needs a complex vector dtype");
  BasisDev B = basis_dev(h->basis);
  KArgs K;
  K.nvec = nvec;
  K.lognv = ilog2(nvec);
  K.x = A.x; K.z = A.z; K.y = A.y; K.acc = A.acc;
  K.a = A.a; K.b = A.b; K.c = A.c; K.w_re = A.w_re; K.w_im = A.w_im;
  K.dots = A.dots;
  K.want = A.dots ? (A.want_dots ? A.want_dots : 7) : 0;
  K.skip_diag = A.skip_diag;
  K.probe = A.probe;
  K.counter = ctx->d_counter;
  const int64_t total = h->basis->dim * nvec;
  const int grid = grid_for(total, 256);
  if (K.want) {
    int rc = ensure_partials(ctx, (size_t)grid * nvec * 4);
    if (rc) return rc;
  }
  K.partials = ctx->d_partials;
  const bool single = (A.dtype == EL_F32 || A.dtype == EL_C64);
  if (single) {
    int rc = ham_diag32(ctx, h);
    if (rc) return rc;
  }
  if (row_kernel_ok(h, A)) return launch_apply_row(ctx, h, A, B, K);
  if (!h->px.empty() && (B.layout == EL_LAYOUT_FULL || B.layout == EL_LAYOUT_TABLE) && B.n <= 32 &&
      B.dim < ((int64_t)1 << 31)) {
    const size_t sm = (size_t)B.n * B.n * (single ? sizeof(float) : sizeof(double)) * 2;
    switch (A.dtype) {
      case EL_F32: k_apply_hop<float, false><<<grid, 256, sm, ctx->stream>>>(B, ham_args<float>(h, h->d_diagV32), K, h->d_hop, h->d_pxA, h->npxA); break;
      case EL_F64: k_apply_hop<double, false><<<grid, 256, sm, ctx->stream>>>(B, ham_args<double>(h, h->d_diagV64), K, h->d_hop, h->d_pxA, h->npxA); break;
      case EL_C64: k_apply_hop<float, true><<<grid, 256, sm, ctx->stream>>>(B, ham_args<float>(h, h->d_diagV32), K, h->d_hop, h->d_pxA, h->npxA); break;
      case EL_C128: k_apply_hop<double, true><<<grid, 256, sm, ctx->stream>>>(B, ham_args<double>(h, h->d_diagV64), K, h->d_hop, h->d_pxA, h->npxA); break;
      default: return fail(ctx, EL_EINVAL, "unknown dtype %d", A.dtype);
    }
    EL_LAUNCH_CHECK(ctx);
    return EL_OK;
  }
  switch (A.dtype) {
    case EL_F32:
      k_apply<float, false><<<grid, 256, 0, ctx->stream>>>(B, ham_args<float>(h, h->d_diagV32), K);
      break;
    case EL_F64:
      k_apply<double, false><<<grid, 256, 0, ctx->stream>>>(B, ham_args<double>(h, h->d_diagV64), K);
      break;
    case EL_C64:
      k_apply<float, true><<<grid, 256, 0, ctx->stream>>>(B, ham_args<float>(h, h->d_diagV32), K);
      break;
    case EL_C128:
      k_apply<double, true><<<grid, 256, 0, ctx->stream>>>(B, ham_args<double>(h, h->d_diagV64), K);
      break;
    default:
      return fail(ctx, EL_EINVAL, "unknown dtype %d", A.dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_diag_v(el_ctx *ctx, el_ham *h) {
  BasisDev B = basis_dev(h->basis);
  const int n = h->n;
  double *d_V = nullptr;
  EL_CUDA_TRY(ctx, cudaMalloc(&d_V, (size_t)n * n * sizeof(double)));
  cudaError_t e = el::copy(ctx, d_V, h->Vbits.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_diag_v<<<grid_for(B.dim, 256), 256, (size_t)n * n * sizeof(double), ctx->stream>>>(
        B, n, d_V, h->d_diagV64, nullptr);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_V);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "diag_v");
  return EL_OK;
}

__global__ void k_to_f32(int64_t len, const double *a, float *b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

int ham_diag32(el_ctx *ctx, el_ham *h) {
  if (h->d_diagV32) return EL_OK;
  const int64_t dim = h->basis->dim;
  EL_CUDA_TRY(ctx, cudaMalloc(&h->d_diagV32, (size_t)dim * sizeof(float)));
  k_to_f32<<<grid_for(dim, 256), 256, 0, ctx->stream>>>(dim, h->d_diagV64, h->d_diagV32);
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_full_diag(el_ctx *ctx, el_ham *h, int dtype, void *out) {
  BasisDev B = basis_dev(h->basis);
  HamArgs<double> H = ham_args<double>(h, h->d_diagV64);
  if (dtype == EL_F64)
    k_full_diag<double><<<grid_for(B.dim, 256), 256, 0, ctx->stream>>>(B, H, (double *)out);
  else if (dtype == EL_F32)
    k_full_diag<float><<<grid_for(B.dim, 256), 256, 0, ctx->stream>>>(B, H, (float *)out);
  else
    return fail(ctx, EL_EINVAL, "diagonal dtype must be EL_F32 or EL_F64");
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int gershgorin(el_ctx *ctx, el_ham *h, double *lo, double *hi, double *norm1) {
  BasisDev B = basis_dev(h->basis);
  HamArgs<double> H = ham_args<double>(h, h->d_diagV64);
  const int grid = grid_for(B.dim, 256);
  int rc = ensure_partials(ctx, (size_t)grid * 3);
  if (rc) return rc;
  k_gershgorin<<<grid, 256, 0, ctx->stream>>>(B, H, ctx->d_partials, ctx->d_counter, ctx->d_scalars);
  EL_LAUNCH_CHECK(ctx);
  EL_CUDA_TRY(ctx, el::copy(ctx, ctx->h_scalars, ctx->d_scalars, 3 * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *lo = ctx->h_scalars[0];
  *hi = ctx->h_scalars[1];
  if (norm1) *norm1 = ctx->h_scalars[2];
  return EL_OK;
}

int launch_axpby(el_ctx *ctx, int dtype, int64_t len, double a_re, double a_im,
                 const void *x, double b_re, double b_im, void *y, double *norm2_out) {
  const int grid = grid_for(len, 256);
  if (norm2_out) {
    int rc = ensure_partials(ctx, (size_t)grid);
    if (rc) return rc;
  }
  switch (dtype) {
    case EL_F32: k_axpby<float, false><<<grid, 256, 0, ctx->stream>>>(len, a_re, a_im, (const float *)x, b_re, b_im, (float *)y, ctx->d_partials, ctx->d_counter, norm2_out); break;
    case EL_F64: k_axpby<double, false><<<grid, 256, 0, ctx->stream>>>(len, a_re, a_im, (const double *)x, b_re, b_im, (double *)y, ctx->d_partials, ctx->d_counter, norm2_out); break;
    case EL_C64: k_axpby<float, true><<<grid, 256, 0, ctx->stream>>>(len, a_re, a_im, (const float *)x, b_re, b_im, (float *)y, ctx->d_partials, ctx->d_counter, norm2_out); break;
    case EL_C128: k_axpby<double, true><<<grid, 256, 0, ctx->stream>>>(len, a_re, a_im, (const double *)x, b_re, b_im, (double *)y, ctx->d_partials, ctx->d_counter, norm2_out); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_gemv_t(el_ctx *ctx, int dtype, int64_t len, int k, const void *V,
                  int64_t ld, const void *w, double *dots_out) {
  if (k <= 0) return EL_OK;
  // one CTA per SM and column group: each thread walks many rows, so the
  // block reduction is paid once per many rows
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  int gx = grid_for(len, 256);
  const int ngroups = (k + GJ - 1) / GJ;
  const int gcap = std::max(1, (2 * sms + ngroups - 1) / ngroups);   // about two CTAs per SM in total
  if (gx > gcap) gx = gcap;
  dim3 grid(gx, ngroups);
  int rc = ensure_partials(ctx, (size_t)gx * k * 2);
  if (rc) return rc;
  switch (dtype) {
    case EL_F32: k_gemv_t<float, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, (const float *)w, ctx->d_partials); break;
    case EL_F64: k_gemv_t<double, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, (const double *)w, ctx->d_partials); break;
    case EL_C64: k_gemv_t<float, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, (const float *)w, ctx->d_partials); break;
    case EL_C128: k_gemv_t<double, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, (const double *)w, ctx->d_partials); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  k_sum_partials<<<(2 * k + 255) / 256, 256, 0, ctx->stream>>>(gx, k, ctx->d_partials, dots_out);
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_gemv_n_sub(el_ctx *ctx, int dtype, int64_t len, int k, const void *V,
                      int64_t ld, const double *coef, void *w) {
  if (k <= 0) return EL_OK;
  const int grid = grid_for(len, 256);
  switch (dtype) {
    case EL_F32: k_gemv_n<float, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, coef, (float *)w, true); break;
    case EL_F64: k_gemv_n<double, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, coef, (double *)w, true); break;
    case EL_C64: k_gemv_n<float, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, coef, (float *)w, true); break;
    case EL_C128: k_gemv_n<double, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, coef, (double *)w, true); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_gemv_n(el_ctx *ctx, int dtype, int64_t len, int k, const void *V,
                  int64_t ld, const double *coef_dev, void *out) {
  if (k <= 0) return EL_OK;
  const int grid = grid_for(len, 256);
  switch (dtype) {
    case EL_F32: k_gemv_n<float, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, coef_dev, (float *)out, false); break;
    case EL_F64: k_gemv_n<double, false><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, coef_dev, (double *)out, false); break;
    case EL_C64: k_gemv_n<float, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const float *)V, ld, coef_dev, (float *)out, false); break;
    case EL_C128: k_gemv_n<double, true><<<grid, 256, 0, ctx->stream>>>(len, k, (const double *)V, ld, coef_dev, (double *)out, false); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_fill_gauss(el_ctx *ctx, int dtype, int64_t len, uint64_t seed, void *out) {
  const int grid = grid_for(len, 256);
  switch (dtype) {
    case EL_F32: k_fill_gauss<float><<<grid, 256, 0, ctx->stream>>>(len, seed, (float *)out); break;
    case EL_F64: k_fill_gauss<double><<<grid, 256, 0, ctx->stream>>>(len, seed, (double *)out); break;
    case EL_C64: k_fill_gauss<float><<<grid_for(2 * len, 256), 256, 0, ctx->stream>>>(2 * len, seed, (float *)out); break;
    case EL_C128: k_fill_gauss<double><<<grid_for(2 * len, 256), 256, 0, ctx->stream>>>(2 * len, seed, (double *)out); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_fill_rademacher(el_ctx *ctx, int dtype, int64_t dim, int nvec,
                           uint64_t seed, int64_t probe0, int nvalid, void *out) {
  const int grid = grid_for(dim * nvec, 256);
  if (dtype == EL_F32)
    k_fill_rademacher<float><<<grid, 256, 0, ctx->stream>>>(dim, nvec, seed, probe0, nvalid, (float *)out);
  else if (dtype == EL_F64)
    k_fill_rademacher<double><<<grid, 256, 0, ctx->stream>>>(dim, nvec, seed, probe0, nvalid, (double *)out);
  else
    return fail(ctx, EL_EINVAL, "probes need a real dtype");
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_probe_copy(el_ctx *ctx, int dtype, int64_t dim, int nvec,
                      const int8_t *probes_dev, void *out) {
  const int grid = grid_for(dim * nvec, 256);
  if (dtype == EL_F32)
    k_probe_copy<float><<<grid, 256, 0, ctx->stream>>>(dim, nvec, probes_dev, (float *)out);
  else if (dtype == EL_F64)
    k_probe_copy<double><<<grid, 256, 0, ctx->stream>>>(dim, nvec, probes_dev, (double *)out);
  else
    return fail(ctx, EL_EINVAL, "probes need a real dtype");
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_scale(el_ctx *ctx, int dtype, int64_t len, const double *scale_dev,
                 int invert_sqrt, void *x) {
  const int64_t n = is_complex(dtype) ? 2 * len : len;
  const int grid = grid_for(n, 256);
  if (dtype == EL_F32 || dtype == EL_C64)
    k_scale<float><<<grid, 256, 0, ctx->stream>>>(n, scale_dev, invert_sqrt, (float *)x);
  else
    k_scale<double><<<grid, 256, 0, ctx->stream>>>(n, scale_dev, invert_sqrt, (double *)x);
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int launch_observables(el_ctx *ctx, el_ham *h, int dtype, const void *psi, double *out_dev) {
  BasisDev B = basis_dev(h->basis);
  const int grid = grid_for(B.dim, 256);
  int rc = ensure_partials(ctx, (size_t)grid * (B.n + 1));
  if (rc) return rc;
  switch (dtype) {
    case EL_F32: k_observables<float, false><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, ctx->d_partials, ctx->d_counter, out_dev); break;
    case EL_F64: k_observables<double, false><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, ctx->d_partials, ctx->d_counter, out_dev); break;
    case EL_C64: k_observables<float, true><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, ctx->d_partials, ctx->d_counter, out_dev); break;
    case EL_C128: k_observables<double, true><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, ctx->d_partials, ctx->d_counter, out_dev); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

}  // namespace el

// ------------------------------------------------------------------ C ABI

extern "C" {

int el_ham_create(el_ctx *ctx, el_basis *basis, const double *omega_re,
                  const double *omega_im, const double *delta, int n_pairs,
                  const int32_t *pi, const int32_t *pj, const double *V, el_ham **out) {
  if (!ctx || !basis || !out || !omega_re || !delta) return EL_EINVAL;
  *out = nullptr;
  if (n_pairs < 0 || (n_pairs > 0 && (!pi || !pj || !V))) return fail(ctx, EL_EINVAL, "bad pair list");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int n = basis->n;
  el_ham *h = new el_ham();
  h->basis = basis;
  h->n = n;
  memset(h->om_re, 0, sizeof h->om_re);
  memset(h->om_im, 0, sizeof h->om_im);
  memset(h->delta, 0, sizeof h->delta);
  memset(h->loss, 0, sizeof h->loss);
  h->Vbits.assign((size_t)n * n, 0.0);
  for (int p = 0; p < n_pairs; ++p) {
    const int i = pi[p], j = pj[p];
    if (i < 0 || j < 0 || i >= n || j >= n || i == j || !std::isfinite(V[p])) {
      delete h;
      return fail(ctx, EL_EINVAL, "pair %d: bad sites (%d, %d) or non-finite V", p, i, j);
    }
    const int qi = n - 1 - i, qj = n - 1 - j;
    h->Vbits[(size_t)qi * n + qj] += V[p];
    if (qi != qj) h->Vbits[(size_t)qj * n + qi] += V[p];
  }
  int rc = el_ham_set_drive(ctx, h, omega_re, omega_im, delta);
  if (rc) { delete h; return rc; }
  cudaError_t e = cudaMalloc(&h->d_diagV64, (size_t)basis->dim * sizeof(double));
  if (e != cudaSuccess) { delete h; return el::fail(ctx, EL_ENOMEM, "cannot allocate diagonal (%s)", cudaGetErrorString(e)); }
  rc = el::launch_diag_v(ctx, h);
  if (rc) { el_ham_destroy(h); return rc; }
  *out = h;
  return EL_OK;
}

int el_ham_set_drive(el_ctx *ctx, el_ham *h, const double *omega_re,
                     const double *omega_im, const double *delta) {
  if (!ctx || !h || !omega_re || !delta) return EL_EINVAL;
  const int n = h->n;
  bool cplx = false;
  for (int i = 0; i < n; ++i) {
    const double ore = omega_re[i], oim = omega_im ? omega_im[i] : 0.0, d = delta[i];
    if (!std::isfinite(ore) || !std::isfinite(oim) || !std::isfinite(d))
      return fail(ctx, EL_EINVAL, "Om/delta must be finite");
    const int q = n - 1 - i;
    h->om_re[q] = ore;
    h->om_im[q] = oim;
    h->delta[q] = d;
    if (oim != 0.0) cplx = true;
  }
  h->drive_complex = cplx;
  h->complex_drive = h->drive_complex || h->px_complex || h->lossy;
  return EL_OK;
}

int el_ham_set_loss(el_ctx *ctx, el_ham *h, const double *gamma) {
  if (!ctx || !h) return EL_EINVAL;
  const int n = h->n;
  // channels.py:69-76: diagonal (delta_i - 0.5 i gamma_i 1e-3 / CONV) n_i
  const double conv = 2.0 * 3.14159265358979323846 * 1e-3;
  bool any = false;
  double loss[EL_MAX_SITES] = {0.0};
  for (int i = 0; gamma && i < n; ++i) {
    if (!std::isfinite(gamma[i])) return fail(ctx, EL_EINVAL, "gamma must be finite");
    loss[n - 1 - i] = -0.5 * gamma[i] * 1e-3 / conv;
    if (gamma[i] != 0.0) any = true;
  }
  memcpy(h->loss, loss, sizeof loss);
  h->lossy = any;
  h->complex_drive = h->drive_complex || h->px_complex || h->lossy;
  return EL_OK;
}

int el_ham_set_exchange(el_ctx *ctx, el_ham *h, int n_pairs, const int32_t *pi,
                        const int32_t *pj, const double *J_re, const double *J_im,
                        const double *A_re, const double *A_im) {
  if (!ctx || !h) return EL_EINVAL;
  if (n_pairs < 0 || (n_pairs > 0 && (!pi || !pj))) return fail(ctx, EL_EINVAL, "bad exchange pair list");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int n = h->n;
  std::vector<ExPair> px;
  bool cplx = false;
  for (int p = 0; p < n_pairs; ++p) {
    const int i = pi[p], j = pj[p];
    ExPair e;
    e.jre = J_re ? J_re[p] : 0.0;
    e.jim = J_im ? J_im[p] : 0.0;
    e.are = A_re ? A_re[p] : 0.0;
    e.aim = A_im ? A_im[p] : 0.0;
    if (i < 0 || j < 0 || i >= n || j >= n || i == j)
      return fail(ctx, EL_EINVAL, "exchange pair %d: bad sites (%d, %d)", p, i, j);
    if (!std::isfinite(e.jre) || !std::isfinite(e.jim) || !std::isfinite(e.are) || !std::isfinite(e.aim))
      return fail(ctx, EL_EINVAL, "exchange pair %d: non-finite J or A", p);
    if (e.jre == 0.0 && e.jim == 0.0 && e.are == 0.0 && e.aim == 0.0) continue;
    e.bi = n - 1 - i;
    e.bj = n - 1 - j;
    if (e.jim != 0.0 || e.aim != 0.0) cplx = true;
    px.push_back(e);
  }
  // hop table of the J channels and the list of A pairs
  std::vector<double> hop(2 * (size_t)n * n, 0.0);
  std::vector<ExPair> pxA;
  for (const ExPair &e : px) {
    // row (i, j) = (r, g): bit bi set, bj clear -> J; row (g, r) -> conj(J)
    hop[(size_t)e.bi * n + e.bj] += e.jre;
    hop[(size_t)n * n + (size_t)e.bi * n + e.bj] += e.jim;
    hop[(size_t)e.bj * n + e.bi] += e.jre;
    hop[(size_t)n * n + (size_t)e.bj * n + e.bi] -= e.jim;
    if (e.are != 0.0 || e.aim != 0.0) pxA.push_back(e);
  }
  ExPair *d = nullptr, *dA = nullptr;
  double *dh = nullptr;
  auto upload = [&](void **dst, const void *src, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e != cudaSuccess) return e;
    e = el::copy(ctx, *dst, src, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e;
  };
  if (!px.empty()) {
    cudaError_t e = upload((void **)&d, px.data(), px.size() * sizeof(ExPair));
    if (e == cudaSuccess) e = upload((void **)&dh, hop.data(), hop.size() * sizeof(double));
    if (e == cudaSuccess && !pxA.empty()) e = upload((void **)&dA, pxA.data(), pxA.size() * sizeof(ExPair));
    if (e != cudaSuccess) {
      cudaFree(d); cudaFree(dh); cudaFree(dA);
      cudaGetLastError();
      return el::fail(ctx, EL_ENOMEM, "cannot store exchange channels (%s)", cudaGetErrorString(e));
    }
  }
  // the previous lists may still be read by work queued on the stream
  if (h->d_px || h->d_hop || h->d_pxA) {
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(h->d_px);
    cudaFree(h->d_hop);
    cudaFree(h->d_pxA);
  }
  h->d_px = d;
  h->d_hop = dh;
  h->d_pxA = dA;
  h->npxA = (int)pxA.size();
  h->px.swap(px);
  h->px_complex = cplx;
  h->complex_drive = h->drive_complex || h->px_complex || h->lossy;
  return EL_OK;
}

int el_ham_diag(el_ctx *ctx, el_ham *h, int dtype, void *out) {
  if (!ctx || !h || !out) return EL_EINVAL;
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  return el::launch_full_diag(ctx, h, dtype, out);
}

int el_ham_destroy(el_ham *h) {
  if (!h) return EL_OK;
  if (h->basis) cudaSetDevice(h->basis->device);
  if (h->d_diagV64) cudaFree(h->d_diagV64);
  if (h->d_diagV32) cudaFree(h->d_diagV32);
  if (h->d_px) cudaFree(h->d_px);
  if (h->d_hop) cudaFree(h->d_hop);
  if (h->d_pxA) cudaFree(h->d_pxA);
  delete h;
  return EL_OK;
}

int el_hv(el_ctx *ctx, el_ham *h, int dtype, int nvec, const void *x, void *y) {
  if (!ctx || !h || !x || !y) return EL_EINVAL;
  if (x == y) return el::fail(ctx, EL_EINVAL, "el_hv: x and y must not alias");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  ApplyArgs A;
  memset(&A, 0, sizeof A);
  A.dtype = dtype;
  A.nvec = nvec;
  A.x = x;
  A.y = y;
  A.a = 1.0;
  return el::launch_apply(ctx, h, A);
}

int el_hv_host(el_ctx *ctx, el_ham *h, int dtype, int nvec, const void *x_host, void *y_host) {
  if (!ctx || !h || !x_host || !y_host) return EL_EINVAL;
  const int es = el::dtype_size(dtype);
  if (!es) return el::fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = (size_t)h->basis->dim * nvec * es;
  // device copies in the context's cached workspace (kept between calls)
  char *buf = (char *)el::workspace(ctx, 14, 2 * bytes);
  if (!buf) return EL_ENOMEM;
  void *dx = buf, *dy = buf + bytes;
  cudaError_t e = el::copy(ctx, dx, x_host, bytes, cudaMemcpyHostToDevice);
  int rc = EL_OK;
  if (e == cudaSuccess) {
    rc = el_hv(ctx, h, dtype, nvec, dx, dy);
    if (rc == EL_OK) {
      e = el::copy(ctx, y_host, dy, bytes, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
  }
  if (rc) return rc;
  if (e != cudaSuccess) return el::cuda_fail(ctx, e, "el_hv_host");
  return EL_OK;
}

int el_observables(el_ctx *ctx, el_ham *h, int dtype, const void *psi,
                   double *n_site_host, double *norm_host) {
  if (!ctx || !h || !psi) return EL_EINVAL;
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int n = h->n;
  int rc = el::launch_observables(ctx, h, dtype, psi, ctx->d_scalars);
  if (rc) return rc;
  EL_CUDA_TRY(ctx, el::copy(ctx, ctx->h_scalars, ctx->d_scalars, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (n_site_host)
    for (int i = 0; i < n; ++i) n_site_host[i] = ctx->h_scalars[n - 1 - i];
  if (norm_host) *norm_host = ctx->h_scalars[n];
  return EL_OK;
}

}  // extern "C"
