// TMA-fed tiled KPM recurrence on the full 2^N basis (14 <= N <= 25).
//
// Same two-group pass scheme as el_kpm_full.cu (see its header): the
// sigma^x part of H splits by row bit into X_A (row bits [0, a)) and X_B
// (row bits [a, N)); a pass over the tiles of one group completes
//   t_m     = p_m + s_m X_G t_{m-1}
// and starts
//   p_{m+1} = 2(D-c)/r t_m + (2/r) X_G t_m - t_{m-1},
// reading two vectors and writing two per Chebyshev step.
//
// Here every byte of tile traffic moves by TMA, not through the LSU pipe:
//   - vectors are [probe][row] arrays (one probe per cell), so an A tile
//     (2^a consecutive rows) is one 64 KB box (two 128-byte-swizzled 32 KB
//     boxes for the two-layout FP32 A pass of 14-bit tiles, k_kpm_tx_a);
//   - a B tile holds the C lowest row bits as a contiguous piece of 32 bytes
//     (C = 3 for FP32: one DRAM sector) or 16 bytes (C = 1 for FP64), carried
//     but not flipped, plus row bits a..N-1; its 2^(N-a) pieces lie 2^a rows
//     apart and move as one 5-D box (one TMA instruction).  The tile index
//     enumerates row bits C..a-1.  a = 14 (FP32) / 13 (FP64) at N = 25 keeps
//     both tiles at 64 KB;
//   - the t_{m-1} tile of the next work item is prefetched into a second
//     buffer while the current one is processed;
//   - t_m and p_{m+1} are written into shared memory and stored by TMA.
// Shared memory per CTA: three 64 KB buffers (S_cur, S_next, S2) = 192 KB.
// Waits on the TMA transaction barriers are bounded; on timeout the kernel
// records an error flag (read by the host) and finishes without hanging.
#include "el_internal.cuh"

#define EL_KPM_MAXN 25   // sites of the tiled full-basis passes

#include <algorithm>
#include <cuda.h>
#include <cudaTypedefs.h>

namespace {

using el::fail;

// One probe per cell.  CARRY: low row bits a B tile keeps as one contiguous
// piece; LOGCH: log2 of the cells in a 256-byte A-map chunk.
template <typename T> struct Cell {
  typedef T U;
  static constexpr int PU = 1;
  static constexpr int CARRY = sizeof(T) == 4 ? 3 : 1;
  static constexpr int LOGCH = sizeof(T) == 4 ? 6 : 5;
};

__device__ __forceinline__ float z8(float) { return 0.f; }
__device__ __forceinline__ double z8(double) { return 0.0; }
__device__ __forceinline__ float fma8(float s, float x, float y) { return fmaf(s, x, y); }
__device__ __forceinline__ double fma8(double s, double x, double y) { return fma(s, x, y); }
__device__ __forceinline__ float sub8(float a, float b) { return a - b; }
__device__ __forceinline__ double sub8(double a, double b) { return a - b; }
__device__ __forceinline__ float scl8(float s, float x) { return s * x; }
__device__ __forceinline__ double scl8(double s, double x) { return s * x; }
__device__ __forceinline__ float get8(float v, int) { return v; }
__device__ __forceinline__ double get8(double v, int) { return v; }


enum { KIND_A = 0, KIND_B = 1 };
enum { MODE_STEP = 0, MODE_PROLOGUE = 1, MODE_LAST = 2 };

template <typename T>
struct TmaArgs {
  int n, a, mode, ng, log_tiles;
  // FP32 passes: the diagonal from tile sums instead of a d2 array (V
  // between row bits [n][n] and delta per row bit, FP64), d2 = s2 d + s2c;
  // wtab: per tile, OTF_ROW doubles {wH_0 .. wH_{TB-1}, ..., cH}
  const double *vbits;
  const double *wtab;
  double delta_b[32];
  double s2, s2c;
  int64_t dim, tiles, items;
  T s_m, two_r, pro_alpha, pro_beta;
  T amp[16];
  // apply passes (single vector): y = D x + X_A x + cz z, then y += X_B x
  const T *dfull, *z;
  T *y;
  T cz;
  const T *d2;
  double *partials;
  unsigned int *counter;
  double *dots;
  int *err;
};

// Work item -> (probe group, tile), group-major: the CTAs working at the
// same time hold adjacent tiles of one probe group, so the 32-byte pieces of
// neighbouring B tiles share DRAM pages.  (A tile-major order, which would
// share each diagonal tile in L2 across the probe groups, measured 1.7x
// slower in FP32 and 3.2x in FP64 for losing that locality.)
template <typename T>
__device__ __forceinline__ int item_group(const TmaArgs<T> &A, int64_t item) {
  return (int)(item >> A.log_tiles);
}
template <typename T>
__device__ __forceinline__ uint32_t item_tile(const TmaArgs<T> &A, int64_t item) {
  return (uint32_t)(item & (A.tiles - 1));
}

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait: gives up after a fixed number of polls and flags the error.
__device__ __forceinline__ void mbar_wait(uint64_t *bar, unsigned parity, int *err) {
  for (int it = 0; it < (1 << 20); ++it)
    if (mbar_try(bar, parity)) return;
  atomicExch(err, 1);
}
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *m, int c0, int c1, int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_load5(void *dst, const CUtensorMap *m, int c0, int c1, int c2, int c3, int c4,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      ::"r"(smem_u32(dst)), "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_store3(const CUtensorMap *m, int c0, int c1, int c2, const void *src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
               ::"l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src)) : "memory");
}
__device__ __forceinline__ void tma_store5(const CUtensorMap *m, int c0, int c1, int c2, int c3, int c4,
                                           const void *src) {
  asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
               ::"l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(src)) : "memory");
}
// Untiled bulk copy global -> shared (16-byte aligned addresses, size a
// multiple of 16), completing on the mbarrier of the tile it travels with.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tile <-> tensor-map coordinates.  A: 3-D map {256-byte chunk, chunk index,
// probe}; B: 5-D map {low-bit piece, tile, h_lo, h_hi, probe}, one box per
// tile (h = the row bits above a, split so that no box side exceeds 256).
template <int KIND, typename T>
__device__ __forceinline__ void tile_load(const TmaArgs<T> &A, void *dst, const CUtensorMap *m,
                                          uint32_t tile, int g, uint64_t *bar) {
  if (KIND == KIND_A) {
    tma_load3(dst, m, 0, (int)(tile << (A.a - Cell<T>::LOGCH)), g, bar);
  } else {
    tma_load5(dst, m, 0, (int)tile, 0, 0, g, bar);
  }
}
template <int KIND, typename T>
__device__ __forceinline__ void tile_store(const TmaArgs<T> &A, const CUtensorMap *m, uint32_t tile,
                                           int g, const void *src) {
  if (KIND == KIND_A) {
    tma_store3(m, 0, (int)(tile << (A.a - Cell<T>::LOGCH)), g, src);
  } else {
    tma_store5(m, 0, (int)tile, 0, 0, g, src);
  }
}

template <int KIND, int C>
__device__ __forceinline__ uint32_t row_of(int a, uint32_t tile, int l) {
  if (KIND == KIND_A) return (tile << a) + (uint32_t)l;
  return (uint32_t)(l & ((1 << C) - 1)) + ((uint32_t)(l >> C) << a) + (tile << C);
}

// Index of cell l of a tile in the (row-ordered) diagonal array.
template <typename T, int KIND, int TB>
__device__ __forceinline__ size_t d2_index(int a, uint32_t tile, int l) {
  return row_of<KIND, Cell<T>::CARRY>(a, tile, l);
}

// Row bit of tile bit k, and of tile-index bit i.
template <int KIND, int C>
__device__ __forceinline__ int tile_rowbit(int a, int k) {
  return KIND == KIND_A ? k : (k < C ? k : a + k - C);
}
template <int KIND, int C>
__device__ __forceinline__ int index_rowbit(int a, int i) {
  return KIND == KIND_A ? a + i : C + i;
}

// h[j] += sum_{k in [K0, KMAX)} amp_k * S[(tid ^ 2^k) + NT*j] for the R cells
// of this thread (NT = 2^KMAX threads).  Bit-outer order: one address per
// bit, R independent FMA chains per bit.
template <typename T, int R, int K0, int KMAX>
__device__ __forceinline__ void gather_all(const T *S, int tid, const TmaArgs<T> &A, T (&h)[R]) {
#pragma unroll
  for (int k = K0; k < KMAX; ++k) {
    const T *base = S + (tid ^ (1 << k));
    const T a = A.amp[k];
#pragma unroll
    for (int j = 0; j < R; ++j) h[j] = fma8(a, base[(1 << KMAX) * j], h[j]);
  }
}

// d2 = 2 (D - c) / r of this thread's R cells of a tile.  FP32 passes form
// it from the per-thread, per-CTA and per-tile sums in FP64 and round once
// (as a precomputed FP32 array would be rounded); FP64 passes read the d2
// array (their registers have no room for the sums).
template <typename T> struct OnTheFly { static constexpr bool value = sizeof(T) == 4; };

// Per-tile couplings of the FP32 passes, one 128-byte row per tile:
// slot k < TB holds wH_k = sum over the tile's set index bits i of
// V(row bit of tile bit k, row bit of index bit i); the last slot holds cH,
// the diagonal of the set index bits alone (their delta plus the V among
// them); the slots between are zero.  The row travels with the tile's TMA
// load, so no thread sums couplings while the others wait.
constexpr int OTF_ROW = 16;
struct DeltaBits { double v[32]; };

template <int KIND, int C>
__global__ void k_otf_table(int n, int a, int TB, int log_tiles, int64_t tiles, const double *__restrict__ vbits,
                            DeltaBits delta, double *__restrict__ out) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= tiles * OTF_ROW) return;
  const uint32_t tile = (uint32_t)(gid / OTF_ROW);
  const int slot = (int)(gid % OTF_ROW);
  double sacc = 0.0;
  if (slot < TB) {
    const int K = tile_rowbit<KIND, C>(a, slot);
    for (int i = 0; i < log_tiles; ++i)
      if ((tile >> i) & 1u) sacc += vbits[K * n + index_rowbit<KIND, C>(a, i)];
  } else if (slot == OTF_ROW - 1) {
    for (int i = 0; i < log_tiles; ++i) {
      if (!((tile >> i) & 1u)) continue;
      const int I = index_rowbit<KIND, C>(a, i);
      sacc += delta.v[I];
      for (int i2 = 0; i2 < i; ++i2)
        if ((tile >> i2) & 1u) sacc += vbits[I * n + index_rowbit<KIND, C>(a, i2)];
    }
  }
  out[gid] = sacc;
}

template <typename T, int KIND, int TB, int LNT>
__device__ __forceinline__ void tile_diag(const TmaArgs<T> &A, uint32_t tile, int tid, double cT,
                                          const double *cTJ, const double *tJ, const double *wH, double cH,
                                          const T *__restrict__ d2, T (&dv)[1 << (TB - LNT)]) {
  constexpr int RB = TB - LNT;
  constexpr int R = 1 << RB;
  constexpr int NT = 1 << LNT;
  if constexpr (!OnTheFly<T>::value) {
#pragma unroll
    for (int j = 0; j < R; ++j) dv[j] = d2[d2_index<T, KIND, TB>(A.a, tile, tid + NT * j)];
  } else {
    double base = cT + cH;
    for (int x = 0; x < LNT; ++x)
      if ((tid >> x) & 1) base += wH[x];
    double u[RB > 0 ? RB : 1];
#pragma unroll
    for (int k = 0; k < RB; ++k) u[k] = cTJ[k * NT + tid] + wH[LNT + k];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      double dj = base + tJ[j];
#pragma unroll
      for (int k = 0; k < RB; ++k)
        if ((j >> k) & 1) dj += u[k];
      dv[j] = (T)fma(A.s2, dj, A.s2c);
    }
  }
}

template <typename T, int TB, int KIND, int LNT>
__global__ void __launch_bounds__(1 << LNT, 1)
k_kpm_tma(const TmaArgs<T> A, const __grid_constant__ CUtensorMap mapP,
          const __grid_constant__ CUtensorMap mapQ) {
  typedef typename Cell<T>::U U;
  constexpr int PU = Cell<T>::PU;
  constexpr int C = Cell<T>::CARRY;
  constexpr int NT = 1 << LNT;               // threads per CTA
  constexpr int R = (1 << TB) / NT;          // cells per thread (TB >= LNT)
  constexpr int LOGNT = LNT;
  constexpr int NWARP = NT / 32;
  constexpr int K0 = (KIND == KIND_B) ? C : 0;
  constexpr unsigned TILE_BYTES = (1u << TB) * (unsigned)sizeof(T);
  static_assert(TILE_BYTES <= 65536, "three tile buffers must fit in shared memory");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  U *const Sb0 = reinterpret_cast<U *>(smem_raw);
  U *const Sb1 = reinterpret_cast<U *>(smem_raw + TILE_BYTES);
  U *const S2 = reinterpret_cast<U *>(smem_raw + 2 * TILE_BYTES);
  __shared__ __align__(8) uint64_t bar[3];   // S buffers 0/1, S2
  __shared__ double wred[NWARP][2 * PU];
  // The diagonal of a cell's row, d = sum_b delta_b + sum_{b<b'} V_bb' over
  // its set row bits, split over the three sets of bits a cell's row has:
  // the thread's index bits (T, fixed per thread), its register bits (J,
  // the cell's slot j) and the tile index bits (H, fixed per tile):
  //   d = cT + tJ[j] + cH + sum_{x in T} wH_x + sum_{k in J(j)} (cTJ_k + wH_k)
  // with cT, cTJ per thread once, tJ per CTA once, and cH, wH_k (the
  // couplings of every tile bit to the tile's set index bits) per tile.
  constexpr int RB = TB - LNT;               // register bits
  constexpr bool OTF = OnTheFly<T>::value;
  __shared__ double sV[OTF ? EL_KPM_MAXN * EL_KPM_MAXN : 1];
  __shared__ double tJ[OTF ? R : 1];
  __shared__ double cTJ[OTF ? (RB > 0 ? RB : 1) * NT : 1];   // [k][tid]: couplings of the thread bits to register bit k
  __shared__ __align__(16) double wHt[2][OTF_ROW];   // the table rows of the tiles in S buffers 0/1
  constexpr unsigned WROW_BYTES = OTF ? OTF_ROW * sizeof(double) : 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ndots = A.ng * PU * 2;
  const int nb = A.n;
  double *dacc = A.partials + (size_t)blockIdx.x * ndots;
  for (int i = tid; i < ndots; i += NT) dacc[i] = 0.0;
  if constexpr (OTF)
    for (int i = tid; i < nb * nb; i += NT) sV[i] = A.vbits[i];
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    fence_async_smem();
  }
  __syncthreads();
  double cT = 0.0;
  if constexpr (OTF) {
    for (int x = 0; x < LNT; ++x) {
      if (!((tid >> x) & 1)) continue;
      const int X = tile_rowbit<KIND, C>(A.a, x);
      cT += A.delta_b[X];
      for (int x2 = 0; x2 < x; ++x2)
        if ((tid >> x2) & 1) cT += sV[X * nb + tile_rowbit<KIND, C>(A.a, x2)];
    }
#pragma unroll
    for (int k = 0; k < RB; ++k) {
      const int K = tile_rowbit<KIND, C>(A.a, LNT + k);
      double sacc = 0.0;
      for (int x = 0; x < LNT; ++x)
        if ((tid >> x) & 1) sacc += sV[tile_rowbit<KIND, C>(A.a, x) * nb + K];
      cTJ[k * NT + tid] = sacc;
    }
    for (int j = tid; j < R; j += NT) {
      double v = 0.0;
      for (int k = 0; k < RB; ++k) {
        if (!((j >> k) & 1)) continue;
        const int K = tile_rowbit<KIND, C>(A.a, LNT + k);
        v += A.delta_b[K];
        for (int k2 = 0; k2 < k; ++k2)
          if ((j >> k2) & 1) v += sV[K * nb + tile_rowbit<KIND, C>(A.a, LNT + k2)];
      }
      tJ[j] = v;
    }
  }
  unsigned par[3] = {0u, 0u, 0u};
  const T *__restrict__ d2 = A.d2;
  int cur = 0;
  int64_t item = blockIdx.x;
  // per-thread FP64 sums of <t,t> and <t,t_prev> for the current probe group
  double acc_tt[PU], acc_tq[PU];
#pragma unroll
  for (int q = 0; q < PU; ++q) { acc_tt[q] = 0.0; acc_tq[q] = 0.0; }
  int gacc = item_group(A, item);
  if (tid == 0 && item < A.items) {
    const uint32_t tile = item_tile(A, item);
    mbar_expect(&bar[0], TILE_BYTES + WROW_BYTES);
    tile_load<KIND>(A, Sb0, &mapQ, tile, gacc, &bar[0]);
    if constexpr (OTF) bulk_load(wHt[0], A.wtab + (size_t)tile * OTF_ROW, WROW_BYTES, &bar[0]);
  }
  for (; item < A.items; item += gridDim.x) {
    const int g = item_group(A, item);
    const uint32_t tile = item_tile(A, item);
    const int64_t nxt = item + gridDim.x;
    if (g != gacc) {   // uniform across the CTA: flush the previous group's sums
#pragma unroll
      for (int q = 0; q < PU; ++q) {
        double x = acc_tt[q], y = acc_tq[q];
        for (int o = 16; o > 0; o >>= 1) {
          x += __shfl_xor_sync(0xffffffffu, x, o);
          y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (lane == 0) { wred[warp][2 * q] = x; wred[warp][2 * q + 1] = y; }
        acc_tt[q] = 0.0; acc_tq[q] = 0.0;
      }
      __syncthreads();
      if (tid < 2 * PU) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
        dacc[gacc * PU * 2 + tid] += sum;
      }
      gacc = g;
    }
    U *S = cur ? Sb1 : Sb0;
    U *Sn = cur ? Sb0 : Sb1;
    // S2 is refilled only after (1) the previous item's S2 store has read it
    // (in a step pass that store is the older of the item's two groups and
    // the S store may still be reading Sn; in the prologue it is the only
    // group) and (2) every thread has finished the previous item, whose last
    // pass reads S2 after its final barrier.
    if (tid == 0) {
      if (A.mode == MODE_PROLOGUE) bulk_wait_read<0>();
      else bulk_wait_read<1>();
    }
    __syncthreads();
    if (tid == 0 && A.mode != MODE_PROLOGUE) {
      mbar_expect(&bar[2], TILE_BYTES);
      tile_load<KIND>(A, S2, &mapP, tile, g, &bar[2]);
    }
    if (cur) { mbar_wait(&bar[1], par[1], A.err); par[1] ^= 1u; }
    else { mbar_wait(&bar[0], par[0], A.err); par[0] ^= 1u; }

    U own[R], hx[R];
#pragma unroll
    for (int j = 0; j < R; ++j) { own[j] = S[tid + NT * j]; hx[j] = z8(U{}); }
    // X_G t_{m-1} (or X_G t_0 in the prologue): shared bits, then the upper
    // tile bits, whose partners are this thread's own cells
    gather_all<T, R, K0, LOGNT>(S, tid, A, hx);
#pragma unroll
    for (int b = 0; (1 << b) < R; ++b)
#pragma unroll
      for (int j = 0; j < R; ++j) hx[j] = fma8(A.amp[LOGNT + b], own[j ^ (1 << b)], hx[j]);
    if (tid == 0 && nxt < A.items) {
      // prefetch the next t_{m-1} tile once the previous S store has read Sn
      bulk_wait_read<0>();
      const int gn = item_group(A, nxt);
      const uint32_t tn = item_tile(A, nxt);
      uint64_t *bn = cur ? &bar[0] : &bar[1];
      mbar_expect(bn, TILE_BYTES + WROW_BYTES);
      tile_load<KIND>(A, Sn, &mapQ, tn, gn, bn);
      if constexpr (OTF) bulk_load(wHt[cur ^ 1], A.wtab + (size_t)tn * OTF_ROW, WROW_BYTES, bn);
    }
    // per-tile products: two interleaved FP32 partial sums per quantity,
    // widened to FP64 once per tile
    T pt[PU][2], pq[PU][2];
#pragma unroll
    for (int q = 0; q < PU; ++q) { pt[q][0] = pt[q][1] = pq[q][0] = pq[q][1] = (T)0; }
    if (A.mode == MODE_PROLOGUE) {
      // p_1 = (D-c)/r t_0 + pro_beta X_G t_0 -> S2 -> P
      T dv[R];
      tile_diag<T, KIND, TB, LNT>(A, tile, tid, cT, cTJ, tJ, wHt[cur], wHt[cur][OTF_ROW - 1], d2, dv);
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int l = tid + NT * j;
        S2[l] = fma8(A.pro_beta, hx[j], scl8(A.pro_alpha * dv[j], own[j]));
#pragma unroll
        for (int q = 0; q < PU; ++q) pt[q][j & 1] = fma(get8(own[j], q), get8(own[j], q), pt[q][j & 1]);
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0) { tile_store<KIND>(A, &mapP, tile, g, S2); bulk_commit(); }
    } else {
      mbar_wait(&bar[2], par[2], A.err);
      par[2] ^= 1u;
      // t_m = p_m + s_m X_G t_{m-1}
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int l = tid + NT * j;
        const U t = fma8(A.s_m, hx[j], S2[l]);
        if (A.mode != MODE_LAST) S2[l] = t;
        hx[j] = t;
#pragma unroll
        for (int q = 0; q < PU; ++q) {
          pt[q][j & 1] = fma(get8(t, q), get8(t, q), pt[q][j & 1]);
          pq[q][j & 1] = fma(get8(t, q), get8(own[j], q), pq[q][j & 1]);
        }
      }
      if (A.mode != MODE_LAST) {
        fence_async_smem();
        __syncthreads();
        if (tid == 0) { tile_store<KIND>(A, &mapP, tile, g, S2); bulk_commit(); }
        // p_{m+1} = d2 t_m + (2/r) X_G t_m - t_{m-1}  (t_m in hx[], t_{m-1} in own[])
        // the diagonal of this thread's rows, loaded before the gathers so
        // that its latency hides behind them
        T dv[R];
        tile_diag<T, KIND, TB, LNT>(A, tile, tid, cT, cTJ, tJ, wHt[cur], wHt[cur][OTF_ROW - 1], d2, dv);
        U h2[R];
#pragma unroll
        for (int j = 0; j < R; ++j) h2[j] = z8(U{});
        gather_all<T, R, K0, LOGNT>(S2, tid, A, h2);
#pragma unroll
        for (int b = 0; (1 << b) < R; ++b)
#pragma unroll
          for (int j = 0; j < R; ++j) h2[j] = fma8(A.amp[LOGNT + b], hx[j ^ (1 << b)], h2[j]);
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const int l = tid + NT * j;
          S[l] = sub8(fma8(A.two_r, h2[j], scl8(dv[j], hx[j])), S[l]);   // S[l] = t_{m-1}
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) { tile_store<KIND>(A, &mapQ, tile, g, S); bulk_commit(); }
      }
    }
    // per-tile products: FP32 tree sums over the R cells, widened to FP64
#pragma unroll
    for (int q = 0; q < PU; ++q) {
      acc_tt[q] += (double)pt[q][0] + (double)pt[q][1];
      acc_tq[q] += (double)pq[q][0] + (double)pq[q][1];
    }
    cur ^= 1;
  }
  // flush the last group
#pragma unroll
  for (int q = 0; q < PU; ++q) {
    double x = acc_tt[q], y = acc_tq[q];
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) { wred[warp][2 * q] = x; wred[warp][2 * q + 1] = y; }
  }
  __syncthreads();
  if (tid < 2 * PU && blockIdx.x < A.items) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
    dacc[gacc * PU * 2 + tid] += sum;
  }
  if (tid == 0) bulk_wait_all();
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

// --------------------------------------------- 16-byte vector helpers
//
// Used by the single-vector FP64 tiled H x below: every access is a
// 16-byte vector (double2) of consecutive cells, so the lowest tile bit is a
// register bit: cell l = v + VN (tid + NT q) for vector lane v and block q.
template <typename T> struct V16;
template <> struct V16<double> { static constexpr int N = 2, LOG = 1; };

__device__ __forceinline__ void ld16(const double *p, double *d) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  d[0] = v.x; d[1] = v.y;
}
__device__ __forceinline__ void st16(double *p, const double *d) {
  *reinterpret_cast<double2 *>(p) = make_double2(d[0], d[1]);
}
__device__ __forceinline__ void stcs16(double *p, const double *d) {
  __stcs(reinterpret_cast<double2 *>(p), make_double2(d[0], d[1]));
}
__device__ __forceinline__ void ldg16(const double *p, double *d) {
  const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
  d[0] = v.x; d[1] = v.y;
}

// h[j] += amp[k] x[partner_k(j)] over every flipped bit k of the tile for
// this thread's R cells: x in registers (src) and, for the thread-index
// bits, in shared memory (S, natural cell order).
template <typename T, int TB, int KIND, int LNT, bool SHF, int R, int C = Cell<T>::CARRY>
__device__ __forceinline__ void xapply_tile(const T *S, const T (&src)[R], T (&h)[R], const T *amp, int tid) {
  constexpr int VN = V16<T>::N, VB = V16<T>::LOG;
  constexpr int NT = 1 << LNT;
  constexpr int QB = TB - VB - LNT;
  constexpr int QR = 1 << QB;
  // bits inside the 16-byte vector
#pragma unroll
  for (int b = 0; b < VB; ++b) {
    if (KIND == KIND_B && b < C) continue;
    const T a = amp[b];
#pragma unroll
    for (int j = 0; j < R; ++j) h[j] = fma8(a, src[j ^ (1 << b)], h[j]);
  }
  // block bits (above the thread index)
#pragma unroll
  for (int b = 0; b < QB; ++b) {
    const T a = amp[VB + LNT + b];
#pragma unroll
    for (int j = 0; j < R; ++j) h[j] = fma8(a, src[j ^ (VN << b)], h[j]);
  }
  // thread-index bits: lanes (shuffles or shared loads), then warps
#pragma unroll
  for (int b = 0; b < LNT; ++b) {
    const int k = VB + b;
    if (KIND == KIND_B && k < C) continue;
    const T a = amp[k];
    if (SHF && b < 5) {
#pragma unroll
      for (int j = 0; j < R; ++j) h[j] = fma8(a, __shfl_xor_sync(0xffffffffu, src[j], 1 << b), h[j]);
    } else {
      const T *base = S + (size_t)VN * (tid ^ (1 << b));
#pragma unroll
      for (int q = 0; q < QR; ++q) {
        T w[VN];
        ld16(base + (size_t)VN * NT * q, w);
#pragma unroll
        for (int v = 0; v < VN; ++v) h[VN * q + v] = fma8(a, w[v], h[VN * q + v]);
      }
    }
  }
}

// global cell index (within one probe group) of the first cell of 16-byte
// block l0 of a tile
template <typename T, int KIND, int CR = Cell<T>::CARRY>
__device__ __forceinline__ size_t gcell(int a, uint32_t tile, int l0) {
  return row_of<KIND, CR>(a, tile, l0);
}

// ------------------------------------------------------ single-vector H x
//
// y = H x + cz z on the full basis as two tiled passes over one vector (the
// Lanczos steps of the spectral bounds): the B pass (tiles of 2^C-row
// pieces 2^a rows apart) writes y = X_B x, the A pass (tiles of 2^a
// consecutive rows) completes y = D x + X_A x + cz z + y and forms <x,x>,
// <x,y>, <y,y>.  x arrives by TMA, double-buffered; z, D and y move by
// 16-byte loads and stores, so the strided B pieces of y are only written
// (the reads of y are contiguous A rows).  Seven vector moves per product,
// instead of the row kernel's repeated DRAM reads of every high-bit partner.
template <typename T, int NWARP>
__device__ __forceinline__ void hv_finish_dots(const TmaArgs<T> &A, double sxx, double sxy, double syy,
                                               double (*wred)[3]);

template <typename T, int TB, int KIND, int LNT>
__global__ void __launch_bounds__(1 << LNT, 1)
k_hv_pass(const TmaArgs<T> A, const __grid_constant__ CUtensorMap mapX) {
  constexpr int VN = V16<T>::N, VB = V16<T>::LOG;
  constexpr int NT = 1 << LNT;
  constexpr int QB = TB - VB - LNT;
  static_assert(QB >= 0, "tile smaller than one vector per thread");
  constexpr int QR = 1 << QB;
  constexpr int R = VN * QR;
  constexpr int NWARP = NT / 32;
  constexpr unsigned TILE_BYTES = (1u << TB) * (unsigned)sizeof(T);
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  T *const buf0 = reinterpret_cast<T *>(smem_raw);
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ double wred[NWARP][3];
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_async_smem();
  }
  __syncthreads();
  unsigned par[2] = {0u, 0u};
  int cur = 0;
  int64_t item = blockIdx.x;
  if (tid == 0 && item < A.items) {
    mbar_expect(&bar[0], TILE_BYTES);
    tile_load<KIND>(A, buf0, &mapX, (uint32_t)item, 0, &bar[0]);
  }
  double sxx = 0.0, sxy = 0.0, syy = 0.0;
  for (; item < A.items; item += gridDim.x) {
    const uint32_t tile = (uint32_t)item;
    const int64_t nxt = item + gridDim.x;
    if (tid == 0 && nxt < A.items) {   // the other buffer was released at the end of the last item
      mbar_expect(&bar[cur ^ 1], TILE_BYTES);
      tile_load<KIND>(A, buf0 + (size_t)(cur ^ 1) * (1u << TB), &mapX, (uint32_t)nxt, 0, &bar[cur ^ 1]);
    }
    mbar_wait(&bar[cur], par[cur], A.err);
    par[cur] ^= 1u;
    const T *S = buf0 + (size_t)cur * (1u << TB);
    T own[R], h[R];
#pragma unroll
    for (int q = 0; q < QR; ++q) ld16(S + (size_t)VN * (tid + NT * q), own + VN * q);
#pragma unroll
    for (int j = 0; j < R; ++j) h[j] = z8(T{});
    xapply_tile<T, TB, KIND, LNT, true, R>(S, own, h, A.amp, tid);
#pragma unroll
    for (int q = 0; q < QR; ++q) {
      const int l0 = VN * (tid + NT * q);
      const size_t row = gcell<T, KIND>(A.a, tile, l0);
      T yv[VN];
      if (KIND == KIND_A) {
        T dv[VN], zv[VN], yb[VN];
        ldg16(A.dfull + row, dv);
        ldg16(A.y + row, yb);
        if (A.z) ldg16(A.z + row, zv);
#pragma unroll
        for (int v = 0; v < VN; ++v) {
          T t = fma8(dv[v], own[VN * q + v], h[VN * q + v] + yb[v]);
          if (A.z) t = fma8(A.cz, zv[v], t);
          yv[v] = t;
          const double xo = (double)own[VN * q + v], yn = (double)t;
          sxx += xo * xo;
          sxy += xo * yn;
          syy += yn * yn;
        }
      } else {
#pragma unroll
        for (int v = 0; v < VN; ++v) yv[v] = h[VN * q + v];
      }
      // B pieces: default L2 policy, so the neighbouring tile's half of the
      // 32-byte sector joins it before the sector is written back
      if (KIND == KIND_B) st16(A.y + row, yv);
      else stcs16(A.y + row, yv);
    }
    __syncthreads();   // every thread is done with this buffer: the next prefetch may fill it
    cur ^= 1;
  }
  if constexpr (KIND == KIND_A) hv_finish_dots<T, NWARP>(A, sxx, sxy, syy, wred);
}

// A pass: CTA sums of <x,x>, <x,y>, <y,y>, then the last CTA adds them up
template <typename T, int NWARP>
__device__ __forceinline__ void hv_finish_dots(const TmaArgs<T> &A, double sxx, double sxy, double syy,
                                               double (*wred)[3]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    sxx += __shfl_xor_sync(0xffffffffu, sxx, o);
    sxy += __shfl_xor_sync(0xffffffffu, sxy, o);
    syy += __shfl_xor_sync(0xffffffffu, syy, o);
  }
  if (lane == 0) { wred[warp][0] = sxx; wred[warp][1] = sxy; wred[warp][2] = syy; }
  __syncthreads();
  double *mine = A.partials + (size_t)blockIdx.x * 3;
  if (tid < 3) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
    mine[tid] = sum;
  }
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(A.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (tid < 3) {
    double sum = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) sum += __ldcg(&A.partials[(size_t)b * 3 + tid]);
    A.dots[tid == 0 ? 0 : (tid == 1 ? 1 : 3)] = sum;
  }
  if (tid == 3) A.dots[2] = 0.0;
  if (tid == 0) *A.counter = 0u;
}

// ------------------------------------------- A pass with two thread layouts
//
// FP32, 14-bit A tiles (N = 24, 25).  The single-layout pass gathers nine of
// the 14 tile bits through shared memory in each of its two X applications.
// Here the tile is held in shared memory with the TMA 128-byte swizzle
// (float index l at l ^ (((l >> 5) & 7) << 2)), which makes two thread
// layouts conflict-free:
//   L1 ("columns"): cell l = tid + 512 j -- lanes hold bits 0..4, warps
//       bits 5..8, the 32 register slots bits 9..13;
//   L2 ("rows"): thread tid holds the 32 cells of row tid (bits 5..13 =
//       tid, bits 0..4 in registers), read and written as eight 16-byte
//       vectors whose swizzled positions differ across each quarter-warp.
// An X application then gathers only bits 5..8 (L1) and takes bits 9..13
// (L1) and 0..4 (L2) from registers; the two partial sums meet in the
// buffer the result goes to anyway:
//   t_m: L1 adds s X_{5..13} t_{m-1} into the p_m tile, L2 adds
//        s X_{0..4} t_{m-1} and completes t_m (and the dot products);
//   p_{m+1}: L2 writes d2 t_m - t_{m-1} + (2/r) X_{0..4} t_m over t_{m-1},
//        L1 adds (2/r) X_{5..13} t_m.
// About 21 four-byte shared-pipe moves per cell instead of 25.  The tile's
// row of coupling sums (k_otf_table) travels with its t_{m-1} tile, as in
// k_kpm_tma.
__device__ __forceinline__ int swz128(int l) { return l ^ (((l >> 5) & 7) << 2); }

__device__ __forceinline__ void tile_load_swz(const TmaArgs<float> &A, void *dst, const CUtensorMap *m,
                                              uint32_t tile, int g, uint64_t *bar) {
  tma_load3(dst, m, 0, (int)(tile << 9), g, bar);
  tma_load3((char *)dst + 32768, m, 0, (int)((tile << 9) + 256), g, bar);
}
__device__ __forceinline__ void wrow_load(const TmaArgs<float> &A, double *dst, uint32_t tile, uint64_t *bar) {
  bulk_load(dst, A.wtab + (size_t)tile * OTF_ROW, OTF_ROW * sizeof(double), bar);
}
__device__ __forceinline__ void tile_store_swz(const CUtensorMap *m, uint32_t tile, int g, const void *src) {
  tma_store3(m, 0, (int)(tile << 9), g, src);
  tma_store3(m, 0, (int)((tile << 9) + 256), g, (const char *)src + 32768);
}

__global__ void __launch_bounds__(512, 1)
k_kpm_tx_a(const TmaArgs<float> A, const __grid_constant__ CUtensorMap mapP,
           const __grid_constant__ CUtensorMap mapQ) {
  typedef float T;
  constexpr int NT = 512, R = 32, NWARP = 16, TB = 14;
  constexpr unsigned TILE_BYTES = 65536;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  T *const Sb0 = reinterpret_cast<T *>(smem_raw);
  T *const Sb1 = reinterpret_cast<T *>(smem_raw + TILE_BYTES);
  T *const S2 = reinterpret_cast<T *>(smem_raw + 2 * TILE_BYTES);
  __shared__ __align__(8) uint64_t bar[3];
  __shared__ double wred[NWARP][2];
  __shared__ double sV[EL_KPM_MAXN * EL_KPM_MAXN];
  __shared__ double tJ[32];        // delta + V of the register bits 0..4 of slot c
  __shared__ double cTJ[5 * NT];   // [k][tid]: couplings of the row bits 5..13 of tid to bit k
  __shared__ __align__(16) double wHt[2][OTF_ROW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ndots = A.ng * 2;
  const int nb = A.n;
  double *dacc = A.partials + (size_t)blockIdx.x * ndots;
  for (int i = tid; i < ndots; i += NT) dacc[i] = 0.0;
  for (int i = tid; i < nb * nb; i += NT) sV[i] = A.vbits[i];
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    fence_async_smem();
  }
  __syncthreads();
  // diagonal sums of the L2 layout: thread bits = row bits 5..13, slots = bits 0..4
  double cT = 0.0;
  for (int x = 0; x < 9; ++x) {
    if (!((tid >> x) & 1)) continue;
    cT += A.delta_b[5 + x];
    for (int x2 = 0; x2 < x; ++x2)
      if ((tid >> x2) & 1) cT += sV[(5 + x) * nb + 5 + x2];
  }
  for (int k = 0; k < 5; ++k) {
    double acc = 0.0;
    for (int x = 0; x < 9; ++x)
      if ((tid >> x) & 1) acc += sV[(5 + x) * nb + k];
    cTJ[k * NT + tid] = acc;
  }
  if (tid < 32) {
    double v = 0.0;
    for (int k = 0; k < 5; ++k) {
      if (!((tid >> k) & 1)) continue;
      v += A.delta_b[k];
      for (int k2 = 0; k2 < k; ++k2)
        if ((tid >> k2) & 1) v += sV[k * nb + k2];
    }
    tJ[tid] = v;
  }
  unsigned par[3] = {0u, 0u, 0u};
  int cur = 0;
  int64_t item = blockIdx.x;
  double acc_tt = 0.0, acc_tq = 0.0;
  int gacc = item_group(A, item);
  if (tid == 0 && item < A.items) {
    mbar_expect(&bar[0], TILE_BYTES + OTF_ROW * 8);
    tile_load_swz(A, Sb0, &mapQ, item_tile(A, item), gacc, &bar[0]);
    wrow_load(A, wHt[0], item_tile(A, item), &bar[0]);
  }
  const int rowq = tid & 7;    // swizzle of this thread's row (L2)
  // L1 cells tid + 512 j differ from tid only in bits 9..13, which the
  // swizzle does not read: their positions are swz(tid) + 512 j
  const int sw1 = swz128(tid);
  for (; item < A.items; item += gridDim.x) {
    const int g = item_group(A, item);
    const uint32_t tile = item_tile(A, item);
    const int64_t nxt = item + gridDim.x;
    if (g != gacc) {
      double x = acc_tt, y = acc_tq;
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) { wred[warp][0] = x; wred[warp][1] = y; }
      acc_tt = 0.0; acc_tq = 0.0;
      __syncthreads();
      if (tid < 2) {
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
        dacc[gacc * 2 + tid] += sum;
      }
      gacc = g;
    }
    T *S = cur ? Sb1 : Sb0;
    T *Sn = cur ? Sb0 : Sb1;
    if (tid == 0) bulk_wait_read<1>();   // the previous t_m store has read S2
    __syncthreads();
    if (tid == 0) {
      mbar_expect(&bar[2], TILE_BYTES);
      tile_load_swz(A, S2, &mapP, tile, g, &bar[2]);
    }
    if (cur) { mbar_wait(&bar[1], par[1], A.err); par[1] ^= 1u; }
    else { mbar_wait(&bar[0], par[0], A.err); par[0] ^= 1u; }
    // the diagonal of this thread's row-layout cells (FP64 sums, rounded
    // once), formed here so that it overlaps the first gathers
    T dvr[R];
    {
      const double *wH = wHt[cur];
      double base = cT + wH[OTF_ROW - 1];
      for (int x = 0; x < 9; ++x)
        if ((tid >> x) & 1) base += wH[5 + x];
      double u[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) u[k] = cTJ[k * NT + tid] + wH[k];
#pragma unroll
      for (int c = 0; c < R; ++c) {
        double dj = base + tJ[c];
#pragma unroll
        for (int k = 0; k < 5; ++k)
          if ((c >> k) & 1) dj += u[k];
        dvr[c] = (T)fma(A.s2, dj, A.s2c);
      }
    }

    // ---- L1: s X_{5..13} t_{m-1} added into the p_m tile
    {
      T own[R], h[R];
#pragma unroll
      for (int j = 0; j < R; ++j) { own[j] = S[sw1 + NT * j]; h[j] = 0.f; }
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        const T a = A.amp[9 + b];
#pragma unroll
        for (int j = 0; j < R; ++j) h[j] = fmaf(a, own[j ^ (1 << b)], h[j]);
      }
#pragma unroll
      for (int k = 5; k < 9; ++k) {
        const T a = A.amp[k];
        const T *Sp = S + swz128(tid ^ (1 << k));
#pragma unroll
        for (int j = 0; j < R; ++j) h[j] = fmaf(a, Sp[NT * j], h[j]);
      }
      if (tid == 0 && nxt < A.items) {
        bulk_wait_read<0>();   // the previous p_{m+1} store has read Sn
        uint64_t *bn = cur ? &bar[0] : &bar[1];
        mbar_expect(bn, TILE_BYTES + OTF_ROW * 8);
        tile_load_swz(A, Sn, &mapQ, item_tile(A, nxt), item_group(A, nxt), bn);
        wrow_load(A, wHt[cur ^ 1], item_tile(A, nxt), bn);
      }
      mbar_wait(&bar[2], par[2], A.err);
      par[2] ^= 1u;
#pragma unroll
      for (int j = 0; j < R; ++j) S2[sw1 + NT * j] = fmaf(A.s_m, h[j], S2[sw1 + NT * j]);
    }
    __syncthreads();
    // ---- L2: s X_{0..4} t_{m-1} completes t_m in this thread's row
    T o2[R], t2[R];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int off = 32 * tid + 4 * (q ^ rowq);
      const float4 ov = *reinterpret_cast<const float4 *>(S + off);
      const float4 pv = *reinterpret_cast<const float4 *>(S2 + off);
      o2[4 * q] = ov.x; o2[4 * q + 1] = ov.y; o2[4 * q + 2] = ov.z; o2[4 * q + 3] = ov.w;
      t2[4 * q] = pv.x; t2[4 * q + 1] = pv.y; t2[4 * q + 2] = pv.z; t2[4 * q + 3] = pv.w;
    }
#pragma unroll
    for (int b = 0; b < 5; ++b) {
      const T a = A.s_m * A.amp[b];
#pragma unroll
      for (int c = 0; c < R; ++c) t2[c] = fmaf(a, o2[c ^ (1 << b)], t2[c]);
    }
    T pt[2] = {0.f, 0.f}, pq[2] = {0.f, 0.f};
#pragma unroll
    for (int c = 0; c < R; ++c) {
      pt[c & 1] = fmaf(t2[c], t2[c], pt[c & 1]);
      pq[c & 1] = fmaf(t2[c], o2[c], pq[c & 1]);
    }
    if (A.mode != MODE_LAST) {
#pragma unroll
      for (int q = 0; q < 8; ++q)
        *reinterpret_cast<float4 *>(S2 + 32 * tid + 4 * (q ^ rowq)) =
            make_float4(t2[4 * q], t2[4 * q + 1], t2[4 * q + 2], t2[4 * q + 3]);
      fence_async_smem();
      __syncthreads();
      if (tid == 0) { tile_store_swz(&mapP, tile, g, S2); bulk_commit(); }
      // ---- L2: p_{m+1} partial = d2 t_m - t_{m-1} + (2/r) X_{0..4} t_m over t_{m-1}
      {
        // o2 (t_{m-1}) becomes the p_{m+1} partial in place
#pragma unroll
        for (int c = 0; c < R; ++c) o2[c] = fmaf(dvr[c], t2[c], -o2[c]);
#pragma unroll
        for (int b = 0; b < 5; ++b) {
          const T a = A.amp[b] * A.two_r;
#pragma unroll
          for (int c = 0; c < R; ++c) o2[c] = fmaf(a, t2[c ^ (1 << b)], o2[c]);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
          *reinterpret_cast<float4 *>(S + 32 * tid + 4 * (q ^ rowq)) =
              make_float4(o2[4 * q], o2[4 * q + 1], o2[4 * q + 2], o2[4 * q + 3]);
      }
      __syncthreads();
      // ---- L1: (2/r) X_{5..13} t_m added into the p_{m+1} tile
      {
        T tl[R], h[R];
#pragma unroll
        for (int j = 0; j < R; ++j) { tl[j] = S2[sw1 + NT * j]; h[j] = 0.f; }
#pragma unroll
        for (int b = 0; b < 5; ++b) {
          const T a = A.amp[9 + b];
#pragma unroll
          for (int j = 0; j < R; ++j) h[j] = fmaf(a, tl[j ^ (1 << b)], h[j]);
        }
#pragma unroll
        for (int k = 5; k < 9; ++k) {
          const T a = A.amp[k];
          const T *Sp = S2 + swz128(tid ^ (1 << k));
#pragma unroll
          for (int j = 0; j < R; ++j) h[j] = fmaf(a, Sp[NT * j], h[j]);
        }
#pragma unroll
        for (int j = 0; j < R; ++j) S[sw1 + NT * j] = fmaf(A.two_r, h[j], S[sw1 + NT * j]);
      }
      fence_async_smem();
      __syncthreads();
      if (tid == 0) { tile_store_swz(&mapQ, tile, g, S); bulk_commit(); }
    }
    acc_tt += (double)pt[0] + (double)pt[1];
    acc_tq += (double)pq[0] + (double)pq[1];
    cur ^= 1;
  }
  {
    double x = acc_tt, y = acc_tq;
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) { wred[warp][0] = x; wred[warp][1] = y; }
  }
  __syncthreads();
  if (tid < 2 && blockIdx.x < A.items) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) sum += wred[w][tid];
    dacc[gacc * 2 + tid] += sum;
  }
  if (tid == 0) bulk_wait_all();
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

// probes -> cells [probe group][row]; probe p = g*PU + lane
template <typename T>
__global__ void k_cells8(int64_t dim, int ng, uint64_t seed, int64_t probe0, int nvalid,
                         const int8_t *probes, T *out) {
  constexpr int PU = Cell<T>::PU;
  const int64_t total = dim * ng * PU;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int lane = (int)(t % PU);
    const int64_t cell = t / PU;
    const int64_t row = cell % dim;
    const int g = (int)(cell / dim);
    const int p = g * PU + lane;
    T v = 0;
    if (p < nvalid)
      v = probes ? (T)probes[(int64_t)p * dim + row]
                 : (T)el::rademacher(seed, (uint64_t)(probe0 + p), (uint64_t)row);
    out[t] = v;
  }
}

template <typename T>
__global__ void k_d2_8(int n, int64_t dim, const double *diagV, const double *delta_bits, double c,
                       double r, T *out) {
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < dim;
       row += (int64_t)gridDim.x * blockDim.x) {
    double d = diagV[row];
    for (int k = 0; k < n; ++k) if ((row >> k) & 1) d += delta_bits[k];
    out[row] = (T)(2.0 * (d - c) / r);
  }
}


PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// A map: {chunk cells (256 B), chunks, probes};
// B map: {piece cells (2^C), 2^(a-C) tiles, hb, 2^(n-a) / hb, probes}
template <typename T>
int make_maps(el_ctx *ctx, void *base, int n, int a, int ng, int hb, CUtensorMap *mA, CUtensorMap *mB,
              int C = Cell<T>::CARRY) {
  auto enc = encode_fn();
  if (!enc) return fail(ctx, EL_ECUDA, "cuTensorMapEncodeTiled unavailable");
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  constexpr int LOGCH = Cell<T>::LOGCH;
  const uint64_t dim = 1ull << n, cb = sizeof(T);
  const uint64_t e256 = 256 / cb, epc = 1ull << C;
  {
    cuuint64_t gdim[3] = {e256, dim * cb / 256, (cuuint64_t)ng};
    cuuint64_t gstr[2] = {256, dim * cb};
    cuuint32_t box[3] = {(cuuint32_t)e256, (cuuint32_t)(1u << (a - LOGCH)), 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(mA, dt, 3, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ctx, EL_ECUDA, "tensor map A encode failed (%d)", (int)r);
  }
  {
    const uint64_t hhi = (1ull << (n - a)) / (uint64_t)hb;
    cuuint64_t gdim[5] = {epc, 1ull << (a - C), (cuuint64_t)hb, hhi, (cuuint64_t)ng};
    cuuint64_t gstr[4] = {epc * cb, (1ull << a) * cb, (uint64_t)hb * (1ull << a) * cb, dim * cb};
    cuuint32_t box[5] = {(cuuint32_t)epc, 1, (cuuint32_t)hb, (cuuint32_t)hhi, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    // 256-byte L2 promotion: a 32-byte piece brings the pieces of the next
    // tiles, which the neighbouring CTAs are about to load (measured best
    // of none / 64 / 128 / 256 bytes)
    CUresult r = enc(mB, dt, 5, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ctx, EL_ECUDA, "tensor map B encode failed (%d)", (int)r);
  }
  return EL_OK;
}

// A map with the 128-byte swizzle for the two-layout A pass (FP32): rows of
// 32 floats, boxes of 256 rows (two per 14-bit tile).
int make_map_a_swz(el_ctx *ctx, void *base, int n, int ng, CUtensorMap *m) {
  auto enc = encode_fn();
  if (!enc) return fail(ctx, EL_ECUDA, "cuTensorMapEncodeTiled unavailable");
  const uint64_t dim = 1ull << n;
  cuuint64_t gdim[3] = {32, dim / 32, (cuuint64_t)ng};
  cuuint64_t gstr[2] = {128, dim * 4};
  cuuint32_t box[3] = {32, 256, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, gdim, gstr, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, EL_ECUDA, "swizzled tensor map A encode failed (%d)", (int)r);
  return EL_OK;
}

template <typename T>
int run_tma(el_ctx *ctx, el_ham *h, int nvalid_total, int chunk, uint64_t seed,
            const int8_t *probes_host, int num, double c, double r, std::vector<double> &acc) {
  constexpr int PU = Cell<T>::PU;
  constexpr int C = Cell<T>::CARRY;
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  const int ng = chunk / PU;
  const size_t vb = (size_t)dim * chunk * sizeof(T);
  // FP32: no diagonal array (formed in the kernel from V and delta, FP64);
  // FP64: the d2 array, in row order
  constexpr bool OTF = OnTheFly<T>::value;
  const size_t dbytes = OTF ? 0 : (size_t)dim * sizeof(T);
  // a: A-tile bits; the B tile has n - a + C bits; both at most 64 KB
  const int amax = sizeof(T) == 4 ? 14 : 13;
  const int a = std::min(amax, std::max((n + C + 1) / 2, n + C - amax));
  const int TBA = a, TBB = n - a + C;
  const int64_t tilesA = dim >> a, tilesB = (int64_t)1 << (a - C);
  const size_t vbits_bytes = 5120;   // EL_KPM_MAXN^2 doubles, rounded up to 256 bytes
  static_assert(EL_KPM_MAXN * EL_KPM_MAXN * sizeof(double) <= 5120, "V table slot");
  const size_t wtab_bytes = OTF ? (size_t)(tilesA + tilesB) * OTF_ROW * sizeof(double) : 0;
  char *buf = (char *)el::workspace(ctx, 6, 2 * vb + dbytes + 256 + vbits_bytes + wtab_bytes);
  if (!buf) return EL_ENOMEM;
  void *P = buf, *Q = buf + vb;
  T *d2 = OTF ? nullptr : reinterpret_cast<T *>(buf + 2 * vb);
  int *d_err = reinterpret_cast<int *>(buf + 2 * vb + dbytes);
  double *d_vbits = reinterpret_cast<double *>(buf + 2 * vb + dbytes + 256);
  double *d_wtab[2] = {nullptr, nullptr};   // [KIND_A, KIND_B]
  if constexpr (OTF) {
    d_wtab[KIND_A] = reinterpret_cast<double *>(buf + 2 * vb + dbytes + 256 + vbits_bytes);
    d_wtab[KIND_B] = d_wtab[KIND_A] + tilesA * OTF_ROW;
    EL_CUDA_TRY(ctx, el::copy(ctx, d_vbits, h->Vbits.data(), (size_t)n * n * sizeof(double),
                              cudaMemcpyHostToDevice));
    DeltaBits db;
    memset(&db, 0, sizeof db);
    for (int k = 0; k < n && k < 32; ++k) db.v[k] = h->delta[k];
    auto lg = [](int64_t t) { int l = 0; while (((int64_t)1 << l) < t) ++l; return l; };
    k_otf_table<KIND_A, C><<<el::grid_for(tilesA * OTF_ROW, 256), 256, 0, ctx->stream>>>(
        n, a, TBA, lg(tilesA), tilesA, d_vbits, db, d_wtab[KIND_A]);
    EL_LAUNCH_CHECK(ctx);
    k_otf_table<KIND_B, C><<<el::grid_for(tilesB * OTF_ROW, 256), 256, 0, ctx->stream>>>(
        n, a, TBB, lg(tilesB), tilesB, d_vbits, db, d_wtab[KIND_B]);
    EL_LAUNCH_CHECK(ctx);
  }
  const int M = (num + 1) / 2;
  double *d_dots = (double *)el::workspace(ctx, 7, (size_t)(M + 1) * chunk * 2 * sizeof(double));
  if (!d_dots) return EL_ENOMEM;
  int8_t *d_probe8 = nullptr;
  if (probes_host) {
    d_probe8 = (int8_t *)el::workspace(ctx, 2, (size_t)dim * chunk);
    if (!d_probe8) return EL_ENOMEM;
  }
  EL_CUDA_TRY(ctx, cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  if (!OTF) {
    double *d_delta = (double *)el::workspace(ctx, 8, 64 * sizeof(double));
    if (!d_delta) return EL_ENOMEM;
    EL_CUDA_TRY(ctx, el::copy(ctx, d_delta, h->delta, 64 * sizeof(double), cudaMemcpyHostToDevice));
    k_d2_8<T><<<el::grid_for(dim, 256), 256, 0, ctx->stream>>>(n, dim, h->d_diagV64, d_delta, c, r, d2);
    EL_LAUNCH_CHECK(ctx);
  }
  const int hb = (int)std::min<int64_t>(256, (int64_t)1 << (n - a));
  CUtensorMap mA[2], mB[2];   // [P buffer, Q buffer]
  int rc = make_maps<T>(ctx, P, n, a, ng, hb, &mA[0], &mB[0]);
  if (rc) return rc;
  rc = make_maps<T>(ctx, Q, n, a, ng, hb, &mA[1], &mB[1]);
  if (rc) return rc;
  const bool use_tx = sizeof(T) == 4 && TBA == 14;
  CUtensorMap mAs[2];
  if (use_tx) {
    rc = make_map_a_swz(ctx, P, n, ng, &mAs[0]);
    if (rc) return rc;
    rc = make_map_a_swz(ctx, Q, n, ng, &mAs[1]);
    if (rc) return rc;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  auto launch = [&](int kind, int mode, double s_m, int pbuf, double *dots) -> int {
    TmaArgs<T> A;
    memset(&A, 0, sizeof A);
    const int TB = kind == KIND_B ? TBB : TBA;
    A.n = n; A.a = a; A.mode = mode; A.ng = ng; A.dim = dim;
    A.tiles = kind == KIND_A ? tilesA : tilesB;
    A.items = A.tiles * ng;
    A.log_tiles = 0;
    while (((int64_t)1 << A.log_tiles) < A.tiles) ++A.log_tiles;
    A.vbits = d_vbits;
    A.wtab = d_wtab[kind];
    for (int k = 0; k < n && k < 32; ++k) A.delta_b[k] = h->delta[k];
    A.s2 = 2.0 / r;
    A.s2c = -2.0 * c / r;
    A.s_m = (T)s_m; A.two_r = (T)(2.0 / r); A.pro_alpha = (T)0.5; A.pro_beta = (T)(1.0 / r);
    for (int k = 0; k < TB && k < 16; ++k) {
      int rowbit = (kind == KIND_A) ? k : (k >= C ? a + k - C : -1);
      A.amp[k] = (T)((rowbit >= 0) ? 0.5 * h->om_re[rowbit] : 0.0);
    }
    A.d2 = d2; A.dots = dots; A.err = d_err; A.counter = ctx->d_counter;
    const int grid = (int)std::min<int64_t>(A.items, sms);
    int e = el::ensure_partials(ctx, (size_t)grid * ng * PU * 2);
    if (e) return e;
    A.partials = ctx->d_partials;
    const CUtensorMap &mp = kind == KIND_A ? mA[pbuf] : mB[pbuf];
    const CUtensorMap &mq = kind == KIND_A ? mA[pbuf ^ 1] : mB[pbuf ^ 1];
    const size_t smem = (size_t)3 * ((size_t)1 << TB) * sizeof(T);
    // FP32, large tiles: 512 threads with 2^(TB-9) cells each (one more tile
    // bit per thread in registers, one fewer shared-memory gather per cell per
    // X application) measured faster than 1024 or 256 threads.  FP64 keeps
    // 1024 threads: twice the registers per cell made 512 threads slower.
    const int lnt = (sizeof(T) == 4 && TB >= 12) ? 9 : 10;
    bool ok = false;
    if constexpr (sizeof(T) == 4) {
      if (use_tx && kind == KIND_A && mode != MODE_PROLOGUE) {
        cudaFuncSetAttribute(k_kpm_tx_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_kpm_tx_a<<<grid, 512, smem, ctx->stream>>>(A, mAs[pbuf], mAs[pbuf ^ 1]);
        EL_LAUNCH_CHECK(ctx);
        return EL_OK;
      }
    }
#define EL_TCASE(TBV, KV, LV)                                                                     \
  if (TB == TBV && kind == KV && lnt == LV) {                                                     \
    cudaFuncSetAttribute(k_kpm_tma<T, TBV, KV, LV>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                         (int)smem);                                                              \
    k_kpm_tma<T, TBV, KV, LV><<<grid, 1 << LV, smem, ctx->stream>>>(A, mp, mq);                   \
    ok = true;                                                                                    \
  }
    EL_TCASE(10, KIND_A, 10) EL_TCASE(11, KIND_A, 10) EL_TCASE(10, KIND_B, 10) EL_TCASE(11, KIND_B, 10)
    if constexpr (sizeof(T) == 4) {
      EL_TCASE(12, KIND_A, 9) EL_TCASE(13, KIND_A, 9) EL_TCASE(12, KIND_B, 9) EL_TCASE(13, KIND_B, 9)
      EL_TCASE(14, KIND_A, 9) EL_TCASE(14, KIND_B, 9)
    } else {
      EL_TCASE(12, KIND_A, 10) EL_TCASE(13, KIND_A, 10) EL_TCASE(12, KIND_B, 10) EL_TCASE(13, KIND_B, 10)
    }
#undef EL_TCASE
    if (!ok) return fail(ctx, EL_EINVAL, "TMA pass with %d tile bits not instantiated", TB);
    EL_LAUNCH_CHECK(ctx);
    return EL_OK;
  };
  std::vector<double> hd((size_t)(M + 1) * chunk * 2);
  for (int done = 0; done < nvalid_total; done += chunk) {
    const int b = std::min(chunk, nvalid_total - done);
    if (probes_host)
      EL_CUDA_TRY(ctx, el::copy(ctx, d_probe8, probes_host + (size_t)done * dim, (size_t)dim * b,
                                cudaMemcpyHostToDevice));
    // t_0 -> Q (buffer 1); the prologue writes p_1 into P (buffer 0)
    k_cells8<T><<<el::grid_for(dim * chunk, 256), 256, 0, ctx->stream>>>(
        dim, ng, seed, done, b, d_probe8, reinterpret_cast<T *>(Q));
    EL_LAUNCH_CHECK(ctx);
    int pbuf = 0;   // index of the buffer holding P this pass
    rc = launch(KIND_B, MODE_PROLOGUE, 0.0, pbuf, d_dots);
    if (rc) return rc;
    for (int m = 1; m <= M; ++m) {
      if ((m & 63) == 0 && el::cancelled(ctx)) return fail(ctx, EL_ECANCEL, "cancelled");
      const int kind = (m & 1) ? KIND_A : KIND_B;
      rc = launch(kind, m == M ? MODE_LAST : MODE_STEP, m == 1 ? 1.0 / r : 2.0 / r, pbuf,
                  d_dots + (size_t)m * chunk * 2);
      if (rc) return rc;
      pbuf ^= 1;
    }
    EL_CUDA_TRY(ctx, el::copy(ctx, hd.data(), d_dots, hd.size() * sizeof(double), cudaMemcpyDeviceToHost));
    int herr = 0;
    EL_CUDA_TRY(ctx, el::copy(ctx, &herr, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (herr) return fail(ctx, EL_ECUDA, "TMA transaction wait timed out in the KPM pass");
    for (int p = 0; p < b; ++p) {
      const double mu0 = hd[(size_t)p * 2];
      const double mu1 = hd[((size_t)chunk + p) * 2 + 1];
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

// Tiled single-vector H x for the spectral bounds (FP64, full basis).
struct el_hv_plan {
  int n = 0, a = 0, hb = 0;
  double *dfull = nullptr;          // [dim] D = diag V + sum delta n
  void *bufs[3] = {nullptr, nullptr, nullptr};
  CUtensorMap mA[3], mB[3];
  int *err = nullptr;
};

namespace el {

int hv_tiled_fill(el_ctx *ctx, el_ham *h, void *const bufs[3], int slot, el_hv_plan *P);

bool hv_tiled_eligible(const el_ham *h, int dtype) {
  return h->basis->layout == EL_LAYOUT_FULL && !h->complex_drive && h->px.empty() && !h->lossy &&
         dtype == EL_F64 && h->n >= 20 && h->n <= 25 && encode_fn() != nullptr;
}

// Plan the tiled product over the three Lanczos buffers (each dim doubles);
// the diagonal array and error flag come from workspace slot `slot`.
int hv_tiled_plan(el_ctx *ctx, el_ham *h, void *const bufs[3], int slot, el_hv_plan **out) {
  *out = nullptr;
  el_hv_plan *P = new el_hv_plan();
  const int rc = hv_tiled_fill(ctx, h, bufs, slot, P);
  if (rc) { delete P; return rc; }
  *out = P;
  return EL_OK;
}

void hv_tiled_free(el_hv_plan *P) { delete P; }

int hv_tiled_fill(el_ctx *ctx, el_ham *h, void *const bufs[3], int slot, el_hv_plan *P) {
  typedef double T;
  constexpr int C = Cell<T>::CARRY;
  const int n = h->n;
  const int64_t dim = h->basis->dim;
  char *ws = (char *)workspace(ctx, slot, (size_t)dim * sizeof(T) + 64);
  if (!ws) return EL_ENOMEM;
  P->n = n;
  P->dfull = reinterpret_cast<T *>(ws);
  P->err = reinterpret_cast<int *>(ws + (size_t)dim * sizeof(T));
  EL_CUDA_TRY(ctx, cudaMemsetAsync(P->err, 0, sizeof(int), ctx->stream));
  double *d_delta = (double *)workspace(ctx, 8, 64 * sizeof(double));
  if (!d_delta) return EL_ENOMEM;
  EL_CUDA_TRY(ctx, copy(ctx, d_delta, h->delta, 64 * sizeof(double), cudaMemcpyHostToDevice));
  // 2 (d - 0) / 2 = d exactly
  k_d2_8<T><<<grid_for(dim, 256), 256, 0, ctx->stream>>>(n, dim, h->d_diagV64, d_delta, 0.0, 2.0, P->dfull);
  EL_LAUNCH_CHECK(ctx);
  const int amax = 13;
  P->a = std::min(amax, std::max((n + C + 1) / 2, n + C - amax));
  P->hb = (int)std::min<int64_t>(256, (int64_t)1 << (n - P->a));
  for (int b = 0; b < 3; ++b) {
    P->bufs[b] = bufs[b];
    const int rc = make_maps<T>(ctx, bufs[b], n, P->a, 1, P->hb, &P->mA[b], &P->mB[b]);
    if (rc) return rc;
  }
  return EL_OK;
}

// y = H x + cz z (z may be null), dots[0..3] = <x,x>, <x,y>, 0, <y,y>;
// x, y, z are three of the planned buffers (ix, iy, iz indices; iz < 0: none).
int hv_tiled(el_ctx *ctx, el_ham *h, el_hv_plan *P, int ix, int iy, int iz, double cz, double *dots) {
  typedef double T;
  constexpr int C = Cell<T>::CARRY;
  const int n = P->n, a = P->a;
  const int64_t dim = h->basis->dim;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  for (int pass = 0; pass < 2; ++pass) {
    const int kind = pass == 0 ? KIND_B : KIND_A;   // X_B x first, then the rest and the dots
    TmaArgs<T> A;
    memset(&A, 0, sizeof A);
    const int TB = kind == KIND_B ? n - a + C : a;
    A.n = n; A.a = a; A.ng = 1; A.dim = dim;
    A.tiles = kind == KIND_A ? (dim >> a) : ((int64_t)1 << (a - C));
    A.items = A.tiles;
    for (int k = 0; k < TB && k < 16; ++k) {
      const int rowbit = (kind == KIND_A) ? k : (k >= C ? a + k - C : -1);
      A.amp[k] = (T)((rowbit >= 0) ? 0.5 * h->om_re[rowbit] : 0.0);
    }
    A.dfull = P->dfull;
    A.z = iz >= 0 ? reinterpret_cast<const T *>(P->bufs[iz]) : nullptr;
    A.cz = cz;
    A.y = reinterpret_cast<T *>(P->bufs[iy]);
    A.err = P->err;
    A.counter = ctx->d_counter;
    A.dots = dots;
    const int grid = (int)std::min<int64_t>(A.items, sms);
    int e = ensure_partials(ctx, (size_t)grid * 3);
    if (e) return e;
    A.partials = ctx->d_partials;
    const CUtensorMap &mx = kind == KIND_A ? P->mA[ix] : P->mB[ix];
    const size_t smem = (size_t)2 * ((size_t)1 << TB) * sizeof(T);
    bool ok = false;
#define EL_HCASE(TBV, KV)                                                                          \
  if (TB == TBV && kind == KV) {                                                                   \
    auto kern = k_hv_pass<T, TBV, KV, (TBV - V16<T>::LOG < 9 ? TBV - V16<T>::LOG : 9)>;            \
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);            \
    kern<<<grid, 1 << (TBV - V16<T>::LOG < 9 ? TBV - V16<T>::LOG : 9), smem, ctx->stream>>>(A, mx); \
    ok = true;                                                                                     \
  }
    EL_HCASE(11, KIND_A) EL_HCASE(12, KIND_A) EL_HCASE(13, KIND_A)
    EL_HCASE(10, KIND_B) EL_HCASE(11, KIND_B) EL_HCASE(12, KIND_B) EL_HCASE(13, KIND_B)
#undef EL_HCASE
    if (!ok) return fail(ctx, EL_EINVAL, "tiled H x with %d tile bits not instantiated", TB);
    EL_LAUNCH_CHECK(ctx);
  }
  return EL_OK;
}

int hv_tiled_error(el_ctx *ctx, el_hv_plan *P) {
  int herr = 0;
  EL_CUDA_TRY(ctx, copy(ctx, &herr, P->err, sizeof(int), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return herr ? fail(ctx, EL_ECUDA, "TMA transaction wait timed out in the tiled H x") : EL_OK;
}

bool kpm_tma_eligible(const el_ham *h, int dtype, int chunk) {
  if (h->basis->layout != EL_LAYOUT_FULL || h->complex_drive) return false;
  if (!h->px.empty()) return false;   // sigma^x channels only
  if (h->n < 20 || h->n > 25) return false;
  if (dtype != EL_F32 && dtype != EL_F64) return false;
  return chunk >= 1 && chunk <= 128;
}

int kpm_tma(el_ctx *ctx, el_ham *h, int dtype, int num, int nvec, int chunk, uint64_t seed,
            const int8_t *probes_host, double c, double r, double *mu_host) {
  std::vector<double> acc(num + 1, 0.0);
  int rc = (dtype == EL_F32)
               ? run_tma<float>(ctx, h, nvec, chunk, seed, probes_host, num, c, r, acc)
               : run_tma<double>(ctx, h, nvec, chunk, seed, probes_host, num, c, r, acc);
  if (rc) return rc;
  const double norm = 1.0 / ((double)nvec * (double)h->basis->dim);
  for (int k = 0; k <= num; ++k) mu_host[k] = acc[k] * norm;
  return EL_OK;
}

}  // namespace el
