// Spin observables of a state on the device: the per-site and pair
// expectations that the evolution reports at every output time.
//
// For a state v on the basis of `ham` one launch computes, per requested
// item, three FP64 sums over the rows s of the basis (p = |v_s|^2):
//   norm item         sum p
//   site item i       <n_i>      = sum_{s_i = r} p
//                     <sigma-_i> = sum_{s_i = g} conj(v_s) v_{s + i}   (flip target in the basis)
//   pair item (i, j)  <n_i n_j>  = sum_{s_i = s_j = r} p
//                     <sigma+_i sigma-_j> = sum_{s_i = g, s_j = r} conj(v_t) v_s,
//                                           t = s with i -> r, j -> g (in the basis)
//   Pauli item        <P> = sum_s conj(v_t) c(s) v_s for P = prod of sigma^x/y/z
//                     on distinct sites, t = s ^ (x and y sites), c(s) = i^e with
//                     e = #(y on g) + 3 #(y on r) + 2 #(z on r)  (mod 4), since
//                     sigma^y|g> = i|r>, sigma^y|r> = -i|g>, sigma^z|r> = -|r>
// which are observables.py:117-159 spin_observables (full basis) and
// observables.py:162-205 spin_observables_basis (restricted basis: targets
// outside the basis drop out), the <n_i n_j> of observables.py:40-47
// corr_matrix and PauliPlan.expect (observables.py:486-622) for the Pauli
// strings.  Items come in groups of eight, one group per blockIdx.y; a
// thread keeps the 24 sums of its group in registers over a grid-stride
// loop of rows, so v is read once per group and every flip target once per
// item.  Block sums go to per-block partials and a second kernel adds them
// in a fixed order (deterministic results).
#include "el_internal.cuh"

#include <vector>

namespace {

using el::fail;

constexpr int kGroup = 6;   // items per launch column: 6 x 3 FP64 sums fit the registers of 2 CTAs per SM
enum { kNoItem = 0, kNormItem, kSiteItem, kPairItem, kPauliItem };

struct ObsItem {
  int kind;
  int bi, bj;         // bit positions of sites i (site and pair items) and j (pair items)
  int pad_;
  uint64_t fm, ym, zm;  // Pauli item: flipped bits (x and y), y bits, z bits
};

template <typename S, bool C>
__device__ __forceinline__ void load_amp(const S *__restrict__ psi, int64_t r, double &re, double &im) {
  if constexpr (C) { re = (double)psi[2 * r]; im = (double)psi[2 * r + 1]; }
  else { re = (double)psi[r]; im = 0.0; }
}

template <typename S, bool C>
__global__ void __launch_bounds__(256, 2) k_obs_items(BasisDev B, const S *__restrict__ psi,
                                                   const ObsItem *__restrict__ items,
                                                   double *__restrict__ partials, int K) {
  __shared__ double red[8][kGroup * 3];
  __shared__ ObsItem it[kGroup];
  const int g = blockIdx.y;
  if (threadIdx.x < kGroup) it[threadIdx.x] = items[g * kGroup + threadIdx.x];
  __syncthreads();
  double acc[kGroup][3];
#pragma unroll
  for (int q = 0; q < kGroup; ++q) acc[q][0] = acc[q][1] = acc[q][2] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.dim; r += stride) {
    const uint64_t code = el::unrank_row(B, r);
    double re, im;
    load_amp<S, C>(psi, r, re, im);
    const double p = re * re + im * im;
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int kind = it[q].kind;
      if (kind == kNoItem) continue;
      if (kind == kNormItem) { acc[q][0] += p; continue; }
      if (kind == kPauliItem) {
        const uint64_t ym = it[q].ym;
        const int64_t t = it[q].fm ? el::rank_any(B, code ^ it[q].fm) : r;
        if (t >= 0) {
          const int e = (__popcll(ym & ~code) + 3 * __popcll(ym & code) + 2 * __popcll(it[q].zm & code)) & 3;
          double wr, wi;
          load_amp<S, C>(psi, t, wr, wi);
          // conj(v_t) v_s, then times i^e
          const double ar = wr * re + wi * im, ai = wr * im - wi * re;
          const double cr = (e == 0) ? ar : (e == 1) ? -ai : (e == 2) ? -ar : ai;
          const double ci = (e == 0) ? ai : (e == 1) ? ar : (e == 2) ? -ai : -ar;
          acc[q][1] += cr;
          acc[q][2] += ci;
        }
        continue;
      }
      const int bi = it[q].bi, bj = it[q].bj;
      const bool si = (code >> bi) & 1ULL;
      if (kind == kSiteItem) {
        if (si) { acc[q][0] += p; continue; }
        const int64_t t = el::flip_target(B, code, r, bi);
        if (t >= 0) {
          double wr, wi;
          load_amp<S, C>(psi, t, wr, wi);
          acc[q][1] += re * wr + im * wi;   // conj(v_s) v_t
          acc[q][2] += re * wi - im * wr;
        }
        continue;
      }
      const bool sj = (code >> bj) & 1ULL;
      if (si && sj) acc[q][0] += p;
      if (!si && sj) {
        // on chain / ring sectors: clear bit j (which keeps the state in the
        // sector), then set bit i -- two O(1) single flips instead of a
        // re-rank; other layouts rank the target directly (on a
        // fixed-excitation sector the intermediate state is outside it)
        int64_t t;
        if (B.layout == EL_LAYOUT_CHAIN || B.layout == EL_LAYOUT_RING) {
          const int64_t t1 = el::flip_target(B, code, r, bj);
          t = (t1 >= 0) ? el::flip_target(B, code ^ (1ULL << bj), t1, bi) : -1;
        } else {
          t = el::rank_any(B, code ^ ((1ULL << bi) | (1ULL << bj)));
        }
        if (t >= 0) {
          double wr, wi;
          load_amp<S, C>(psi, t, wr, wi);
          acc[q][1] += wr * re + wi * im;   // conj(v_t) v_s
          acc[q][2] += wr * im - wi * re;
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kGroup; ++q) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double v = acc[q][c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[warp][q * 3 + c] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < kGroup * 3) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    partials[(size_t)blockIdx.x * K + (size_t)g * kGroup * 3 + threadIdx.x] = s;
  }
}

__global__ void k_obs_sum(int nparts, int K, const double *__restrict__ partials, double *__restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += partials[(size_t)b * K + k];
    out[k] = s;
  }
}

ObsItem item(int kind, int bi, int bj) {
  ObsItem it;
  memset(&it, 0, sizeof it);
  it.kind = kind;
  it.bi = bi;
  it.bj = bj;
  return it;
}

// Evaluate `items` (padded here to whole groups) on psi; out[3 q .. 3 q + 2]
// receives the three sums of item q.
int run_items(el_ctx *ctx, el_ham *h, int dtype, const void *psi, std::vector<ObsItem> &items,
              std::vector<double> &out) {
  while (items.size() % kGroup) items.push_back(item(kNoItem, 0, 0));
  const int ngroups = (int)(items.size() / kGroup);
  if (ngroups > 65535) return fail(ctx, EL_EINVAL, "too many observables (%zu)", items.size());
  const int K = ngroups * kGroup * 3;
  BasisDev B = el::basis_dev(h->basis);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  int gx = el::grid_for(B.dim, 256);
  if (gx > 2 * sms) gx = 2 * sms;
  ObsItem *d_items = (ObsItem *)el::workspace(ctx, 9, items.size() * sizeof(ObsItem));
  double *d_out = (double *)el::workspace(ctx, 10, (size_t)K * sizeof(double));
  if (!d_items || !d_out) return EL_ENOMEM;
  int rc = el::ensure_partials(ctx, (size_t)gx * K);
  if (rc) return rc;
  EL_CUDA_TRY(ctx, el::copy(ctx, d_items, items.data(), items.size() * sizeof(ObsItem), cudaMemcpyHostToDevice));
  const dim3 grid(gx, ngroups);
  switch (dtype) {
    case EL_F32: k_obs_items<float, false><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, d_items, ctx->d_partials, K); break;
    case EL_F64: k_obs_items<double, false><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, d_items, ctx->d_partials, K); break;
    case EL_C64: k_obs_items<float, true><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, d_items, ctx->d_partials, K); break;
    case EL_C128: k_obs_items<double, true><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, d_items, ctx->d_partials, K); break;
    default: return fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  }
  EL_LAUNCH_CHECK(ctx);
  k_obs_sum<<<(K + 255) / 256, 256, 0, ctx->stream>>>(gx, K, ctx->d_partials, d_out);
  EL_LAUNCH_CHECK(ctx);
  out.assign(K, 0.0);
  EL_CUDA_TRY(ctx, el::copy(ctx, out.data(), d_out, (size_t)K * sizeof(double), cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return EL_OK;
}

}  // namespace

extern "C" int el_spin_observables(el_ctx *ctx, el_ham *h, int dtype, const void *psi,
                                   int n_pairs, const int32_t *pi, const int32_t *pj,
                                   double *n_site, double *norm, double *sigma_minus,
                                   double *nn, double *xy) {
  if (!ctx || !h || !psi) return EL_EINVAL;
  const int n = h->n;
  if (n_pairs < 0 || (n_pairs > 0 && (!pi || !pj))) return fail(ctx, EL_EINVAL, "bad pair list");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<ObsItem> items;
  items.push_back(item(kNormItem, 0, 0));
  for (int i = 0; i < n; ++i) items.push_back(item(kSiteItem, n - 1 - i, 0));
  for (int p = 0; p < n_pairs; ++p) {
    const int i = pi[p], j = pj[p];
    if (i < 0 || j < 0 || i >= n || j >= n || i == j)
      return fail(ctx, EL_EINVAL, "pair %d: bad sites (%d, %d)", p, i, j);
    items.push_back(item(kPairItem, n - 1 - i, n - 1 - j));
  }
  std::vector<double> out;
  int rc = run_items(ctx, h, dtype, psi, items, out);
  if (rc) return rc;
  if (norm) *norm = out[0];
  for (int i = 0; i < n; ++i) {
    const double *o = &out[3 * (1 + i)];
    if (n_site) n_site[i] = o[0];
    if (sigma_minus) { sigma_minus[2 * i] = o[1]; sigma_minus[2 * i + 1] = o[2]; }
  }
  for (int p = 0; p < n_pairs; ++p) {
    const double *o = &out[3 * (1 + n + p)];
    if (nn) nn[p] = o[0];
    if (xy) { xy[2 * p] = o[1]; xy[2 * p + 1] = o[2]; }
  }
  return EL_OK;
}

extern "C" int el_pauli_expect(el_ctx *ctx, el_ham *h, int dtype, const void *psi, int n_strings,
                               const int32_t *offsets, const int32_t *sites, const char *axes,
                               double *out_host) {
  if (!ctx || !h || !psi || (n_strings > 0 && (!offsets || !sites || !axes || !out_host))) return EL_EINVAL;
  if (n_strings < 0) return fail(ctx, EL_EINVAL, "n_strings must be >= 0");
  if (n_strings == 0) return EL_OK;
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int n = h->n;
  std::vector<ObsItem> items;
  for (int q = 0; q < n_strings; ++q) {
    ObsItem it = item(kPauliItem, 0, 0);
    uint64_t used = 0;
    if (offsets[q + 1] <= offsets[q]) return fail(ctx, EL_EINVAL, "Pauli string %d is empty", q);
    for (int k = offsets[q]; k < offsets[q + 1]; ++k) {
      const int site = sites[k];
      if (site < 0 || site >= n) return fail(ctx, EL_EINVAL, "Pauli string %d: site %d out of range", q, site);
      const uint64_t bit = 1ULL << (n - 1 - site);
      if (used & bit) return fail(ctx, EL_EINVAL, "Pauli string %d: site %d appears twice", q, site);
      used |= bit;
      switch (axes[k]) {
        case 'x': it.fm |= bit; break;
        case 'y': it.fm |= bit; it.ym |= bit; break;
        case 'z': it.zm |= bit; break;
        default: return fail(ctx, EL_EINVAL, "Pauli string %d: axis must be x, y or z", q);
      }
    }
    items.push_back(it);
  }
  std::vector<double> out;
  int rc = run_items(ctx, h, dtype, psi, items, out);
  if (rc) return rc;
  for (int q = 0; q < n_strings; ++q) {
    out_host[2 * q] = out[3 * q + 1];
    out_host[2 * q + 1] = out[3 * q + 2];
  }
  return EL_OK;
}
