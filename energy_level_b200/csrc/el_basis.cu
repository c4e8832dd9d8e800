// Basis construction, code expansion and ranking.
//
// Order and identity follow the reference: independent sets of the blockade
// graph in ascending code order (basis.py:24-47 independent_states, a DFS whose
// leaf order is ascending because site 0 is the most significant bit) and
// fixed-popcount codes in ascending order (matrix_free.py:12-38).
#include "el_internal.cuh"

#include <algorithm>
#include <unordered_map>

namespace {

using el::fail;

// Expand codes of the TABLE layout: one warp per allowed prefix group, lanes
// write consecutive suffixes, so stores are coalesced.
__global__ void k_codes_table(int64_t ngroups, const uint64_t *grp_prefix,
                              const int64_t *grp_off, const int32_t *grp_cls,
                              const int64_t *cls_off, const uint32_t *suf_list,
                              int L, uint64_t *codes) {
  const int lane = threadIdx.x & 31;
  int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = warp; g < ngroups; g += nwarps) {
    const uint64_t hi = grp_prefix[g] << L;
    const int64_t base = grp_off[g];
    const int32_t c = grp_cls[g];
    const int64_t s0 = cls_off[c], cnt = cls_off[c + 1] - s0;
    for (int64_t j = lane; j < cnt; j += 32) codes[base + j] = hi | suf_list[s0 + j];
  }
}

__global__ void k_codes_unrank(BasisDev B, uint64_t *codes) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.dim;
       r += (int64_t)gridDim.x * blockDim.x)
    codes[r] = el::unrank_row(B, r);
}

__global__ void k_rank(BasisDev B, const uint64_t *codes, int64_t count,
                       int64_t *ranks) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    ranks[i] = el::rank_any(B, codes[i]);
}

uint64_t fib_u64(int i) {
  uint64_t a = 0, b = 1;
  for (int k = 0; k < i; ++k) { uint64_t t = a + b; a = b; b = t; }
  return a;
}

// Build the prefix/suffix tables.  `charge` < 0: blockade constraint from
// b->adj; otherwise codes with popcount == charge.
int build_tables(el_ctx *ctx, el_basis *b, int charge, int64_t max_states) {
  const int n = b->n;
  const uint64_t cap_entries = 1ULL << 25;
  int L = (n + 1) / 2;
  for (;; --L) {
    if (L < 1 && n > 0) return fail(ctx, EL_EINVAL, "constraint too irregular for table ranking");
    const int P = n - L;
    if (P > 26) return fail(ctx, EL_EINVAL, "n=%d too large for table ranking", n);
    const uint64_t lowmask = (L >= 64) ? ~0ULL : ((1ULL << L) - 1ULL);
    const uint64_t npre = 1ULL << P, nsuf = 1ULL << L;
    // prefix pass
    std::vector<int64_t> pre_off(npre, -1);
    std::vector<int32_t> pre_cls(npre, 0);
    std::vector<uint64_t> cls_key;
    std::unordered_map<uint64_t, int> cls_id;
    std::vector<uint8_t> pre_ok(npre, 0);
    std::vector<uint64_t> pre_forbid(npre, 0);
    // prefix validity DP: ok[p] = ok[p without lowest bit] and no edge to it
    pre_ok[0] = 1;
    for (uint64_t p = 1; p < npre; ++p) {
      const int j = __builtin_ctzll(p);
      const uint64_t rest = p & (p - 1);
      const int q = L + j;  // bit position of this prefix bit
      if (charge >= 0) {
        pre_ok[p] = (__builtin_popcountll(p) <= charge);
      } else {
        pre_ok[p] = pre_ok[rest] && !((rest << L) & b->adj[q]);
        pre_forbid[p] = pre_forbid[rest] | (b->adj[q] & lowmask);
      }
    }
    bool too_many = false;
    for (uint64_t p = 0; p < npre; ++p) {
      if (!pre_ok[p]) continue;
      uint64_t key = (charge >= 0) ? (uint64_t)__builtin_popcountll(p) : pre_forbid[p];
      auto it = cls_id.find(key);
      int c;
      if (it == cls_id.end()) {
        c = (int)cls_key.size();
        cls_id.emplace(key, c);
        cls_key.push_back(key);
        if ((uint64_t)cls_key.size() * nsuf > cap_entries) { too_many = true; break; }
      } else {
        c = it->second;
      }
      pre_cls[p] = c;
    }
    if (too_many) continue;
    const int ncls = (int)cls_key.size();
    // suffix validity for the blockade: internal independence DP
    std::vector<uint8_t> suf_ok(nsuf, 1);
    if (charge < 0) {
      for (uint64_t s = 1; s < nsuf; ++s) {
        const int j = __builtin_ctzll(s);
        const uint64_t rest = s & (s - 1);
        suf_ok[s] = suf_ok[rest] && !(rest & b->adj[j]);
      }
    }
    std::vector<int32_t> suf_rank((size_t)ncls * nsuf, -1);
    std::vector<int64_t> cls_off(ncls + 1, 0);
    std::vector<uint32_t> suf_list;
    for (int c = 0; c < ncls; ++c) {
      cls_off[c] = (int64_t)suf_list.size();
      int32_t r = 0;
      for (uint64_t s = 0; s < nsuf; ++s) {
        bool ok;
        if (charge >= 0) ok = (int)__builtin_popcountll(s) + (int)cls_key[c] == charge;
        else ok = suf_ok[s] && !(s & cls_key[c]);
        if (ok) {
          suf_rank[(size_t)c * nsuf + s] = r++;
          suf_list.push_back((uint32_t)s);
        }
      }
    }
    cls_off[ncls] = (int64_t)suf_list.size();
    int64_t off = 0;
    for (uint64_t p = 0; p < npre; ++p) {
      if (!pre_ok[p]) continue;
      const int c = pre_cls[p];
      const int64_t cnt = cls_off[c + 1] - cls_off[c];
      if (cnt == 0) { pre_ok[p] = 0; continue; }
      pre_off[p] = off;
      off += cnt;
    }
    if (max_states > 0 && off > max_states)
      return fail(ctx, EL_EINVAL, "restricted basis dimension %lld exceeds max_states=%lld",
                  (long long)off, (long long)max_states);
    if (off == 0) return fail(ctx, EL_EINVAL, "empty basis");
    b->L = L;
    b->ncls = ncls;
    b->dim = off;
    b->h_pre_off.swap(pre_off);
    b->h_pre_cls.swap(pre_cls);
    b->h_suf_rank.swap(suf_rank);
    b->h_suf_list.swap(suf_list);
    b->h_cls_off.swap(cls_off);
    return EL_OK;
  }
}

int upload_tables(el_ctx *ctx, el_basis *b) {
  const size_t npre = b->h_pre_off.size();
  EL_CUDA_TRY(ctx, cudaMalloc(&b->d_pre_off, npre * sizeof(int64_t)));
  EL_CUDA_TRY(ctx, cudaMalloc(&b->d_pre_cls, npre * sizeof(int32_t)));
  EL_CUDA_TRY(ctx, cudaMalloc(&b->d_suf_rank, b->h_suf_rank.size() * sizeof(int32_t)));
  EL_CUDA_TRY(ctx, el::copy(ctx, b->d_pre_off, b->h_pre_off.data(), npre * sizeof(int64_t), cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, b->d_pre_cls, b->h_pre_cls.data(), npre * sizeof(int32_t), cudaMemcpyHostToDevice));
  EL_CUDA_TRY(ctx, el::copy(ctx, b->d_suf_rank, b->h_suf_rank.data(), b->h_suf_rank.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  // groups for the code expansion
  std::vector<uint64_t> gp;
  std::vector<int64_t> go;
  std::vector<int32_t> gc;
  for (size_t p = 0; p < npre; ++p)
    if (b->h_pre_off[p] >= 0) { gp.push_back(p); go.push_back(b->h_pre_off[p]); gc.push_back(b->h_pre_cls[p]); }
  uint64_t *d_gp = nullptr; int64_t *d_go = nullptr, *d_co = nullptr; int32_t *d_gc = nullptr;
  uint32_t *d_sl = nullptr;
  int rc = EL_OK;
  cudaError_t e = cudaSuccess;
  do {
    if ((e = cudaMalloc(&b->d_codes, (size_t)b->dim * sizeof(uint64_t))) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_gp, gp.size() * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_go, go.size() * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_gc, gc.size() * 4)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_co, b->h_cls_off.size() * 8)) != cudaSuccess) break;
    if ((e = cudaMalloc(&d_sl, std::max<size_t>(1, b->h_suf_list.size()) * 4)) != cudaSuccess) break;
    el::copy(ctx, d_gp, gp.data(), gp.size() * 8, cudaMemcpyHostToDevice);
    el::copy(ctx, d_go, go.data(), go.size() * 8, cudaMemcpyHostToDevice);
    el::copy(ctx, d_gc, gc.data(), gc.size() * 4, cudaMemcpyHostToDevice);
    el::copy(ctx, d_co, b->h_cls_off.data(), b->h_cls_off.size() * 8, cudaMemcpyHostToDevice);
    el::copy(ctx, d_sl, b->h_suf_list.data(), b->h_suf_list.size() * 4, cudaMemcpyHostToDevice);
    const int64_t ng = (int64_t)gp.size();
    int grid = el::grid_for(ng * 32, 256);
    k_codes_table<<<grid, 256, 0, ctx->stream>>>(ng, d_gp, d_go, d_gc, d_co, d_sl, b->L, b->d_codes);
    ctx->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  } while (0);
  if (e != cudaSuccess) rc = el::cuda_fail(ctx, e, "table upload");
  cudaFree(d_gp); cudaFree(d_go); cudaFree(d_gc); cudaFree(d_co); cudaFree(d_sl);
  return rc;
}

}  // namespace

extern "C" {

int el_basis_build(el_ctx *ctx, int n, const int32_t *edges, int n_edges,
                   int kind, int k, int64_t max_states, el_basis **out) {
  if (!ctx || !out) return EL_EINVAL;
  *out = nullptr;
  if (n < 1 || n > 63) return fail(ctx, EL_EINVAL, "n must be in [1, 63], got %d", n);
  if (kind != EL_BASIS_FULL && kind != EL_BASIS_BLOCKADE && kind != EL_BASIS_CHARGE)
    return fail(ctx, EL_EINVAL, "unknown basis kind %d", kind);
  if (n_edges < 0 || (n_edges > 0 && !edges)) return fail(ctx, EL_EINVAL, "bad edge list");
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  el_basis *b = new el_basis();
  b->n = n;
  b->kind = kind;
  b->device = ctx->device;
  memset(b->adj, 0, sizeof b->adj);
  int rc = EL_OK;
  if (kind == EL_BASIS_BLOCKADE) {
    // validate + deduplicate like basis.py:12-21
    std::vector<std::pair<int, int>> es;
    for (int e = 0; e < n_edges; ++e) {
      int i = edges[2 * e], j = edges[2 * e + 1];
      if (i < 0 || j < 0 || i >= n || j >= n || i == j) {
        delete b;
        return fail(ctx, EL_EINVAL, "blockade edge out of range or self loop: (%d, %d)", i, j);
      }
      if (i > j) std::swap(i, j);
      es.emplace_back(i, j);
    }
    std::sort(es.begin(), es.end());
    es.erase(std::unique(es.begin(), es.end()), es.end());
    for (auto &e : es) {
      const int qi = n - 1 - e.first, qj = n - 1 - e.second;
      b->adj[qi] |= 1ULL << qj;
      b->adj[qj] |= 1ULL << qi;
    }
    bool chain = (int)es.size() == n - 1 && n >= 2;
    for (int i = 0; chain && i < n - 1; ++i) chain = es[i] == std::make_pair(i, i + 1);
    bool ring = false;
    if (!chain && n >= 3 && (int)es.size() == n) {
      ring = true;
      // sorted order: (0,1), (0,n-1), (1,2), ..., (n-2,n-1)
      std::vector<std::pair<int, int>> want;
      for (int i = 0; i < n - 1; ++i) want.emplace_back(i, i + 1);
      want.emplace_back(0, n - 1);
      std::sort(want.begin(), want.end());
      ring = (want == es);
    }
    if (es.empty()) {
      b->layout = EL_LAYOUT_FULL;
    } else if (chain) {
      b->layout = EL_LAYOUT_CHAIN;
    } else if (ring) {
      b->layout = EL_LAYOUT_RING;
    } else {
      b->layout = EL_LAYOUT_TABLE;
    }
    if (b->layout == EL_LAYOUT_CHAIN) b->dim = (n + 2 <= 93) ? (int64_t)fib_u64(n + 2) : -1;
    if (b->layout == EL_LAYOUT_RING) b->dim = (int64_t)(fib_u64(n + 1) + fib_u64(n - 1));
    if (b->layout == EL_LAYOUT_FULL) {
      if (n > 34) { delete b; return fail(ctx, EL_EINVAL, "full basis limited to n <= 34"); }
      b->dim = 1LL << n;
    }
    if (b->layout == EL_LAYOUT_TABLE) {
      rc = build_tables(ctx, b, -1, max_states);
    } else if (max_states > 0 && b->dim > max_states) {
      rc = fail(ctx, EL_EINVAL, "restricted basis dimension %lld exceeds max_states=%lld",
                (long long)b->dim, (long long)max_states);
    }
  } else if (kind == EL_BASIS_CHARGE) {
    if (k < 0 || k > n) { delete b; return fail(ctx, EL_EINVAL, "charge sector k=%d out of [0, %d]", k, n); }
    b->layout = EL_LAYOUT_TABLE;
    rc = build_tables(ctx, b, k, max_states);
  } else {
    if (n > 34) { delete b; return fail(ctx, EL_EINVAL, "full basis limited to n <= 34"); }
    b->layout = EL_LAYOUT_FULL;
    b->dim = 1LL << n;
  }
  if (rc == EL_OK && b->dim > (1LL << 34))
    rc = fail(ctx, EL_EINVAL, "basis dimension %lld too large", (long long)b->dim);
  if (rc == EL_OK && b->layout == EL_LAYOUT_TABLE) rc = upload_tables(ctx, b);
  if (rc != EL_OK) {
    el_basis_destroy(b);
    return rc;
  }
  *out = b;
  return EL_OK;
}

int el_basis_info(const el_basis *b, int64_t *dim, int *layout) {
  if (!b) return EL_EINVAL;
  if (dim) *dim = b->dim;
  if (layout) *layout = b->layout;
  return EL_OK;
}

int el_basis_codes(el_ctx *ctx, el_basis *b, uint64_t *codes) {
  if (!ctx || !b || !codes) return EL_EINVAL;
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (b->layout == EL_LAYOUT_TABLE) {
    EL_CUDA_TRY(ctx, el::copy(ctx, codes, b->d_codes, (size_t)b->dim * 8, cudaMemcpyDeviceToDevice));
    return EL_OK;
  }
  BasisDev B = el::basis_dev(b);
  k_codes_unrank<<<el::grid_for(b->dim, 256), 256, 0, ctx->stream>>>(B, codes);
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int el_basis_rank(el_ctx *ctx, el_basis *b, const uint64_t *codes, int64_t count,
                  int64_t *ranks) {
  if (!ctx || !b || (count > 0 && (!codes || !ranks)) || count < 0) return EL_EINVAL;
  if (count == 0) return EL_OK;
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  BasisDev B = el::basis_dev(b);
  k_rank<<<el::grid_for(count, 256), 256, 0, ctx->stream>>>(B, codes, count, ranks);
  EL_LAUNCH_CHECK(ctx);
  return EL_OK;
}

int el_basis_destroy(el_basis *b) {
  if (!b) return EL_OK;
  cudaSetDevice(b->device);
  if (b->d_pre_off) cudaFree(b->d_pre_off);
  if (b->d_pre_cls) cudaFree(b->d_pre_cls);
  if (b->d_suf_rank) cudaFree(b->d_suf_rank);
  if (b->d_codes) cudaFree(b->d_codes);
  delete b;
  return EL_OK;
}

}  // extern "C"
