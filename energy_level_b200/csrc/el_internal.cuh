// Internal declarations shared by the translation units of libel_b200.so.
//
// Layout of a basis on the device (all code words are uint64, bit position
// k = n-1-site, so site 0 is the most significant bit as in the reference's
// basis.py:6-9):
//   FULL   rank(code) = code
//   CHAIN  nearest-neighbour path; the ascending independent sets are ranked by
//          rank(c) = sum_{k set} F(k+2)  (Zeckendorf; F(1)=F(2)=1)
//   RING   nearest-neighbour cycle; codes with the top bit clear rank as a
//          path of n-1 sites, codes with it set follow with weights F(k+1)
//   TABLE  any constraint: code = (prefix << L) | suffix, a prefix table gives
//          the group offset and constraint class, a per-class suffix table the
//          rank inside the group.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <cstring>
#include <cstdio>
#include <cmath>

#include "../../include/energy_level_b200.h"

#define EL_MAX_SITES 64

struct el_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  const volatile int32_t *cancel = nullptr;
  int64_t launches = 0;
  int64_t h2d_bytes = 0;   // host->device bytes copied by the library
  int64_t d2h_bytes = 0;   // device->host bytes copied by the library
  // deterministic reduction scratch: per-block partials + completion counter
  double *d_partials = nullptr;
  size_t partial_cap = 0;  // doubles
  unsigned int *d_counter = nullptr;
  // small device result area and pinned host mirror
  double *d_scalars = nullptr;   // EL_SCALARS doubles
  double *h_scalars = nullptr;   // pinned
  // cached device workspace slots (grown on demand, freed with the context)
  void *ws_ptr[16] = {nullptr};
  size_t ws_size[16] = {0};
  int adjoint_mode = 0;    // EL_ADJ_*: how el_adjoint_pulse schedules its sweeps
};
#define EL_SCALARS 4096

struct el_basis {
  int kind = 0;     // EL_BASIS_*
  int layout = 0;   // EL_LAYOUT_*
  int n = 0;
  int64_t dim = 0;
  uint64_t adj[EL_MAX_SITES];  // by bit position: bit positions adjacent to it
  // TABLE layout
  int L = 0;        // suffix bits
  int ncls = 0;
  std::vector<int64_t> h_pre_off;   // [2^P], -1 if the prefix is not allowed
  std::vector<int32_t> h_pre_cls;   // [2^P]
  std::vector<int32_t> h_suf_rank;  // [ncls << L], -1 if not allowed
  std::vector<uint32_t> h_suf_list; // concatenated ascending allowed suffixes
  std::vector<int64_t> h_cls_off;   // [ncls+1] offsets into h_suf_list
  int64_t *d_pre_off = nullptr;
  int32_t *d_pre_cls = nullptr;
  int32_t *d_suf_rank = nullptr;
  uint64_t *d_codes = nullptr;      // [dim] (TABLE layout only)
  int device = 0;
};

// Basis description passed to kernels by value.
struct BasisDev {
  int layout;
  int n;
  int L;
  int pad_;
  int64_t dim;
  const int64_t *pre_off;
  const int32_t *pre_cls;
  const int32_t *suf_rank;
  const uint64_t *codes;
  uint64_t adj[EL_MAX_SITES];
  uint64_t fib[EL_MAX_SITES + 3];  // fib[i] = F(i), F(1)=F(2)=1
};

// One two-site exchange channel pair (bit positions bi, bj of sites i, j):
// J moves an excitation between the sites, A creates or removes both.
struct ExPair {
  int32_t bi, bj;
  double jre, jim;   // J: amplitude conj(J) into a row with (i, j) = (g, r), J into (r, g)
  double are, aim;   // A: amplitude A into a row with (r, r), conj(A) into (g, g)
};

struct el_hv_plan;   // el_kpm_tma.cu

struct el_ham {
  el_basis *basis = nullptr;
  int n = 0;
  // per bit position k (site n-1-k)
  double om_re[EL_MAX_SITES];
  double om_im[EL_MAX_SITES];
  double delta[EL_MAX_SITES];
  std::vector<double> Vbits;   // [n*n] by bit positions, symmetric
  double *d_diagV64 = nullptr;  // per-row sum of V_ij n_i n_j (FP64)
  float *d_diagV32 = nullptr;   // FP32 copy, built on first use
  // exchange channels (I2 J, I3 A); empty for the Omega/delta/V model
  std::vector<ExPair> px;
  ExPair *d_px = nullptr;
  // the same channels for the hop kernel: J as a table hop[a][b] (bit
  // positions, a row with bit a = r and bit b = g gains hop[a][b] x[row with
  // the excitation moved from a to b]; re/im, n*n each) and the pairs with a
  // nonzero A in their own list
  double *d_hop = nullptr;     // [2][n*n]
  ExPair *d_pxA = nullptr;
  int npxA = 0;
  bool drive_complex = false;     // Omega has an imaginary part
  bool px_complex = false;        // some J or A has an imaginary part
  // loss: imaginary diagonal -gamma_i/2 (in the evolution's units) per bit
  double loss[EL_MAX_SITES];
  bool lossy = false;             // some gamma != 0: H is not Hermitian
  bool complex_drive = false;     // H is complex: drive_complex || px_complex || lossy
};

// ---------------------------------------------------------------- helpers

namespace el {

int fail(el_ctx *ctx, int code, const char *fmt, ...);
int cuda_fail(el_ctx *ctx, cudaError_t e, const char *where);
bool cancelled(el_ctx *ctx);
int ensure_partials(el_ctx *ctx, size_t doubles);
BasisDev basis_dev(const el_basis *b);
int ham_diag32(el_ctx *ctx, el_ham *h);
int dtype_size(int dtype);
int grid_for(int64_t work, int block);
// Cached device workspace `slot` of at least `bytes` bytes (nullptr on failure,
// with the error recorded on ctx).
void *workspace(el_ctx *ctx, int slot, size_t bytes);

// Asynchronous copy on the context stream, counting host<->device bytes.
inline cudaError_t copy(el_ctx *ctx, void *dst, const void *src, size_t bytes,
                        cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice) ctx->h2d_bytes += (int64_t)bytes;
  else if (kind == cudaMemcpyDeviceToHost) ctx->d2h_bytes += (int64_t)bytes;
  return cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream);
}

#define EL_CUDA_TRY(ctx, expr)                                   \
  do {                                                           \
    cudaError_t e_ = (expr);                                     \
    if (e_ != cudaSuccess) return el::cuda_fail(ctx, e_, #expr); \
  } while (0)

#define EL_LAUNCH_CHECK(ctx)                                          \
  do {                                                                \
    (ctx)->launches++;                                                \
    cudaError_t e_ = cudaGetLastError();                              \
    if (e_ != cudaSuccess) return el::cuda_fail(ctx, e_, "launch"); \
  } while (0)

// ------------------------------------------------------- device helpers

__host__ __device__ inline uint64_t splitmix64(uint64_t x) {
  // SplitMix64 finaliser (Steele, Lea, Flood 2014; constants from Vigna's
  // public-domain reference).
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// Counter-based value for (seed, stream, index): independent of launch shape.
__host__ __device__ inline uint64_t counter_hash(uint64_t seed, uint64_t stream,
                                                 uint64_t index) {
  return splitmix64(splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ULL)) + index);
}

// Rademacher +-1 for probe `p`, row `r`.
__host__ __device__ inline int rademacher(uint64_t seed, uint64_t p, uint64_t r) {
  return (counter_hash(seed, p + 1, r) >> 63) ? -1 : 1;
}

// Row -> code and code -> rank for each layout --------------------------------

__device__ __forceinline__ uint64_t unrank_row(const BasisDev &B, int64_t row) {
  if (B.layout == EL_LAYOUT_FULL) return (uint64_t)row;
  if (B.layout == EL_LAYOUT_TABLE) return B.codes[row];
  uint64_t r = (uint64_t)row, c = 0;
  const int n = B.n;
  if (B.layout == EL_LAYOUT_CHAIN) {
    for (int k = n - 1; k >= 0; --k) {
      uint64_t w = B.fib[k + 2];
      if (r >= w) { c |= 1ULL << k; r -= w; }
    }
    return c;
  }
  // RING
  if (r < B.fib[n + 1]) {
    for (int k = n - 2; k >= 0; --k) {
      uint64_t w = B.fib[k + 2];
      if (r >= w) { c |= 1ULL << k; r -= w; }
    }
    return c;
  }
  r -= B.fib[n + 1];
  c = 1ULL << (n - 1);
  for (int k = n - 3; k >= 1; --k) {
    uint64_t w = B.fib[k + 1];
    if (r >= w) { c |= 1ULL << k; r -= w; }
  }
  return c;
}

// Full rank of an allowed code (no validity check for CHAIN/RING).
__device__ __forceinline__ int64_t rank_code_ring(const BasisDev &B, uint64_t c) {
  const int n = B.n;
  int64_t r = 0;
  if ((c >> (n - 1)) & 1ULL) {
    r = (int64_t)B.fib[n + 1];
    uint64_t m = c & ~(1ULL << (n - 1));
    while (m) { int k = __ffsll((long long)m) - 1; r += (int64_t)B.fib[k + 1]; m &= m - 1; }
  } else {
    uint64_t m = c;
    while (m) { int k = __ffsll((long long)m) - 1; r += (int64_t)B.fib[k + 2]; m &= m - 1; }
  }
  return r;
}

// Rank of any code: -1 if the code is not in the basis.
__device__ __forceinline__ int64_t rank_any(const BasisDev &B, uint64_t c) {
  const int n = B.n;
  if (n < 64 && (c >> n) != 0) return -1;
  if (B.layout == EL_LAYOUT_FULL) return (int64_t)c;
  if (B.layout == EL_LAYOUT_TABLE) {
    uint64_t p = c >> B.L, s = c & ((1ULL << B.L) - 1ULL);
    int64_t off = B.pre_off[p];
    if (off < 0) return -1;
    int32_t rr = B.suf_rank[((uint64_t)B.pre_cls[p] << B.L) + s];
    return rr < 0 ? -1 : off + rr;
  }
  // CHAIN / RING: independence check, then arithmetic rank
  uint64_t m = c;
  while (m) {
    int k = __ffsll((long long)m) - 1;
    if (c & B.adj[k]) return -1;
    m &= m - 1;
  }
  if (B.layout == EL_LAYOUT_CHAIN) {
    int64_t r = 0;
    m = c;
    while (m) { int k = __ffsll((long long)m) - 1; r += (int64_t)B.fib[k + 2]; m &= m - 1; }
    return r;
  }
  return rank_code_ring(B, c);
}

// Target row of flipping bit k of `code` (row `row`); -1 if outside the basis.
__device__ __forceinline__ int64_t flip_target(const BasisDev &B, uint64_t code,
                                               int64_t row, int k) {
  const uint64_t bit = 1ULL << k;
  const bool set = (code & bit) != 0;
  if (B.layout == EL_LAYOUT_FULL) return row ^ (int64_t)bit;
  if (B.layout == EL_LAYOUT_TABLE) {
    if (!set && (code & B.adj[k])) return -1;
    uint64_t t = code ^ bit;
    uint64_t p = t >> B.L, s = t & ((1ULL << B.L) - 1ULL);
    int64_t off = B.pre_off[p];
    if (off < 0) return -1;
    int32_t rr = B.suf_rank[((uint64_t)B.pre_cls[p] << B.L) + s];
    return rr < 0 ? -1 : off + rr;
  }
  if (!set && (code & B.adj[k])) return -1;
  if (B.layout == EL_LAYOUT_CHAIN) {
    int64_t w = (int64_t)B.fib[k + 2];
    return set ? row - w : row + w;
  }
  // RING
  const int n = B.n;
  if (k == n - 1) return rank_code_ring(B, code ^ bit);
  const bool top = (code >> (n - 1)) & 1ULL;
  int64_t w = (int64_t)(top ? B.fib[k + 1] : B.fib[k + 2]);
  return set ? row - w : row + w;
}

// ------------------------------------------------------------ scalar types

template <typename S> struct Cx { S re, im; };

template <typename S, bool C> struct VecT;
template <typename S> struct VecT<S, false> { typedef S type; };
template <> struct VecT<float, true> { typedef float2 type; };
template <> struct VecT<double, true> { typedef double2 type; };

}  // namespace el

// ------------------------------------------------------------ launchers
// Generic fused row kernel:  y = a*(H x) + b*x + c*z ;  acc += w*y ;
// dots over rows per vector: [xx, Re<x,y>, Im<x,y>, yy] (FP64, deterministic).

struct ApplyArgs {
  int dtype;           // EL_F32 / EL_F64 / EL_C64 / EL_C128
  int nvec;
  const void *x;
  const void *z;       // may be null
  void *y;             // may be null (only dots/acc wanted)
  void *acc;           // may be null
  double a, b, c;
  double w_re, w_im;   // acc coefficient
  double *dots;        // device [nvec*4] or null
  int want_dots;       // bitmask: 1 xx, 2 xy, 4 yy
  const void *probe;   // real dtypes: slot 2 of dots = <y, probe> (may be null)
  int skip_diag;       // 1: H without its diagonal (off-diagonal part only)
  const double *row_diag_scale;  // unused hook, keep null
};

namespace el {
int launch_apply(el_ctx *ctx, el_ham *h, const ApplyArgs &A);
int launch_diag_v(el_ctx *ctx, el_ham *h);
int launch_full_diag(el_ctx *ctx, el_ham *h, int dtype, void *out);
// Gershgorin interval of H over the basis (host results).
// norm1 (optional): max over rows of |d_r| + sum |offdiag| (a bound on the
// 1-norm and the 2-norm of H, also when H has a loss diagonal).
int gershgorin(el_ctx *ctx, el_ham *h, double *lo, double *hi, double *norm1 = nullptr);
// y[i] = alpha*x[i] + beta*y[i] and optional ||y||^2 (dots[0]); real or complex
int launch_axpby(el_ctx *ctx, int dtype, int64_t len, double a_re, double a_im,
                 const void *x, double b_re, double b_im, void *y,
                 double *norm2_out);
// dots_out[j] = <V_j, w> for j < k (V: k vectors of length len, contiguous,
// leading dimension ld); complex results as (re, im) pairs.
int launch_gemv_t(el_ctx *ctx, int dtype, int64_t len, int k, const void *V,
                  int64_t ld, const void *w, double *dots_out);
// w -= sum_j coef_j V_j  (coef: device complex pairs [k][2])
int launch_gemv_n_sub(el_ctx *ctx, int dtype, int64_t len, int k,
                      const void *V, int64_t ld, const double *coef, void *w);
// out = sum_j coef_j V_j (coef host-side copied into scalars area)
int launch_gemv_n(el_ctx *ctx, int dtype, int64_t len, int k, const void *V,
                  int64_t ld, const double *coef_dev, void *out);
int launch_fill_gauss(el_ctx *ctx, int dtype, int64_t len, uint64_t seed,
                      void *out);
int launch_fill_rademacher(el_ctx *ctx, int dtype, int64_t dim, int nvec,
                           uint64_t seed, int64_t probe0, int nvalid, void *out);
int launch_probe_copy(el_ctx *ctx, int dtype, int64_t dim, int nvec,
                      const int8_t *probes_dev, void *out);
int launch_scale(el_ctx *ctx, int dtype, int64_t len, const double *scale_dev,
                 int invert_sqrt, void *x);
int launch_observables(el_ctx *ctx, el_ham *h, int dtype, const void *psi,
                       double *out_dev);
// Chebyshev propagator plan for exp(-i CONV H tau) (el_evolve.cu):
// H = a Htil + b from the Gershgorin interval, coefficients c_0..c_M.
struct ChebPlan {
  double a = 1, b = 0;
  int M = 1;
  std::vector<double> c_re, c_im;
};
int cheb_plan(el_ctx *ctx, el_ham *h, double tau_ns, double tol, ChebPlan *plan);
// The expansion for a spectrum inside [lo, hi] (what cheb_plan does after
// its Gershgorin bound).
void cheb_plan_bounds(double lo, double hi, double tau_ns, double tol, ChebPlan *plan);
// The whole adjoint gradient as one cooperative launch (el_adjoint_coop.cu):
// vectors in buf (K+1 checkpoints, Mmax+1 terms, 3 adjoint vectors, lambda),
// per-term dots into hg, the objective into F.
template <typename S>
int adjoint_coop(el_ctx *ctx, el_ham *h, int K, const std::vector<ChebPlan> &plans, int Mmax,
                 const double *omega_k, const double *delta_k, const std::vector<double> &ash,
                 const std::vector<double> &bsh, const void *psi0, const void *target, const double *obs_diag,
                 void *buf, std::vector<double> &hg, double &F);
// Tiled single-vector FP64 H x on the full basis, 20 <= N <= 25 (el_kpm_tma.cu):
// a plan over three vector buffers, then y = H x + cz z per call with
// <x,x>, <x,y>, 0, <y,y> in dots[0..3].
bool hv_tiled_eligible(const el_ham *h, int dtype);
int hv_tiled_plan(el_ctx *ctx, el_ham *h, void *const bufs[3], int slot, el_hv_plan **out);
int hv_tiled(el_ctx *ctx, el_ham *h, el_hv_plan *P, int ix, int iy, int iz, double cz, double *dots);
int hv_tiled_error(el_ctx *ctx, el_hv_plan *P);
void hv_tiled_free(el_hv_plan *P);

// TMA-fed tiled full-basis KPM recurrence (el_kpm_tma.cu), 20 <= N <= 25
bool kpm_tma_eligible(const el_ham *h, int dtype, int chunk);
int kpm_tma(el_ctx *ctx, el_ham *h, int dtype, int num, int nvec, int chunk, uint64_t seed,
            const int8_t *probes_host, double c, double r, double *mu_host);
// tiled full-basis KPM recurrence (el_kpm_full.cu)
bool kpm_full_eligible(const el_ham *h, int dtype, int chunk, int mode);
int kpm_full(el_ctx *ctx, el_ham *h, int dtype, int num, int nvec, int chunk, uint64_t seed,
             const int8_t *probes_host, double c, double r, double *mu_host);
}  // namespace el
