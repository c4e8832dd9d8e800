// Site occupations without allocation: el_observables_noalloc.
//
// Same result as el_observables (per-site <n_i> and the squared norm of a
// device state), for callers that must not allocate device memory once they
// are running -- for example an evolution driver that measures <n_i> between
// propagation steps in a process whose own pool has already reserved the free
// HBM for state vectors, where a cudaMalloc would fail or, like cudaFree,
// could stall the device.  el_observables may grow the context's reduction
// buffer with cudaMalloc on its first call for a larger basis; this variant
// never does: its reduction scratch is one static device array of fixed size,
// and it calls no allocating function (no cudaMalloc/cudaFree, no library that
// allocates).  Results go through the context's pinned result area, which
// el_ctx_create allocated.
//
// Limits and rules:
//  * at most EL_NOALLOC_MAX_SITES sites (n + 1 partial sums per block, for at
//    most EL_NOALLOC_BLOCKS blocks); a larger system returns EL_EINVAL with a
//    message, and el_observables serves it;
//  * the scratch's completion counter must be zero when a launch starts: it
//    is zero when the module loads and the last block of every launch resets
//    it; the partial sums and the result need no initial value (each block
//    writes its own slot before the last block reads them);
//  * the scratch is shared by every caller on a device, so calls on one
//    device must not overlap in time (two host threads, or two streams with
//    launches in flight together): overlapping calls race on the counter and
//    the partial sums and return wrong values.  Serialise them;
//  * the first call on each device looks up the scratch's address with
//    cudaGetSymbolAddress, which can load this library's device code; make
//    that first call before any stream capture starts on the device.
#include "el_internal.cuh"

#include <atomic>

#define EL_NOALLOC_MAX_SITES 40
#define EL_NOALLOC_BLOCKS 592          // 4 blocks of 256 threads per SM of a B200
#define EL_NOALLOC_HEADER 128          // doubles: counter word, then the result
#define EL_NOALLOC_DOUBLES (EL_NOALLOC_HEADER + EL_NOALLOC_BLOCKS * (EL_NOALLOC_MAX_SITES + 1))
#define EL_NOALLOC_MAX_DEVICES 64

namespace {

// [0]: completion counter (low 32 bits), [64, 64 + n]: result (bit order),
// [EL_NOALLOC_HEADER, ...): per-block partial sums, n + 1 per block.
// 195,200 bytes per device.
static __device__ __align__(256) double g_noalloc_scratch[EL_NOALLOC_DOUBLES];

std::atomic<double *> g_scratch_ptr[EL_NOALLOC_MAX_DEVICES];

template <typename S, bool C>
__global__ void __launch_bounds__(256) k_observables_static(BasisDev B, const S *psi, double *scratch) {
  __shared__ double ws[8][EL_NOALLOC_MAX_SITES + 1];
  __shared__ bool last;
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
  double *out = scratch + 64;
  double *partials = scratch + EL_NOALLOC_HEADER;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = B.n;
  for (int k = threadIdx.x; k < 8 * (EL_NOALLOC_MAX_SITES + 1); k += blockDim.x) (&ws[0][0])[k] = 0.0;
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

// Device address of the scratch array on `device` (looked up once per device).
int scratch_for(el_ctx *ctx, int device, double **out) {
  if (device < 0 || device >= EL_NOALLOC_MAX_DEVICES)
    return el::fail(ctx, EL_EINVAL, "el_observables_noalloc: device %d outside [0, %d)", device,
                    EL_NOALLOC_MAX_DEVICES);
  double *p = g_scratch_ptr[device].load(std::memory_order_acquire);
  if (!p) {
    // the caller made `device` current
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return el::fail(ctx, EL_ECUDA, "el_observables_noalloc: cudaGetSymbolAddress failed (%s)",
                      cudaGetErrorString(e));
    }
    g_scratch_ptr[device].store(p, std::memory_order_release);
  }
  *out = p;
  return EL_OK;
}

}  // namespace

extern "C" int el_observables_noalloc(el_ctx *ctx, el_ham *h, int dtype, const void *psi,
                                      double *n_site_host, double *norm_host) {
  if (!ctx || !h || !psi) return EL_EINVAL;
  const int n = h->n;
  if (n > EL_NOALLOC_MAX_SITES)
    return el::fail(ctx, EL_EINVAL,
                    "el_observables_noalloc: %d sites exceed its static scratch limit of %d sites; "
                    "use el_observables", n, EL_NOALLOC_MAX_SITES);
  if (dtype != EL_F32 && dtype != EL_F64 && dtype != EL_C64 && dtype != EL_C128)
    return el::fail(ctx, EL_EINVAL, "unknown dtype %d", dtype);
  EL_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  double *scratch = nullptr;
  int rc = scratch_for(ctx, ctx->device, &scratch);
  if (rc) return rc;
  const BasisDev B = el::basis_dev(h->basis);
  int64_t g = (B.dim + 255) / 256;
  const int grid = (int)(g < 1 ? 1 : (g > EL_NOALLOC_BLOCKS ? EL_NOALLOC_BLOCKS : g));
  switch (dtype) {
    case EL_F32: k_observables_static<float, false><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, scratch); break;
    case EL_F64: k_observables_static<double, false><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, scratch); break;
    case EL_C64: k_observables_static<float, true><<<grid, 256, 0, ctx->stream>>>(B, (const float *)psi, scratch); break;
    default: k_observables_static<double, true><<<grid, 256, 0, ctx->stream>>>(B, (const double *)psi, scratch); break;
  }
  EL_LAUNCH_CHECK(ctx);
  EL_CUDA_TRY(ctx, el::copy(ctx, ctx->h_scalars, scratch + 64, (n + 1) * sizeof(double),
                            cudaMemcpyDeviceToHost));
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (n_site_host)
    for (int i = 0; i < n; ++i) n_site_host[i] = ctx->h_scalars[n - 1 - i];
  if (norm_host) *norm_host = ctx->h_scalars[n];
  return EL_OK;
}
