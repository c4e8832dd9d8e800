// Context, error handling and small shared utilities of libel_b200.so.
#include "el_internal.cuh"

#include <cstdarg>

namespace el {

int fail(el_ctx *ctx, int code, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int cuda_fail(el_ctx *ctx, cudaError_t e, const char *where) {
  return fail(ctx, EL_ECUDA, "CUDA error %d (%s) at %s", (int)e,
              cudaGetErrorString(e), where);
}

bool cancelled(el_ctx *ctx) { return ctx && ctx->cancel && *ctx->cancel != 0; }

int ensure_partials(el_ctx *ctx, size_t doubles) {
  if (doubles <= ctx->partial_cap) return EL_OK;
  // queued kernels may still use the old buffer
  EL_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->d_partials) cudaFree(ctx->d_partials);
  ctx->d_partials = nullptr;
  ctx->partial_cap = 0;
  size_t cap = doubles < (1u << 16) ? (1u << 16) : doubles;
  EL_CUDA_TRY(ctx, cudaMalloc(&ctx->d_partials, cap * sizeof(double)));
  ctx->partial_cap = cap;
  return EL_OK;
}

int dtype_size(int dtype) {
  switch (dtype) {
    case EL_F32: return 4;
    case EL_F64: return 8;
    case EL_C64: return 8;
    case EL_C128: return 16;
  }
  return 0;
}

int grid_for(int64_t work, int block) {
  int64_t g = (work + block - 1) / block;
  const int64_t cap = 148 * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

void *workspace(el_ctx *ctx, int slot, size_t bytes) {
  if (slot < 0 || slot >= 16) { fail(ctx, EL_EINVAL, "bad workspace slot"); return nullptr; }
  if (bytes == 0) bytes = 16;
  if (ctx->ws_size[slot] >= bytes) return ctx->ws_ptr[slot];
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    fail(ctx, EL_ECUDA, "stream synchronisation failed before workspace growth");
    return nullptr;
  }
  if (ctx->ws_ptr[slot]) cudaFree(ctx->ws_ptr[slot]);
  ctx->ws_ptr[slot] = nullptr;
  ctx->ws_size[slot] = 0;
  cudaError_t e = cudaMalloc(&ctx->ws_ptr[slot], bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(ctx, EL_ENOMEM, "cannot allocate %zu bytes of workspace (%s)", bytes, cudaGetErrorString(e));
    ctx->ws_ptr[slot] = nullptr;
    return nullptr;
  }
  ctx->ws_size[slot] = bytes;
  return ctx->ws_ptr[slot];
}

BasisDev basis_dev(const el_basis *b) {
  BasisDev B;
  memset(&B, 0, sizeof B);
  B.layout = b->layout;
  B.n = b->n;
  B.L = b->L;
  B.dim = b->dim;
  B.pre_off = b->d_pre_off;
  B.pre_cls = b->d_pre_cls;
  B.suf_rank = b->d_suf_rank;
  B.codes = b->d_codes;
  for (int k = 0; k < EL_MAX_SITES; ++k) B.adj[k] = b->adj[k];
  B.fib[0] = 0;
  B.fib[1] = 1;
  for (int i = 2; i < EL_MAX_SITES + 3; ++i) B.fib[i] = B.fib[i - 1] + B.fib[i - 2];
  return B;
}

}  // namespace el

extern "C" {

int el_version(void) { return 100; }

int el_ctx_create(int device, void *stream, el_ctx **out) {
  if (!out) return EL_EINVAL;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= 0) return EL_ECUDA;
  if (device < 0 || device >= count) return EL_EINVAL;
  el_ctx *ctx = new el_ctx();
  ctx->device = device;
  ctx->stream = (cudaStream_t)stream;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaMalloc(&ctx->d_counter, 64 * sizeof(unsigned int)) != cudaSuccess ||
      cudaMemset(ctx->d_counter, 0, 64 * sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&ctx->d_scalars, EL_SCALARS * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&ctx->h_scalars, EL_SCALARS * sizeof(double)) != cudaSuccess) {
    el_ctx_destroy(ctx);
    return EL_ECUDA;
  }
  *out = ctx;
  return EL_OK;
}

int el_ctx_destroy(el_ctx *ctx) {
  if (!ctx) return EL_OK;
  cudaSetDevice(ctx->device);
  if (ctx->d_partials) cudaFree(ctx->d_partials);
  if (ctx->d_counter) cudaFree(ctx->d_counter);
  if (ctx->d_scalars) cudaFree(ctx->d_scalars);
  if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
  for (int i = 0; i < 16; ++i) if (ctx->ws_ptr[i]) cudaFree(ctx->ws_ptr[i]);
  delete ctx;
  return EL_OK;
}

int el_ctx_set_stream(el_ctx *ctx, void *stream) {
  if (!ctx) return EL_EINVAL;
  ctx->stream = (cudaStream_t)stream;
  return EL_OK;
}

int el_ctx_set_cancel(el_ctx *ctx, const volatile int32_t *flag) {
  if (!ctx) return EL_EINVAL;
  ctx->cancel = flag;
  return EL_OK;
}

const char *el_last_error(const el_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

int64_t el_ctx_launches(const el_ctx *ctx) { return ctx ? ctx->launches : -1; }

int el_ctx_bytes(const el_ctx *ctx, int64_t *h2d, int64_t *d2h) {
  if (!ctx) return EL_EINVAL;
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  return EL_OK;
}

}  // extern "C"
