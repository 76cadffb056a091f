// extern "C" entry points of libmtlgpu (declared in include/mtlgpu.h).
// Every entry validates its arguments, never throws, and returns an
// mtlgpu_status; CUDA failures are reported as MTLGPU_CUDA_ERROR with the
// runtime's message kept in the context (mtlgpu_last_error).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>

#include "internal.h"

namespace mtlgpu {

mtlgpu_status set_cuda_error(Ctx* ctx, cudaError_t e, const char* what) {
  if (ctx) {
    ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  }
  cudaGetLastError();  // clear the sticky-free error state
  return e == cudaErrorMemoryAllocation ? MTLGPU_OUT_OF_MEMORY : MTLGPU_CUDA_ERROR;
}

mtlgpu_status take_device_error(Ctx* ctx) {
  int h = 0;
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h != 0) {
    MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->last_error = std::string("device reported: ") + mtlgpu_status_string(h);
    return (mtlgpu_status)h;
  }
  return MTLGPU_OK;
}

mtlgpu_status dot_launch(Ctx* ctx, int n, const double* x, const double* y, double* d_out,
                         int order);
mtlgpu_status axpby_launch(Ctx* ctx, int n, double alpha, const double* x, double beta, double* y);

namespace {

mtlgpu_status set_device(Ctx* ctx) {
  MTLGPU_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  return MTLGPU_OK;
}

mtlgpu_status ctx_init(Ctx* ctx) {
  MTLGPU_TRY_CUDA(ctx, cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount,
                                              ctx->device));
  if (const char* m = std::getenv("MTLGPU_SWEEP_BLOCKS_PER_SM")) ctx->sweep_blocks_per_sm = std::atoi(m);
  if (const char* m = std::getenv("MTLGPU_SWEEP")) {
    if (!std::strcmp(m, "part")) ctx->part_sweeps = 1;
    if (!std::strcmp(m, "ticket")) ctx->part_sweeps = 0;
  }
  if (const char* m = std::getenv("MTLGPU_PART_ROWS")) ctx->part_rows = std::atoi(m);
  {
    // the context's own pool (a failure leaves the device's default pool)
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    if (cudaMemPoolCreate(&ctx->pool, &props) == cudaSuccess) {
      unsigned long long keep = kPoolKeepBytes;
      cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
      cudaGetLastError();
      ctx->pool = nullptr;
    }
  }
  MTLGPU_TRY(dalloc(ctx, &ctx->d_partials, (size_t)kMaxPartials * kPartialWidth));
  MTLGPU_TRY(dalloc(ctx, &ctx->d_counters, kNumCounters));
  MTLGPU_TRY(dalloc(ctx, &ctx->d_scalars, 64));
  MTLGPU_TRY(dalloc(ctx, &ctx->d_error, 1));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, sizeof(unsigned) * kNumCounters,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_scalars, 0, sizeof(double) * 64, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&ctx->h_scalars), 64 * sizeof(double)));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return MTLGPU_OK;
}

mtlgpu_status read_scalar(Ctx* ctx, const double* d, double* h) {
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->h_scalars, d, sizeof(double), cudaMemcpyDeviceToHost,
                                       ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *h = ctx->h_scalars[0];
  return MTLGPU_OK;
}

mtlgpu_status csr_finish_create(Csr* A) {
  mtlgpu_status s = csr_analyse(A);
  if (s != MTLGPU_OK) return s;
  return MTLGPU_OK;
}

void csr_release(Csr* A) {
  Ctx* ctx = A->ctx;
  release_workspaces(A, nullptr);
  dfree(ctx, A->d_rp);
  dfree(ctx, A->d_ci);
  dfree(ctx, A->d_v);
  dfree(ctx, A->d_v32);
  dfree(ctx, A->d_diag);
  dfree(ctx, A->d_bin_rows);
  dfree(ctx, A->d_meta);
  sell_free(ctx, &A->sell);
  dfree(ctx, A->d_trp);
  dfree(ctx, A->d_tci);
  dfree(ctx, A->d_tv);
}

}  // namespace

// A new handle that takes ownership of device CSR arrays built by the library
// (assembly, generators); they are freed with the handle, or here on failure.
mtlgpu_status csr_adopt(Ctx* ctx, int n_rows, int n_cols, int nnz, int32_t* d_rp, int32_t* d_ci,
                        double* d_v, Csr** out) {
  *out = nullptr;
  mtlgpu_csr* A = new (std::nothrow) mtlgpu_csr();
  if (!A) {
    dfree(ctx, d_rp);
    dfree(ctx, d_ci);
    dfree(ctx, d_v);
    return MTLGPU_OUT_OF_MEMORY;
  }
  A->ctx = ctx;
  A->n_rows = n_rows;
  A->n_cols = n_cols;
  A->nnz = nnz;
  A->d_rp = d_rp;
  A->d_ci = d_ci;
  A->d_v = d_v;
  mtlgpu_status s = csr_finish_create(A);
  if (s != MTLGPU_OK) {
    csr_release(A);
    delete A;
    return s;
  }
  *out = A;
  return MTLGPU_OK;
}

mtlgpu_status csr_assemble(Ctx* ctx, const Csr* base, int n_rows, int n_cols, long long count,
                           const int32_t* d_rows, const int32_t* d_cols, const double* d_vals,
                           const uint8_t* d_ops, int updater, Csr** out);  // assemble.cu
mtlgpu_status csr_laplacian(Ctx* ctx, int dim, int a, int b, Csr** out);   // assemble.cu

}  // namespace mtlgpu

using namespace mtlgpu;

extern "C" {

int mtlgpu_abi_version(void) { return MTLGPU_ABI_VERSION; }

const char* mtlgpu_status_string(int s) {
  switch (s) {
    case MTLGPU_OK: return "ok";
    case MTLGPU_MAX_ITER: return "too many iterations";
    case MTLGPU_INVALID_ARG: return "invalid argument";
    case MTLGPU_NOT_SQUARE: return "matrix not square";
    case MTLGPU_MISSING_DIAGONAL: return "missing diagonal";
    case MTLGPU_ZERO_PIVOT: return "zero, negative or non-finite pivot";
    case MTLGPU_BREAKDOWN: return "unexpected orthogonality (breakdown)";
    case MTLGPU_TIMEOUT: return "bounded device wait timed out";
    case MTLGPU_INTERRUPTED: return "interrupted";
    case MTLGPU_CUDA_ERROR: return "CUDA error";
    case MTLGPU_NOT_SORTED: return "CSR rows not sorted or duplicate column";
    case MTLGPU_INDEX_RANGE: return "column index out of range";
    case MTLGPU_OUT_OF_MEMORY: return "out of device memory";
    case MTLGPU_INCOMPATIBLE_SIZE: return "incompatible size";
    case MTLGPU_NOT_SUPPORTED: return "not supported";
    default: return "unknown status";
  }
}

mtlgpu_status mtlgpu_ctx_create_on_stream(int device, void* stream, mtlgpu_ctx** out) {
  if (!out) return MTLGPU_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return MTLGPU_CUDA_ERROR;
  }
  mtlgpu_ctx* c = new (std::nothrow) mtlgpu_ctx();
  if (!c) return MTLGPU_OUT_OF_MEMORY;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return MTLGPU_CUDA_ERROR;
  }
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
    c->own_stream = false;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return MTLGPU_CUDA_ERROR;
    }
    c->own_stream = true;
  }
  mtlgpu_status s = ctx_init(c);
  if (s != MTLGPU_OK) {
    mtlgpu_ctx_destroy(c);
    return s;
  }
  *out = c;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_ctx_create(int device, mtlgpu_ctx** out) {
  return mtlgpu_ctx_create_on_stream(device, nullptr, out);
}

mtlgpu_status mtlgpu_ctx_destroy(mtlgpu_ctx* c) {
  if (!c) return MTLGPU_INVALID_ARG;
  cudaSetDevice(c->device);
  dfree(c, c->d_partials);
  dfree(c, c->d_counters);
  dfree(c, c->d_scalars);
  dfree(c, c->d_error);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->h_scalars) cudaFreeHost(c->h_scalars);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  // memory still held by handles of this context is released with the
  // pool once those handles free it
  if (c->pool) cudaMemPoolDestroy(c->pool);
  delete c;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_ctx_synchronize(mtlgpu_ctx* c) {
  if (!c) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return take_device_error(c);
}

void* mtlgpu_ctx_stream(mtlgpu_ctx* c) { return c ? (void*)c->stream : nullptr; }

mtlgpu_status mtlgpu_ctx_set_spin_limit(mtlgpu_ctx* c, long long polls) {
  if (!c || polls < 1) return MTLGPU_INVALID_ARG;
  c->spin_limit = polls;
  return MTLGPU_OK;
}

const char* mtlgpu_last_error(mtlgpu_ctx* c) { return c ? c->last_error.c_str() : "no context"; }

mtlgpu_status mtlgpu_malloc(mtlgpu_ctx* c, size_t bytes, void** out) {
  if (!c || !out) return MTLGPU_INVALID_ARG;
  char* p = nullptr;
  MTLGPU_TRY(dalloc(c, &p, bytes));
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  *out = p;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_free(mtlgpu_ctx* c, void* p) {
  if (!c) return MTLGPU_INVALID_ARG;
  if (p) MTLGPU_TRY_CUDA(c, cudaFreeAsync(p, c->stream));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_memcpy_h2d(mtlgpu_ctx* c, void* d, const void* h, size_t bytes) {
  if (!c || (bytes && (!d || !h))) return MTLGPU_INVALID_ARG;
  if (bytes) MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c->stream));
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_memcpy_d2h(mtlgpu_ctx* c, void* h, const void* d, size_t bytes) {
  if (!c || (bytes && (!d || !h))) return MTLGPU_INVALID_ARG;
  if (bytes) MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, c->stream));
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return MTLGPU_OK;
}

// ---- CSR -------------------------------------------------------------------
static mtlgpu_status csr_create_common(mtlgpu_ctx* c, int n_rows, int n_cols, int nnz,
                                       const int32_t* rp, const int32_t* ci, const double* v,
                                       cudaMemcpyKind kind, mtlgpu_csr** out) {
  if (!c || !out || n_rows < 0 || n_cols < 0 || nnz < 0 || !rp || (nnz > 0 && (!ci || !v)))
    return MTLGPU_INVALID_ARG;
  *out = nullptr;
  MTLGPU_TRY(set_device(c));
  if (kind == cudaMemcpyHostToDevice && (rp[0] != 0 || rp[n_rows] != nnz))
    return MTLGPU_INVALID_ARG;
  mtlgpu_csr* A = new (std::nothrow) mtlgpu_csr();
  if (!A) return MTLGPU_OUT_OF_MEMORY;
  A->ctx = c;
  A->n_rows = n_rows;
  A->n_cols = n_cols;
  A->nnz = nnz;
  mtlgpu_status s = MTLGPU_OK;
  if ((s = dalloc(c, &A->d_rp, n_rows + 1)) != MTLGPU_OK ||
      (s = dalloc(c, &A->d_ci, nnz)) != MTLGPU_OK ||
      (s = dalloc(c, &A->d_v, nnz)) != MTLGPU_OK) {
    csr_release(A);
    delete A;
    return s;
  }
  cudaError_t e = cudaMemcpyAsync(A->d_rp, rp, sizeof(int32_t) * (n_rows + 1), kind, c->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(A->d_ci, ci, sizeof(int32_t) * nnz, kind, c->stream);
  if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(A->d_v, v, sizeof(double) * nnz, kind, c->stream);
  if (e != cudaSuccess) {
    s = set_cuda_error(c, e, "csr upload");
    csr_release(A);
    delete A;
    return s;
  }
  s = csr_finish_create(A);
  if (s != MTLGPU_OK) {
    csr_release(A);
    delete A;
    return s;
  }
  *out = A;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_create(mtlgpu_ctx* c, int n_rows, int n_cols, int nnz,
                                const int32_t* rp, const int32_t* ci, const double* v,
                                mtlgpu_csr** out) {
  return csr_create_common(c, n_rows, n_cols, nnz, rp, ci, v, cudaMemcpyHostToDevice, out);
}

mtlgpu_status mtlgpu_csr_create_device(mtlgpu_ctx* c, int n_rows, int n_cols, int nnz,
                                       const int32_t* rp, const int32_t* ci, const double* v,
                                       mtlgpu_csr** out) {
  return csr_create_common(c, n_rows, n_cols, nnz, rp, ci, v, cudaMemcpyDeviceToDevice, out);
}

mtlgpu_status mtlgpu_csr_set_values(mtlgpu_csr* A, const double* h_vals, const double* d_vals) {
  if (!A || (!h_vals == !d_vals)) return MTLGPU_INVALID_ARG;
  Ctx* c = A->ctx;
  if (A->nnz)
    MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(A->d_v, h_vals ? h_vals : d_vals, sizeof(double) * A->nnz,
                                       h_vals ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                       c->stream));
  // Solver graphs recorded on this matrix captured pointers to the derived
  // copies below: release them (they are re-recorded on the next solve).
  release_workspaces(A, nullptr);
  dfree(c, A->d_v32);
  dfree(c, A->d_trp);
  dfree(c, A->d_tci);
  dfree(c, A->d_tv);
  if (A->spmv_kernel == 2) {
    dfree(c, A->sell.d_val32);  // rebuilt by the next mixed-precision solve
    MTLGPU_TRY(sell_refill(c, A->d_rp, A->d_ci, A->d_v, 0, &A->sell));
  }
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_destroy(mtlgpu_csr* A) {
  if (!A) return MTLGPU_INVALID_ARG;
  Ctx* c = A->ctx;
  csr_release(A);
  cudaStreamSynchronize(c->stream);
  delete A;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_assemble(mtlgpu_ctx* c, const mtlgpu_csr* base, int n_rows, int n_cols,
                                  long long count, const int32_t* d_rows, const int32_t* d_cols,
                                  const double* d_vals, const uint8_t* d_ops, int updater,
                                  mtlgpu_csr** out) {
  if (!c || !out || n_rows < 0 || n_cols < 0 || count < 0 ||
      (count > 0 && (!d_rows || !d_cols || !d_vals)) || updater < MTLGPU_UPDATE_STORE ||
      updater > MTLGPU_UPDATE_TIMES)
    return MTLGPU_INVALID_ARG;
  if (base && (base->ctx != c || base->n_rows != n_rows || base->n_cols != n_cols))
    return MTLGPU_INCOMPATIBLE_SIZE;
  *out = nullptr;
  MTLGPU_TRY(set_device(c));
  Csr* A = nullptr;
  MTLGPU_TRY(csr_assemble(c, base, n_rows, n_cols, count, d_rows, d_cols, d_vals, d_ops, updater,
                          &A));
  *out = static_cast<mtlgpu_csr*>(A);
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_laplacian2d(mtlgpu_ctx* c, int m, int n, mtlgpu_csr** out) {
  if (!c || !out || m < 0 || n < 0) return MTLGPU_INVALID_ARG;
  *out = nullptr;
  MTLGPU_TRY(set_device(c));
  Csr* A = nullptr;
  MTLGPU_TRY(csr_laplacian(c, 2, m, n, &A));
  *out = static_cast<mtlgpu_csr*>(A);
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_laplacian3d(mtlgpu_ctx* c, int N, mtlgpu_csr** out) {
  if (!c || !out || N < 0) return MTLGPU_INVALID_ARG;
  *out = nullptr;
  MTLGPU_TRY(set_device(c));
  Csr* A = nullptr;
  MTLGPU_TRY(csr_laplacian(c, 3, N, N, &A));
  *out = static_cast<mtlgpu_csr*>(A);
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_info(const mtlgpu_csr* A, int* n_rows, int* n_cols, int* nnz) {
  if (!A) return MTLGPU_INVALID_ARG;
  if (n_rows) *n_rows = A->n_rows;
  if (n_cols) *n_cols = A->n_cols;
  if (nnz) *nnz = A->nnz;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_csr_device_arrays(const mtlgpu_csr* A, const int32_t** rp,
                                       const int32_t** ci, const double** v) {
  if (!A) return MTLGPU_INVALID_ARG;
  if (rp) *rp = A->d_rp;
  if (ci) *ci = A->d_ci;
  if (v) *v = A->d_v;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_spmv(mtlgpu_csr* A, const double* x, double* y, double alpha, double beta) {
  if (!A || (A->n_rows && (!x || !y)) || x == y) return MTLGPU_INVALID_ARG;
  SpmvArgs a;
  a.epi = EPI_AXPBY;
  a.alpha = alpha;
  a.beta = beta;
  MTLGPU_TRY(spmv_launch<double>(A, x, y, a));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_cg_direction_product(mtlgpu_csr* A, int prec, const void* d_z, double beta,
                                          const void* d_p, void* d_p_out, void* d_q,
                                          double* d_pq) {
  if (!A || (prec != MTLGPU_FP32 && prec != MTLGPU_FP64)) return MTLGPU_INVALID_ARG;
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  if (A->n_rows && (!d_z || !d_p_out || !d_q || !d_pq || d_p_out == d_z || d_p_out == d_p ||
                    d_q == d_z || d_q == d_p || d_q == d_p_out))
    return MTLGPU_INVALID_ARG;
  if (prec == MTLGPU_FP32) {
    MTLGPU_TRY(csr_ensure_fp32(A));
    return cg_direction_product<float>(A, static_cast<const float*>(d_z), beta,
                                       static_cast<const float*>(d_p),
                                       static_cast<float*>(d_p_out), static_cast<float*>(d_q),
                                       d_pq);
  }
  return cg_direction_product<double>(A, static_cast<const double*>(d_z), beta,
                                      static_cast<const double*>(d_p),
                                      static_cast<double*>(d_p_out), static_cast<double*>(d_q),
                                      d_pq);
}

mtlgpu_status mtlgpu_spmv_f32(mtlgpu_csr* A, const float* x, float* y) {
  if (!A || (A->n_rows && (!x || !y)) || x == y) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY(csr_ensure_fp32(A));
  SpmvArgs a;
  a.epi = EPI_AXPBY;
  a.alpha = 1.0;
  a.beta = 0.0;
  MTLGPU_TRY(spmv_launch<float>(A, x, y, a));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_spmv_transposed(mtlgpu_csr* A, const double* x, double* y) {
  if (!A || (A->n_rows && (!x || !y)) || x == y) return MTLGPU_INVALID_ARG;
  return spmv_transposed_launch(A, x, y);
}

// ---- BLAS-1 ----------------------------------------------------------------
mtlgpu_status mtlgpu_dot(mtlgpu_ctx* c, int n, const double* x, const double* y, double* h) {
  if (!c || n < 0 || !h || (n && (!x || !y))) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY(dot_launch(c, n, x, y, c->d_scalars + 8, 0));
  return read_scalar(c, c->d_scalars + 8, h);
}

mtlgpu_status mtlgpu_unary_dot(mtlgpu_ctx* c, int n, const double* x, double* h) {
  return mtlgpu_dot(c, n, x, x, h);
}

mtlgpu_status mtlgpu_two_norm(mtlgpu_ctx* c, int n, const double* x, double* h) {
  double s = 0;
  MTLGPU_TRY(mtlgpu_dot(c, n, x, x, &s));
  *h = std::sqrt(s);
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_axpy(mtlgpu_ctx* c, int n, double alpha, const double* x, double* y) {
  if (!c || n < 0 || (n && (!x || !y))) return MTLGPU_INVALID_ARG;
  return axpby_launch(c, n, alpha, x, 1.0, y);
}

mtlgpu_status mtlgpu_xpay(mtlgpu_ctx* c, int n, const double* x, double beta, double* y) {
  if (!c || n < 0 || (n && (!x || !y))) return MTLGPU_INVALID_ARG;
  return axpby_launch(c, n, 1.0, x, beta, y);
}

// ---- preconditioners --------------------------------------------------------
mtlgpu_status mtlgpu_pc_create(mtlgpu_csr* A, int kind, int prec, mtlgpu_pc** out) {
  if (!A || !out || kind < MTLGPU_PC_IDENTITY || kind > MTLGPU_PC_IC0 ||
      (prec != MTLGPU_FP64 && prec != MTLGPU_FP32))
    return MTLGPU_INVALID_ARG;
  *out = nullptr;
  if (A->n_rows != A->n_cols) return MTLGPU_NOT_SQUARE;
  mtlgpu_pc* P = new (std::nothrow) mtlgpu_pc();
  if (!P) return MTLGPU_OUT_OF_MEMORY;
  P->A = A;
  P->kind = kind;
  P->prec = prec;
  mtlgpu_status s = pc_build(P);
  if (s != MTLGPU_OK) {
    pc_release(P);
    delete P;
    return s;
  }
  *out = P;
  return P->factor_status ? (mtlgpu_status)P->factor_status : MTLGPU_OK;
}

mtlgpu_status mtlgpu_pc_destroy(mtlgpu_pc* P) {
  if (!P) return MTLGPU_INVALID_ARG;
  release_workspaces(P->A, P);
  pc_release(P);
  cudaStreamSynchronize(P->A->ctx->stream);
  delete P;
  return MTLGPU_OK;
}

static mtlgpu_status pc_apply_common(mtlgpu_pc* P, const double* r, double* z, bool adjoint) {
  if (!P || (P->n && (!r || !z)) || (r == z && P->n)) return MTLGPU_INVALID_ARG;
  MTLGPU_TRY(pc_apply_t<double>(P, r, z, adjoint, nullptr, false, false));
  return take_device_error(P->A->ctx);
}

mtlgpu_status mtlgpu_pc_apply(mtlgpu_pc* P, const double* r, double* z) {
  return pc_apply_common(P, r, z, false);
}

mtlgpu_status mtlgpu_pc_adjoint_apply(mtlgpu_pc* P, const double* r, double* z) {
  return pc_apply_common(P, r, z, true);
}

mtlgpu_status mtlgpu_pc_apply_f32(mtlgpu_pc* P, const float* r, float* z) {
  if (!P || (P->n && (!r || !z)) || (r == z && P->n) ||
      (P->prec != MTLGPU_FP32 && P->kind != MTLGPU_PC_IDENTITY))
    return MTLGPU_INVALID_ARG;
  return pc_apply_t<float>(P, r, z, false, nullptr, false, false);
}

mtlgpu_status mtlgpu_pc_sweep(mtlgpu_pc* P, int which, const double* in, double* out) {
  if (!P || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0) || in == out)
    return MTLGPU_INVALID_ARG;
  const SweepPlan& S = which == MTLGPU_LOWER ? P->lower : P->upper;
  MTLGPU_TRY(sweep_launch<double>(P->A->ctx, S, in, out, false, nullptr));
  return take_device_error(P->A->ctx);
}

mtlgpu_status mtlgpu_pc_sweep_f32(mtlgpu_pc* P, int which, const float* in, float* out) {
  if (!P || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0) || in == out ||
      P->prec != MTLGPU_FP32)
    return MTLGPU_INVALID_ARG;
  const SweepPlan& S = which == MTLGPU_LOWER ? P->lower : P->upper;
  MTLGPU_TRY(sweep_launch<float>(P->A->ctx, S, in, out, false, nullptr));
  return take_device_error(P->A->ctx);
}

mtlgpu_status mtlgpu_pc_set_jacobi_sweeps(mtlgpu_pc* P, int iters) {
  if (!P || iters < 0 || iters > 64) return MTLGPU_INVALID_ARG;
  if (iters == P->jacobi_iters) return MTLGPU_OK;
  // solver graphs recorded with the other kind of apply are stale
  release_workspaces(P->A, P);
  MTLGPU_TRY(pc_set_jacobi(P, iters));
  return take_device_error(P->A->ctx);
}

mtlgpu_status mtlgpu_pc_sweep_kind(const mtlgpu_pc* P, int which, int prec, int* kind) {
  if (!P || !kind || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0)) return MTLGPU_INVALID_ARG;
  const SweepPlan& S = which == MTLGPU_LOWER ? P->lower : P->upper;
  const int pi = prec == MTLGPU_FP32 ? 1 : 0;
  if (P->jacobi_iters > 0)
    *kind = 2;
  else
    *kind = (S.part && S.part->prec[pi].ready) ? 1 : 0;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_pc_factor_info(const mtlgpu_pc* P, int which, int* nnz, int* n_levels) {
  if (!P || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0)) return MTLGPU_INVALID_ARG;
  if (nnz) *nnz = which == MTLGPU_LOWER ? P->nnz_L : P->nnz_U;
  if (n_levels) *n_levels = which == MTLGPU_LOWER ? P->lower.n_levels : P->upper.n_levels;
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_pc_get_factor(const mtlgpu_pc* P, int which, int32_t* rp, int32_t* ci,
                                   double* v) {
  if (!P || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0)) return MTLGPU_INVALID_ARG;
  Ctx* c = P->A->ctx;
  const bool lo = which == MTLGPU_LOWER;
  const int nnz = lo ? P->nnz_L : P->nnz_U;
  const int32_t* drp = lo ? P->d_Lrp : P->d_Urp;
  const int32_t* dci = lo ? P->d_Lci : P->d_Uci;
  const double* dv = lo ? P->d_Lv : P->d_Uv;
  if (rp) MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(rp, drp, sizeof(int32_t) * (P->n + 1),
                                             cudaMemcpyDeviceToHost, c->stream));
  if (ci && nnz) MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(ci, dci, sizeof(int32_t) * nnz,
                                                    cudaMemcpyDeviceToHost, c->stream));
  if (v && nnz) {
    MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(v, dv, sizeof(double) * nnz, cudaMemcpyDeviceToHost,
                                       c->stream));
    MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
    if (P->prec == MTLGPU_FP32)  // FP32 factors: report the stored (rounded) values
      for (int j = 0; j < nnz; j++) v[j] = (double)(float)v[j];
  }
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return MTLGPU_OK;
}

mtlgpu_status mtlgpu_pc_get_levels(const mtlgpu_pc* P, int which, int32_t* lev) {
  if (!P || !lev || (P->kind != MTLGPU_PC_IC0 && P->kind != MTLGPU_PC_ILU0))
    return MTLGPU_INVALID_ARG;
  Ctx* c = P->A->ctx;
  const SweepPlan& S = which == MTLGPU_LOWER ? P->lower : P->upper;
  if (P->n)
    MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(lev, S.d_level, sizeof(int32_t) * P->n,
                                       cudaMemcpyDeviceToHost, c->stream));
  MTLGPU_TRY_CUDA(c, cudaStreamSynchronize(c->stream));
  return MTLGPU_OK;
}

// ---- solvers ----------------------------------------------------------------
void mtlgpu_iter_params_default(mtlgpu_iter_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_iter = 1000;
  p->rtol = 1e-10;
  p->atol = 0.0;
  p->norm_r0 = -1.0;
  p->mode = MTLGPU_SOLVE_FP64;
  p->inner_rtol = 1e-4;
}

mtlgpu_status mtlgpu_solve_krylov(int method, mtlgpu_csr* A, mtlgpu_pc* L, mtlgpu_pc* R,
                                  int param, double* x, const double* b,
                                  const mtlgpu_iter_params* prm, mtlgpu_iter_result* res) {
  if (!A || !prm || !res || (A->n_rows && (!x || !b)) || prm->max_iter < 0 || param < 0)
    return MTLGPU_INVALID_ARG;
  if (method == MTLGPU_CG || method == MTLGPU_BICGSTAB) {
    if (R) return MTLGPU_INVALID_ARG;  // cg / bicgstab take one preconditioner
    return mtlgpu_solve(method, A, L, x, b, prm, res);
  }
  MTLGPU_TRY(set_device(A->ctx));
  const long long launches_before = A->ctx->launches;
  mtlgpu_status s = solve_krylov_impl(method, A, L, R, param, x, b, prm, res);
  res->status = s;
  res->kernel_launches = A->ctx->launches - launches_before;
  return s;
}

mtlgpu_status mtlgpu_solve(int method, mtlgpu_csr* A, mtlgpu_pc* P, double* x, const double* b,
                           const mtlgpu_iter_params* prm, mtlgpu_iter_result* res) {
  if (!A || !prm || !res || (A->n_rows && (!x || !b)) || prm->max_iter < 0)
    return MTLGPU_INVALID_ARG;
  if (method >= MTLGPU_BICG && method <= MTLGPU_GMRES)
    return mtlgpu_solve_krylov(method, A, P, nullptr, 0, x, b, prm, res);
  MTLGPU_TRY(set_device(A->ctx));
  const long long launches_before = A->ctx->launches;
  mtlgpu_status s = solve_impl(method, A, P, x, b, prm, res);
  res->status = s;
  res->kernel_launches = A->ctx->launches - launches_before;
  return s;
}

mtlgpu_status mtlgpu_solve_host(int method, mtlgpu_csr* A, mtlgpu_pc* P, double* hx,
                                const double* hb, const mtlgpu_iter_params* prm,
                                mtlgpu_iter_result* res) {
  if (!A || !prm || !res || (A->n_rows && (!hx || !hb))) return MTLGPU_INVALID_ARG;
  Ctx* c = A->ctx;
  const int n = A->n_rows;
  double *dx = nullptr, *db = nullptr;
  MTLGPU_TRY(dalloc(c, &dx, n));
  MTLGPU_TRY(dalloc(c, &db, n));
  MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(dx, hx, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  MTLGPU_TRY_CUDA(c, cudaMemcpyAsync(db, hb, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  mtlgpu_status s = mtlgpu_solve(method, A, P, dx, db, prm, res);
  cudaMemcpyAsync(hx, dx, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
  dfree(c, dx);
  dfree(c, db);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess && s == MTLGPU_OK) s = set_cuda_error(c, e, "solve_host copy-out");
  return s;
}

mtlgpu_status mtlgpu_csr_autotune(mtlgpu_csr* A, int* choice) {
  if (!A) return MTLGPU_INVALID_ARG;
  int c = 0;
  float ms[3];
  MTLGPU_TRY(csr_autotune_spmv(A, &c, ms));
  if (choice) *choice = c;
  return MTLGPU_OK;
}

}  // extern "C"
