// Host-side structures shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "mtlgpu.h"

namespace mtlgpu {

// Maximum number of partial sums a reduction kernel writes (one per block).
constexpr int kMaxPartials = 4096;
// Device scratch for reductions: partial sums are stored as up to 4 doubles
// per block slot.
constexpr int kPartialWidth = 4;
// Number of independent "last block" counters (one per reduction site that
// may be in flight in one stream-ordered sequence).
constexpr int kNumCounters = 64;
// Freed device memory a context's pool keeps mapped for reuse.
constexpr unsigned long long kPoolKeepBytes = 4ull << 30;

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long spin_limit = 1ll << 26;
  int num_sms = 148;
  std::string last_error;
  // reduction scratch
  double* d_partials = nullptr;   // kMaxPartials * kPartialWidth
  unsigned* d_counters = nullptr; // kNumCounters
  double* d_scalars = nullptr;    // 64 scalar result slots
  double* h_scalars = nullptr;    // pinned mirror (64)
  int* d_error = nullptr;         // device error word: 0 ok, else mtlgpu_status
  // Stream-ordered pool for every device allocation of this context.  Freed
  // memory stays mapped up to kPoolKeepBytes, so per-call scratch (the
  // staging vectors of mtlgpu_solve_host, temporary arrays) is not unmapped
  // and mapped again at every synchronisation as with the default pool.
  cudaMemPool_t pool = nullptr;
  long long launches = 0;         // kernels launched on this context (host-side count)
  // Resident CTAs per SM for the triangular sweeps (fewer pollers contend
  // less for L2; 2 measured best on B200).  Benchmark override:
  // MTLGPU_SWEEP_BLOCKS_PER_SM.
  int sweep_blocks_per_sm = 2;
  // Partitioned sweeps (part_sweep.cu), built at preconditioner creation:
  // 2 = automatic (factors with narrow levels), 1 = always (MTLGPU_SWEEP=part),
  // 0 = never (MTLGPU_SWEEP=ticket); rows per part (MTLGPU_PART_ROWS).
  int part_sweeps = 2;
  int part_rows = 16384;
};

// Row-binned SpMV plan: rows grouped by length, each bin processed by a
// kernel instantiation with G lanes per row (G = 2..32) or a CTA per row.
struct SpmvBin {
  int group;        // lanes per row; 0 = CTA per row
  int begin, count; // slice of the bin row list
};

// SELL-32 copy of a CSR matrix or of a factor's off-diagonal part (sell.cu):
// slices of 32 rows, entries column-major inside a slice, padding column -1;
// the stored (inverted) diagonal of a factor separately.
struct Sell {
  int n = 0, n_slices = 0;
  long long n_ent = 0;             // padded entries
  int max_width = 0;               // largest slice width (entries per row)
  bool unit_diag = false;
  bool round64 = false;            // double copy holds float-rounded values
  bool col_scaled = false;         // entry (r, c) stored as a_rc * dinv[c]
  int32_t* d_slice_ptr = nullptr;  // n_slices + 1 entry offsets (multiples of 32)
  int32_t* d_col = nullptr;
  // column - row as 16 bits (padding: -32768), built when every entry lies
  // within 32,767 of its row (banded / stencil patterns): the streaming
  // kernels then read 2 bytes of index per entry instead of 4
  int16_t* d_dcol = nullptr;
  double* d_val = nullptr;
  float* d_val32 = nullptr;
  double* d_dinv = nullptr;
  float* d_dinv32 = nullptr;
};

struct Pc;
struct XWork;  // workspace of the other Krylov methods (krylov_ext.cu)
// Solver workspace cache entry (buffers + instantiated graph; krylov.cu).
struct WorkspaceEntry {
  Pc* P;
  int method, prec;
  void* ws;
};

struct Csr {
  Ctx* ctx = nullptr;
  std::vector<WorkspaceEntry> workspaces;
  std::vector<XWork*> xwork;
  int n_rows = 0, n_cols = 0, nnz = 0;
  int32_t* d_rp = nullptr;
  int32_t* d_ci = nullptr;
  double* d_v = nullptr;
  float* d_v32 = nullptr;          // FP32 copy, built on demand
  int32_t* d_diag = nullptr;       // position of the diagonal entry per row (-1 if none)
  int max_row = 0;
  double mean_row = 0;
  // binning
  bool uniform = true;             // one bin covering all rows, no row list
  int uniform_group = 8;
  int32_t* d_bin_rows = nullptr;   // rows ordered by bin (when !uniform)
  std::vector<SpmvBin> bins;
  int tuned_rows_per_group = 1;    // autotuner choice (1 or 2 rows per pass)
  // CSR-stream row blocks: block b = rows [meta[b].x, meta[b+1].x), entries
  // [meta[b].y, meta[b+1].y); <= 32 rows and <= 256 entries, or one longer row
  int2* d_meta = nullptr;
  int n_blk = 0;
  int spmv_kernel = 0;             // 0 = CSR-stream, 1 = row-binned groups, 2 = SELL-32
  Sell sell;                       // SELL-32 copy (spmv_kernel == 2)
  // batched solves: CTAs per system (cluster size), lanes per row, and the
  // row count below which a system is solved by one CTA; picked by
  // mtlgpu_batched_autotune
  int batch_cs = 4, batch_g = 8, batch_small = 4096;
  void* batch_work = nullptr;      // cached batched configuration (batched_cluster.cu)
  // transpose (built on demand for A^T x)
  int32_t* d_trp = nullptr;
  int32_t* d_tci = nullptr;
  double* d_tv = nullptr;
};

// Partitioned form of a sweep (part_sweep.cu): rows split into P parts, one
// CTA each; per precision (0: double, 1: float) a stream of block records.
struct PartPlan {
  int P = 0;
  int max_rows = 0;
  long long ext_entries = 0;         // entries read from another part
  struct Prec {
    bool ready = false;
    int vals_bytes = 0, offs_bytes = 0, slot_bytes = 0, smem_bytes = 0, n_blocks = 0;
    int32_t* d_part_blk = nullptr;   // P+1: block range of each part
    int32_t* d_blk_off16 = nullptr;  // n_blocks+1: record offsets in 16-byte units
    unsigned char* d_rec = nullptr;  // record stream
  } prec[2];
};

// One triangular sweep, stored in processing (level) order.
// Row t of the plan is original row row_of[t]; its off-diagonal entries are
// ci/val[rp[t] .. rp[t+1]); dinv[t] is its (inverted) diagonal, absent for a
// unit diagonal.  Tasks never cross a level boundary: task k covers plan rows
// [task_ptr[k], task_ptr[k+1]).
struct SweepPlan {
  int n = 0, nnz_off = 0, n_levels = 0, n_tasks = 0;
  int group = 4;                   // lanes per row
  bool unit_diag = false;
  bool reverse = false;            // upper sweep
  int32_t* d_rp = nullptr;
  int32_t* d_ci = nullptr;
  double* d_val = nullptr;
  float* d_val32 = nullptr;
  double* d_dinv = nullptr;
  float* d_dinv32 = nullptr;
  int32_t* d_row_of = nullptr;
  int32_t* d_task_ptr = nullptr;
  int32_t* d_level_ptr = nullptr;  // plan rows of each level
  int32_t* d_level = nullptr;      // level of each ORIGINAL row
  unsigned* d_ticket = nullptr;    // [0] = task ticket, [1] = finished warps
  PartPlan* part = nullptr;        // partitioned form, when built and fitting
};

struct Pc {
  Csr* A = nullptr;
  int kind = MTLGPU_PC_IDENTITY;
  int prec = MTLGPU_FP64;
  int n = 0;
  double* d_inv_diag = nullptr;    // Jacobi
  float* d_inv_diag32 = nullptr;
  // factors in the reference's CSR layout (for export)
  int nnz_L = 0, nnz_U = 0;
  int32_t *d_Lrp = nullptr, *d_Lci = nullptr, *d_Urp = nullptr, *d_Uci = nullptr;
  double *d_Lv = nullptr, *d_Uv = nullptr;
  SweepPlan lower, upper;          // solve sweeps
  SweepPlan adj_lower, adj_upper;  // adjoint sweeps (ILU only; built on demand)
  bool adj_built = false;
  double* d_tmp = nullptr;         // y0 of solve_lower (per handle, never static)
  float* d_tmp32 = nullptr;
  int factor_status = MTLGPU_OK;
  // Triangular solves as Jacobi iterations (0: exact sweeps).
  int jacobi_iters = 0;
  Sell jac_lower, jac_upper;
  double* d_jtmp = nullptr;
  float* d_jtmp32 = nullptr;
};

// ---- error plumbing ------------------------------------------------------
mtlgpu_status set_cuda_error(Ctx* ctx, cudaError_t e, const char* what);
#define MTLGPU_TRY_CUDA(ctx, call)                                        \
  do {                                                                    \
    cudaError_t _e = (call);                                              \
    if (_e != cudaSuccess) return ::mtlgpu::set_cuda_error((ctx), _e, #call); \
  } while (0)
#define MTLGPU_TRY(call)                      \
  do {                                        \
    mtlgpu_status _s = (call);                \
    if (_s != MTLGPU_OK) return _s;           \
  } while (0)

// Reads and clears the device error word (synchronises the stream).
mtlgpu_status take_device_error(Ctx* ctx);

template <typename T>
mtlgpu_status dalloc(Ctx* ctx, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e =
      ctx->pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), count * sizeof(T),
                                          ctx->pool, ctx->stream)
                : cudaMallocAsync(reinterpret_cast<void**>(p), count * sizeof(T), ctx->stream);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("device allocation failed: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? MTLGPU_OUT_OF_MEMORY : MTLGPU_CUDA_ERROR;
  }
  return MTLGPU_OK;
}
template <typename T>
void dfree(Ctx* ctx, T*& p) {
  if (p) cudaFreeAsync(p, ctx->stream);
  p = nullptr;
}

// ---- internal launchers (implemented in the .cu files) --------------------
mtlgpu_status csr_analyse(Csr* A);                 // spmv.cu: row lengths, bins, diag
mtlgpu_status csr_ensure_fp32(Csr* A);             // spmv.cu
mtlgpu_status csr_ensure_transpose(Csr* A);        // analysis.cu

// SpMV epilogues
enum SpmvEpilogue { EPI_AXPBY = 0, EPI_DOT_X2 = 1, EPI_RESID = 2 };
struct SpmvArgs {
  int epi = EPI_AXPBY;
  double alpha = 1, beta = 0;
  const void* x2 = nullptr;        // EPI_DOT_X2: partial += x2[row] * (A x)[row]
  const void* b = nullptr;         // EPI_RESID: y = b - A x, partial += y^2
  double* out = nullptr;           // device scalar receiving the reduction
  const int* skip = nullptr;       // device flag: nonzero -> kernel returns at once
};
// T = double or float (vector and value type).
template <typename T>
mtlgpu_status spmv_launch(Csr* A, const T* x, T* y, const SpmvArgs& args);
mtlgpu_status spmv_transposed_launch(Csr* A, const double* x, double* y);
mtlgpu_status csr_autotune_spmv(Csr* A, int* choice, float* ms);

// Batched PCG in one persistent cluster launch (batched_cluster.cu).
bool batched_cluster_supported(const Pc* P);
void release_batch_work(Csr* A, const Pc* only_P);
mtlgpu_status solve_batched_cluster(Csr* A, Pc* P, int count, const int32_t* h_off, double* d_x,
                                    const double* d_b, const mtlgpu_iter_params* prm,
                                    mtlgpu_iter_result* res, int cs, int g, int small_rows,
                                    float* ms_out);

// Sweeps (sweep.cu): out must be prefilled with the sentinel when
// prefilled == true; otherwise the launcher fills it first.
template <typename T>
mtlgpu_status sweep_launch(Ctx* ctx, const SweepPlan& P, const T* in, T* out, bool prefilled,
                           const int* skip);
template <typename T>
mtlgpu_status fill_sentinel(Ctx* ctx, T* p, int n);

// Partitioned sweeps (part_sweep.cu).  part_plan_build runs outside stream
// capture; without a usable plan (disabled, or a part that does not fit
// shared memory) S->part stays null and sweeps use sweep_kernel.
mtlgpu_status part_plan_build(Ctx* ctx, SweepPlan* S, bool with_fp32);
void part_plan_free(Ctx* ctx, SweepPlan* S);
void part_plan_free_one(Ctx* ctx, PartPlan* PP, int prec);
template <typename T>
bool part_sweep_ready(const SweepPlan& S, const T* out);
template <typename T>
mtlgpu_status part_sweep_launch(Ctx* ctx, const SweepPlan& S, const T* in, T* out,
                                const int* skip);

// SELL-32 layouts (sell.cu).  diag_pos: 0 = every entry kept (a matrix, or
// a unit-diagonal factor), 1 = the first entry of each row is the diagonal,
// 2 = the last one; the diagonal then goes to d_dinv.
long long sell_padded_entries(int n, const int32_t* h_rp, int diag_pos);
mtlgpu_status sell_build(Ctx* ctx, int n, const int32_t* d_rp, const int32_t* d_ci,
                         const double* d_v, int diag_pos, bool fp64, bool fp32, bool round64,
                         bool scale_cols, Sell* J);
mtlgpu_status sell_refill(Ctx* ctx, const int32_t* d_rp, const int32_t* d_ci, const double* d_v,
                          int diag_pos, Sell* J);
mtlgpu_status sell_ensure_fp32(Ctx* ctx, const int32_t* d_rp, const int32_t* d_ci,
                               const double* d_v, int diag_pos, Sell* J);
void sell_free(Ctx* ctx, Sell* J);

// Jacobi-iteration triangular solves (jacobi_sweep.cu).
template <typename T>
mtlgpu_status jacobi_solve(Ctx* ctx, const Sell& J, int k, const T* v, T* out, T* scratch,
                           const int* skip, const T* dot_with = nullptr,
                           double* dot_out = nullptr);
template <typename T>
mtlgpu_status jacobi_solve_from(Ctx* ctx, const Sell& J, int k, int first, const T* v, T* out,
                                T* scratch, const int* skip, const T* dot_with = nullptr,
                                double* dot_out = nullptr);
mtlgpu_status pc_set_jacobi(Pc* P, int iters);

// Preconditioned CG with Jacobi-applied IC(0)/ILU(0) in three kernels per
// iteration (cg_fused.cu).  `st` is the solve's device SolverState.
struct SolverState;
bool cg_fused_eligible(Csr* A, Pc* P, int prec);
template <typename T>
mtlgpu_status cg_fused_prologue(Csr* A, Pc* P, SolverState* st, const T* r, T* z, T* p, T* q);
template <typename T>
mtlgpu_status bicg_fused_s_apply(Csr* A, Pc* P, SolverState* st, const T* r, const T* v, T* s,
                                 T* shat);
template <typename T>
mtlgpu_status bicg_t_product(Csr* A, SolverState* st, const T* shat, const T* s, T* t);
template <typename T>
mtlgpu_status cg_direction_product(Csr* A, const T* z, double beta, const T* p, T* p_next, T* q,
                                   double* d_pq);
template <typename T>
mtlgpu_status cg_fused_iteration(Csr* A, Pc* P, SolverState* st, T* x, const T* r, T* r_next,
                                 const T* p, T* p_next, T* z, T* q);

// Analysis (analysis.cu)
mtlgpu_status build_sweep_plan(Ctx* ctx, int n, const int32_t* d_rp, const int32_t* d_ci,
                               const double* d_v, bool lower, bool unit_diag, bool diag_last,
                               SweepPlan* plan);
void free_sweep_plan(Ctx* ctx, SweepPlan* plan);
mtlgpu_status sweep_plan_make_fp32(Ctx* ctx, SweepPlan* plan);
mtlgpu_status compute_levels(Ctx* ctx, int n, const int32_t* d_rp, const int32_t* d_ci,
                             bool lower, int32_t* d_level, int* n_levels);
mtlgpu_status scan_i32(Ctx* ctx, const int32_t* in, int32_t* out, int n);
mtlgpu_status csr_transpose(Ctx* ctx, int n_rows, int n_cols, int nnz, const int32_t* d_rp,
                            const int32_t* d_ci, const double* d_v, int32_t* d_trp,
                            int32_t* d_tci, double* d_tv);

// Factorisations (factor.cu)
mtlgpu_status pc_build(Pc* P);
void pc_release(Pc* P);
mtlgpu_status pc_ensure_adjoint(Pc* P);
template <typename T>
mtlgpu_status pc_apply_t(Pc* P, const T* r, T* z, bool adjoint, const int* skip,
                         bool prefilled_tmp, bool prefilled_out, double* rho_out = nullptr);

// BLAS-1 (blas1.cu): results land in device scalar slots.
mtlgpu_status dot_launch(Ctx* ctx, int n, const double* x, const double* y, double* d_out,
                         int order);
mtlgpu_status axpby_launch(Ctx* ctx, int n, double alpha, const double* x, double beta, double* y);

// The other Krylov methods (krylov_ext.cu)
mtlgpu_status solve_krylov_impl(int method, Csr* A, Pc* L, Pc* R, int param, double* d_x,
                                const double* d_b, const mtlgpu_iter_params* prm,
                                mtlgpu_iter_result* res);
void release_xwork(Csr* A, const Pc* only_P);

// Krylov driver (krylov.cu)
mtlgpu_status solve_impl(int method, Csr* A, Pc* P, double* d_x, const double* d_b,
                         const mtlgpu_iter_params* prm, mtlgpu_iter_result* res);
void release_workspaces(Csr* A, Pc* only_P);

int sm_count(Ctx* ctx);
unsigned* counter_slot(Ctx* ctx, int i);

}  // namespace mtlgpu

struct mtlgpu_ctx : mtlgpu::Ctx {};
struct mtlgpu_csr : mtlgpu::Csr {};
struct mtlgpu_pc : mtlgpu::Pc {};
