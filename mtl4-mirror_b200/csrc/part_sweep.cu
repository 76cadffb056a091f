// Partitioned triangular sweeps for sm_100a.
//
// Same arithmetic as lower_trisolve_t::apply(int_<5>/<6>) and
// upper_trisolve_t::apply(int_<3>) (mtl/operation/lower_trisolve.hpp:173-209,
// upper_trisolve.hpp:160-176): for each row r in dependency order
//     rr = v[r];  for each off-diagonal entry j (stored order): rr -= F[r][j] * w[j];
//     w[r] = rr * dia[r]        (no multiply for a unit diagonal)
// with every multiply and subtract rounded separately, so results are
// bit-identical to the reference's sequential loops.
//
// Why a second sweep design.  The level-ordered sync-free sweep (sweep.cu)
// pays one dependency hop through L2 per level -- a store on one SM, a poll
// on another, 0.3-0.5 us each way on B200 -- so a 128^3 IC(0) factor with
// 382 levels costs ~0.5 ms whatever its bytes.  Here the rows are split into
// P parts, one CTA each (P <= SM count, one resident CTA per SM), chosen so
// that long dependency chains stay inside a part:
//   1. chains: walking rows in level order, a row extends the chain of its
//      farthest dependency one level below it (for a grid in natural order
//      that is the pencil along the slowest index), if that chain still ends
//      there;
//   2. parts: recursive bisection of the chain adjacency graph by BFS
//      distance from a pseudo-peripheral chain, balanced by row count.
// A part's CTA processes its rows level by level.  Values of its own rows
// live in shared memory (one __syncthreads per block of a level); a
// dependency on another part is read from the NaN-boxed output vector in
// global memory (bounded poll), so only part boundaries pay an L2 hop.
//
// Data of a part is a stream of 16-byte aligned block records (<= 256 rows
// of one level each): header, row entry offsets, gather list (the rows' own
// indices, then the external dependencies), entry references (>= 0: slot in
// the part's shared-memory values; < 0: -(1 + gather index)), entry values,
// inverted diagonals.  A ring of kRing slots is filled with cp.async kRing-1
// blocks ahead; the gathers (right-hand sides and external values, 16-byte
// chunks through L2, placed right after the block's record in its slot)
// kAhead blocks ahead, as soon as their record has landed.  An external value
// still unset when gathered is polled again at use.
//
// Co-residency: the grid is P <= SM count CTAs whose shared memory admits one
// CTA per SM, and a CTA only waits for rows of lower levels, which their CTAs
// reach without waiting on it; every wait is bounded (MTLGPU_TIMEOUT).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"

namespace mtlgpu {

using namespace dev;

namespace {

constexpr int kPartThreads = 256;
constexpr int kRing = 8;   // record slots in flight
constexpr int kAhead = 3;  // gathers issued this many blocks ahead
static_assert(kRing >= 2 * kAhead + 1, "a gather needs its record landed");

struct RecHdr {
  int nrows, nent, ngather, slot0;
};

__host__ __device__ __forceinline__ int a16(int b) { return (b + 15) & ~15; }

// Section offsets of a block record (identical on host and device).
struct RecLayout {
  int row_beg, gsrc, ref, val, dinv, bytes;
  __host__ __device__ RecLayout(const RecHdr& h, int tsize, bool unit) {
    row_beg = 16;
    gsrc = row_beg + a16(4 * (h.nrows + 1));
    ref = gsrc + a16(4 * h.ngather);
    val = ref + a16(4 * h.nent);
    dinv = val + a16(tsize * h.nent);
    bytes = dinv + (unit ? 0 : a16(tsize * h.nrows));
  }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
__global__ void __launch_bounds__(kPartThreads, 1)
    part_sweep_kernel(const int32_t* __restrict__ part_blk, const int32_t* __restrict__ blk_off16,
                      const unsigned char* __restrict__ recs, int vals_bytes, int offs_bytes,
                      int slot_bytes, int unit_diag, const T* __restrict__ in, T* out, int* err,
                      long long limit, const int* skip) {
  if (skip && ld_relaxed(skip)) return;
  extern __shared__ __align__(16) unsigned char sm[];
  T* vals = reinterpret_cast<T*>(sm);
  int32_t* offs = reinterpret_cast<int32_t*>(sm + vals_bytes);
  unsigned char* ring = sm + vals_bytes + offs_bytes;
  const int tid = threadIdx.x;
  const int b0 = part_blk[blockIdx.x];
  const int nb = part_blk[blockIdx.x + 1] - b0;
  for (int i = tid; i <= nb; i += kPartThreads) offs[i] = blk_off16[b0 + i];
  __syncthreads();

  auto slot = [&](int k) { return ring + (k % kRing) * slot_bytes; };
  auto copy_rec = [&](int k) {
    const unsigned char* src = recs + (size_t)offs[k] * 16;
    const int chunks = offs[k + 1] - offs[k];
    unsigned char* dst = slot(k);
    for (int c = tid; c < chunks; c += kPartThreads) cp_async16(dst + 16 * c, src + 16 * c);
  };
  auto gather = [&](int k) {
    unsigned char* s = slot(k);
    const RecHdr h = *reinterpret_cast<const RecHdr*>(s);
    const RecLayout L(h, (int)sizeof(T), unit_diag != 0);
    const int* gsrc = reinterpret_cast<const int*>(s + L.gsrc);
    unsigned char* g = s + L.bytes;
    for (int i = tid; i < h.ngather; i += kPartThreads) {
      const T* p = (i < h.nrows ? in : out) + gsrc[i];
      cp_async16(g + 16 * i,
                 reinterpret_cast<const void*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15)));
    }
  };

  // prologue: records of blocks 0 .. kRing-2, then the first kAhead gathers
  for (int k = 0; k < kRing - 1 && k < nb; ++k) copy_rec(k);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int k = 0; k < kAhead; ++k) {
    if (k < nb) gather(k);
    cp_async_commit();
  }

  for (int t = 0; t < nb; ++t) {
    // Block t's gathers (and, earlier, its record) have landed, and every
    // thread is done with block t-1, whose slot is refilled next.
    cp_async_wait<kAhead - 1>();
    __syncthreads();
    if (t + kRing - 1 < nb) copy_rec(t + kRing - 1);
    if (t + kAhead < nb) gather(t + kAhead);
    cp_async_commit();

    const unsigned char* s = slot(t);
    const RecHdr h = *reinterpret_cast<const RecHdr*>(s);
    if (tid < h.nrows) {
      const RecLayout L(h, (int)sizeof(T), unit_diag != 0);
      const int* row_beg = reinterpret_cast<const int*>(s + L.row_beg);
      const int* gsrc = reinterpret_cast<const int*>(s + L.gsrc);
      const int* ref = reinterpret_cast<const int*>(s + L.ref);
      const T* val = reinterpret_cast<const T*>(s + L.val);
      const unsigned char* g = s + L.bytes;
      auto gathered = [&](int i) -> T {
        const T* p = (i < h.nrows ? in : out) + gsrc[i];
        return *reinterpret_cast<const T*>(g + 16 * i + (reinterpret_cast<uintptr_t>(p) & 15));
      };
      T rr = gathered(tid);
      const int e1 = row_beg[tid + 1];
      for (int e = row_beg[tid]; e < e1; ++e) {
        const int r = ref[e];
        T w;
        if (r >= 0) {
          w = vals[r];
        } else {
          const int gi = -r - 1;
          w = gathered(gi);
          if (Box<T>::is(w)) w = wait_value(out + gsrc[gi], limit, err);
        }
        rr = sub_rn(rr, mul_rn(val[e], w));
      }
      if (!unit_diag) rr = mul_rn(rr, reinterpret_cast<const T*>(s + L.dinv)[tid]);
      rr = canonical(rr);
      vals[h.slot0 + tid] = rr;
      st_relaxed(out + gsrc[tid], rr);
    }
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Host-side partitioning.

int env_int(const char* name, int dflt) {
  const char* s = std::getenv(name);
  return (s && *s) ? std::atoi(s) : dflt;
}

// Recursive bisection of the chain graph (CSR adj_ptr/adj) into `parts`
// parts balanced by row count (len); result in part_of[chain].
struct Bisector {
  const std::vector<int>& adj_ptr;
  const std::vector<int>& adj;
  const std::vector<int>& len;
  std::vector<int>& part_of;
  std::vector<int> member, seen;
  int stamp = 0;

  Bisector(const std::vector<int>& ap, const std::vector<int>& a, const std::vector<int>& l,
           std::vector<int>& po)
      : adj_ptr(ap), adj(a), len(l), part_of(po), member(l.size(), -1), seen(l.size(), -1) {}

  // BFS order over the members of set `set_id` from `start`, continuing from
  // the next unvisited member (in `nodes` order) when a component runs out.
  void bfs(const std::vector<int>& nodes, int set_id, int start, std::vector<int>& order) {
    const int vs = ++stamp;
    order.clear();
    size_t head = 0, next_unvisited = 0;
    auto push = [&](int c) {
      seen[c] = vs;
      order.push_back(c);
    };
    push(start);
    while (order.size() < nodes.size()) {
      if (head == order.size()) {
        while (seen[nodes[next_unvisited]] == vs) ++next_unvisited;
        push(nodes[next_unvisited]);
      }
      const int c = order[head++];
      for (int k = adj_ptr[c]; k < adj_ptr[c + 1]; ++k) {
        const int d = adj[k];
        if (member[d] == set_id && seen[d] != vs) push(d);
      }
    }
  }

  void run(std::vector<int>& nodes, int parts, int first, int& set_counter) {
    if (parts <= 1 || nodes.size() <= 1) {
      for (int c : nodes) part_of[c] = first;
      return;
    }
    const int set_id = ++set_counter;
    for (int c : nodes) member[c] = set_id;
    std::vector<int> order;
    // pseudo-peripheral start: BFS sweeps from the first node
    bfs(nodes, set_id, nodes[0], order);
    bfs(nodes, set_id, order.back(), order);
    bfs(nodes, set_id, order.back(), order);
    long long total = 0;
    for (int c : nodes) total += len[c];
    const int p1 = parts / 2;
    const long long target = total * p1 / parts;
    std::vector<int> a, b;
    long long acc = 0;
    for (int c : order) {
      if (a.empty() || (b.empty() && acc + len[c] / 2 <= target)) {
        a.push_back(c);
        acc += len[c];
      } else {
        b.push_back(c);
      }
    }
    if (b.empty()) {
      b.push_back(a.back());
      a.pop_back();
    }
    std::vector<int>().swap(nodes);
    std::vector<int>().swap(order);
    run(a, p1, first, set_counter);
    run(b, parts - p1, first + p1, set_counter);
  }
};

}  // namespace

// Host side of the partitioning: the level-ordered plan in, block records
// out (pure host code; part_plan_build copies the plan down and the records
// up).  Returns false when a part or a row does not fit shared memory.
struct PartInput {
  int n = 0, n_levels = 0;
  bool unit_diag = false, with_fp32 = false;
  const int32_t *lp = nullptr, *row_of = nullptr, *rp = nullptr, *ci = nullptr;
  const double *val = nullptr, *dinv = nullptr;
  int num_sms = 148, rows_per_part = 16384, smem_optin = 232448;
};
struct HostPart {
  int P = 0, max_rows = 0;
  long long ext_entries = 0;
  struct Prec {
    int vals_bytes = 0, offs_bytes = 0, slot_bytes = 0, smem_bytes = 0;
    std::vector<unsigned char> stream;
    std::vector<int32_t> blk_off16, part_blk;
  } prec[2];
};

bool part_plan_host(const PartInput& in, HostPart* out) {
  const int n = in.n;
  std::vector<int32_t> pos_of(n), lev(n);
  for (int p = 0; p < n; ++p) pos_of[in.row_of[p]] = p;
  for (int l = 0; l < in.n_levels; ++l)
    for (int p = in.lp[l]; p < in.lp[l + 1]; ++p) lev[p] = l;

  const int rows_per_part = std::max(64, in.rows_per_part);
  int P = (int)std::min<long long>(in.num_sms, ((long long)n + rows_per_part - 1) / rows_per_part);
  P = std::max(1, P);
  const int max_chain = std::max(1, ((n + P - 1) / P) / 4);

  // 1. chains
  std::vector<int> chain_of(n), tail, clen;
  for (int p = 0; p < n; ++p) {
    const int r = in.row_of[p];
    int best = -1;
    long long best_dist = -1;
    for (int e = in.rp[p]; e < in.rp[p + 1]; ++e) {
      const int q = pos_of[in.ci[e]];
      if (lev[q] != lev[p] - 1) continue;
      const int ch = chain_of[q];
      if (tail[ch] != q || clen[ch] >= max_chain) continue;
      const long long dist = std::llabs((long long)in.ci[e] - r);
      if (dist > best_dist) best_dist = dist, best = ch;
    }
    if (best < 0) {
      best = (int)tail.size();
      tail.push_back(p);
      clen.push_back(0);
    }
    chain_of[p] = best;
    tail[best] = p;
    clen[best]++;
  }
  const int nc = (int)tail.size();

  // 2. chain adjacency (unique neighbours, both directions)
  std::vector<int> cptr(nc + 1, 0), crows(n);
  for (int p = 0; p < n; ++p) cptr[chain_of[p] + 1]++;
  for (int c = 0; c < nc; ++c) cptr[c + 1] += cptr[c];
  {
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int p = 0; p < n; ++p) crows[fill[chain_of[p]]++] = p;
  }
  std::vector<int> mark(nc, -1), out_ptr(nc + 1, 0), out_adj;
  for (int c = 0; c < nc; ++c) {
    for (int k = cptr[c]; k < cptr[c + 1]; ++k) {
      const int p = crows[k];
      for (int e = in.rp[p]; e < in.rp[p + 1]; ++e) {
        const int d = chain_of[pos_of[in.ci[e]]];
        if (d != c && mark[d] != c) {
          mark[d] = c;
          out_adj.push_back(d);
        }
      }
    }
    out_ptr[c + 1] = (int)out_adj.size();
  }
  std::vector<int> in_ptr(nc + 1, 0), in_adj(out_adj.size());
  for (int d : out_adj) in_ptr[d + 1]++;
  for (int c = 0; c < nc; ++c) in_ptr[c + 1] += in_ptr[c];
  {
    std::vector<int> fill(in_ptr.begin(), in_ptr.end() - 1);
    for (int c = 0; c < nc; ++c)
      for (int k = out_ptr[c]; k < out_ptr[c + 1]; ++k) in_adj[fill[out_adj[k]]++] = c;
  }
  std::vector<int> adj_ptr(nc + 1, 0), adj;
  std::fill(mark.begin(), mark.end(), -1);
  for (int c = 0; c < nc; ++c) {
    for (int k = out_ptr[c]; k < out_ptr[c + 1]; ++k)
      if (mark[out_adj[k]] != c) mark[out_adj[k]] = c, adj.push_back(out_adj[k]);
    for (int k = in_ptr[c]; k < in_ptr[c + 1]; ++k)
      if (mark[in_adj[k]] != c) mark[in_adj[k]] = c, adj.push_back(in_adj[k]);
    adj_ptr[c + 1] = (int)adj.size();
  }
  std::vector<int>().swap(out_adj);
  std::vector<int>().swap(in_adj);

  // 3. parts
  std::vector<int> part_of_chain(nc, 0);
  {
    std::vector<int> nodes(nc);
    for (int c = 0; c < nc; ++c) nodes[c] = c;
    Bisector B(adj_ptr, adj, clen, part_of_chain);
    int sets = 0;
    B.run(nodes, P, 0, sets);
  }

  // 4. rows of each part in level order (plan order is level order); slots
  std::vector<int> part_ptr(P + 1, 0), part_rows(n), slot_of(n), part_of(n);
  for (int p = 0; p < n; ++p) part_of[p] = part_of_chain[chain_of[p]];
  for (int p = 0; p < n; ++p) part_ptr[part_of[p] + 1]++;
  for (int q = 0; q < P; ++q) part_ptr[q + 1] += part_ptr[q];
  {
    std::vector<int> fill(part_ptr.begin(), part_ptr.end() - 1);
    for (int p = 0; p < n; ++p) {
      slot_of[p] = fill[part_of[p]] - part_ptr[part_of[p]];
      part_rows[fill[part_of[p]]++] = p;
    }
  }
  int max_rows = 0;
  for (int q = 0; q < P; ++q) max_rows = std::max(max_rows, part_ptr[q + 1] - part_ptr[q]);

  const int smem_optin = in.smem_optin;
  out->P = P;
  out->max_rows = max_rows;
  long long ext_entries = 0;

  // 5. block records, per precision.  A slot holds one block's record and,
  // right after it, the block's gather area (16 bytes per gathered value).
  for (int prec = 0; prec < (in.with_fp32 ? 2 : 1); ++prec) {
    const int ts = prec == 0 ? 8 : 4;
    const int vals_bytes = a16(max_rows * ts);
    int offs_bytes = 8192;
    bool ok = false;
    std::vector<unsigned char> stream;
    std::vector<int32_t> blk_off16, part_blk;
    int slot_bytes = 0;
    for (int attempt = 0; attempt < 3 && !ok; ++attempt) {
      slot_bytes = ((smem_optin - vals_bytes - offs_bytes - 1024) / kRing) & ~15;
      if (slot_bytes < 2048) break;
      stream.clear();
      blk_off16.assign(1, 0);
      part_blk.assign(1, 0);
      ext_entries = 0;
      int max_blocks = 0;
      bool fits = true;
      for (int q = 0; q < P && fits; ++q) {
        int nblk = 0;
        for (int i = part_ptr[q], iend = part_ptr[q + 1]; i < iend;) {
          // grow a block from row i: one level, <= kPartThreads rows, fits a slot
          RecHdr h{0, 0, 0, i - part_ptr[q]};
          int j = i;
          const int l0 = lev[part_rows[i]];
          while (j < iend && h.nrows < kPartThreads && lev[part_rows[j]] == l0) {
            const int p = part_rows[j];
            int ext = 0;
            for (int e = in.rp[p]; e < in.rp[p + 1]; ++e) ext += part_of[pos_of[in.ci[e]]] != q;
            const RecHdr t{h.nrows + 1, h.nent + in.rp[p + 1] - in.rp[p], h.ngather + 1 + ext, h.slot0};
            if (RecLayout(t, ts, in.unit_diag).bytes + 16 * t.ngather > slot_bytes) break;
            h = t;
            ++j;
          }
          if (j == i) {  // one row alone does not fit a slot
            fits = false;
            break;
          }
          const RecLayout L(h, ts, in.unit_diag);
          const size_t base = stream.size();
          stream.resize(base + L.bytes, 0);
          unsigned char* rec = stream.data() + base;
          std::memcpy(rec, &h, sizeof(h));
          int32_t* rb = reinterpret_cast<int32_t*>(rec + L.row_beg);
          int32_t* gs = reinterpret_cast<int32_t*>(rec + L.gsrc);
          int32_t* rf = reinterpret_cast<int32_t*>(rec + L.ref);
          // gather list: the rows' own right-hand sides first, then externals
          int ne = 0, ng = h.nrows;
          for (int k = 0; k < h.nrows; ++k) {
            const int p = part_rows[i + k];
            rb[k] = ne;
            gs[k] = in.row_of[p];
            for (int e = in.rp[p]; e < in.rp[p + 1]; ++e, ++ne) {
              const int qd = pos_of[in.ci[e]];
              if (part_of[qd] == q) {
                rf[ne] = slot_of[qd];
              } else {
                gs[ng] = in.ci[e];
                rf[ne] = -(ng + 1);
                ++ng;
              }
              if (ts == 8)
                reinterpret_cast<double*>(rec + L.val)[ne] = in.val[e];
              else
                reinterpret_cast<float*>(rec + L.val)[ne] = (float)in.val[e];
            }
            if (!in.unit_diag) {
              if (ts == 8)
                reinterpret_cast<double*>(rec + L.dinv)[k] = in.dinv[p];
              else
                reinterpret_cast<float*>(rec + L.dinv)[k] = (float)in.dinv[p];
            }
          }
          rb[h.nrows] = ne;
          ext_entries += ng - h.nrows;
          blk_off16.push_back((int32_t)(stream.size() / 16));
          ++nblk;
          i = j;
        }
        max_blocks = std::max(max_blocks, nblk);
        part_blk.push_back(part_blk.back() + nblk);
      }
      if (!fits || stream.size() / 16 >= (size_t)INT32_MAX) break;
      const int need_offs = a16(4 * (max_blocks + 1));
      if (need_offs > offs_bytes) {
        offs_bytes = need_offs;  // retry with a smaller ring
        continue;
      }
      ok = true;
    }
    const int smem = vals_bytes + offs_bytes + kRing * slot_bytes;
    if (!ok || smem > smem_optin) return false;
    HostPart::Prec& V = out->prec[prec];
    V.vals_bytes = vals_bytes;
    V.offs_bytes = offs_bytes;
    V.slot_bytes = slot_bytes;
    V.smem_bytes = smem;
    V.stream.swap(stream);
    V.blk_off16.swap(blk_off16);
    V.part_blk.swap(part_blk);
    out->ext_entries = ext_entries;
  }
  return true;
}

// Built at preconditioner creation (outside any stream capture).
mtlgpu_status part_plan_build(Ctx* ctx, SweepPlan* S, bool with_fp32) {
  part_plan_free(ctx, S);
  if (!ctx->part_sweeps) return MTLGPU_OK;
  const int n = S->n;
  if (n == 0) return MTLGPU_OK;

  // host copies of the level-ordered plan
  std::vector<int32_t> lp(S->n_levels + 1), row_of(n), rp(n + 1), ci(S->nnz_off);
  std::vector<double> val(S->nnz_off), dinv(S->unit_diag ? 0 : n);
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(lp.data(), S->d_level_ptr, 4 * lp.size(),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(row_of.data(), S->d_row_of, 4 * (size_t)n,
                                       cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(rp.data(), S->d_rp, 4 * (size_t)(n + 1),
                                       cudaMemcpyDeviceToHost, ctx->stream));
  if (S->nnz_off) {
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(ci.data(), S->d_ci, 4 * ci.size(), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(val.data(), S->d_val, 8 * val.size(),
                                         cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (!S->unit_diag)
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(dinv.data(), S->d_dinv, 8 * (size_t)n,
                                         cudaMemcpyDeviceToHost, ctx->stream));
  MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

  PartInput in;
  in.n = n;
  in.n_levels = S->n_levels;
  in.unit_diag = S->unit_diag;
  in.with_fp32 = with_fp32;
  in.lp = lp.data();
  in.row_of = row_of.data();
  in.rp = rp.data();
  in.ci = ci.data();
  in.val = val.data();
  in.dinv = dinv.data();
  in.num_sms = ctx->num_sms;
  in.rows_per_part = ctx->part_rows;
  MTLGPU_TRY_CUDA(ctx, cudaDeviceGetAttribute(&in.smem_optin,
                                              cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  HostPart H;
  if (!part_plan_host(in, &H)) return MTLGPU_OK;  // sweeps keep the ticket kernel

  PartPlan* PP = new PartPlan();
  PP->P = H.P;
  PP->max_rows = H.max_rows;
  PP->ext_entries = H.ext_entries;
  for (int prec = 0; prec < (with_fp32 ? 2 : 1); ++prec) {
    HostPart::Prec& hp = H.prec[prec];
    auto& V = PP->prec[prec];
    V.vals_bytes = hp.vals_bytes;
    V.offs_bytes = hp.offs_bytes;
    V.slot_bytes = hp.slot_bytes;
    V.smem_bytes = hp.smem_bytes;
    V.n_blocks = (int)hp.blk_off16.size() - 1;
    mtlgpu_status st = MTLGPU_OK;
    if ((st = dalloc(ctx, &V.d_blk_off16, hp.blk_off16.size())) != MTLGPU_OK ||
        (st = dalloc(ctx, &V.d_rec, hp.stream.size())) != MTLGPU_OK ||
        (st = dalloc(ctx, &V.d_part_blk, hp.part_blk.size())) != MTLGPU_OK) {
      S->part = PP;
      part_plan_free(ctx, S);
      return st;
    }
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(V.d_blk_off16, hp.blk_off16.data(),
                                         4 * hp.blk_off16.size(), cudaMemcpyHostToDevice,
                                         ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(V.d_rec, hp.stream.data(), hp.stream.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
    MTLGPU_TRY_CUDA(ctx, cudaMemcpyAsync(V.d_part_blk, hp.part_blk.data(), 4 * hp.part_blk.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
    int occ = 0;
    if (prec == 0) {
      MTLGPU_TRY_CUDA(ctx, cudaFuncSetAttribute(part_sweep_kernel<double>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                in.smem_optin));
      MTLGPU_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &occ, part_sweep_kernel<double>, kPartThreads, V.smem_bytes));
    } else {
      MTLGPU_TRY_CUDA(ctx, cudaFuncSetAttribute(part_sweep_kernel<float>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                in.smem_optin));
      MTLGPU_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &occ, part_sweep_kernel<float>, kPartThreads, V.smem_bytes));
    }
    MTLGPU_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // host buffers die after this
    // one resident CTA per part, all at once
    V.ready = occ >= 1 && (long long)occ * ctx->num_sms >= PP->P;
    if (!V.ready) part_plan_free_one(ctx, PP, prec);
  }
  S->part = PP;
  return MTLGPU_OK;
}

void part_plan_free_one(Ctx* ctx, PartPlan* PP, int prec) {
  auto& V = PP->prec[prec];
  dfree(ctx, V.d_blk_off16);
  dfree(ctx, V.d_rec);
  dfree(ctx, V.d_part_blk);
  V.ready = false;
}

void part_plan_free(Ctx* ctx, SweepPlan* S) {
  if (!S->part) return;
  part_plan_free_one(ctx, S->part, 0);
  part_plan_free_one(ctx, S->part, 1);
  delete S->part;
  S->part = nullptr;
}

template <typename T>
bool part_sweep_ready(const SweepPlan& S) {
  return S.part && S.part->prec[sizeof(T) == 8 ? 0 : 1].ready;
}

template <typename T>
mtlgpu_status part_sweep_launch(Ctx* ctx, const SweepPlan& S, const T* in, T* out,
                                const int* skip) {
  const auto& V = S.part->prec[sizeof(T) == 8 ? 0 : 1];
  ctx->launches++;
  part_sweep_kernel<T><<<S.part->P, kPartThreads, V.smem_bytes, ctx->stream>>>(
      V.d_part_blk, V.d_blk_off16, V.d_rec, V.vals_bytes, V.offs_bytes, V.slot_bytes,
      S.unit_diag ? 1 : 0, in, out, ctx->d_error, ctx->spin_limit, skip);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template bool part_sweep_ready<double>(const SweepPlan&);
template bool part_sweep_ready<float>(const SweepPlan&);
template mtlgpu_status part_sweep_launch<double>(Ctx*, const SweepPlan&, const double*, double*,
                                                 const int*);
template mtlgpu_status part_sweep_launch<float>(Ctx*, const SweepPlan&, const float*, float*,
                                                const int*);

}  // namespace mtlgpu
