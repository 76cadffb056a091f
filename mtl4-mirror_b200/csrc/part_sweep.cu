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
//   2. parts: two topological orders of the chain dependency graph cut
//      into strips and tiles, balanced by row count, so that dependencies
//      between parts all point forward (no two parts wait on each other in
//      turn).
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
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "internal.h"
#include "tma.cuh"

namespace mtlgpu {

using namespace dev;

namespace {

// Automatic selection: partitioned sweeps for factors with at most this many
// rows per level.
constexpr int kAutoRowsPerLevel = 1024;

constexpr int kPartThreads = 256;   // consumer threads: rows per block at most
constexpr int kProducers = 64;      // producer threads (two warps): copies and gathers
constexpr int kCtaThreads = kPartThreads + kProducers;
// Ring depth per value type: kRing record slots in flight, gathers issued
// kAhead blocks ahead (a gather needs its record landed: kRing >= 2 kAhead).
// FP64 values take more shared memory, which leaves room for fewer slots.
template <typename T> struct Ring;
template <> struct Ring<double> { static constexpr int kRing = 10, kAhead = 5; };
template <> struct Ring<float> { static constexpr int kRing = 16, kAhead = 8; };
static_assert(Ring<double>::kRing >= 2 * Ring<double>::kAhead, "ring too shallow");
static_assert(Ring<float>::kRing >= 2 * Ring<float>::kAhead, "ring too shallow");
constexpr int kRegEnt = 4;  // entries per row held in registers (more: read from the slot)

// Block record: a 48-byte header, then structure-of-arrays sections whose
// byte offsets the header holds (0: absent), all 16-byte aligned:
//   out[nrows]        natural index of each row (right-hand side and result)
//   ref[K][nrows]     first K entries of each row: >= 0 slot of a value of
//                     this part; kNoEntry: padding; else -(1 + 4 e + lane):
//                     lane of the e-th gathered 16-byte chunk of `out`
//   val[K][nrows]     their values
//   dia[nrows]        inverted diagonal (absent for a unit diagonal)
//   over[nrows]       entries beyond K: (start << 8) | count in the lists
//   over_ref[nover], over_val[nover]
//   gext[next]        natural index of each external value
// A slot holds the record and then its gather area: rhs[nrows] (element
// size) and next 16-byte chunks.
struct RecHdr {
  int nrows, next, nover, slot0;
  int off_ref, off_val, off_dia, off_over;
  int off_gext, bytes, K, pad;
};
static_assert(sizeof(RecHdr) == 48, "record header is three 16-byte words");
constexpr int kNoEntry = INT32_MIN;

__host__ __device__ __forceinline__ int a16(int b) { return (b + 15) & ~15; }

// Fills the section offsets of h from its counts.
__host__ __device__ inline void rec_layout(RecHdr& h, int ts, bool unit) {
  int o = 48 + a16(4 * h.nrows);
  h.off_ref = o;
  o += a16(4 * h.K * h.nrows);
  h.off_val = o;
  o += a16(ts * h.K * h.nrows);
  h.off_dia = unit ? 0 : o;
  if (!unit) o += a16(ts * h.nrows);
  h.off_over = h.nover ? o : 0;
  if (h.nover) o += a16(4 * h.nrows) + a16(4 * h.nover) + a16(ts * h.nover);
  h.off_gext = o;
  o += a16(4 * h.next);
  h.bytes = o;
}
__host__ __device__ __forceinline__ int slot_need(const RecHdr& h, int ts) {
  return h.bytes + a16(ts * h.nrows) + 16 * h.next;
}

__device__ __forceinline__ void consumer_sync() {  // the kPartThreads consumer threads only
  asm volatile("bar.sync 1, %0;" ::"n"(kPartThreads) : "memory");
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

template <typename T>
__global__ void __launch_bounds__(kCtaThreads, 1)
    part_sweep_kernel(const int32_t* __restrict__ part_blk, const int32_t* __restrict__ blk_off16,
                      const unsigned char* __restrict__ recs, int vals_bytes, int offs_bytes,
                      int slot_bytes, const T* __restrict__ in, T* out, int* err,
                      long long limit, const int* skip) {
  constexpr int kRing = Ring<T>::kRing, kAhead = Ring<T>::kAhead;
  constexpr int kTs = (int)sizeof(T);
  if (skip && ld_relaxed(skip)) return;
  extern __shared__ __align__(16) unsigned char sm[];
  // Per slot: rec_full (its record copied), full (record and gathers landed),
  // empty (every consumer warp done with it).
  __shared__ unsigned long long rec_full[kRing], full[kRing], empty[kRing];
  __shared__ int abort_flag;
  T* vals = reinterpret_cast<T*>(sm);
  int32_t* offs = reinterpret_cast<int32_t*>(sm + vals_bytes);
  unsigned char* ring = sm + vals_bytes + offs_bytes;
  const int tid = threadIdx.x;
  const int b0 = part_blk[blockIdx.x];
  const int nb = part_blk[blockIdx.x + 1] - b0;
  for (int i = tid; i <= nb; i += kCtaThreads) offs[i] = blk_off16[b0 + i];
  if (tid < kRing) {
    mbar_init(&rec_full[tid], 1);
    mbar_init(&full[tid], kProducers);
    mbar_init(&empty[tid], kPartThreads / 32);
    // make the initialised barriers visible to the bulk-copy (async) proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (tid == 0) abort_flag = 0;
  __syncthreads();
  auto slot = [&](int k) { return ring + (k % kRing) * slot_bytes; };

  if (tid >= kPartThreads) {
    // ---- producer warps: records kRing blocks ahead of the consumers, the
    // gathers of a block kAhead loop steps after its record
    const int pt = tid - kPartThreads;
    int last_rec = -1;  // pt 0: last record whose bulk copy was issued
    for (int k = 0; k < nb + kAhead; ++k) {
      if (k < nb) {
        if (k >= kRing && !mbar_wait(&empty[k % kRing], ((k / kRing) - 1) & 1, limit)) {
          atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
          abort_flag = 1;
          break;
        }
        if (pt == 0) {  // the record: one bulk copy
          const unsigned bytes = (unsigned)(offs[k + 1] - offs[k]) * 16u;
          mbar_arrive_expect_tx(&rec_full[k % kRing], bytes);
          bulk_copy_g2s(slot(k), recs + (size_t)offs[k] * 16, bytes, &rec_full[k % kRing]);
          last_rec = k;
        }
      }
      const int j = k - kAhead;
      if (j >= 0) {
        if (!mbar_wait(&rec_full[j % kRing], (j / kRing) & 1, limit)) {
          atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
          abort_flag = 1;
          break;
        }
        // right-hand sides at element size (the input is not written during
        // the sweep), external values as 16-byte chunks through L2
        unsigned char* s = slot(j);
        const RecHdr& h = *reinterpret_cast<const RecHdr*>(s);
        const int nrows = h.nrows, ng = h.nrows + h.next;
        const int* orow = reinterpret_cast<const int*>(s + 48);
        const int* gext = reinterpret_cast<const int*>(s + h.off_gext);
        unsigned char* g = s + h.bytes;
        unsigned char* ge = g + a16(kTs * nrows) - 16 * nrows;
        for (int i = pt; i < ng; i += kProducers) {
          if (i < nrows)
            cp_async_ca<kTs>(g + kTs * i, in + orow[i]);
          else
            cp_async16(ge + 16 * i, reinterpret_cast<const void*>(
                                        reinterpret_cast<uintptr_t>(out + gext[i - nrows]) &
                                        ~uintptr_t(15)));
        }
        mbar_arrive_cp_async(&full[j % kRing]);
      }
    }
    // After an abort, record copies may still be in flight into this CTA's
    // shared memory: the issuing thread waits for the last phase of every
    // slot it filled before leaving (shared memory stays valid while any
    // thread of the CTA runs).  On a normal exit those phases have completed
    // and each wait returns at once.  A global -> shared bulk copy always
    // completes; the wait is still bounded, by at least 2^24 polls.
    if (pt == 0) {
      const long long drain = limit > (1ll << 24) ? limit : (1ll << 24);
      for (int k = last_rec - kRing + 1 > 0 ? last_rec - kRing + 1 : 0; k <= last_rec; ++k)
        mbar_wait(&rec_full[k % kRing], (unsigned)(k / kRing) & 1u, drain);
    }
    cp_async_wait<0>();
    return;
  }

  // ---- consumer warps: one row per thread and block
  const int lane = tid & 31;
  struct Row {
    int nrows = 0, slot0 = 0, out_idx = 0, over = 0;
    T rhs = T(0), dia = T(1);
    int ref[kRegEnt];
    T val[kRegEnt];
    T wext[kRegEnt];  // prefetched external value (sentinel: not ready then)
  };
  // Block k's row for this thread, into registers before the block's barrier.
  auto load_row = [&](int k, Row& R) {
    const unsigned char* s = slot(k);
    const RecHdr h = *reinterpret_cast<const RecHdr*>(s);
    R.nrows = h.nrows;
    R.slot0 = h.slot0;
    if (tid >= h.nrows) return;
    R.out_idx = reinterpret_cast<const int*>(s + 48)[tid];
    R.rhs = reinterpret_cast<const T*>(s + h.bytes)[tid];
    R.dia = h.off_dia ? reinterpret_cast<const T*>(s + h.off_dia)[tid] : T(1);
    R.over = h.off_over ? reinterpret_cast<const int*>(s + h.off_over)[tid] : 0;
    const int* ref = reinterpret_cast<const int*>(s + h.off_ref) + tid;
    const T* val = reinterpret_cast<const T*>(s + h.off_val) + tid;
    const unsigned char* ge = s + h.bytes + a16(kTs * h.nrows);
#pragma unroll
    for (int q = 0; q < kRegEnt; ++q) {
      R.ref[q] = kNoEntry;
      if (q < h.K) {
        const int r = ref[q * h.nrows];
        R.ref[q] = r;
        R.val[q] = val[q * h.nrows];
        if (r < 0 && r != kNoEntry) {
          const int code = -r - 1;
          R.wext[q] = reinterpret_cast<const T*>(ge + 16 * (code >> 2))[code & 3];
        }
      }
    }
  };

  Row R;
  if (nb > 0) {
    if (!(mbar_wait(&rec_full[0], 0, limit) && mbar_wait(&full[0], 0, limit))) {
      atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
      abort_flag = 1;
    }
    consumer_sync();
    if (!abort_flag) load_row(0, R);
  }
  for (int t = 0; t < nb; ++t) {
    // Block t+1 has landed; the values of block t-1 are in shared memory.
    if (t + 1 < nb && !(mbar_wait(&rec_full[(t + 1) % kRing], ((t + 1) / kRing) & 1, limit) &&
                        mbar_wait(&full[(t + 1) % kRing], ((t + 1) / kRing) & 1, limit))) {
      atomicCAS(err, 0, (int)MTLGPU_TIMEOUT);
      abort_flag = 1;
    }
    consumer_sync();
    if (abort_flag) break;
    if (tid < R.nrows) {
      T w[kRegEnt];
#pragma unroll
      for (int q = 0; q < kRegEnt; ++q) w[q] = R.ref[q] >= 0 ? vals[R.ref[q]] : R.wext[q];
      T rr = R.rhs;
#pragma unroll
      for (int q = 0; q < kRegEnt; ++q) {
        if (R.ref[q] != kNoEntry) {
          if (R.ref[q] < 0 && Box<T>::is(w[q])) {  // not ready when gathered: poll
            const unsigned char* s = slot(t);
            const int e = (-R.ref[q] - 1) >> 2;
            const int off_gext = reinterpret_cast<const RecHdr*>(s)->off_gext;
            w[q] = wait_value(out + reinterpret_cast<const int*>(s + off_gext)[e], limit, err);
          }
          rr = sub_rn(rr, mul_rn(R.val[q], w[q]));
        }
      }
      if (R.over) {  // entries beyond K, straight from the slot
        const unsigned char* s = slot(t);
        const RecHdr& h = *reinterpret_cast<const RecHdr*>(s);
        const int* oref = reinterpret_cast<const int*>(s + h.off_over + a16(4 * h.nrows));
        const T* oval =
            reinterpret_cast<const T*>(s + h.off_over + a16(4 * h.nrows) + a16(4 * h.nover));
        const int* gext = reinterpret_cast<const int*>(s + h.off_gext);
        const unsigned char* ge = s + h.bytes + a16(kTs * h.nrows);
        const int e0 = R.over >> 8, e1 = e0 + (R.over & 255);
        for (int e = e0; e < e1; ++e) {
          const int r = oref[e];
          T wv;
          if (r >= 0) {
            wv = vals[r];
          } else {
            const int code = -r - 1;
            wv = reinterpret_cast<const T*>(ge + 16 * (code >> 2))[code & 3];
            if (Box<T>::is(wv)) wv = wait_value(out + gext[code >> 2], limit, err);
          }
          rr = sub_rn(rr, mul_rn(oval[e], wv));
        }
      }
      rr = canonical(mul_rn(rr, R.dia));
      vals[R.slot0 + tid] = rr;
      st_relaxed(out + R.out_idx, rr);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[t % kRing]);  // this warp is done with slot t
    if (t + 1 < nb) load_row(t + 1, R);
  }
}

// ---------------------------------------------------------------------------
// Host-side partitioning.

int env_int(const char* name, int dflt) {
  const char* s = std::getenv(name);
  return (s && *s) ? std::atoi(s) : dflt;
}

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
  // optional: the part of each row (natural index), e.g. from the geometry
  // the caller knows; parts are then 0 .. max+1 and chains are not formed
  const int32_t* part_of_row = nullptr;
};
struct HostPart {
  int P = 0, max_rows = 0, n_chains = 0;
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

  std::vector<int> part_of(n);
  if (in.part_of_row) {
    P = 0;
    for (int p = 0; p < n; ++p) P = std::max(P, in.part_of_row[in.row_of[p]] + 1);
    if (P > in.num_sms) return false;
    for (int p = 0; p < n; ++p) part_of[p] = in.part_of_row[in.row_of[p]];
  } else {
    // 1. chains.  Level by level, each row claims the chain ending at one of
    // its dependencies one level below; claims are granted farthest first
    // (largest |column - row|), so that on a grid in natural order the
    // chains are the pencils along the slowest index.
    std::vector<int> chain_of(n, -1), tail, clen;
    struct Claim {
      long long dist;
      int p, q;
    };
    std::vector<Claim> claims;
    for (int l = 0; l < in.n_levels; ++l) {
      claims.clear();
      for (int p = in.lp[l]; p < in.lp[l + 1]; ++p) {
        const int r = in.row_of[p];
        for (int e = in.rp[p]; e < in.rp[p + 1]; ++e) {
          const int q = pos_of[in.ci[e]];
          if (lev[q] == l - 1) claims.push_back({std::llabs((long long)in.ci[e] - r), p, q});
        }
      }
      std::stable_sort(claims.begin(), claims.end(),
                       [](const Claim& a, const Claim& b) { return a.dist > b.dist; });
      for (const Claim& c : claims) {
        if (chain_of[c.p] >= 0) continue;
        const int ch = chain_of[c.q];
        if (tail[ch] != c.q || clen[ch] >= max_chain) continue;
        chain_of[c.p] = ch;
        tail[ch] = c.p;
        clen[ch]++;
      }
      for (int p = in.lp[l]; p < in.lp[l + 1]; ++p) {
        if (chain_of[p] >= 0) continue;
        chain_of[p] = (int)tail.size();
        tail.push_back(p);
        clen.push_back(1);
      }
    }
    const int nc = (int)tail.size();

    // 2. chain dependency graph: out_adj[c] = chains that c's rows depend on,
    // in_adj[c] = chains depending on c (unique entries)
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

    // 3. parts.  Two topological orders of the chain dependency graph
    // (Kahn's algorithm taking, among the ready chains, the one whose first
    // row has the smallest index -- L1 -- or the largest -- L2; on a grid in
    // natural order these are the row-major and column-major orders of the
    // pencils).  sqrt(P) strips are cut along L1 and each strip into tiles
    // along L2, balanced by row count.  Every dependency then points to the
    // same or a later part, so neighbouring parts never wait on each other
    // in turn, and on a grid the tiles are rectangles whose boundaries a
    // dependency path crosses about 2 sqrt(P) times.
    std::vector<int> part_of_chain(nc, 0);
    {
      std::vector<int> head(nc);
      for (int p = n - 1; p >= 0; --p) head[chain_of[p]] = in.row_of[p];
      auto kahn = [&](bool smallest_first) {
        std::vector<int> rank(nc, -1), indeg(nc);
        for (int c = 0; c < nc; ++c) indeg[c] = out_ptr[c + 1] - out_ptr[c];
        auto cmp = [&](int a, int b) {  // heap order: top = next to take
          return smallest_first ? head[a] > head[b] : head[a] < head[b];
        };
        std::vector<int> heap;
        for (int c = 0; c < nc; ++c)
          if (indeg[c] == 0) heap.push_back(c);
        std::make_heap(heap.begin(), heap.end(), cmp);
        int next = 0, scan = 0;
        while (next < nc) {
          if (heap.empty()) {  // a cycle between chains: release the first one left
            while (rank[scan] >= 0) ++scan;
            indeg[scan] = 0;
            heap.push_back(scan);
          }
          std::pop_heap(heap.begin(), heap.end(), cmp);
          const int c = heap.back();
          heap.pop_back();
          if (rank[c] >= 0) continue;
          rank[c] = next++;
          for (int k = in_ptr[c]; k < in_ptr[c + 1]; ++k) {
            const int d = in_adj[k];
            if (rank[d] < 0 && --indeg[d] == 0) {
              heap.push_back(d);
              std::push_heap(heap.begin(), heap.end(), cmp);
            }
          }
        }
        return rank;
      };
      const std::vector<int> L1 = kahn(true), L2 = kahn(false);
      std::vector<int> order(nc);
      for (int c = 0; c < nc; ++c) order[L1[c]] = c;
      long long total = 0;
      for (int c = 0; c < nc; ++c) total += clen[c];
      const int S = std::max(1, std::min(P, (int)std::lround(std::sqrt((double)P))));
      size_t pos = 0;
      int first_part = 0;
      long long done_rows = 0;
      for (int st = 0; st < S; ++st) {
        const int ps = P / S + (st < P % S ? 1 : 0);
        const long long strip_end = total * (first_part + ps) / P;
        std::vector<int> strip;
        while (pos < order.size() &&
               (strip.empty() || st == S - 1 || done_rows + clen[order[pos]] / 2 <= strip_end)) {
          strip.push_back(order[pos]);
          done_rows += clen[order[pos]];
          ++pos;
        }
        std::sort(strip.begin(), strip.end(), [&](int a, int b) { return L2[a] < L2[b]; });
        long long sw = 0, acc = 0;
        for (int c : strip) sw += clen[c];
        int k = 0;
        for (int c : strip) {
          while (k < ps - 1 && acc + clen[c] / 2 > sw * (k + 1) / ps) ++k;
          part_of_chain[c] = first_part + k;
          acc += clen[c];
        }
        first_part += ps;
      }
    }
    for (int p = 0; p < n; ++p) part_of[p] = part_of_chain[chain_of[p]];
    out->n_chains = nc;
  }

  // 4. rows of each part in level order (plan order is level order); slots
  std::vector<int> part_ptr(P + 1, 0), part_rows(n), slot_of(n);
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

  // entries per row held in the record's fixed columns
  int K = 0;
  for (int p = 0; p < n; ++p) K = std::max(K, in.rp[p + 1] - in.rp[p]);
  K = std::min(K, kRegEnt);

  // 5. block records, per precision.  A slot holds one block's record and,
  // right after it, the block's gather area.
  for (int prec = 0; prec < (in.with_fp32 ? 2 : 1); ++prec) {
    const int ts = prec == 0 ? 8 : 4;
    const int kRing = prec == 0 ? Ring<double>::kRing : Ring<float>::kRing;
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
          RecHdr h{};
          h.slot0 = i - part_ptr[q];
          h.K = K;
          int j = i;
          const int l0 = lev[part_rows[i]];
          while (j < iend && h.nrows < kPartThreads && lev[part_rows[j]] == l0) {
            const int p = part_rows[j];
            const int ne = in.rp[p + 1] - in.rp[p];
            int ext = 0;
            for (int e = in.rp[p]; e < in.rp[p + 1]; ++e) ext += part_of[pos_of[in.ci[e]]] != q;
            RecHdr t = h;
            t.nrows += 1;
            t.next += ext;
            t.nover += std::max(0, ne - K);
            rec_layout(t, ts, in.unit_diag);
            if (ne - K > 255 || slot_need(t, ts) > slot_bytes) break;
            h = t;
            ++j;
          }
          if (j == i) {  // one row alone does not fit a slot
            fits = false;
            break;
          }
          rec_layout(h, ts, in.unit_diag);
          const size_t base = stream.size();
          stream.resize(base + h.bytes, 0);
          unsigned char* rec = stream.data() + base;
          std::memcpy(rec, &h, sizeof(h));
          int32_t* orow = reinterpret_cast<int32_t*>(rec + 48);
          int32_t* rf = reinterpret_cast<int32_t*>(rec + h.off_ref);
          int32_t* gext = reinterpret_cast<int32_t*>(rec + h.off_gext);
          int32_t* over = h.off_over ? reinterpret_cast<int32_t*>(rec + h.off_over) : nullptr;
          int32_t* oref = h.off_over ? over + a16(4 * h.nrows) / 4 : nullptr;
          unsigned char* oval = h.off_over ? rec + h.off_over + a16(4 * h.nrows) + a16(4 * h.nover)
                                           : nullptr;
          auto put_val = [&](unsigned char* base_v, int idx, double v) {
            if (ts == 8)
              reinterpret_cast<double*>(base_v)[idx] = v;
            else
              reinterpret_cast<float*>(base_v)[idx] = (float)v;
          };
          const int lanes = 16 / ts;
          int ng = 0, no = 0;
          for (int k = 0; k < h.nrows; ++k) {
            const int p = part_rows[i + k];
            orow[k] = in.row_of[p];
            const int ne = in.rp[p + 1] - in.rp[p];
            if (over) over[k] = ne > K ? (no << 8) | (ne - K) : 0;
            for (int q2 = 0; q2 < K; ++q2) rf[q2 * h.nrows + k] = kNoEntry;
            for (int e = in.rp[p], c = 0; e < in.rp[p + 1]; ++e, ++c) {
              const int qd = pos_of[in.ci[e]];
              int r;
              if (part_of[qd] == q) {
                r = slot_of[qd];
              } else {
                gext[ng] = in.ci[e];
                r = -(1 + 4 * ng + in.ci[e] % lanes);
                ++ng;
              }
              if (c < K) {
                rf[c * h.nrows + k] = r;
                put_val(rec + h.off_val, c * h.nrows + k, in.val[e]);
              } else {
                oref[no] = r;
                put_val(oval, no, in.val[e]);
                ++no;
              }
            }
            if (!in.unit_diag) put_val(rec + h.off_dia, k, in.dinv[p]);
          }
          ext_entries += ng;
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
  const int n = S->n;
  if (n == 0 || ctx->part_sweeps == 0) return MTLGPU_OK;
  // automatic choice: the partitioned sweep where levels are narrow (few rows
  // per level, long dependency chains) and factor rows short (2-D 5-point
  // grids, where it measured 16 % faster); the level-ordered ticket sweep
  // where levels are wide (3-D grids) or rows long (27-point factors: 5.7 ms
  // partitioned against under 1 ms for the ticket sweep at 48^3)
  if (ctx->part_sweeps == 2 &&
      (S->n_levels == 0 || n / S->n_levels > kAutoRowsPerLevel ||
       (long long)S->nnz_off * 2 > 5ll * n))
    return MTLGPU_OK;

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
      cudaFuncAttributes fa{};
      MTLGPU_TRY_CUDA(ctx, cudaFuncGetAttributes(&fa, part_sweep_kernel<double>));
      MTLGPU_TRY_CUDA(ctx, cudaFuncSetAttribute(part_sweep_kernel<double>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                in.smem_optin - (int)fa.sharedSizeBytes));
      MTLGPU_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &occ, part_sweep_kernel<double>, kCtaThreads, V.smem_bytes));
    } else {
      cudaFuncAttributes fa{};
      MTLGPU_TRY_CUDA(ctx, cudaFuncGetAttributes(&fa, part_sweep_kernel<float>));
      MTLGPU_TRY_CUDA(ctx, cudaFuncSetAttribute(part_sweep_kernel<float>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                in.smem_optin - (int)fa.sharedSizeBytes));
      MTLGPU_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                               &occ, part_sweep_kernel<float>, kCtaThreads, V.smem_bytes));
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

// External values are read as 16-byte chunks whose lane the records fix, so
// the output vector must be 16-byte aligned (device allocations are).
template <typename T>
bool part_sweep_ready(const SweepPlan& S, const T* out) {
  return S.part && S.part->prec[sizeof(T) == 8 ? 0 : 1].ready &&
         (reinterpret_cast<uintptr_t>(out) & 15) == 0;
}

template <typename T>
mtlgpu_status part_sweep_launch(Ctx* ctx, const SweepPlan& S, const T* in, T* out,
                                const int* skip) {
  const auto& V = S.part->prec[sizeof(T) == 8 ? 0 : 1];
  ctx->launches++;
  part_sweep_kernel<T><<<S.part->P, kCtaThreads, V.smem_bytes, ctx->stream>>>(
      V.d_part_blk, V.d_blk_off16, V.d_rec, V.vals_bytes, V.offs_bytes, V.slot_bytes, in, out,
      ctx->d_error, ctx->spin_limit, skip);
  MTLGPU_TRY_CUDA(ctx, cudaGetLastError());
  return MTLGPU_OK;
}

template bool part_sweep_ready<double>(const SweepPlan&, const double*);
template bool part_sweep_ready<float>(const SweepPlan&, const float*);
template mtlgpu_status part_sweep_launch<double>(Ctx*, const SweepPlan&, const double*, double*,
                                                 const int*);
template mtlgpu_status part_sweep_launch<float>(Ctx*, const SweepPlan&, const float*, float*,
                                                const int*);

}  // namespace mtlgpu
