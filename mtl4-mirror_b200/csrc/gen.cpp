// Host-side fixture generators (include/mtlgpu_fixtures.h).  These build the
// synthetic inputs; they are not part of the solve path.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "mtlgpu_fixtures.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * 0x1.0p-53; }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  // Box-Muller: two uniforms -> two normals
  bool have = false;
  double spare = 0;
  double normal() {
    if (have) {
      have = false;
      return spare;
    }
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    const double r = std::sqrt(-2.0 * std::log(u1)), t = 6.283185307179586 * u2;
    spare = r * std::sin(t);
    have = true;
    return r * std::cos(t);
  }
};

struct RowWriter {
  int32_t* rp;
  int32_t* ci;
  double* v;
  long long nnz = 0;
  void begin(long long row) {
    if (rp) rp[row] = (int32_t)nnz;
  }
  void put(long long c, double w) {
    if (ci) ci[nnz] = (int32_t)c, v[nnz] = w;
    nnz++;
  }
  void end(long long rows) {
    if (rp) rp[rows] = (int32_t)nnz;
  }
};

double harmonic(double a, double b) { return 2.0 * a * b / (a + b); }

void build_graph(int n, double avg_deg, double shift_frac, uint64_t seed, int32_t* rp, int32_t* ci,
                 double* v, long long* nnz_out) {
  SplitMix64 g(seed);
  const long long m = std::llround(double(n) * avg_deg / 2.0);
  std::vector<int32_t> ei(m), ej(m);
  for (long long e = 0; e < m; e++) {
    int i, j;
    do {
      i = (int)std::min<double>(n - 1, std::floor(g.uniform() * n));
      j = (int)std::min<double>(n - 1, std::floor(g.uniform() * n));
    } while (i == j);
    ei[e] = i;
    ej[e] = j;
  }
  std::vector<int64_t> start(n + 1, 0);
  for (long long e = 0; e < m; e++) start[ei[e] + 1]++, start[ej[e] + 1]++;
  for (int i = 0; i < n; i++) start[i + 1] += start[i];
  std::vector<int32_t> nb(2 * m);
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  for (long long e = 0; e < m; e++) nb[fill[ei[e]]++] = ej[e], nb[fill[ej[e]]++] = ei[e];
  const double shift = shift_frac * avg_deg;
  RowWriter w{rp, ci, v};
  for (int i = 0; i < n; i++) {
    std::sort(nb.begin() + start[i], nb.begin() + start[i + 1]);
    w.begin(i);
    double deg = 0;
    bool diag_done = false;
    long long k = start[i];
    while (k < start[i + 1]) {
      const int c = nb[k];
      long long k2 = k;
      while (k2 < start[i + 1] && nb[k2] == c) k2++;
      const double wt = double(k2 - k);
      deg += wt;
      if (!diag_done && c > i) {
        w.put(i, 0.0);  // placeholder, set below
        diag_done = true;
      }
      w.put(c, -wt);
      k = k2;
    }
    if (!diag_done) w.put(i, 0.0);
    if (v) {  // locate the diagonal entry of this row and set it
      long long b = rp ? rp[i] : 0;
      for (long long q = b; q < w.nnz; q++)
        if (ci[q] == i) v[q] = deg + shift;
    }
  }
  w.end(n);
  *nnz_out = w.nnz;
}

}  // namespace

extern "C" {

long long mtlgpu_gen_laplacian2d(int m, int n, int32_t* rp, int32_t* ci, double* v) {
  RowWriter w{rp, ci, v};
  for (long long i = 0; i < m; i++)
    for (long long j = 0; j < n; j++) {
      const long long row = i * n + j;
      w.begin(row);
      if (i > 0) w.put(row - n, -1.0);
      if (j > 0) w.put(row - 1, -1.0);
      w.put(row, 4.0);
      if (j < n - 1) w.put(row + 1, -1.0);
      if (i < m - 1) w.put(row + n, -1.0);
    }
  w.end((long long)m * n);
  return w.nnz;
}

long long mtlgpu_gen_laplacian3d(int N, int32_t* rp, int32_t* ci, double* v) {
  RowWriter w{rp, ci, v};
  const long long NN = (long long)N * N;
  for (long long i = 0; i < N; i++)
    for (long long j = 0; j < N; j++)
      for (long long k = 0; k < N; k++) {
        const long long row = (i * N + j) * N + k;
        w.begin(row);
        if (i > 0) w.put(row - NN, -1.0);
        if (j > 0) w.put(row - N, -1.0);
        if (k > 0) w.put(row - 1, -1.0);
        w.put(row, 6.0);
        if (k < N - 1) w.put(row + 1, -1.0);
        if (j < N - 1) w.put(row + N, -1.0);
        if (i < N - 1) w.put(row + NN, -1.0);
      }
  w.end(NN * N);
  return w.nnz;
}

long long mtlgpu_gen_convdiff27(int N, uint64_t seed, int32_t* rp, int32_t* ci, double* v) {
  const long long n = (long long)N * N * N;
  if (!rp) {
    const long long s = 3ll * N - 2;
    return s * s * s;
  }
  SplitMix64 g(seed);
  std::vector<double> kap(n), ux(n), uy(n), uz(n);
  for (long long c = 0; c < n; c++) kap[c] = std::exp(0.5 * g.normal());
  g.have = false;
  for (long long c = 0; c < n; c++) {
    ux[c] = g.uniform(-1, 1);
    uy[c] = g.uniform(-1, 1);
    uz[c] = g.uniform(-1, 1);
  }
  RowWriter w{rp, ci, v};
  for (long long i = 0; i < N; i++)
    for (long long j = 0; j < N; j++)
      for (long long k = 0; k < N; k++) {
        const long long c = (i * N + j) * N + k;
        w.begin(c);
        double diag = 0;
        long long diag_pos = -1;
        for (int di = -1; di <= 1; di++)
          for (int dj = -1; dj <= 1; dj++)
            for (int dk = -1; dk <= 1; dk++) {
              const long long ii = i + di, jj = j + dj, kk = k + dk;
              const bool inside = ii >= 0 && ii < N && jj >= 0 && jj < N && kk >= 0 && kk < N;
              if (di == 0 && dj == 0 && dk == 0) {
                diag_pos = w.nnz;
                w.put(c, 0.0);
                continue;
              }
              const int d2 = di * di + dj * dj + dk * dk;
              const double wd = 1.0 / d2;
              const long long nbi = inside ? (ii * N + jj) * N + kk : c;
              const double D = harmonic(kap[c], kap[nbi]) * wd;
              const double flow = ux[c] * di + uy[c] * dj + uz[c] * dk;
              const double C = std::max(0.0, -flow) * wd;
              diag += D + C;
              if (inside) w.put(nbi, -(D + C));
            }
        if (v) v[diag_pos] = (1.0 + 1e-3) * diag;
      }
  w.end(n);
  return w.nnz;
}

long long mtlgpu_gen_random_graph(int n, double avg_deg, double shift_frac, uint64_t seed,
                                  int32_t* rp, int32_t* ci, double* v) {
  long long nnz = 0;
  if (!rp) {
    // sizes need the pattern: build once into scratch
    std::vector<int32_t> trp(n + 1);
    build_graph(n, avg_deg, shift_frac, seed, trp.data(), nullptr, nullptr, &nnz);
    return nnz;
  }
  build_graph(n, avg_deg, shift_frac, seed, rp, ci, v, &nnz);
  return nnz;
}

long long mtlgpu_gen_fv2d(int N, double sigma, double corr, uint64_t seed, int32_t* rp,
                          int32_t* ci, double* v) {
  const long long n = (long long)N * N;
  if (!rp) return 5 * n - 4ll * N;
  SplitMix64 g(seed);
  std::vector<double> wn(n), tmp(n), f(n);
  for (long long c = 0; c < n; c++) wn[c] = g.normal();
  const int rad = (int)std::ceil(3 * corr);
  std::vector<double> ker(2 * rad + 1);
  for (int t = -rad; t <= rad; t++) ker[t + rad] = std::exp(-0.5 * (t / corr) * (t / corr));
  for (long long i = 0; i < N; i++)
    for (long long j = 0; j < N; j++) {
      double s = 0;
      for (int t = -rad; t <= rad; t++) {
        const long long jj = j + t;
        if (jj >= 0 && jj < N) s += ker[t + rad] * wn[i * N + jj];
      }
      tmp[i * N + j] = s;
    }
  for (long long i = 0; i < N; i++)
    for (long long j = 0; j < N; j++) {
      double s = 0;
      for (int t = -rad; t <= rad; t++) {
        const long long ii = i + t;
        if (ii >= 0 && ii < N) s += ker[t + rad] * tmp[ii * N + j];
      }
      f[i * N + j] = s;
    }
  double mean = 0, var = 0;
  for (long long c = 0; c < n; c++) mean += f[c];
  mean /= n;
  for (long long c = 0; c < n; c++) var += (f[c] - mean) * (f[c] - mean);
  var /= n;
  const double sd = var > 0 ? std::sqrt(var) : 1.0;
  std::vector<double> kap(n);
  for (long long c = 0; c < n; c++) kap[c] = std::exp(sigma * (f[c] - mean) / sd);
  RowWriter w{rp, ci, v};
  for (long long i = 0; i < N; i++)
    for (long long j = 0; j < N; j++) {
      const long long c = i * N + j;
      const double kc = kap[c];
      const double tn = i > 0 ? harmonic(kc, kap[c - N]) : 2 * kc;
      const double tw = j > 0 ? harmonic(kc, kap[c - 1]) : 2 * kc;
      const double te = j < N - 1 ? harmonic(kc, kap[c + 1]) : 2 * kc;
      const double ts = i < N - 1 ? harmonic(kc, kap[c + N]) : 2 * kc;
      w.begin(c);
      if (i > 0) w.put(c - N, -tn);
      if (j > 0) w.put(c - 1, -tw);
      w.put(c, tn + tw + te + ts);
      if (j < N - 1) w.put(c + 1, -te);
      if (i < N - 1) w.put(c + N, -ts);
    }
  w.end(n);
  return w.nnz;
}

long long mtlgpu_gen_graph_batch(int count, int n_min, int n_max, double deg_min, double deg_max,
                                 double shift_frac, uint64_t seed, int64_t* sizes, int32_t* rp,
                                 int32_t* ci, double* v) {
  SplitMix64 g(seed);
  std::vector<int> ns(count);
  std::vector<double> ds(count);
  std::vector<uint64_t> seeds(count);
  for (int s = 0; s < count; s++) {
    ns[s] = (int)std::llround(std::exp(g.uniform(std::log((double)n_min), std::log((double)n_max))));
    ds[s] = g.uniform(deg_min, deg_max);
    seeds[s] = g.next();
  }
  std::vector<long long> nnz(count);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  auto run_sizes = [&](unsigned t) {
    for (int s = (int)t; s < count; s += (int)hw) {
      std::vector<int32_t> trp(ns[s] + 1);
      build_graph(ns[s], ds[s], shift_frac, seeds[s], trp.data(), nullptr, nullptr, &nnz[s]);
    }
  };
  {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < hw; t++) th.emplace_back(run_sizes, t);
    for (auto& x : th) x.join();
  }
  long long total = 0;
  for (int s = 0; s < count; s++) {
    if (sizes) sizes[2 * s] = ns[s], sizes[2 * s + 1] = nnz[s];
    total += nnz[s];
  }
  if (!rp) return total;
  std::vector<long long> roff(count), eoff(count);
  long long ro = 0, eo = 0;
  for (int s = 0; s < count; s++) {
    roff[s] = ro;
    eoff[s] = eo;
    ro += ns[s] + 1;
    eo += nnz[s];
  }
  auto run_fill = [&](unsigned t) {
    for (int s = (int)t; s < count; s += (int)hw) {
      long long dummy = 0;
      build_graph(ns[s], ds[s], shift_frac, seeds[s], rp + roff[s], ci + eoff[s], v + eoff[s],
                  &dummy);
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < hw; t++) th.emplace_back(run_fill, t);
  for (auto& x : th) x.join();
  return total;
}

void mtlgpu_gen_uniform(long long n, uint64_t seed, double a, double b, double* out) {
  SplitMix64 g(seed);
  for (long long i = 0; i < n; i++) out[i] = g.uniform(a, b);
}

void mtlgpu_gen_normal(long long n, uint64_t seed, double* out) {
  SplitMix64 g(seed);
  for (long long i = 0; i < n; i++) out[i] = g.normal();
}

void mtlgpu_gen_csr_mult(int n, const int32_t* rp, const int32_t* ci, const double* v,
                         const double* x, double* y) {
  for (long long i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = rp[i]; j < rp[i + 1]; j++) t += v[j] * x[ci[j]];
    y[i] = t;
  }
}

}  // extern "C"
