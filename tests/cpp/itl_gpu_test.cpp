// Reference-style programs for the C++ layer <mtlgpu/mtl.hpp> (standalone
// mode, no MTL4 headers).  Each case follows one of the reference's own test
// programs, with the same calls (y = A * x, solve(P, x), itl::cg(A, x, b, P,
// iter) ...) on device types, and prints one JSON line with what it measured;
// tests/test_cpp_layer.py checks the lines against the oracle and the golden
// fixtures.  A failed check inside a case throws, as the reference's tests do
// (MTL_THROW_IF), and the program exits non-zero.
//
//   itl_gpu_test spmv        matrix_vector_product_test.cpp:43-89
//   itl_gpu_test dot         dot_test.cpp:33-44
//   itl_gpu_test ic0_float   itl/test/ic_0_test.cpp:17-36
//   itl_gpu_test cg          config-1 PCG-IC(0) through cyclic_iteration
//   itl_gpu_test bicgstab    BiCGSTAB + ILU(0) on a 27-point operator
//   itl_gpu_test mixed       PCG-IC(0) with FP32 inner solves + FP64 refinement
//   itl_gpu_test errors      exceptions for bad input
#include <mtlgpu/mtl.hpp>
#include <mtlgpu_fixtures.h>

#include <cstdio>
#include <cstring>
#include <sstream>
#include <vector>

namespace {

using Matrix = mtl::gpu::compressed2D<double>;
using Vector = mtl::gpu::dense_vector<double>;

struct HostCsr {
  int n = 0;
  std::vector<int32_t> rp, ci;
  std::vector<double> v;
  Matrix device() const {
    return Matrix(n, n, int(v.size()), rp.data(), ci.data(), v.data());
  }
};

HostCsr laplacian2d(int m, int k) {
  HostCsr h;
  h.n = m * k;
  const long long nnz = mtlgpu_gen_laplacian2d(m, k, nullptr, nullptr, nullptr);
  h.rp.resize(h.n + 1);
  h.ci.resize(nnz);
  h.v.resize(nnz);
  mtlgpu_gen_laplacian2d(m, k, h.rp.data(), h.ci.data(), h.v.data());
  return h;
}

HostCsr convdiff27(int N, uint64_t seed) {
  HostCsr h;
  h.n = N * N * N;
  const long long nnz = mtlgpu_gen_convdiff27(N, seed, nullptr, nullptr, nullptr);
  h.rp.resize(h.n + 1);
  h.ci.resize(nnz);
  h.v.resize(nnz);
  mtlgpu_gen_convdiff27(N, seed, h.rp.data(), h.ci.data(), h.v.data());
  return h;
}

HostCsr laplacian3d(int N) {
  HostCsr h;
  h.n = N * N * N;
  const long long nnz = mtlgpu_gen_laplacian3d(N, nullptr, nullptr, nullptr);
  h.rp.resize(h.n + 1);
  h.ci.resize(nnz);
  h.v.resize(nnz);
  mtlgpu_gen_laplacian3d(N, h.rp.data(), h.ci.data(), h.v.data());
  return h;
}

void check(bool ok, const char* what) {
  if (!ok) throw mtl::runtime_error(what);
}

// b = A * x_true with x_true ~ U[-1, 1] (seeded), computed on the host.
std::vector<double> rhs(const HostCsr& h, uint64_t seed) {
  std::vector<double> xt(h.n), b(h.n);
  mtlgpu_gen_uniform(h.n, seed, -1.0, 1.0, xt.data());
  mtlgpu_gen_csr_mult(h.n, h.rp.data(), h.ci.data(), h.v.data(), xt.data(), b.data());
  return b;
}

double true_rel_resid(const HostCsr& h, const std::vector<double>& x, const std::vector<double>& b) {
  std::vector<double> ax(h.n);
  mtlgpu_gen_csr_mult(h.n, h.rp.data(), h.ci.data(), h.v.data(), x.data(), ax.data());
  double r = 0, nb = 0;
  for (int i = 0; i < h.n; ++i) {
    r += (b[i] - ax[i]) * (b[i] - ax[i]);
    nb += b[i] * b[i];
  }
  return std::sqrt(r / nb);
}

// matrix_vector_product_test: v = row 12 of the 5x5-grid Laplacian,
// w = A * v gives the 13-point stencil 1 / 2 -8 2 / 1 -8 20 -8 1 ...
void case_spmv() {
  HostCsr h = laplacian2d(5, 5);
  Matrix A = h.device();
  std::vector<double> row(h.n, 0.0);
  for (int j = h.rp[12]; j < h.rp[13]; ++j) row[h.ci[j]] = h.v[j];
  Vector v(row), w(h.n);
  w = A * v;
  check(w[12] == 20 && w[13] == -8 && w[14] == 1 && w[15] == 0 && w[17] == -8 && w[18] == 2 &&
            w[22] == 1,
        "wrong stencil after w = A * v");
  w += A * v;
  check(w[12] == 40 && w[18] == 4, "wrong stencil after w += A * v");
  w -= A * v;
  check(w[12] == 20 && w[18] == 2, "wrong stencil after w -= A * v");
  Vector u(h.n);
  mult(A, v, u);
  check(u[13] == -8, "mult(A, v, u)");
  std::printf("{\"case\": \"spmv\", \"w12\": %g, \"w18\": %g}\n", w[12], w[18]);
}

// dot_test: u = 1..9, dot(u, u) = 285
void case_dot() {
  std::vector<double> h(9);
  for (int i = 0; i < 9; ++i) h[i] = i + 1;
  Vector u(h);
  const double d = dot(u, u), un = unary_dot(u), nrm = two_norm(u);
  check(d == 285.0 && un == 285.0, "dot(u, u) != 285");
  check(std::abs(nrm - std::sqrt(285.0)) < 1e-14, "two_norm");
  Vector x(9, 1.0);
  x += 2.0 * u;  // 3, 5, ..., 19
  check(x[8] == 19.0, "x += alpha * u");
  std::printf("{\"case\": \"dot\", \"dot\": %.17g, \"two_norm\": %.17g}\n", d, nrm);
}

// ic_0_test: 3x3-grid Laplacian, ic_0<Matrix, float>, y = solve(P, iota)
void case_ic0_float() {
  HostCsr h = laplacian2d(3, 3);
  Matrix A = h.device();
  itl::pc::ic_0<Matrix, float> P(A);
  std::vector<double> io(h.n);
  for (int i = 0; i < h.n; ++i) io[i] = i;
  Vector x(io), y(h.n);
  y = solve(P, x);
  std::vector<double> yh = y.to_host();
  std::printf("{\"case\": \"ic0_float\", \"y\": [");
  for (int i = 0; i < h.n; ++i) std::printf("%s%.17g", i ? ", " : "", yh[i]);
  std::printf("]}\n");
}

// PCG-IC(0) on the 100 x 100 Laplacian (b = A x_true, x_true ~ U[-1,1] seed 0,
// rtol 1e-10, 1000 iterations), logged every 50 iterations.
void case_cg() {
  HostCsr h = laplacian2d(100, 100);
  Matrix A = h.device();
  std::vector<double> bh = rhs(h, 0);
  Vector b(bh), x(h.n, 0.0);
  itl::pc::ic_0<Matrix> P(A);
  std::ostringstream log;
  itl::cyclic_iteration<double> iter(b, 1000, 1.e-10, 0.0, 50, log);
  iter.suppress_resume(true);
  const int err = itl::cg(A, x, b, P, iter);
  int lines = 0;
  for (char c : log.str()) lines += c == '\n';
  std::printf(
      "{\"case\": \"cg\", \"error\": %d, \"iterations\": %d, \"resid\": %.17g, \"norm_r0\": %.17g, "
      "\"converged\": %d, \"log_lines\": %d, \"true_rel\": %.17g}\n",
      err, iter.iterations(), iter.resid(), iter.norm_r0(), int(iter.is_converged()), lines,
      true_rel_resid(h, x.to_host(), bh));
}

void case_bicgstab() {
  HostCsr h = convdiff27(8, 2);
  Matrix A = h.device();
  std::vector<double> bh = rhs(h, 1);  // the fixture seeds x_true with 1
  Vector b(bh), x(h.n, 0.0);
  itl::pc::ilu_0<Matrix> P(A);
  itl::basic_iteration<double> iter(b, 1000, 1.e-10);
  const int err = itl::bicgstab(A, x, b, P, iter);
  std::printf(
      "{\"case\": \"bicgstab\", \"error\": %d, \"iterations\": %d, \"resid\": %.17g, "
      "\"true_rel\": %.17g}\n",
      err, iter.iterations(), iter.resid(), true_rel_resid(h, x.to_host(), bh));
}

void case_mixed() {
  HostCsr h = laplacian3d(16);
  Matrix A = h.device();
  std::vector<double> bh = rhs(h, 1);
  Vector b(bh), x(h.n, 0.0);
  itl::pc::ic_0<Matrix, float> P(A);
  itl::basic_iteration<double> iter(b, 2000, 1.e-10);
  const int err = itl::cg(A, x, b, P, iter, mtl::gpu::refinement(1e-5));
  std::printf(
      "{\"case\": \"mixed\", \"error\": %d, \"iterations\": %d, \"resid\": %.17g, "
      "\"true_rel\": %.17g}\n",
      err, iter.iterations(), iter.resid(), true_rel_resid(h, x.to_host(), bh));
}

void case_errors() {
  int caught = 0;
  // row 1 has no diagonal entry
  const int32_t rp[4] = {0, 1, 2, 3}, ci[3] = {0, 0, 2};
  const double v[3] = {2.0, 1.0, 2.0};
  Matrix A(3, 3, 3, rp, ci, v);
  try {
    itl::pc::ilu_0<Matrix> P(A);
  } catch (const mtl::missing_diagonal&) {
    ++caught;
  }
  Vector x(3), y(4);
  try {
    y = A * x;
  } catch (const mtl::incompatible_size&) {
    ++caught;
  }
  const int32_t rp2[3] = {0, 1, 2}, ci2[2] = {0, 1};
  const double v2[2] = {1.0, 1.0};
  Matrix R(2, 3, 2, rp2, ci2, v2);
  Vector x3(3, 1.0), y2(2, 0.0);
  y2 = R * x3;  // rectangular products are fine
  try {
    itl::basic_iteration<double> iter(1.0, 10, 1e-8);
    itl::cg(R, x3, y2, iter);
  } catch (const mtl::matrix_not_square&) {
    ++caught;
  }
  check(caught == 3, "expected three exceptions");
  std::printf("{\"case\": \"errors\", \"caught\": %d}\n", caught);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: itl_gpu_test spmv|dot|ic0_float|cg|bicgstab|mixed|errors\n");
    return 2;
  }
  const std::string c = argv[1];
  try {
    if (c == "spmv") case_spmv();
    else if (c == "dot") case_dot();
    else if (c == "ic0_float") case_ic0_float();
    else if (c == "cg") case_cg();
    else if (c == "bicgstab") case_bicgstab();
    else if (c == "mixed") case_mixed();
    else if (c == "errors") case_errors();
    else {
      std::fprintf(stderr, "unknown case %s\n", c.c_str());
      return 2;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s: %s\n", c.c_str(), e.what());
    return 1;
  }
  return 0;
}
