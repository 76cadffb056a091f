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
//   itl_gpu_test adjoint     linear_solve forward/backward vs finite differences
#include <mtlgpu/mtl.hpp>
#include <mtlgpu_fixtures.h>

#include <cmath>
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

// Differentiable solve on the 2-D finite-volume operator (N x N, log-normal
// kappa): L = 1/2 ||x - x_target||^2, x = A^{-1} b with b a Gaussian source and
// x_target = x + 0.01 N(0,1).  Gradients from linear_solve::backward against
// central finite differences (h = 1e-6) along random directions in b and in
// A's values (perturbations kept symmetric, so A stays SPD for CG).
void case_adjoint() {
  const int N = 32, n = N * N;
  HostCsr h;
  h.n = n;
  const long long nnz = mtlgpu_gen_fv2d(N, 1.0, 8.0, 4, nullptr, nullptr, nullptr);
  h.rp.resize(n + 1);
  h.ci.resize(nnz);
  h.v.resize(nnz);
  mtlgpu_gen_fv2d(N, 1.0, 8.0, 4, h.rp.data(), h.ci.data(), h.v.data());
  std::vector<double> bh(n), noise(n);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      const double x = (i + 0.5) / N - 0.5, y = (j + 0.5) / N - 0.5;
      bh[i * N + j] = std::exp(-(x * x + y * y) / (2 * 0.1 * 0.1));
    }
  mtlgpu_gen_normal(n, 44, noise.data());
  auto loss_of = [&](const std::vector<double>& vals, const std::vector<double>& b,
                     const std::vector<double>& xt) {
    Matrix A(n, n, (int)nnz, h.rp.data(), h.ci.data(), vals.data());
    mtl::gpu::linear_solve S(A, MTLGPU_PC_IC0, true, 1e-14, 20000);
    std::vector<double> x = S.forward(Vector(b)).to_host();
    double L = 0;
    for (int i = 0; i < n; ++i) L += 0.5 * (x[i] - xt[i]) * (x[i] - xt[i]);
    return std::make_pair(L, x);
  };
  Matrix A = h.device();
  mtl::gpu::linear_solve S(A, MTLGPU_PC_IC0, true, 1e-14, 20000);
  std::vector<double> x = S.forward(Vector(bh)).to_host();
  std::vector<double> xt(n), dl(n);
  for (int i = 0; i < n; ++i) xt[i] = x[i] + 0.01 * noise[i];
  for (int i = 0; i < n; ++i) dl[i] = x[i] - xt[i];
  Vector gb(n), gv((int)nnz);
  S.backward(Vector(dl), gb, gv);
  const std::vector<double> gbh = gb.to_host(), gvh = gv.to_host();
  // transpose position of every entry (the pattern is symmetric)
  std::vector<int> tpos(nnz);
  for (int r = 0; r < n; ++r)
    for (int k = h.rp[r]; k < h.rp[r + 1]; ++k) {
      const int c = h.ci[k];
      for (int m = h.rp[c]; m < h.rp[c + 1]; ++m)
        if (h.ci[m] == r) tpos[k] = m;
    }
  const double eps = 1e-6;
  double worst_b = 0, worst_v = 0;
  std::vector<double> dir(n), dv(nnz), tmp(nnz);
  for (int d = 0; d < 8; ++d) {
    mtlgpu_gen_normal(n, 100 + d, dir.data());
    std::vector<double> bp(bh), bm(bh);
    double pred = 0;
    for (int i = 0; i < n; ++i) bp[i] += eps * dir[i], bm[i] -= eps * dir[i], pred += gbh[i] * dir[i];
    const double fd = (loss_of(h.v, bp, xt).first - loss_of(h.v, bm, xt).first) / (2 * eps);
    worst_b = std::max(worst_b, std::abs(fd - pred) / std::max(std::abs(pred), 1e-30));
    mtlgpu_gen_normal(nnz, 200 + d, tmp.data());
    for (long long k = 0; k < nnz; ++k) dv[k] = 0.5 * (tmp[k] + tmp[tpos[k]]);
    std::vector<double> vp(h.v), vm(h.v);
    double predv = 0;
    for (long long k = 0; k < nnz; ++k)
      vp[k] += eps * dv[k], vm[k] -= eps * dv[k], predv += gvh[k] * dv[k];
    const double fdv = (loss_of(vp, bh, xt).first - loss_of(vm, bh, xt).first) / (2 * eps);
    worst_v = std::max(worst_v, std::abs(fdv - predv) / std::max(std::abs(predv), 1e-30));
  }
  std::printf(
      "{\"case\": \"adjoint\", \"forward_iterations\": %d, \"backward_iterations\": %d, "
      "\"fd_rel_err_b\": %.3e, \"fd_rel_err_vals\": %.3e}\n",
      S.forward_iterations(), S.backward_iterations(), worst_b, worst_v);
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

// laplacian_setup_test / the inserter (compressed2D.hpp:662-1151) on device
// matrices: the 5-point Laplacian inserted element by element as
// laplacian_setup.hpp:30-41 does equals the device laplacian_setup and the
// host generator; duplicates fold with the inserter's updater; an index out
// of range raises index_out_of_range.
void case_assemble() {
  const int m = 20, n = 30;
  Matrix A(m * n, m * n), L(0, 0);
  {
    mtl::mat::inserter<Matrix> ins(A, 5);
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) {
        const int row = i * n + j;
        ins(row, row) << 4.0;
        if (j < n - 1) ins(row, row + 1) << -1.0;
        if (i < m - 1) ins(row, row + n) << -1.0;
        if (j > 0) ins(row, row - 1) << -1.0;
        if (i > 0) ins(row, row - n) << -1.0;
      }
  }
  mtl::mat::laplacian_setup(L, m, n);
  HostCsr h = laplacian2d(m, n);
  const mtl::gpu::host_csr a = A.to_host(), l = L.to_host();
  const bool lap_equal = a.starts == l.starts && a.indices == l.indices && a.data == l.data &&
                         a.starts == h.rp && a.indices == h.ci && a.data == h.v;
  // update_plus with duplicates, then `=` and `+=` on top of the result
  Matrix B(3, 4);
  {
    mtl::mat::inserter<Matrix, mtl::operations::update_plus<double>> ins(B);
    ins[2][3] << 1.5;
    ins[0][1] << 2.0;
    ins[2][3] << 0.25;
    ins[1][0] << -1.0;
  }
  {
    mtl::mat::inserter<Matrix> ins(B);
    ins[2][3] += 4.0;   // 1.75 + 4
    ins[0][1] = 7.0;    // overwritten
    ins[0][0] << 3.0;   // new entry
  }
  const mtl::gpu::host_csr b = B.to_host();
  const bool upd_ok = b.starts == std::vector<int32_t>{0, 2, 3, 4} &&
                      b.indices == std::vector<int32_t>{0, 1, 0, 3} &&
                      b.data == std::vector<double>{3.0, 7.0, -1.0, 5.75};
  bool range_error = false;
  try {
    Matrix C(2, 2);
    mtl::mat::inserter<Matrix> ins(C);
    ins[0][2] << 1.0;
    ins.finish();
  } catch (const mtl::index_out_of_range&) {
    range_error = true;
  }
  check(lap_equal && upd_ok && range_error, "device inserter");
  std::printf("{\"case\": \"assemble\", \"laplacian_equal\": %s, \"updaters\": %s, "
              "\"range_error\": %s, \"nnz\": %d}\n",
              lap_equal ? "true" : "false", upd_ok ? "true" : "false",
              range_error ? "true" : "false", A.nnz());
}

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
    else if (c == "adjoint") case_adjoint();
    else if (c == "assemble") case_assemble();
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
