// Drop-in check of <mtlgpu/mtl.hpp> against the UNMODIFIED MTL4/ITL headers.
//
// Built only where the MTL4 tree is available (with the project's Boost
// stand-in, oracle/compat), by tests/cpp/Makefile; the binary needs no MTL4
// files at run time.  Each case runs the same reference-style code twice --
// once on mtl::compressed2D / mtl::dense_vector with the reference's own
// itl::cg / itl::bicgstab / preconditioners on the CPU, once on
// mtl::gpu::compressed2D / mtl::gpu::dense_vector, which the reference's
// overload set hands to the device through the specialisations in
// <mtlgpu/mtl.hpp> -- and prints one JSON line comparing the two iteration
// objects and solutions.  tests/test_cpp_layer.py checks the lines.
#include <boost/numeric/mtl/mtl.hpp>
#include <boost/numeric/itl/itl.hpp>

#include <mtlgpu/mtl.hpp>
#include <mtlgpu_fixtures.h>

#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

namespace {

typedef mtl::compressed2D<double> Matrix;
typedef mtl::dense_vector<double> Vector;
typedef mtl::gpu::compressed2D<double> DMatrix;
typedef mtl::gpu::dense_vector<double> DVector;

Vector uniform(int n, uint64_t seed) {
  std::vector<double> h(n);
  mtlgpu_gen_uniform(n, seed, -1.0, 1.0, h.data());
  Vector v(n);
  for (int i = 0; i < n; ++i) v[i] = h[i];
  return v;
}

double max_abs_diff(const Vector& a, const DVector& b) {
  std::vector<double> h = b.to_host();
  double m = 0;
  for (std::size_t i = 0; i < h.size(); ++i) m = std::max(m, std::abs(a[i] - h[i]));
  return m;
}

int count_lines(const std::string& s) {
  int n = 0;
  for (char c : s) n += c == '\n';
  return n;
}

template <typename It>
void print_iter(const char* tag, const It& it) {
  std::printf("\"%s\": {\"iterations\": %d, \"resid\": %.17g, \"norm_r0\": %.17g, \"error\": %d}",
              tag, it.iterations(), it.resid(), it.norm_r0(), int(it.is_converged() ? 0 : 1));
}

// PCG-IC(0) on laplacian_setup(A, 100, 100), b = A * x_true (seed 0), logged
// every 50 iterations: reference CPU vs device, and the device path again
// through itl::cg_solver (the solver class calls cg(...) unqualified).
void case_cg() {
  Matrix A(10000, 10000);
  mtl::mat::laplacian_setup(A, 100, 100);
  Vector xt = uniform(10000, 0), b(10000), x(10000);
  b = A * xt;
  x = 0.0;

  std::ostringstream cpu_log, gpu_log;
  itl::pc::ic_0<Matrix> P(A);
  itl::cyclic_iteration<double> it(b, 1000, 1.e-10, 0.0, 50, cpu_log);
  it.suppress_resume(true);
  itl::cg(A, x, b, P, it);

  DMatrix dA(A);
  DVector db(b), dx(10000, 0.0);
  itl::pc::ic_0<DMatrix> dP(dA);
  itl::cyclic_iteration<double> dit(b, 1000, 1.e-10, 0.0, 50, gpu_log);
  dit.suppress_resume(true);
  itl::cg(dA, dx, db, dP, dit);

  itl::cg_solver<DMatrix, itl::pc::ic_0<DMatrix>, itl::pc::identity<DMatrix>> solver(dA, dP);
  DVector dx2(10000, 0.0);
  itl::basic_iteration<double> sit(b, 1000, 1.e-10);
  solver.solve(dx2, db, sit);

  Vector back(10000);
  dx.copy_to(back);
  std::printf("{\"case\": \"cg\", ");
  print_iter("cpu", it);
  std::printf(", ");
  print_iter("gpu", dit);
  std::printf(", ");
  print_iter("gpu_solver_class", sit);
  std::printf(", \"cpu_log_lines\": %d, \"gpu_log_lines\": %d, \"x_max_diff\": %.3g, "
              "\"copy_back_max_diff\": %.3g, \"x_true_max_err\": %.3g}\n",
              count_lines(cpu_log.str()), count_lines(gpu_log.str()), max_abs_diff(x, dx),
              max_abs_diff(back, dx), max_abs_diff(xt, dx));
}

// BiCGSTAB + ILU(0) on the 27-point convection-diffusion operator (8^3,
// seed 2; b = A * x_true, x_true seed 1), the matrix entering MTL4 through
// compressed2D's raw-array constructor.
void case_bicgstab() {
  const int N = 8, n = N * N * N;
  const long long nnz = mtlgpu_gen_convdiff27(N, 2, nullptr, nullptr, nullptr);
  std::vector<int32_t> rp(n + 1), ci(nnz);
  std::vector<double> v(nnz);
  mtlgpu_gen_convdiff27(N, 2, rp.data(), ci.data(), v.data());
  std::vector<std::size_t> rps(rp.begin(), rp.end()), cis(ci.begin(), ci.end());
  Matrix A(n, n, std::size_t(nnz), rps.data(), cis.data(), v.data());
  Vector xt = uniform(n, 1), b(n), x(n);
  b = A * xt;
  x = 0.0;
  itl::pc::ilu_0<Matrix> P(A);
  itl::basic_iteration<double> it(b, 1000, 1.e-10);
  itl::bicgstab(A, x, b, P, it);

  DMatrix dA(A);
  DVector db(b), dx(n, 0.0);
  itl::pc::ilu_0<DMatrix> dP(dA);
  itl::basic_iteration<double> dit(b, 1000, 1.e-10);
  itl::bicgstab(dA, dx, db, dP, dit);
  std::printf("{\"case\": \"bicgstab\", ");
  print_iter("cpu", it);
  std::printf(", ");
  print_iter("gpu", dit);
  std::printf(", \"x_max_diff\": %.3g}\n", max_abs_diff(x, dx));
}

// ic_0<Matrix, float> on the 3x3 grid, y = solve(P, iota) (ic_0_test.cpp), and
// ilu_0 solve / adjoint_solve on the same matrix.
void case_pc() {
  Matrix A(9, 9);
  mtl::mat::laplacian_setup(A, 3, 3);
  Vector x(9), y(9), ya(9), yi(9);
  for (int i = 0; i < 9; ++i) x[i] = i;
  itl::pc::ic_0<Matrix, float> P(A);
  y = solve(P, x);
  itl::pc::ilu_0<Matrix> Q(A);
  yi = solve(Q, x);
  ya = adjoint_solve(Q, x);

  DMatrix dA(A);
  DVector dxv(x), dy(9), dyi(9), dya(9);
  itl::pc::ic_0<DMatrix, float> dP(dA);
  dy = solve(dP, dxv);
  itl::pc::ilu_0<DMatrix> dQ(dA);
  dyi = solve(dQ, dxv);
  dya = adjoint_solve(dQ, dxv);
  std::printf("{\"case\": \"pc\", \"ic0_float_max_diff\": %.3g, \"ilu0_max_diff\": %.3g, "
              "\"ilu0_adjoint_max_diff\": %.3g}\n",
              max_abs_diff(y, dy), max_abs_diff(yi, dyi), max_abs_diff(ya, dya));
}

// The other Krylov methods called exactly as the reference's tests call them,
// on mtl::compressed2D (CPU) and on mtl::gpu::compressed2D (device), ILU(0)
// on the left, identity on the right, 27-point convection-diffusion 6^3.
void case_krylov() {
  const int N = 6, n = N * N * N;
  const long long nnz = mtlgpu_gen_convdiff27(N, 2, nullptr, nullptr, nullptr);
  std::vector<int32_t> rp(n + 1), ci(nnz);
  std::vector<double> v(nnz);
  mtlgpu_gen_convdiff27(N, 2, rp.data(), ci.data(), v.data());
  std::vector<std::size_t> rps(rp.begin(), rp.end()), cis(ci.begin(), ci.end());
  Matrix A(n, n, std::size_t(nnz), rps.data(), cis.data(), v.data());
  Vector xt = uniform(n, 1), b(n);
  b = A * xt;
  DMatrix dA(A);
  DVector db(b);
  itl::pc::ilu_0<Matrix> L(A);
  itl::pc::identity<Matrix> R(A);
  itl::pc::ilu_0<DMatrix> dL(dA);
  itl::pc::identity<DMatrix> dR(dA);
  const char* names[] = {"bicg", "cgs", "bicgstab_2", "bicgstab_ell", "tfqmr", "qmr", "idr_s",
                         "gmres"};
  std::printf("{\"case\": \"krylov\"");
  for (int m = 0; m < 8; ++m) {
    const int max_it = m == 5 ? 60 : 400;
    Vector x(n, 0.0);
    DVector dx(n, 0.0);
    itl::basic_iteration<double> it(b, max_it, 1.e-8), dit(b, max_it, 1.e-8);
    int e = 0, de = 0;
    switch (m) {
      case 0: e = itl::bicg(A, x, b, L, it); de = itl::bicg(dA, dx, db, dL, dit); break;
      case 1: e = itl::cgs(A, x, b, L, it); de = itl::cgs(dA, dx, db, dL, dit); break;
      case 2: e = itl::bicgstab_2(A, x, b, L, it); de = itl::bicgstab_2(dA, dx, db, dL, dit); break;
      case 3:
        e = itl::bicgstab_ell(A, x, b, L, R, it, 4);
        de = itl::bicgstab_ell(dA, dx, db, dL, dR, dit, 4);
        break;
      case 4: e = itl::tfqmr(A, x, b, L, R, it); de = itl::tfqmr(dA, dx, db, dL, dR, dit); break;
      case 5: e = itl::qmr(A, x, b, L, R, it); de = itl::qmr(dA, dx, db, dL, dR, dit); break;
      case 6:
        mtl::seed<double>::counter = 0;
        e = itl::idr_s(A, x, b, L, R, it, 2);
        de = itl::idr_s(dA, dx, db, dL, dR, dit, 2);
        break;
      case 7: e = itl::gmres(A, x, b, L, R, it, 8); de = itl::gmres(dA, dx, db, dL, dR, dit, 8); break;
    }
    std::printf(", \"%s\": {\"cpu\": [%d, %d], \"gpu\": [%d, %d], \"x_max_diff\": %.3g}",
                names[m], it.iterations(), e, dit.iterations(), de, max_abs_diff(x, dx));
  }
  std::printf("}\n");
}

// The same insertion code on mtl::compressed2D (the reference's inserter)
// and on mtl::gpu::compressed2D (assembled on the device): seeded triplets
// with duplicates, `<<` with update_plus, `=` and `+=` mixed, into a matrix
// that already holds entries.  The CSR arrays must be identical.
template <typename M>
void insert_all(M& A, const std::vector<int>& r, const std::vector<int>& c,
                const std::vector<double>& v, const std::vector<int>& how) {
  mtl::mat::inserter<M, mtl::operations::update_plus<double>> ins(A, 3);
  for (size_t k = 0; k < r.size(); ++k) {
    if (how[k] == 0) ins[r[k]][c[k]] = v[k];
    else if (how[k] == 1) ins[r[k]][c[k]] += v[k];
    else ins[r[k]][c[k]] << v[k];
  }
}

void case_assemble() {
  const int nr = 400, nc = 300, cnt = 20000;
  std::vector<int> r(cnt), c(cnt), how(cnt);
  std::vector<double> v(cnt), u(cnt);
  mtlgpu_gen_uniform(cnt, 91, -1.0, 1.0, v.data());
  mtlgpu_gen_uniform(cnt, 92, 0.0, 1.0, u.data());
  for (int k = 0; k < cnt; ++k) {
    r[k] = int(u[k] * nr) % nr;
    c[k] = (r[k] * 3 + k % 11) % nc;
    how[k] = k % 3;
  }
  Matrix A(nr, nc);
  insert_all(A, std::vector<int>(r.begin(), r.begin() + 5000),
             std::vector<int>(c.begin(), c.begin() + 5000),
             std::vector<double>(v.begin(), v.begin() + 5000), std::vector<int>(5000, 2));
  insert_all(A, r, c, v, how);
  DMatrix dA(nr, nc);
  insert_all(dA, std::vector<int>(r.begin(), r.begin() + 5000),
             std::vector<int>(c.begin(), c.begin() + 5000),
             std::vector<double>(v.begin(), v.begin() + 5000), std::vector<int>(5000, 2));
  insert_all(dA, r, c, v, how);
  const mtl::gpu::host_csr h = dA.to_host();
  bool same = int(A.nnz()) == dA.nnz();
  for (int i = 0; same && i <= nr; ++i) same = int(A.ref_major()[i]) == h.starts[i];
  for (int j = 0; same && j < dA.nnz(); ++j)
    same = int(A.ref_minor()[j]) == h.indices[j] && A.data[j] == h.data[j];
  // laplacian_setup on both matrix types
  Matrix L(1, 1);
  DMatrix dL(1, 1);
  mtl::mat::laplacian_setup(L, 17, 23);
  mtl::mat::laplacian_setup(dL, 17, 23);
  const mtl::gpu::host_csr hl = dL.to_host();
  bool lap = int(L.nnz()) == dL.nnz();
  for (int j = 0; lap && j < dL.nnz(); ++j)
    lap = int(L.ref_minor()[j]) == hl.indices[j] && L.data[j] == hl.data[j];
  std::printf("{\"case\": \"assemble\", \"nnz\": %d, \"identical\": %s, "
              "\"laplacian_identical\": %s}\n",
              dA.nnz(), same ? "true" : "false", lap ? "true" : "false");
}

}  // namespace

int main(int argc, char** argv) {
  const std::string c = argc > 1 ? argv[1] : "";
  try {
    if (c == "cg") case_cg();
    else if (c == "bicgstab") case_bicgstab();
    else if (c == "pc") case_pc();
    else if (c == "assemble") case_assemble();
    else if (c == "krylov") case_krylov();
    else {
      std::fprintf(stderr, "usage: mtl4_dropin cg|bicgstab|pc|assemble|krylov\n");
      return 2;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s: %s\n", c.c_str(), e.what());
    return 1;
  }
  return 0;
}
