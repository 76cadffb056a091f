// C entry points over the UNMODIFIED MTL4/ITL headers, for use as the CPU
// test oracle and as the timed CPU baseline (the reference's own code path).
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
// the reference sources where they lie (include path only; nothing is copied),
// together with the project-written Boost stand-in in oracle/compat/.  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
// Every function builds mtl::compressed2D from the caller's CSR arrays through
// the raw-array constructor (mtl/matrix/compressed2D.hpp:355-364) with 32-bit
// unsigned indices (mat::parameters<..., unsigned>, mtl/matrix/parameter.hpp:29-47,
// the index type the reference's own timing programs use) and then calls the
// reference's public API exactly as its tests do:
//   y = A * x, y += A * x, y -= A * x      matrix_vector_product_test.cpp:43-89
//   itl::pc::ic_0 / ilu_0 / diagonal / identity, solve(P, x), adjoint_solve
//   itl::cg(A, x, b, P, iter), itl::bicgstab(A, x, b, P, iter)   cg.hpp:75-112,
//   bicgstab.hpp:27-78, with basic_iteration semantics (basic_iteration.hpp:24-164).
#include <boost/numeric/mtl/mtl.hpp>
#include <boost/numeric/itl/itl.hpp>

#ifdef _OPENMP
#include <omp.h>
#endif
#include <chrono>
#include <cstring>
#include <vector>

namespace {

typedef mtl::mat::parameters<mtl::row_major, mtl::index::c_index, mtl::non_fixed::dimensions, false,
                             unsigned>
    upara;
typedef mtl::mat::compressed2D<double, upara> matrix_type;
typedef mtl::dense_vector<double> vector_type;

matrix_type make_matrix(int n, int nnz, const int* rp, const int* ci, const double* v) {
  std::vector<unsigned> major(rp, rp + n + 1), minor(ci, ci + nnz);
  std::vector<double> data(v, v + nnz);
  return matrix_type(unsigned(n), unsigned(n), unsigned(nnz), major.data(),
                     nnz ? minor.data() : nullptr, nnz ? data.data() : nullptr);
}

vector_type make_vector(int n, const double* x) {
  vector_type r(n);
  for (int i = 0; i < n; ++i) r[i] = x[i];
  return r;
}

void store_vector(const vector_type& v, double* out) {
  for (std::size_t i = 0; i < mtl::size(v); ++i) out[i] = v[i];
}

template <typename M>
int export_csr(const M& A, int* rp, int* ci, double* v) {
  const int n = int(num_rows(A));
  const int nnz = int(A.nnz());
  if (rp) {
    for (int i = 0; i <= n; ++i) rp[i] = int(A.ref_major()[i]);
    for (int j = 0; j < nnz; ++j) ci[j] = int(A.ref_minor()[j]);
    for (int j = 0; j < nnz; ++j) v[j] = double(A.data[j]);
  }
  return nnz;
}

// Records the residual passed to every termination test; otherwise exactly
// basic_iteration (the solvers are templated on the iteration type, so this
// finished() is the one they call).
struct recording_iteration : itl::basic_iteration<double> {
  typedef itl::basic_iteration<double> super;
  recording_iteration(double nr0, int max_iter, double rtol, double atol, double* hist, int cap)
      : super(nr0, max_iter, rtol, atol), hist(hist), cap(cap), count(0) {}
  bool finished(const double& r) {
    if (hist && count < cap) hist[count] = r;
    ++count;
    return super::finished(r);
  }
  template <typename Vector>
  bool finished(const Vector& r) {
    return finished(double(two_norm(r)));
  }
  bool finished() const { return super::finished(); }
  double* hist;
  int cap, count;
};

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

enum { PC_IDENTITY = 0, PC_DIAGONAL = 1, PC_ILU0 = 2, PC_IC0 = 3, PC_ILU0_FLOAT = 4, PC_IC0_FLOAT = 5 };

template <typename PC>
int run_solver(int method, const matrix_type& A, vector_type& x, const vector_type& b, const PC& P,
               recording_iteration& iter) {
  if (method == 0) return itl::cg(A, x, b, P, iter);
  return itl::bicgstab(A, x, b, P, iter);
}

}  // namespace

extern "C" {

// laplacian_setup(A, m, n) (mtl/matrix/laplacian_setup.hpp:25-44); returns nnz.
// With rp == nullptr only the size is returned.
int ref_laplacian_setup(unsigned m, unsigned n, int* rp, int* ci, double* v) {
  matrix_type A(m * n, m * n);
  mtl::mat::laplacian_setup(A, m, n);
  return export_csr(A, rp, ci, v);
}

// mode 0: y = A*x, 1: y += A*x, 2: y -= A*x  (crtp_base_vector.hpp:92-103,192-200,269-277)
int ref_spmv(int n, int nnz, const int* rp, const int* ci, const double* v, const double* x,
             double* y, int mode) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  vector_type xv = make_vector(n, x), yv = make_vector(n, y);
  if (mode == 0)
    yv = A * xv;
  else if (mode == 1)
    yv += A * xv;
  else
    yv -= A * xv;
  store_vector(yv, y);
  return 0;
}

// Mean seconds of `reps` products w = A*v (sparse_matrix_vector_timing.cpp:66-73).
double ref_spmv_time(int n, int nnz, const int* rp, const int* ci, const double* v, const double* x,
                     int reps) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  vector_type xv = make_vector(n, x), yv(n);
  yv = A * xv;
  auto t0 = std::chrono::steady_clock::now();
  for (int r = 0; r < reps; ++r) yv = A * xv;
  return seconds_since(t0) / reps;
}

double ref_dot(int n, const double* x, const double* y) {
  vector_type a = make_vector(n, x), b = make_vector(n, y);
  return dot(a, b);
}

double ref_two_norm(int n, const double* x) {
  vector_type a = make_vector(n, x);
  return two_norm(a);
}

double ref_unary_dot(int n, const double* x) {
  vector_type a = make_vector(n, x);
  return unary_dot(a);
}

// IC(0) factors (itl/pc/ic_0.hpp:136-186): U = upper factor with inverted
// diagonal first, L = trans(U) copy with inverted diagonal last.  Both have
// nnz_u entries; returns nnz_u (sizes only when Urp == nullptr).
// as_float != 0 selects ic_0<Matrix, float> (factorise in double, store float).
int ref_ic0(int n, int nnz, const int* rp, const int* ci, const double* v, int as_float, int* Lrp,
            int* Lci, double* Lv, int* Urp, int* Uci, double* Uv) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  if (as_float) {
    itl::pc::ic_0<matrix_type, float> P(A);
    export_csr(P.get_L(), Lrp, Lci, Lv);
    return export_csr(P.get_U(), Urp, Uci, Uv);
  }
  itl::pc::ic_0<matrix_type> P(A);
  export_csr(P.get_L(), Lrp, Lci, Lv);
  return export_csr(P.get_U(), Urp, Uci, Uv);
}

// ILU(0) factors (itl/pc/ilu_0.hpp:45-82): L strict lower (unit diagonal not
// stored), U upper with inverted diagonal first.  Writes nnz of L and U to
// nnz_lu[0..1].
int ref_ilu0(int n, int nnz, const int* rp, const int* ci, const double* v, int as_float, int* nnz_lu,
             int* Lrp, int* Lci, double* Lv, int* Urp, int* Uci, double* Uv) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  if (as_float) {
    itl::pc::ilu_0<matrix_type, float> P(A);
    nnz_lu[0] = export_csr(P.get_L(), Lrp, Lci, Lv);
    nnz_lu[1] = export_csr(P.get_U(), Urp, Uci, Uv);
    return 0;
  }
  itl::pc::ilu_0<matrix_type> P(A);
  nnz_lu[0] = export_csr(P.get_L(), Lrp, Lci, Lv);
  nnz_lu[1] = export_csr(P.get_U(), Urp, Uci, Uv);
  return 0;
}

// z = solve(P, r) or adjoint_solve(P, r) for the given preconditioner kind.
int ref_pc_apply(int pc, int n, int nnz, const int* rp, const int* ci, const double* v,
                 const double* r, double* z, int adjoint) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  vector_type rv = make_vector(n, r), zv(n);
  switch (pc) {
    case PC_DIAGONAL: {
      itl::pc::diagonal<matrix_type> P(A);
      if (adjoint) zv = adjoint_solve(P, rv); else zv = solve(P, rv);
      break;
    }
    case PC_ILU0: {
      itl::pc::ilu_0<matrix_type> P(A);
      if (adjoint) zv = adjoint_solve(P, rv); else zv = solve(P, rv);
      break;
    }
    case PC_IC0: {
      itl::pc::ic_0<matrix_type> P(A);
      if (adjoint) zv = adjoint_solve(P, rv); else zv = solve(P, rv);
      break;
    }
    case PC_ILU0_FLOAT: {
      itl::pc::ilu_0<matrix_type, float> P(A);
      if (adjoint) zv = adjoint_solve(P, rv); else zv = solve(P, rv);
      break;
    }
    case PC_IC0_FLOAT: {
      itl::pc::ic_0<matrix_type, float> P(A);
      if (adjoint) zv = adjoint_solve(P, rv); else zv = solve(P, rv);
      break;
    }
    default:
      zv = rv;
  }
  store_vector(zv, z);
  return 0;
}

// Full solve.  method 0 = itl::cg, 1 = itl::bicgstab.  The iteration object is
// basic_iteration(norm_r0, max_iter, rtol, atol) with norm_r0 = two_norm(b)
// when norm_r0 < 0 (the (r0, ...) constructor used by the reference tests).
// x holds the initial guess on entry and the solution on exit.
// out[0] = iterations, out[1] = last residual, out[2] = norm_r0,
// out[3] = seconds in the preconditioner constructor, out[4] = seconds in the
// solver call, out[5] = number of termination tests recorded.
// Returns the solver's error code (0 converged, 1 too many iterations), or
// -2 when the reference threw itl::unexpected_orthogonality, -3 for other
// MTL exceptions.
int ref_solve(int method, int pc, int n, int nnz, const int* rp, const int* ci, const double* v,
              const double* b, double* x, int max_iter, double rtol, double atol, double norm_r0,
              double* hist, int hist_cap, double* out) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  vector_type bv = make_vector(n, b), xv = make_vector(n, x);
  if (norm_r0 < 0) norm_r0 = two_norm(bv);
  recording_iteration iter(norm_r0, max_iter, rtol, atol, hist, hist_cap);
  int err = 0;
  double tf = 0, ts = 0;
  try {
    auto t0 = std::chrono::steady_clock::now();
    switch (pc) {
      case PC_IDENTITY: {
        itl::pc::identity<matrix_type> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      case PC_DIAGONAL: {
        itl::pc::diagonal<matrix_type> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      case PC_ILU0: {
        itl::pc::ilu_0<matrix_type> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      case PC_IC0: {
        itl::pc::ic_0<matrix_type> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      case PC_ILU0_FLOAT: {
        itl::pc::ilu_0<matrix_type, float> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      case PC_IC0_FLOAT: {
        itl::pc::ic_0<matrix_type, float> P(A);
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        err = run_solver(method, A, xv, bv, P, iter);
        break;
      }
      default:
        return -4;
    }
    ts = seconds_since(t0);
  } catch (itl::unexpected_orthogonality&) {
    err = -2;
  } catch (mtl::runtime_error&) {
    err = -3;
  } catch (mtl::logic_error&) {
    err = -3;
  }
  store_vector(xv, x);
  if (out) {
    out[0] = iter.iterations();
    out[1] = iter.resid();
    out[2] = norm_r0;
    out[3] = tf;
    out[4] = ts;
    out[5] = iter.count;
  }
  return err;
}

// Assembly through mtl::mat::inserter<compressed2D, Updater>
// (compressed2D.hpp:662-1151, update.hpp:26-111).  The matrix starts as the
// base CSR (base_nnz entries, possibly none); then every triplet k goes in as
// ins[rows[k]][cols[k]] << vals[k] (the class updater: 0 store, 1 plus,
// 2 minus, 3 times), or, with syntax != nullptr, as syntax[k] == 0:
// ins[r][c] = v, 1: ins[r][c] += v, 2: ins[r][c] << v.  slot_size is the
// inserter's (5 when 0).  The result is exported to rp / ci / v (capacity
// base_nnz + count entries); returns nnz, -1 on an updater out of range.
// *seconds receives the time from the inserter's construction to its
// destruction.
int ref_assemble(int n_rows, int n_cols, int base_nnz, const int* brp, const int* bci,
                 const double* bv, long long count, const int* rows, const int* cols,
                 const double* vals, const unsigned char* syntax, int updater, int slot_size,
                 int* rp, int* ci, double* v, double* seconds) {
  const unsigned nr = unsigned(n_rows), nc = unsigned(n_cols);
  matrix_type A(nr, nc);
  if (base_nnz > 0) {
    std::vector<unsigned> major(brp, brp + n_rows + 1), minor(bci, bci + base_nnz);
    std::vector<double> data(bv, bv + base_nnz);
    matrix_type B(nr, nc, unsigned(base_nnz), major.data(),
                  minor.data(), data.data());
    A = B;
  }
  const unsigned slots = slot_size > 0 ? unsigned(slot_size) : 5u;
  auto run = [&](auto updater_tag) {
    typedef decltype(updater_tag) U;
    auto t0 = std::chrono::steady_clock::now();
    {
      mtl::mat::inserter<matrix_type, U> ins(A, slots);
      for (long long k = 0; k < count; ++k) {
        const unsigned r = unsigned(rows[k]), c = unsigned(cols[k]);
        if (!syntax || syntax[k] == 2)
          ins[r][c] << vals[k];
        else if (syntax[k] == 0)
          ins[r][c] = vals[k];
        else
          ins[r][c] += vals[k];
      }
    }
    if (seconds) *seconds = seconds_since(t0);
  };
  switch (updater) {
    case 0: run(mtl::operations::update_store<double>()); break;
    case 1: run(mtl::operations::update_plus<double>()); break;
    case 2: run(mtl::operations::update_minus<double>()); break;
    case 3: run(mtl::operations::update_times<double>()); break;
    default: return -1;
  }
  return export_csr(A, rp, ci, v);
}

// The other ITL Krylov methods, called as the reference's tests call them:
//   method 2 bicg(A, x, b, L, iter)                     itl/krylov/bicg.hpp:22-63
//          3 cgs(A, x, b, L, iter)                      itl/krylov/cgs.hpp:23-65
//          4 bicgstab_2(A, x, b, L, iter)               itl/krylov/bicgstab_2.hpp:33-131
//          5 bicgstab_ell(A, x, b, L, R, iter, param)   itl/krylov/bicgstab_ell.hpp:37-132
//          6 tfqmr(A, x, b, L, R, iter)                 itl/krylov/tfqmr.hpp:26-100
//          7 qmr(A, x, b, L, R, iter)                   itl/krylov/qmr.hpp:24-109
//          8 idr_s(A, x, b, L, R, iter, param)          itl/krylov/idr_s.hpp:30-105
//          9 gmres(A, x, b, L, R, iter, param)          itl/krylov/gmres.hpp:121-135
// pc_left / pc_right: 0 identity, 1 diagonal, 2 ilu_0, 3 ic_0.  idr_s's
// random shadow space is drawn as in a fresh process (mtl::seed counter
// reset to 0 before the call, mtl/operation/random.hpp:27-37).  Returns and
// fills out[] as ref_solve does.
int ref_solve_krylov(int method, int pc_left, int pc_right, int param, int n, int nnz,
                     const int* rp, const int* ci, const double* v, const double* b, double* x,
                     int max_iter, double rtol, double atol, double norm_r0, double* hist,
                     int hist_cap, double* out) {
  matrix_type A = make_matrix(n, nnz, rp, ci, v);
  vector_type bv = make_vector(n, b), xv = make_vector(n, x);
  if (norm_r0 < 0) norm_r0 = two_norm(bv);
  recording_iteration iter(norm_r0, max_iter, rtol, atol, hist, hist_cap);
  int err = 0;
  double tf = 0, ts = 0;
  auto with_pc = [&](int kind, auto&& body) {
    switch (kind) {
      case PC_IDENTITY: { itl::pc::identity<matrix_type> P(A); body(P); break; }
      case PC_DIAGONAL: { itl::pc::diagonal<matrix_type> P(A); body(P); break; }
      case PC_ILU0: { itl::pc::ilu_0<matrix_type> P(A); body(P); break; }
      case PC_IC0: { itl::pc::ic_0<matrix_type> P(A); body(P); break; }
      default: err = -4;
    }
  };
  try {
    auto t0 = std::chrono::steady_clock::now();
    with_pc(pc_left, [&](auto& L) {
      with_pc(pc_right, [&](auto& R) {
        tf = seconds_since(t0);
        t0 = std::chrono::steady_clock::now();
        const size_t prm = size_t(param);
        switch (method) {
          case 2: err = itl::bicg(A, xv, bv, L, iter); break;
          case 3: err = itl::cgs(A, xv, bv, L, iter); break;
          case 4: err = itl::bicgstab_2(A, xv, bv, L, iter); break;
          case 5: err = itl::bicgstab_ell(A, xv, bv, L, R, iter, prm ? prm : 8); break;
          case 6: err = itl::tfqmr(A, xv, bv, L, R, iter); break;
          case 7: err = itl::qmr(A, xv, bv, L, R, iter); break;
          case 8:
            mtl::seed<double>::counter = 0;
            err = itl::idr_s(A, xv, bv, L, R, iter, prm ? prm : 8);
            break;
          case 9: err = itl::gmres(A, xv, bv, L, R, iter, prm ? prm : 8); break;
          default: err = -4;
        }
        ts = seconds_since(t0);
      });
    });
  } catch (itl::unexpected_orthogonality&) {
    err = -2;
  } catch (mtl::runtime_error&) {
    err = -3;
  } catch (mtl::logic_error&) {
    err = -3;
  }
  store_vector(xv, x);
  if (out) {
    out[0] = iter.iterations();
    out[1] = iter.resid();
    out[2] = norm_r0;
    out[3] = tf;
    out[4] = ts;
    out[5] = iter.count;
  }
  return err;
}

// Build-flavour tag, so callers can report how the baseline was compiled.
const char* ref_build_info(void) {
#ifdef MTL_WITH_OPENMP
  return "MTL4 reference headers, OpenMP (MTL_WITH_OPENMP)";
#else
  return "MTL4 reference headers, serial";
#endif
}

int ref_omp_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
