// MTL4/ITL names over the mtlgpu C ABI -- header-only C++.
//
// Reference code of the form
//
//     itl::pc::ic_0<Matrix>        P(A);                    // itl/pc/ic_0.hpp:57
//     itl::cyclic_iteration<double> iter(b, 1000, 1e-10);   // itl/iteration/cyclic_iteration.hpp:44
//     itl::cg(A, x, b, P, iter);                            // itl/krylov/cg.hpp:75-112
//
// runs on the GPU when Matrix is mtl::gpu::compressed2D<double> and x, b are
// mtl::gpu::dense_vector<double>.  The whole solve runs on the device through
// mtlgpu_solve; afterwards the residual sequence the device recorded is
// replayed through the caller's iteration object (finished(r) / ++iter in the
// reference's order), so the object ends in the state the reference's loop
// leaves it in: iterations(), resid(), error_code(), and the log lines a
// cyclic_iteration prints.
//
// Two modes.
//  * With MTL4: include <boost/numeric/mtl/mtl.hpp> and
//    <boost/numeric/itl/itl.hpp> BEFORE this header.  The reference's own
//    iteration classes, exceptions and preconditioner templates are used;
//    this header adds partial specialisations of itl::pc::identity, diagonal,
//    ilu_0 and ic_0 for mtl::gpu::compressed2D, itl::cg / itl::bicgstab
//    overloads that overload resolution prefers for device arguments (also
//    from inside itl::cg_solver / bicgstab_solver, through argument-dependent
//    lookup), and conversions from and to mtl::compressed2D / dense_vector.
//  * Standalone (no MTL4 headers seen): the same names are defined here with
//    the reference's interfaces -- basic_iteration, cyclic_iteration,
//    noisy_iteration (itl/iteration/*.hpp), the exception types
//    (mtl/utility/exception.hpp:95-232, itl/utility/exception.hpp:22-31) and
//    the preconditioner templates -- so reference-style code compiles without
//    MTL4.
//
// Errors: the C ABI's status codes are raised as the reference's exceptions
// (missing_diagonal, matrix_not_square, incompatible_size,
// index_out_of_range, itl::unexpected_orthogonality for a BiCGSTAB
// breakdown).  A zero pivot is not an error, as in the reference, which
// carries on with inf/NaN factor entries.
//
// Ownership follows the C ABI: matrices and vectors own device buffers,
// preconditioners share their factor handle between copies (the reference
// copies factors by value; the device factors are immutable, so sharing them
// is not observable) and must not outlive their matrix.
#ifndef MTLGPU_MTL_HPP
#define MTLGPU_MTL_HPP

#include <cmath>
#include <cstdint>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../mtlgpu.h"

#if defined(ITL_ITL_INCLUDE) && defined(MTL_MTL_INCLUDE)
#define MTLGPU_WITH_MTL4 1
#elif defined(ITL_ITL_INCLUDE) || defined(MTL_MTL_INCLUDE) || defined(ITL_BASIC_ITERATION_INCLUDE)
#error "include both <boost/numeric/mtl/mtl.hpp> and <boost/numeric/itl/itl.hpp> before <mtlgpu/mtl.hpp>"
#endif

// ---------------------------------------------------------------------------
// Standalone definitions of the reference's names (skipped with MTL4).
#ifndef MTLGPU_WITH_MTL4
namespace mtl {

struct index_out_of_range : std::out_of_range {
  explicit index_out_of_range(const char* s = "Index out of range") : std::out_of_range(s) {}
};
struct domain_error : std::domain_error {
  explicit domain_error(const char* s = "Argument out of domain") : std::domain_error(s) {}
};
struct incompatible_size : domain_error {
  explicit incompatible_size(const char* s = "Arguments have incompatible size.")
      : domain_error(s) {}
};
struct matrix_not_square : domain_error {
  explicit matrix_not_square(const char* s = "Matrix must be square for this operation.")
      : domain_error(s) {}
};
struct missing_diagonal : domain_error {
  explicit missing_diagonal(const char* s = "Diagonal entry missing or not where it belongs to.")
      : domain_error(s) {}
};
struct runtime_error : std::runtime_error {
  explicit runtime_error(const char* s = "Run-time error") : std::runtime_error(s) {}
};
struct logic_error : std::logic_error {
  explicit logic_error(const char* s = "Logic error") : std::logic_error(s) {}
};

template <typename T>
struct Collection;

}  // namespace mtl

namespace itl {

struct search_space_exhaustion : mtl::runtime_error {
  explicit search_space_exhaustion(
      const char* s = "Iterative solvers that exhausted the search space, i.e. search "
                      "direction(s) parallel to already visited Krylov subspace")
      : mtl::runtime_error(s) {}
};
struct unexpected_orthogonality : search_space_exhaustion {};

/// Iteration control with the interface of itl::basic_iteration
/// (itl/iteration/basic_iteration.hpp:24-164): converged when
/// resid <= rtol * ||r0|| or resid <= atol (atol only when ||r0|| == 0);
/// error 1 after max_iter iterations.
template <class Real>
class basic_iteration {
 public:
  typedef basic_iteration self;
  typedef Real real;

  template <class Vector>
  basic_iteration(const Vector& r0, int max_iter, Real rtol, Real atol = Real(0))
      : norm_r0_(std::abs(two_norm(r0))), max_iter_(max_iter), rtol_(rtol), atol_(atol) {}
  basic_iteration(Real norm_r0, int max_iter, Real rtol, Real atol = Real(0))
      : norm_r0_(norm_r0), max_iter_(max_iter), rtol_(rtol), atol_(atol) {}
  virtual ~basic_iteration() {}

  bool check_max() {
    if (i_ >= max_iter_) {
      error_ = 1;
      finished_ = true;
      msg_ = "Too many iterations.";
    }
    return finished_;
  }
  template <class Vector>
  bool finished(const Vector& r) {
    return test(Real(two_norm(r)));
  }
  bool finished(const Real& r) { return test(r); }
  bool finished() const { return finished_; }
  template <class T>
  int terminate(const T& r) {
    finished(r);
    return error_;
  }

  self& operator++() {
    ++i_;
    return *this;
  }
  self& operator+=(int n) {
    i_ += n;
    return *this;
  }
  bool first() const { return i_ <= 1; }
  virtual operator int() const { return error_; }
  virtual int error_code() const { return error_; }
  bool is_converged() const { return finished_ && error_ == 0; }
  int iterations() const { return i_; }
  int max_iterations() const { return max_iter_; }
  void set_max_iterations(int m) { max_iter_ = m; }
  void restart() { i_ = 0; }
  Real resid() const { return resid_; }
  Real relresid() const { return resid_ / norm_r0_; }
  Real normb() const { return norm_r0_; }
  Real norm_r0() const { return norm_r0_; }
  void set_norm_r0(Real r0) { norm_r0_ = r0; }
  Real tol() const { return rtol_; }
  Real atol() const { return atol_; }
  int fail(int code) {
    error_ = code;
    return error_code();
  }
  int fail(int code, const std::string& msg) {
    error_ = code;
    msg_ = msg;
    return error_code();
  }
  void set(Real v) { norm_r0_ = v; }
  void set_quite(bool q) { quiet_ = q; }
  bool is_quite() const { return quiet_; }
  void suppress_resume(bool s) { suppress_ = s; }
  bool resume_suppressed() const { return suppress_; }

 protected:
  bool test(Real r) {
    resid_ = r;
    const bool conv = norm_r0_ == 0 ? resid_ <= atol_ : (resid_ <= rtol_ * norm_r0_ || resid_ <= atol_);
    if (conv) return finished_ = true;
    return check_max();
  }

  int error_ = 0, i_ = 0;
  Real norm_r0_;
  int max_iter_;
  Real rtol_, atol_, resid_ = Real(0);
  std::string msg_;
  bool finished_ = false, quiet_ = false, suppress_ = false;
};

/// itl::cyclic_iteration (itl/iteration/cyclic_iteration.hpp:24-101): prints
/// "iteration i: resid r" every `cycle` iterations and a resume from
/// error_code().
template <class Real, class OStream = std::ostream>
class cyclic_iteration : public basic_iteration<Real> {
  typedef basic_iteration<Real> super;

 public:
  template <class Vector>
  cyclic_iteration(const Vector& r0, int max_iter, Real rtol, Real atol = Real(0),
                   int cycle = 100, OStream& out = std::cout)
      : super(r0, max_iter, rtol, atol), cycle_(cycle), out_(out) {}
  cyclic_iteration(Real r0, int max_iter, Real rtol, Real atol = Real(0), int cycle = 100,
                   OStream& out = std::cout)
      : super(r0, max_iter, rtol, atol), cycle_(cycle), out_(out) {}

  bool finished() { return super::finished(); }
  template <typename T>
  bool finished(const T& r) {
    const bool ret = super::finished(r);
    if (!this->quiet_ && this->i_ % cycle_ == 0 && (multi_print_ || this->i_ != last_print_)) {
      out_ << "iteration " << this->i_ << ": resid " << this->resid() << std::endl;
      last_print_ = this->i_;
    }
    return ret;
  }
  cyclic_iteration& operator++() {
    ++this->i_;
    return *this;
  }
  cyclic_iteration& operator+=(int n) {
    this->i_ += n;
    return *this;
  }
  operator int() const { return error_code(); }
  bool is_multi_print() const { return multi_print_; }
  void set_multi_print(bool m) { multi_print_ = m; }
  void set_cycle(int c) { cycle_ = c; }
  int error_code() const {
    if (!this->suppress_)
      out_ << "finished! error code = " << this->error_ << '\n'
           << this->iterations() << " iterations\n"
           << this->resid() << " is actual final residual. \n"
           << this->relresid() << " is actual relative tolerance achieved. \n"
           << "Relative tol: " << this->rtol_ << "  Absolute tol: " << this->atol_ << '\n'
           << "Convergence:  " << std::pow(this->relresid(), 1.0 / double(this->iterations()))
           << std::endl;
    return this->error_;
  }

 protected:
  int cycle_, last_print_ = -1;
  bool multi_print_ = false;
  OStream& out_;
};

/// itl::noisy_iteration (itl/iteration/noisy_iteration.hpp:21-30): prints
/// every iteration.
template <class Real, class OStream = std::ostream>
class noisy_iteration : public cyclic_iteration<Real, OStream> {
 public:
  template <class Vector>
  noisy_iteration(const Vector& r0, int max_iter, Real rtol, Real atol = Real(0),
                  OStream& out = std::cout)
      : cyclic_iteration<Real, OStream>(r0, max_iter, rtol, atol, 1, out) {}
};

namespace pc {
template <typename Matrix, typename Value = double>
class identity;
template <typename Matrix, typename Value = typename mtl::Collection<Matrix>::value_type>
class diagonal;
template <typename Matrix, typename Value = typename mtl::Collection<Matrix>::value_type>
class ilu_0;
template <typename Matrix, typename Value = typename mtl::Collection<Matrix>::value_type>
class ic_0;
}  // namespace pc
}  // namespace itl
#endif  // !MTLGPU_WITH_MTL4

// ---------------------------------------------------------------------------
// Device types.
namespace mtl {
namespace gpu {

/// Raise the reference's exception for a C-ABI status (OK and MAX_ITER pass).
inline void throw_on(int status, mtlgpu_ctx* ctx = nullptr) {
  switch (status) {
    case MTLGPU_OK:
    case MTLGPU_MAX_ITER:
    case MTLGPU_ZERO_PIVOT:  // the reference carries on with inf/NaN entries
      return;
    case MTLGPU_NOT_SQUARE: throw mtl::matrix_not_square();
    case MTLGPU_MISSING_DIAGONAL: throw mtl::missing_diagonal();
    case MTLGPU_INCOMPATIBLE_SIZE: throw mtl::incompatible_size();
    case MTLGPU_INDEX_RANGE: throw mtl::index_out_of_range();
    case MTLGPU_BREAKDOWN: throw itl::unexpected_orthogonality();
    case MTLGPU_INVALID_ARG:
    case MTLGPU_NOT_SORTED: throw mtl::logic_error(mtlgpu_status_string(status));
    default: {
      std::string m = mtlgpu_status_string(status);
      if (ctx && mtlgpu_last_error(ctx)) m += std::string(": ") + mtlgpu_last_error(ctx);
      throw mtl::runtime_error(m.c_str());
    }
  }
}

/// A device and its stream (one mtlgpu_ctx).  default_context() is a
/// process-wide context on device 0, created on first use.
class context {
 public:
  explicit context(int device = 0) {
    mtlgpu_ctx* c = nullptr;
    throw_on(mtlgpu_ctx_create(device, &c));
    ctx_.reset(c, [](mtlgpu_ctx* p) { mtlgpu_ctx_destroy(p); });
  }
  mtlgpu_ctx* get() const { return ctx_.get(); }
  void synchronize() const { throw_on(mtlgpu_ctx_synchronize(get()), get()); }
  static context& default_context() {
    static context c(0);
    return c;
  }

 private:
  std::shared_ptr<mtlgpu_ctx> ctx_;
};

template <typename Value>
class dense_vector;
template <typename Value>
class compressed2D;

template <typename Value>
struct scaled_vector {  // alpha * v
  Value alpha;
  const dense_vector<Value>* v;
};
template <typename Value>
struct mat_cvec_product {  // A * x
  const compressed2D<Value>* A;
  const dense_vector<Value>* x;
};
template <typename Value>
struct trans_mat_cvec_product {  // trans(A) * x
  const compressed2D<Value>* A;
  const dense_vector<Value>* x;
};
template <typename Pc, typename Value>
struct pc_solve {  // solve(P, r)
  const Pc* P;
  const dense_vector<Value>* r;
  bool adjoint;
};

/// Device vector of float64 (mtl::dense_vector on the device).
template <typename Value = double>
class dense_vector {
  static_assert(std::is_same<Value, double>::value, "device vectors are float64");

 public:
  typedef Value value_type;
  typedef int size_type;

  explicit dense_vector(int n = 0, context& c = context::default_context()) : ctx_(c) { alloc(n); }
  dense_vector(int n, Value v, context& c = context::default_context()) : ctx_(c) {
    alloc(n);
    *this = v;
  }
  dense_vector(const std::vector<Value>& h, context& c = context::default_context()) : ctx_(c) {
    alloc(int(h.size()));
    upload(h.data());
  }
#ifdef MTLGPU_WITH_MTL4
  template <typename P>
  explicit dense_vector(const mtl::vec::dense_vector<Value, P>& h,
                        context& c = context::default_context())
      : ctx_(c) {
    alloc(int(mtl::size(h)));
    if (n_) upload(&h[0]);
  }
  /// Copy back into an MTL4 vector of the same size.
  template <typename P>
  void copy_to(mtl::vec::dense_vector<Value, P>& h) const {
    if (int(mtl::size(h)) != n_) throw mtl::incompatible_size();
    if (n_) download(&h[0]);
  }
#endif
  dense_vector(const dense_vector& o) : ctx_(o.ctx_) {
    alloc(o.n_);
    copy_from(o);
  }
  dense_vector(dense_vector&& o) noexcept : ctx_(o.ctx_), n_(o.n_), d_(std::move(o.d_)) { o.n_ = 0; }
  dense_vector& operator=(const dense_vector& o) {
    if (this != &o) {
      if (o.n_ != n_) throw mtl::incompatible_size();
      copy_from(o);
    }
    return *this;
  }

  int size() const { return n_; }
  Value* data() { return static_cast<Value*>(d_.get()); }
  const Value* data() const { return static_cast<const Value*>(d_.get()); }
  context& ctx() const { return ctx_; }

  void upload(const Value* h) {
    if (n_) throw_on(mtlgpu_memcpy_h2d(ctx_.get(), data(), h, sizeof(Value) * n_), ctx_.get());
  }
  void download(Value* h) const {
    if (n_)
      throw_on(mtlgpu_memcpy_d2h(ctx_.get(), h, data(), sizeof(Value) * n_), ctx_.get());
  }
  std::vector<Value> to_host() const {
    std::vector<Value> h(n_);
    download(h.data());
    return h;
  }
  /// Element read (one device-to-host copy; for tests and checks).
  Value operator[](int i) const {
    if (i < 0 || i >= n_) throw mtl::index_out_of_range();
    Value v;
    throw_on(mtlgpu_memcpy_d2h(ctx_.get(), &v, data() + i, sizeof(Value)), ctx_.get());
    return v;
  }

  dense_vector& operator=(Value v) {  // x = 0.0
    std::vector<Value> h(n_, v);
    upload(h.data());
    return *this;
  }
  dense_vector& operator=(const mat_cvec_product<Value>& p) { return spmv(p, 1.0, 0.0); }
  dense_vector& operator+=(const mat_cvec_product<Value>& p) { return spmv(p, 1.0, 1.0); }
  dense_vector& operator-=(const mat_cvec_product<Value>& p) { return spmv(p, -1.0, 1.0); }
  dense_vector& operator=(const trans_mat_cvec_product<Value>& p);
  dense_vector& operator+=(const scaled_vector<Value>& s) {  // x += alpha * p
    check_size(s.v->n_);
    throw_on(mtlgpu_axpy(ctx_.get(), n_, s.alpha, s.v->data(), data()), ctx_.get());
    return *this;
  }
  dense_vector& operator-=(const scaled_vector<Value>& s) {
    return *this += scaled_vector<Value>{-s.alpha, s.v};
  }
  dense_vector& operator+=(const dense_vector& o) { return *this += scaled_vector<Value>{1.0, &o}; }
  dense_vector& operator-=(const dense_vector& o) { return *this += scaled_vector<Value>{-1.0, &o}; }
  template <typename Pc>
  dense_vector& operator=(const pc_solve<Pc, Value>& s) {
    if (s.adjoint)
      s.P->adjoint_solve(*s.r, *this);
    else
      s.P->solve(*s.r, *this);
    return *this;
  }

 private:
  void alloc(int n) {
    if (n < 0) throw mtl::logic_error("negative vector size");
    n_ = n;
    void* p = nullptr;
    if (n) throw_on(mtlgpu_malloc(ctx_.get(), sizeof(Value) * n, &p), ctx_.get());
    mtlgpu_ctx* c = ctx_.get();
    d_.reset(p, [c](void* q) {
      if (q) mtlgpu_free(c, q);
    });
  }
  void check_size(int m) const {
    if (m != n_) throw mtl::incompatible_size();
  }
  void copy_from(const dense_vector& o) {
    if (!n_) return;
    *this = 0.0;
    *this += scaled_vector<Value>{1.0, &o};
  }
  dense_vector& spmv(const mat_cvec_product<Value>& p, double alpha, double beta);

  context& ctx_;
  int n_ = 0;
  std::shared_ptr<void> d_;
};

template <typename Value>
inline scaled_vector<Value> operator*(Value alpha, const dense_vector<Value>& v) {
  return {alpha, &v};
}
template <typename Value>
inline int size(const dense_vector<Value>& v) {
  return v.size();
}
/// dot(x, y) (mtl/operation/dot.hpp:226-232)
template <typename Value>
inline Value dot(const dense_vector<Value>& x, const dense_vector<Value>& y) {
  if (x.size() != y.size()) throw mtl::incompatible_size();
  Value r = 0;
  throw_on(mtlgpu_dot(x.ctx().get(), x.size(), x.data(), y.data(), &r), x.ctx().get());
  return r;
}
/// two_norm(x) (mtl/operation/two_norm.hpp:33-57)
template <typename Value>
inline Value two_norm(const dense_vector<Value>& x) {
  Value r = 0;
  throw_on(mtlgpu_two_norm(x.ctx().get(), x.size(), x.data(), &r), x.ctx().get());
  return r;
}
/// unary_dot(x) = x . x (mtl/operation/unary_dot.hpp:29-65)
template <typename Value>
inline Value unary_dot(const dense_vector<Value>& x) {
  Value r = 0;
  throw_on(mtlgpu_unary_dot(x.ctx().get(), x.size(), x.data(), &r), x.ctx().get());
  return r;
}

/// A factor or matrix copied to the host in CSR form (get_L()/get_U()).
struct host_csr {
  int num_rows = 0, num_cols = 0;
  std::vector<int32_t> starts, indices;
  std::vector<double> data;
  double operator()(int r, int c) const {  // element lookup; 0 when not stored
    for (int j = starts[r]; j < starts[r + 1]; ++j)
      if (indices[j] == c) return data[j];
    return 0.0;
  }
};

/// CSR matrix on the device (mtl::compressed2D<double>): int32 row starts and
/// column indices, float64 values, rows sorted by column.
template <typename Value = double>
class compressed2D {
  static_assert(std::is_same<Value, double>::value, "device matrices hold float64 values");

 public:
  typedef Value value_type;
  typedef int size_type;

  /// The raw-array constructor of compressed2D (mtl/matrix/compressed2D.hpp:355-364).
  compressed2D(int num_rows, int num_cols, int nnz, const int32_t* starts, const int32_t* indices,
               const Value* data, context& c = context::default_context())
      : ctx_(c) {
    create(num_rows, num_cols, nnz, starts, indices, data);
  }
#ifdef MTLGPU_WITH_MTL4
  /// Copy an MTL4 compressed2D to the device (address_major/minor/data,
  /// mtl/matrix/compressed2D.hpp:610-620).
  template <typename P>
  explicit compressed2D(const mtl::mat::compressed2D<Value, P>& A,
                        context& c = context::default_context())
      : ctx_(c) {
    const int n = int(A.num_rows()), m = int(A.num_cols()), nnz = int(A.nnz());
    std::vector<int32_t> s(A.ref_major().begin(), A.ref_major().end());
    std::vector<int32_t> ix(A.ref_minor().begin(), A.ref_minor().end());
    create(n, m, nnz, s.data(), ix.data(), nnz ? A.address_data() : nullptr);
  }
#endif
  /// An empty num_rows x num_cols matrix (compressed2D(r, c), filled by an
  /// inserter or laplacian_setup).
  compressed2D(int num_rows, int num_cols, context& c = context::default_context()) : ctx_(c) {
    change_dim(num_rows, num_cols);
  }
  /// change_dim (compressed2D.hpp:441-451): new dimensions, no entries.
  void change_dim(int num_rows, int num_cols) {
    std::vector<int32_t> s(size_t(num_rows) + 1, 0);
    create(num_rows, num_cols, 0, s.data(), nullptr, nullptr);
  }
  /// Take ownership of a handle built by the library (assembly, generators).
  void adopt(mtlgpu_csr* A) {
    int n = 0, m = 0, nz = 0;
    throw_on(mtlgpu_csr_info(A, &n, &m, &nz), ctx_.get());
    h_.reset(A, [](mtlgpu_csr* p) { mtlgpu_csr_destroy(p); });
    n_rows_ = n;
    n_cols_ = m;
    nnz_ = nz;
  }
  /// The CSR arrays copied to the host.
  host_csr to_host() const {
    host_csr h;
    h.num_rows = n_rows_;
    h.num_cols = n_cols_;
    h.starts.resize(size_t(n_rows_) + 1);
    h.indices.resize(size_t(nnz_));
    h.data.resize(size_t(nnz_));
    const int32_t *rp = nullptr, *ci = nullptr;
    const double* v = nullptr;
    throw_on(mtlgpu_csr_device_arrays(handle(), &rp, &ci, &v), ctx_.get());
    throw_on(mtlgpu_memcpy_d2h(ctx_.get(), h.starts.data(), rp, sizeof(int32_t) * h.starts.size()),
             ctx_.get());
    if (nnz_) {
      throw_on(mtlgpu_memcpy_d2h(ctx_.get(), h.indices.data(), ci, sizeof(int32_t) * nnz_),
               ctx_.get());
      throw_on(mtlgpu_memcpy_d2h(ctx_.get(), h.data.data(), v, sizeof(double) * nnz_), ctx_.get());
    }
    return h;
  }
  int num_rows() const { return n_rows_; }
  int num_cols() const { return n_cols_; }
  int nnz() const { return nnz_; }
  mtlgpu_csr* handle() const { return h_.get(); }
  context& ctx() const { return ctx_; }
  /// Pick SpMV row-bin thresholds by timing candidates on this matrix.
  int autotune() {
    int choice = 0;
    throw_on(mtlgpu_csr_autotune(handle(), &choice), ctx_.get());
    return choice;
  }

 private:
  void create(int n, int m, int nnz, const int32_t* s, const int32_t* ix, const Value* v) {
    mtlgpu_csr* A = nullptr;
    throw_on(mtlgpu_csr_create(ctx_.get(), n, m, nnz, s, ix, v, &A), ctx_.get());
    h_.reset(A, [](mtlgpu_csr* p) { mtlgpu_csr_destroy(p); });
    n_rows_ = n;
    n_cols_ = m;
    nnz_ = nnz;
  }
  context& ctx_;
  std::shared_ptr<mtlgpu_csr> h_;
  int n_rows_ = 0, n_cols_ = 0, nnz_ = 0;
};

template <typename Value>
inline int num_rows(const compressed2D<Value>& A) {
  return A.num_rows();
}
template <typename Value>
inline int num_cols(const compressed2D<Value>& A) {
  return A.num_cols();
}
template <typename Value>
inline int size(const compressed2D<Value>& A) {
  return A.num_rows() * A.num_cols();
}
template <typename Value>
inline mat_cvec_product<Value> operator*(const compressed2D<Value>& A, const dense_vector<Value>& x) {
  return {&A, &x};
}
/// Updater code of the C ABI for an updater type (mtl/operation/update.hpp:26-111).
template <typename Updater>
struct updater_code {
  static const int value = MTLGPU_UPDATE_STORE;
};

/// Insertion into a device matrix with the semantics of
/// mtl::mat::inserter<compressed2D, Updater> (mtl/matrix/compressed2D.hpp:
/// 662-1151): ins[r][c] << v applies the inserter's updater, ins[r][c] = v
/// stores, ins[r][c] += v adds; entries the matrix already holds are kept
/// and updated.  Triplets are collected on the host and assembled on the
/// device (mtlgpu_csr_assemble) by finish() or the destructor, as the
/// reference's inserter finishes in its destructor.  The slot size is
/// accepted for interface compatibility; it never changes the result.
template <typename Updater>
class device_inserter {
 public:
  typedef double value_type;
  explicit device_inserter(compressed2D<double>& A, int slot_size = 5) : A_(A) {
    (void)slot_size;
  }
  device_inserter(const device_inserter&) = delete;
  device_inserter& operator=(const device_inserter&) = delete;
  ~device_inserter() {
    try {
      finish();
    } catch (...) {  // a destructor must not throw; call finish() to see errors
    }
  }
  struct proxy {
    device_inserter& ins;
    int r, c;
    template <typename V>
    proxy& operator<<(const V& v) {
      ins.add(r, c, double(v), updater_code<Updater>::value);
      return *this;
    }
    template <typename V>
    proxy& operator=(const V& v) {
      ins.add(r, c, double(v), MTLGPU_UPDATE_STORE);
      return *this;
    }
    template <typename V>
    proxy& operator+=(const V& v) {
      ins.add(r, c, double(v), MTLGPU_UPDATE_PLUS);
      return *this;
    }
  };
  struct bracket {
    device_inserter& ins;
    int r;
    proxy operator[](int c) { return {ins, r, c}; }
  };
  bracket operator[](int r) { return {*this, r}; }
  proxy operator()(int r, int c) { return {*this, r, c}; }

  /// Assembles the collected triplets into the matrix (once).
  void finish() {
    if (done_) return;
    done_ = true;
    mtlgpu_ctx* ctx = A_.ctx().get();
    const long long n = (long long)rows_.size();
    void *dr = nullptr, *dc = nullptr, *dv = nullptr, *dop = nullptr;
    auto release = [&]() {
      for (void* p : {dr, dc, dv, dop})
        if (p) mtlgpu_free(ctx, p);
    };
    mtlgpu_csr* out = nullptr;
    int st = MTLGPU_OK;
    if (n > 0) {
      st = mtlgpu_malloc(ctx, sizeof(int32_t) * n, &dr);
      if (st == MTLGPU_OK) st = mtlgpu_malloc(ctx, sizeof(int32_t) * n, &dc);
      if (st == MTLGPU_OK) st = mtlgpu_malloc(ctx, sizeof(double) * n, &dv);
      if (st == MTLGPU_OK) st = mtlgpu_malloc(ctx, n, &dop);
      if (st == MTLGPU_OK) st = mtlgpu_memcpy_h2d(ctx, dr, rows_.data(), sizeof(int32_t) * n);
      if (st == MTLGPU_OK) st = mtlgpu_memcpy_h2d(ctx, dc, cols_.data(), sizeof(int32_t) * n);
      if (st == MTLGPU_OK) st = mtlgpu_memcpy_h2d(ctx, dv, vals_.data(), sizeof(double) * n);
      if (st == MTLGPU_OK) st = mtlgpu_memcpy_h2d(ctx, dop, ops_.data(), n);
    }
    if (st == MTLGPU_OK)
      st = mtlgpu_csr_assemble(ctx, A_.nnz() ? A_.handle() : nullptr, A_.num_rows(),
                               A_.num_cols(), n, static_cast<const int32_t*>(dr),
                               static_cast<const int32_t*>(dc), static_cast<const double*>(dv),
                               static_cast<const uint8_t*>(dop), updater_code<Updater>::value,
                               &out);
    release();
    throw_on(st, ctx);
    A_.adopt(out);
  }

 private:
  void add(int r, int c, double v, int op) {
    rows_.push_back(r);
    cols_.push_back(c);
    vals_.push_back(v);
    ops_.push_back(uint8_t(op));
  }
  compressed2D<double>& A_;
  std::vector<int32_t> rows_, cols_;
  std::vector<double> vals_;
  std::vector<uint8_t> ops_;
  bool done_ = false;
};

template <typename Value>
struct transposed_view {
  const compressed2D<Value>* A;
};
template <typename Value>
inline transposed_view<Value> trans(const compressed2D<Value>& A) {
  return {&A};
}
template <typename Value>
inline trans_mat_cvec_product<Value> operator*(const transposed_view<Value>& T,
                                               const dense_vector<Value>& x) {
  return {T.A, &x};
}
/// mult(A, x, y): y = A * x (mtl/operation/mult.hpp:43-55)
template <typename Value>
inline void mult(const compressed2D<Value>& A, const dense_vector<Value>& x, dense_vector<Value>& y) {
  y = A * x;
}

template <typename Value>
dense_vector<Value>& dense_vector<Value>::spmv(const mat_cvec_product<Value>& p, double alpha,
                                               double beta) {
  if (p.A->num_cols() != p.x->size() || p.A->num_rows() != n_) throw mtl::incompatible_size();
  if (p.x->data() == data()) throw mtl::logic_error("y = A * x with y aliasing x");
  throw_on(mtlgpu_spmv(p.A->handle(), p.x->data(), data(), alpha, beta), ctx_.get());
  return *this;
}
template <typename Value>
dense_vector<Value>& dense_vector<Value>::operator=(const trans_mat_cvec_product<Value>& p) {
  if (p.A->num_rows() != p.x->size() || p.A->num_cols() != n_) throw mtl::incompatible_size();
  throw_on(mtlgpu_spmv_transposed(p.A->handle(), p.x->data(), data()), ctx_.get());
  return *this;
}

/// Device preconditioner shared by the itl::pc specialisations.
class device_pc {
 public:
  device_pc(const compressed2D<double>& A, int kind, int prec) : A_(&A) {
    if (kind == MTLGPU_PC_IDENTITY) return;
    mtlgpu_pc* P = nullptr;
    const int st = mtlgpu_pc_create(A.handle(), kind, prec, &P);
    if (P) h_.reset(P, [](mtlgpu_pc* p) { mtlgpu_pc_destroy(p); });
    factor_status_ = st;
    throw_on(st, A.ctx().get());
  }
  mtlgpu_pc* handle() const { return h_.get(); }
  /// MTLGPU_ZERO_PIVOT when a pivot was zero/negative/non-finite, else OK.
  int factor_status() const { return factor_status_; }

  void solve(const dense_vector<double>& r, dense_vector<double>& z) const { apply(r, z, false); }
  void adjoint_solve(const dense_vector<double>& r, dense_vector<double>& z) const {
    apply(r, z, true);
  }
  dense_vector<double> solve(const dense_vector<double>& r) const {
    dense_vector<double> z(r.size(), r.ctx());
    apply(r, z, false);
    return z;
  }
  dense_vector<double> adjoint_solve(const dense_vector<double>& r) const {
    dense_vector<double> z(r.size(), r.ctx());
    apply(r, z, true);
    return z;
  }

 protected:
  host_csr factor(int which) const {
    host_csr f;
    int nnz = 0;
    throw_on(mtlgpu_pc_factor_info(handle(), which, &nnz, nullptr), A_->ctx().get());
    f.num_rows = f.num_cols = A_->num_rows();
    f.starts.resize(f.num_rows + 1);
    f.indices.resize(nnz);
    f.data.resize(nnz);
    throw_on(mtlgpu_pc_get_factor(handle(), which, f.starts.data(), f.indices.data(), f.data.data()),
             A_->ctx().get());
    return f;
  }

 private:
  void apply(const dense_vector<double>& r, dense_vector<double>& z, bool adj) const {
    if (r.size() != A_->num_rows() || z.size() != r.size()) throw mtl::incompatible_size();
    if (!handle()) {  // identity
      z = r;
      return;
    }
    const int st = adj ? mtlgpu_pc_adjoint_apply(handle(), r.data(), z.data())
                       : mtlgpu_pc_apply(handle(), r.data(), z.data());
    throw_on(st, A_->ctx().get());
  }
  const compressed2D<double>* A_;
  std::shared_ptr<mtlgpu_pc> h_;
  int factor_status_ = MTLGPU_OK;
};

template <typename V>
struct factor_precision {
  static_assert(std::is_same<V, double>::value || std::is_same<V, float>::value,
                "factors are stored as double or float");
  static const int value = std::is_same<V, float>::value ? MTLGPU_FP32 : MTLGPU_FP64;
};

/// Iterative refinement request for itl::cg / itl::bicgstab: the inner
/// Krylov solve, its factors and its SpMV run in FP32, the outer residual
/// r = b - A x, the update x += d and the stopping norm in FP64.  Needs a
/// preconditioner with float factors (ic_0<M, float>, ilu_0<M, float>,
/// diagonal<M, float>) or identity.
struct refinement {
  double inner_rtol = 0;  // 0: library default
  int inner_max_iter = 0;
  int max_outer = 0;
  refinement() {}
  explicit refinement(double rtol, int inner_max = 0, int outer = 0)
      : inner_rtol(rtol), inner_max_iter(inner_max), max_outer(outer) {}
};

/// Differentiable solve x = A^{-1} b with autograd-Function semantics and no
/// PyTorch dependency: forward(b) solves and keeps x; backward(dL/dx) solves
/// the adjoint A^T lambda = dL/dx with the same preconditioned Krylov path
/// and returns dL/db = lambda and dL/dvals(A)[k] = -lambda_i x_j for every
/// stored entry k = (i, j) of A.  symmetric = true: CG on A for both solves
/// (A^T = A); false: BiCGSTAB on A and on A^T (a transposed handle and its
/// own preconditioner).
class linear_solve {
 public:
  explicit linear_solve(const compressed2D<double>& A, int pc_kind = MTLGPU_PC_IC0,
                        bool symmetric = true, double rtol = 1e-12, int max_iter = 10000)
      : A_(&A), sym_(symmetric), rtol_(rtol), max_iter_(max_iter), x_(A.num_rows(), A.ctx()) {
    mtlgpu_ctx* c = A.ctx().get();
    P_ = make_pc(A.handle(), pc_kind, c);
    if (!symmetric) {
      mtlgpu_csr* t = nullptr;
      throw_on(mtlgpu_csr_create_transpose(A.handle(), &t), c);
      AT_.reset(t, [](mtlgpu_csr* q) { mtlgpu_csr_destroy(q); });
      PT_ = make_pc(t, pc_kind, c);
    }
  }
  /// x = A^{-1} b (kept for backward)
  const dense_vector<double>& forward(const dense_vector<double>& b) {
    x_ = 0.0;
    fwd_it_ = solve(A_->handle(), P_.get(), x_, b);
    return x_;
  }
  /// dL/db and dL/dvals(A) from dL/dx at the last forward solution
  void backward(const dense_vector<double>& dl_dx, dense_vector<double>& grad_b,
                dense_vector<double>& grad_vals) {
    if (grad_vals.size() != A_->nnz() || grad_b.size() != A_->num_rows())
      throw mtl::incompatible_size();
    grad_b = 0.0;
    bwd_it_ = sym_ ? solve(A_->handle(), P_.get(), grad_b, dl_dx)
                   : solve(AT_.get(), PT_.get(), grad_b, dl_dx);
    throw_on(mtlgpu_csr_values_grad(A_->handle(), grad_b.data(), x_.data(), grad_vals.data()),
             A_->ctx().get());
  }
  const dense_vector<double>& x() const { return x_; }
  int forward_iterations() const { return fwd_it_; }
  int backward_iterations() const { return bwd_it_; }

 private:
  static std::shared_ptr<mtlgpu_pc> make_pc(mtlgpu_csr* M, int kind, mtlgpu_ctx* c) {
    if (kind == MTLGPU_PC_IDENTITY) return nullptr;
    mtlgpu_pc* P = nullptr;
    const int st = mtlgpu_pc_create(M, kind, MTLGPU_FP64, &P);
    std::shared_ptr<mtlgpu_pc> h(P, [](mtlgpu_pc* q) {
      if (q) mtlgpu_pc_destroy(q);
    });
    throw_on(st, c);
    return h;
  }
  int solve(mtlgpu_csr* M, mtlgpu_pc* P, dense_vector<double>& x, const dense_vector<double>& b) {
    mtlgpu_iter_params p;
    mtlgpu_iter_params_default(&p);
    p.max_iter = max_iter_;
    p.rtol = rtol_;
    mtlgpu_iter_result r;
    const int st = mtlgpu_solve(sym_ ? MTLGPU_CG : MTLGPU_BICGSTAB, M, P, x.data(), b.data(), &p, &r);
    if (st == MTLGPU_MAX_ITER) throw mtl::runtime_error("linear_solve: iteration limit reached");
    throw_on(st, A_->ctx().get());
    return r.iterations;
  }
  const compressed2D<double>* A_;
  bool sym_;
  double rtol_;
  int max_iter_;
  dense_vector<double> x_;
  std::shared_ptr<mtlgpu_pc> P_, PT_;
  std::shared_ptr<mtlgpu_csr> AT_;
  int fwd_it_ = 0, bwd_it_ = 0;
};

namespace detail {

template <typename Pc>
inline mtlgpu_pc* pc_handle(const Pc& P) {
  return P.handle();
}

/// Run one device solve and replay its residual sequence through `iter` in
/// the order the reference's loop calls the termination test:
/// CG (itl/krylov/cg.hpp:93-110): finished(r0), then per iteration ++iter,
/// finished(r_k); BiCGSTAB (itl/krylov/bicgstab.hpp:40-73): finished(r0),
/// then per iteration ++iter, finished(s_k), finished(r_k).
template <typename Iteration>
int solve(int method, const compressed2D<double>& A, dense_vector<double>& x,
          const dense_vector<double>& b, mtlgpu_pc* P, Iteration& iter, const refinement* mixed) {
  typedef typename Iteration::real Real;
  if (A.num_rows() != A.num_cols()) throw mtl::matrix_not_square();
  if (x.size() != A.num_cols() || b.size() != A.num_rows()) throw mtl::incompatible_size();
  mtlgpu_iter_params p;
  mtlgpu_iter_params_default(&p);
  p.max_iter = iter.max_iterations() - iter.iterations();
  p.rtol = iter.tol();
  p.atol = iter.atol();
  p.norm_r0 = iter.norm_r0();
  std::vector<double> hist;
  if (mixed) {
    p.mode = MTLGPU_SOLVE_MIXED_REFINED;
    p.inner_rtol = mixed->inner_rtol;
    p.inner_max_iter = mixed->inner_max_iter;
    p.max_outer = mixed->max_outer;
  } else {
    hist.resize(size_t(2) * (p.max_iter > 0 ? p.max_iter : 0) + 2);
    p.h_resid_history = hist.data();
    p.history_cap = int(hist.size());
  }
  mtlgpu_iter_result res;
  const int st = mtlgpu_solve(method, A.handle(), P, x.data(), b.data(), &p, &res);
  if (st != MTLGPU_OK && st != MTLGPU_MAX_ITER && st != MTLGPU_BREAKDOWN)
    throw_on(st, A.ctx().get());
  if (mixed) {
    iter += res.iterations;
    iter.finished(Real(res.true_resid));
  } else {
    const int per_iter = method == MTLGPU_BICGSTAB ? 2 : 1;
    bool done = res.history_len == 0 || iter.finished(Real(hist[0]));
    for (int k = 1; !done && k < res.history_len;) {
      ++iter;
      for (int t = 0; t < per_iter && k < res.history_len && !done; ++t, ++k)
        done = iter.finished(Real(hist[k]));
    }
    if (st == MTLGPU_BREAKDOWN) {
      if (!done) ++iter;
      throw itl::unexpected_orthogonality();
    }
  }
  return iter;
}

/// The other Krylov methods (mtlgpu_solve_krylov).  The device records every
/// residual the reference's loop passes to finished(); they are replayed
/// through `iter` one per iteration after the first (bicg, cgs: finished(r0),
/// then ++iter, finished(r_k)); for the methods that test several times per
/// iteration or at the top of their loop, the iteration object is advanced
/// to the device's count and given the last residual.  A breakdown returns
/// iter.fail(code) as the reference does; idr_s's singular LU raises
/// mtl::runtime_error ("matrix singular").
template <typename Iteration>
int solve_krylov(int method, const compressed2D<double>& A, dense_vector<double>& x,
                 const dense_vector<double>& b, mtlgpu_pc* L, mtlgpu_pc* R, int param,
                 Iteration& iter) {
  typedef typename Iteration::real Real;
  if (A.num_rows() != A.num_cols()) throw mtl::matrix_not_square();
  if (x.size() != A.num_cols() || b.size() != A.num_rows()) throw mtl::incompatible_size();
  mtlgpu_iter_params p;
  mtlgpu_iter_params_default(&p);
  p.max_iter = iter.max_iterations() - iter.iterations();
  p.rtol = iter.tol();
  p.atol = iter.atol();
  p.norm_r0 = iter.norm_r0();
  std::vector<double> hist(size_t(param + 4) * size_t(p.max_iter > 0 ? p.max_iter + 2 : 2));
  p.h_resid_history = hist.data();
  p.history_cap = int(hist.size());
  mtlgpu_iter_result res;
  const int st = mtlgpu_solve_krylov(method, A.handle(), L, R, param, x.data(), b.data(), &p,
                                     &res);
  if (st != MTLGPU_OK && st != MTLGPU_MAX_ITER && st != MTLGPU_BREAKDOWN)
    throw_on(st, A.ctx().get());
  const int n_hist = std::min(res.history_len, int(hist.size()));
  if (method == MTLGPU_BICG || method == MTLGPU_CGS) {
    bool done = n_hist == 0 || iter.finished(Real(hist[0]));
    for (int k = 1; !done && k < n_hist; ++k) {
      ++iter;
      done = iter.finished(Real(hist[k]));
    }
    while (iter.iterations() < res.iterations) ++iter;  // breakdown inside an iteration
  } else {
    iter += res.iterations;
    iter.finished(Real(res.resid));
  }
  if (st == MTLGPU_BREAKDOWN) {
    if (method == MTLGPU_IDR_S) throw mtl::runtime_error("matrix singular");
    return iter.fail(res.error);
  }
  return iter;
}

}  // namespace detail
}  // namespace gpu

#ifndef MTLGPU_WITH_MTL4
// The updaters of mtl/operation/update.hpp:26-111 (standalone definitions).
namespace operations {
template <typename Element>
struct update_store {
  template <typename Value>
  Element& operator()(Element& x, const Value& y) { return x = Element(y); }
  template <typename Value>
  Element init(const Value& y) { return y; }
};
template <typename Element>
struct update_plus {
  template <typename Value>
  Element& operator()(Element& x, const Value& y) { return x += Element(y); }
  template <typename Value>
  Element init(const Value& y) { return y; }
};
template <typename Element>
struct update_minus {
  template <typename Value>
  Element& operator()(Element& x, const Value& y) { return x -= Element(y); }
  template <typename Value>
  Element init(const Value& y) { return -y; }
};
template <typename Element>
struct update_times {
  template <typename Value>
  Element& operator()(Element& x, const Value& y) { return x *= y; }
  template <typename Value>
  Element init(const Value& y) { return y; }
};
}  // namespace operations
namespace mat {
/// mtl::mat::inserter (mtl/matrix/inserter.hpp:33-52), for device matrices.
template <typename Matrix, typename Updater = operations::update_store<double>>
struct inserter;
}  // namespace mat
#endif

namespace gpu {
template <>
struct updater_code<mtl::operations::update_plus<double>> {
  static const int value = MTLGPU_UPDATE_PLUS;
};
template <>
struct updater_code<mtl::operations::update_minus<double>> {
  static const int value = MTLGPU_UPDATE_MINUS;
};
template <>
struct updater_code<mtl::operations::update_times<double>> {
  static const int value = MTLGPU_UPDATE_TIMES;
};
}  // namespace gpu

namespace mat {
/// mtl::mat::inserter<gpu::compressed2D<double>, Updater>: the reference's
/// inserter interface, assembled on the device (gpu::device_inserter).
template <typename Updater>
struct inserter<gpu::compressed2D<double>, Updater> : gpu::device_inserter<Updater> {
  explicit inserter(gpu::compressed2D<double>& A, int slot_size = 5)
      : gpu::device_inserter<Updater>(A, slot_size) {}
};

/// laplacian_setup(A, m, n) (mtl/matrix/laplacian_setup.hpp:25-44) on a
/// device matrix: the m*n x m*n 5-point Laplacian generated on the device.
inline void laplacian_setup(gpu::compressed2D<double>& A, unsigned m, unsigned n) {
  mtlgpu_csr* out = nullptr;
  gpu::throw_on(mtlgpu_csr_laplacian2d(A.ctx().get(), int(m), int(n), &out), A.ctx().get());
  A.adopt(out);
}
}  // namespace mat

#ifdef MTLGPU_WITH_MTL4
template <typename V>
struct Collection<gpu::compressed2D<V>> {
  typedef V value_type;
  typedef V const_reference;
  typedef int size_type;
};
template <typename V>
struct Collection<gpu::dense_vector<V>> {
  typedef V value_type;
  typedef V const_reference;
  typedef int size_type;
};
#else
template <typename V>
struct Collection<gpu::compressed2D<V>> {
  typedef V value_type;
  typedef int size_type;
};
template <typename V>
struct Collection<gpu::dense_vector<V>> {
  typedef V value_type;
  typedef int size_type;
};
#endif
}  // namespace mtl

// ---------------------------------------------------------------------------
// itl::pc specialisations and itl::cg / itl::bicgstab for device arguments.
namespace itl {
namespace pc {

/// identity<M> (itl/pc/identity.hpp:24-71)
template <typename Value>
class identity<mtl::gpu::compressed2D<double>, Value> : public mtl::gpu::device_pc {
 public:
  explicit identity(const mtl::gpu::compressed2D<double>& A)
      : device_pc(A, MTLGPU_PC_IDENTITY, MTLGPU_FP64) {}
};

/// diagonal<M, V> (itl/pc/diagonal.hpp:28-103): z_i = r_i / a_ii.
template <typename Value>
class diagonal<mtl::gpu::compressed2D<double>, Value> : public mtl::gpu::device_pc {
 public:
  explicit diagonal(const mtl::gpu::compressed2D<double>& A)
      : device_pc(A, MTLGPU_PC_DIAGONAL, mtl::gpu::factor_precision<Value>::value) {}
};

/// ilu_0<M, V> (itl/pc/ilu_0.hpp:86-92, factorisation 45-82): L strictly
/// lower with unit diagonal, U upper with the inverted diagonal first.
template <typename Value>
class ilu_0<mtl::gpu::compressed2D<double>, Value> : public mtl::gpu::device_pc {
 public:
  typedef Value value_type;
  explicit ilu_0(const mtl::gpu::compressed2D<double>& A)
      : device_pc(A, MTLGPU_PC_ILU0, mtl::gpu::factor_precision<Value>::value) {}
  mtl::gpu::host_csr get_L() const { return factor(MTLGPU_LOWER); }
  mtl::gpu::host_csr get_U() const { return factor(MTLGPU_UPPER); }
};

/// ic_0<M, V> (itl/pc/ic_0.hpp:39-194): U upper with the inverted diagonal
/// first, L = trans(U) with it last.
template <typename Value>
class ic_0<mtl::gpu::compressed2D<double>, Value> : public mtl::gpu::device_pc {
 public:
  typedef Value value_type;
  explicit ic_0(const mtl::gpu::compressed2D<double>& A)
      : device_pc(A, MTLGPU_PC_IC0, mtl::gpu::factor_precision<Value>::value) {}
  mtl::gpu::host_csr get_L() const { return factor(MTLGPU_LOWER); }
  mtl::gpu::host_csr get_U() const { return factor(MTLGPU_UPPER); }
};

#define MTLGPU_PC_FREE_SOLVE(PC)                                                                  \
  template <typename V>                                                                           \
  inline mtl::gpu::pc_solve<PC<mtl::gpu::compressed2D<double>, V>, double> solve(                 \
      const PC<mtl::gpu::compressed2D<double>, V>& P, const mtl::gpu::dense_vector<double>& r) {  \
    return {&P, &r, false};                                                                       \
  }                                                                                               \
  template <typename V>                                                                           \
  inline mtl::gpu::pc_solve<PC<mtl::gpu::compressed2D<double>, V>, double> adjoint_solve(         \
      const PC<mtl::gpu::compressed2D<double>, V>& P, const mtl::gpu::dense_vector<double>& r) {  \
    return {&P, &r, true};                                                                        \
  }
// solve(P, x) / adjoint_solve(P, x) (itl/pc/ilu.hpp:189-205, ic_0.hpp:257-269,
// diagonal.hpp:90-103, identity.hpp)
MTLGPU_PC_FREE_SOLVE(identity)
MTLGPU_PC_FREE_SOLVE(diagonal)
MTLGPU_PC_FREE_SOLVE(ilu_0)
MTLGPU_PC_FREE_SOLVE(ic_0)
#undef MTLGPU_PC_FREE_SOLVE

}  // namespace pc

/// itl::cg(A, x, b, P, iter) on the device (itl/krylov/cg.hpp:75-112).
template <typename Preconditioner, typename Iteration>
int cg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
       const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter) {
  return mtl::gpu::detail::solve(MTLGPU_CG, A, x, b, mtl::gpu::detail::pc_handle(P), iter, nullptr);
}
/// itl::cg(A, x, b, iter) without preconditioner (cg.hpp:39-69).
template <typename Iteration>
int cg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
       const mtl::gpu::dense_vector<double>& b, Iteration& iter) {
  return mtl::gpu::detail::solve(MTLGPU_CG, A, x, b, nullptr, iter, nullptr);
}
/// itl::cg with a (ignored) right preconditioner (cg.hpp:115-121).
template <typename Preconditioner, typename RightPreconditioner, typename Iteration>
int cg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
       const mtl::gpu::dense_vector<double>& b, const Preconditioner& P,
       const RightPreconditioner&, Iteration& iter) {
  return cg(A, x, b, P, iter);
}
/// PCG with FP32 inner solves and FP64 iterative refinement.
template <typename Preconditioner, typename Iteration>
int cg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
       const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter,
       const mtl::gpu::refinement& how) {
  return mtl::gpu::detail::solve(MTLGPU_CG, A, x, b, mtl::gpu::detail::pc_handle(P), iter, &how);
}

/// itl::bicgstab(A, x, b, P, iter) on the device (itl/krylov/bicgstab.hpp:27-78).
template <typename Preconditioner, typename Iteration>
int bicgstab(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
             const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter) {
  return mtl::gpu::detail::solve(MTLGPU_BICGSTAB, A, x, b, mtl::gpu::detail::pc_handle(P), iter,
                                 nullptr);
}
/// BiCGSTAB with FP32 inner solves and FP64 iterative refinement.
template <typename Preconditioner, typename Iteration>
int bicgstab(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
             const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter,
             const mtl::gpu::refinement& how) {
  return mtl::gpu::detail::solve(MTLGPU_BICGSTAB, A, x, b, mtl::gpu::detail::pc_handle(P), iter,
                                 &how);
}

/// itl::bicg(A, x, b, M, iter) on the device (itl/krylov/bicg.hpp:22-63).
template <typename Preconditioner, typename Iteration>
int bicg(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
         const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_BICG, A, x, b, mtl::gpu::detail::pc_handle(P),
                                        nullptr, 0, iter);
}
/// itl::cgs(A, x, b, M, iter) (itl/krylov/cgs.hpp:23-65).
template <typename Preconditioner, typename Iteration>
int cgs(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
        const mtl::gpu::dense_vector<double>& b, const Preconditioner& P, Iteration& iter) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_CGS, A, x, b, mtl::gpu::detail::pc_handle(P),
                                        nullptr, 0, iter);
}
/// itl::bicgstab_2(A, x, b, L, iter) (itl/krylov/bicgstab_2.hpp:33-131).
template <typename Preconditioner, typename Iteration>
int bicgstab_2(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
               const mtl::gpu::dense_vector<double>& b, const Preconditioner& L, Iteration& iter) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_BICGSTAB_2, A, x, b,
                                        mtl::gpu::detail::pc_handle(L), nullptr, 2, iter);
}
/// itl::bicgstab_ell(A, x, b, L, R, iter, l) (itl/krylov/bicgstab_ell.hpp:37-132).
template <typename LeftPreconditioner, typename RightPreconditioner, typename Iteration>
int bicgstab_ell(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
                 const mtl::gpu::dense_vector<double>& b, const LeftPreconditioner& L,
                 const RightPreconditioner& R, Iteration& iter, size_t l) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_BICGSTAB_ELL, A, x, b,
                                        mtl::gpu::detail::pc_handle(L),
                                        mtl::gpu::detail::pc_handle(R), int(l), iter);
}
/// itl::tfqmr(A, x, b, L, R, iter) (itl/krylov/tfqmr.hpp:26-100).
template <typename LeftPreconditioner, typename RightPreconditioner, typename Iteration>
int tfqmr(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
          const mtl::gpu::dense_vector<double>& b, const LeftPreconditioner& L,
          const RightPreconditioner& R, Iteration& iter) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_TFQMR, A, x, b, mtl::gpu::detail::pc_handle(L),
                                        mtl::gpu::detail::pc_handle(R), 0, iter);
}
/// itl::qmr(A, x, b, L, R, iter) (itl/krylov/qmr.hpp:24-109).
template <typename LeftPreconditioner, typename RightPreconditioner, typename Iteration>
int qmr(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
        const mtl::gpu::dense_vector<double>& b, LeftPreconditioner& L,
        const RightPreconditioner& R, Iteration& iter) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_QMR, A, x, b, mtl::gpu::detail::pc_handle(L),
                                        mtl::gpu::detail::pc_handle(R), 0, iter);
}
/// itl::idr_s(A, x, b, L, R, iter, s) (itl/krylov/idr_s.hpp:30-105); both
/// preconditioners are ignored, as by the reference.
template <typename LeftPreconditioner, typename RightPreconditioner, typename Iteration>
int idr_s(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
          const mtl::gpu::dense_vector<double>& b, const LeftPreconditioner&,
          const RightPreconditioner&, Iteration& iter, size_t s) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_IDR_S, A, x, b, nullptr, nullptr, int(s), iter);
}
/// itl::gmres(A, x, b, L, R, iter, restart) (itl/krylov/gmres.hpp:121-135).
template <typename LeftPreconditioner, typename RightPreconditioner, typename Iteration>
int gmres(const mtl::gpu::compressed2D<double>& A, mtl::gpu::dense_vector<double>& x,
          const mtl::gpu::dense_vector<double>& b, LeftPreconditioner& L, RightPreconditioner& R,
          Iteration& iter, typename mtl::Collection<mtl::gpu::dense_vector<double>>::size_type restart) {
  return mtl::gpu::detail::solve_krylov(MTLGPU_GMRES, A, x, b, mtl::gpu::detail::pc_handle(L),
                                        mtl::gpu::detail::pc_handle(R), int(restart), iter);
}

}  // namespace itl

#endif  // MTLGPU_MTL_HPP
