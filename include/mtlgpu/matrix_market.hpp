// Matrix Market reader for the CSR handle -- header-only, host code.
//
// Reads what mtl::io::matrix_market_istream::read (mtl/io/matrix_market.hpp:
// 44-219, read_matrix 101-211) reads into a compressed2D, with the same
// meaning:
//   - header "%%MatrixMarket matrix <coordinate|array> <real|integer|pattern>
//     <general|symmetric|skew-symmetric|hermitian>", then '%' comment lines,
//     then "rows cols [nnz]";
//   - coordinate entries "i j [v]" are 1-based; an off-diagonal entry of a
//     symmetric (or real hermitian) file is also stored at (j, i), of a
//     skew-symmetric file with the opposite sign;
//   - pattern entries store the value 0 (as the reference does);
//   - an entry given twice keeps the last value (the reference's inserter
//     stores, it does not add);
//   - array files list rows x cols values column by column, each stored;
//   - complex files and malformed input raise io::format_error (a
//     std::runtime_error; the reference raises mtl::runtime_error).
// The result is CSR with int32 indices and every row sorted by column: the
// arrays mtlgpu_csr_create and mtl::gpu::compressed2D take.
#ifndef MTLGPU_MATRIX_MARKET_HPP
#define MTLGPU_MATRIX_MARKET_HPP

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <fstream>
#include <istream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace mtlgpu {
namespace io {

struct csr_matrix {
  int n_rows = 0, n_cols = 0;
  std::vector<int32_t> starts{0}, indices;
  std::vector<double> data;
  int nnz() const { return (int)indices.size(); }
};

/// Raised for input the reference's reader rejects.
struct format_error : std::runtime_error {
  explicit format_error(const std::string& s) : std::runtime_error(s) {}
};

inline csr_matrix read_matrix_market(std::istream& in) {
  auto lower = [](std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return std::tolower(c); });
    return s;
  };
  std::string line;
  if (!std::getline(in, line)) throw format_error("empty Matrix Market input");
  std::istringstream head(line);
  std::string marker, object, format, field, symmetry;
  head >> marker >> object >> format >> field >> symmetry;
  if (marker != "%%MatrixMarket") throw format_error("File not in Matrix Market format");
  // object and field are compared as written, format and symmetry after
  // lowering them (matrix_market.hpp:171-196)
  if (object != "matrix") throw format_error("Try to read matrix from non-matrix file");
  format = lower(format);
  symmetry = lower(symmetry);
  if (format != "coordinate" && format != "array") throw format_error("unknown Matrix Market format");
  if (field == "complex") throw format_error("Cannot convert complex value in real");
  if (field != "real" && field != "integer" && field != "pattern")
    throw format_error("Unknown tag for matrix value type in file");
  int sym = 0;  // 0 general, 1 symmetric/hermitian, -1 skew
  if (symmetry == "symmetric" || symmetry == "hermitian")
    sym = 1;
  else if (symmetry == "skew-symmetric")
    sym = -1;
  else if (symmetry != "general")
    throw format_error("unknown Matrix Market symmetry");
  // comments, then the size line
  do {
    if (!std::getline(in, line)) throw format_error("missing size line");
  } while (line.empty() || line[0] == '%' ||
           line.find_first_not_of(" \t\r") == std::string::npos);
  std::istringstream sz(line);
  long long rows = -1, cols = -1, entries = -1;
  sz >> rows >> cols;
  if (format == "coordinate") sz >> entries;
  if (rows < 0 || cols < 0 || (format == "coordinate" && entries < 0) || rows > INT32_MAX ||
      cols > INT32_MAX)
    throw format_error("bad Matrix Market size line");
  // row -> (column -> value); later entries overwrite earlier ones
  std::vector<std::map<int32_t, double>> rowmap((size_t)rows);
  auto put = [&](long long r, long long c, double v) {
    if (r < 0 || r >= rows || c < 0 || c >= cols) throw format_error("entry out of range");
    rowmap[(size_t)r][(int32_t)c] = v;
  };
  if (format == "coordinate") {
    for (long long k = 0; k < entries; ++k) {
      long long i, j;
      double v = 0;
      if (!(in >> i >> j)) break;  // fewer entries than announced: stop, as the reference does
      if (field == "integer") {    // read as an integer, as the reference reads a long
        long long iv = 0;
        if (!(in >> iv)) throw format_error("missing value");
        v = (double)iv;
      } else if (field == "real") {
        if (!(in >> v)) throw format_error("missing value");
      }
      put(i - 1, j - 1, v);
      if (i != j && sym != 0) put(j - 1, i - 1, sym * v);
    }
  } else {
    for (long long c = 0; c < cols; ++c)
      for (long long r = 0; r < rows; ++r) {
        double v = 0;
        if (field == "integer") {
          long long iv = 0;
          if (!(in >> iv)) throw format_error("missing array value");
          v = (double)iv;
        } else if (field != "pattern" && !(in >> v)) {
          throw format_error("missing array value");
        }
        put(r, c, v);
      }
  }
  csr_matrix A;
  A.n_rows = (int)rows;
  A.n_cols = (int)cols;
  for (auto& row : rowmap) {
    for (auto& e : row) {
      A.indices.push_back(e.first);
      A.data.push_back(e.second);
    }
    A.starts.push_back((int32_t)A.indices.size());
  }
  return A;
}

inline csr_matrix read_matrix_market(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw format_error("cannot open " + path);
  return read_matrix_market(f);
}

}  // namespace io
}  // namespace mtlgpu

#endif  // MTLGPU_MATRIX_MARKET_HPP
