// Matrix Market: <mtlgpu/matrix_market.hpp> against the reference's own
// reader (mtl::io::matrix_market_istream, mtl/io/matrix_market.hpp) on the
// same inputs.  Host-only; built where the MTL4 headers are present.  Prints
// one JSON line per case with whether both readers give the same CSR arrays.
#include <boost/numeric/mtl/mtl.hpp>

#include <mtlgpu/matrix_market.hpp>

#include <cstdio>
#include <sstream>
#include <string>
#include <vector>

namespace {

const char* kCases[][2] = {
    {"general", "%%MatrixMarket matrix coordinate real general\n% a comment\n3 4 5\n"
                "1 1 2.5\n3 4 -1\n2 2 4\n1 3 0.5\n3 1 7\n"},
    {"symmetric", "%%MatrixMarket matrix coordinate real symmetric\n4 4 6\n1 1 4\n2 1 -1\n"
                  "2 2 4\n3 2 -1\n4 4 4\n4 1 -0.5\n"},
    {"skew", "%%MatrixMarket matrix coordinate real skew-symmetric\n3 3 2\n2 1 1.5\n3 2 -2\n"},
    {"pattern", "%%MatrixMarket matrix coordinate pattern general\n3 3 4\n1 1\n2 3\n3 1\n3 3\n"},
    {"integer", "%%MatrixMarket matrix coordinate integer symmetric\n3 3 3\n1 1 5\n3 1 -2\n3 3 9\n"},
    {"duplicate", "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n1 1 3\n2 2 5\n"},
    {"array", "%%MatrixMarket matrix array real general\n2 3\n1\n2\n0\n4\n5\n6\n"},
    // an integer file holding a fraction: the value is read as an integer
    // and the reader stops at the leftover ".5"
    {"integer_fraction", "%%MatrixMarket matrix coordinate integer general\n2 2 2\n1 1 1.5\n"
                         "2 2 3\n"},
    // format and symmetry are compared after lowering them
    {"mixed_case_format", "%%MatrixMarket matrix COORDINATE real General\n2 2 1\n1 2 3\n"},
};

// Input both readers must reject.
const char* kRejected[][2] = {
    {"field_double", "%%MatrixMarket matrix coordinate double general\n1 1 1\n1 1 1\n"},
    {"object_case", "%%MatrixMarket Matrix coordinate real general\n1 1 1\n1 1 1\n"},
    {"field_case", "%%MatrixMarket matrix coordinate Real general\n1 1 1\n1 1 1\n"},
};

}  // namespace

// With file arguments: compare both readers on each file and print the CSR
// arrays of ours (one JSON line per file).
int compare_files(int argc, char** argv) {
  int fails = 0;
  for (int a = 1; a < argc; ++a) {
    mtl::compressed2D<double> R;
    mtl::io::matrix_market_istream mm(argv[a]);
    mm >> R;
    mtlgpu::io::csr_matrix G = mtlgpu::io::read_matrix_market(std::string(argv[a]));
    bool same = int(num_rows(R)) == G.n_rows && int(num_cols(R)) == G.n_cols &&
                int(R.nnz()) == G.nnz();
    for (int i = 0; same && i <= G.n_rows; ++i) same = int(R.ref_major()[i]) == G.starts[i];
    for (int k = 0; same && k < G.nnz(); ++k)
      same = int(R.ref_minor()[k]) == G.indices[k] && R.data[k] == G.data[k];
    fails += !same;
    std::printf("{\"file\": \"%s\", \"same\": %d, \"rows\": %d, \"cols\": %d, \"starts\": [",
                argv[a], int(same), G.n_rows, G.n_cols);
    for (size_t i = 0; i < G.starts.size(); ++i) std::printf("%s%d", i ? ", " : "", G.starts[i]);
    std::printf("], \"indices\": [");
    for (size_t i = 0; i < G.indices.size(); ++i) std::printf("%s%d", i ? ", " : "", G.indices[i]);
    std::printf("], \"data\": [");
    for (size_t i = 0; i < G.data.size(); ++i) std::printf("%s%.17g", i ? ", " : "", G.data[i]);
    std::printf("]}\n");
  }
  return fails ? 1 : 0;
}

int main(int argc, char** argv) {
  if (argc > 1) return compare_files(argc, argv);
  int fails = 0;
  for (auto& c : kCases) {
    std::istringstream s1(c[1]), s2(c[1]);
    mtl::compressed2D<double> R;
    mtl::io::matrix_market_istream mm(s1);
    mm >> R;
    mtlgpu::io::csr_matrix G = mtlgpu::io::read_matrix_market(s2);
    bool same = int(num_rows(R)) == G.n_rows && int(num_cols(R)) == G.n_cols &&
                int(R.nnz()) == G.nnz();
    for (int i = 0; same && i <= G.n_rows; ++i) same = int(R.ref_major()[i]) == G.starts[i];
    for (int k = 0; same && k < G.nnz(); ++k)
      same = int(R.ref_minor()[k]) == G.indices[k] && R.data[k] == G.data[k];
    fails += !same;
    std::printf("{\"case\": \"%s\", \"same\": %d, \"nnz_ref\": %d, \"nnz\": %d}\n", c[0], int(same),
                int(R.nnz()), G.nnz());
  }
  for (auto& c : kRejected) {
    std::istringstream s1(c[1]), s2(c[1]);
    bool ref_threw = false, ours_threw = false;
    try {
      mtl::compressed2D<double> R;
      mtl::io::matrix_market_istream mm(s1);
      mm >> R;
    } catch (...) {
      ref_threw = true;
    }
    try {
      mtlgpu::io::read_matrix_market(s2);
    } catch (const mtlgpu::io::format_error&) {
      ours_threw = true;
    }
    const bool same = ref_threw && ours_threw;
    fails += !same;
    std::printf("{\"case\": \"%s\", \"same\": %d, \"rejected_ref\": %d, \"rejected\": %d}\n",
                c[0], int(same), int(ref_threw), int(ours_threw));
  }
  return fails ? 1 : 0;
}
