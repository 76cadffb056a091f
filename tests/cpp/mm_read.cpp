// Reads a Matrix Market file with <mtlgpu/matrix_market.hpp> and prints its
// CSR arrays as one JSON object (for tests/test_matrix_market.py).
#include <mtlgpu/matrix_market.hpp>

#include <cstdio>

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  try {
    const mtlgpu::io::csr_matrix A = mtlgpu::io::read_matrix_market(std::string(argv[1]));
    std::printf("{\"rows\": %d, \"cols\": %d, \"starts\": [", A.n_rows, A.n_cols);
    for (size_t i = 0; i < A.starts.size(); ++i) std::printf("%s%d", i ? ", " : "", A.starts[i]);
    std::printf("], \"indices\": [");
    for (size_t i = 0; i < A.indices.size(); ++i) std::printf("%s%d", i ? ", " : "", A.indices[i]);
    std::printf("], \"data\": [");
    for (size_t i = 0; i < A.data.size(); ++i) std::printf("%s%.17g", i ? ", " : "", A.data[i]);
    std::printf("]}\n");
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
