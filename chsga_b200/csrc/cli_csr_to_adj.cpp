// Drop-in for the reference's csr_to_adj (src/csr_to_adj.cpp): a CSR text
// file to the AdjacencyGraph file, the concatenated labels and the label
// offsets, byte for byte as the reference writes them.
//
//   csr_to_adj IN.csr OUT.adj OUT.labels OUT.label_offsets
#include "cli_common.hpp"

int main(int argc, char** argv) {
  if (argc < 5) {
    std::cerr << "Usage: csr2adj IN.csr OUT.adj OUT.labels OUT.label_offsets\n";
    return 2;
  }
  if (chsga_csr_text_to_adj(argv[1], argv[2], argv[3], argv[4]) != CHSGA_OK) {
    std::cerr << chsga_last_error_global() << "\n";
    return 3;
  }
  return 0;
}
