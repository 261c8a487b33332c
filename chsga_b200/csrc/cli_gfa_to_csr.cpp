// Counterpart of the reference's handlegraph_to_csr (src/handlegraph_to_csr.cpp)
// reading GFA v1 instead of a libbdsg PackedGraph (see chsga_gfa_to_csr_text):
//
//   gfa_to_csr <graph.gfa> <string_csr_out> <char_csr_out>
//
// Both outputs are in handlegraph_to_csr's CSR text layout, the input of
// csr_to_adj.
#include "cli_common.hpp"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::cerr << "Usage: " << argv[0] << " <graph.gfa> <string_csr_out> <char_csr_out>\n";
    return 1;
  }
  if (chsga_gfa_to_csr_text(argv[1], argv[2], argv[3]) != CHSGA_OK) {
    std::cerr << chsga_last_error_global() << "\n";
    return 1;
  }
  return 0;
}
