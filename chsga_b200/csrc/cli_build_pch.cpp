// Drop-in for build_pch (src/CHoverrides/build_pch.cpp): contraction
// hierarchy of a string graph, written as the hierarchy file ConSGA reads
// with -c.
//
//   build_pch -i string.adj -o string.out [-v string.label_offsets]
//             [-p max_pop_count] [-s select_fraction] [-k weight_bound] [-d]
//             [-g cuda_device]
//
// Differences from the reference driver: -k only sets the weight bound (the
// reference's case 'k' falls through into 'v', build_pch.cpp:79-88); -b
// (degree-bounded contraction, which leaves same-level hierarchy edges) is
// rejected; -t/-q (query verification counts) are accepted and ignored; -g
// (not in the reference) runs each round's witness searches on that CUDA
// device, with the same resulting hierarchy.
#include <getopt.h>

#include <chrono>
#include <cstring>

#include "cli_common.hpp"
#include "host_graph.hpp"

namespace chsga {
HostPch build_pch(const HostCsr& g, const std::vector<uint64_t>& offs, const chsga_pch_opts& o);
}

int main(int argc, char* argv[]) {
  if (argc < 3) {
    std::fprintf(stderr,
                 "WeightedGraph only\n"
                 "Usage: %s [-i input_graph]\n"
                 "Options:\n"
                 "\t-o,\toutput_ch_graph\n"
                 "\t-p,\tmax_pop_count\n"
                 "\t-s,\tselect fraction\n"
                 "\t-k,\tshortcut weight bound\n"
                 "\t-v,\tlabel offsets (shortcut weights count the skipped labels)\n"
                 "\t-d,\tprint per round detail\n"
                 "\t-g,\tCUDA device for the witness searches\n",
                 argv[0]);
    return 0;
  }
  const char *in = nullptr, *out = nullptr, *offs_path = nullptr;
  chsga_pch_opts o{};
  o.max_pop_count = 500;
  o.sample_bound = 1.0;
  o.seed = 0x5EED;
  int c;
  while ((c = getopt(argc, argv, "i:o:p:s:t:q:b:dk:v:g:")) != -1) {
    switch (c) {
      case 'i': in = optarg; break;
      case 'o': out = optarg; break;
      case 'p': {
        long v = std::atol(optarg);
        if (v < 0) cli::die("Error: max_pop_count must be non negative", "");
        o.max_pop_count = (uint32_t)v;
        break;
      }
      case 's':
        o.sample_bound = std::atof(optarg);
        if (o.sample_bound <= 0 || o.sample_bound > 1)
          cli::die("Error: selection_fraction must be larger than 0 and smaller than or equal to 1", "");
        break;
      case 't':
      case 'q': break;
      case 'b': cli::die("Error: -b (degree-bounded contraction) is not supported", "");
      case 'd': o.print_detail = 1; break;
      case 'k': {
        double v = std::atof(optarg);
        if (v < 0) cli::die("Error: k (shortcut weight bound) must be non-negative", "");
        o.weight_bound = (uint64_t)v;
        break;
      }
      case 'v': offs_path = optarg; break;
      case 'g':
        o.use_gpu = 1;
        o.device = std::atoi(optarg);
        break;
      default: std::fprintf(stderr, "Error: Unknown option %c\n", optopt); return EXIT_FAILURE;
    }
  }
  if (!in) cli::die("Error: -i input_graph is required", "");
  try {
    chsga::HostCsr g = chsga::read_adj(in);
    std::vector<uint64_t> offs;
    if (offs_path) {
      offs = chsga::read_label_offsets(offs_path);
      if (offs.size() != g.n + 1) cli::die("Error: label offsets do not match the graph", offs_path);
      o.use_label_lengths = 1;
    }
    auto t0 = std::chrono::high_resolution_clock::now();
    chsga::HostPch p = chsga::build_pch(g, offs, o);
    double sec = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
    std::cout << "[ build time ] : " << sec << " sec\n";
    if (out) {
      t0 = std::chrono::high_resolution_clock::now();
      chsga::write_pch(out, p);
      sec = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
      std::cout << "[ write time ] : " << sec << " sec\n";
    }
  } catch (const std::exception& e) {
    cli::die("build_pch", e.what());
  }
  return 0;
}
