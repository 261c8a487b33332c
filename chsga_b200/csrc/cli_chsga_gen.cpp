// Writes a seeded synthetic workload: the five ConSGA input files
// (<prefix>.char.adj, .string.adj, .string.out, .char.labels,
// .string.label_offsets) and a FASTA of simulated reads.
//
//   chsga_gen -o prefix [-B backbone_len] [-g bubble_gap] [-m snp,indel,alt]
//             [-S seed] [-n reads] [-L len_min[,len_max]] [-e sub,indel,N]
//             [-R read_seed] [-V vlen_max]
#include <getopt.h>

#include <cstring>
#include <sstream>

#include "cli_common.hpp"

static std::vector<double> nums(const char* s) {
  std::vector<double> v;
  std::stringstream ss(s);
  std::string t;
  while (std::getline(ss, t, ',')) v.push_back(std::atof(t.c_str()));
  return v;
}

int main(int argc, char** argv) {
  chsga_gen_graph_cfg g{100000, 1, 1.0 / (0.01 + 0.001), 0.01 / 0.011, 0.001 / 0.011, 0.0,
                        1, 10, 50, 300, 1, 32};
  chsga_gen_reads_cfg r{200, 7, 150, 150, 0.01, 0.003, 0.001, 3};
  std::string prefix;
  int c;
  while ((c = getopt(argc, argv, "o:B:g:m:S:n:L:e:R:V:I:")) != -1) {
    switch (c) {
      case 'o': prefix = optarg; break;
      case 'B': g.backbone_len = std::strtoull(optarg, nullptr, 10); break;
      case 'g': g.bubble_gap_mean = std::atof(optarg); break;
      case 'm': {
        auto v = nums(optarg);
        if (v.size() != 3) cli::die("-m wants snp,indel,alt", optarg);
        g.p_snp = v[0];
        g.p_indel = v[1];
        g.p_alt = v[2];
        break;
      }
      case 'I': {
        auto v = nums(optarg);
        if (v.size() != 4) cli::die("-I wants indel_min,indel_max,alt_min,alt_max", optarg);
        g.indel_min = (uint32_t)v[0];
        g.indel_max = (uint32_t)v[1];
        g.alt_min = (uint32_t)v[2];
        g.alt_max = (uint32_t)v[3];
        break;
      }
      case 'S': g.seed = std::strtoull(optarg, nullptr, 10); break;
      case 'n': r.count = std::strtoull(optarg, nullptr, 10); break;
      case 'L': {
        auto v = nums(optarg);
        r.len_min = (uint32_t)v[0];
        r.len_max = (uint32_t)(v.size() > 1 ? v[1] : v[0]);
        break;
      }
      case 'e': {
        auto v = nums(optarg);
        if (v.size() != 3) cli::die("-e wants sub,indel,N", optarg);
        r.sub_rate = v[0];
        r.indel_rate = v[1];
        r.n_rate = v[2];
        break;
      }
      case 'R': r.seed = std::strtoull(optarg, nullptr, 10); break;
      case 'V': g.vlen_max = (uint32_t)std::atoi(optarg); break;
      default: cli::die("usage: chsga_gen -o prefix [options]", "");
    }
  }
  if (prefix.empty()) cli::die("usage: chsga_gen -o prefix [options]", "");
  chsga_host_graph* h = nullptr;
  cli::check(chsga_gen_graph(&g, &h), nullptr, "chsga_gen_graph");
  chsga_pch_opts po{500, 1.0, 0, 1, 0x5EED, 0, 0, 0, 0};
  cli::check(chsga_build_pch(h, &po), nullptr, "chsga_build_pch");
  cli::check(chsga_graph_write_files(h, prefix.c_str()), nullptr, "chsga_graph_write_files");
  chsga_reads* rd = nullptr;
  cli::check(chsga_gen_reads(h, &r, &rd), nullptr, "chsga_gen_reads");
  cli::check(chsga_reads_write_fasta(rd, (prefix + ".reads.fa").c_str()), nullptr, "write reads");
  chsga_graph_stats s{};
  chsga_graph_get_stats(h, &s);
  std::cout << "chars " << s.num_chars << " strings " << s.num_strings << " string_edges "
            << s.num_string_edges << " pch_levels " << s.pch_levels << " reads " << r.count << "\n";
  chsga_reads_free(rd);
  chsga_graph_free(h);
  return 0;
}
