// Drop-in for ConSGA_mismatchN_dag (src/ConSGA.cpp): score-only alignment of
// every read against the graph, printed as the reference prints it. Built a
// second time with -DCHSGA_MATCH_N as ConSGA_matchN_dag (matchN scoring).
//
//   ConSGA_mismatchN_dag -I char.adj -i string.adj -c string.out
//                        -r reads -l char.labels -o string.label_offsets
//
// Environment (extensions; the reference has no equivalents):
//   CHSGA_MAX_READS   reads to load, default 5 like src/load_reads.hpp:5; 0 = all
//   CHSGA_SLOTS       0 (default): one read per launch sequence; 2..128:
//                     the batched engine with that many read slots
//   CHSGA_DEVICE      CUDA device ordinal
#include <getopt.h>

#include <chrono>

#include "cli_common.hpp"

int main(int argc, char** argv) {
  char *orig_char = nullptr, *orig_str = nullptr, *contr_str = nullptr, *reads_f = nullptr,
       *labels_f = nullptr, *offsets_f = nullptr;
  int opt;
  while ((opt = getopt(argc, argv, "I:C:i:c:r:l:o:a:s:N:M:y:")) != -1) {
    switch (opt) {
      case 'I': orig_char = optarg; break;
      case 'i': orig_str = optarg; break;
      case 'c': contr_str = optarg; break;
      case 'r': reads_f = optarg; break;
      case 'l': labels_f = optarg; break;
      case 'o': offsets_f = optarg; break;
      default:
        std::cerr << "Usage: " << argv[0]
                  << " -I orig_char -i orig_string -c contr_string"
                     " -r reads_file -l labels_file -o offsets_file"
                     " \n";
        return EXIT_FAILURE;
    }
  }
  if (!orig_char || !orig_str || !contr_str || !reads_f || !labels_f || !offsets_f) {
    std::cerr << "Error: missing required arguments\n";
    return EXIT_FAILURE;
  }
  chsga_reads* reads = nullptr;
  {
    chsga_status s = chsga_reads_load(reads_f, cli::env_u64("CHSGA_MAX_READS", 5), &reads);
    if (s != CHSGA_OK) cli::die("terminate: load_reads", chsga_last_error_global());
  }
  auto t_in = std::chrono::steady_clock::now();
  chsga_host_graph* g = nullptr;
  chsga_status s = chsga_graph_read_files(orig_char, orig_str, contr_str, labels_f, offsets_f, &g);
  if (s != CHSGA_OK) cli::die("Cannot load inputs", chsga_last_error_global());
  chsga_opts o{};
  o.device = (int)cli::env_u64("CHSGA_DEVICE", 0);
  o.flags = cli::scoring_flags();
  chsga_ctx* ctx = nullptr;
  cli::check(chsga_open(&o, &ctx), nullptr, "chsga_open");
  auto t_ch = std::chrono::steady_clock::now();
  cli::check(chsga_load_host_graph(ctx, g), ctx, "chsga_load_graph");
  const double ch_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_ch).count();
  std::cout << "input ch time: " << ch_time << '\n';
  const double in_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_in).count();
  std::cout << "input time: " << in_time << '\n' << std::flush;

  const uint64_t n = chsga_reads_count(reads);
  const char* data = chsga_reads_data(reads);
  const uint64_t* offs = chsga_reads_offsets(reads);
  std::vector<const char*> ptrs(n);
  std::vector<uint32_t> lens(n);
  for (uint64_t i = 0; i < n; ++i) {
    ptrs[i] = data + offs[i];
    lens[i] = (uint32_t)(offs[i + 1] - offs[i]);
  }
  std::vector<int32_t> scores(n);
  std::vector<double> total(n), subst(n), ins(n);
  const uint32_t slots = (uint32_t)cli::env_u64("CHSGA_SLOTS", 0);
  auto t0 = std::chrono::high_resolution_clock::now();
  if (slots > 1) {
    chsga_batch_opts b{slots, 8, 1, 0, 0, 0};
    cli::check(chsga_align_scores_batched(ctx, ptrs.data(), lens.data(), (uint32_t)n, &b,
                                          scores.data()),
               ctx, "chsga_align_scores_batched");
    const double sec = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
    for (uint64_t i = 0; i < n; ++i) total[i] = sec / (double)n;
  } else {
    // align_combo aligns the reads one after another (src/align.hpp:488)
    for (uint64_t i = 0; i < n; ++i) {
      auto r0 = std::chrono::steady_clock::now();
      cli::check(chsga_align_scores(ctx, &ptrs[i], &lens[i], 1, &scores[i]), ctx,
                 "chsga_align_scores");
      total[i] = std::chrono::duration<double>(std::chrono::steady_clock::now() - r0).count();
    }
  }
  // the row kernel and the hierarchy closure run as one device sequence; their
  // per-phase split is not measured here
  std::cout << "Average times (skipping first read), 95% CI:\n";
  cli::print_mean_with_moe_t(" Total", total);
  std::cout << " Substitutions: NA\n Insertions: NA\n";
  auto t1 = std::chrono::high_resolution_clock::now();
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::cout << "[total over " << n << " reads] : " << ms << " ms\n";
  std::cout << "score: ";
  for (uint64_t i = 0; i < n; ++i) std::cout << (int64_t)scores[i] << (i + 1 < n ? " " : "");
  std::cout << '\n';
  chsga_close(ctx);
  chsga_graph_free(g);
  chsga_reads_free(reads);
  return 0;
}
