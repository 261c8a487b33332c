// Drop-in for ConSGA_traceback_mismatchN_dag (src/ConSGA_traceback.cpp).
// Built a second time with -DCHSGA_MATCH_N as ConSGA_traceback_matchN_dag.
//
//   ConSGA_traceback_mismatchN_dag [-b] -I char.adj -i string.adj -c string.out
//       -r reads -l char.labels -o string.label_offsets [-k rows] [-d dir]
//
// CHSGA_SLOTS >= 4 traces all reads through chsga_align_traceback_batched
// (same paths; unless CHSGA_CKPT_FILES asks for checkpoint row files).
//
// Default mode verifies: forward scores, traceback of every read, then each
// path is rescored under the fixed costs and must equal the forward score and
// end on the last read row; exit status 0 iff all checks pass. -b times the
// traceback of each read. Checkpoint rows are kept in pinned host memory; with
// CHSGA_CKPT_FILES=1 they are also written as <dir>/read_<i>/row_<r>.bin and
// erased after use like the reference (CHSGA_KEEP_CKPT=1 keeps them).
// CHSGA_HBM_CAP_BYTES caps the full score matrix (default 85% of free HBM).
#include <getopt.h>

#include <chrono>

#include "cli_common.hpp"

int main(int argc, char** argv) {
  char *orig_char = nullptr, *orig_str = nullptr, *contr_str = nullptr, *reads_f = nullptr,
       *labels_f = nullptr, *offsets_f = nullptr;
  int64_t k = 500;
  std::string dir = "/tmp/consga_traceback_ckpts";
  bool benchmark = false;
  int opt;
  while ((opt = getopt(argc, argv, "bI:i:c:r:l:o:k:d:")) != -1) {
    switch (opt) {
      case 'b': benchmark = true; break;
      case 'I': orig_char = optarg; break;
      case 'i': orig_str = optarg; break;
      case 'c': contr_str = optarg; break;
      case 'r': reads_f = optarg; break;
      case 'l': labels_f = optarg; break;
      case 'o': offsets_f = optarg; break;
      case 'k': k = std::stoll(optarg); break;
      case 'd': dir = optarg; break;
      default:
        std::cerr << "Usage: " << argv[0]
                  << " [-b] -I orig_char -i orig_string -c contracted"
                     " -r reads -l labels -o offsets"
                     " [-k checkpoint_every_k_rows] [-d ckpt_dir]\n";
        return EXIT_FAILURE;
    }
  }
  if (!orig_char || !orig_str || !contr_str || !reads_f || !labels_f || !offsets_f) {
    std::cerr << "Error: missing required arguments\n";
    return EXIT_FAILURE;
  }
  if (k <= 0) cli::die("Error: -k must be positive", "");
  chsga_reads* reads = nullptr;
  if (chsga_reads_load(reads_f, cli::env_u64("CHSGA_MAX_READS", 5), &reads) != CHSGA_OK)
    cli::die("terminate: load_reads", chsga_last_error_global());
  chsga_host_graph* g = nullptr;
  if (chsga_graph_read_files(orig_char, orig_str, contr_str, labels_f, offsets_f, &g) != CHSGA_OK)
    cli::die("Cannot load inputs", chsga_last_error_global());
  chsga_graph_host view{};
  chsga_graph_view(g, &view);
  chsga_opts o{};
  o.device = (int)cli::env_u64("CHSGA_DEVICE", 0);
  o.flags = cli::scoring_flags();
  o.hbm_cap_bytes = cli::env_u64("CHSGA_HBM_CAP_BYTES", 0);
  chsga_ctx* ctx = nullptr;
  cli::check(chsga_open(&o, &ctx), nullptr, "chsga_open");
  cli::check(chsga_load_host_graph(ctx, g), ctx, "chsga_load_graph");
  const bool files = cli::env_u64("CHSGA_CKPT_FILES", 0) != 0;
  const bool keep = cli::env_u64("CHSGA_KEEP_CKPT", 0) != 0;

  const uint64_t n = chsga_reads_count(reads);
  const char* data = chsga_reads_data(reads);
  const uint64_t* offs = chsga_reads_offsets(reads);
  auto read_of = [&](uint64_t i) { return data + offs[i]; };
  auto len_of = [&](uint64_t i) { return (uint32_t)(offs[i + 1] - offs[i]); };
  auto run_tb = [&](uint64_t ri, chsga_tb_result* r) {
    std::string rdir = dir + "/read_" + std::to_string(ri);
    chsga_tb_opts t{k, files ? rdir.c_str() : nullptr, keep ? 1 : 0, 0};
    cli::check(chsga_align_traceback(ctx, read_of(ri), len_of(ri), &t, r), ctx,
               "chsga_align_traceback");
  };

  if (benchmark) {
    std::vector<double> per_read;
    auto t0 = std::chrono::high_resolution_clock::now();
    for (uint64_t ri = 0; ri < n; ++ri) {
      auto r0 = std::chrono::high_resolution_clock::now();
      chsga_tb_result r{};
      run_tb(ri, &r);
      chsga_tb_result_free(&r);
      per_read.push_back(
          std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - r0).count());
    }
    const double ms = std::chrono::duration<double, std::milli>(
                          std::chrono::high_resolution_clock::now() - t0).count();
    std::cout << "Average times (skipping first read), 95% CI:\n";
    cli::print_mean_with_moe_z(" Total", per_read);
    std::cout << " Substitutions: NA sec\n";
    std::cout << " Insertions:    NA sec\n";
    std::cout << "[total over " << n << " reads] : " << ms << " ms\n";
    chsga_close(ctx);
    return 0;
  }

  std::cout << "=== Forward-pass scores (align_combo) ===\n";
  std::vector<const char*> ptrs(n);
  std::vector<uint32_t> lens(n);
  std::vector<int32_t> ref(n);
  std::vector<double> tot(n);
  for (uint64_t i = 0; i < n; ++i) {
    ptrs[i] = read_of(i);
    lens[i] = len_of(i);
    auto r0 = std::chrono::steady_clock::now();
    cli::check(chsga_align_scores(ctx, &ptrs[i], &lens[i], 1, &ref[i]), ctx, "chsga_align_scores");
    tot[i] = std::chrono::duration<double>(std::chrono::steady_clock::now() - r0).count();
  }
  std::cout << "Average times (skipping first read), 95% CI:\n";
  cli::print_mean_with_moe_t(" Total", tot);
  std::cout << " Substitutions: NA\n Insertions: NA\n";
  for (uint64_t i = 0; i < n; ++i) std::cout << "read[" << i << "] score=" << ref[i] << "\n";

  std::cout << "\n=== Traceback results (align_combo_with_traceback) ===\n";
  std::cout << "  (checkpoint every k=" << k << " rows, dir=" << dir << ")\n";
  auto t0 = std::chrono::high_resolution_clock::now();
  std::vector<chsga_tb_result> res(n);
  const uint32_t slots = (uint32_t)cli::env_u64("CHSGA_SLOTS", 0);
  if (slots >= 4 && !files) {
    // every read at once: full-matrix reads through the batched engine
    chsga_tb_opts t{k, nullptr, keep ? 1 : 0, 0};
    cli::check(chsga_align_traceback_batched(ctx, ptrs.data(), lens.data(), (uint32_t)n, &t,
                                             std::min<uint32_t>(slots, 64), res.data()),
               ctx, "chsga_align_traceback_batched");
  } else {
    for (uint64_t ri = 0; ri < n; ++ri) run_tb(ri, &res[ri]);
  }
  const double ms = std::chrono::duration<double, std::milli>(
                        std::chrono::high_resolution_clock::now() - t0).count();
  bool all_ok = true;
  for (uint64_t ri = 0; ri < n; ++ri) {
    const chsga_tb_result& r = res[ri];
    const char* rd = read_of(ri);
    std::string cigar(chsga_ops_to_cigar(r.ops, r.num_ops, nullptr, 0), '\0');
    chsga_ops_to_cigar(r.ops, r.num_ops, cigar.data(), cigar.size() + 1);
    int path_score = 0, read_pos = -1;
    for (uint64_t j = 0; j < r.num_ops; ++j) {
      const chsga_op& op = r.ops[j];
      if (op.op == CHSGA_OP_DELETE) {
        path_score += 1;
        read_pos = (int)op.row;
      } else if (op.op == CHSGA_OP_MATCHSUB) {
        // byte equality, as the reference's check (ConSGA_traceback.cpp:198-199),
        // in its matchN build too: an N-matched step counts as a substitution
        path_score += view.labels[op.vertex] == rd[op.row] ? 0 : 1;
        read_pos = (int)op.row;
      } else {
        path_score += 1;
      }
    }
    const bool score_ok = path_score == ref[ri];
    const bool len_ok = read_pos == (int)len_of(ri) - 1;
    std::cout << "read[" << ri << "] = \"" << std::string(rd, len_of(ri)) << "\"\n"
              << "  CIGAR      : " << cigar << "\n"
              << "  path_score : " << path_score << "  ref_score  : " << ref[ri]
              << "  score_ok   : " << (score_ok ? "YES" : "FAIL") << "\n"
              << "  last_row   : " << read_pos << "  expected   : " << (len_of(ri) - 1)
              << "  row_ok     : " << (len_ok ? "YES" : "FAIL") << "\n";
    if (!score_ok || !len_ok) all_ok = false;
    chsga_tb_result_free(&res[ri]);
  }
  std::cout << "\n[traceback time] " << ms << " ms\n";
  std::cout << "\n[RESULT] " << (all_ok ? "ALL CHECKS PASSED" : "SOME CHECKS FAILED") << "\n";
  chsga_close(ctx);
  chsga_graph_free(g);
  chsga_reads_free(reads);
  return all_ok ? 0 : 1;
}
