// Host-side containers for the alignment inputs and the file formats that
// fill them. Layouts follow the reference's producers:
//   AdjacencyGraph text (src/csr_to_adj.cpp:46-114): "AdjacencyGraph", n, m,
//     n offsets (the final offset is implied), m targets, then optionally m
//     weights ("1.0" as csr_to_adj writes them).
//   labels (src/ConSGA.cpp:159-170): raw bytes, every '\n' skipped.
//   label offsets (src/ConSGA.cpp:175-185): whitespace-separated integers.
//   hierarchy file (-c): the upstream write_pbbs_format layout lives in the
//     Parallel-Contraction-Hierarchy library, which is not available, so the
//     hierarchy is stored in the binary layout documented at write_pch().
//   checkpoint rows (src/traceback.hpp:215-237): raw native int32 x N.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "common.hpp"

namespace chsga {

struct HostCsr {
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> offset;  // n+1
  std::vector<uint32_t> target;  // m
  std::vector<uint32_t> weight;  // m, or empty = every weight 1
  uint32_t w(uint64_t e) const { return weight.empty() ? 1u : weight[e]; }
};

// Rank-ordered contraction hierarchy (PchGraph after setOrderedLayer,
// src/CHoverrides/build_pch.hpp:1199-1220).
struct HostPch {
  bool present = false;
  uint64_t n = 0, m = 0, rm = 0;
  std::vector<uint32_t> rank;          // n, by original id
  std::vector<uint32_t> level;         // n, by rank
  std::vector<uint32_t> layer_offset;  // layers+1
  std::vector<uint32_t> cc_offset;     // ccs+1
  std::vector<uint64_t> up_offset;     // n+1
  std::vector<uint32_t> up_v, up_w;    // m
  std::vector<uint64_t> down_offset;   // n+1
  std::vector<uint32_t> down_v, down_w;// rm
};

struct HostReads {
  std::vector<char> data;
  std::vector<uint64_t> offsets{0};
  uint64_t count() const { return offsets.size() - 1; }
  uint32_t len(uint64_t i) const { return (uint32_t)(offsets[i + 1] - offsets[i]); }
  const char* seq(uint64_t i) const { return data.data() + offsets[i]; }
  void add(const char* s, size_t n) {
    data.insert(data.end(), s, s + n);
    offsets.push_back(data.size());
  }
};

HostCsr read_adj(const std::string& path);
void write_adj(const std::string& path, const HostCsr& g);
std::vector<char> read_labels(const std::string& path);
void write_labels(const std::string& path, const std::vector<char>& labels);
std::vector<uint64_t> read_label_offsets(const std::string& path);
void write_label_offsets(const std::string& path, const std::vector<uint64_t>& offs);
HostPch read_pch(const std::string& path);
void write_pch(const std::string& path, const HostPch& p);
void validate_pch(const HostPch& p, uint64_t num_strings);
HostReads read_reads(const std::string& path, uint64_t max_reads);
void write_fasta(const std::string& path, const HostReads& r);

std::string ckpt_row_path(const std::string& dir, int64_t row);
void write_ckpt_row(const std::string& dir, int64_t row, const int32_t* data, uint64_t n);
void read_ckpt_row(const std::string& dir, int64_t row, int32_t* data, uint64_t n);

}  // namespace chsga

struct chsga_host_graph {
  std::vector<char> labels;
  chsga::HostCsr char_graph;
  chsga::HostCsr string_graph;
  std::vector<uint64_t> label_offsets;
  chsga::HostPch pch;
};

struct chsga_reads {
  chsga::HostReads r;
};
