/* ORACLE STAND-IN — test infrastructure, not product code.
 *
 * src/load_reads.hpp includes "kseq.h" from PaSGAL's ext/kseq, which is not
 * present. This project-written header provides the part of that interface
 * load_reads uses (KSEQ_INIT, kseq_t with seq.s/seq.l, kseq_init, kseq_read,
 * kseq_destroy) with the usual FASTA/FASTQ record rules: a record starts at
 * '>' or '@'; sequence lines run until a line starting with '>', '+' or '@';
 * a FASTQ quality block ends once it is as long as the sequence. kseq_read
 * returns the sequence length, -1 at end of input, -2 on a malformed record.
 */
#pragma once
#include <zlib.h>

#include <string>

struct kseq_str_t {
  char* s;
  size_t l;
};

struct kseq_t {
  gzFile fp;
  std::string buf;
  size_t pos;
  bool eof;
  int last_char;
  std::string seq_store;
  kseq_str_t seq;
};

namespace chsga_kseq {
inline int getc_(kseq_t* k) {
  if (k->pos >= k->buf.size()) {
    if (k->eof) return -1;
    char tmp[1 << 16];
    int n = gzread(k->fp, tmp, sizeof(tmp));
    if (n <= 0) {
      k->eof = true;
      return -1;
    }
    k->buf.assign(tmp, tmp + n);
    k->pos = 0;
  }
  return (unsigned char)k->buf[k->pos++];
}
/* reads the rest of a line into out (appending), stripping a trailing '\r';
 * returns -1 if the input ended before any char */
inline int line_(kseq_t* k, std::string* out) {
  int c, got = 0;
  while ((c = getc_(k)) >= 0 && c != '\n') {
    got = 1;
    if (out) out->push_back((char)c);
  }
  if (out && !out->empty() && out->back() == '\r') out->pop_back();
  return (c < 0 && !got) ? -1 : 0;
}
}  // namespace chsga_kseq

#define KSEQ_INIT(type_t, __read) static_assert(true, "kseq stand-in")

inline kseq_t* kseq_init(gzFile fp) {
  kseq_t* k = new kseq_t();
  k->fp = fp;
  k->pos = 0;
  k->eof = false;
  k->last_char = 0;
  k->seq.s = nullptr;
  k->seq.l = 0;
  return k;
}

inline void kseq_destroy(kseq_t* k) { delete k; }

inline int kseq_read(kseq_t* k) {
  using namespace chsga_kseq;
  int c;
  if (k->last_char == 0) {
    while ((c = getc_(k)) >= 0 && c != '>' && c != '@') {
    }
    if (c < 0) return -1;
  }
  k->last_char = 0;
  line_(k, nullptr); /* name and comment */
  k->seq_store.clear();
  while ((c = getc_(k)) >= 0 && c != '>' && c != '+' && c != '@') {
    if (c == '\n') continue;
    k->seq_store.push_back((char)c);
    line_(k, &k->seq_store);
  }
  if (c == '>' || c == '@') k->last_char = c;
  k->seq.s = k->seq_store.data();
  k->seq.l = k->seq_store.size();
  if (c != '+') return (int)k->seq.l;
  line_(k, nullptr); /* rest of the '+' line */
  std::string qual;
  while (qual.size() < k->seq_store.size()) {
    if (line_(k, &qual) < 0) break;
  }
  k->seq.s = k->seq_store.data();
  if (qual.size() != k->seq_store.size()) return -2;
  return (int)k->seq.l;
}
