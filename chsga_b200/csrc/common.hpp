// Shared host-side definitions for libchsga: status codes, the error type
// that carries them to the C-ABI, and a deterministic random generator used
// by the synthetic-input tools.
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/chsga.h"

namespace chsga {

// Every failure inside the library is thrown as ChsgaError and converted to
// a status code plus a message at the C-ABI boundary (no exception crosses it).
struct ChsgaError : std::runtime_error {
  chsga_status status;
  ChsgaError(chsga_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void fail(chsga_status s, const std::string& msg) { throw ChsgaError(s, msg); }
inline void require(bool ok, chsga_status s, const std::string& msg) {
  if (!ok) fail(s, msg);
}
// A literal message becomes a string only when the check fails (checks run
// per element of inputs with hundreds of millions of them). Messages built
// from parts are formed before the call: in such loops, test first and
// call fail().
inline void require(bool ok, chsga_status s, const char* msg) {
  if (!ok) fail(s, msg);
}

// splitmix64 seeding + xoshiro256** stream. Fixed arithmetic so generated
// inputs are identical on every machine and library version.
struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& v : s) v = splitmix(x);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in [0, n) by 128-bit multiply (bias < 2^-64 * n, irrelevant here)
  uint64_t below(uint64_t n) { return (uint64_t)(((__uint128_t)next() * n) >> 64); }
  // uniform integer in [lo, hi]
  int64_t range(int64_t lo, int64_t hi) { return lo + (int64_t)below((uint64_t)(hi - lo + 1)); }
  // uniform double in [0, 1)
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace chsga
