// Sampled chance mode (ChanceMode::Sampled, crates/solver/src/tree.rs:128-136):
// the random number generator the reference's tree builder draws from and the
// stratified card sample it draws (crates/solver/src/sampling.rs:9-54).
//
// The generator is rand 0.9.5's StdRng, which is rand_chacha 0.9.0's
// ChaCha12Rng: the ChaCha block function (D. J. Bernstein, "ChaCha, a variant
// of Salsa20", 2008) with 12 rounds, a 256-bit key, a 64-bit block counter
// from 0 (words 12-13) and a 64-bit stream id of 0 (words 14-15); its output
// is the keystream read as little-endian 32-bit words, and a 64-bit draw
// joins two consecutive words, low word first. StdRng::seed_from_u64 (rand_core
// 0.9) expands the u64 seed into the 32-byte key with eight steps of the PCG32
// generator (M. E. O'Neill, "PCG: A Family of Simple Fast Space-Efficient
// Statistically Good Algorithms for Random Number Generation", 2014: an LCG
// step followed by the XSH-RR output function), each step giving one key word.
// A uniform f64 in [0, 1) is the top 53 bits of a 64-bit draw times 2^-53
// (rand 0.9's StandardUniform for f64).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace dcfr {

class StdRng {
 public:
  explicit StdRng(uint64_t seed) {
    uint64_t s = seed;
    for (int i = 0; i < 8; i++) {
      s = s * 6364136223846793005ull + 11634580027462260723ull;
      const uint32_t xs = (uint32_t)(((s >> 18) ^ s) >> 27);
      const uint32_t rot = (uint32_t)(s >> 59);
      key_[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
  }

  uint64_t next_u64() {
    if (pos_ >= 16) refill();
    const uint64_t lo = words_[pos_], hi = words_[pos_ + 1];
    pos_ += 2;
    return lo | (hi << 32);
  }

  double next_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }

  // One ChaCha block (rounds = 12 for StdRng) at the given counter and stream.
  static void block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
    uint32_t x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u};
    for (int i = 0; i < 8; i++) x[4 + i] = key[i];
    x[12] = (uint32_t)counter;
    x[13] = (uint32_t)(counter >> 32);
    x[14] = (uint32_t)stream;
    x[15] = (uint32_t)(stream >> 32);
    uint32_t w[16];
    for (int i = 0; i < 16; i++) w[i] = x[i];
    for (int r = 0; r < rounds; r += 2) {
      quarter(w, 0, 4, 8, 12);
      quarter(w, 1, 5, 9, 13);
      quarter(w, 2, 6, 10, 14);
      quarter(w, 3, 7, 11, 15);
      quarter(w, 0, 5, 10, 15);
      quarter(w, 1, 6, 11, 12);
      quarter(w, 2, 7, 8, 13);
      quarter(w, 3, 4, 9, 14);
    }
    for (int i = 0; i < 16; i++) out[i] = w[i] + x[i];
  }

 private:
  static uint32_t rotl(uint32_t v, int n) { return (v << n) | (v >> (32 - n)); }
  static void quarter(uint32_t* w, int a, int b, int c, int d) {
    w[a] += w[b]; w[d] = rotl(w[d] ^ w[a], 16);
    w[c] += w[d]; w[b] = rotl(w[b] ^ w[c], 12);
    w[a] += w[b]; w[d] = rotl(w[d] ^ w[a], 8);
    w[c] += w[d]; w[b] = rotl(w[b] ^ w[c], 7);
  }
  // Draws are always 64-bit, so they never straddle a block: reading the
  // keystream one block at a time gives the same words as rand_chacha's
  // four-block buffer.
  void refill() {
    block(key_, counter_++, 0, 12, words_);
    pos_ = 0;
  }

  uint32_t key_[8];
  uint64_t counter_ = 0;
  uint32_t words_[16];
  int pos_ = 16;
};

// sample_cards (sampling.rs:9-54): k of the available cards (ascending card
// ids, card = rank * 4 + suit), each suit represented in proportion to the
// cards it has left (largest remainder, ties broken by a random key), and
// within a suit ranks spread evenly from a random offset. Four draws for the
// remainder keys (suits 0..3), then one offset draw per suit with a quota.
inline std::vector<int> sample_cards(const std::vector<int>& available, size_t k, StdRng& rng) {
  if (k >= available.size()) return available;
  std::vector<int> by_suit[4];
  for (int c : available) by_suit[c & 3].push_back(c);
  for (auto& v : by_suit) std::sort(v.begin(), v.end(), [](int a, int b) { return (a >> 2) < (b >> 2); });
  const double total = (double)available.size();
  size_t quota[4];
  struct Frac {
    double frac, key;
    int suit;
  } fr[4];
  for (int s = 0; s < 4; s++) {
    const double exact = (double)k * (double)by_suit[s].size() / total;
    const double fl = std::floor(exact);
    quota[s] = (size_t)fl;
    fr[s] = {exact - fl, rng.next_f64(), s};
  }
  size_t assigned = quota[0] + quota[1] + quota[2] + quota[3];
  // Descending by (fraction, key, suit).
  std::sort(fr, fr + 4, [](const Frac& a, const Frac& b) {
    if (a.frac != b.frac) return a.frac > b.frac;
    if (a.key != b.key) return a.key > b.key;
    return a.suit > b.suit;
  });
  for (const Frac& f : fr) {
    if (assigned >= k) break;
    if (quota[f.suit] < by_suit[f.suit].size()) {
      quota[f.suit]++;
      assigned++;
    }
  }
  std::vector<int> out;
  for (int s = 0; s < 4; s++) {
    const size_t m = by_suit[s].size(), q = quota[s];
    if (q == 0) continue;
    const double step = (double)m / (double)q;
    const double offset = rng.next_f64() * step;
    for (size_t j = 0; j < q; j++) {
      const size_t idx = std::min((size_t)std::floor(offset + (double)j * step), m - 1);
      out.push_back(by_suit[s][idx]);
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

}  // namespace dcfr
