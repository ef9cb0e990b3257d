// The random streams fit-null draws from, restated from their published
// algorithms so that probe vectors and the VR marker split follow the same
// sequence as saige-rs:
//  - ChaCha with 8 rounds (Bernstein 2008), 64-bit block counter in words
//    12-13 and 64-bit stream id in words 14-15, four blocks per refill — the
//    ChaCha8Rng of rand_chacha 0.3.1;
//  - SeedableRng::seed_from_u64 of rand_core 0.6.4: the 32-byte key is filled
//    with PCG32 (XSH-RR, O'Neill 2014) outputs;
//  - rand 0.8.5 mappings: bool = sign bit of next_u32; uniform integers in
//    [low, high) by widening multiply with the "(range << lz) - 1" zone.
//  - SliceRandom::shuffle of rand 0.8.5 (Fisher-Yates from the back; indices by
//    the u32 gen_range when they fit).
// Used by ai_reml.rs:121-130 (probes), fit_null.rs:234-240 (VR draws) and
// variance_ratio.rs:116-120 (the order in which VR markers are tried).
#pragma once
#include <stdint.h>

#include <array>

#if defined(__CUDACC__)
#define SG_HD __host__ __device__
#else
#define SG_HD
#endif

namespace saige {

// One ChaCha8 block: key words 4-11, 64-bit counter in words 12-13, stream 0.
SG_HD inline void chacha8_block(const uint32_t* key, uint64_t ctr, uint32_t* out) {
  uint32_t in[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                     key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                     static_cast<uint32_t>(ctr), static_cast<uint32_t>(ctr >> 32), 0u, 0u};
  uint32_t s[16];
  for (int i = 0; i < 16; ++i) s[i] = in[i];
  auto rotl = [](uint32_t v, int c) { return (v << c) | (v >> (32 - c)); };
  auto qr = [&](int a, int b, int c, int d) {
    s[a] += s[b]; s[d] = rotl(s[d] ^ s[a], 16);
    s[c] += s[d]; s[b] = rotl(s[b] ^ s[c], 12);
    s[a] += s[b]; s[d] = rotl(s[d] ^ s[a], 8);
    s[c] += s[d]; s[b] = rotl(s[b] ^ s[c], 7);
  };
  for (int dr = 0; dr < 4; ++dr) {
    qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
    qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; ++i) out[i] = s[i] + in[i];
}

class ChaCha8 {
 public:
  explicit ChaCha8(uint64_t seed) {
    uint64_t st = seed;
    for (int w = 0; w < 8; ++w) {
      st = st * 6364136223846793005ull + 11634580027462260723ull;
      uint32_t xs = static_cast<uint32_t>(((st >> 18) ^ st) >> 27);
      uint32_t rot = static_cast<uint32_t>(st >> 59);
      key_[w] = (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
  }

  uint32_t next_u32() {
    if (pos_ == 64) refill();
    return buf_[pos_++];
  }
  uint64_t next_u64() {
    uint64_t lo = next_u32();
    uint64_t hi = next_u32();
    return lo | (hi << 32);
  }
  bool gen_bool() { return static_cast<int32_t>(next_u32()) < 0; }

  // Key words (set by the seed); word w of the stream is word w % 16 of block w / 16.
  const uint32_t* key() const { return key_; }

  // gen_range(low..high) for u32, high > low: the 32-bit widening multiply.
  uint32_t gen_range_u32(uint32_t low, uint32_t high) {
    const uint32_t range = high - low;
    const uint32_t zone = (range << __builtin_clz(range)) - 1u;
    while (true) {
      const uint64_t wide = static_cast<uint64_t>(next_u32()) * range;
      if (static_cast<uint32_t>(wide) <= zone) return low + static_cast<uint32_t>(wide >> 32);
    }
  }

  // SliceRandom::shuffle of rand 0.8.5: Fisher-Yates from the back, the index
  // drawn with gen_range(0..i+1) on u32 when i+1 fits in 32 bits.
  template <class T>
  void shuffle(T* v, size_t len) {
    for (size_t i = len; i-- > 1;) {
      const size_t j = (i + 1) <= 0xFFFFFFFFull ? gen_range_u32(0, (uint32_t)(i + 1))
                                                 : (size_t)gen_range(0, (uint64_t)(i + 1));
      T t = v[i];
      v[i] = v[j];
      v[j] = t;
    }
  }

  // gen_range(low..high) for usize/u64, high > low.
  uint64_t gen_range(uint64_t low, uint64_t high) {
    const uint64_t range = high - low;
    const uint64_t zone = (range << __builtin_clzll(range)) - 1;
    while (true) {
      const unsigned __int128 wide = static_cast<unsigned __int128>(next_u64()) * range;
      if (static_cast<uint64_t>(wide) <= zone) return low + static_cast<uint64_t>(wide >> 64);
    }
  }

 private:
  void refill() {
    for (int b = 0; b < 4; ++b) chacha8_block(key_, counter_ + b, buf_.data() + 16 * b);
    counter_ += 4;
    pos_ = 0;
  }

  uint32_t key_[8];
  uint64_t counter_ = 0;
  std::array<uint32_t, 64> buf_{};
  int pos_ = 64;
};

}  // namespace saige
