// Row sampling of the boosting loop, for the CPU oracle (test
// infrastructure only; the product has its own implementation).
//   next_random:       xorshift64* state update and output,
//                      src/boosting/booster.cpp:1219-1225
//   random_subsample:  the first (Index)(n * ratio) entries of 0..n-1
//                      shuffled by std::shuffle with std::mt19937_64 seeded
//                      by one next_random() draw, src/core/dataset.cpp:552-562
// std::shuffle and std::mt19937_64 are called (not restated), so the
// permutation is libstdc++'s, as in the reference build.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <random>
#include <vector>

extern "C" uint64_t tco_next_random(uint64_t* state) {
  uint64_t s = *state;
  s ^= s >> 12;
  s ^= s << 25;
  s ^= s >> 27;
  *state = s;
  return s * 0x2545F4914F6CDD1DULL;
}

extern "C" uint32_t tco_random_subsample(uint32_t n, float ratio, uint64_t seed, uint32_t* out) {
  const uint32_t m = static_cast<uint32_t>(n * ratio);  // Index * Float, as the reference
  std::vector<uint32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::mt19937_64 rng(seed);
  std::shuffle(idx.begin(), idx.end(), rng);
  std::copy(idx.begin(), idx.begin() + m, out);
  return m;
}
