// Row sampling of the boosting loop, for the CPU oracle (test
// infrastructure only; the product has its own implementation).
//   next_random:       xorshift64* state update and output,
//                      src/boosting/booster.cpp:1219-1225
//   random_subsample:  the first (Index)(n * ratio) entries of 0..n-1
//                      shuffled by std::shuffle with std::mt19937_64 seeded
//                      by one next_random() draw, src/core/dataset.cpp:552-562
//   goss_subsample:    below, src/core/dataset.cpp:494-549
// std::shuffle, std::nth_element, std::mt19937_64 and
// std::uniform_int_distribution are called (not restated), so the
// permutations are libstdc++'s, as in the reference build.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <random>
#include <utility>
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

// Dataset::goss_subsample (src/core/dataset.cpp:494-549) over |g| already
// taken per row (absg; softmax: the largest |g| over the classes,
// src/boosting/booster.cpp:1327-1348): the rows of the (uint32)(n * top)
// largest values after std::nth_element over (value, row) pairs in
// descending order, then (uint32)(n * other) rows (at most the rest) of a
// partial Fisher-Yates shuffle of the rest as nth_element left it, each
// position drawn by std::uniform_int_distribution<uint32_t> over
// std::mt19937_64(seed).  Rows are written in that order; returns the count.
extern "C" uint32_t tco_goss_subsample(uint32_t n, const float* absg, float top_rate, float other_rate,
                                       uint64_t seed, uint32_t* out) {
  const uint32_t top_n = static_cast<uint32_t>(n * top_rate);  // Index * Float, as the reference
  uint32_t other_n = static_cast<uint32_t>(n * other_rate);
  if (top_n == 0 && other_n == 0) return 0;
  std::vector<std::pair<float, uint32_t>> a(n);
  for (uint32_t i = 0; i < n; ++i) a[i] = {absg[i], i};
  auto desc = [](const std::pair<float, uint32_t>& l, const std::pair<float, uint32_t>& r) {
    return l.first > r.first;
  };
  if (top_n > 0 && top_n < n) std::nth_element(a.begin(), a.begin() + top_n, a.end(), desc);
  uint32_t m = 0;
  for (uint32_t i = 0; i < top_n && i < n; ++i) out[m++] = a[i].second;
  if (other_n > 0 && top_n < n) {
    const uint32_t rest = n - top_n;
    other_n = std::min(other_n, rest);
    std::mt19937_64 rng(seed);
    for (uint32_t i = 0; i < other_n; ++i) {
      std::uniform_int_distribution<uint32_t> pick(i, rest - 1);
      const uint32_t j = pick(rng);
      if (i != j) std::swap(a[top_n + i], a[top_n + j]);
      out[m++] = a[top_n + i].second;
    }
  }
  return m;
}
