// hj_ranges.h -- the free ranges of a batch's particle pool (host only, no
// CUDA), first fit: admission takes room for a bunch, retirement gives it
// back and merges it with its free neighbours.
#pragma once

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

namespace hj_ranges {

// (start, length) of each free range: sorted, disjoint and never adjacent.
using Ranges = std::vector<std::pair<int64_t, int64_t>>;

// Room for n particles, rounded up to a multiple of 4 (at least 4, so every
// bunch starts on a 32-byte boundary), from the first free range that holds
// it.  Returns false, changing nothing, when none does.
inline bool take(Ranges& fr, int64_t n, int64_t* start, int64_t* cap) {
  const int64_t need = std::max<int64_t>((n + 3) / 4 * 4, 4);
  for (size_t i = 0; i < fr.size(); ++i) {
    auto& r = fr[i];
    if (r.second >= need) {
      *start = r.first;
      *cap = need;
      r.first += need;
      r.second -= need;
      if (r.second == 0) fr.erase(fr.begin() + i);
      return true;
    }
  }
  return false;
}

// Return [start, start + cap) to the free ranges.
inline void give(Ranges& fr, int64_t start, int64_t cap) {
  auto it = std::lower_bound(fr.begin(), fr.end(), std::make_pair(start, (int64_t)0));
  it = fr.insert(it, {start, cap});
  size_t i = it - fr.begin();
  if (i + 1 < fr.size() && fr[i].first + fr[i].second == fr[i + 1].first) {
    fr[i].second += fr[i + 1].second;
    fr.erase(fr.begin() + i + 1);
  }
  if (i > 0 && fr[i - 1].first + fr[i - 1].second == fr[i].first) {
    fr[i - 1].second += fr[i].second;
    fr.erase(fr.begin() + i);
  }
}

// Length of the largest free range.
inline int64_t largest(const Ranges& fr) {
  int64_t m = 0;
  for (const auto& r : fr) m = std::max(m, r.second);
  return m;
}

}  // namespace hj_ranges
