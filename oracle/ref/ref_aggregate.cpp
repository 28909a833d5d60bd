// Harness around the reference's CPU hash aggregation,
// reference/db_operators/aggregate.cpp (compiled from where it lies).
// Test infrastructure only.
//
// hash_table_aggregate<T, U> (aggregate.cpp:40-83) accumulates with `+=` into
// thread-local absl::flat_hash_maps and merges them under omp critical.  The
// harness instantiates it with an int64 {SUM, COUNT, MIN, MAX} accumulator
// whose += merges all four, and orders the groups by key afterwards.
#include <algorithm>
#include <cstdint>
#include <vector>

struct PdAgg {
  int64_t sum, count, min, max;
  PdAgg &operator+=(const PdAgg &o) {
    sum += o.sum;
    count += o.count;
    if (o.min < min) min = o.min;
    if (o.max > max) max = o.max;
    return *this;
  }
};

#define main pimdal_ref_aggregate_main
#include "aggregate.cpp"
#undef main

extern "C" {

void pimdal_ref_set_threads(int t) { omp_set_num_threads(t); }
uint64_t pimdal_ref_aggregate_num_blocks(void) { return NUM_BLOCKS; }

// Group by int32 key: SUM/COUNT/MIN/MAX of int64 values, groups ascending by
// signed key.  Returns the number of groups.
uint64_t pimdal_ref_group_by(const int32_t *key, const int64_t *val, uint64_t n,
                             int32_t *out_key, int64_t *out_sum, int64_t *out_count,
                             int64_t *out_min, int64_t *out_max) {
  std::vector<PdAgg> v(n);
  for (uint64_t i = 0; i < n; i++) v[i] = {val[i], 1, val[i], val[i]};
  const uint32_t *k = reinterpret_cast<const uint32_t *>(key);
  absl::flat_hash_map<uint32_t, PdAgg> t = hash_table_aggregate(k, k + n, v.data(), v.data() + n);
  std::vector<std::pair<int32_t, PdAgg>> g;
  g.reserve(t.size());
  for (auto &e : t) g.push_back({(int32_t)e.first, e.second});
  std::sort(g.begin(), g.end(),
            [](const std::pair<int32_t, PdAgg> &a, const std::pair<int32_t, PdAgg> &b) {
              return a.first < b.first;
            });
  for (uint64_t i = 0; i < g.size(); i++) {
    out_key[i] = g[i].first;
    out_sum[i] = g[i].second.sum;
    out_count[i] = g[i].second.count;
    out_min[i] = g[i].second.min;
    out_max[i] = g[i].second.max;
  }
  return g.size();
}
}
