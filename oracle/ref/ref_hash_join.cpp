// Harness around the reference's CPU radix-partitioned hash join,
// reference/db_operators/hash_join.cpp (compiled from where it lies).
// Test infrastructure only.
//
// partition() and join_partitions() (hash_join.cpp:57-157) are templates over
// the element type.  The harness instantiates them for a row that carries a
// payload next to the key: it converts to uint32_t for hash() (:20-25) and
// hashes / compares on the key only, so the absl::flat_hash_set built per
// partition maps a probe key to the stored build row, payload included.
#include <cstdint>
#include <utility>
#include <vector>

struct PdRow {
  uint32_t key;
  uint32_t aux;
  operator uint32_t() const { return key; }
  bool operator==(const PdRow &o) const { return key == o.key; }
  template <typename H>
  friend H AbslHashValue(H h, const PdRow &r) {
    return H::combine(std::move(h), r.key);
  }
};

#define main pimdal_ref_hash_join_main
#include "hash_join.cpp"
#undef main

extern "C" {

void pimdal_ref_set_threads(int t) { omp_set_num_threads(t); }
uint64_t pimdal_ref_hash_join_num_blocks(void) { return NUM_BLOCKS; }

// Joins build (key, payload) with probe keys (row id = index).  Writes, in the
// reference's output order (partition by partition), the build payload and
// the probe row id of every match; returns the match count.  Scratch output
// rows the reference leaves unwritten are skipped.
uint64_t pimdal_ref_hash_join(const uint32_t *bkey, const uint32_t *bpay, uint64_t nb,
                              const uint32_t *pkey, uint64_t np, uint32_t part_n,
                              uint32_t *out_payload, uint32_t *out_rowid) {
  std::vector<PdRow> inner(nb), outer(np), inner_res(np), outer_res(np);
  for (uint64_t i = 0; i < nb; i++) inner[i] = {bkey[i], bpay[i]};
  for (uint64_t i = 0; i < np; i++) outer[i] = {pkey[i], (uint32_t)i};
  for (uint64_t i = 0; i < np; i++) outer_res[i] = {0, 0xFFFFFFFFu};
  arrow::BufferVector ip = partition(inner.data(), inner.data() + nb, part_n);
  arrow::BufferVector op = partition(outer.data(), outer.data() + np, part_n);
  uint64_t joined = join_partitions(ip, op, part_n, inner_res.data(), outer_res.data());
  uint64_t k = 0;
  for (uint64_t i = 0; i < np && k < joined; i++) {
    if (outer_res[i].aux == 0xFFFFFFFFu) continue;
    out_payload[k] = inner_res[i].aux;
    out_rowid[k] = outer_res[i].aux;
    k++;
  }
  return joined;
}
}
