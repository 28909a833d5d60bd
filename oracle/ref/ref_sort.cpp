// Harness around the reference's CPU sort, reference/db_operators/sort.cpp
// (compiled from where it lies).  Test infrastructure only.
//
// sort_kernel (sort.cpp:30-40) is std::copy + __gnu_parallel::sort of one
// key column.  Sorting (key, original index) pairs with it and mapping the
// index back to the row-id column gives the stable key/row-id sort.
#include <cstdint>
#include <vector>

struct PdPairU {
  uint32_t key, idx;
  bool operator<(const PdPairU &o) const { return key < o.key || (key == o.key && idx < o.idx); }
};
struct PdPairS {
  int32_t key;
  uint32_t idx;
  bool operator<(const PdPairS &o) const { return key < o.key || (key == o.key && idx < o.idx); }
};

#define main pimdal_ref_sort_main
#include "sort.cpp"
#undef main

extern "C" {

void pimdal_ref_set_threads(int t) { omp_set_num_threads(t); }

// The reference kernel as shipped: sort of a uint32 key column.
void pimdal_ref_sort_keys(const uint32_t *in, uint32_t *out, uint64_t n) {
  sort_kernel(const_cast<uint32_t *>(in), out, n);
}

// The reference kernel on pairs that the caller packed beforehand: each
// 64-bit word is a PdPairU (key in the low half, index in the high half, as
// the struct lies in memory), so the timed call is sort_kernel alone.
void pimdal_ref_sort_packed(const uint64_t *in, uint64_t *out, uint64_t n) {
  sort_kernel(reinterpret_cast<PdPairU *>(const_cast<uint64_t *>(in)),
              reinterpret_cast<PdPairU *>(out), n);
}

// Stable sort of (key, ptr) by key; ptr == NULL means row id = index.
void pimdal_ref_sort_pairs(const uint32_t *key, const uint32_t *ptr, uint64_t n, int is_signed,
                           uint32_t *out_key, uint32_t *out_ptr) {
  if (is_signed) {
    std::vector<PdPairS> in(n), out(n);
    for (uint64_t i = 0; i < n; i++) in[i] = {(int32_t)key[i], (uint32_t)i};
    sort_kernel(in.data(), out.data(), n);
    for (uint64_t i = 0; i < n; i++) {
      out_key[i] = (uint32_t)out[i].key;
      out_ptr[i] = ptr ? ptr[out[i].idx] : out[i].idx;
    }
  } else {
    std::vector<PdPairU> in(n), out(n);
    for (uint64_t i = 0; i < n; i++) in[i] = {key[i], (uint32_t)i};
    sort_kernel(in.data(), out.data(), n);
    for (uint64_t i = 0; i < n; i++) {
      out_key[i] = out[i].key;
      out_ptr[i] = ptr ? ptr[out[i].idx] : out[i].idx;
    }
  }
}
}
