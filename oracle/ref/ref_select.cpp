// Harness around the reference's CPU selection, reference/db_operators/select.cpp
// (compiled from where it lies; nothing copied).  Test infrastructure only.
//
// select.cpp hard-codes its predicate (select.cpp:33-36, 10 <= v < 30).  The
// harness instantiates the reference's own sel_cnt_kernel / sel_out_kernel
// templates (select.cpp:38-75) for a one-field wrapper type whose predicate
// specialisation evaluates the closed interval [g_lo, g_hi] instead.
#include <cstdint>
#include <vector>

struct PdSelVal {
  int32_t v;
};
static int64_t g_lo = 0, g_hi = 0;

#define main pimdal_ref_select_main
#include "select.cpp"
#undef main

template <>
inline bool predicate<PdSelVal>(PdSelVal e) {
  return e.v >= g_lo && e.v <= g_hi;
}

extern "C" {

uint64_t pimdal_ref_select_num_blocks(void) { return NUM_BLOCKS; }

void pimdal_ref_set_threads(int t) { omp_set_num_threads(t); }

// Count pass only (sel_cnt_kernel, select.cpp:39-58): exact with any threads.
uint64_t pimdal_ref_sel_count(const int32_t *in, uint64_t n, int64_t lo, int64_t hi) {
  g_lo = lo;
  g_hi = hi;
  std::vector<uint64_t> counts(NUM_BLOCKS + 1, 0);
  const PdSelVal *b = reinterpret_cast<const PdSelVal *>(in);
  return sel_cnt_kernel(b, b + n, counts.data());
}

// The reference's select() body (select.cpp:77-100): count, serial prefix,
// scatter.  `out` needs count + 1 slots (sel_out_kernel writes every element,
// the last one past the end, select.cpp:69-72).
uint64_t pimdal_ref_select(const int32_t *in, uint64_t n, int64_t lo, int64_t hi, int32_t *out) {
  g_lo = lo;
  g_hi = hi;
  std::vector<uint64_t> counts(NUM_BLOCKS + 1, 0);
  const PdSelVal *b = reinterpret_cast<const PdSelVal *>(in);
  uint64_t selected = sel_cnt_kernel(b, b + n, counts.data());
  counts[0] = 0;
  for (uint64_t i = 0; i < NUM_BLOCKS; i++) counts[i + 1] += counts[i];
  sel_out_kernel(b, b + n, reinterpret_cast<PdSelVal *>(out), counts.data());
  return selected;
}
}
