// Harness around the reference's CPU sort-merge join,
// reference/db_operators/sort_merge_join.cpp (compiled from where it lies).
// Test infrastructure only.
//
// sort_merge_join_kernel (sort_merge_join.cpp:48-103) sorts uint32 key
// columns and merges them block by block with one cursor shared by all
// OpenMP threads.  Run with one thread, an outer size that is a multiple of
// 8000 equal to BUFFER_SIZE, and every outer key present in the inner
// relation, it writes, for each outer key in ascending order, the matching
// inner key.  Inputs need one element of slack (the cursor is read before it
// is bounds-checked, :93).
#include <cstdint>

#define main pimdal_ref_smj_main
#include "sort_merge_join.cpp"
#undef main

extern "C" {

void pimdal_ref_set_threads(int t) { omp_set_num_threads(t); }
uint64_t pimdal_ref_smj_buffer_size(void) { return BUFFER_SIZE; }

void pimdal_ref_smj(const uint32_t *inner, uint64_t ni, const uint32_t *outer, uint64_t no,
                    uint32_t *inner_res, uint32_t *outer_res) {
  sort_merge_join_kernel(const_cast<uint32_t *>(inner), const_cast<uint32_t *>(outer), inner_res,
                         outer_res, ni, no);
}
}
