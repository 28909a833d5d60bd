/* Harness around the reference's hash functions, pimdal/hash/hash_func.h
 * (compiled from where it lies, nothing copied).  Test infrastructure only.
 *
 * The Bloom-filter loops themselves live in pimdal/hash/hash_steps.c, which
 * needs the DPU runtime (mram, barriers, mutexes) and cannot be compiled
 * here; the two loops below restate insert_bloom_filter (hash_steps.c:143-152)
 * and probe_bloom_filter (:163-185) around the reference's own hash_func[]
 * table, as filter_kernel (pimdal/join/hash_join.c:116-149) and match_kernel
 * (:236-341) apply them partition by partition.  What this pins is the hash
 * functions, which decide every filter bit. */
#include <stdint.h>
#include <string.h>

#include "hash_func.h"

#define REF_FILTER_SIZE 16384u /* hash_steps.c:15 */
#define REF_FILTER_BYTES (REF_FILTER_SIZE / 8u)

/* which = 0: hash0; which = 1..4: hash_func[which - 1] (hash1..hash4). */
void pimdal_ref_hash(int which, const uint32_t *key, uint64_t n, uint32_t *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = which == 0 ? hash0(key[i]) : hash_func[which - 1](key[i]);
}

void pimdal_ref_bloom_build(const uint32_t *key, const uint64_t *part_sizes, uint32_t part_n,
                            uint8_t *filters) {
  for (uint32_t p = 0; p < part_n; p++) {
    uint8_t *out = filters + (uint64_t)p * REF_FILTER_BYTES;
    memset(out, 0, REF_FILTER_BYTES);
    for (uint32_t filter = 0; filter < 4; filter++)
      for (uint64_t i = part_sizes[p]; i < part_sizes[p + 1]; i++) {
        uint32_t bit = hash_func[filter](key[i]) % REF_FILTER_SIZE;
        out[bit / 8] = out[bit / 8] | (uint8_t)(1u << (bit % 8));
      }
  }
}

uint64_t pimdal_ref_bloom_match(const uint8_t *filters, const uint32_t *key, const uint32_t *ptr,
                                const uint64_t *part_sizes, uint32_t part_n, uint32_t *out_key,
                                uint32_t *out_ptr, uint64_t *match_sizes) {
  uint64_t selected = 0;
  match_sizes[0] = 0;
  for (uint32_t p = 0; p < part_n; p++) {
    const uint8_t *f = filters + (uint64_t)p * REF_FILTER_BYTES;
    uint64_t hits = 0;
    for (uint64_t i = part_sizes[p]; i < part_sizes[p + 1]; i++) {
      uint32_t hit = 1;
      for (uint32_t filter = 0; filter < 4; filter++) {
        uint32_t bit = hash_func[filter](key[i]) % REF_FILTER_SIZE;
        if ((f[bit / 8] & ((uint8_t)1 << (bit % 8))) == 0) {
          hit = 0;
          break;
        }
      }
      if (hit) {
        out_key[selected] = key[i];
        out_ptr[selected] = ptr ? ptr[i] : (uint32_t)i;
        selected++;
        hits++;
      }
    }
    match_sizes[p + 1] = hits;
  }
  return selected;
}
