/*
 * oracle.h -- CPU oracle for the pimdal_b200 operators.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this library, and only as the checker
 * (or the timed CPU baseline); the product path never calls it.
 *
 * Plain-C restatement of the reference algorithms, each function citing the
 * reference lines it follows and the reference defect it fixes.  Pinned by
 * the tests against the reference's own CPU operators (reference/db_operators
 * compiled through the harnesses in oracle/ref/ into oracle/_ref/) and against the golden
 * fixtures in tests/golden/.
 */
#ifndef PIMDAL_ORACLE_H_
#define PIMDAL_ORACLE_H_

#include <stdint.h>

/* Selection: reference/db_operators/select.cpp:38-100 (count per 8000-row
 * block, serial prefix, scatter) + row ids as in
 * pimdal/main/select/dpu/kernel_select.c:31-36 (create_ptr).  Selected means
 * lo <= v <= hi (xor invert).  Returns the count. */
uint64_t oracle_select(const uint32_t *in, uint64_t n, int is_signed, int64_t lo, int64_t hi,
                       int invert, const uint32_t *in_ptr, uint64_t ptr_base, uint32_t *out_key,
                       uint32_t *out_ptr);

/* Stable ascending sort of (key, ptr) by key (sort.cpp:30-40 made stable and
 * paired).  in_ptr NULL = row id index. */
void oracle_sort_pairs(const uint32_t *key, const uint32_t *ptr, uint64_t n, int is_signed,
                       uint32_t *out_key, uint32_t *out_ptr);

/* Merge join of key-sorted relations (pimdal/join/sort_merge.c:54-83,
 * reference/db_operators/sort_merge_join.cpp:80-102) emitting every matching
 * (outer ptr, inner ptr) pair, outer-major.  Returns the match count; writes
 * at most cap pairs. */
uint64_t oracle_smj_merge(const uint32_t *ikey, const uint32_t *iptr, uint64_t ni,
                          const uint32_t *okey, const uint32_t *optr, uint64_t no, int is_signed,
                          uint32_t *out_outer, uint32_t *out_inner, uint64_t cap);

/* Hash join (reference/db_operators/hash_join.cpp:20-157): Fibonacci-hash
 * partitioning into part_n partitions, then per partition build a table of
 * the build rows and probe it.  Emits (build payload, probe row id) for every
 * match, partition by partition.  Returns the match count. */
uint64_t oracle_hash_join(const uint32_t *bkey, const uint32_t *bpay, uint64_t nb,
                          const uint32_t *pkey, const uint32_t *prow, uint64_t np, uint32_t part_n,
                          uint32_t *out_payload, uint32_t *out_rowid, uint64_t cap);

/* Radix partition by bits [shift - log2(part_n), shift) of hash0(key)
 * (pimdal/join/hash_join.c:154-235 with hash_steps.c:198-294, hash_func.h:5-14),
 * stable.  part_sizes[p] = start of partition p, part_sizes[part_n] = n. */
void oracle_part_hash0(const uint32_t *key, const uint32_t *ptr, uint64_t n, uint32_t shift,
                       uint32_t part_n, uint32_t *out_key, uint32_t *out_ptr, uint64_t *part_sizes);

/* Hash group-by (reference/db_operators/aggregate.cpp:40-83): int32 key,
 * int64 value; exact int64 SUM / COUNT / MIN / MAX; groups ascending by key.
 * val NULL = every value 1.  Returns the number of groups. */
uint64_t oracle_group_by(const int32_t *key, const int64_t *val, uint64_t n, int32_t *out_key,
                         int64_t *out_sum, int64_t *out_count, int64_t *out_min, int64_t *out_max);

/* Sort group-by (pimdal/aggregate/aggregate.c:31-44, 82-158): stable sort by
 * key, then run-length reduction of equal keys. */
uint64_t oracle_sort_group_by(const int32_t *key, const int64_t *val, uint64_t n, int32_t *out_key,
                              int64_t *out_sum, int64_t *out_count, int64_t *out_min,
                              int64_t *out_max);

/* Bloom-filter semi-join prefilter (pimdal/join/hash_join.c:116-149 and
 * :236-341, pimdal/hash/hash_steps.c:143-185): filters of ORACLE_FILTER_BITS
 * bits (hash_steps.c:15-16), one per partition of partitioned keys, and the
 * ordered compaction of the rows that hit their partition's filter.
 * oracle_hash(0, k) is hash0, oracle_hash(K, k) is hashK (K = 1..4). */
#define ORACLE_FILTER_BITS 16384u
#define ORACLE_FILTER_BYTES (ORACLE_FILTER_BITS / 8u)
uint32_t oracle_hash(int which, uint32_t key);
void oracle_bloom_build(const uint32_t *key, const uint64_t *part_sizes, uint32_t part_n,
                        uint8_t *filters);
uint64_t oracle_bloom_match(const uint8_t *filters, const uint32_t *key, const uint32_t *ptr,
                            uint64_t n, const uint64_t *part_sizes, uint32_t part_n,
                            uint32_t *out_key, uint32_t *out_ptr, uint64_t cap,
                            uint64_t *match_sizes);

#endif
