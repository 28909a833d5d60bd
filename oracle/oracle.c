/*
 * oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Restates the reference's CPU operators (reference/db_operators) in plain C,
 * single-threaded, with these named fixes:
 *  F1 select.cpp:69-72 writes every element at out[counts[block]+block_cnt],
 *     racing with the next block and writing one past the end: here only
 *     selected elements are written.
 *  F2 select.cpp:16 / hash_join.cpp:18 / aggregate.cpp:17 NUM_BLOCKS =
 *     BUFFER_SIZE/8000 truncates and skips the tail rows: here the last
 *     partial block is processed.
 *  F3 sort.cpp:30-40 sorts keys only and is not stable: here (key, row id)
 *     pairs are sorted stably.
 *  F4 sort_merge_join.cpp:81-101 shares one cursor across threads, leaves
 *     per-block gaps, clamps block_end wrongly (:87) and emits at most one
 *     match per outer row: here one cursor, no gaps, every match emitted.
 *  F5 aggregate.cpp:59 sums int32 into int32 (overflow) and outputs in hash
 *     order: here int64 SUM/COUNT/MIN/MAX, groups ordered by key.
 *  F6 hash_join.cpp:131-135 builds a flat_hash_set, so duplicate build keys
 *     collapse to one: here every build row is kept (identical when build
 *     keys are unique, as in the reference's own inputs).
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#define BLOCK 8000u

static inline int64_t key_val(uint32_t k, int is_signed) {
  return is_signed ? (int64_t)(int32_t)k : (int64_t)k;
}

/* ---------------------------------------------------------------- select */
uint64_t oracle_select(const uint32_t *in, uint64_t n, int is_signed, int64_t lo, int64_t hi,
                       int invert, const uint32_t *in_ptr, uint64_t ptr_base, uint32_t *out_key,
                       uint32_t *out_ptr) {
  uint64_t nblocks = (n + BLOCK - 1) / BLOCK; /* F2 */
  uint64_t *counts = (uint64_t *)calloc(nblocks + 1, sizeof(uint64_t));
  /* count pass (select.cpp:39-58) */
  for (uint64_t b = 0; b < nblocks; b++) {
    uint64_t end = (b + 1) * BLOCK < n ? (b + 1) * BLOCK : n, c = 0;
    for (uint64_t i = b * BLOCK; i < end; i++) {
      int64_t v = key_val(in[i], is_signed);
      c += ((v >= lo && v <= hi) != (invert != 0));
    }
    counts[b + 1] = c;
  }
  /* serial prefix (select.cpp:86-89) */
  for (uint64_t b = 0; b < nblocks; b++) counts[b + 1] += counts[b];
  /* scatter pass (select.cpp:61-75), F1 */
  for (uint64_t b = 0; b < nblocks; b++) {
    uint64_t end = (b + 1) * BLOCK < n ? (b + 1) * BLOCK : n, c = counts[b];
    for (uint64_t i = b * BLOCK; i < end; i++) {
      int64_t v = key_val(in[i], is_signed);
      if ((v >= lo && v <= hi) != (invert != 0)) {
        if (out_key) out_key[c] = in[i];
        if (out_ptr) out_ptr[c] = in_ptr ? in_ptr[i] : (uint32_t)(ptr_base + i);
        c++;
      }
    }
  }
  uint64_t total = counts[nblocks];
  free(counts);
  return total;
}

/* ------------------------------------------------------------ stable sort */
typedef struct {
  uint32_t key;
  uint32_t idx;
} kv_t;

static int kv_less(const kv_t *a, const kv_t *b, int is_signed) {
  return key_val(a->key, is_signed) < key_val(b->key, is_signed);
}

/* Bottom-up merge sort: stable (F3). */
static void merge_sort_kv(kv_t *a, uint64_t n, int is_signed) {
  kv_t *tmp = (kv_t *)malloc((n ? n : 1) * sizeof(kv_t));
  kv_t *src = a, *dst = tmp;
  for (uint64_t w = 1; w < n; w *= 2) {
    for (uint64_t lo = 0; lo < n; lo += 2 * w) {
      uint64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
      uint64_t i = lo, j = mid, k = lo;
      while (i < mid && j < hi) dst[k++] = kv_less(&src[j], &src[i], is_signed) ? src[j++] : src[i++];
      while (i < mid) dst[k++] = src[i++];
      while (j < hi) dst[k++] = src[j++];
    }
    kv_t *t = src;
    src = dst;
    dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(kv_t));
  free(tmp);
}

void oracle_sort_pairs(const uint32_t *key, const uint32_t *ptr, uint64_t n, int is_signed,
                       uint32_t *out_key, uint32_t *out_ptr) {
  kv_t *a = (kv_t *)malloc((n ? n : 1) * sizeof(kv_t));
  for (uint64_t i = 0; i < n; i++) {
    a[i].key = key[i];
    a[i].idx = (uint32_t)i;
  }
  merge_sort_kv(a, n, is_signed);
  for (uint64_t i = 0; i < n; i++) {
    out_key[i] = a[i].key;
    out_ptr[i] = ptr ? ptr[a[i].idx] : a[i].idx;
  }
  free(a);
}

/* ------------------------------------------------------------ merge join */
uint64_t oracle_smj_merge(const uint32_t *ikey, const uint32_t *iptr, uint64_t ni,
                          const uint32_t *okey, const uint32_t *optr, uint64_t no, int is_signed,
                          uint32_t *out_outer, uint32_t *out_inner, uint64_t cap) {
  /* One cursor over the inner relation (F4): for each outer row advance past
   * smaller inner keys (sort_merge.c:61-72), then emit every equal inner row. */
  uint64_t out = 0, i = 0;
  for (uint64_t o = 0; o < no; o++) {
    int64_t ok = key_val(okey[o], is_signed);
    while (i < ni && key_val(ikey[i], is_signed) < ok) i++;
    for (uint64_t j = i; j < ni && key_val(ikey[j], is_signed) == ok; j++) {
      if (out < cap) {
        out_outer[out] = optr[o];
        out_inner[out] = iptr[j];
      }
      out++;
    }
  }
  return out;
}

/* ------------------------------------------------------------- hash join */
/* Fibonacci hash of hash_join.cpp:20-25. */
static inline uint32_t fib_hash(uint32_t input) {
  uint64_t x = (uint64_t)input * 11400714785074694791ull;
  return (uint32_t)__builtin_bswap64(x);
}

uint64_t oracle_hash_join(const uint32_t *bkey, const uint32_t *bpay, uint64_t nb,
                          const uint32_t *pkey, const uint32_t *prow, uint64_t np, uint32_t part_n,
                          uint32_t *out_payload, uint32_t *out_rowid, uint64_t cap) {
  /* partition() (hash_join.cpp:57-119): histogram, prefix, stable scatter. */
  uint64_t *bstart = (uint64_t *)calloc(part_n + 1, sizeof(uint64_t));
  uint64_t *pstart = (uint64_t *)calloc(part_n + 1, sizeof(uint64_t));
  uint32_t *bidx = (uint32_t *)malloc((nb ? nb : 1) * sizeof(uint32_t));
  uint32_t *pidx = (uint32_t *)malloc((np ? np : 1) * sizeof(uint32_t));
  for (uint64_t i = 0; i < nb; i++) bstart[fib_hash(bkey[i]) % part_n + 1]++;
  for (uint64_t i = 0; i < np; i++) pstart[fib_hash(pkey[i]) % part_n + 1]++;
  for (uint32_t p = 0; p < part_n; p++) {
    bstart[p + 1] += bstart[p];
    pstart[p + 1] += pstart[p];
  }
  uint64_t *bcur = (uint64_t *)malloc(part_n * sizeof(uint64_t));
  uint64_t *pcur = (uint64_t *)malloc(part_n * sizeof(uint64_t));
  memcpy(bcur, bstart, part_n * sizeof(uint64_t));
  memcpy(pcur, pstart, part_n * sizeof(uint64_t));
  for (uint64_t i = 0; i < nb; i++) bidx[bcur[fib_hash(bkey[i]) % part_n]++] = (uint32_t)i;
  for (uint64_t i = 0; i < np; i++) pidx[pcur[fib_hash(pkey[i]) % part_n]++] = (uint32_t)i;

  /* join_partitions() (hash_join.cpp:121-157): per partition, an
   * open-addressing table of the build rows, then the probe loop.  F6. */
  uint64_t out = 0;
  uint64_t maxb = 0;
  for (uint32_t p = 0; p < part_n; p++)
    if (bstart[p + 1] - bstart[p] > maxb) maxb = bstart[p + 1] - bstart[p];
  uint64_t cap_slots = 16;
  while (cap_slots < 2 * maxb + 1) cap_slots *= 2;
  int64_t *slot = (int64_t *)malloc(cap_slots * sizeof(int64_t));
  for (uint32_t p = 0; p < part_n; p++) {
    for (uint64_t s = 0; s < cap_slots; s++) slot[s] = -1;
    for (uint64_t b = bstart[p]; b < bstart[p + 1]; b++) {
      uint32_t row = bidx[b];
      uint64_t h = ((uint64_t)bkey[row] * 0x9E3779B97F4A7C15ull) & (cap_slots - 1);
      while (slot[h] >= 0) h = (h + 1) & (cap_slots - 1);
      slot[h] = row;
    }
    for (uint64_t q = pstart[p]; q < pstart[p + 1]; q++) {
      uint32_t prow_i = pidx[q];
      uint32_t k = pkey[prow_i];
      uint64_t h = ((uint64_t)k * 0x9E3779B97F4A7C15ull) & (cap_slots - 1);
      while (slot[h] >= 0) {
        if (bkey[slot[h]] == k) {
          if (out < cap) {
            out_payload[out] = bpay[slot[h]];
            out_rowid[out] = prow ? prow[prow_i] : prow_i;
          }
          out++;
        }
        h = (h + 1) & (cap_slots - 1);
      }
    }
  }
  free(slot);
  free(bstart);
  free(pstart);
  free(bidx);
  free(pidx);
  free(bcur);
  free(pcur);
  return out;
}

/* -------------------------------------------------------- hash partition */
static inline uint32_t hash0(uint32_t key) { /* pimdal/hash/hash_func.h:5-14 */
  key += 272333u;
  key += ~(key << 5);
  key ^= (key >> 18);
  key += (key << 11);
  key ^= (key >> 17);
  return key;
}

void oracle_part_hash0(const uint32_t *key, const uint32_t *ptr, uint64_t n, uint32_t shift,
                       uint32_t part_n, uint32_t *out_key, uint32_t *out_ptr, uint64_t *part_sizes) {
  uint32_t bits = 0;
  while ((1u << bits) < part_n) bits++;
  uint32_t sh = shift - bits;
  memset(part_sizes, 0, (part_n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n; i++) part_sizes[((hash0(key[i]) >> sh) & (part_n - 1)) + 1]++;
  for (uint32_t p = 0; p < part_n; p++) part_sizes[p + 1] += part_sizes[p];
  uint64_t *cur = (uint64_t *)malloc(part_n * sizeof(uint64_t));
  memcpy(cur, part_sizes, part_n * sizeof(uint64_t));
  for (uint64_t i = 0; i < n; i++) {
    uint64_t d = cur[(hash0(key[i]) >> sh) & (part_n - 1)]++;
    out_key[d] = key[i];
    out_ptr[d] = ptr ? ptr[i] : (uint32_t)i;
  }
  free(cur);
}

/* ---------------------------------------------------------- bloom filter */
/* The four filter hashes, hash1..hash4 of pimdal/hash/hash_func.h:16-58
 * (hash_func[] at :60), restated: an add of a constant, then shift-add /
 * shift-xor mixing steps with the constants and shifts of each function. */
static uint32_t bloom_hash(int f, uint32_t k) {
  static const uint32_t add[4] = {593627u, 274277u, 855467u, 176521u};
  static const uint8_t sh[4][4] = {{22, 26, 10, 28}, {13, 20, 3, 9}, {4, 21, 5, 16}, {10, 25, 5, 24}};
  k += add[f];
  k += ~(k << sh[f][0]);
  k ^= (k >> sh[f][1]);
  k += (k << sh[f][2]);
  k ^= (k >> sh[f][3]);
  return k;
}

uint32_t oracle_hash(int which, uint32_t key) { return which == 0 ? hash0(key) : bloom_hash(which - 1, key); }

/* filter_kernel (pimdal/join/hash_join.c:116-149) with insert_bloom_filter
 * (pimdal/hash/hash_steps.c:143-152): per partition, a zeroed filter of
 * ORACLE_FILTER_BITS bits with bit hashK(key) % ORACLE_FILTER_BITS set for
 * K = 1..4.  Bit b lives in byte b / 8 at bit b % 8. */
void oracle_bloom_build(const uint32_t *key, const uint64_t *part_sizes, uint32_t part_n,
                        uint8_t *filters) {
  for (uint32_t p = 0; p < part_n; p++) {
    uint8_t *f = filters + (uint64_t)p * ORACLE_FILTER_BYTES;
    memset(f, 0, ORACLE_FILTER_BYTES);
    for (uint64_t i = part_sizes[p]; i < part_sizes[p + 1]; i++)
      for (int h = 0; h < 4; h++) {
        uint32_t bit = bloom_hash(h, key[i]) % ORACLE_FILTER_BITS;
        f[bit / 8] |= (uint8_t)(1u << (bit % 8));
      }
  }
}

/* match_kernel (pimdal/join/hash_join.c:236-341) with probe_bloom_filter
 * (hash_steps.c:163-185): the rows of each partition whose key has all four
 * bits set in the partition's filter, in input order; match_sizes[0] = 0 and
 * match_sizes[p + 1] = kept rows of partition p.  Rows of [0, n) outside
 * every partition are not kept (the reference reads past part_sizes there,
 * hash_join.c:268-273).  Writes at most cap rows; returns the total. */
uint64_t oracle_bloom_match(const uint8_t *filters, const uint32_t *key, const uint32_t *ptr,
                            uint64_t n, const uint64_t *part_sizes, uint32_t part_n,
                            uint32_t *out_key, uint32_t *out_ptr, uint64_t cap,
                            uint64_t *match_sizes) {
  uint64_t c = 0;
  match_sizes[0] = 0;
  for (uint32_t p = 0; p < part_n; p++) {
    const uint8_t *f = filters + (uint64_t)p * ORACLE_FILTER_BYTES;
    uint64_t hits = 0;
    uint64_t end = part_sizes[p + 1] < n ? part_sizes[p + 1] : n;
    for (uint64_t i = part_sizes[p]; i < end; i++) {
      int hit = 1;
      for (int h = 0; h < 4 && hit; h++) {
        uint32_t bit = bloom_hash(h, key[i]) % ORACLE_FILTER_BITS;
        hit = (f[bit / 8] >> (bit % 8)) & 1;
      }
      if (!hit) continue;
      if (c < cap) {
        out_key[c] = key[i];
        if (out_ptr) out_ptr[c] = ptr ? ptr[i] : (uint32_t)i;
      }
      c++;
      hits++;
    }
    match_sizes[p + 1] = hits;
  }
  return c;
}

/* -------------------------------------------------------------- group by */
typedef struct {
  int32_t key;
  int64_t sum, count, min, max;
} grp_t;

static int grp_cmp(const void *a, const void *b) {
  int32_t x = ((const grp_t *)a)->key, y = ((const grp_t *)b)->key;
  return (x > y) - (x < y);
}

static uint64_t emit_groups(grp_t *g, uint64_t ng, int32_t *out_key, int64_t *out_sum,
                            int64_t *out_count, int64_t *out_min, int64_t *out_max) {
  qsort(g, ng, sizeof(grp_t), grp_cmp);
  for (uint64_t i = 0; i < ng; i++) {
    out_key[i] = g[i].key;
    out_sum[i] = g[i].sum;
    out_count[i] = g[i].count;
    out_min[i] = g[i].min;
    out_max[i] = g[i].max;
  }
  return ng;
}

static inline void grp_add(grp_t *g, int64_t v) {
  g->sum = (int64_t)((uint64_t)g->sum + (uint64_t)v); /* exact mod 2^64, F5 */
  g->count++;
  if (v < g->min) g->min = v;
  if (v > g->max) g->max = v;
}

static int64_t *grp_table_new(uint64_t cap) {
  int64_t *slot = (int64_t *)malloc(cap * sizeof(int64_t));
  for (uint64_t s = 0; s < cap; s++) slot[s] = -1;
  return slot;
}

static inline uint64_t grp_home(int32_t key, uint64_t cap) {
  return ((uint64_t)(uint32_t)key * 0x9E3779B97F4A7C15ull) >> 20 & (cap - 1);
}

uint64_t oracle_group_by(const int32_t *key, const int64_t *val, uint64_t n, int32_t *out_key,
                         int64_t *out_sum, int64_t *out_count, int64_t *out_min, int64_t *out_max) {
  /* hash_table_aggregate (aggregate.cpp:40-83): find-or-insert per row into a
   * table that doubles when half full, as absl::flat_hash_map grows. */
  uint64_t cap = 16, gcap = 8;
  int64_t *slot = grp_table_new(cap);
  grp_t *g = (grp_t *)malloc(gcap * sizeof(grp_t));
  uint64_t ng = 0;
  for (uint64_t i = 0; i < n; i++) {
    int64_t v = val ? val[i] : 1;
    uint64_t h = grp_home(key[i], cap);
    while (slot[h] >= 0 && g[slot[h]].key != key[i]) h = (h + 1) & (cap - 1);
    if (slot[h] < 0) {
      if (2 * (ng + 1) > cap) { /* grow, rehash every group, then find the slot again */
        free(slot);
        cap *= 2;
        slot = grp_table_new(cap);
        for (uint64_t q = 0; q < ng; q++) {
          uint64_t t = grp_home(g[q].key, cap);
          while (slot[t] >= 0) t = (t + 1) & (cap - 1);
          slot[t] = (int64_t)q;
        }
        h = grp_home(key[i], cap);
        while (slot[h] >= 0) h = (h + 1) & (cap - 1);
      }
      if (ng == gcap) {
        gcap *= 2;
        g = (grp_t *)realloc(g, gcap * sizeof(grp_t));
      }
      slot[h] = (int64_t)ng;
      g[ng].key = key[i];
      g[ng].sum = 0;
      g[ng].count = 0;
      g[ng].min = INT64_MAX;
      g[ng].max = INT64_MIN;
      ng++;
    }
    grp_add(&g[slot[h]], v);
  }
  uint64_t r = emit_groups(g, ng, out_key, out_sum, out_count, out_min, out_max);
  free(slot);
  free(g);
  return r;
}

uint64_t oracle_sort_group_by(const int32_t *key, const int64_t *val, uint64_t n, int32_t *out_key,
                              int64_t *out_sum, int64_t *out_count, int64_t *out_min,
                              int64_t *out_max) {
  kv_t *a = (kv_t *)malloc((n ? n : 1) * sizeof(kv_t));
  for (uint64_t i = 0; i < n; i++) {
    a[i].key = (uint32_t)key[i];
    a[i].idx = (uint32_t)i;
  }
  merge_sort_kv(a, n, 1);
  /* aggregate() (aggregate.c:31-44): new group when the key changes. */
  grp_t *g = (grp_t *)malloc((n ? n : 1) * sizeof(grp_t));
  uint64_t ng = 0;
  for (uint64_t i = 0; i < n; i++) {
    int64_t v = val ? val[a[i].idx] : 1;
    if (i == 0 || a[i].key != a[i - 1].key) {
      g[ng].key = (int32_t)a[i].key;
      g[ng].sum = 0;
      g[ng].count = 0;
      g[ng].min = INT64_MAX;
      g[ng].max = INT64_MIN;
      ng++;
    }
    grp_add(&g[ng - 1], v);
  }
  uint64_t r = emit_groups(g, ng, out_key, out_sum, out_count, out_min, out_max);
  free(a);
  free(g);
  return r;
}
