// Device-resident descriptors of a batched run (pimdal_group_batch_*,
// pimdal_hash_join_batch_*): many independent operator instances executed by
// one persistent launch per phase, fed by a device work queue.  Built on the
// host once per plan (batch.cu), read by the kernels in groupby.cu and
// hashjoin.cu.
#pragma once

#include "common.cuh"

// One group-by instance (pimdal_aggr_arguments_t resolved to device memory).
struct pd_gb_inst {
  const uint32_t *key;
  const int64_t *val;  // NULL: every value is 1
  uint64_t n;
  uint32_t *out_key;
  int64_t *out_sum, *out_count, *out_min, *out_max;
  uint64_t out_cap;
  uint64_t *d_count;   // results[i].t_count
  uint64_t slot0;      // first slot of its table in the plan's global table
  uint32_t slots;      // table slots
  uint32_t mode;       // shared-table mode (warp tables, CTA table, direct)
  uint32_t wrep;       // warp-table replicas
  uint32_t flip;       // 0x80000000 for signed keys (ascending output order)
};

struct pd_gb_batch {
  const pd_gb_inst *inst;
  uint32_t count;
  const uint2 *items;       // (instance, first row) of each work item, instance-major
  uint32_t nitems;
  uint32_t rows_per_item;   // a multiple of 128
  unsigned long long *gtab; // all instances' 32-byte slots
  uint64_t total_slots;
  const uint64_t *slot0;    // count + 1 prefix of table slots
  uint32_t *counters;       // work-queue claim counters (2 words, self-resetting)
  unsigned long long *ngroups;  // occupied slots of all instances (device)
  uint32_t *inst_groups;    // groups per instance
  uint64_t *inst_start;     // first position of each instance in the ordered list
  uint32_t *ckey, *cslot, *skey, *sslot, *ikey, *islot;  // total_slots each
  void *sort_ws;
  uint32_t inst_bits;       // bits of an instance index
  uint32_t *d_error;
};

// One hash-join instance (pimdal_hash_join_arguments_t resolved to device
// memory); it is never partitioned.
struct pd_hj_inst {
  const uint32_t *bkey, *bpay;  // bpay NULL: payload = build row id
  uint64_t nb;
  const uint32_t *pkey, *prow;  // prow NULL: row id = probe index
  uint64_t np;
  uint32_t *out_pay, *out_row;
  uint64_t cap;
  uint64_t *d_count;            // results[i].t_count
  unsigned long long *table;    // 2^bits slots
  uint32_t *header;             // side count (word 0), duplicate flag (word 2)
  uint32_t bits;
  uint32_t pad;
  uint64_t tile0;               // first probe tile of this instance
};

struct pd_hj_batch {
  const pd_hj_inst *inst;
  uint32_t count;
  const uint64_t *tile0;        // count + 1 prefix of probe tiles
  uint64_t total_tiles;
  const uint2 *bitems;          // (instance, first build row) of each build item
  uint32_t nbitems;
  uint32_t build_rows_per_item;
  unsigned long long *tables;   // all instances' tables, contiguous
  uint64_t table_words;
  uint32_t *headers;            // 8 words per instance
  uint64_t *status;             // total_tiles look-back words
  uint32_t *epoch;              // device epoch of the look-back words
  uint32_t *counters;           // claim counters (2 words, self-resetting)
  uint32_t *d_error;
};

int pd_gb_batch_run(pimdal_ctx *ctx, const pd_gb_batch &b, cudaStream_t s);
int pd_hj_batch_run(pimdal_ctx *ctx, const pd_hj_batch &b, cudaStream_t s);
size_t pd_gb_batch_shared_bytes();
// Shared-table mode and replicas for an expected group count (same rule as
// the plain hash group-by).
void pd_gb_mode(uint64_t expected, uint32_t *mode, uint32_t *wrep);
// Probe tile rows of the hash join; log2 of the slots of its table for nb
// build rows at a load factor (same rule as pimdal_hash_join).
uint32_t pd_hj_tile_rows();
uint32_t pd_hj_table_bits(uint64_t nb, uint32_t load_pct);
