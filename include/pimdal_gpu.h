/*
 * pimdal_gpu.h -- C ABI of the B200 (sm_100a) implementation of PIMDAL's
 * data-parallel operator layer: selection, stable radix sort, sort-merge join,
 * radix-partitioned / L2-resident hash join, and hash / sort group-by.
 *
 * Every entry point mirrors one DPU library call of the reference.  The
 * argument structs keep the reference's field meaning; what changes is:
 *   - 32-bit MRAM addresses become 64-bit device pointers (columns resident
 *     in HBM, caller-owned);
 *   - function-pointer predicates / combiners become small descriptors;
 *   - every call takes a context (workspace + device error word) and a
 *     CUDA stream, and returns a status code instead of `return 0`;
 *   - counts are uint64 and are written to DEVICE memory (results structs),
 *     so calls never block the host.
 *
 * Threading: all work is stream-ordered.  A context may be used from one
 * stream at a time (its workspace and lookback status words are shared by
 * consecutive calls); use one context per concurrently-running stream.
 *
 * Device-side failures (a bounded spin that gave up, a hash table that ran
 * out of slots, an output buffer that was too small) never trap: kernels set
 * bits in the context's device error word; pimdal_ctx_sync_status() waits for
 * the stream and turns the word into a status code.
 */
#ifndef PIMDAL_GPU_H_
#define PIMDAL_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIMDAL_ABI_VERSION 1

/* ------------------------------------------------------------------------- */
/* Status codes (replace the reference's unconditional `return 0` and the     */
/* host-side DPU_ASSERT / dpu::DpuError).                                     */
/* ------------------------------------------------------------------------- */
typedef enum {
  PIMDAL_OK = 0,
  PIMDAL_ERR_ARG = 1,            /* bad argument (null pointer, size, enum)   */
  PIMDAL_ERR_OOM = 2,            /* device allocation failed                 */
  PIMDAL_ERR_WORKSPACE = 3,      /* caller-provided workspace too small      */
  PIMDAL_ERR_TABLE_FULL = 4,     /* hash table has no free slot              */
  PIMDAL_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait gave up       */
  PIMDAL_ERR_CUDA = 6,           /* a CUDA runtime call or launch failed     */
  PIMDAL_ERR_CAPACITY = 7,       /* output buffer smaller than the result    */
  PIMDAL_ERR_BUDGET = 8,         /* admission rejected by the HBM byte budget*/
  PIMDAL_ERR_NOT_SUPPORTED = 9
} pimdal_status_t;

typedef void *pimdal_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* The reference's pair type: key_ptr32 {uint32 key; uint32 ptr;}
 * (pimdal/main/select/shared/datatype.h:8-12, key_ptr_t alias at :35). */
typedef struct {
  uint32_t key;
  uint32_t ptr;
} pimdal_key_ptr32_t;

/* Column element types accepted at the boundary. */
typedef enum { PIMDAL_U32 = 0, PIMDAL_I32 = 1, PIMDAL_I64 = 2, PIMDAL_U8 = 3 } pimdal_dtype_t;

/* Input/output layout: structure-of-arrays columns (key column + row-id
 * column) or the reference's array of key_ptr32 pairs. */
typedef enum { PIMDAL_LAYOUT_COLUMNS = 0, PIMDAL_LAYOUT_PAIRS = 1 } pimdal_layout_t;

/* ------------------------------------------------------------------------- */
/* Context                                                                    */
/* ------------------------------------------------------------------------- */
typedef struct pimdal_ctx pimdal_ctx_t;

/* Creates a context on `device`.  Allocates only the device error word and
 * the lookback status words (a few MB), zeroed. */
int pimdal_ctx_create(pimdal_ctx_t **ctx, int device);
int pimdal_ctx_destroy(pimdal_ctx_t *ctx);

/* Hands the context a caller-owned scratch buffer (device memory, 256-byte
 * aligned).  Without one, the context grows its own buffer with cudaMalloc
 * when a call needs more (never during stream capture).  Each operator's
 * *_workspace_size() query gives the bytes it needs. */
int pimdal_ctx_set_workspace(pimdal_ctx_t *ctx, void *ptr, size_t bytes);

/* Waits for `stream`, reads and clears the device error word, and returns the
 * first error code it holds (PIMDAL_OK when none). */
int pimdal_ctx_sync_status(pimdal_ctx_t *ctx, pimdal_stream_t stream);

/* Number of kernels this context launched so far (for accounting). */
uint64_t pimdal_ctx_launch_count(const pimdal_ctx_t *ctx);

/* Per-kernel device timing.  While enabled, every launch of the library's
 * kernels is bracketed by CUDA events recorded on the launching stream;
 * pimdal_ctx_kernel_time() waits for them and returns, for one kernel id,
 * the number of launches and their summed duration since the last read. */
typedef enum {
  PIMDAL_KERNEL_SELECT = 0,
  PIMDAL_KERNEL_GEN = 1,
  PIMDAL_KERNEL_SORT_HIST = 2,   /* radix sort: all-digit histogram pass   */
  PIMDAL_KERNEL_SORT_PASS = 3,   /* radix sort: one onesweep digit pass    */
  PIMDAL_KERNEL_SMJ_MERGE = 4,   /* merge-path join                        */
  PIMDAL_KERNEL_PARTITION = 5,   /* hash radix partition                   */
  PIMDAL_KERNEL_HJ_BUILD = 6,
  PIMDAL_KERNEL_HJ_PROBE = 7,
  PIMDAL_KERNEL_GROUP = 8,       /* hash group-by                          */
  PIMDAL_KERNEL_SEGREDUCE = 9,   /* sort group-by segmented reduction      */
  PIMDAL_KERNEL_OTHER = 10,
  PIMDAL_KERNEL_FILTER = 11,     /* Bloom filter build                     */
  PIMDAL_KERNEL_MATCH = 12,      /* Bloom filter probe + ordered compaction*/
  PIMDAL_KERNEL_FUSED = 13,      /* fused select -> join -> group-by pass  */
  PIMDAL_KERNEL_SCAN_AGG = 14,   /* fused select -> arithmetic -> group-by */
  PIMDAL_KERNEL_COUNT = 15
} pimdal_kernel_id_t;
int pimdal_ctx_set_profiling(pimdal_ctx_t *ctx, int enable);
int pimdal_ctx_kernel_time(pimdal_ctx_t *ctx, int kernel_id, uint64_t *launches,
                           double *total_ms);

const char *pimdal_status_string(int status);
int pimdal_abi_version(void);

/* ------------------------------------------------------------------------- */
/* Seeded counter-based column generator (replaces the thread-count-dependent */
/* std::default_random_engine generators of reference/db_operators/          */
/* shared.cpp:10-60).  Value i depends only on (seed, stream_id, i), so CPU   */
/* and GPU produce identical columns for any launch shape.                    */
/* ------------------------------------------------------------------------- */
typedef enum {
  PIMDAL_GEN_UNIFORM = 0,      /* lo + floor(u * (hi-lo+1)), inclusive range    */
  PIMDAL_GEN_PERM = 1,         /* perm_domain(row)  (distinct values)           */
  PIMDAL_GEN_PERM_UNIFORM = 2, /* perm_domain(uniform index in [lo, hi])        */
  PIMDAL_GEN_PERM_ZIPF = 3,    /* perm_domain(zipf index over cdf[0..cdf_n))    */
  PIMDAL_GEN_PROBE = 4         /* join probe: Bernoulli(match_permille/1000)
                                  picks perm_domain(idx) with idx < lo (a build
                                  key) or perm_domain(lo + idx) (a non-key);
                                  idx uniform over [0, lo) or zipf via cdf     */
} pimdal_gen_kind_t;

typedef struct {
  int32_t kind;          /* pimdal_gen_kind_t */
  int32_t out_dtype;     /* PIMDAL_U32 / PIMDAL_I32 (4 bytes) or PIMDAL_I64 */
  uint64_t seed;
  uint64_t stream_id;    /* independent sub-stream per column */
  int64_t lo, hi;        /* uniform range (inclusive) / PROBE: build count */
  uint64_t perm_domain;  /* permutation domain size (0 = 2^32) */
  const double *cdf;     /* device pointer: zipf CDF (ascending), or NULL */
  uint64_t cdf_n;
  uint32_t match_permille; /* PROBE only */
  uint32_t pad;
} pimdal_gen_spec_t;

/* dst[i] = value(row_offset + i) for i < n. */
int pimdal_gen_column(pimdal_ctx_t *ctx, const pimdal_gen_spec_t *spec, void *dst,
                      uint64_t n, uint64_t row_offset, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Selection.  Replaces sel_kernel(sel_arguments_t*, sel_results_t*)          */
/* (pimdal/select/sel.h:7-21, sel.c:81-150) together with the create_ptr /   */
/* out_val glue of pimdal/main/select/dpu/kernel_select.c:31-42, and the CPU  */
/* sel_cnt_kernel / sel_out_kernel of reference/db_operators/select.cpp:39-75.*/
/* Output is stable: selected rows appear in ascending input order.           */
/* ------------------------------------------------------------------------- */
typedef enum {
  PIMDAL_PRED_LT = 0,      /* v <  lo            */
  PIMDAL_PRED_LE = 1,      /* v <= lo            */
  PIMDAL_PRED_GT = 2,      /* v >  lo            */
  PIMDAL_PRED_GE = 3,      /* v >= lo            */
  PIMDAL_PRED_EQ = 4,      /* v == lo            */
  PIMDAL_PRED_NE = 5,      /* v != lo            */
  PIMDAL_PRED_BETWEEN = 6, /* lo <= v && v <= hi */
  PIMDAL_PRED_RANGE = 7    /* lo <= v && v <  hi */
} pimdal_pred_op_t;

/* Replaces `bool (*pred)(const key_ptr_t)` (sel.h:11). */
typedef struct {
  int32_t op;    /* pimdal_pred_op_t */
  int32_t pad;
  int64_t lo;
  int64_t hi;
} pimdal_pred_t;

typedef struct {
  uint64_t size;          /* sel_arguments_t.size: number of elements          */
  const void *in;         /* sel_arguments_t.in: key column (key_dtype) or pairs */
  const uint32_t *in_ptr; /* row-id column; NULL = ptr_base + index (create_ptr) */
  uint64_t ptr_base;
  void *out;              /* sel_arguments_t.out: selected keys (or pairs)      */
  uint32_t *out_ptr;      /* selected row ids (COLUMNS layout); may be NULL     */
  pimdal_pred_t pred;     /* sel_arguments_t.pred                               */
  int32_t key_dtype;      /* PIMDAL_I32 or PIMDAL_U32                            */
  int32_t layout;         /* pimdal_layout_t                                    */
} pimdal_sel_arguments_t;

typedef struct {
  uint64_t t_count; /* sel_results_t.t_count (sel.h:14-16) */
} pimdal_sel_results_t;

int pimdal_sel_workspace_size(const pimdal_sel_arguments_t *args, size_t *bytes);
/* `d_result` is device memory. */
int pimdal_sel_kernel(pimdal_ctx_t *ctx, const pimdal_sel_arguments_t *args,
                      pimdal_sel_results_t *d_result, pimdal_stream_t stream);

/* Selection that allocates nothing -- no counterpart in the reference.  For
 * callers that cannot call cudaMalloc: a host whose memory manager owns every
 * device allocation (a database buffer pool, a framework's caching
 * allocator), or a latency-critical path where an allocation could block on
 * a device-wide synchronisation.  No context is needed: the caller passes
 * only its own input, output and result buffers.  Same arguments and results
 * as pimdal_sel_kernel, on the current device.  Scratch is a fixed 32 KiB
 * device array inside the library (held by every GPU that loads the library
 * until the process exits), so at most 2^29 rows per call with 16-byte-
 * aligned input and row ids (2^24 otherwise); larger calls return
 * PIMDAL_ERR_WORKSPACE before anything is launched.  The first call on a
 * device looks up and clears that array; make that first call before any
 * stream capture.  Every call shares the array: calls that overlap on the
 * GPU race and must not be issued.  A device-side failure sets
 * d_result->t_count to UINT64_MAX. */
int pimdal_sel_kernel_noalloc(const pimdal_sel_arguments_t *args, pimdal_sel_results_t *d_result,
                              pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Sort.  Replaces sort_part_kernel + sort_kernel (pimdal/sort/sort.h:7-25,  */
/* sort_keyval.c:114-179) and the CPU sort_kernel of                          */
/* reference/db_operators/sort.cpp:30-40.  Stable ascending sort of          */
/* (key, row id) pairs by key: equal keys keep their input order, so the     */
/* result is fully determined.  nr_elements < 2^30.                          */
/* ------------------------------------------------------------------------- */
typedef struct {
  uint64_t nr_elements;   /* sort_arguments_t.nr_elements                      */
  const void *in;         /* sort_arguments_t.in: key column or pairs          */
  const uint32_t *in_ptr; /* row ids (COLUMNS); NULL = ptr_base + index         */
  uint64_t ptr_base;
  void *out;              /* sort_arguments_t.out: sorted keys or pairs (!= in) */
  uint32_t *out_ptr;      /* sorted row ids (COLUMNS); NULL = keys only         */
  int32_t key_dtype;      /* PIMDAL_U32 or PIMDAL_I32 (signed order)            */
  int32_t layout;         /* pimdal_layout_t                                    */
  uint32_t begin_bit;     /* sort on key bits [begin_bit, end_bit)              */
  uint32_t end_bit;       /* 0 = 32                                             */
} pimdal_sort_arguments_t;

int pimdal_sort_workspace_size(const pimdal_sort_arguments_t *args, size_t *bytes);
int pimdal_sort_kernel(pimdal_ctx_t *ctx, const pimdal_sort_arguments_t *args,
                       pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Sort-merge join.  pimdal_smj_merge replaces merge_kernel of               */
/* pimdal/join/sort_merge.h:6-23 (sort_merge.c:86-152): both relations are   */
/* sorted by key; for every pair of rows with equal keys it emits            */
/* (outer ptr, inner ptr) (sort_merge.c:76-77).  Every match is emitted,     */
/* duplicates on both sides included, outer-major then inner order.  With a  */
/* unique inner key (the reference's inputs) this equals the reference.      */
/* ------------------------------------------------------------------------- */
typedef struct {
  const void *inner;           /* merge_arguments_t.inner: sorted inner keys   */
  const uint32_t *inner_ptr;   /* inner row ids / payloads                     */
  uint64_t size_inner;         /* merge_arguments_t.size_inner                 */
  const void *outer;           /* merge_arguments_t.outer: sorted outer keys   */
  const uint32_t *outer_ptr;
  uint64_t size_outer;         /* merge_arguments_t.size_outer                 */
  uint32_t *out_outer;         /* merge_arguments_t.out, column of outer ptrs  */
  uint32_t *out_inner;         /* ... and of inner ptrs                        */
  uint64_t out_capacity;       /* rows available in out_outer / out_inner      */
  int32_t key_dtype;           /* PIMDAL_I32 or PIMDAL_U32                      */
  int32_t pad;
} pimdal_smj_merge_arguments_t;

typedef struct {
  uint64_t t_count; /* merge_results_t.t_count / .out_n: total matches (even
                       when larger than out_capacity, which then raises
                       PIMDAL_ERR_CAPACITY at pimdal_ctx_sync_status) */
} pimdal_merge_results_t;

int pimdal_smj_merge_workspace_size(const pimdal_smj_merge_arguments_t *args, size_t *bytes);
int pimdal_smj_merge(pimdal_ctx_t *ctx, const pimdal_smj_merge_arguments_t *args,
                     pimdal_merge_results_t *d_result, pimdal_stream_t stream);

/* Whole sort-merge join of two unsorted relations (the pipeline of
 * pimdal/main/join/sort and reference/db_operators/sort_merge_join.cpp:48-156):
 * stable sort of both sides by key, then the merge.  Output: for every match,
 * the inner payload and the outer payload (payload NULL = row id). */
typedef struct {
  const void *inner_key;
  const uint32_t *inner_payload;
  uint64_t size_inner;
  const void *outer_key;
  const uint32_t *outer_payload;
  uint64_t size_outer;
  uint32_t *out_inner_payload;
  uint32_t *out_outer_payload;
  uint64_t out_capacity;
  int32_t key_dtype;
  int32_t pad;
} pimdal_smj_arguments_t;

int pimdal_sort_merge_join_workspace_size(const pimdal_smj_arguments_t *args, size_t *bytes);
int pimdal_sort_merge_join(pimdal_ctx_t *ctx, const pimdal_smj_arguments_t *args,
                           pimdal_merge_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Ingress of a host column into device memory.  Replaces the scatter of     */
/* Arrow buffers to the DPUs (populate_mram / dist_table,                     */
/* pimdal/support/transfer_helper.h, after the parquet read of                */
/* pimdal/main/tpc_h/reader/read_table.cpp:18-34): copies bytes from host     */
/* memory to dst on the stream.  A pageable source is copied chunk by chunk  */
/* by several host threads (PIMDAL_INGEST_THREADS, default 8) into pinned     */
/* staging buffers of PIMDAL_INGEST_CHUNK bytes owned by the context (made by */
/* the first call that needs them), so host copies overlap each other and the */
/* transfers; a pinned (page-locked or registered) source is copied directly. */
/* A pageable source may be reused on return (every host read is done); a    */
/* pinned source is read by the transfer itself, so it must stay unchanged   */
/* until the stream reaches the copy, as with cudaMemcpyAsync.  The device   */
/* copy completes in stream order.                                           */
/* ------------------------------------------------------------------------- */
#define PIMDAL_INGEST_CHUNK (16u << 20)
int pimdal_ingest(pimdal_ctx_t *ctx, const void *host_src, size_t bytes, void *dst,
                  pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Radix partition.  Replaces part_kernel (pimdal/join/hash_join.h:23-31,    */
/* hash_join.c:154-235): element e goes to partition                         */
/* (hash0(e.key) >> (shift - log2(part_n))) & (part_n - 1), hash0 being the  */
/* reference's pimdal/hash/hash_func.h:5-14.  Stable.  part_sizes[p] is the  */
/* first row of partition p, part_sizes[part_n] = size (uint64, device).     */
/* ------------------------------------------------------------------------- */
typedef struct {
  const void *in;           /* part_arguments_t.in_ptr: uint32 key column      */
  const uint32_t *in_ptr;   /* row ids; NULL = index                           */
  uint64_t size;            /* part_arguments_t.size                           */
  uint32_t shift;           /* part_arguments_t.shift (<= 32)                  */
  uint32_t part_n;          /* part_arguments_t.part_n: power of 2, <= 65536   */
  void *part_out;           /* part_arguments_t.part_ptr: partitioned keys     */
  uint32_t *part_out_ptr;   /* partitioned row ids (may be NULL)               */
  uint64_t *part_sizes;     /* part_arguments_t.part_sizes: part_n + 1 entries */
  int32_t layout;           /* PIMDAL_LAYOUT_COLUMNS                           */
  int32_t pad;
} pimdal_part_arguments_t;

int pimdal_part_workspace_size(const pimdal_part_arguments_t *args, size_t *bytes);
int pimdal_part_kernel(pimdal_ctx_t *ctx, const pimdal_part_arguments_t *args,
                       pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Hash tables.  pimdal_hash_kernel replaces hash_kernel                      */
/* (pimdal/join/hash_join.h:6-13, hash_join.c:40-115): a linear-probing       */
/* table of table_size 64-bit slots (payload << 32 | key), built with         */
/* atomicCAS, in caller memory of pimdal_hash_table_bytes(table_size) bytes.  */
/* pimdal_hj_probe replaces merge_kernel (hash_join.h:44-57,                  */
/* hash_join.c:343-430): for every probe row and every build row with the     */
/* same key it emits (probe ptr, build payload), in probe order.              */
/* ------------------------------------------------------------------------- */
typedef struct {
  const void *in_key;       /* hash_arguments_t.in_ptr: build keys (uint32)    */
  const uint32_t *in_ptr;   /* build payloads / row ids; NULL = index          */
  uint64_t size;            /* hash_arguments_t.size                           */
  void *table_ptr;          /* hash_arguments_t.table_ptr                      */
  uint64_t table_size;      /* hash_arguments_t.table_size: slots, power of 2  */
} pimdal_hash_arguments_t;

typedef struct {
  const void *table_ptr;    /* merge_arguments_t.table_ptr (built above)       */
  uint64_t table_size;      /* merge_arguments_t.size: slots                   */
  const void *in_key;       /* merge_arguments_t.in_ptr: probe keys            */
  const uint32_t *in_ptr;   /* probe row ids; NULL = index                     */
  uint64_t size;            /* probe rows                                      */
  uint32_t *out_outer;      /* merge_arguments_t.out_ptr: probe ptr per match  */
  uint32_t *out_inner;      /* ... and build payload per match                 */
  uint64_t out_capacity;
} pimdal_probe_arguments_t;

size_t pimdal_hash_table_bytes(uint64_t table_size);
int pimdal_hash_kernel(pimdal_ctx_t *ctx, const pimdal_hash_arguments_t *args,
                       pimdal_stream_t stream);
int pimdal_hj_probe(pimdal_ctx_t *ctx, const pimdal_probe_arguments_t *args,
                    pimdal_merge_results_t *d_result, pimdal_stream_t stream);

/* Whole hash join (the pipeline of pimdal/main/join/hash and
 * reference/db_operators/hash_join.cpp:159-219).  A table that fits
 * l2_budget_bytes is built and probed directly; for a larger one both
 * relations are first radix-partitioned by the top bits of the key hash
 * whose next bits give a key's home bucket, so the rows of one partition
 * touch one L2-sized slice of the table, and the partitioned rows are built
 * and probed in partition order.  Output per match: build payload and probe
 * row id; partitions in order, probe order within a partition (probe order
 * overall when not partitioned).  With duplicate build keys the matches of
 * one probe row come in table order.
 * partition_bits 9..16 selects shared-memory partitions instead: both
 * relations are partitioned 2^partition_bits ways (stable passes of at most
 * 6 bits) so that one partition's build rows fit a table in one CTA's shared
 * memory (the reference CPU join's 16384 cache-sized partitions,
 * hash_join.cpp:57-157); load_factor_pct and l2_budget_bytes are then
 * unused.  Same output order, except that a partition with more than 12288
 * build rows is joined in chunks of build rows, its output chunk-major. */
typedef struct {
  const void *build_key;          /* uint32 / int32 keys                          */
  const uint32_t *build_payload;  /* NULL = build row id                          */
  uint64_t size_build;            /* < 2^32                                       */
  const void *probe_key;
  const uint32_t *probe_ptr;      /* NULL = probe row id                          */
  uint64_t size_probe;            /* < 2^30                                       */
  uint32_t *out_build_payload;
  uint32_t *out_probe_ptr;
  uint64_t out_capacity;
  uint32_t partition_bits;        /* 0 = auto, 0xFFFFFFFF = never partition, 1..8   */
                                  /* (L2-sized) or 9..16 (shared-memory partitions) */
  uint32_t load_factor_pct;       /* table load factor in percent; 0 = 50          */
  uint64_t l2_budget_bytes;       /* 0 = 48 MiB                                   */
} pimdal_hash_join_arguments_t;

int pimdal_hash_join_workspace_size(const pimdal_hash_join_arguments_t *args, size_t *bytes);
int pimdal_hash_join(pimdal_ctx_t *ctx, const pimdal_hash_join_arguments_t *args,
                     pimdal_merge_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Bloom-filter semi-join prefilter.  pimdal_filter_kernel replaces           */
/* filter_kernel (pimdal/join/hash_join.h:15-21,64-66; hash_join.c:116-149;   */
/* insert_bloom_filter, pimdal/hash/hash_steps.c:143-152): for every          */
/* partition p of already-partitioned keys (rows [part_sizes[p],              */
/* part_sizes[p+1])), a filter of PIMDAL_FILTER_BITS bits is zeroed and bit   */
/* hashK(key) % PIMDAL_FILTER_BITS is set for K = 1..4, hashK being the       */
/* reference's hash1..hash4 (pimdal/hash/hash_func.h:16-60).  Filter p is     */
/* bytes [p, p+1) * PIMDAL_FILTER_BYTES of filter_ptr; bit b is bit b % 8 of  */
/* byte b / 8, as in the reference, so filters are interchangeable with it.   */
/* pimdal_match_kernel replaces match_kernel (hash_join.h:33-42,74-76;        */
/* hash_join.c:236-341; probe_bloom_filter, hash_steps.c:163-185): keeps the  */
/* rows r < size whose key finds all four bits set in the filter of r's       */
/* partition, in input order.  match_sizes[0] = 0 and match_sizes[p+1] = kept */
/* rows of partition p (uint64, device); t_count = all kept rows.  Rows that  */
/* lie in no partition are not kept.  part_sizes must be non-decreasing.      */
/* pimdal_match_kernel takes 8 bytes per 2048 input rows of the context's     */
/* workspace.                                                                */
/* ------------------------------------------------------------------------- */
#define PIMDAL_FILTER_BITS 16384
#define PIMDAL_FILTER_BYTES (PIMDAL_FILTER_BITS / 8)

typedef struct {
  const void *in;              /* filter_arguments_t.in_ptr: partitioned keys    */
  void *filter_ptr;            /* filter_arguments_t.filter_ptr: part_n filters, */
                               /* 16-byte aligned                                */
  const uint64_t *part_sizes;  /* filter_arguments_t.part_sizes: part_n + 1      */
                               /* row offsets (device)                           */
  uint32_t part_n;             /* filter_arguments_t.part_n (>= 1)               */
  int32_t layout;              /* PIMDAL_LAYOUT_COLUMNS (uint32 keys) or         */
                               /* PIMDAL_LAYOUT_PAIRS (key_ptr32 pairs)          */
} pimdal_filter_arguments_t;

typedef struct {
  const void *filter_ptr;      /* match_arguments_t.filter_ptr                   */
  uint64_t size;               /* match_arguments_t.size: input rows (< 2^31)    */
  const void *part_ptr;        /* match_arguments_t.part_ptr: partitioned keys   */
  const uint32_t *part_row;    /* row ids (columns layout); NULL = row index     */
  void *out_ptr;               /* match_arguments_t.out_ptr: kept keys (pairs)   */
  uint32_t *out_row;           /* kept row ids (columns layout; may be NULL)     */
  uint64_t out_capacity;       /* rows of room in the outputs                    */
  uint64_t *match_sizes;       /* match_arguments_t.match_sizes: part_n + 1      */
  const uint64_t *part_sizes;  /* match_arguments_t.part_sizes: part_n + 1       */
  uint32_t part_n;             /* match_arguments_t.part_n (>= 1)                */
  int32_t layout;              /* PIMDAL_LAYOUT_COLUMNS or PIMDAL_LAYOUT_PAIRS   */
} pimdal_match_arguments_t;

int pimdal_filter_kernel(pimdal_ctx_t *ctx, const pimdal_filter_arguments_t *args,
                         pimdal_stream_t stream);
int pimdal_match_workspace_size(const pimdal_match_arguments_t *args, size_t *bytes);
int pimdal_match_kernel(pimdal_ctx_t *ctx, const pimdal_match_arguments_t *args,
                        pimdal_merge_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Group-by.  Replaces group_kernel (pimdal/aggregate/aggregate.h:7-25):      */
/* the hash variant of aggregate_hash.c:123-194 and the sort variant of       */
/* aggregate.c:82-158, plus the host merge and order_by of                    */
/* pimdal/main/aggregate/hash/host/host_aggregate_sync.cpp:71-95, and the CPU */
/* hash_table_aggregate of reference/db_operators/aggregate.cpp:40-83.  The   */
/* combiner function pointer (aggregate.h:11; UNIQUE / COUNT / SUM of         */
/* groupby.h:17-21) becomes a fixed set of exact int64 aggregates -- any of   */
/* SUM (wrapping mod 2^64), COUNT, MIN, MAX -- each requested by passing its  */
/* output column.  Groups come out ascending by key (signed for I32).         */
/* ------------------------------------------------------------------------- */
typedef enum {
  PIMDAL_GROUP_AUTO = 0, /* hash */
  PIMDAL_GROUP_HASH = 1, /* shared-memory tables + global table, then key order */
  PIMDAL_GROUP_SORT = 2  /* stable radix sort, then reduce-by-key              */
} pimdal_group_method_t;

typedef struct {
  uint64_t size;           /* aggr_arguments_t.size: rows (< 2^30)              */
  const void *in;          /* aggr_arguments_t.in: group keys (int32 / uint32)  */
  const int64_t *in_val;   /* values; NULL = 1 for every row                    */
  void *out;               /* aggr_arguments_t.out: group keys, ascending       */
  int64_t *out_sum;        /* per group; any of these may be NULL               */
  int64_t *out_count;
  int64_t *out_min;
  int64_t *out_max;
  uint64_t out_capacity;   /* groups room in the outputs                        */
  uint64_t expected_groups;/* hash method: table sizing hint (0 = min(size, 2^22)) */
  int32_t key_dtype;       /* PIMDAL_I32 or PIMDAL_U32                           */
  int32_t method;          /* pimdal_group_method_t                             */
} pimdal_aggr_arguments_t;

typedef struct {
  uint64_t t_count; /* aggr_results_t.t_count: number of groups */
} pimdal_aggr_results_t;

int pimdal_group_workspace_size(const pimdal_aggr_arguments_t *args, size_t *bytes);
int pimdal_group_kernel(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *args,
                        pimdal_aggr_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Pipeline glue between operators.  Replaces the separate DPU passes of     */
/* arithmetic_kernel (pimdal/general/arithmetic.c:35-67), the reduce chains  */
/* (pimdal/general/reduce.c:42-77) and the column <-> pair conversions of    */
/* the query pipelines (pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156)    */
/* with fused single-pass gathers.                                           */
/* ------------------------------------------------------------------------- */
/* out[i] = col[idx[i]] for i < n. */
int pimdal_gather_u32(pimdal_ctx_t *ctx, const uint32_t *col, const uint32_t *idx, uint64_t n,
                      uint32_t *out, pimdal_stream_t stream);

typedef struct {
  uint64_t size;               /* joined rows                                   */
  const uint32_t *match_row;   /* per joined row: index into sel_rows           */
  const uint32_t *match_attr;  /* per joined row: the dimension attribute       */
  const uint32_t *sel_rows;    /* selected fact rows (NULL: match_row is the row) */
  const int64_t *price;        /* fact columns, indexed by fact row             */
  const int32_t *discount;     /* percent, 0..100                               */
  const uint8_t *flag;         /* second group column (NULL: none)              */
  uint32_t attr_mult;          /* key = attr * attr_mult + flag[row] (uint32,   */
  uint32_t pad;                /* wrapping)                                     */
  uint32_t *out_key;           /* group key per joined row                      */
  int64_t *out_val;            /* price * (100 - discount) per joined row       */
} pimdal_revenue_arguments_t;

int pimdal_revenue_keys(pimdal_ctx_t *ctx, const pimdal_revenue_arguments_t *args,
                        pimdal_stream_t stream);

/* Fused filter -> join -> group-by of one query over a fact range: the chain  */
/* the reference's TPC-H pipelines run as sel_kernel, merge_kernel,           */
/* arithmetic_kernel and group_kernel with host steps between them (e.g.      */
/* pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156), in one pass.  Fact row  */
/* r < size takes part when date_lo <= date[r] <= date_hi; it is joined       */
/* through a table built by pimdal_hash_kernel (every build row whose key is  */
/* jkey[r] contributes, its payload being the attribute); the group key is    */
/* attr * attr_mult + (flag ? flag[r] : 0) in 32-bit arithmetic that wraps,   */
/* exactly as pimdal_revenue_keys computes it, and the value                  */
/* price[r] * (100 - discount[r]).  Output: the groups with at least one row, */
/* ascending by key, with SUM (int64, wrapping) and COUNT -- exactly what     */
/* selection + gather + pimdal_hj_probe + pimdal_revenue_keys +               */
/* pimdal_group_kernel return.  Group keys must be < key_space (at most       */
/* PIMDAL_FUSED_MAX_KEYS); a larger one raises PIMDAL_ERR_ARG at              */
/* pimdal_ctx_sync_status.  Scratch: key_space * 16 bytes of the context's    */
/* workspace.                                                                 */
#define PIMDAL_FUSED_MAX_KEYS 4096
typedef struct {
  uint64_t size;               /* fact rows in the range                        */
  const int32_t *date;         /* filter column                                 */
  int32_t date_lo, date_hi;    /* inclusive bounds                              */
  const uint32_t *jkey;        /* join key per fact row                         */
  const void *table_ptr;       /* table of pimdal_hash_kernel                   */
  uint64_t table_size;         /* its slots                                     */
  const uint8_t *flag;         /* second group column (NULL: none)              */
  const int64_t *price;
  const int32_t *discount;     /* percent, 0..100                               */
  uint32_t attr_mult;          /* key = attr * attr_mult + flag[row]            */
  uint32_t key_space;          /* keys are < key_space (1..PIMDAL_FUSED_MAX_KEYS) */
  uint32_t *out_key;           /* groups, ascending                             */
  int64_t *out_sum;
  int64_t *out_count;
  uint64_t out_capacity;
} pimdal_select_join_aggregate_arguments_t;

int pimdal_select_join_aggregate_workspace_size(
    const pimdal_select_join_aggregate_arguments_t *args, size_t *bytes);
int pimdal_select_join_aggregate(pimdal_ctx_t *ctx,
                                 const pimdal_select_join_aggregate_arguments_t *args,
                                 pimdal_aggr_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Fused select -> arithmetic -> group-by scan.  Replaces the chains that the */
/* reference's query pipelines run as separate DPU kernels with host steps    */
/* between them: one sel_kernel per predicate with load_next gathers in       */
/* between, arithmetic_kernel (pimdal/general/arithmetic.c:35-67) and         */
/* reduce_kernel (pimdal/general/reduce.c:42-77) -- e.g. the Q6 chain of      */
/* pimdal/main/tpc_h/query6/dpu/kernel_q6.c:112-156 -- and the per-row sums   */
/* and group-by of pimdal/main/tpc_h/query1/dpu/kernel_q1_1.c:84-170 with     */
/* kernel_q1_2.c.                                                              */
/*                                                                            */
/* Row i < size is the table row r = rows ? rows[i] : i.  It takes part when  */
/* every predicate holds on its column at r.  Its group key is                */
/* sum_g group[g].col[r] * group[g].mult (uint32, wrapping; 0 without group   */
/* columns) and must be < key_space, else PIMDAL_ERR_ARG is raised at         */
/* pimdal_ctx_sync_status.  Expression e is the int64 product (wrapping) of   */
/* its terms, term t being (negate ? -col[r] : col[r]) + add, or the constant */
/* add when col is NULL.  Output: the groups with at least one row, ascending */
/* by key: out_key, out_count and one SUM (int64, wrapping) per expression in */
/* out_sum[e] (NULL: not written).  Columns are PIMDAL_I32, PIMDAL_U32,        */
/* PIMDAL_I64 or PIMDAL_U8 (zero-extended) values.  Scratch:                  */
/* key_space * (n_exprs + 1) * 8 bytes of the context's workspace.            */
/* ------------------------------------------------------------------------- */
#define PIMDAL_SA_MAX_PREDS 4
#define PIMDAL_SA_MAX_GROUP_COLS 2
#define PIMDAL_SA_MAX_EXPRS 6
#define PIMDAL_SA_MAX_TERMS 3
#define PIMDAL_SA_MAX_KEYS 1024

typedef struct {
  const void *col;
  int32_t dtype;           /* pimdal_dtype_t                                   */
  int32_t pad;
  pimdal_pred_t pred;      /* the predicate on col (sel_arguments_t.pred)      */
} pimdal_column_pred_t;

typedef struct {
  const void *col;
  int32_t dtype;
  uint32_t mult;           /* key += col[r] * mult                             */
} pimdal_group_col_t;

typedef struct {
  const void *col;         /* NULL: the term is the constant add               */
  int32_t dtype;
  int32_t negate;          /* term = -col[r] + add                             */
  int64_t add;
} pimdal_term_t;

typedef struct {
  pimdal_term_t term[PIMDAL_SA_MAX_TERMS];
  uint32_t n_terms;        /* 1..PIMDAL_SA_MAX_TERMS                           */
  uint32_t pad;
} pimdal_expr_t;

typedef struct {
  uint64_t size;                                  /* rows scanned (< 2^32)    */
  const uint32_t *rows;                           /* NULL: row i is i         */
  pimdal_column_pred_t pred[PIMDAL_SA_MAX_PREDS];
  uint32_t n_preds;
  uint32_t n_group;
  pimdal_group_col_t group[PIMDAL_SA_MAX_GROUP_COLS];
  uint32_t key_space;                             /* 1..PIMDAL_SA_MAX_KEYS    */
  uint32_t n_exprs;                               /* 0..PIMDAL_SA_MAX_EXPRS   */
  pimdal_expr_t expr[PIMDAL_SA_MAX_EXPRS];
  uint32_t *out_key;
  int64_t *out_count;
  int64_t *out_sum[PIMDAL_SA_MAX_EXPRS];
  uint64_t out_capacity;                          /* groups room              */
} pimdal_select_aggregate_arguments_t;

int pimdal_select_aggregate_workspace_size(const pimdal_select_aggregate_arguments_t *args,
                                           size_t *bytes);
int pimdal_select_aggregate(pimdal_ctx_t *ctx, const pimdal_select_aggregate_arguments_t *args,
                            pimdal_aggr_results_t *d_result, pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Per-row arithmetic: replaces arithmetic_kernel (pimdal/general/            */
/* arithmetic.c:35-67, arithmetic.h:7-19), which multiplies two columns       */
/* element by element, and the DPU pipelines' per-row projections such as the */
/* revenue price * (100 - discount) of                                        */
/* pimdal/main/tpc_h/query3/dpu/kernel_q3_5.c:107 or the comparison column of */
/* query4/dpu/kernel_q4_2.c:104-106 (commit - receipt < 0).                    */
/*                                                                            */
/* out[i] = expr - minus (each as in pimdal_select_aggregate: the int64       */
/* product, wrapping, of its terms; minus with 0 terms is 0) at row           */
/* r = rows ? rows[i] : i, for i < size, shifted right (arithmetically) by    */
/* shift bits; out_dtype PIMDAL_I64 stores it whole, PIMDAL_I32 its low 32    */
/* bits (shift = 32: the high word).  With a single column term this is a     */
/* gather (a load_next) of any column type.                                   */
/* ------------------------------------------------------------------------- */
typedef struct {
  uint64_t size;                /* rows (< 2^32)                                 */
  const uint32_t *rows;         /* NULL: row i is i                              */
  pimdal_expr_t expr;           /* 1..PIMDAL_SA_MAX_TERMS terms                  */
  pimdal_expr_t minus;          /* 0..PIMDAL_SA_MAX_TERMS terms                  */
  void *out;                    /* size values of out_dtype                      */
  int32_t out_dtype;            /* PIMDAL_I64 or PIMDAL_I32                      */
  uint32_t shift;               /* 0..63                                         */
} pimdal_project_arguments_t;

int pimdal_project(pimdal_ctx_t *ctx, const pimdal_project_arguments_t *args,
                   pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Batched form: many independent group-by or hash-join instances, each phase */
/* one persistent launch fed by a device work queue.  No reference counterpart */
/* (the reference runs one operator instance per DPU launch, e.g. the        */
/* dpu_launch loops of pimdal/main/aggregate/hash/host/host_aggregate_sync.cpp */
/* and pimdal/main/join/hash/host/host_join_sync.cpp); every instance gets    */
/* what pimdal_group_kernel / pimdal_hash_join (unpartitioned) return for the */
/* same arguments.                                                           */
/*                                                                           */
/* A plan holds the instances' descriptors, the work items, the tables and   */
/* the scratch in device memory allocated when it is created (not inside a   */
/* stream capture).  pimdal_batch_run then launches a fixed kernel sequence  */
/* that reads nothing from the host, so it can be captured into a CUDA graph */
/* and replayed; the inputs are read and the outputs written at run time.    */
/* ------------------------------------------------------------------------- */
typedef struct pimdal_batch pimdal_batch_t;

typedef struct {
  uint32_t rows_per_item;   /* rows of one work item, a multiple of 128 (0 = 65536) */
  uint32_t load_factor_pct; /* hash-table load factor in percent, 10..90 (0 = 50)   */
  uint32_t reserved[2];
} pimdal_batch_tuning_t;

typedef enum { PIMDAL_BATCH_GROUP = 0, PIMDAL_BATCH_HASH_JOIN = 1 } pimdal_batch_kind_t;

/* d_results: device array of count results (instance i -> d_results[i]). */
int pimdal_group_batch_create(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *args,
                              uint32_t count, const pimdal_batch_tuning_t *tuning,
                              pimdal_aggr_results_t *d_results, pimdal_batch_t **plan);
int pimdal_hash_join_batch_create(pimdal_ctx_t *ctx, const pimdal_hash_join_arguments_t *args,
                                  uint32_t count, const pimdal_batch_tuning_t *tuning,
                                  pimdal_merge_results_t *d_results, pimdal_batch_t **plan);
int pimdal_batch_run(pimdal_ctx_t *ctx, pimdal_batch_t *plan, pimdal_stream_t stream);
int pimdal_batch_device_bytes(const pimdal_batch_t *plan, size_t *bytes);
int pimdal_batch_destroy(pimdal_batch_t *plan);

/* Autotuner: times the candidate work-item sizes and load factors on these  */
/* instances (running them, so their outputs are written), returns the      */
/* fastest and caches it in the context under the batch's shape (kind,      */
/* count, row and group totals and maxima).  A later call for the same shape */
/* returns the cached choice without running.  args is a                     */
/* pimdal_aggr_arguments_t or pimdal_hash_join_arguments_t array; d_results  */
/* as for the create call.  *cached tells whether the choice came from the   */
/* cache.                                                                    */
int pimdal_batch_autotune(pimdal_ctx_t *ctx, int kind, const void *args, uint32_t count,
                          void *d_results, pimdal_batch_tuning_t *best, int *cached,
                          pimdal_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Autotuner of the plain operators (the batch autotuner's counterpart for    */
/* single calls).  The hash join's partition fan-out and table load factor    */
/* (L2-sized partitions) or shared-memory partition count, and the           */
/* high-cardinality hash group-by's mode (hash-partitioned chunks or         */
/* one direct global table) and partition count are chosen per input shape.   */
/* pimdal_*_autotune runs the call once per candidate on the given arguments  */
/* (writing the outputs; the last run is the chosen candidate's), keeps the   */
/* fastest in the context under the call's shape (the log2 of its sizes; for  */
/* the join also the L2 budget; for the group-by the expected groups and      */
/* whether values are given), and returns it.  A later call of the same       */
/* shape whose arguments leave the choice to the library (hash join:          */
/* partition_bits = 0 and load_factor_pct = 0; group-by: method HASH or AUTO) */
/* uses it; a later autotune of a cached shape returns it without running     */
/* (*cached = 1).  The workspace-size queries of such calls cover every       */
/* candidate.  A group-by with nothing to choose (few groups, the sort       */
/* method) runs once with the library's choice and returns group_mode 0.     */
/* ------------------------------------------------------------------------- */
typedef struct {
  uint32_t partition_bits;   /* hash join: 0xFFFFFFFF = unpartitioned, else 1..16      */
  uint32_t load_factor_pct;  /* hash join: table load factor in percent                */
  uint32_t group_mode;       /* group-by: 0 library's choice, 1 partitioned, 2 direct  */
  uint32_t group_part_bits;  /* group-by, partitioned: log2 of the hash partitions     */
  float ms;                  /* the chosen candidate's device time (0 when not timed)  */
  uint32_t candidates;       /* candidates timed (0 when cached or nothing to choose)  */
} pimdal_tuning_t;

int pimdal_hash_join_autotune(pimdal_ctx_t *ctx, const pimdal_hash_join_arguments_t *args,
                              pimdal_merge_results_t *d_result, pimdal_tuning_t *best,
                              int *cached, pimdal_stream_t stream);
int pimdal_group_autotune(pimdal_ctx_t *ctx, const pimdal_aggr_arguments_t *args,
                          pimdal_aggr_results_t *d_result, pimdal_tuning_t *best, int *cached,
                          pimdal_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* PIMDAL_GPU_H_ */
