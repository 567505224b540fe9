/*
 * sj_join.h — C ABI of the B200 (sm_100a) equi-hash-join.
 *
 * This is the drop-in boundary that replaces the three cuDF calls inside Sirius's
 * physical hash-join operator, `sirius_physical_hash_join::execute`
 * (src/op/sirius_physical_hash_join.cpp:1527-1955):
 *
 *   build   cudf::hash_join(keys, compare_nulls(), stream)           (:1620)
 *           cudf::distinct_hash_join(keys, UNEQUAL, 0.5, stream)      (:1614-1615, :1852)
 *   probe   hash_join::inner_join(probe_keys, {}, stream)             (:1688)
 *           distinct_hash_join::inner_join(probe_keys, stream)        (:1671)
 *           cudf::inner_join(left_keys, right_keys, nulls, stream)    (:1872)
 *   gather  gather_join_output -> cudf::gather(...) x2                (:1299-1359, :1336, :1348)
 *
 * Conventions (the cuDF ones the operator already uses):
 *   - a column is a contiguous array of fixed-width values plus an optional validity bitmask of
 *     32-bit words; bit (validity_offset + i) % 32 of word (validity_offset + i) / 32 set means
 *     row i is valid (not NULL);
 *   - row ids are int32 (cudf::size_type, src/op/sirius_physical_hash_join.cpp:1305-1306);
 *   - "probe" = left = input_batches[0], "build" = right = input_batches[1]
 *     (src/op/sirius_physical_hash_join.cpp:1157-1158);
 *   - output columns are [probe payload columns..., build payload columns...], the order
 *     gather_join_output assembles (src/op/sirius_physical_hash_join.cpp:1350-1355).
 *
 * Every pointer argument named d_* or carrying column data is device memory on the current
 * device. Every call is stream-ordered on the given stream unless its comment says it
 * synchronizes. Calls on distinct tables are thread-safe; probes of one built table may run
 * concurrently from many threads and streams (the BUILD_PROBE pattern, one writer then many
 * readers, src/op/sirius_physical_hash_join.cpp:1585-1588, :1624).
 *
 * Errors are returned as sj_status; a human-readable message for the last failing call on the
 * calling thread is available from sj_last_error(). No call throws across the ABI.
 */
#ifndef SJ_JOIN_H
#define SJ_JOIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same export style as Sirius's FFI layer (SIRIUS_FFI_EXPORT, src/include/sirius_ffi.hpp:37). */
#ifndef SJ_EXPORT
#define SJ_EXPORT __attribute__((visibility("default")))
#endif

/* Binary-compatible with cudaStream_t; 0 is the legacy default stream. */
typedef struct CUstream_st* sj_stream_t;

/* Status codes. The adapter maps SJ_ERR_OOM to rmm::out_of_memory so that Sirius's
 * oom_reschedule path still fires (src/pipeline/gpu_pipeline_task.cpp:386-437); everything else
 * becomes std::runtime_error, as the operator's own misuse errors are
 * (src/op/sirius_physical_hash_join.cpp:1548-1564). */
typedef enum sj_status {
  SJ_OK             = 0,
  SJ_ERR_OOM        = 1, /* the allocator returned NULL */
  SJ_ERR_TABLE_FULL = 2, /* a bounded insert ran out of slots */
  SJ_ERR_INVALID    = 3, /* bad argument (types, sizes, null pointers, alignment) */
  SJ_ERR_DEVICE     = 4, /* a CUDA runtime call failed */
  SJ_ERR_TIMEOUT    = 5, /* a bounded wait gave up */
  SJ_ERR_CAPACITY   = 6, /* more output rows than the capacity the caller gave */
  SJ_ERR_BUSY       = 7  /* admission refused (memory budget / queue full) */
} sj_status;

/* Fixed-width column types. Keys must be SJ_INT32 or SJ_INT64 (cuDF INT32/INT64 and the types
 * Sirius stores in them, e.g. DATE / TIMESTAMP); payloads may be any of these. */
typedef enum sj_type {
  SJ_TYPE_INVALID = 0,
  SJ_INT8         = 1,
  SJ_INT16        = 2,
  SJ_INT32        = 3,
  SJ_INT64        = 4,
  SJ_FLOAT32      = 5,
  SJ_FLOAT64      = 6,
  SJ_BOOL8        = 7,
  SJ_UINT32       = 8,
  SJ_UINT64       = 9
} sj_type;

/* A read-only column view (cudf::column_view: data<T>() , null_mask(), offset(), size()). */
typedef struct sj_column {
  const void* data;         /* row 0 of the column (head + offset already applied) */
  const uint32_t* validity; /* NULL = all rows valid */
  int64_t validity_offset;  /* bit index of row 0 inside validity */
  int64_t num_rows;
  int32_t type;             /* sj_type */
  int32_t reserved;
} sj_column;

/* A writable output column: num_rows is given by the call's capacity. */
typedef struct sj_mut_column {
  void* data;
  uint32_t* validity; /* required iff the matching input payload column has validity */
  int32_t type;       /* sj_type, must equal the input payload type */
  int32_t reserved;
} sj_mut_column;

/* Device memory comes from the caller (Sirius: the cuCascade reservation-aware RMM resource the
 * task attached to its stream, src/pipeline/gpu_pipeline_task.cpp:523-525). Passing NULL where
 * an sj_alloc* is accepted uses cudaMallocAsync / cudaFreeAsync on the call's stream. */
typedef struct sj_alloc {
  void* ctx;
  void* (*alloc)(void* ctx, size_t bytes, sj_stream_t stream);
  void (*free)(void* ctx, void* ptr, size_t bytes, sj_stream_t stream);
} sj_alloc;

/* NULL semantics of the key comparison: cudf::null_equality as the operator caches it in
 * compare_nulls_ (src/op/sirius_physical_hash_join.cpp:252-264). UNEQUAL: NULL never matches.
 * EQUAL: NULL matches NULL (every key IS NOT DISTINCT FROM). */
typedef enum sj_null_equality { SJ_NULLS_UNEQUAL = 0, SJ_NULLS_EQUAL = 1 } sj_null_equality;

/* Table layout. AUTO builds a DISTINCT table when the valid build keys are unique and a GROUPED
 * table otherwise; GROUPED forces the grouped layout. */
typedef enum sj_layout {
  SJ_LAYOUT_AUTO     = 0,
  SJ_LAYOUT_DISTINCT = 1, /* one slot per build row, keys unique (cudf::distinct_hash_join) */
  SJ_LAYOUT_GROUPED  = 2  /* one slot per distinct key + a row-id range (cudf::hash_join multiset) */
} sj_layout;

/* Slot encoding chosen at build time from the key range. */
typedef enum sj_slot_kind {
  SJ_SLOT_PACKED64 = 0, /* (key - key_min) << rid_bits | row id, inserted by 64-bit atomicCAS */
  SJ_SLOT_WIDE128  = 1  /* {int64 key, row id} pair, inserted by 128-bit atomicCAS */
} sj_slot_kind;

/* Output reservation of the single-pass probe: matches are always compacted warp-aggregated
 * (prefix over the lanes' hit counts); the range is then reserved with one atomicAdd per warp or
 * one per CTA tile. AUTO picks per-CTA for probes of 2^20 rows or more. */
/* How probe matches reserve output positions: one atomicAdd per warp, per CTA tile (for probes of
 * 2^20 rows or more under AUTO), or per warp with warps taking tiles from a shared counter. */
typedef enum sj_aggregation {
  SJ_AGG_AUTO = 0,
  SJ_AGG_WARP = 1,
  SJ_AGG_CTA = 2,
  SJ_AGG_WARP_DYNAMIC = 3
} sj_aggregation;

/* Tunables. Zero-initialised fields take defaults (sj_default_params fills them in). */
/* How a DISTINCT probe reads its rows and writes its output. DIRECT: lanes write their own
 * matches at positions ranked by warp ballots (no shared-memory staging of matches); it serves
 * outputs of row ids, up to 2 probe payloads and up to 3 build payloads of 4 or 8 bytes without
 * NULLs (attached build payloads: 8-byte fields). DIRECT_TMA: DIRECT with the probe rows (keys,
 * payloads) bulk-copied into shared memory two tiles ahead by the TMA engine; needs 16-byte
 * aligned probe columns. STAGED: matches are staged per warp in shared memory and written column
 * by column; it serves every output shape. AUTO takes DIRECT where it applies, else STAGED. */
typedef enum sj_probe_kernel {
  SJ_PROBE_KERNEL_AUTO = 0,
  SJ_PROBE_KERNEL_STAGED = 1,
  SJ_PROBE_KERNEL_DIRECT = 2,
  SJ_PROBE_KERNEL_DIRECT_TMA = 3
} sj_probe_kernel;

/* L2 eviction priority of the table loads of a probe (PTX createpolicy / L2::cache_hint). */
typedef enum sj_l2_priority {
  SJ_L2_AUTO = 0,       /* the default below */
  SJ_L2_NORMAL = 1,     /* plain loads */
  SJ_L2_EVICT_LAST = 2  /* table lines evicted after the probe stream's */
} sj_l2_priority;

typedef struct sj_join_params {
  int32_t layout;           /* sj_layout */
  int32_t null_equality;    /* sj_null_equality */
  float load_factor;        /* slots in use / slots; default 0.5 (the distinct_hash_join value) */
  int32_t block_size;       /* threads per CTA for probe kernels; default 256 */
  int32_t group_width;      /* accepted and ignored: a single join's probe uses one lane per key,
                               which loads a whole 32-byte bucket (4 or 2 slots) at once. Lanes
                               sharing one key are the batched path's sj_batch_params.group_width,
                               where one lane per key measured fastest. Default 1 */
  int32_t partition_bits;   /* radix bits of the partitioned variant: 0 = automatic (partition
                               when the table and its attached payloads outgrow L2), -1 = never,
                               1..10 = that many bits (2^bits partitions) */
  int32_t force_wide;       /* 1 = use SJ_SLOT_WIDE128 even when the packed encoding fits */
  int32_t ctas_per_sm;      /* grid = ctas_per_sm * SM count for grid-stride kernels; default 4 */
  int32_t aggregation;      /* sj_aggregation: how probe matches reserve output positions */
  int32_t probe_kernel;     /* sj_probe_kernel: write-out of DISTINCT probes; default AUTO */
  int32_t rows_per_lane;    /* probe rows per lane and tile of the direct kernel: 2 or 4; 0 = 2 */
  int32_t probe_partition_mb; /* partitioned probe: table megabytes per probe partition (the part
                                 of the table one sweep keeps in L2); 0 = default (48) */
  int32_t table_l2_priority;  /* sj_l2_priority of the table's slot and record loads in the
                                 direct probe kernels */
  int32_t bloom_bits_per_key; /* > 0: the build also produces the join's dynamic filter (the
                                 blocked Bloom filter of sj_bloom_build, that many bits per build
                                 row), its bits set by the insert pass itself, so the filter costs no
                                 second read of the build keys; read it with sj_table_bloom. One key
                                 column only. 0 = none */
  int32_t reserved[2];
} sj_join_params;

typedef struct sj_table sj_table;

typedef struct sj_table_info {
  int64_t build_rows;      /* rows of the build key column */
  int64_t valid_rows;      /* rows with a non-NULL key */
  int64_t null_rows;       /* rows with a NULL key */
  int64_t distinct_keys;   /* distinct non-NULL keys */
  int64_t num_slots;       /* slots in the open-addressing table */
  int64_t device_bytes;    /* bytes held on the device by the table */
  int64_t key_min;         /* smallest valid key (0 if none) */
  int64_t key_max;         /* largest valid key (-1 if none) */
  int32_t layout;          /* sj_layout actually built (DISTINCT or GROUPED) */
  int32_t slot_kind;       /* sj_slot_kind */
  int32_t rid_bits;        /* row-id bits of a packed slot */
  int32_t key_type;        /* sj_type of the key */
  int32_t partition_bits;  /* radix bits used (0 = not partitioned) */
  int32_t max_group;       /* largest number of build rows sharing one key */
} sj_table_info;

/* ---------------------------------------------------------------------------------------------
 * Core join: build, probe, gather.
 * ------------------------------------------------------------------------------------------- */

/* Fill *params with defaults. */
SJ_EXPORT void sj_default_params(sj_join_params* params);

/* Build a hash table over the build keys (replaces the cudf::hash_join / distinct_hash_join
 * constructors, src/op/sirius_physical_hash_join.cpp:1614-1620). Row ids in the table are the
 * build column's row indices. num_keys 1..4: several INT32/INT64 key columns form a composite key
 * (the operator's multi-column conditions, prepare_join_keys, :1234-1291), packed exactly into one
 * 64-bit key from the build's per-column value ranges — refused with SJ_ERR_INVALID when the ranges
 * need more than 63 bits; every probe of the table then passes the same number of key columns.
 * Rows with a NULL key (any NULL column) are not inserted under SJ_NULLS_UNEQUAL; under
 * SJ_NULLS_EQUAL a NULL column compares equal to NULL column by column. The key columns are only
 * read during the call; the caller keeps the build batch alive for the gather, as the operator
 * does (:1593).
 * Synchronizes `stream` (once to size the table from the key range, once to choose the layout);
 * the reference synchronizes after the build as well (:1622). */
SJ_EXPORT sj_status sj_build(const sj_column* keys, int32_t num_keys, const sj_join_params* params,
                             const sj_alloc* alloc, sj_stream_t stream, sj_table** out);

/* sj_build plus attached build payload columns (the build-side columns the operator projects,
 * rhs_output_columns, src/op/sirius_physical_hash_join.cpp:1339-1353). The table keeps its own
 * copy of them in table-position order, so a probe's payload gather reads the rows stored next to
 * the matched slot's partition instead of the build batch at random; pass build_payload = NULL to
 * sj_probe_gather to gather them. With radix partitioning (large tables) positions follow
 * partition order and every partition's slots and payload rows stay L2-resident while its probes
 * run. Costs one copy of the attached columns in device memory. */
SJ_EXPORT sj_status sj_build_ex(const sj_column* keys, int32_t num_keys, const sj_column* payload,
                                int32_t num_payload, const sj_join_params* params, const sj_alloc* alloc,
                                sj_stream_t stream, sj_table** out);

/* Free the table's device memory, stream-ordered on `stream` (on_finalize_operator frees each
 * slot's table on its device, src/op/sirius_physical_hash_join.cpp:2084-2097). */
SJ_EXPORT sj_status sj_table_destroy(sj_table* table, sj_stream_t stream);

SJ_EXPORT sj_status sj_table_get_info(const sj_table* table, sj_table_info* info);

/* Probe keys of every sj_probe_* call: the table's number of key columns. A single key column
 * may be of the other integer type than the table's (the reference's key casts,
 * prepare_join_keys, src/op/sirius_physical_hash_join.cpp:1234-1291): INT32 probe keys widen
 * exactly into an INT64 table; INT64 probe keys narrow exactly into an INT32 table when in range
 * and otherwise never match (they stay non-NULL); a table whose INT32 keys span the whole INT32
 * range refuses INT64 probes with SJ_ERR_INVALID. Composite-key columns may mix types freely.
 *
 * Count the INNER matches of the probe keys (the size pass cuDF runs before retrieval for the
 * multiset inner_join). Writes the count to *d_count (device int64). Stream-ordered. */
SJ_EXPORT sj_status sj_probe_count(const sj_table* table, const sj_column* probe_keys,
                                   int32_t num_keys, const sj_alloc* alloc, sj_stream_t stream,
                                   int64_t* d_count);

/* INNER probe fused with the payload gather (replaces inner_join + gather_join_output,
 * src/op/sirius_physical_hash_join.cpp:1671, :1688, :1299-1359).
 * For every (probe row i, build row j) with equal keys it writes, at one output position p:
 *   out_probe_rid[p] = i, out_build_rid[p] = j   (either pointer may be NULL: not written)
 *   out_probe_payload[c][p] = probe_payload[c][i]
 *   out_build_payload[c][p] = build_payload[c][j]
 * and validity bits copied from the payload columns (NULLIFY is not needed for INNER).
 * build_payload == NULL with num_build_payload == the number of columns attached by sj_build_ex
 * gathers the attached columns (in attach order) instead of caller columns.
 * *d_count (device int64) receives the total number of matches M; only positions p < capacity
 * are written, so the call succeeded iff M <= capacity (read *d_count after the stream).
 * A negative *d_count means a bounded device wait of the DIRECT_TMA kernel ran out (report it as
 * SJ_ERR_TIMEOUT; the outputs are incomplete).
 * A DISTINCT table never has M > probe rows. Output order is unspecified, as cuDF's is.
 * Stream-ordered; scratch for GROUPED tables comes from `alloc`. */
SJ_EXPORT sj_status sj_probe_gather(const sj_table* table, const sj_column* probe_keys,
                                    int32_t num_keys, const sj_column* probe_payload,
                                    int32_t num_probe_payload, const sj_column* build_payload,
                                    int32_t num_build_payload, int32_t* out_probe_rid,
                                    int32_t* out_build_rid, const sj_mut_column* out_probe_payload,
                                    const sj_mut_column* out_build_payload, int64_t capacity,
                                    const sj_alloc* alloc, sj_stream_t stream, int64_t* d_count);

/* Join types of the operator's BUILD_PROBE path on a built table
 * (src/op/sirius_physical_hash_join.cpp:1640-1700; MARK: resolve_mark_join_result, :1461-1525). */
typedef enum sj_join_kind {
  SJ_JOIN_INNER = 0,
  SJ_JOIN_LEFT = 1,  /* INNER rows + every probe row without a match (NULL keys included) */
  SJ_JOIN_SEMI = 2,  /* probe rows with at least one match, each once */
  SJ_JOIN_ANTI = 3,  /* probe rows without a match (NULL keys included: NOT EXISTS) */
  SJ_JOIN_MARK = 4,  /* one BOOL8 per probe row, SQL three-valued (IN) */
  SJ_JOIN_FULL = 5   /* LEFT rows + every build row without a match (NULL keys included) */
} sj_join_kind;

/* Row id written for the missing side of an outer row (cuDF's JoinNoneValue). */
#define SJ_NO_ROW ((int32_t)0x80000000)

/* A join of `kind` on a built table; the counterpart of sj_probe_gather for every join type.
 *   INNER: exactly sj_probe_gather.
 *   LEFT:  the INNER rows at positions [0, M), then one row per unmatched probe row with
 *          out_build_rid = SJ_NO_ROW and NULL build payloads; every out_build_payload must have a
 *          validity buffer. *d_count = total rows.
 *   FULL:  the LEFT rows, then one row per unmatched build row (NULL keys included) with
 *          out_probe_rid = SJ_NO_ROW and NULL probe payloads; every output payload needs a validity
 *          buffer, and build payloads must be caller columns (build_payload != NULL), since
 *          NULL-key build rows are not stored in the table. A FULL join of several probe batches
 *          would need their matches combined; this call covers one probe input.
 *   SEMI / ANTI: out_probe_rid and the probe payloads of the selected probe rows (build outputs
 *          unused). *d_count = rows.
 *   MARK:  out_mark[i] = 1 if probe row i has a match, else 0, for every probe row; out_mark_validity
 *          (bitmask, may be NULL only when no row can be NULL) marks NULL the unmatched rows whose
 *          probe key is NULL, or every unmatched row when the build side has a NULL key (the IN rule
 *          of resolve_mark_join_result; the table must use SJ_NULLS_UNEQUAL). *d_count = probe rows.
 * Rows beyond `capacity` are not written (*d_count still counts them). Stream-ordered. */
SJ_EXPORT sj_status sj_probe_join(const sj_table* table, sj_join_kind kind, const sj_column* probe_keys,
                                  int32_t num_keys, const sj_column* probe_payload, int32_t num_probe_payload,
                                  const sj_column* build_payload, int32_t num_build_payload, int32_t* out_probe_rid,
                                  int32_t* out_build_rid, const sj_mut_column* out_probe_payload,
                                  const sj_mut_column* out_build_payload, int64_t capacity, uint8_t* out_mark,
                                  uint32_t* out_mark_validity, const sj_alloc* alloc, sj_stream_t stream,
                                  int64_t* d_count);

/* Hash partitioning of a table (the partition operator's hash_partition,
 * src/op/partition/gpu_partition_impl.cpp:29-110, which splits both sides of a partitioned join).
 * The `num_columns` columns (up to 8; include the key columns to have them reordered too) are written
 * to out_columns in partition order; partition p occupies rows [d_offsets[p], d_offsets[p+1]) and
 * d_offsets (device, num_partitions + 1 int64) ends with the row count. The partition of a row is
 * the top log2(num_partitions) bits of mix64 of its key — the key itself for one key column without
 * NULLs (the same function that splits a radix-partitioned table), else a fold over the 1..4 key
 * columns; rows with a NULL key column go to partition 0. Equal keys land in the same partition in
 * every table. num_partitions: a power of two, 1..1024. Order within a partition is unspecified.
 * Stream-ordered; scratch from `alloc`. */
SJ_EXPORT sj_status sj_hash_partition(const sj_column* keys, int32_t num_keys, const sj_column* columns,
                                      int32_t num_columns, int32_t num_partitions, const sj_mut_column* out_columns,
                                      int64_t* d_offsets, const sj_alloc* alloc, sj_stream_t stream);

/* Dynamic filter from the build keys (src/cuda/sirius_dynamic_bloom_filter.cu, published by the
 * hash join at src/op/sirius_physical_hash_join.cpp:1960-2069): a blocked Bloom filter of 32-byte
 * blocks, `bits_per_key` bits per key (0 = 16), 8 bits set per key in one block, so a probe row is
 * tested with one sector read. NULL keys are not inserted. sj_bloom_contains writes one byte per
 * probe row: 1 = may be in the build keys (no false negatives), 0 = not; rows with a NULL probe key
 * test 0 and, when out_validity is given, get a NULL bit there (the probe's NULLs). For an exact
 * in-list filter use a built table: sj_probe_join(SJ_JOIN_MARK) gives the same mask without false
 * positives. Stream-ordered. */
typedef struct sj_bloom sj_bloom;
SJ_EXPORT sj_status sj_bloom_build(const sj_column* keys, int32_t bits_per_key, const sj_alloc* alloc,
                                   sj_stream_t stream, sj_bloom** out);
SJ_EXPORT sj_status sj_bloom_contains(const sj_bloom* bloom, const sj_column* probe_keys, uint8_t* out_mask,
                                      uint32_t* out_validity, sj_stream_t stream);
SJ_EXPORT int64_t sj_bloom_bytes(const sj_bloom* bloom);
/* The dynamic filter a table's build produced (sj_join_params.bloom_bits_per_key > 0), or NULL.
 * It is the filter sj_bloom_build would make from the same key column, bit for bit; test it with
 * sj_bloom_contains. The table owns it: it lives until sj_table_destroy (do not destroy it). */
SJ_EXPORT const sj_bloom* sj_table_bloom(const sj_table* table);
SJ_EXPORT sj_status sj_bloom_destroy(sj_bloom* bloom, sj_stream_t stream);

/* One-shot INNER join (STANDARD mode: cudf::inner_join(left_keys, right_keys, compare_nulls(),
 * stream), src/op/sirius_physical_hash_join.cpp:1872, followed by gather_join_output): builds a
 * throwaway table on build_keys, probes it with probe_keys and gathers. Same output contract as
 * sj_probe_gather. Synchronizes `stream` like sj_build. */
SJ_EXPORT sj_status sj_inner_join(const sj_column* build_keys, const sj_column* probe_keys,
                                  int32_t num_keys, const sj_column* probe_payload,
                                  int32_t num_probe_payload, const sj_column* build_payload,
                                  int32_t num_build_payload, int32_t* out_probe_rid,
                                  int32_t* out_build_rid, const sj_mut_column* out_probe_payload,
                                  const sj_mut_column* out_build_payload, int64_t capacity,
                                  const sj_join_params* params, const sj_alloc* alloc,
                                  sj_stream_t stream, int64_t* d_count);

/* ---------------------------------------------------------------------------------------------
 * Batched joins: thousands of independent small INNER joins in one persistent launch.
 * ------------------------------------------------------------------------------------------- */

/* One join of a batch. Keys are SJ_INT32 or SJ_INT64 (one type for the whole batch); each side
 * carries at most one payload column (data == NULL: none). Outputs follow sj_probe_gather:
 * every match writes probe row id, build row id and the payloads at one position < capacity;
 * the join's match count is read with sj_batch_plan_counts. Duplicated build keys are allowed
 * (all matches are produced). Key validity is honoured (NULL never matches). */
typedef struct sj_batch_join {
  sj_column build_key;
  sj_column build_payload;
  sj_column probe_key;
  sj_column probe_payload;
  int32_t* out_probe_rid;
  int32_t* out_build_rid;
  sj_mut_column out_probe_payload;
  sj_mut_column out_build_payload;
  int64_t capacity;
} sj_batch_join;

/* Tunables of the batched launch (0 = default; the autotuner picks them per GPU and size class). */
typedef struct sj_batch_params {
  int32_t block_size;   /* threads per CTA: 128, 256 or 512; default 256 */
  int32_t group_width;  /* lanes cooperating on one probe key: 1, 2, 4 or 8; default 1 */
  float load_factor;    /* table slots in use / slots; default 0.5 */
  int32_t tile_rows;    /* rows per work item; default 4096 */
  int32_t ctas_per_sm;  /* resident CTAs per SM of the persistent grid; default 4 */
  int32_t reserved[7];
} sj_batch_params;

typedef struct sj_batch_plan sj_batch_plan;

/* Plan a batch: sizes every join's table, lays out one table arena and the work queue (every
 * join's build tiles, then every join's probe tiles), and uploads the descriptors. The column
 * pointers are read by each launch, so the caller may refill the same buffers between launches.
 * Allocates through `alloc`; stream-ordered. */
SJ_EXPORT sj_status sj_batch_plan_create(const sj_batch_join* joins, int32_t num_joins,
                                         const sj_batch_params* params, const sj_alloc* alloc,
                                         sj_stream_t stream, sj_batch_plan** out);

/* Run every join of the plan in ONE persistent kernel launch (plus memset nodes that reset the
 * tables, counters and queue). A probe work item waits — bounded, then flags an error — until its
 * join's build tiles are done. Stream-ordered, no host synchronisation, capturable. */
SJ_EXPORT sj_status sj_batch_plan_launch(sj_batch_plan* plan, sj_stream_t stream);

/* Capture sj_batch_plan_launch into a CUDA graph once (on `stream`) and replay it: the whole batch
 * is one graph launch. */
SJ_EXPORT sj_status sj_batch_plan_replay(sj_batch_plan* plan, sj_stream_t stream);

/* The comparison point: the same joins with one build launch and one probe launch per join. */
SJ_EXPORT sj_status sj_batch_plan_launch_per_join(sj_batch_plan* plan, sj_stream_t stream);

/* Copy the per-join match counts (int64[num_joins], device) and the plan's error word (device
 * int32: 0 = ok, 1 = a probe item timed out waiting for its build) into caller memory. */
SJ_EXPORT sj_status sj_batch_plan_counts(const sj_batch_plan* plan, int64_t* d_counts, int32_t* d_error,
                                         sj_stream_t stream);

SJ_EXPORT sj_status sj_batch_plan_destroy(sj_batch_plan* plan, sj_stream_t stream);

/* ---------------------------------------------------------------------------------------------
 * Serving: resident tables, probe requests admitted continuously against a memory budget
 * (the BUILD_PROBE pattern, src/op/sirius_physical_hash_join.cpp:1585-1624, with admission in the
 * manner of exec::admission_control, src/include/exec/admission_control.hpp:39-104).
 * ------------------------------------------------------------------------------------------- */

typedef struct sj_server sj_server;

typedef struct sj_server_config {
  int32_t slots;                /* requests on the GPU at once, one CUDA stream each; default 4 */
  int32_t max_skip;             /* times the queue head may be passed by smaller requests; 8 */
  int64_t memory_budget_bytes;  /* device bytes for request outputs + scratch; default 120 GiB */
  int64_t reserve_bytes;        /* device memory the server's pool takes up front and keeps, so
                                   requests are served without growing it; default 0 */
  int32_t batch_small;          /* 0 (default): requests of fewer than 65,536 rows into tables whose
                                   attached payloads are 8-byte fields without NULLs (at most 3)
                                   are batched: all such queued requests run as one kernel launch
                                   on the server's batch stream while it is idle; -1: every request
                                   runs alone on a slot stream */
  int32_t reserved[5];
} sj_server_config;

/* A finished request. Output buffers are device memory owned by the server until
 * sj_server_release(request_id); columns are [probe row id, build row id, attached build
 * payloads...] with `count` valid rows. Times are seconds on one steady clock. */
typedef struct sj_request_result {
  uint64_t request_id;
  int32_t status;   /* sj_status of the request */
  int32_t table_id;
  int64_t count;
  int64_t probe_rows;
  int32_t* probe_rid;
  int32_t* build_rid;
  void* build_payload[8];
  uint32_t* build_validity[8]; /* NULL where the payload column has no validity */
  double t_submit;  /* sj_server_submit returned */
  double t_admit;   /* admitted onto a slot */
  double t_done;    /* its last GPU operation finished */
} sj_request_result;

/* Start a server on the current device (its worker thread runs until sj_server_destroy). */
SJ_EXPORT sj_status sj_server_create(const sj_server_config* config, sj_server** out);

/* Build a resident table (unique keys: DISTINCT layout) with its attached payload columns.
 * Synchronizes. *table_id receives the table's id. */
SJ_EXPORT sj_status sj_server_add_table(sj_server* server, const sj_column* key, const sj_column* payload,
                                        int32_t num_payload, const sj_join_params* params,
                                        int32_t* table_id);

/* Queue a probe request: INNER join of `probe_key` (device column, valid until the request
 * completes) with table `table_id`. Returns immediately; the worker admits the request when a slot
 * is free and its outputs + scratch fit the budget. A request larger than the whole budget fails
 * with SJ_ERR_BUSY. */
SJ_EXPORT sj_status sj_server_submit(sj_server* server, int32_t table_id, const sj_column* probe_key,
                                     uint64_t request_id);

/* Move up to `capacity` finished requests into `out`, waiting up to `wait_ms` for at least one.
 * Returns the number written (>= 0) or a negative sj_status. */
SJ_EXPORT int32_t sj_server_poll(sj_server* server, sj_request_result* out, int32_t capacity, int32_t wait_ms);

/* Free a finished request's output buffers (returns their bytes to the budget). */
SJ_EXPORT sj_status sj_server_release(sj_server* server, uint64_t request_id);

/* Stop the worker after the queued and in-flight requests finish and free everything. */
SJ_EXPORT sj_status sj_server_destroy(sj_server* server);

/* The one-shot INNER join of sj_inner_join with every column in HOST memory (pinned memory for
 * full speed): the operator's whole join when its batches live in host memory, as the reference's
 * memory spaces allow (batches are moved to the device before a GPU operator runs, and results
 * are read back after it; src/op/sirius_physical_hash_join.cpp:1527-1955 runs in between).
 * The build side is copied to the device and built with its payloads attached (sj_build_ex). The
 * probe side streams through in chunks of `chunk_rows` rows (0 = 8M; rounded up to a multiple of
 * 32). Chunk i+2 uploads on one copy stream while chunk i is probed on `stream` and chunk i-1's
 * output downloads on another copy stream, so host-to-device and device-to-host traffic overlap.
 * The output has the same columns and meaning as sj_inner_join, with probe row ids of the whole
 * probe. It is written to host buffers in chunk order, and rows past `capacity` are not written.
 * *out_count (a host pointer) receives the full match count.
 * Key columns may carry NULLs (validity at any offset). Payload columns with NULLs are refused
 * with SJ_ERR_INVALID. Device memory comes from `alloc`: the build copy, then the table, plus two
 * input and two output chunk slots. Returns when every output row is on the host. */
SJ_EXPORT sj_status sj_inner_join_host(const sj_column* build_keys, const sj_column* probe_keys,
                                       int32_t num_keys, const sj_column* probe_payload,
                                       int32_t num_probe_payload, const sj_column* build_payload,
                                       int32_t num_build_payload, int32_t* out_probe_rid,
                                       int32_t* out_build_rid,
                                       const sj_mut_column* out_probe_payload,
                                       const sj_mut_column* out_build_payload, int64_t capacity,
                                       int64_t chunk_rows, const sj_join_params* params,
                                       const sj_alloc* alloc, sj_stream_t stream, int64_t* out_count);

/* The one-shot INNER join of sj_inner_join for callers that cannot allocate device memory: code
 * held to a device-memory reservation that is already fully committed (an allocation attempt
 * there would be refused and rescheduled as out-of-memory), latency-critical host threads that
 * must not wait in the driver's allocator, and hosts whose allocator belongs to another component.
 * No counterpart in the reference: Sirius's join always allocates through its memory pool.
 * Every byte of scratch (hash table, build statistics, grouped-probe match list) comes from one
 * 64 MiB `static __device__` array per GPU; no cudaMalloc, cudaFree or allocator callback is used.
 * The driver commits the array when it loads the library's device code: at the first call on a
 * device under lazy module loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2), at
 * library load under EAGER. A caller whose memory will be fully committed later makes one warm-up
 * call while 64 MiB are still free; every GPU that ran the entry point then holds the array until
 * the process exits. Outputs follow sj_probe_gather's contract (caller-provided device buffers,
 * *d_count = matches). Inputs whose worst-case scratch exceeds the array are rejected with
 * SJ_ERR_INVALID before any GPU work; at load factor 0.5 that allows 2^19 build rows with up to
 * 1.9M probe rows, or 2^20 build rows with up to 600K probe rows. The table is never
 * radix-partitioned and builds no dynamic filter: every params field is honoured except
 * partition_bits, probe_partition_mb and bloom_bits_per_key.
 * All calls share the array and leave their data in it; each call re-initialises what it reads,
 * but calls that overlap on the GPU race: serialise them (one stream, or synchronise between).
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make it before any stream capture begins on the device. Synchronizes `stream`
 * like sj_build. */
SJ_EXPORT sj_status sj_inner_join_noalloc(const sj_column* build_keys, const sj_column* probe_keys,
                                          int32_t num_keys, const sj_column* probe_payload,
                                          int32_t num_probe_payload, const sj_column* build_payload,
                                          int32_t num_build_payload, int32_t* out_probe_rid,
                                          int32_t* out_build_rid,
                                          const sj_mut_column* out_probe_payload,
                                          const sj_mut_column* out_build_payload, int64_t capacity,
                                          const sj_join_params* params, sj_stream_t stream,
                                          int64_t* d_count);

/* ---------------------------------------------------------------------------------------------
 * Diagnostics.
 * ------------------------------------------------------------------------------------------- */

SJ_EXPORT const char* sj_status_string(sj_status status);

/* Message of the last failing call on this thread ("" if none). */
SJ_EXPORT const char* sj_last_error(void);

/* Opt-in per-kernel timing. While enabled (process-wide), every kernel the library launches from
 * the calling thread is bracketed by a CUDA event pair on its stream; sj_timing_collect waits for
 * those events, writes up to `capacity` (name, milliseconds) records in launch order, clears the
 * log and returns the number of records. Names are static strings. Off by default. Turning it on
 * creates a pool of 512 events for the calling thread, so the timed launches create none. */
typedef struct sj_kernel_time {
  const char* name;
  float ms;
  int32_t reserved;
} sj_kernel_time;

SJ_EXPORT void sj_timing_enable(int32_t on);
SJ_EXPORT int32_t sj_timing_collect(sj_kernel_time* out, int32_t capacity);

/* Test hook for the library's bounded device waits: runs, in one small kernel, the batched join's
 * wait for a join's build tiles on a counter that nothing increments, and the TMA probe ring's wait
 * for a stage's bulk copies on an mbarrier that nothing arrives on, each limited to `polls` polls
 * (1..2^20). d_status: device int32[3]; after the stream, d_status[0] / d_status[1] are 1 when the
 * build wait / the mbarrier wait gave up (as they must), 0 otherwise; d_status[2] is scratch. The
 * library reports such a timeout as SJ_ERR_TIMEOUT (a batch's error word bit 0, a probe's negative
 * count). No counterpart in the reference. Stream-ordered. */
SJ_EXPORT sj_status sj_debug_wait_timeout(int32_t polls, sj_stream_t stream, int32_t* d_status);

/* ABI version: major * 10000 + minor * 100 + patch. */
SJ_EXPORT int32_t sj_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SJ_JOIN_H */
