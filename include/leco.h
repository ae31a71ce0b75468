/*
 * leco.h -- C ABI of the B200 (sm_100a) LeCo integer codec.
 *
 * Drop-in boundary for the reference's per-block codec classes
 * (yhliu918/Learn-to-Compress):
 *   Leco_int<T>             headers/piecewise_fix_integer_template.h:14-338
 *   FOR_int<T>              headers/FOR_integer_template.h:14-249
 *   Delta_int<T>            headers/delta_integer_template.h:14-158
 *   Leco_int_poly<T,2>      headers/poly_fix_integer_template.h:15-292
 *   Leco_cost_merge_double_wo_round<uint64_t> (variable-length segments)
 *                           headers/piecewise_cost_merge_integer_template_double_wo_round.h:18-700
 * each with init / encodeArray8_int / decodeArray8 / randomdecodeArray8.
 *
 * The reference encodes a column as independent per-block byte strings held by
 * its driver (experiments/leco_int_fix_template.cpp:108-127).  Here a column is
 *   payload  : the reference block images concatenated, byte for byte,
 *   offsets  : uint64 byte offset of block b in payload, offsets[nblocks] = total,
 * so block b is exactly what the reference's encodeArray8_int writes for values
 * [b*block_size, min(n, (b+1)*block_size)).  Payload buffers must be 8-byte
 * aligned and extend LECO_PAYLOAD_SLACK bytes past the last block (kernels read
 * whole 8-byte words).
 *
 * Conventions: all pointers named d_* are device pointers, h_* host pointers;
 * every call is asynchronous on `stream` unless documented otherwise; status 0 =
 * success, negative = error (leco_last_error() describes the last one on the
 * calling thread).  No call allocates device memory unless its comment says so.
 * The library keeps per-device addresses of its own device variables (the error
 * word, the built-in encoder scratch) from the first call on each device, so the
 * device must not be reset (cudaDeviceReset) while the library is in use.
 */
#ifndef LECO_B200_H_
#define LECO_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *leco_stream_t; /* == cudaStream_t */

enum leco_codec {
  LECO_CODEC_LINEAR = 0, /* Leco_int<T>: OLS line + midpoint shift, signed residuals */
  LECO_CODEC_FOR = 1,    /* FOR_int<T>: frame of reference, unsigned offsets        */
  LECO_CODEC_DELTA = 2,  /* Delta_int<T>: signed first differences                  */
  LECO_CODEC_POLY2 = 3,  /* Leco_int_poly<T,2>: degree-2 normal-equation fit        */
  LECO_CODEC_VARLEN = 4, /* Leco_cost_merge_double_wo_round<uint64_t> segments      */
  LECO_CODEC_LINEAR_F32 = 5 /* piecewise_fix_op_max (u32 only, legacy): f32 slope,
                               13-byte header, raw u32 body when l >= 31
                               (piecewise_fix_op_minimize_maxerror.h:45-186).
                               Encode (leco_encode, leco_encode_host,
                               leco_block_encode), decode, random access, sum,
                               directory, zone map, validation.  The encoder's
                               difference lists for the reference's additive bulk
                               decoder are not produced: leco_decode returns the
                               stored values directly. */
};

/* Value type = bytes per value. */
enum leco_dtype { LECO_U32 = 4, LECO_U64 = 8 };

/* How the encoder fits the block model.
 * LECO_FIT_REFERENCE: the reference's sequential FP64 moment sums
 *   (headers/lr.h:66-85, headers/polynomial_regression_internals.hpp:111-137),
 *   so every block image is byte-identical to the reference encoder's.
 * LECO_FIT_EXACT: exact 128-bit integer moment sums (parallel reduction), one
 *   rounding to FP64, then the reference's formula.  Deterministic for any
 *   launch shape; the stored model is what the reference decoder recomputes, so
 *   the streams still decode bit-exactly in the reference's own decoder. */
enum leco_fit_mode { LECO_FIT_REFERENCE = 0, LECO_FIT_EXACT = 1 };

enum leco_status {
  LECO_OK = 0,
  LECO_ERR_ARG = -1,         /* bad argument (null pointer, size, codec/dtype)      */
  LECO_ERR_CUDA = -2,        /* a CUDA runtime call failed                           */
  LECO_ERR_CORRUPT = -3,     /* a block header or offset is not a valid stream       */
  LECO_ERR_NOMEM = -4,       /* device or host allocation failed / admission refused */
  LECO_ERR_TIMEOUT = -5,     /* a bounded device wait gave up (error word set)       */
  LECO_ERR_UNSUPPORTED = -6, /* codec/dtype combination not provided                 */
  LECO_ERR_CAPACITY = -7     /* output buffer smaller than the encoded size          */
};

#define LECO_PAYLOAD_SLACK 64u
#define LECO_MAX_BLOCK 16384u

/* Directory entry derived from a block header (32 bytes), kept device-resident
 * so random access reads one L2-resident sector of metadata per lookup:
 *   word0 = absolute bit address of field 0 | (l << 56) | (kind << 48)
 *   a0,a1,a2 = model (theta0/theta1, poly coefficients, FOR base or Delta base
 *   as raw 64-bit patterns). */
typedef struct leco_dir_entry {
  uint64_t word0;
  double a0, a1, a2;
} leco_dir_entry;

/* ---- sizing (host, no device work) ------------------------------------ */

/* Number of blocks of a column. */
uint64_t leco_num_blocks(uint64_t n, uint32_t block_size);
/* Upper bound on payload bytes (including LECO_PAYLOAD_SLACK). */
uint64_t leco_max_payload_bytes(int codec, int dtype, uint64_t n, uint32_t block_size);
/* Bytes of device workspace leco_encode needs (caller allocates). */
uint64_t leco_encode_workspace_bytes(int codec, int dtype, uint64_t n, uint32_t block_size, int fit_mode);
/* Exact byte size of one reference block image with l-bit fields
 * (headers/bit_write.h:257-323 and :326-390 padding rules). */
uint64_t leco_block_bytes(int codec, int dtype, uint32_t l, uint32_t nvalues);

/* ---- column encode / decode / random access (device buffers) ---------- */

/* Encodes n values (d_values, dtype) in blocks of block_size with `codec`
 * (LINEAR, FOR, DELTA, POLY2; LINEAR_F32 for u32, the loop of
 * piecewise_fix_op_max::encodeArray8 in experiments/fix_int.cpp:70-80).  Writes the concatenated reference block images
 * to d_payload (capacity payload_cap bytes, see leco_max_payload_bytes),
 * d_offsets[nblocks+1] and, when d_dir != NULL, the directory (nblocks
 * entries).  Replaces the driver loop over <Codec>::encodeArray8_int
 * (experiments/leco_int_fix_template.cpp:111-127).  One single-pass kernel
 * (plus a sequential-fit kernel for LECO_FIT_REFERENCE columns whose FP64 sums
 * round), a block-size prefix sum by decoupled look-back through d_workspace.
 * d_payload must be 16-byte aligned (the images are written in 16-byte stores). */
int leco_encode(int codec, int dtype, const void *d_values, uint64_t n, uint32_t block_size, int fit_mode,
                uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets, leco_dir_entry *d_dir,
                void *d_workspace, uint64_t workspace_bytes, leco_stream_t stream);

/* Same as leco_encode, for callers that cannot allocate device memory (no counterpart in the
 * reference, whose encoder only writes host memory).  An engine whose buffer manager owns all
 * device memory, or a latency-critical thread that must not call cudaMalloc/cudaFree (they can
 * synchronize the whole device), can pass just the input and output buffers: the encoder's
 * scratch lives in a fixed array inside the library (1 MiB per GPU that loads the library, held
 * until the process exits).  Columns are limited to leco_encode_noalloc_max_blocks() blocks
 * (32768); larger ones are rejected with LECO_ERR_ARG.  The first call on each device resolves
 * the array's device address (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  Every call uses the same array and the scratch is re-zeroed by each call: calls whose
 * work overlaps on the GPU (different streams, no ordering between them) race and must not be
 * issued.  Allocates nothing.  The resolved address belongs to the CUDA context of that
 * first call: do not reset the device (cudaDeviceReset) while this library is in use. */
int leco_encode_noalloc(int codec, int dtype, const void *d_values, uint64_t n, uint32_t block_size, int fit_mode,
                        uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets, leco_dir_entry *d_dir,
                        leco_stream_t stream);
/* Largest column, in blocks, that leco_encode_noalloc accepts. */
uint64_t leco_encode_noalloc_max_blocks(void);

/* Decodes a whole column into d_out[n].  Replaces <Codec>::decodeArray8 per block
 * (piecewise_fix_integer_template.h:142-204, FOR_integer_template.h:83-112,
 * delta_integer_template.h:89-127, poly_fix_integer_template.h:93-158).  A block
 * is raw iff l == 8*sizeof(T) (the reference's random-access rule; its bulk
 * decoders also treat l == 8*sizeof(T)-1 as raw, which mis-decodes such blocks). */
int leco_decode(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                uint32_t block_size, void *d_out, leco_stream_t stream);

/* Decodes values [first, first+count) of a column into d_out[count]
 * (range scan: only the touched blocks are read). */
int leco_decode_range(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                      uint32_t block_size, uint64_t first, uint64_t count, void *d_out, leco_stream_t stream);

/* Builds the device directory from the block headers (after an import). */
int leco_build_directory(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                         uint32_t block_size, leco_dir_entry *d_dir, leco_stream_t stream);

/* Random access: d_out[i] = value d_idx[i] of the column, for i < m.  Replaces
 * the per-index randomdecodeArray8 loop (experiments/leco_int_fix_template.cpp:189-207;
 * piecewise_fix_integer_template.h:305-337, FOR_integer_template.h:218-245,
 * delta_integer_template.h:132-154, poly_fix_integer_template.h:259-291).
 * d_dir may be NULL (headers are then parsed from the payload). Indices >= n
 * yield 0 and set the column error word (see leco_check). */
int leco_gather(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets,
                const leco_dir_entry *d_dir, uint64_t n, uint32_t block_size, const uint64_t *d_idx, uint64_t m,
                void *d_out, leco_stream_t stream);

/* Sum of all decoded values mod 2^64, written to *d_sum, without
 * materialising the values (compressed-domain summation; the reference has
 * one only for its legacy u32 codec, piecewise_fix_op.h:187-282).
 * d_partials: device scratch of leco_sum_workspace_bytes() bytes. */
uint64_t leco_sum_workspace_bytes(uint64_t n, uint32_t block_size);
int leco_sum(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
             uint32_t block_size, uint64_t *d_sum, void *d_partials, leco_stream_t stream);

/* ---- predicate pushdown ------------------------------------------------------
 * Indices of the values that pass a filter, found without decoding the column to
 * memory.  Output: uint32 global value indices b*block_size + k (the reference's
 * uint32_t out), blocks in order, within a block in the order the reference's
 * method emits them; at most out_cap are written and *d_count receives the full
 * count.  Columns of LINEAR (Leco_int<T>) or FOR (FOR_int<T>) blocks, n < 2^32.
 * d_ws: leco_filter_workspace_bytes() bytes of 8-byte aligned device scratch.
 * A raw LINEAR block (l == 8*sizeof(T)), which the reference's filters read as a
 * model, is filtered on its stored values here. */
uint64_t leco_filter_workspace_bytes(uint64_t n, uint32_t block_size);

/* Values above `filter`: Leco_int<T>::filter_range
 * (piecewise_fix_integer_template.h:206-252: scan from the model's threshold index)
 * or FOR_int<T>::filter_range (FOR_integer_template.h:115-160) on every block, as the
 * filter experiment calls them (experiments/leco_int_fix_template.cpp:244-256).
 * d_zone_min / d_zone_max (each nullable): per-block minima / maxima (leco_zonemap).
 * Blocks whose maximum is <= filter are skipped unread, as the experiment's zone map
 * does (:247-249); blocks whose minimum is above it match from the threshold index on
 * without their fields being read (the same indices the reference emits). */
int leco_filter_range(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                      uint32_t block_size, uint64_t filter, const uint64_t *d_zone_min, const uint64_t *d_zone_max,
                      uint32_t *d_out, uint64_t out_cap, uint64_t *d_count, void *d_ws, uint64_t ws_bytes,
                      leco_stream_t stream);

/* Close-range filter: filter_range_close (piecewise_fix_integer_template.h:254-303,
 * FOR_integer_template.h:166-215) on every block, as the close-range experiments call
 * it (leco_int_fix_template.cpp:290-322, FOR_int_fix_template.cpp:303-322).
 * FOR: values v with filter1 < v % base < filter2.  LINEAR: for the windows
 * (filter1 + p*base, filter2 + p*base), p = 0, 1, ..., the values inside each window
 * among the indices the block's model allows, windows in order; with d_zone_min
 * (per-block minima) each block's first window is derived from its minimum as the
 * experiment does (:299-304), without it every block starts at (filter1, filter2).
 * 1 <= base <= INT32_MAX (the codecs take it as int).  The reference appends each
 * window's indices after the previous ones only for l == 0 blocks (for l > 0 it
 * writes every window from the block's first output slot again, :280); here they
 * are always appended, and the count is the reference's.  A LINEAR block that
 * needs more than 65536 windows sets the error word (leco_check returns
 * LECO_ERR_UNSUPPORTED); the reference's loop costs windows x block length there. */
int leco_filter_range_close(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                            uint32_t block_size, uint64_t filter1, uint64_t filter2, uint64_t base,
                            const uint64_t *d_zone_min, uint32_t *d_out, uint64_t out_cap, uint64_t *d_count,
                            void *d_ws, uint64_t ws_bytes, leco_stream_t stream);

/* Per-block minimum and maximum of the decoded values, as uint64 (the filter
 * experiments' zone map, experiments/leco_int_fix_template.cpp:219-239, built there
 * from the raw column; here from the compressed one).  Any fixed-block codec. */
int leco_zonemap(int codec, int dtype, const uint8_t *d_payload, const uint64_t *d_offsets, uint64_t n,
                 uint32_t block_size, uint64_t *d_min, uint64_t *d_max, leco_stream_t stream);

/* ---- variable-length segments (Leco_cost_merge_double_wo_round<uint64_t>) ----
 * headers/piecewise_cost_merge_integer_template_double_wo_round.h:18-700.  A column is
 * payload (segment images back to back), offsets[nseg + 1] and starts[nseg] (value
 * index of each segment's first value, starts[0] = 0; segment s covers
 * [starts[s], starts[s+1]) and the last one ends at n). */

/* Host partitioner (encodeArray8_int's split + merge passes, :283-570): coarse blocks
 * as the reference driver cuts them (n / coarse_blocks values each), `delta` = the
 * reference's merge penalty in bits.  Writes the segment starts (<= starts_cap) and
 * *nseg.  threads <= 0: all host cores. */
int leco_varlen_partition(const uint64_t *h_values, uint64_t n, uint32_t coarse_blocks, int64_t delta,
                          uint64_t *h_starts, uint64_t starts_cap, uint64_t *nseg, int threads);
/* The same partitioner on the GPU (same segment starts bit for bit): one thread per
 * coarse block, each with a private scratch slot in d_ws (the segment list of the
 * split/merge phase, then the segment starts and sizes of the pairwise passes).
 * d_values on the device; writes d_starts (<= starts_cap; the error word records an
 * overflow) and *d_nseg on the device.  d_ws: leco_varlen_partition_workspace_bytes()
 * bytes, 256-byte aligned (about 56 bytes per value of the coarse block size per
 * resident thread, plus 4 bytes per value). */
uint64_t leco_varlen_partition_workspace_bytes(uint64_t n, uint32_t coarse_blocks);
int leco_varlen_partition_device(const uint64_t *d_values, uint64_t n, uint32_t coarse_blocks, int64_t delta,
                                 uint64_t *d_starts, uint64_t starts_cap, uint64_t *d_nseg, void *d_ws, uint64_t ws_bytes,
                                 leco_stream_t stream);
uint64_t leco_varlen_max_payload_bytes(uint64_t n, uint64_t nseg);
/* Device workspace of leco_varlen_encode: the look-back status words and ticket,
 * and for LECO_FIT_REFERENCE the segments' sequential fits (16 bytes a segment). */
uint64_t leco_varlen_workspace_bytes(uint64_t nseg);
/* Longest segment leco_varlen_encode accepts (values). */
uint64_t leco_varlen_max_segment(void);
/* Writes every segment image (newsegment / newsegment_1 / newsegment_2, :134-272) for the
 * given starts; LECO_FIT_REFERENCE gives the reference's bytes.  max_segment_len bounds the
 * longest segment (0 = leco_varlen_max_segment()); it sizes the per-segment staging. */
int leco_varlen_encode(const uint64_t *d_values, uint64_t n, const uint64_t *d_starts, uint64_t nseg,
                       uint32_t max_segment_len, int fit_mode,
                       uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets, void *d_workspace,
                       uint64_t workspace_bytes, leco_stream_t stream);
/* decodeArray8 over all segments (:573-626); a raw segment yields its own values.
 * d_out: 8-byte aligned. */
int leco_varlen_decode(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                       uint64_t n, uint64_t *d_out, leco_stream_t stream);
/* randomdecodeArray8 for each index (:636-698): binary search of the device start array. */
int leco_varlen_gather(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                       uint64_t n, const uint64_t *d_idx, uint64_t m, uint64_t *d_out, leco_stream_t stream);
/* Sum of all values mod 2^64 without materialising them. */
int leco_varlen_sum(const uint8_t *d_payload, const uint64_t *d_offsets, const uint64_t *d_starts, uint64_t nseg,
                    uint64_t n, uint64_t *d_sum, leco_stream_t stream);

/* ---- batch engine: many columns, one persistent launch per pass --------
 * No counterpart in the reference, whose drivers loop over the blocks of one
 * column (experiments/leco_int_fix_template.cpp:111-127, :145-153). */

typedef struct leco_column_desc {
  int32_t codec;       /* LINEAR, FOR, DELTA or POLY2                          */
  int32_t dtype;       /* LECO_U32 or LECO_U64                                 */
  uint32_t block_size; /* values per block, 1..16384                           */
  uint16_t group_threads; /* batch engine: threads per block, 32/64/128/256;
                             0 = 32 for blocks of <= 512 values, else 256       */
  uint16_t unroll;     /* batch engine: unroll depth 1/2/4 (0 = 2): the decoder
                          writes `unroll` 16-byte chunks per thread step, the u64
                          LeCo encoder keeps 2*unroll 16-byte loads in flight   */
  uint64_t n;          /* values in the column                                 */
  const void *d_values;/* encode input (n values)                              */
  void *d_out;         /* decode output (n values); may be NULL if never decoded */
  uint8_t *d_payload;  /* block images (leco_max_payload_bytes capacity)       */
  uint64_t payload_cap;
  uint64_t *d_offsets; /* nblocks + 1                                          */
  leco_dir_entry *d_dir; /* nblocks entries or NULL                            */
} leco_column_desc;

typedef struct leco_batch leco_batch; /* opaque */

/* Builds a batch over ncols column descriptors (copied).  Allocates the device
 * descriptor table and the batch workspace (the only allocations of the batch
 * engine); sizes the persistent grids so every CTA is resident.  A column's
 * work items hold 256/group_threads blocks, one per group of a 256-thread CTA;
 * an item's shared memory (enc_smem per block x blocks per item) must stay
 * within 200 KB, else LECO_ERR_ARG.  The committed autotune table gives
 * block_size, group_threads and unroll per column shape. */
int leco_batch_create(const leco_column_desc *h_cols, uint32_t ncols, int fit_mode, leco_batch **out);
int leco_batch_destroy(leco_batch *b);
uint64_t leco_batch_total_blocks(const leco_batch *b);
/* Encodes every block of every column with one persistent launch pulling
 * (column, block) items from an atomic work queue (plus the sequential-fit pass
 * for reference-fit columns that need it). */
int leco_batch_encode(leco_batch *b, leco_stream_t stream);
/* Decodes every column into its d_out (aligned to the column's value size) with one
 * persistent launch. */
int leco_batch_decode(leco_batch *b, leco_stream_t stream);
/* Captures the pass(es) (1 encode, 2 decode, 3 both) into a CUDA graph on the
 * first call and replays the graph on every call. */
int leco_batch_run_graph(leco_batch *b, int passes, leco_stream_t stream);
/* The same work as one leco_encode / leco_decode call per column (baseline). */
int leco_batch_encode_per_column(leco_batch *b, leco_stream_t stream);
int leco_batch_decode_per_column(leco_batch *b, leco_stream_t stream);

/* ---- serving: continuous batching of lookups and range scans -----------
 * No counterpart in the reference (its random access is a per-index CPU loop,
 * experiments/leco_int_fix_template.cpp:189-207).  Columns stay resident in HBM
 * (encoded with leco_encode / leco_batch_*); requests from any thread are
 * admitted by free device memory for their index and output buffers, coalesced
 * into one kernel launch per batch, and several batches overlap on the GPU. */

enum leco_request_kind { LECO_REQ_LOOKUP = 0, LECO_REQ_RANGE = 1 };

typedef struct leco_request {
  uint32_t column;       /* index into the server's columns                          */
  uint32_t kind;         /* LECO_REQ_LOOKUP or LECO_REQ_RANGE                         */
  uint64_t count;        /* lookups, or values in the range                           */
  const uint64_t *h_idx; /* LOOKUP: count indices (pinned host memory for async copy) */
  uint64_t first;        /* RANGE: first value                                        */
  void *h_out;           /* count results (pinned host memory for async copy)         */
} leco_request;

typedef struct leco_server_options {
  uint32_t slots;                  /* batches in flight (streams); 0 -> 4                  */
  uint32_t max_requests_per_batch; /* 0 -> 1024; 1 with slots = 1 = per-request launches   */
  uint32_t max_items_per_batch;    /* CTAs per batch launch; 0 -> 65536                    */
  uint32_t reserved;
  uint64_t hbm_budget_bytes;       /* device arena for indices + results; 0 -> 1/4 of free */
} leco_server_options;

typedef struct leco_server_stats {
  uint64_t completed, lookups, scanned_values, batches, max_requests_in_batch, arena_bytes;
  double p50_us, p99_us, mean_us, max_us; /* submit -> results in the client's buffer */
} leco_server_stats;

typedef struct leco_server leco_server; /* opaque */

/* Starts a server (one host thread) over encoded resident columns; allocates
 * its device arena and per-slot item tables. */
int leco_server_create(const leco_column_desc *h_cols, uint32_t ncols, const leco_server_options *opt, leco_server **out);
/* Queues a request (thread-safe, returns at once).  LECO_ERR_NOMEM if the request
 * could never fit the server's device budget. */
int leco_server_submit(leco_server *sv, const leco_request *req, uint64_t *req_id);
/* Blocks until the request's results are in its h_out; *latency_us = submit -> done. */
int leco_server_wait(leco_server *sv, uint64_t req_id, double *latency_us);
/* Blocks until every submitted request has completed. */
int leco_server_drain(leco_server *sv);
int leco_server_get_stats(leco_server *sv, leco_server_stats *out);
int leco_server_reset_stats(leco_server *sv);
int leco_server_destroy(leco_server *sv);

/* ---- host-buffer entry points (synchronous; allocate device memory) ----
 * These are the reference-facing calls: host in, host out, the same
 * arguments as the reference's per-column driver loops.  Their device memory
 * comes from a memory pool of this library, one per device, which keeps up to
 * 1 GiB mapped between calls (so repeated calls do not map their buffers
 * afresh) until the process ends. */

/* Encodes h_values[n]; writes payload bytes and offsets[nblocks+1] to host
 * buffers; *out_bytes = compressed size. */
int leco_encode_host(int codec, int dtype, const void *h_values, uint64_t n, uint32_t block_size, int fit_mode,
                     uint8_t *h_payload, uint64_t payload_cap, uint64_t *h_offsets, uint64_t *out_bytes);
/* Decodes a host column into h_out[n]; copies are pipelined with the kernels. */
int leco_decode_host(int codec, int dtype, const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t n,
                     uint32_t block_size, void *h_out);
/* Random access from host indices into host output. */
int leco_gather_host(int codec, int dtype, const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t n,
                     uint32_t block_size, const uint64_t *h_idx, uint64_t m, void *h_out);

/* ---- per-block drop-in (one reference block, host buffers) ------------
 * Byte-for-byte the reference methods' contracts; used by include/leco_codecs.hpp.
 * Synchronous.  Each calling thread keeps one stream, a device buffer and a pinned
 * host buffer (both grow to the largest block seen) for these calls, from its first
 * per-block call on a device until leco_thread_release() or the end of the process. */

/* <Codec>::encodeArray8_int(data, length, res, nvalue): returns bytes written
 * to h_out (which must hold leco_block_bytes(..., 8*dtype, length)), or a
 * negative status. */
int64_t leco_block_encode(int codec, int dtype, const void *h_values, uint32_t length, int fit_mode, uint8_t *h_out);
/* <Codec>::decodeArray8(in, length, out, nvalue). in_bytes = image size. */
int leco_block_decode(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length, void *h_out);
/* <Codec>::randomdecodeArray8(in, to_find, NULL, 0) into *h_value. */
int leco_block_random(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length,
                      uint32_t to_find, void *h_value);
/* Frees the calling thread's per-block stream and buffers (no counterpart in the
 * reference, whose per-block calls need no resources).  Call it before a thread
 * that made per-block calls exits, if the process goes on. */
int leco_thread_release(void);

/* Leco_int<T> / FOR_int<T>::filter_range(in, length, filter, out, block_id)
 * (close = 0; piecewise_fix_integer_template.h:206-252, FOR_integer_template.h:115-160) or
 * filter_range_close(in, length, out, block_id, filter1, filter2, base)
 * (close = 1; :254-303, :166-215) on one block image: indices block_start + k into h_out
 * (at most out_cap written).  Returns the count (which may exceed out_cap) or a negative
 * status.  block_start = block_id * block_size, as the reference computes it. */
int64_t leco_block_filter(int codec, int dtype, const uint8_t *h_in, uint64_t in_bytes, uint32_t length,
                          uint32_t block_start, int close, uint64_t filter1, uint64_t filter2, uint64_t base,
                          uint32_t *h_out, uint64_t out_cap);

/* ---- container file, import / export ------------------------------------
 * The reference has no file format: its drivers hold each block as a separate
 * malloc'ed byte string (experiments/leco_int_fix_template.cpp:108-127).  A column
 * container stores payload + offsets (+ segment starts) behind a 64-byte header
 * with a checksum; reading checks the header, the offsets, the checksum and every
 * block header before anything reaches a kernel (LECO_ERR_CORRUPT otherwise). */
typedef struct leco_container_info {
  int codec;            /* enum leco_codec                                   */
  int dtype;            /* LECO_U32 / LECO_U64                               */
  uint32_t block_size;  /* fixed-block codecs; 0 for variable-length          */
  uint64_t n;           /* values                                            */
  uint64_t nunits;      /* blocks or segments                                */
  uint64_t payload_bytes;
  int has_starts;       /* variable-length: segment starts stored            */
} leco_container_info;

/* Writes a column from host buffers (atomically: a temporary file renamed). */
int leco_container_write(const char *path, const leco_container_info *info, const uint8_t *h_payload,
                         const uint64_t *h_offsets, const uint64_t *h_starts);
/* Reads the header (and checks offsets/starts) without the payload. */
int leco_container_info_read(const char *path, leco_container_info *info);
/* Reads a column into host buffers (payload_cap >= payload_bytes). */
int leco_container_read(const char *path, uint8_t *h_payload, uint64_t payload_cap, uint64_t *h_offsets,
                        uint64_t *h_starts);
/* Device-buffer forms (synchronous; staged through host memory).  load: payload_cap >=
 * payload_bytes + LECO_PAYLOAD_SLACK (the slack is zero-filled). */
int leco_container_save_device(const char *path, const leco_container_info *info, const uint8_t *d_payload,
                               const uint64_t *d_offsets, const uint64_t *d_starts, leco_stream_t stream);
int leco_container_load_device(const char *path, uint8_t *d_payload, uint64_t payload_cap, uint64_t *d_offsets,
                               uint64_t *d_starts, leco_stream_t stream);
/* The reference drivers' per-block byte strings (block_start_vec[i], sizes) <-> a
 * column's payload + offsets, byte for byte.  export: h_blocks may be NULL to get the
 * sizes only; otherwise each h_blocks[i] must hold h_sizes[i] bytes. */
int leco_import_blocks(const uint8_t *const *h_blocks, const uint64_t *h_sizes, uint64_t nblocks, uint8_t *h_payload,
                       uint64_t payload_cap, uint64_t *h_offsets);
int leco_export_blocks(const uint8_t *h_payload, const uint64_t *h_offsets, uint64_t nblocks, uint8_t *const *h_blocks,
                       uint64_t *h_sizes);

/* ---- validation / errors ------------------------------------------------ */

/* Host-side validation of an imported column before any launch: offsets
 * monotone and within payload_bytes, each header's l legal for the codec and
 * each image size equal to leco_block_bytes(). Returns LECO_OK or
 * LECO_ERR_CORRUPT (first bad block in *bad_block). */
int leco_validate_host(int codec, int dtype, const uint8_t *h_payload, uint64_t payload_bytes,
                       const uint64_t *h_offsets, uint64_t n, uint32_t block_size, uint64_t *bad_block);
/* Reads and clears the device error word (bad index, bad header, bounded-wait
 * timeout). Synchronous. Returns LECO_OK, LECO_ERR_CORRUPT or LECO_ERR_TIMEOUT. */
int leco_check(leco_stream_t stream);
/* TEST HOOK, not part of the codec interface (no counterpart in the reference):
 * the failure-detection test calls it; applications have no use for it.
 * Runs the encoder's look-back wait on a predecessor that never publishes, with
 * at most spin_limit polls (the encoder itself uses about 4 million, ~1-2 s), and
 * returns what leco_check reports afterwards: LECO_ERR_TIMEOUT when the bounded
 * wait gave up as designed (*h_result = ~0).  Synchronous; the context stays usable. */
int leco_test_bounded_wait(uint32_t spin_limit, uint64_t *h_result);
/* Message of the last error on this thread ("" if none). */
const char *leco_last_error(void);
/* Library version string. */
const char *leco_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LECO_B200_H_ */
