/*
 * gpusw_b200.h -- C ABI of the B200 Gotoh scoring engine (libgpusw_sm100.so).
 *
 * Plain C types only: pointers, sizes and int status codes. No exception crosses the ABI;
 * every call returns GPUSW_OK (0) or an error code, and gpusw_last_error() gives the
 * message. A context owns one CUDA stream on one device plus every device buffer it
 * allocates; calls on one context must be serialised by the caller (one context per host
 * thread, or a lock around it). Host buffers passed in or out belong to the caller.
 *
 * Each entry point names the interface of the reference package (freiburgermsu/gpuSW,
 * Python) that it replaces. The package's Python side binds these symbols with ctypes
 * (gpusw_b200/_native.py).
 */
#ifndef GPUSW_B200_H
#define GPUSW_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The Python layer maps them onto the reference's exception classes
 * (src/gpusw/errors.py:5-31): INVALID -> ValueError, NO_GPU -> NoGpuError,
 * SCHEME -> SchemeError, OVERFLOW -> OverflowRiskError, the rest -> GpuSWError. */
#define GPUSW_OK 0
#define GPUSW_ERR_INVALID 1      /* bad argument: null pointer, index out of range, ... */
#define GPUSW_ERR_NO_GPU 2       /* no CUDA device / driver */
#define GPUSW_ERR_CUDA 3         /* a CUDA call failed */
#define GPUSW_ERR_MEMORY 4       /* device memory budget exceeded / allocation failed */
#define GPUSW_ERR_OVERFLOW 5     /* scores cannot be represented even in int32 */
#define GPUSW_ERR_SCHEME 6       /* no scheme set, or scheme values out of range */
#define GPUSW_ERR_QUEUE_FULL 7   /* serving: admission refused (no slot / memory) */
#define GPUSW_ERR_NOT_FOUND 8    /* unknown handle or request id */
#define GPUSW_ERR_CANCELLED 9    /* serving: the request was cancelled */
#define GPUSW_ERR_TIMEOUT 10     /* a bounded wait ran out */
#define GPUSW_ERR_UNSUPPORTED 11 /* input this routine does not take (the caller uses its own) */

/* Alignment modes (src/gpusw/scheme.py:19, MODES). */
#define GPUSW_MODE_LOCAL 0
#define GPUSW_MODE_GLOBAL 1
#define GPUSW_MODE_SEMIGLOBAL 2

/* Integer width policy (src/gpusw/scheme.py:116-141, Scheme.resolve_dtype).
 * AUTO: every pair in int16 (two alignments per 32-bit register); pairs whose int16 run
 * may have overflowed are rescored in int32 -- the integers equal an all-int32 run.
 * INT16: same kernels; the caller has already checked the static envelope.
 * INT32: every pair in int32. */
#define GPUSW_DTYPE_AUTO 0
#define GPUSW_DTYPE_INT16 1
#define GPUSW_DTYPE_INT32 2

typedef struct gpusw_ctx gpusw_ctx;

/* Counters of the last call and of the context's lifetime. Times come from CUDA events
 * recorded on the context's stream. */
typedef struct gpusw_stats {
  double last_kernel_ms;      /* scoring + rescoring + top-k kernels of the last call */
  double last_score_ms;       /* scoring + int32 rescoring kernels only */
  double last_topk_ms;        /* top-k kernels only */
  double last_total_ms;       /* the last call's device work including its copies */
  double last_cells;          /* DP cells of the last call (sum of |q| * |r|) */
  int64_t last_pairs;         /* alignments scored by the last call */
  int64_t last_overflow;      /* int16 cells rescored in int32 by the last call */
  int64_t last_launches;      /* kernels launched by the last call */
  int64_t total_launches;     /* kernels launched by this context */
  int64_t total_overflow;     /* int16 rescores over the context's lifetime */
  int64_t device_bytes;       /* device memory currently held by the context */
  int64_t last_inter_items;   /* threads' items (one or two alignments) of the last call that
                                 the inter-sequence pairs kernel scored */
} gpusw_stats;

/* Library version (major * 10000 + minor * 100 + patch). */
int gpusw_version(void);

/* Number of visible CUDA devices (0 when there is no driver/GPU; never an error).
 * Replaces src/gpusw/_compile.py:39-46 (gpu_available). */
int gpusw_device_count(int *count);

/* Create / destroy a context on `device`. Replaces the device binding of
 * src/gpusw/backends/cuda.py:30-35 (device_scope). */
int gpusw_ctx_create(int device, gpusw_ctx **out);
void gpusw_ctx_destroy(gpusw_ctx *ctx);

/* Message of the last failed call on `ctx` (or of the last failed gpusw_ctx_create when
 * ctx is NULL). Valid until the next call on the context. */
const char *gpusw_last_error(const gpusw_ctx *ctx);

/* Set the scoring scheme: mode, gap open/extend (<= 0), semiglobal free-end flags, and the
 * (ns x ns) int32 substitution table, row = reference code, column = query code, last
 * row/column = sentinel. Replaces src/gpusw/_compile.py:55-93 (get_module: the baked
 * MODE/GOPEN/GEXT/FREE_Q/FREE_R/NS, and get_sub: the SUB upload). */
int gpusw_set_scheme(gpusw_ctx *ctx, int mode, int gap_open, int gap_extend, int free_q,
                     int free_r, int ns, const int32_t *sub);

/* Upload one encoded sequence set (codes in [0, ns), offsets[n + 1], int32 like the
 * reference's Encoded). The library packs it (2, 4, 5 or 8 bits per residue, picked from
 * the largest code) and keeps it resident; *out_db receives the handle. Replaces
 * src/gpusw/backends/__init__.py:57-59 (Backend.upload of codes and offsets). */
int gpusw_db_upload(gpusw_ctx *ctx, const uint8_t *codes, const int32_t *offsets, int32_t n,
                    int32_t *out_db);

/* Packed image of an encoded set, for storing it (host only, no GPU): the exact byte
 * layout gpusw_db_upload sends to the device -- packed words (every sequence 16-byte
 * aligned, then 64 zero slack words) | int64 word offsets | int32 lengths, each part on a
 * 256-byte boundary. With image == NULL only *out_need (bytes), *out_bits and *out_nwords
 * (packed words without the slack) are set; otherwise image_bytes must be at least
 * *out_need. Errors set gpusw_last_error(NULL). Replaces the per-process re-encoding of a
 * reference set (src/gpusw/aligner.py:69-77, src/gpusw/encode.py:204-215): a set packed
 * once is stored and uploaded as is by gpusw_db_upload_image. */
int gpusw_pack_image(const uint8_t *codes, const int32_t *offsets, int32_t n, void *image,
                     int64_t image_bytes, int64_t *out_need, int32_t *out_bits,
                     int64_t *out_nwords);

/* Upload a packed image made by gpusw_pack_image (n sequences, `bits` per residue,
 * nwords packed words) without packing it again. The image is checked before it is used:
 * its size, word offsets and lengths must agree, and its largest stored code is found
 * (and checked against the scheme at scoring time, as for gpusw_db_upload). Same handle
 * semantics as gpusw_db_upload. */
int gpusw_db_upload_image(gpusw_ctx *ctx, const void *image, int64_t image_bytes, int32_t n,
                          int32_t bits, int64_t nwords, int32_t *out_db);

/* Release a sequence set. */
int gpusw_db_free(gpusw_ctx *ctx, int32_t db);

/* Bits per residue the set was packed with, or a negative status. */
int gpusw_db_bits(gpusw_ctx *ctx, int32_t db);

/* Cross product: out[a * n_refs + b] = score(query qlist[a] of qdb, reference b of rdb),
 * int32, host buffer of nq * n_refs. Replaces src/gpusw/backends/cuda.py:47-66 (run_cross)
 * and :87-91 (as_host), kernel sw_cross of src/gpusw/kernel.py:161-175. */
int gpusw_score_cross(gpusw_ctx *ctx, int32_t qdb, int32_t rdb, const int32_t *qlist,
                      int32_t nq, int dtype, int32_t *out);

/* Per-query top-k: out_idx/out_score are host (nq, min(k, n_refs)) int32, best first,
 * ties broken by the lower reference index (the order of a stable sort of -scores).
 * Queries are scored in blocks that keep the score block within the context's memory
 * budget. Replaces src/gpusw/aligner.py:169-195 (Aligner.top_k) together with
 * src/gpusw/backends/cuda.py:93-106 (Backend.topk). */
int gpusw_topk(gpusw_ctx *ctx, int32_t qdb, int32_t rdb, const int32_t *qlist, int32_t nq,
               int32_t k, int dtype, int32_t *out_idx, int32_t *out_score);

/* Explicit pairs: out[i] = score(query qi[i] of qdb, reference rj[i] of rdb). Indices are
 * validated before any launch (GPUSW_ERR_INVALID on an out-of-range index). Replaces
 * src/gpusw/backends/cuda.py:68-85 (run_pairs), kernel sw_pairs of
 * src/gpusw/kernel.py:178-190. */
int gpusw_score_pairs(gpusw_ctx *ctx, int32_t qdb, int32_t rdb, const int32_t *qi,
                      const int32_t *rj, int64_t n, int dtype, int32_t *out);

/* Zipped pairs from host buffers in one call: out[i] = score(query i, reference i) for
 * i < n, with query i at q_codes[q_offsets[i] .. q_offsets[i + 1]) and reference i at
 * r_codes[r_offsets[i] .. r_offsets[i + 1]) (code bytes, int32 offsets of n + 1 entries,
 * the reference package's Encoded layout). Equal to gpusw_db_upload of both sets followed
 * by gpusw_score_pairs with qi = rj = 0..n-1, but pipelined: chunks of 131,072 pairs are
 * packed on the host while the GPU scores the previous chunk, on two streams, so host
 * packing, copies and kernels overlap; nothing stays resident after the call. Replaces
 * src/gpusw/__init__.py:145-189 (align_pairs with pairs=None) with its
 * src/gpusw/aligner.py:69-87 uploads and src/gpusw/backends/cuda.py:68-85 (run_pairs).
 * On an error (decreasing offsets, a code >= the scheme's table side) out[] is
 * unspecified. */
int gpusw_score_pairs_zip(gpusw_ctx *ctx, const uint8_t *q_codes, const int32_t *q_offsets,
                          const uint8_t *r_codes, const int32_t *r_offsets, int64_t n,
                          int dtype, int32_t *out);

/* Best-cell coordinates of explicit pairs (int32): for every pair, out_score receives the
 * maximum of H over all cells and out_rend/out_qend the 0-based reference row and query
 * column of the first cell holding it in row-major order (reference row, then query
 * column), or -1 when no cell scores above 0 in local mode. anchored = 0 runs the context's
 * local scheme (the end of the best local alignment; out_score is then the local score);
 * anchored = 1 runs the same table and gaps with both sequences anchored at their start
 * (global boundaries, best cell anywhere) -- on reversed prefixes this gives the start of an
 * optimal local alignment ending at a known cell. Replaces the CPU re-alignment the
 * reference's examples use to recover coordinates (examples/legacy_16s_gpu_align.py:280-292,
 * docs/DESIGN.md:95-96); the reference itself is score-only. */
int gpusw_locate_pairs(gpusw_ctx *ctx, int32_t qdb, int32_t rdb, const int32_t *qi,
                       const int32_t *rj, int64_t n, int anchored, int32_t *out_score,
                       int32_t *out_rend, int32_t *out_qend);

/* Engine options. plain != 0 selects the one-batch-per-call form (queries in input order,
 * one kernel shape per batch, no length binning, no graph) used as the comparison point
 * of the batched form. mem_budget bounds the score blocks of gpusw_topk (bytes, 0 keeps the
 * default of 4 GiB). flags: GPUSW_OPT_NO_AUTOTUNE keeps the modelled kernel-shape costs,
 * GPUSW_OPT_NO_GRAPHS runs every call eagerly instead of replaying cached CUDA graphs,
 * GPUSW_OPT_ONE_LAUNCH scores a local-mode cross product of several streaming-kernel shapes
 * in one persistent launch over every shape's work items (costliest first) instead of one
 * launch per shape on up to four streams (the default: on the uneven-length protein top-10
 * the single launch measured 7 % slower, its registers being the most any shape needs),
 * GPUSW_OPT_NO_INTER keeps every explicit pair on the team kernels (by default, int16 pairs
 * of queries up to 160 residues or of 193 to 224 go to the inter-sequence kernel, one thread
 * per two alignments, when the query set holds only codes 0..3, the scheme's values fit a
 * byte and the call has enough of them to keep every thread busy). */
#define GPUSW_OPT_NO_AUTOTUNE 1
#define GPUSW_OPT_NO_GRAPHS 2
#define GPUSW_OPT_ONE_LAUNCH 4
#define GPUSW_OPT_NO_INTER 8
int gpusw_set_options(gpusw_ctx *ctx, int plain, int64_t mem_budget, int flags);

/* Autotune the streaming cross-product kernel for the current scheme: every compiled
 * shape (team size G x columns per lane W) is timed once on synthetic full-width
 * columns (256 queries) against 4,096 synthetic 300-residue references, enough work
 * items to fill the GPU for every shape; the measured device time per (column pair,
 * reference, column pass) replaces the modelled cost when the planner bins queries by
 * length, so the bin edges are the crossover points of the measured costs. Tables are
 * kept per (alphabet size, int width) in the context; calls run it on first use unless
 * gpusw_set_options disabled it. us_per_row_pass (may be NULL) receives up to n entries
 * (microseconds, one per shape). No reference counterpart. */
int gpusw_autotune(gpusw_ctx *ctx, int width, double *us_per_row_pass, int32_t n);

/* Read (get) or install (set) the autotuner table of the current scheme's alphabet size
 * and `width` (1 = int32, 2 = int16x2), so that a caller can keep tables across processes.
 * get returns the number of entries copied (0 when the context has no table yet, negative
 * status on error); set replaces the table and drops cached plans. No reference
 * counterpart. */
int gpusw_get_tune(gpusw_ctx *ctx, int width, double *us_per_row_pass, int32_t n);
int gpusw_set_tune(gpusw_ctx *ctx, int width, const double *us_per_row_pass, int32_t n);

/* Name of CUDA device `device` (for cache keys); returns a status. */
int gpusw_device_name(int device, char *buf, int32_t len);

/* Counters (see gpusw_stats). Replaces src/gpusw/aligner.py:212 (Aligner.gcups): GCUPS =
 * last_cells / last_kernel_ms / 1e6. */
int gpusw_get_stats(gpusw_ctx *ctx, gpusw_stats *out);

/* Block until the context's stream is idle. */
int gpusw_sync(gpusw_ctx *ctx);

/* Sustained int16x2 add-max (DPX) instruction rate of the device, measured by a short
 * self-timed kernel: *ops_per_s lane-operations per second. The denominator of the
 * scoring kernels' instruction roofline. No reference counterpart (measurement only). */
int gpusw_measure_dpx_rate(gpusw_ctx *ctx, double *ops_per_s);

/* Write `bytes` of zeros into a scratch buffer on the context's stream (evicts the L2
 * between timed steps of a benchmark). No reference counterpart (measurement only). */
int gpusw_flush_l2(gpusw_ctx *ctx, int64_t bytes);

/* Explicit pairs scored without any allocation by the library, for callers that own all
 * device memory and cannot let a library call cudaMalloc: code running inside a framework's
 * caching allocator or a fixed arena sized at start-up, plugin hosts that forbid allocation
 * in their callbacks, or latency-bound loops that cannot pay the device-wide
 * synchronisation a cudaFree implies. No counterpart in the reference (which allocates
 * through CuPy on every call).
 *
 * Inputs and output are the caller's device memory, in the reference's own encoding: code
 * bytes with int32 offsets (n_seq + 1) for the queries and the references, int32 pair
 * indices qi/rj[n], int32 out[n] (out[i] = score of query qi[i] vs reference rj[i]). The
 * substitution table `sub` (ns x ns int32, row = reference code) is a host array.
 * max_len must bound every sequence length. Scores are computed in int32 and equal
 * gpusw_score_pairs. The kernel's scratch (work counter, error word, table, multi-pass
 * boundary strips) lives in a 32 MiB file-scope device array that every GPU loading this
 * library holds until exit; sizes beyond it are rejected (GPUSW_ERR_MEMORY): ns <= 64, and
 * with max_len above 256 the strips need max_len x 8 bytes per team (about 260,000
 * residues at most). The first call on a device looks up the array's device address with
 * that device current; make that first call before any stream capture. Every call shares
 * the array and resets its counter and error word; calls that overlap on the GPU (on
 * different streams or threads) race on it and must be serialised by the caller. Runs on
 * `stream` (a cudaStream_t, NULL for the legacy default stream) and returns after the
 * stream is idle. Bad indices, lengths above max_len, decreasing offsets and codes >= ns
 * are found on the device before any code is used, the pair is skipped (its out[] entry
 * left as it was) and the call returns GPUSW_ERR_INVALID. Offsets must lie inside the
 * caller's code buffers (their sizes are not passed, so they cannot be checked). The
 * shared-memory limit of the kernel is raised once per device, so the first call on each
 * GPU makes that setting too. Messages go to errbuf (errlen bytes, may be NULL). */
int gpusw_score_pairs_noalloc(const uint8_t *q_codes, const int32_t *q_offsets, int32_t nq,
                              const uint8_t *r_codes, const int32_t *r_offsets, int32_t nr,
                              const int32_t *qi, const int32_t *rj, int32_t n, int mode,
                              int gap_open, int gap_extend, int free_q, int free_r, int ns,
                              const int32_t *sub, int32_t max_len, int32_t *out, void *stream,
                              char *errbuf, int32_t errlen);

/* ---------------------------------------------------------------------------------
 * Serving: continuous batching over a resident reference set.
 *
 * A server keeps the reference set `rdb` of `ctx` resident and answers top-k requests.
 * A scheduler thread admits pending requests in arrival order while a slot (an execution
 * stream) and the device-memory budget allow, merges the admitted requests into one batch
 * (up to max_batch_queries queries), and launches the batch asynchronously; batches on
 * different slots overlap on the device. Each request's top-k equals what gpusw_topk
 * returns for its queries alone. `ctx` must not be used for other calls while its server
 * exists. No reference counterpart (the reference has no serving layer); this is the
 * serving pattern of the scoring path.
 * --------------------------------------------------------------------------------- */
typedef struct gpusw_server gpusw_server;

#define GPUSW_REQ_PENDING 0
#define GPUSW_REQ_RUNNING 1
#define GPUSW_REQ_DONE 2
#define GPUSW_REQ_CANCELLED 3

typedef struct gpusw_server_stats {
  int64_t submitted, completed, cancelled, rejected;
  int64_t pending, running;      /* requests waiting / on the device now */
  int64_t batches;               /* launched batches */
  double mean_batch_queries;
  double p50_ms, p99_ms, mean_ms, max_ms;  /* submit -> done latency of completed requests */
  double cells;                  /* DP cells of completed requests */
  double wall_s;                 /* seconds since the first submit */
  double gcups;                  /* cells / wall_s / 1e9 */
  int64_t device_bytes;          /* device memory held by the server's slots */
} gpusw_server_stats;

/* Create a server over reference set `rdb` of `ctx` (scheme as set on ctx at this time).
 * mem_budget bounds the device memory of in-flight batches (0: 4 GiB); max_slots (1-8)
 * bounds concurrent batches; max_pending bounds queued requests (submit then returns
 * GPUSW_ERR_QUEUE_FULL). */
int gpusw_server_create(gpusw_ctx *ctx, int32_t rdb, int32_t k, int dtype, int64_t mem_budget,
                        int32_t max_slots, int32_t max_batch_queries, int32_t max_pending,
                        gpusw_server **out);

/* Queue one request of nq encoded queries (codes/offsets as for gpusw_db_upload; copied,
 * the caller may free them on return). *req_id receives its id. */
int gpusw_server_submit(gpusw_server *srv, const uint8_t *codes, const int32_t *offsets,
                        int32_t nq, int64_t *req_id);

/* State of a request. When it is done, its (nq, min(k, n_refs)) top-k is copied into
 * out_idx/out_score (may be NULL to discard) and the request is released; a cancelled
 * request is released as well. Waits at most timeout_ms (0: no wait) for completion;
 * GPUSW_ERR_NOT_FOUND for unknown or already released ids. */
int gpusw_server_poll(gpusw_server *srv, int64_t req_id, int32_t timeout_ms, int32_t *state,
                      int32_t *out_idx, int32_t *out_score);

/* Cancel a request: a pending one is dropped at once, a running one has its results
 * discarded when its batch finishes. */
int gpusw_server_cancel(gpusw_server *srv, int64_t req_id);

int gpusw_server_get_stats(gpusw_server *srv, gpusw_server_stats *out);

/* Message of the last failed call on the server. */
const char *gpusw_server_last_error(const gpusw_server *srv);

/* Stop the scheduler (waiting at most for the in-flight batches) and free the server. */
void gpusw_server_destroy(gpusw_server *srv);
/* Least work per batch in DP cells (0: the default, 3e12, about half a second on one B200).
 * Batches are cut by work, not by request: a batch takes this much, or an equal share per
 * slot of all the queued work when that is larger; a request above it runs as several
 * parts, and while others wait no request takes more than half of a batch, so small
 * requests queued behind a large one share the next batch. Smaller values lower latency at
 * light load; under a backlog batches grow anyway. No reference counterpart (the reference
 * has no server). */
int gpusw_server_set_batch_cells(gpusw_server *srv, double cells);

/* ------------------------------------------------------------------ FASTA (host only)
 * Native reader and encoder for FASTA text, replacing the reference's Python reader and
 * per-sequence encoding loop (src/gpusw/encode.py:89-120, :196-225) with one pass over
 * the bytes; no CUDA call, so it also runs without a GPU. `lut` is the scheme's 256-entry
 * code table (case folding included) and `sentinel` its out-of-alphabet code; with
 * unknown_error != 0 the first byte mapping to the sentinel fails the parse with
 * GPUSW_ERR_INVALID, and gpusw_fasta_bad_record / _bad_byte name it. Text with a byte
 * >= 0x80 or one of \v \f \x1c-\x1f returns GPUSW_ERR_UNSUPPORTED (the caller's Unicode
 * reader handles it). On any return *out, when set, must be freed with gpusw_fasta_free. */
typedef struct gpusw_fasta gpusw_fasta;
int gpusw_fasta_parse(const char *data, int64_t len, const uint8_t *lut, int32_t sentinel,
                      int unknown_error, gpusw_fasta **out);
int32_t gpusw_fasta_count(const gpusw_fasta *f);            /* records */
int64_t gpusw_fasta_residues(const gpusw_fasta *f);         /* total codes */
const uint8_t *gpusw_fasta_codes(const gpusw_fasta *f);     /* residues codes */
const int32_t *gpusw_fasta_offsets(const gpusw_fasta *f);   /* count + 1 offsets */
const char *gpusw_fasta_ids(const gpusw_fasta *f);          /* ids, concatenated */
const int64_t *gpusw_fasta_id_offsets(const gpusw_fasta *f); /* count + 1 offsets into ids */
const char *gpusw_fasta_error(const gpusw_fasta *f);
int64_t gpusw_fasta_bad_record(const gpusw_fasta *f);
int32_t gpusw_fasta_bad_byte(const gpusw_fasta *f);
void gpusw_fasta_free(gpusw_fasta *f);

#ifdef __cplusplus
}
#endif

#endif /* GPUSW_B200_H */
