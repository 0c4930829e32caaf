/* crystal_b200.h -- C ABI of the B200 execution layer for crystal-sycl's fused
 * star-join query pipeline (fact scan -> predicate -> dimension perfect-hash
 * build/probe -> group-by aggregate).
 *
 * Every entry point is plain C: pointers, sizes and int status codes; no C++
 * types and no exceptions cross it.  Functions return CX_OK (0) on success or a
 * negative CX_E_* code; cx_last_error() then describes the failure (per thread).
 *
 * The reference hands generated source to ICompiler::compile and the resulting
 * library to IExecutor::execute (include/core/execution.h:291-301), both behind
 * QueryEngine::executeQuery (src/core/execution.cpp:652-725).  The functions
 * below replace that pair: cx_compile stands where AdaptiveCppCompiler::compile
 * shelled out to `acpp` (src/core/execution.cpp:114-151), and cx_execute stands
 * where DynamicLibraryExecutor::execute dlopen()ed the library and called its
 * `execute_query(ExecutionContext*)` (src/core/execution.cpp:161-192).  The
 * execution context mirrors db::ExecutionContext's named buffers
 * (include/core/execution.h:131-282).
 */
#ifndef CRYSTAL_B200_H
#define CRYSTAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CX_ABI_VERSION 1

enum {
  CX_OK = 0,
  CX_E_INVALID = -1,     /* bad argument or plan */
  CX_E_COMPILE = -2,     /* NVRTC rejected the source (log filled) */
  CX_E_CUDA = -3,        /* a CUDA runtime/driver call failed */
  CX_E_MISSING = -4,     /* a buffer the query binds is not in the context */
  CX_E_CAPACITY = -5,    /* a caller buffer or the memory budget is too small */
  CX_E_KERNEL = -6,      /* a kernel raised an error code (see cx_ctx_kernel_error) */
  CX_E_NO_DEVICE = -7,   /* no CUDA device */
  CX_E_REJECTED = -8,    /* admission control refused a request */
  CX_E_PENDING = -9      /* a request has not finished within the wait */
};

typedef struct cx_module cx_module;     /* compiled query: cubin + launch plan */
typedef struct cx_exec_ctx cx_exec_ctx; /* named device buffers + scratch + timing */

/* Launch shape for generated scan kernels (the autotuner's search space). */
typedef struct cx_tuning {
  int block_threads;     /* BLOCK_THREADS, multiple of 32 (default 1024) */
  int items_per_thread;  /* ITEMS_PER_THREAD (default 4) */
  int stages;            /* TMA staging depth; 0 = read fact columns directly (default) */
  int ctas_per_sm;       /* persistent CTAs per SM, capped by occupancy (default 16) */
  int group_placement;   /* 0 auto, 1 shared-memory group tables, 2 global atomics, 3 register
                          * accumulators (tiny domains), 4 per-thread shared-memory accumulators
                          * (tiny domains; auto picks them when they fit the group budget) */
  int smem_group_budget; /* bytes a shared-memory group table may use */
  int bitmap_budget;     /* bytes of shared memory for exact join membership bitmaps (0 = none;
                            default 48 KiB) */
  int group_merge;       /* 0 auto, 1 merge equal groups within a warp first (for a plan with one
                            OR / multi-value join: a warp-uniform expansion loop), 2 per-lane
                            atomics, 3 shared scans: per-row atomics above 32 groups only */
  int producer_warps;    /* shared scans: warps that build query masks (0 = 3/8 of the block) */
  int parametric;        /* plain kernels: 1 = integer literals become launch parameters
                            (one module per plan shape, literals passed to cx_execute_params) */
  int prefetch;          /* unstaged plain scans (stages = 0): 0 = each column loaded where the
                            pipeline first reads it, 1 = vector loads of every column at the tile
                            start (default), 2 = as 1 with the next tile's loads issued a tile
                            ahead, 3 = as 1 with the warp's next tile prefetched into L2 (one
                            bulk prefetch per column, no registers held) */
  int wait_limit_us;     /* every wait of a kernel on an mbarrier gives up after this many
                            microseconds (global timer) and raises kernel error 1 (CX_E_KERNEL
                            from cx_ctx_sync); default 500000, range 1 .. 60000000 */
  int debug_stall;       /* test hook for the bounded-wait path: 1 = every CTA of the scan first
                            waits on a barrier that nothing completes, so the wait runs out
                            (kernel error 1) with no copy in flight; 0 in normal use */
  int compact;           /* plain grouped scans without expanding joins, unstaged vector loads:
                            1 = each warp queues the rows that pass the join bitmaps and fact
                            filters (ballot / popc into shared memory) and runs payload fetches,
                            remaining probes and the group update on 32 queued rows at a time;
                            2 = the same on 64 queued rows at a time (two rows per lane, their
                            gathers in flight together, half as many drains) */
  int table_budget;      /* bytes of shared memory for payload tables (default 0 = none; the
                            autotuner tries 96 KiB): a join whose payload's catalog range has at
                            most 254 values keeps one byte per hash slot -- membership and payload
                            together -- instead of a membership bitmap and a payload load from the
                            hash table */
  int cube;              /* shared scans: 0 = answer every query from per-query row masks; 1, 2 or
                            4 (default 4) = the program also carries the aggregate-cube path, which
                            cx_shared_execute takes when every column the batch's predicates and
                            GROUP BY keys read has a registered range (cx_ctx_set_column_range) of
                            at most 65,536 values and each shape's cube has at most 16,777,216
                            cells: one pass adds every fact row into one cell per plan shape, then
                            each query sums the cells its predicates accept (the value is the
                            cube scan's rows per lane) */
} cx_tuning;

/* Shape of a compiled query's result buffer. */
typedef struct cx_result_info {
  uint64_t groups;          /* perfect-hash group slots (1 for scalar aggregates) */
  uint32_t storage_ts;      /* u64 slots per group while aggregating */
  uint32_t visible_ts;      /* u64 slots per group after finalisation */
  uint64_t result_words;    /* u64 words the caller's result buffer must hold */
  uint64_t validity_words;  /* u64 words of the result validity bitmap */
  uint64_t final_words;     /* u64 words of the final result (groups x ts) */
  int sparse;               /* 1 = fast sparse output (no validity bits set) */
  int finalized;            /* 1 = AVG finalisation compacts to visible_ts */
} cx_result_info;

/* Timing of the last cx_execute on a context (CUDA events, ms). */
typedef struct cx_timing {
  float build_ms;  /* memsets + hash-table build kernels */
  float scan_ms;   /* fused scan/probe/aggregate kernel */
  float post_ms;   /* epilogue / finalisation kernels */
  float total_ms;  /* whole execute */
  int scan_grid;   /* CTAs of the scan launch */
  int gpu_launches;/* kernels launched by the last execute */
  int graph;       /* shared scans: 0 launched directly, 1 replayed a cached graph, 2 captured a new one */
  int mode;        /* shared scans: 0 per-query row masks, 1 aggregate cubes */
} cx_timing;

int cx_abi_version(void);
const char* cx_last_error(void);

/* Default tuning (filled in place). */
void cx_tuning_default(cx_tuning* t);

/* Generates the CUDA C++ source of a star-join plan (S-expression text; see
 * the package's plan builder).  Replaces JITOperatorVisitor::generateCode
 * (src/core/visitor.cpp:4771-4878) for this path.  Writes at most out_cap bytes
 * (NUL-terminated) and the full length to *out_len; call with out=NULL to size. */
int cx_codegen(const char* plan, size_t plan_len, const cx_tuning* tuning, char* out, size_t out_cap,
               size_t* out_len);

/* Rewrites a program emitted by the reference's code generator
 * (JITOperatorVisitor::generateCode, src/core/visitor.cpp:4771-4878: SYCL, an
 * `execute_query(db::ExecutionContext*)` that submits nd_range build and scan
 * kernels) into this library's CUDA skeleton: the kernel bodies are kept, the
 * launch skeleton becomes `__global__` kernels over one argument block plus the
 * embedded launch plan, and the row-count macros (LO_LEN, C_LEN, ...) become the
 * context's table rows.  cx_compile applies it by itself to such sources, so
 * the reference's ICompiler::compile can pass the visitor's text unchanged.
 * Programs that need the host between kernels (dense result materialisation,
 * multi-value hash tables, projections, ORDER BY) return CX_E_INVALID naming
 * the construct.  Same output-buffer contract as cx_codegen. */
int cx_translate_visitor(const char* src, size_t src_len, char* out, size_t out_cap, size_t* out_len);

/* Compiles generated source with NVRTC for sm_100a into an in-memory cubin and
 * parses its embedded launch plan.  `key` names the module in the process-wide
 * cache (the reference keys its cache on "query_" + ABI version + hash(sql),
 * src/core/execution.cpp:696-697); a hit returns the cached module with its
 * reference count raised.  On CX_E_COMPILE the NVRTC log goes to `log`.
 * Replaces ICompiler::compile / AdaptiveCppCompiler::compile. */
int cx_compile(const char* src, size_t src_len, const char* key, cx_module** out, char* log, size_t log_cap);

/* Drops one reference; the cubin is unloaded when the last one goes. */
int cx_module_release(cx_module* m);

int cx_module_result_info(const cx_module* m, cx_result_info* info);

/* Execution context: db::ExecutionContext's buffer registry. */
cx_exec_ctx* cx_ctx_create(void);
void cx_ctx_destroy(cx_exec_ctx* c);
/* Registers a device column as "d_<column>" (ctx->buffers_, execution.h:137). */
int cx_ctx_set_buffer(cx_exec_ctx* c, const char* name, const void* dev_ptr, uint64_t elems);
/* Registers a column's validity words (bit r = row r valid; ctx->null_bitmaps_). */
int cx_ctx_set_null_bitmap(cx_exec_ctx* c, const char* name, const uint64_t* dev_words, uint64_t words);
/* Row count of a table (the reference bakes these in as LO_LEN, C_LEN ...). */
int cx_ctx_set_table_rows(cx_exec_ctx* c, const char* table, uint64_t rows);
/* Caller-owned result and validity buffers (ctx->result_buffer_ /
 * result_validity_buffer_); sizes in u64 words. */
int cx_ctx_set_result(cx_exec_ctx* c, uint64_t* dev_result, uint64_t result_words, uint64_t* dev_validity,
                      uint64_t validity_words);
/* Optional caller-owned scratch for hash tables and group bitmaps.  Without it
 * the context allocates grow-only scratch itself (the reference's
 * getScratchIntBuffer high-water reuse, execution.h:186-207). */
int cx_ctx_set_scratch(cx_exec_ctx* c, void* dev_ptr, uint64_t bytes);
/* Bytes of scratch `m` needs under the context's current table sizes.  A
 * multi-value hash join adds 4 bytes per build row, counted only when `c` is
 * given (NULL: the size-independent part). */
int cx_module_scratch_bytes(const cx_module* m, const cx_exec_ctx* c, uint64_t* bytes);
/* Overrides the multiprocessor count used to size persistent grids (0 = device's). */
int cx_ctx_set_sm_count(cx_exec_ctx* c, int sms);
/* Registers the value range [lo, hi] of column `name` ("d_<column>").  Shared
 * scans turn single-column filters on a ranged column into lookup tables over
 * the first 256 values of the range; filters on unranged columns (or values
 * past the window) are evaluated row by row per query.  The aggregate-cube
 * path (cx_tuning.cube) indexes cells by the values of ranged columns, so it
 * takes the range as a bound: a value outside it raises kernel error 5 (the
 * batch's results are then not valid; re-register the range, or run the batch
 * with cube = 0, whose lookup tables only use the range as a window).  No
 * reference counterpart: the reference plans one query at a time. */
int cx_ctx_set_column_range(cx_exec_ctx* c, const char* name, int64_t lo, int64_t hi);
/* Shared-scan batches are captured once into a CUDA graph and replayed while
 * the batch keeps the same pass shapes (queries per pass, parameters, shared
 * memory assignment, buffers); on by default.  0 launches every kernel directly. */
int cx_ctx_set_graph_replay(cx_exec_ctx* c, int enable);

/* Enqueues the query on `stream` (a cudaStream_t; NULL = legacy default
 * stream).  Asynchronous: call cx_ctx_sync before reading results.  Replaces
 * IExecutor::execute / DynamicLibraryExecutor::execute. */
int cx_execute(cx_module* m, cx_exec_ctx* c, void* stream);
/* cx_execute for a module generated with cx_tuning.parametric = 1: `params`
 * holds the plan's literals in the order of cx_plan_literals.  No reference
 * counterpart: the reference compiles a kernel per query text. */
int cx_execute_params(cx_module* m, cx_exec_ctx* c, const int32_t* params, int nparams, void* stream);
/* Waits for the context's last execute, reads its device error word and fills
 * timing.  Returns CX_E_KERNEL if a kernel raised an error. */
int cx_ctx_sync(cx_exec_ctx* c);
int cx_ctx_timing(const cx_exec_ctx* c, cx_timing* t);
/* Error code raised by a kernel in the last execute (0 = none; 1 = staging
 * wait timeout; 2 = GROUP BY key outside its catalog domain). */
int cx_ctx_kernel_error(const cx_exec_ctx* c, uint32_t* code);

/* ---------------------------------------------------------- shared scans ---
 * A shared scan runs a batch of queries in one pass over the fact table: every
 * fact tile is staged once and every query of the batch is applied to it.
 * Queries are grouped by plan shape (the plan with its integer literals
 * abstracted); one compiled program serves any batch of its shapes, with each
 * query's literals passed as parameters.  No counterpart in the reference,
 * which runs one generated program per query (src/core/execution.cpp:652-725);
 * each query's result buffer is bit-identical to running it alone. */
typedef struct cx_shared_query {
  int shape;              /* index of the query's shape in the program */
  int param_off;          /* offset of its literals in the batch parameter array */
  uint64_t* result;       /* groups x storage_ts u64, device, caller-owned */
  uint64_t result_words;
  uint64_t* validity;     /* validity words, device, caller-owned */
  uint64_t validity_words;
} cx_shared_query;

/* Literals of a plan in the order that numbers its shape's parameters. */
int cx_plan_literals(const char* plan, size_t plan_len, int64_t* out, int cap, int* n);
/* Shared-scan program for `nshapes` plan shapes (one representative plan per
 * shape; its literals are ignored).  Same output contract as cx_codegen; fails
 * with CX_E_INVALID for shapes that cannot share a scan (nullable columns,
 * aggregates other than COUNT/SUM, conflicting joins, OR-joins, multi-value
 * hash joins).  A NULL tuning means 1024 threads, 1 row per thread, 3 staging
 * stages, 1 CTA per SM. */
int cx_shared_codegen(const char* const* plans, const size_t* plan_lens, int nshapes, const cx_tuning* tuning,
                      char* out, size_t out_cap, size_t* out_len);
/* Enqueues one batch (<= 256 queries, <= 4096 parameters) of a compiled shared
 * program on `stream`; cx_ctx_sync waits for it.  The program answers up to 64
 * queries per pass over the fact table; larger batches run as consecutive
 * passes.  Foreign keys of shared joins must be non-zero (the engine checks
 * column minima before batching). */
int cx_shared_execute(cx_module* m, cx_exec_ctx* c, const cx_shared_query* queries, int nq, const int32_t* params,
                      int nparams, void* stream);

/* cx_shared_execute over the fact-table rows [row0, row0 + nrows) only (the
 * range is clipped to the table; nrows = UINT64_MAX runs to its end).  With
 * keep[q] != 0, query q's result and validity words are not zeroed first: the
 * launch adds this range's rows to what earlier ranges left there, so a query
 * can be answered over consecutive launches that each scan one range (the
 * request loop's circular scan lets queries join at any range boundary).
 * keep may be NULL (every query starts from zero). */
int cx_shared_execute_rows(cx_module* m, cx_exec_ctx* c, const cx_shared_query* queries, int nq, const int32_t* params,
                           int nparams, uint64_t row0, uint64_t nrows, const uint8_t* keep, void* stream);

/* Sparse-result compaction: copies every group tuple with a non-zero slot to
 * `dst` in group order and writes the row count to *dev_count (device u64).
 * Same rows as the reference's CompactSparseAggregateResult
 * (src/db/database_instance.cpp:286-307), deterministic order. */
int cx_compact_sparse(const uint64_t* dev_src, uint64_t groups, uint32_t tuple_size, uint64_t* dev_dst,
                      uint64_t* dev_count, void* stream);

/* Sparse-result compaction that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot let this library allocate
 * device memory -- a serving loop that has reserved the whole HBM budget for
 * admitted queries, or an engine whose memory guard must account every device
 * byte before a query runs.  Same output as cx_compact_sparse.  Its scratch is
 * a fixed file-scope device array of 16384 block counts (128 KiB, held by
 * every GPU that loads the library until exit), so `groups` may be at most
 * 16384 * 2048 = 33,554,432; larger inputs return CX_E_CAPACITY (the message
 * in cx_last_error() names the maximum).  A call outside stream capture
 * resolves the array's address in the current device's context; a captured
 * call reuses the address an earlier call on that device resolved, so make the
 * first call on a device before any stream capture.  All calls share the one array: calls
 * whose work overlaps on the GPU (other streams, other threads) race and
 * corrupt each other's results. */
int cx_compact_sparse_noalloc(const uint64_t* dev_src, uint64_t groups, uint32_t tuple_size, uint64_t* dev_dst,
                              uint64_t* dev_count, void* stream);

/* Seeded synthetic column generator (device; no reference counterpart: the
 * reference loads SSB dbgen output from disk, include/crystal/utils.h:242-253).
 * Row r of generator stream `gen_stream` gets lo + below(hash(seed, stream, r),
 * hi - lo + 1); practice_b200/datagen.py restates the same function in numpy. */
int cx_gen_uniform(uint64_t gen_stream, uint64_t seed, int64_t lo, int64_t hi, uint64_t row0, uint64_t rows,
                   int32_t* dev_out, void* stream);
/* yyyymmdd keys of a uniformly drawn day in [1992-01-01, +days). */
int cx_gen_datekey(uint64_t gen_stream, uint64_t seed, uint32_t days, uint64_t row0, uint64_t rows, int32_t* dev_out,
                   void* stream);
/* Seeded Bernoulli validity words: bit r is 0 (NULL) with probability
 * null_permille/1000; unused bits of the last word are 0. */
int cx_gen_validity(uint64_t gen_stream, uint64_t seed, uint64_t rows, uint32_t null_permille, uint64_t* dev_out,
                    void* stream);

/* ------------------------------------------------------------------------
 * Result finalisation on the device.  Replaces the reference's generated
 * post-processing: AggregateDenseCount / AggregateDenseWrite
 * (src/core/visitor.cpp:2589-2697) -- present groups become columnar rows in
 * group order -- and the SortLimit kernels (src/core/visitor.cpp:307-581) --
 * rows ordered by the keys (each compared in its column's result type, a
 * valid value before NULL, ties by row index), then cut to LIMIT.  The row
 * offsets come from a device prefix sum instead of a host loop.
 * ---------------------------------------------------------------------- */
enum { CX_COL_INT64 = 0, CX_COL_UINT64 = 1, CX_COL_FLOAT64 = 2 };

typedef struct cx_result_layout {
  uint64_t groups;                 /* group tuples in the aggregate buffer */
  uint32_t tuple_size;             /* u64 words per tuple (visible columns first) */
  uint32_t columns;                /* visible columns, 1..32 */
  int sparse;                      /* fast sparse output: all-zero tuples dropped, every value valid */
  int scalar;                      /* no GROUP BY: exactly one row */
  const uint8_t* column_type;      /* per column CX_COL_*; NULL = all UINT64 */
  const uint8_t* column_nullable;  /* per column 1 = carries validity; NULL = none */
} cx_result_layout;

typedef struct cx_sort_key {
  int column;
  int descending;
} cx_sort_key;

/* Writes the result rows column by column: column c at dev_columns + c *
 * row_cap, its validity bits at dev_col_validity + c * ((row_cap + 63) / 64).
 * row_cap must cover the group count.  `limit` = UINT64_MAX for none.  Returns
 * the number of rows in *rows (synchronises `stream`). */
int cx_finalize(const uint64_t* dev_result, const uint64_t* dev_validity, const cx_result_layout* layout,
                const cx_sort_key* keys, int nkeys, uint64_t limit, uint64_t* dev_columns,
                uint64_t* dev_col_validity, uint64_t row_cap, uint64_t* rows, void* stream);

/* ------------------------------------------------------------------------
 * Request loop (serving).  No reference counterpart: the reference runs one
 * query per db_cli command on one in-order queue (src/db/database_instance.cpp:23);
 * the admission estimate generalises its device-memory preflight
 * (src/core/execution.cpp:298-404).
 *
 * A server keeps the caller's resident tables (the context passed at create),
 * the compiled programs and per-slot scratch on one GPU.  A scheduler thread
 * admits submitted queries in arrival order while their estimated result and
 * hash/group bytes fit the HBM budget, fuses the admitted shareable queries
 * into shared-scan batches (continuous batching: a batch forms from whatever
 * is waiting when a slot frees up, once at least min_shared_batch wait), runs
 * the others through their plain kernel -- one parametric module per plan
 * shape, so new literals compile nothing -- and overlaps `slots` launches on
 * separate streams.  Results are
 * copied to host memory owned by the server until released.
 * ---------------------------------------------------------------------- */
typedef struct cx_server cx_server;

typedef struct cx_server_config {
  uint64_t budget_bytes;  /* HBM for per-query results, hash tables and batch scratch */
  int max_batch;          /* queries per shared launch, 1..256 (64 per pass) */
  int slots;              /* launches in flight, each on its own stream, 1..8 (default 1) */
  int plain_only;         /* 1: every query runs alone through its plain kernel (baseline loop) */
  int min_shared_batch;   /* fewer waiting shareable queries than this run alone (default 5) */
  cx_tuning shared_tuning;/* launch shape of the shared-scan programs */
  uint64_t chunk_rows;    /* 0: a shared launch scans the whole fact table.  > 0: circular scan --
                             each shared launch scans the next range of this many rows (rounded up
                             to 1024); queries join at any range boundary and finish once they
                             have covered every row, so arrivals wait for one range, not for a
                             whole-table launch */
  uint64_t cube_bytes;    /* per slot: most device bytes the aggregate cubes of one shared launch may
                             take (cx_tuning.cube); a batch whose cubes need more runs the
                             per-query path.  0 = budget_bytes / (2 x slots) */
} cx_server_config;

typedef struct cx_request_info {
  int status;             /* CX_OK when answered, else the request's error */
  uint32_t kernel_error;  /* kernel error code of its launch (0 = none) */
  uint64_t words;         /* u64 words of its result (final layout) */
  uint64_t validity_words;/* u64 words of its validity bitmap */
  double queue_ms;        /* submit -> launch */
  double latency_ms;      /* submit -> result in host memory */
  int batch_size;         /* queries answered by the same launch (1 = alone) */
  int shared;             /* 1 = answered by a shared scan, 0 = by its plain kernel */
} cx_request_info;

typedef struct cx_server_stats {
  uint64_t submitted, completed, rejected, launches;
  double p50_ms, p99_ms, max_ms;  /* latency of completed requests */
  double mean_batch;              /* queries per launch */
  double queries_per_s;           /* completed / (last completion - first submit) */
  uint64_t budget_bytes, peak_reserved_bytes;
} cx_server_stats;

void cx_server_config_default(cx_server_config* cfg);
/* Starts a server on the current device over the tables bound in `tables`
 * (buffers, row counts, value ranges; copied at create). */
int cx_server_create(const cx_exec_ctx* tables, const cx_server_config* cfg, cx_server** out);
/* Compiles what a plan needs ahead of its first submission (its shared
 * program shape or its plain kernel), so no request waits for NVRTC. */
int cx_server_prepare(cx_server* s, const char* plan, size_t plan_len);
/* Same, compiling the plan's plain kernel with `plain_tuning` (e.g. the
 * autotuned launch shape of its shape) for when the plan runs alone. */
int cx_server_prepare_tuned(cx_server* s, const char* plan, size_t plan_len, const cx_tuning* plain_tuning);
/* Queues one query; `id` identifies it to wait / fetch / release.  A plan
 * whose estimated bytes exceed the whole budget is refused (CX_E_REJECTED). */
int cx_server_submit(cx_server* s, const char* plan, size_t plan_len, uint64_t* id);
/* Waits up to timeout_ms (< 0: forever) for a request; CX_E_PENDING if still running. */
int cx_server_wait(cx_server* s, uint64_t id, int timeout_ms, cx_request_info* info);
/* Copies a finished request's result words and validity words. */
int cx_server_fetch(cx_server* s, uint64_t id, uint64_t* words, uint64_t cap, uint64_t* validity, uint64_t vcap);
/* Forgets a finished request and its host copy. */
int cx_server_release(cx_server* s, uint64_t id);
/* Latency and throughput of requests completed since the last reset. */
int cx_server_get_stats(cx_server* s, int reset, cx_server_stats* out);
/* Finishes in-flight work and frees everything. */
int cx_server_destroy(cx_server* s);

#ifdef __cplusplus
}
#endif

#endif /* CRYSTAL_B200_H */
