// cx_internal.h -- library-internal access to execution contexts (not part of
// the C ABI).  Used by the request loop, which runs batches on contexts of its
// own that see the caller's resident tables.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/crystal_b200.h"
#include "cx_codegen.h"

struct cx_exec_ctx;
struct cx_module;

namespace cx_internal {

// Copies the table bindings of `src` (column buffers, validity bitmaps, table
// row counts, column value ranges) into `dst`.
void ctx_copy_tables(const cx_exec_ctx* src, cx_exec_ctx* dst);

// The value range registered for column `name` ("d_<column>"); false if none.
bool ctx_column_range(const cx_exec_ctx* c, const std::string& name, int64_t* lo, int64_t* hi);

// Device bytes the context holds as its own scratch (hash tables, indexes).
uint64_t ctx_scratch_bytes(const cx_exec_ctx* c);

// Scratch bytes cx_shared_execute needs for a batch of queries of `shapes`
// (program shape indexes) on program `m`.
uint64_t shared_scratch_need(const cx_module* m, const cx_exec_ctx* c, const int* shapes, int nq);
// Most bytes of aggregate cubes one shared launch on `c` may take (larger batches run the per-query path).
void ctx_set_cube_cap(cx_exec_ctx* c, uint64_t bytes);
// Checks (once per context and column pair, waiting on `s`) which cube
// attributes of a dimension determine others, so that later scratch estimates
// for program `m` see the cube layout its launches will use.
int ensure_cube_dependencies(const cx_module* m, cx_exec_ctx* c, cudaStream_t s);
// Compiles ahead of the first batch the cube scan of program `m` for the cube
// layout batches on `c` will use (every batch of a program shares one), so no
// batch waits for it.
int prepare_cube_layout(cx_module* m, cx_exec_ctx* c, cudaStream_t s);

// Scratch bytes a context owns after an execute that needs `need` bytes, when
// it owns `own` bytes before (own scratch grows to 1.5x the need).
uint64_t grown_scratch(uint64_t own, uint64_t need);

// The code generator's tuning for a C-ABI tuning (defaults where null).
cx::Tuning to_tuning(const cx_tuning* t);

// Whether `src` is a program of the reference's code generator (a SYCL
// `execute_query(db::ExecutionContext*)` translation unit, not cx_codegen output).
bool is_visitor_program(const std::string& src);

// Rewrites such a program's launch skeleton into this library's (kernel
// bodies kept); throws std::runtime_error naming what it cannot translate.
std::string translate_visitor_program(const std::string& src);

// Rows the context holds for the module's fact table (its first table), 0 if unknown.
uint64_t module_fact_rows(const cx_module* m, const cx_exec_ctx* c);

// Takes one more reference on a module (dropped with cx_module_release).
void module_retain(cx_module* m);

// Enqueues the check whether dimension column `b` determines column `a` (n
// rows, value offsets from lo_a / lo_b, radix_b values of b): tab (radix_b
// ints) ends up mapping each b offset to its a offset, and *flag (zeroed by the
// caller) becomes non-zero when some b offset has two different a offsets.
int fd_check_launch(const int* a, const int* b, long long n, int lo_a, int lo_b, int radix_b, int* tab, unsigned* flag,
                    cudaStream_t s);

// Records `msg` as the calling thread's cx_last_error() and returns `code`.
int set_error(int code, const std::string& msg);

}  // namespace cx_internal
