// cx_internal.h -- library-internal access to execution contexts (not part of
// the C ABI).  Used by the request loop, which runs batches on contexts of its
// own that see the caller's resident tables.
#pragma once

#include <cstdint>
#include <string>

struct cx_exec_ctx;

namespace cx_internal {

// Copies the table bindings of `src` (column buffers, validity bitmaps, table
// row counts, column value ranges) into `dst`.
void ctx_copy_tables(const cx_exec_ctx* src, cx_exec_ctx* dst);

// The value range registered for column `name` ("d_<column>"); false if none.
bool ctx_column_range(const cx_exec_ctx* c, const std::string& name, int64_t* lo, int64_t* hi);

// Device bytes the context holds as its own scratch (hash tables, indexes).
uint64_t ctx_scratch_bytes(const cx_exec_ctx* c);

// Records `msg` as the calling thread's cx_last_error() and returns `code`.
int set_error(int code, const std::string& msg);

}  // namespace cx_internal
