// execution_b200.h -- the two adapters a maintainer adds to crystal-sycl to run
// its query engine on this library: drop the header into the reference's
// include/core/, link db_cli with libcrystal_b200.so, and construct the
// QueryEngine with them instead of AdaptiveCppCompiler / DynamicLibraryExecutor
// (src/db/database_instance.cpp:30-35):
//
//     engine_ = std::make_unique<QueryEngine>(
//         catalog_, std::make_unique<FileBasedQueryCache>(),
//         std::make_unique<NvrtcCompiler>(),
//         std::make_unique<CudaModuleExecutor>(catalog_));
//
// The SQL front end, optimiser and JITOperatorVisitor stay as they are: the
// program the visitor emits goes to cx_compile unchanged (the library
// translates its launch skeleton), and the executor binds the context's
// buffers by name.  Only members that exist in include/core/execution.h and
// include/core/memory.h are used; the one thing ExecutionContext lacks -- the
// row count of each table, which the reference bakes into its programs as the
// LO_LEN / C_LEN / ... macros of include/crystal/utils.h -- comes from the
// catalog the executor is given.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>

#include "core/execution.h"
#include "core/memory.h"
#include "crystal/utils.h"
#include "crystal_b200.h"

namespace db {

// Replaces AdaptiveCppCompiler (src/core/execution.cpp:114-151).  The
// "library path" the engine caches (FileBasedQueryCache) becomes the handle of
// an in-memory module; compile errors surface as std::runtime_error, as the
// acpp path throws them.
class NvrtcCompiler : public ICompiler {
 public:
  std::string compile(const std::string& source_code, const std::string& query_hash) override {
    cx_module* m = nullptr;
    std::string log(1 << 16, '\0');
    if (cx_compile(source_code.data(), source_code.size(), query_hash.c_str(), &m, &log[0], log.size()) != CX_OK)
      throw std::runtime_error(std::string("JIT compilation failed: ") + cx_last_error() + "\n" + log.c_str());
    return "cx:" + std::to_string(reinterpret_cast<std::uintptr_t>(m));
  }
};

// Replaces DynamicLibraryExecutor (src/core/execution.cpp:155-192): instead of
// dlopen() + execute_query(ctx), binds the context's named buffers to a
// library context and runs the module's launch plan on the GPU.
class CudaModuleExecutor : public IExecutor {
 public:
  explicit CudaModuleExecutor(std::shared_ptr<Catalog> catalog) : catalog_(std::move(catalog)) {}

  void execute(const std::string& handle, ExecutionContext* ctx) override {
    if (handle.rfind("cx:", 0) != 0) throw std::runtime_error("not a crystal-b200 module handle: " + handle);
    cx_module* m = reinterpret_cast<cx_module*>(static_cast<std::uintptr_t>(std::stoull(handle.substr(3))));
    cx_exec_ctx* c = cx_ctx_create();
    if (!c) throw std::runtime_error(cx_last_error());
    for (const auto& t : catalog_->getTablesMetadata()) cx_ctx_set_table_rows(c, t.getName().c_str(), t.getSize());
    for (const auto& kv : ctx->buffers_) cx_ctx_set_buffer(c, kv.first.c_str(), kv.second, rows_of(kv.first));
    for (const auto& kv : ctx->null_bitmaps_)
      cx_ctx_set_null_bitmap(c, kv.first.c_str(), kv.second, (rows_of(kv.first) + 63) / 64);
    cx_result_info info{};
    cx_module_result_info(m, &info);
    ctx->result_buffer_->ensureCapacity(info.result_words);
    ctx->ensureResultValidityCapacity(info.result_words);
    cx_ctx_set_result(c, reinterpret_cast<uint64_t*>(ctx->getResultPointer()), info.result_words,
                      ctx->getResultValidityPointer(), info.validity_words);
    int rc = cx_execute(m, c, /*stream=*/nullptr);
    if (rc == CX_OK) rc = cx_ctx_sync(c);
    cx_timing t{};
    cx_ctx_timing(c, &t);
    ctx->timing_.gpu_execute_ms = t.total_ms;
    ctx->timing_.jit_execute_ms = t.total_ms;
    ctx->tuple_size_ = info.finalized ? info.visible_ts : info.storage_ts;
    ctx->result_is_dense_ = false;
    ctx->result_row_count_ = 0;
    ctx->expected_result_size_ = info.result_words;
    const std::string err = rc == CX_OK ? std::string() : std::string(cx_last_error());
    cx_ctx_destroy(c);
    if (rc != CX_OK) throw std::runtime_error(err);  // the REPL catches it (src/cli/terminal_app.cpp:304)
  }

 private:
  // Rows of the table a "d_<column>" buffer belongs to (getTableName, utils.h).
  uint64_t rows_of(const std::string& buffer) const {
    const std::string table = getTableName(buffer.size() > 2 ? buffer.substr(2) : buffer);
    for (const auto& t : catalog_->getTablesMetadata())
      if (t.getName() == table) return t.getSize();
    return 0;
  }

  std::shared_ptr<Catalog> catalog_;
};

}  // namespace db
