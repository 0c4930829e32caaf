// cx_server.cpp -- continuous-batching request loop on one GPU.
//
// The reference answers one query per db_cli command on one in-order queue and
// checks free device memory before each one (preflightDeviceMemoryOrThrow /
// estimateJitTemporaryBytes, src/core/execution.cpp:298-404).  Here a
// scheduler thread serves a stream of queries:
//   * admission in arrival order while the estimated bytes of the admitted
//     queries (results, hash tables, batch scratch) fit the HBM budget;
//   * every admitted shareable query waiting when a slot frees up joins one
//     shared-scan launch (continuous batching), others run through their
//     plain fused kernel; up to `slots` launches overlap on separate streams;
//   * each result is copied to host memory as part of its launch, so a
//     request is finished when its launch's completion event has fired.
// The server is a client of the C ABI (cx_shared_execute, cx_execute) on
// execution contexts of its own that share the caller's resident tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/crystal_b200.h"
#include "cx_codegen.h"
#include "cx_internal.h"
#include "cx_plan.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Plan text with every integer literal blanked: plans that differ only in
// literals share one shape (and one shared-scan program slot).
std::string shape_of(const std::string& text) {
  std::string out;
  out.reserve(text.size());
  size_t i = 0;
  while (i < text.size()) {
    if (text.compare(i, 5, "(int ") == 0) {
      size_t j = i + 5;
      while (j < text.size() && (text[j] == '-' || (text[j] >= '0' && text[j] <= '9'))) ++j;
      out += "(int ?";
      i = j;
      continue;
    }
    out += text[i++];
  }
  return out;
}

struct Request {
  uint64_t id = 0;
  std::string text, shape;
  std::unique_ptr<cx::Plan> plan;
  bool shared = false;
  std::vector<int32_t> lits;
  uint64_t words = 0, vwords = 0, final_words = 0;
  uint64_t est_bytes = 0;
  cx_module* plain = nullptr;  // its plain kernel (parametric unless a literal exceeds int32)
  bool plain_param = false;
  int status = 1;  // 1 queued, 0 running, 2 done
  int rc = CX_OK;
  uint32_t kernel_err = 0;
  double t_submit = 0, t_launch = 0, t_done = 0;
  int batch_size = 0;
  bool ran_shared = false;  // answered by a shared scan (else by its plain kernel)
  // Circular scans: the query runs over consecutive row ranges of the fact
  // table, one per launch, until it has covered every row once.
  bool circ = false;        // joined a circular scan
  bool started = false;     // holds device result buffers and has scanned at least one range
  uint64_t rows_left = 0;   // fact rows it still has to scan
  bool completes = false;   // the launch in flight finishes it
  void* d_res = nullptr;
  void* d_val = nullptr;
  size_t host_off = 0;  // offset of its result in the slot's pinned landing area
  std::vector<uint64_t> h_words, h_val;
};

struct Slot {
  cx_exec_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  bool shared = false;
  cx_module* mod = nullptr;
  std::vector<Request*> reqs;
  uint64_t* pin = nullptr;  // pinned landing area for the launch's results
  size_t pin_words = 0;
  uint64_t reserved = 0;
};

int serr(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return cx_internal::set_error(code, buf);
}

}  // namespace

struct cx_server {
  cx_server_config cfg{};
  int device = 0;
  cx_exec_ctx* tables = nullptr;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  uint64_t reserved = 0, peak_reserved = 0;
  // Shared-scan shapes seen so far and the program compiled for all of them.
  std::vector<std::string> shape_keys;
  std::vector<std::unique_ptr<cx::Plan>> shape_reps;
  std::map<std::string, int> shape_index;
  cx_module* universe = nullptr;
  size_t universe_shapes = 0;
  std::mutex compile_mu;
  std::map<std::string, cx_module*> plain_mods;
  std::map<std::string, cx_tuning> shape_tunings;  // plain launch shape given at prepare, per plan shape
  std::thread th;
  bool stop = false;
  // Circular scans (cfg.chunk_rows > 0): queries between two of their range
  // launches, and where the next range starts.
  std::vector<Request*> circ_idle;
  uint64_t next_row = 0;
  // Statistics since the last reset.
  std::vector<double> lat;
  uint64_t submitted = 0, completed = 0, rejected = 0, launches = 0, launched_queries = 0;
  double first_submit = 0, last_done = 0;
};

namespace {

// Compiles a shared program covering every registered shape (caller holds compile_mu).
int rebuild_universe(cx_server* s) {
  std::vector<std::string> texts;
  std::vector<const cx::Plan*> reps;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->universe && s->universe_shapes == s->shape_reps.size()) return CX_OK;
    for (auto& p : s->shape_reps) reps.push_back(p.get());
  }
  const size_t n = reps.size();
  std::string src;
  try {
    src = cx::generate_shared_cuda(reps, cx_internal::to_tuning(&s->cfg.shared_tuning));
  } catch (const std::exception& e) {
    return serr(CX_E_INVALID, "shared program: %s", e.what());
  }
  cx_module* m = nullptr;
  char log[4096];
  const int rc = cx_compile(src.data(), src.size(), nullptr, &m, log, sizeof log);
  if (rc) return rc;
  // The cube scan for the slots' layout, compiled before any batch needs it
  // (on a context and stream of its own: the scheduler may be running a batch
  // on the slots' contexts meanwhile; the compiled scan is kept by the module).
  {
    cx_exec_ctx* tmp = cx_ctx_create();
    cudaStream_t st = nullptr;
    if (tmp && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
      cx_internal::ctx_copy_tables(s->tables, tmp);
      cx_internal::prepare_cube_layout(m, tmp, st);
      cudaStreamDestroy(st);
    }
    cx_ctx_destroy(tmp);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->universe) cx_module_release(s->universe);
  s->universe = m;
  s->universe_shapes = n;
  return CX_OK;
}

// Parses and classifies a plan; compiles what it needs.  Returns a request
// without an id.
std::string tuning_key(const cx_tuning* t) {
  if (!t) return "default";
  char buf[256];
  snprintf(buf, sizeof buf, "%d/%d/%d/%d/%d/%d/%d/%d/%d/%d/%d/%d/%d/%d", t->block_threads, t->items_per_thread,
           t->stages, t->ctas_per_sm, t->group_placement, t->smem_group_budget, t->bitmap_budget, t->group_merge,
           t->prefetch, t->wait_limit_us, t->debug_stall, t->compact, t->table_budget, t->cube);
  return buf;
}

int make_request(cx_server* s, const char* plan, size_t len, std::unique_ptr<Request>* out,
                 const cx_tuning* plain_tuning = nullptr) {
  auto r = std::make_unique<Request>();
  r->text.assign(plan, len);
  try {
    r->plan = cx::parse_plan(r->text);
  } catch (const std::exception& e) {
    return serr(CX_E_INVALID, "plan: %s", e.what());
  }
  const cx::Plan& p = *r->plan;
  r->shape = shape_of(r->text);
  // Literals become launch parameters (plain and shared) when they fit int32.
  std::vector<const cx::Expr*> lits;
  cx::collect_literals(p, lits);
  bool param_ok = lits.size() <= 64;
  for (const cx::Expr* e : lits) {
    if (e->ival < -2147483647LL || e->ival > 2147483647LL) param_ok = false;
    r->lits.push_back((int32_t)e->ival);
  }
  bool shared = !s->cfg.plain_only && param_ok && cx::shared_shape_ok(p, nullptr);
  if (shared) {
    // The PHT empty sentinel is key 0: every probed foreign key must be > 0.
    for (const auto& st : p.steps) {
      if (st.kind != cx::Step::JoinStep) continue;
      int64_t lo = 0, hi = 0;
      if (!cx_internal::ctx_column_range(s->tables, "d_" + st.join.fks[0], &lo, &hi) || lo <= 0) shared = false;
    }
  }
  // Its plain kernel: one parametric module per plan shape and tuning, so a
  // new literal never waits for NVRTC.  A shape prepared with a tuning keeps
  // it for later submissions.
  cx_module* m = nullptr;
  cx_tuning remembered;
  {
    std::lock_guard<std::mutex> ck(s->compile_mu);
    if (plain_tuning) {
      s->shape_tunings[r->shape] = *plain_tuning;
    } else {
      auto st = s->shape_tunings.find(r->shape);
      if (st != s->shape_tunings.end()) {
        remembered = st->second;
        plain_tuning = &remembered;
      }
    }
    const std::string key = (param_ok ? r->shape : r->text) + "|" + tuning_key(plain_tuning);
    auto it = s->plain_mods.find(key);
    if (it != s->plain_mods.end()) {
      m = it->second;
    } else {
      std::string src;
      try {
        cx::Tuning t = cx_internal::to_tuning(plain_tuning);
        t.parametric = param_ok ? 1 : 0;
        src = cx::generate_cuda(p, t);
      } catch (const std::exception& e) {
        return serr(CX_E_INVALID, "plan: %s", e.what());
      }
      char log[4096];
      const int rc = cx_compile(src.data(), src.size(), nullptr, &m, log, sizeof log);
      if (rc) return rc;
      s->plain_mods[key] = m;
    }
  }
  r->plain = m;
  r->plain_param = param_ok;
  cx_result_info info;
  cx_module_result_info(m, &info);
  uint64_t scratch = 0;
  cx_module_scratch_bytes(m, s->tables, &scratch);
  r->words = std::max<uint64_t>(1, info.result_words);
  r->vwords = std::max<uint64_t>(1, info.validity_words);
  r->final_words = info.final_words;
  const uint64_t groups = p.group_count();
  r->est_bytes = (r->words + r->vwords) * 8 + (shared ? ((groups + 31) / 32) * 4 + 64 + r->lits.size() * 4 : 0);
  if (r->est_bytes + scratch > s->cfg.budget_bytes)
    return serr(CX_E_REJECTED, "cx_server_submit: the query needs %llu bytes, the budget is %llu",
                (unsigned long long)(r->est_bytes + scratch), (unsigned long long)s->cfg.budget_bytes);
  r->shared = shared;
  if (shared) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      auto it = s->shape_index.find(r->shape);
      if (it == s->shape_index.end()) {
        if (s->shape_reps.size() >= 16) {
          r->shared = false;  // the program holds at most 16 shapes; the rest run alone
        } else {
          s->shape_index[r->shape] = (int)s->shape_reps.size();
          s->shape_keys.push_back(r->shape);
          s->shape_reps.push_back(cx::parse_plan(r->text));
        }
      }
    }
    if (r->shared) {
      std::lock_guard<std::mutex> ck(s->compile_mu);
      const int rc = rebuild_universe(s);
      if (rc) return rc;
    }
  }
  *out = std::move(r);
  return CX_OK;
}

// Launches `batch` on `sl` with module `mod` (the scheduler marked the batch
// running and retained `mod` under s->mu; this runs without the lock, so
// submit, wait and the statistics calls are not held up by allocations and
// kernel enqueues).  `shapes` holds each request's shape index in `mod` for a
// shared launch.  On failure the requests carry the error code.
void launch(Slot& sl, std::vector<Request*>& batch, bool shared, cx_module* mod, const std::vector<int>& shapes,
            uint64_t row0 = 0, uint64_t nrows = UINT64_MAX) {
  int rc = CX_OK;
  size_t need = 0;
  for (Request* r : batch) {
    if (!r->completes) continue;  // results of finished queries only
    r->host_off = need;
    need += r->words + r->vwords;
  }
  if (sl.pin_words < need) {
    if (sl.pin) cudaFreeHost(sl.pin);
    sl.pin = nullptr;
    sl.pin_words = 0;
    const size_t grow = need + need / 4;  // some headroom, not a doubling: large results are gigabytes
    if (cudaMallocHost((void**)&sl.pin, grow * 8) != cudaSuccess) rc = CX_E_CUDA;
    else sl.pin_words = grow;
  }
  for (Request* r : batch) {
    if (rc) break;
    if (r->started) continue;  // a circular query keeps its buffers between ranges
    if (cudaMallocAsync(&r->d_res, r->words * 8, sl.stream) != cudaSuccess ||
        cudaMallocAsync(&r->d_val, r->vwords * 8, sl.stream) != cudaSuccess)
      rc = CX_E_CUDA;
  }
  if (!rc && shared) {
    std::vector<cx_shared_query> q(batch.size());
    std::vector<uint8_t> keep(batch.size());
    std::vector<int32_t> params;
    for (size_t i = 0; i < batch.size(); ++i) {
      Request* r = batch[i];
      q[i].shape = shapes[i];
      q[i].param_off = (int)params.size();
      params.insert(params.end(), r->lits.begin(), r->lits.end());
      q[i].result = (uint64_t*)r->d_res;
      q[i].result_words = r->words;
      q[i].validity = (uint64_t*)r->d_val;
      q[i].validity_words = r->vwords;
      keep[i] = r->started ? 1 : 0;
    }
    rc = cx_shared_execute_rows(mod, sl.ctx, q.data(), (int)q.size(), params.data(), (int)params.size(), row0, nrows,
                                keep.data(), sl.stream);
  } else if (!rc) {
    Request* r = batch[0];
    rc = cx_ctx_set_result(sl.ctx, (uint64_t*)r->d_res, r->words, (uint64_t*)r->d_val, r->vwords);
    if (!rc)
      rc = cx_execute_params(mod, sl.ctx, r->plain_param ? r->lits.data() : nullptr,
                             r->plain_param ? (int)r->lits.size() : 0, sl.stream);
  }
  for (Request* r : batch) {
    if (rc) break;
    if (!r->completes) continue;
    if (cudaMemcpyAsync(sl.pin + r->host_off, r->d_res, r->words * 8, cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess ||
        cudaMemcpyAsync(sl.pin + r->host_off + r->words, r->d_val, r->vwords * 8, cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess)
      rc = CX_E_CUDA;
  }
  for (Request* r : batch) {
    if (!r->completes && !rc) continue;  // an error ends every query of the launch
    if (r->d_res) cudaFreeAsync(r->d_res, sl.stream);
    if (r->d_val) cudaFreeAsync(r->d_val, sl.stream);
    r->d_res = r->d_val = nullptr;
  }
  if (!rc && cudaEventRecord(sl.done, sl.stream) != cudaSuccess) rc = CX_E_CUDA;
  if (rc) {
    cudaStreamSynchronize(sl.stream);
    for (Request* r : batch) r->rc = rc;
    cudaEventRecord(sl.done, sl.stream);
  }
}

// Finishes the launch on `sl` once its event fired (caller holds s->mu).
void finish(cx_server* s, Slot& sl) {
  const double t = now_ms();
  int krc = CX_OK;
  uint32_t kerr = 0;
  if (sl.reqs.size() && sl.reqs[0]->rc == CX_OK) {
    krc = cx_ctx_sync(sl.ctx);
    cx_ctx_kernel_error(sl.ctx, &kerr);
  }
  for (Request* r : sl.reqs) {
    if (r->rc == CX_OK && krc != CX_OK && krc != CX_E_KERNEL) r->rc = krc;
    r->kernel_err |= kerr;
    if (r->rc == CX_OK && !r->completes) {
      // A circular query with rows left waits for its next range.
      r->started = true;
      s->circ_idle.push_back(r);
      continue;
    }
    if (r->circ && r->rc != CX_OK && !r->completes) {
      if (r->d_res) cudaFree(r->d_res);
      if (r->d_val) cudaFree(r->d_val);
      r->d_res = r->d_val = nullptr;
    }
    s->reserved -= std::min(s->reserved, r->est_bytes);
    if (r->rc == CX_OK) {
      r->h_words.assign(sl.pin + r->host_off, sl.pin + r->host_off + r->final_words);
      r->h_val.assign(sl.pin + r->host_off + r->words, sl.pin + r->host_off + r->words + (r->final_words + 63) / 64);
    }
    r->status = 2;
    r->t_done = t;
    s->lat.push_back(t - r->t_submit);
    ++s->completed;
    s->last_done = t;
  }
  sl.reserved = 0;
  sl.reqs.clear();
  sl.busy = false;
  cx_module_release(sl.mod);  // the reference the scheduler took for this launch
  sl.mod = nullptr;
}

uint64_t fixed_bytes(cx_server* s) {
  uint64_t b = 0;
  for (const Slot& sl : s->slots) b += cx_internal::ctx_scratch_bytes(sl.ctx);
  return b;
}

void scheduler(cx_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    bool progressed = false;
    for (Slot& sl : s->slots) {
      if (!sl.busy) continue;
      const cudaError_t q = cudaEventQuery(sl.done);
      if (q == cudaErrorNotReady) continue;
      finish(s, sl);
      progressed = true;
    }
    if (progressed) s->cv_done.notify_all();
    const bool circ_mode = s->cfg.chunk_rows > 0 && !s->cfg.plain_only;
    for (Slot& sl : s->slots) {
      if (sl.busy) continue;
      const bool circ_waiting = circ_mode && !s->circ_idle.empty();
      if (s->pending.empty() && !circ_waiting) continue;
      const uint64_t fixed = fixed_bytes(s);
      const uint64_t own = cx_internal::ctx_scratch_bytes(sl.ctx);
      std::vector<Request*> batch;
      Request* head = s->pending.empty() ? nullptr : s->pending.front();
      // Admission: what is reserved, the scratch the slots own, the scratch
      // this launch adds to its slot and the new queries' bytes must fit the
      // budget.  A launch on an idle GPU always goes (sizes were checked
      // against the whole budget at submit).
      auto admit = [&](uint64_t growth, uint64_t add) {
        return s->reserved + fixed + growth + add <= s->cfg.budget_bytes || (s->reserved == 0 && batch.empty());
      };
      auto in_universe = [&](const Request* r) {
        return r->shared && s->universe && s->shape_index.at(r->shape) < (int)s->universe_shapes;
      };
      bool shared = head && in_universe(head);
      if (shared && !circ_waiting) {
        // A short queue runs its head alone through the plain kernel: one
        // shared launch costs about as much as a few plain ones.
        int ready = 0;
        for (Request* r : s->pending) {
          if (!in_universe(r) || ready >= s->cfg.min_shared_batch) break;
          ++ready;
        }
        if (ready < s->cfg.min_shared_batch) shared = false;
      }
      // Queries between two ranges of a circular scan always continue; a
      // non-shareable head runs alone first.
      if (circ_waiting && (!head || in_universe(head))) shared = true;
      if (!shared) {
        uint64_t need = 0;
        cx_module_scratch_bytes(head->plain, sl.ctx, &need);
        if (admit(cx_internal::grown_scratch(own, need) - own, head->est_bytes)) {
          batch.push_back(head);
          s->pending.pop_front();
        }
      } else {
        uint64_t add = 0;
        std::vector<int> shapes;
        if (circ_mode) {
          while (!s->circ_idle.empty() && (int)batch.size() < s->cfg.max_batch) {
            batch.push_back(s->circ_idle.front());
            shapes.push_back(s->shape_index.at(s->circ_idle.front()->shape));
            s->circ_idle.erase(s->circ_idle.begin());
          }
        }
        cx_internal::ensure_cube_dependencies(s->universe, sl.ctx, sl.stream);
        while (!s->pending.empty() && (int)batch.size() < s->cfg.max_batch) {
          Request* r = s->pending.front();
          if (!in_universe(r)) break;
          shapes.push_back(s->shape_index.at(r->shape));
          const uint64_t need = cx_internal::shared_scratch_need(s->universe, sl.ctx, shapes.data(), (int)shapes.size());
          if (!admit(cx_internal::grown_scratch(own, need) - own, add + r->est_bytes)) {
            shapes.pop_back();
            break;
          }
          add += r->est_bytes;
          batch.push_back(r);
          s->pending.pop_front();
        }
      }
      if (batch.empty()) break;
      // The row range of a circular launch; every other launch covers the table.
      uint64_t row0 = 0, nrows = UINT64_MAX;
      if (shared && circ_mode) {
        const uint64_t fact_rows = cx_internal::module_fact_rows(s->universe, sl.ctx);
        row0 = s->next_row < fact_rows ? s->next_row : 0;
        nrows = std::min<uint64_t>(s->cfg.chunk_rows, fact_rows - row0);
        s->next_row = row0 + nrows >= fact_rows ? 0 : row0 + nrows;
        for (Request* r : batch) {
          if (!r->circ) {
            r->circ = true;
            r->rows_left = fact_rows;
          }
          r->rows_left -= std::min(r->rows_left, nrows);
          r->completes = r->rows_left == 0;
        }
      } else {
        for (Request* r : batch) r->completes = true;
      }
      // Mark the batch running and reserve the bytes of its new queries under
      // the lock; the launch itself runs without it.  The slot keeps a
      // reference on the module it launches, so a new shared program compiled
      // meanwhile cannot unload it while its kernels run.
      const double t_launch = now_ms();
      sl.busy = true;
      sl.shared = shared;
      sl.reqs = batch;
      sl.reserved = 0;
      std::vector<int> shapes;
      for (Request* r : batch) {
        if (r->status == 1) {  // first launch of this query
          r->t_launch = t_launch;
          s->reserved += r->est_bytes;
        }
        r->status = 0;
        r->batch_size = (int)batch.size();
        r->ran_shared = shared;
        if (shared) shapes.push_back(s->shape_index.at(r->shape));
      }
      cx_module* mod = shared ? s->universe : head->plain;
      cx_internal::module_retain(mod);
      sl.mod = mod;
      lk.unlock();
      launch(sl, batch, shared, mod, shapes, row0, nrows);
      lk.lock();
      ++s->launches;
      s->launched_queries += batch.size();
      s->peak_reserved = std::max(s->peak_reserved, s->reserved + fixed_bytes(s));
      progressed = true;
    }
    bool busy = false;
    for (const Slot& sl : s->slots) busy = busy || sl.busy;
    if (s->stop && !busy && s->pending.empty() && s->circ_idle.empty()) break;
    if (!progressed) s->cv_sched.wait_for(lk, std::chrono::microseconds(busy ? 20 : 2000));
  }
}

}  // namespace

extern "C" {

void cx_server_config_default(cx_server_config* cfg) {
  if (!cfg) return;
  memset(cfg, 0, sizeof *cfg);
  cfg->budget_bytes = 40ULL << 30;
  cfg->max_batch = 64;
  cfg->slots = 1;
  cfg->min_shared_batch = 5;
  cfg->chunk_rows = 0;
  cfg->plain_only = 0;
  cx_tuning_default(&cfg->shared_tuning);
  cfg->shared_tuning.block_threads = 1024;
  cfg->shared_tuning.items_per_thread = 1;
  cfg->shared_tuning.stages = 3;
  cfg->shared_tuning.ctas_per_sm = 1;
}

int cx_server_create(const cx_exec_ctx* tables, const cx_server_config* cfg, cx_server** out) {
  if (!tables || !out) return serr(CX_E_INVALID, "cx_server_create: NULL argument");
  auto s = std::make_unique<cx_server>();
  if (cfg) s->cfg = *cfg;
  else cx_server_config_default(&s->cfg);
  if (s->cfg.min_shared_batch < 1) s->cfg.min_shared_batch = 1;
  // Range starts stay 4 KiB aligned (bulk-copy alignment of every fact column).
  if (s->cfg.chunk_rows) s->cfg.chunk_rows = (s->cfg.chunk_rows + 1023) / 1024 * 1024;
  if (s->cfg.max_batch < 1 || s->cfg.max_batch > 256 || s->cfg.slots < 1 || s->cfg.slots > 8 || s->cfg.budget_bytes == 0)
    return serr(CX_E_INVALID, "cx_server_create: max_batch 1..256, slots 1..8 and a non-zero budget");
  if (cudaGetDevice(&s->device) != cudaSuccess) return serr(CX_E_NO_DEVICE, "cx_server_create: no CUDA device");
  // Per-query result buffers come from the device's stream-ordered pool; keep
  // freed blocks in the pool up to the budget instead of returning them.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t keep = s->cfg.budget_bytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  s->tables = cx_ctx_create();
  cx_internal::ctx_copy_tables(tables, s->tables);
  s->slots.resize(s->cfg.slots);
  for (Slot& sl : s->slots) {
    sl.ctx = cx_ctx_create();
    cx_internal::ctx_copy_tables(tables, sl.ctx);
    // Batches here change from launch to launch (queries, shapes, row
    // ranges), so a captured graph would be re-captured every time: launch
    // the kernels directly.
    cx_ctx_set_graph_replay(sl.ctx, 0);
    cx_internal::ctx_set_cube_cap(sl.ctx, s->cfg.cube_bytes ? s->cfg.cube_bytes
                                                            : s->cfg.budget_bytes / (2 * (uint64_t)s->cfg.slots));
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
      return serr(CX_E_CUDA, "cx_server_create: stream or event creation failed");
  }
  cx_server* raw = s.release();
  raw->th = std::thread(scheduler, raw);
  *out = raw;
  return CX_OK;
}

int cx_server_prepare(cx_server* s, const char* plan, size_t plan_len) {
  return cx_server_prepare_tuned(s, plan, plan_len, nullptr);
}

int cx_server_prepare_tuned(cx_server* s, const char* plan, size_t plan_len, const cx_tuning* plain_tuning) {
  if (!s || !plan) return serr(CX_E_INVALID, "cx_server_prepare: NULL argument");
  std::unique_ptr<Request> r;
  return make_request(s, plan, plan_len, &r, plain_tuning);
}

int cx_server_submit(cx_server* s, const char* plan, size_t plan_len, uint64_t* id) {
  if (!s || !plan || !id) return CX_E_INVALID;
  const double t = now_ms();
  std::unique_ptr<Request> r;
  const int rc = make_request(s, plan, plan_len, &r);
  if (rc) {
    if (rc == CX_E_REJECTED) {
      std::lock_guard<std::mutex> lk(s->mu);
      ++s->submitted;
      ++s->rejected;
    }
    return rc;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->submitted == 0 || s->first_submit == 0) s->first_submit = t;
  ++s->submitted;
  if (r->est_bytes > s->cfg.budget_bytes) {
    ++s->rejected;
    return serr(CX_E_REJECTED, "cx_server_submit: the query needs %llu bytes, the budget is %llu",
                (unsigned long long)r->est_bytes, (unsigned long long)s->cfg.budget_bytes);
  }
  r->id = s->next_id++;
  r->t_submit = t;
  *id = r->id;
  s->pending.push_back(r.get());
  s->reqs[r->id] = std::move(r);
  s->cv_sched.notify_one();
  return CX_OK;
}

int cx_server_wait(cx_server* s, uint64_t id, int timeout_ms, cx_request_info* info) {
  if (!s) return CX_E_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CX_E_INVALID;
  Request* r = it->second.get();
  auto done = [&] { return r->status == 2; };
  if (timeout_ms < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return CX_E_PENDING;
  if (info) {
    info->status = r->rc;
    info->kernel_error = r->kernel_err;
    info->words = r->final_words;
    info->validity_words = (r->final_words + 63) / 64;
    info->queue_ms = r->t_launch - r->t_submit;
    info->latency_ms = r->t_done - r->t_submit;
    info->batch_size = r->batch_size;
    info->shared = r->ran_shared ? 1 : 0;
  }
  return r->rc;
}

int cx_server_fetch(cx_server* s, uint64_t id, uint64_t* words, uint64_t cap, uint64_t* validity, uint64_t vcap) {
  if (!s) return CX_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CX_E_INVALID;
  Request* r = it->second.get();
  if (r->status != 2) return CX_E_PENDING;
  if (r->rc) return r->rc;
  if (cap < r->h_words.size() || vcap < r->h_val.size()) return CX_E_CAPACITY;
  if (words) memcpy(words, r->h_words.data(), r->h_words.size() * 8);
  if (validity) memcpy(validity, r->h_val.data(), r->h_val.size() * 8);
  return CX_OK;
}

int cx_server_release(cx_server* s, uint64_t id) {
  if (!s) return CX_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return CX_E_INVALID;
  if (it->second->status != 2) return CX_E_PENDING;
  s->reqs.erase(it);
  return CX_OK;
}

int cx_server_get_stats(cx_server* s, int reset, cx_server_stats* out) {
  if (!s || !out) return CX_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof *out);
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->rejected = s->rejected;
  out->launches = s->launches;
  out->budget_bytes = s->cfg.budget_bytes;
  out->peak_reserved_bytes = s->peak_reserved;
  out->mean_batch = s->launches ? (double)s->launched_queries / (double)s->launches : 0.0;
  if (!s->lat.empty()) {
    std::vector<double> v = s->lat;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = v.back();
    const double span = s->last_done - s->first_submit;
    out->queries_per_s = span > 0 ? (double)s->completed / (span / 1000.0) : 0.0;
  }
  if (reset) {
    s->lat.clear();
    s->submitted = s->completed = s->rejected = s->launches = s->launched_queries = 0;
    s->first_submit = s->last_done = 0;
    s->peak_reserved = s->reserved + fixed_bytes(s);
  }
  return CX_OK;
}

int cx_server_destroy(cx_server* s) {
  if (!s) return CX_E_INVALID;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_sched.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.pin) cudaFreeHost(sl.pin);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    cx_ctx_destroy(sl.ctx);
  }
  if (s->universe) cx_module_release(s->universe);
  for (auto& kv : s->plain_mods) cx_module_release(kv.second);
  cx_ctx_destroy(s->tables);
  delete s;
  return CX_OK;
}

}  // extern "C"
