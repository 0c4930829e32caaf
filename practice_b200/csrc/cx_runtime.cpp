// cx_runtime.cpp -- NVRTC compiler, module cache and generic executor behind
// the C ABI in include/crystal_b200.h.
//
// The reference compiles each generated program out of process with `acpp` and
// dlopen()s it (src/core/execution.cpp:114-192); the generated library then
// runs its own host code.  Here the generated source holds device code plus a
// launch plan; NVRTC compiles it in memory for sm_100a and one generic
// executor (this file) runs the plan: memsets, build kernels, the fused scan,
// epilogues.  Driver-API entry points are obtained through the runtime
// (cudaGetDriverEntryPointByVersion), so the library links no libcuda and
// loads on hosts without a GPU.
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/crystal_b200.h"
#include "cx_args.h"
#include "cx_codegen.h"
#include "cx_internal.h"
#include "cx_plan.h"

// Generated at build time from crystal_sm100.cuh and cx_args.h.
#include "cx_embedded.inc"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CX_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(CX_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_));    \
  } while (0)

// ----------------------------------------------------------- driver entry ---
struct Driver {
  CUresult (*ModuleLoadData)(CUmodule*, const void*) = nullptr;
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*ModuleUnload)(CUmodule) = nullptr;
  CUresult (*FuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                           void**, void**) = nullptr;
  CUresult (*Occupancy)(int*, CUfunction, int, size_t) = nullptr;
  CUresult (*GetErrorString)(CUresult, const char**) = nullptr;
  bool ok = false;
};

template <typename F>
bool entry(const char* name, F& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p)
    return false;
  fn = reinterpret_cast<F>(p);
  return true;
}

Driver& driver() {
  static Driver d;
  static std::once_flag once;
  std::call_once(once, [] {
    d.ok = entry("cuModuleLoadData", d.ModuleLoadData) && entry("cuModuleGetFunction", d.ModuleGetFunction) &&
           entry("cuModuleUnload", d.ModuleUnload) && entry("cuFuncSetAttribute", d.FuncSetAttribute) &&
           entry("cuLaunchKernel", d.LaunchKernel) &&
           entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", d.Occupancy) &&
           entry("cuGetErrorString", d.GetErrorString);
  });
  return d;
}

int drv_fail(CUresult r, const char* what) {
  const char* s = "unknown";
  if (driver().GetErrorString) driver().GetErrorString(r, &s);
  return fail(CX_E_CUDA, "%s: %s", what, s);
}

// ------------------------------------------------------------ launch plan ---
struct KernelSpec {
  std::string name, kind;
  int table = 0, block = 128, tile = 512, ctas_per_sm = 1;
  size_t smem = 0;
};

struct LaunchPlan {
  std::vector<std::string> tables;
  struct Col { int slot; std::string name; int table; };
  std::vector<Col> cols;
  std::vector<std::pair<int, std::string>> nulls;
  // A hash table of `words` ints, or (rows_table >= 0) of mult x the row count
  // of that table, known at execute.
  struct Ht { int slot; std::string name; uint64_t words; int rows_table = -1; uint64_t mult = 0; };
  std::vector<Ht> hts;
  std::map<int, uint64_t> htv_words;
  std::map<int, uint64_t> bm_words;
  std::map<int, int> mht_table;                        // multi-value hash table slot -> build table slot
  std::map<int, int> mht_arrays;                       // payload arrays (row ids + published columns) per slot
  uint64_t result_words = 0, groups = 1;
  int storage_ts = 1, visible_ts = 1, sparse = 0;
  uint64_t touched_words = 0;
  bool finalize = false;
  uint64_t fin_groups = 0;
  int fin_vts = 0;
  std::vector<KernelSpec> kernels;
  bool shared = false;
  int shared_maxq = 256, shared_maxp = 4096;           // queries / parameters per shared launch
  uint64_t shared_qb_bytes = 0;                        // shared memory of row bitmaps per query of a pass
  int nparams = -1;                                    // parametric plain kernels: literal count
  bool rows_sized = false;                             // some hash table is sized by a table's rows
  std::map<int, uint64_t> dat_words;                   // shared scans: extra payload attributes per dimension
  std::vector<std::pair<int, std::string>> fcols;      // shared scans: fact filter table columns
  struct SShape { uint64_t groups; int ts, grouped, sparse, nlits, smem_ok, naggs; uint64_t tw; int nseen; };
  std::vector<SShape> sshapes;
  // Shared scans with an aggregate-cube path: its attributes (dimension index
  // and 16-bit field of the entry, or dim -1 for a fact column) and, per shape,
  // its SUM aggregates and attributes in cell order.
  bool cube = false;
  struct CAttr { int dim = -1, field = 0; std::string col; };
  std::vector<CAttr> cattrs;
  struct CShape { int nsums = 0; std::vector<int> attrs; };
  std::vector<CShape> cshapes;
  struct CDim { int table = 0; long long len = 0, keymin = 0; std::string fk, pk; };
  std::vector<CDim> cdims;
};

bool parse_launch_plan(const std::string& src, LaunchPlan& lp, std::string& err) {
  const size_t b = src.find("/*@cx-launch");
  const size_t e = src.find("@*/");
  if (b == std::string::npos || e == std::string::npos || e < b) {
    err = "source has no /*@cx-launch ... @*/ block (not generated by cx_codegen)";
    return false;
  }
  std::istringstream in(src.substr(b + 12, e - b - 12));
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string k;
    if (!(ls >> k)) continue;
    if (k == "v") {
      int v = 0;
      ls >> v;
      if (v != 1) { err = "unsupported launch plan version"; return false; }
    } else if (k == "table") {
      int s; std::string n;
      ls >> s >> n;
      if (s != (int)lp.tables.size()) { err = "table slots out of order"; return false; }
      lp.tables.push_back(n);
    } else if (k == "col") {
      LaunchPlan::Col c;
      ls >> c.slot >> c.name >> c.table;
      lp.cols.push_back(c);
    } else if (k == "null") {
      int s; std::string n;
      ls >> s >> n;
      lp.nulls.emplace_back(s, n);
    } else if (k == "ht") {
      LaunchPlan::Ht h;
      ls >> h.slot >> h.name >> h.words;
      lp.hts.push_back(h);
    } else if (k == "htrows") {
      LaunchPlan::Ht h;
      ls >> h.slot >> h.name >> h.mult >> h.rows_table;
      h.words = h.mult;
      lp.hts.push_back(h);
      lp.rows_sized = true;
    } else if (k == "htv") {
      int s; uint64_t w;
      ls >> s >> w;
      lp.htv_words[s] = w;
    } else if (k == "shared") {
      lp.shared = true;
      int mq = 0, mp = 0;
      if (ls >> mq >> mp) { lp.shared_maxq = mq; lp.shared_maxp = mp; }
      ls.clear();
    } else if (k == "params") {
      ls >> lp.nparams;
      if (lp.nparams > CX_MAX_LITS) { err = "too many literal parameters"; return false; }
    } else if (k == "sqb") {
      ls >> lp.shared_qb_bytes;
    } else if (k == "dat") {
      int s; uint64_t w;
      ls >> s >> w;
      lp.dat_words[s] = w;
    } else if (k == "fcol") {
      int s; std::string n;
      ls >> s >> n;
      if (s != (int)lp.fcols.size() || s >= CX_MAX_FCOLS) { err = "filter table columns out of order"; return false; }
      lp.fcols.emplace_back(s, n);
    } else if (k == "sshape") {
      int i; LaunchPlan::SShape sh;
      ls >> i >> sh.groups >> sh.ts >> sh.grouped >> sh.sparse >> sh.nlits >> sh.smem_ok >> sh.naggs >> sh.tw >> sh.nseen;
      if (i != (int)lp.sshapes.size()) { err = "shape lines out of order"; return false; }
      lp.sshapes.push_back(sh);
    } else if (k == "cube") {
      size_t n = 0;
      ls >> n;
      if (n > CX_MAX_CATTRS) { err = "too many cube attributes"; return false; }
      lp.cube = true;
    } else if (k == "cattr") {
      int id = 0;
      LaunchPlan::CAttr at;
      ls >> id >> at.dim >> at.field >> at.col;
      if (id != (int)lp.cattrs.size() || id >= CX_MAX_CATTRS || at.field < 0 || at.field > 3 || at.dim >= CX_MAX_HTS) {
        err = "cube attribute lines out of order or out of range";
        return false;
      }
      lp.cattrs.push_back(at);
    } else if (k == "cshape") {
      int i = 0, na = 0;
      LaunchPlan::CShape cs;
      ls >> i >> cs.nsums >> na;
      if (i != (int)lp.cshapes.size() || na < 0 || na > CX_MAX_SATTRS || cs.nsums < 0 || cs.nsums > 64) {
        err = "cube shape lines out of order or out of range";
        return false;
      }
      for (int j = 0; j < na; ++j) {
        int id = -1;
        ls >> id;
        if (id < 0 || id >= (int)lp.cattrs.size()) { err = "cube shape names an unknown attribute"; return false; }
        cs.attrs.push_back(id);
      }
      lp.cshapes.push_back(cs);
    } else if (k == "cdim") {
      int i = 0;
      LaunchPlan::CDim cd;
      ls >> i >> cd.table >> cd.len >> cd.keymin >> cd.fk >> cd.pk;
      if (i != (int)lp.cdims.size() || i >= CX_MAX_HTS || cd.len <= 0) { err = "cube dimension lines out of order or out of range"; return false; }
      lp.cdims.push_back(cd);
    } else if (k == "mht") {
      int sl = 0, t = 0, na = 1;
      ls >> sl >> t;
      if (!(ls >> na)) { na = 1; ls.clear(); }
      if (na < 1 || na > 32) { err = "bad payload array count on an mht line"; return false; }
      lp.mht_table[sl] = t;
      lp.mht_arrays[sl] = na;
    } else if (k == "bm") {
      int s; uint64_t w;
      ls >> s >> w;
      lp.bm_words[s] = w;
    } else if (k == "result") {
      ls >> lp.result_words >> lp.groups >> lp.storage_ts >> lp.visible_ts >> lp.sparse;
    } else if (k == "touched") {
      ls >> lp.touched_words;
    } else if (k == "finalize") {
      lp.finalize = true;
      ls >> lp.fin_groups >> lp.fin_vts;
    } else if (k == "kernel") {
      KernelSpec ks;
      ls >> ks.name >> ks.kind >> ks.table >> ks.block;
      if (ks.kind == "build" || ks.kind == "cubeidx" || ks.kind == "tiles" || ks.kind == "tilescan") ls >> ks.tile;
      else if (ks.kind == "scan" || ks.kind == "sharedscan" || ks.kind == "cubescan") ls >> ks.tile >> ks.smem >> ks.ctas_per_sm;
      else { size_t z; ls >> z; }
      lp.kernels.push_back(ks);
    } else {
      err = "unknown launch plan line: " + line;
      return false;
    }
    if (ls.fail()) { err = "malformed launch plan line: " + line; return false; }
  }
  if (lp.cols.size() > CX_MAX_COLS || lp.hts.size() > CX_MAX_HTS || lp.tables.size() > CX_MAX_TABLES) {
    err = "launch plan exceeds argument slots";
    return false;
  }
  for (const auto& h : lp.hts)
    if (h.rows_table >= (int)lp.tables.size() || h.slot < 0 || h.slot >= CX_MAX_HTS) {
      err = "hash table line names a slot or table outside the plan";
      return false;
    }
  for (const auto& k : lp.kernels)
    if ((k.kind == "tiles" || k.kind == "tilescan" || k.kind == "build" || k.kind == "cubeidx") &&
        (k.table < 0 || k.table >= (int)lp.tables.size() || k.tile <= 0 || k.block <= 0 || k.block > 1024)) {
      err = "kernel line " + k.name + " names a table outside the plan or a bad shape";
      return false;
    }
  return true;
}

uint64_t align256(uint64_t x) { return (x + 255) & ~255ULL; }

// Scratch layout of one execute: hash tables, payload validity, group
// touched bits, finalisation staging and the error word.
struct ScratchLayout {
  std::vector<uint64_t> ht_off, htv_off, bm_off;
  uint64_t touched_off = 0, fin_off = 0, err_off = 0, total = 0;
};

// Words of a hash table: fixed, or sized by its table's rows when they are
// known (at least one row's worth before that).
uint64_t ht_words(const LaunchPlan::Ht& h, const std::vector<long long>* rows) {
  if (h.rows_table < 0) return h.words;
  const long long n = rows ? std::max<long long>(1, (*rows)[h.rows_table]) : 1;
  return h.mult * (uint64_t)n;
}

ScratchLayout scratch_layout(const LaunchPlan& lp, const std::vector<long long>* rows = nullptr) {
  ScratchLayout s;
  uint64_t off = 0;
  for (const auto& h : lp.hts) {
    s.ht_off.push_back(off);
    off = align256(off + ht_words(h, rows) * 4);
  }
  for (const auto& h : lp.hts) {
    auto it = lp.htv_words.find(h.slot);
    s.htv_off.push_back(off);
    if (it != lp.htv_words.end()) off = align256(off + it->second * 4);
  }
  for (const auto& h : lp.hts) {
    auto it = lp.bm_words.find(h.slot);
    s.bm_off.push_back(off);
    if (it != lp.bm_words.end()) off = align256(off + it->second * 4);
  }
  s.touched_off = off;
  off = align256(off + lp.touched_words * 4);
  s.fin_off = off;
  if (lp.finalize) {
    const uint64_t vis = lp.fin_groups * (uint64_t)lp.fin_vts;
    off = align256(off + (vis + (vis + 63) / 64 + 1) * 8);
  }
  s.err_off = off;
  off = align256(off + 16);
  s.total = off;
  return s;
}

// Bytes of the row-id payloads of a plan's multi-value hash tables: one int
// per build row, so they are sized when the row counts are known.
// Bytes of one multi-value hash table's payload: its arrays (row ids, then
// the published columns and their validity) of one int per build row each.
uint64_t mht_slot_bytes(const LaunchPlan& lp, int slot, long long build_rows) {
  auto it = lp.mht_arrays.find(slot);
  const uint64_t arrays = it == lp.mht_arrays.end() ? 1 : (uint64_t)it->second;
  return align256((uint64_t)std::max<long long>(1, build_rows) * 4 * arrays);
}

uint64_t mht_payload_bytes(const LaunchPlan& lp, const std::vector<long long>& rows) {
  uint64_t b = 0;
  for (const auto& kv : lp.mht_table) b += mht_slot_bytes(lp, kv.first, rows[kv.second]);
  return b;
}

}  // namespace

// ---------------------------------------------------------------- module ---
struct cx_module {
  std::string key;
  size_t src_hash = 0;
  uint64_t uid = 0;  // unique per module for the life of the process (graph signatures)
  std::vector<char> cubin;
  LaunchPlan lp;
  ScratchLayout sl;
  std::atomic<int> refs{1};
  std::mutex mu;
  struct Loaded {
    CUmodule mod = nullptr;
    std::vector<CUfunction> fns;
    std::vector<int> occupancy;  // scan kernels: CTAs per SM at their smem size
  };
  std::map<int, Loaded> per_device;
  // Shared programs with a cube path: the source, and the cube scan compiled
  // once per cube layout with the layout as constants, per layout and device.
  std::string source;
  struct Spec { CUmodule mod = nullptr; CUfunction fn = nullptr; bool failed = false; };
  std::map<std::string, std::map<int, Spec>> cube_specs;
};

struct cx_exec_ctx {
  std::unordered_map<std::string, std::pair<const void*, uint64_t>> buffers;
  std::unordered_map<std::string, std::pair<const uint64_t*, uint64_t>> nulls;
  std::unordered_map<std::string, uint64_t> rows;
  std::unordered_map<std::string, std::pair<int64_t, int64_t>> ranges;  // registered column value ranges
  uint64_t* result = nullptr;
  uint64_t result_words = 0;
  uint64_t* validity = nullptr;
  uint64_t validity_words = 0;
  void* user_scratch = nullptr;
  uint64_t user_scratch_bytes = 0;
  void* own_scratch = nullptr;
  uint64_t own_scratch_bytes = 0;
  int device = -1;
  int sm_override = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  unsigned int* host_err = nullptr;  // pinned
  void* host_stage = nullptr;        // pinned staging of shared-scan descriptors
  size_t host_stage_bytes = 0;
  bool pending = false;
  cx_timing timing{};
  uint32_t kernel_err = 0;
  // Shared-scan batches replay a captured CUDA graph while their pass shapes repeat.
  bool graph_replay = true;
  uint64_t cube_cap = UINT64_MAX;   // most bytes of aggregate cubes one shared launch may take
  // Functional dependencies between dimension columns checked for cube
  // layouts, by "A|B|buffers|rows|ranges": whether B determines A, and the
  // device table from B's value offset to A's.
  struct Fd { bool holds = false; int* tab = nullptr; };
  std::map<std::string, Fd> fds;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  std::vector<unsigned char> gsig;
  int graph_launches = 0;
};

namespace {

std::mutex g_cache_mu;
std::unordered_map<std::string, cx_module*> g_cache;

int load_on_device(cx_module* m, int dev, cx_module::Loaded** out) {
  std::lock_guard<std::mutex> lk(m->mu);
  auto it = m->per_device.find(dev);
  if (it != m->per_device.end()) { *out = &it->second; return CX_OK; }
  Driver& d = driver();
  if (!d.ok) return fail(CX_E_CUDA, "CUDA driver entry points unavailable");
  cx_module::Loaded L;
  CUresult r = d.ModuleLoadData(&L.mod, m->cubin.data());
  if (r != CUDA_SUCCESS) return drv_fail(r, "cuModuleLoadData");
  for (const auto& k : m->lp.kernels) {
    CUfunction f = nullptr;
    r = d.ModuleGetFunction(&f, L.mod, k.name.c_str());
    if (r != CUDA_SUCCESS) { d.ModuleUnload(L.mod); return drv_fail(r, k.name.c_str()); }
    int occ = 1;
    if (k.kind == "scan" || k.kind == "sharedscan" || k.kind == "cubescan") {
      if (m->lp.shared) {
        r = d.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, 227 * 1024);
        if (r != CUDA_SUCCESS) { d.ModuleUnload(L.mod); return drv_fail(r, "cuFuncSetAttribute(smem)"); }
      } else if (k.smem > 48 * 1024) {
        r = d.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)k.smem);
        if (r != CUDA_SUCCESS) { d.ModuleUnload(L.mod); return drv_fail(r, "cuFuncSetAttribute(smem)"); }
      }
      r = d.Occupancy(&occ, f, k.block, k.smem);
      if (r != CUDA_SUCCESS) { d.ModuleUnload(L.mod); return drv_fail(r, "cuOccupancyMaxActiveBlocksPerMultiprocessor"); }
      if (occ < 1) { d.ModuleUnload(L.mod); return fail(CX_E_CAPACITY, "scan kernel %s cannot be resident (smem %zu)", k.name.c_str(), k.smem); }
    }
    L.fns.push_back(f);
    L.occupancy.push_back(occ);
  }
  auto ins = m->per_device.emplace(dev, std::move(L));
  *out = &ins.first->second;
  return CX_OK;
}

// The cube scan of a shared program compiled with one batch layout as
// constants: the program's prelude, `#define`s of the CXS_* layout macros
// (values from the batch's arguments) and the program's cube region.  Cached
// per layout and device; *fn stays null (the generic kernel runs) if the
// program has no cube region or the compile fails.
int cube_spec_function(cx_module* m, int dev, const CxArgs& a, const std::string& kname, size_t smem_max, CUfunction* fn) {
  *fn = nullptr;
  const std::string& src = m->source;
  const size_t p0 = src.find("@*/"), p1 = src.find("//@cx-prelude-end");
  const size_t r0 = src.find("//@cx-cube-begin"), r1 = src.find("//@cx-cube-end");
  if (p0 == std::string::npos || p1 == std::string::npos || r0 == std::string::npos || r1 == std::string::npos) return CX_OK;
  std::string region = src.substr(r0, r1 - r0);
  // Default lines: "#define NAME (a.field[idx])" or "#define NAME (a.field)".
  std::string defs = "#define CXS_SPEC 1\n";
  std::istringstream in(region);
  std::string line;
  auto value = [&](const std::string& f, int i, bool* ok) -> long long {
    *ok = true;
    auto in_range = [&](int n) { if (i < 0 || i >= n) *ok = false; return *ok; };
    if (f == "cube_dsm_bytes") return a.cube_dsm_bytes;
    if (f == "cube_smem_words") return a.cube_smem_words;
    if (f == "cube_dsm" && in_range(CX_MAX_HTS)) return a.cube_dsm[i];
    if (f == "cube_dgl" && in_range(CX_MAX_HTS)) return a.cube_dgl[i];
    if (f == "cube_desz" && in_range(CX_MAX_HTS)) return a.cube_desz[i];
    if (f == "cube_dbase" && in_range(CX_MAX_HTS)) return a.cube_dbase[i];
    if (f == "cube_dlen" && in_range(CX_MAX_HTS)) return a.cube_dlen[i];
    if (f == "cube_fsh" && in_range(CX_MAX_HTS * 4)) return a.cube_fsh[i];
    if (f == "cube_fmk" && in_range(CX_MAX_HTS * 4)) return a.cube_fmk[i];
    if (f == "cube_stride" && in_range(CX_MAX_SHAPES * CX_MAX_SATTRS)) return a.cube_stride[i];
    if (f == "cube_smem" && in_range(CX_MAX_SHAPES)) return a.cube_smem[i];
    if (f == "cube_cells" && in_range(CX_MAX_SHAPES)) return a.cube_cells[i];
    if (f == "cube_lo" && in_range(CX_MAX_CATTRS)) return a.cube_lo[i];
    if (f == "cube_radix" && in_range(CX_MAX_CATTRS)) return a.cube_radix[i];
    *ok = false;
    return 0;
  };
  while (std::getline(in, line)) {
    if (line.rfind("#define CXS_", 0) != 0) continue;
    std::istringstream ls(line);
    std::string def, name, expr;
    ls >> def >> name >> expr;
    // expr: "(a.field[idx])" or "(a.field)"
    if (expr.size() < 5 || expr.compare(0, 3, "(a.") != 0) return CX_OK;
    std::string body = expr.substr(3, expr.size() - 4);
    int idx = -1;
    const size_t lb = body.find('[');
    if (lb != std::string::npos) {
      idx = atoi(body.c_str() + lb + 1);
      body = body.substr(0, lb);
    }
    bool ok = false;
    const long long v = value(body, idx, &ok);
    if (!ok) return CX_OK;
    defs += "#define " + name + " (" + std::to_string(v) + (body == "cube_cells" ? "LL" : "") + ")\n";
  }
  std::lock_guard<std::mutex> lk(m->mu);
  cx_module::Spec& sp = m->cube_specs[defs][dev];
  if (sp.fn || sp.failed) { *fn = sp.fn; return CX_OK; }
  const std::string prog_src = src.substr(p0 + 3, p1 - p0 - 3) + "\n" + defs + region;
  nvrtcProgram prog;
  const char* headers[] = {kCxEmbeddedCrystalHeader, kCxEmbeddedArgsHeader};
  const char* names[] = {"crystal_sm100.cuh", "cx_args.h"};
  sp.failed = true;
  if (nvrtcCreateProgram(&prog, prog_src.c_str(), "cx_cube_layout.cu", 2, headers, names) != NVRTC_SUCCESS) return CX_OK;
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};
  const bool compiled = nvrtcCompileProgram(prog, 4, opts) == NVRTC_SUCCESS;
  std::vector<char> cubin;
  if (compiled) {
    size_t csz = 0;
    nvrtcGetCUBINSize(prog, &csz);
    cubin.resize(csz);
    nvrtcGetCUBIN(prog, cubin.data());
  }
  nvrtcDestroyProgram(&prog);
  if (!compiled) return CX_OK;
  Driver& d = driver();
  if (d.ModuleLoadData(&sp.mod, cubin.data()) != CUDA_SUCCESS) { sp.mod = nullptr; return CX_OK; }
  CUfunction f = nullptr;
  if (d.ModuleGetFunction(&f, sp.mod, kname.c_str()) != CUDA_SUCCESS ||
      d.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem_max) != CUDA_SUCCESS) {
    d.ModuleUnload(sp.mod);
    sp.mod = nullptr;
    return CX_OK;
  }
  sp.fn = f;
  sp.failed = false;
  *fn = f;
  return CX_OK;
}

int ensure_ctx_device(cx_exec_ctx* c, int dev) {
  if (c->device == dev && c->ev[0]) return CX_OK;
  if (c->ev[0]) {
    for (auto& e : c->ev) { cudaEventDestroy(e); e = nullptr; }
  }
  for (auto& e : c->ev) CX_CUDA(cudaEventCreate(&e));
  if (!c->host_err) CX_CUDA(cudaMallocHost((void**)&c->host_err, sizeof(unsigned int)));
  c->device = dev;
  return CX_OK;
}

// Layout of a batch's aggregate cubes: per attribute its registered range, per
// shape with queries its cell count, mixed-radix strides (last attribute
// varies fastest), global cube offset and, when it fits the per-CTA budget, its
// shared-memory offset.  `why` says why the batch keeps the per-query path.
struct CubePlan {
  bool on = false;
  std::string why;
  std::vector<int> lo, radix;
  std::vector<uint64_t> cells, goff;
  std::vector<std::vector<int>> stride;
  std::vector<int> smem_off;
  uint64_t smem_words = 0, gbytes = 0;
  int chunks = 1;
  std::vector<std::vector<int>> fdsrc;   // per shape and attribute position: source position, -1 none
  std::vector<const int*> fdtab;          // per attribute: its table from the source's value offset
  // Dimensions kept in shared memory as compact words: byte offset (-1: none),
  // bytes per word, per field bit shift and mask, scratch offset and size of
  // the array the index kernel writes.
  std::vector<int> dsm, dgl, desz, dbase, dlen, fsh, fmk;
  std::vector<char> used;                 // per shape: the batch has queries of it
  std::vector<uint64_t> dcomp_off, dcomp_bytes;
  uint64_t dsm_bytes = 0;
};

// Cache key of "column B of a dimension determines column A" on a context:
// both columns' names, buffers, the table's rows and the registered ranges.
bool fd_key(const LaunchPlan& lp, const cx_exec_ctx* c, int a, int b, std::string* key, const int** pa,
            const int** pb, long long* rows) {
  const auto& A = lp.cattrs[a];
  const auto& B = lp.cattrs[b];
  auto ba = c->buffers.find(A.col), bb = c->buffers.find(B.col);
  auto ra = c->ranges.find(A.col), rb = c->ranges.find(B.col);
  if (ba == c->buffers.end() || bb == c->buffers.end() || ra == c->ranges.end() || rb == c->ranges.end()) return false;
  int table = -1;
  for (const auto& col : lp.cols)
    if (col.name == A.col) table = col.table;
  if (table < 0 || table >= (int)lp.tables.size()) return false;
  auto rt = c->rows.find(lp.tables[table]);
  if (rt == c->rows.end()) return false;
  *pa = (const int*)ba->second.first;
  *pb = (const int*)bb->second.first;
  *rows = (long long)rt->second;
  char buf[512];
  snprintf(buf, sizeof buf, "%s|%s|%p|%p|%lld|%lld|%lld|%lld|%lld", A.col.c_str(), B.col.c_str(), (const void*)*pa,
           (const void*)*pb, *rows, (long long)ra->second.first, (long long)ra->second.second,
           (long long)rb->second.first, (long long)rb->second.second);
  *key = buf;
  return true;
}

// Checks, once per context and column pair, which cube attributes of one
// dimension determine which others (on `s`, then waits for it).
int ensure_cube_fds(const LaunchPlan& lp, cx_exec_ctx* c, cudaStream_t s) {
  if (!lp.cube) return CX_OK;
  struct Todo { std::string key; int* tab; };
  std::vector<Todo> todo;
  std::vector<std::tuple<const int*, const int*, long long, int, int, int>> args;
  for (size_t a = 0; a < lp.cattrs.size(); ++a)
    for (size_t b = 0; b < lp.cattrs.size(); ++b) {
      if (a == b || lp.cattrs[a].dim < 0 || lp.cattrs[a].dim != lp.cattrs[b].dim) continue;
      std::string key;
      const int *pa = nullptr, *pb = nullptr;
      long long rows = 0;
      if (!fd_key(lp, c, (int)a, (int)b, &key, &pa, &pb, &rows) || c->fds.count(key)) continue;
      const auto& ra = c->ranges.at(lp.cattrs[a].col);
      const auto& rb = c->ranges.at(lp.cattrs[b].col);
      const int64_t radix_b = rb.second - rb.first + 1;
      if (radix_b <= 0 || radix_b > 65536 || ra.second - ra.first + 1 > 65536 || !pa || !pb) {
        c->fds[key] = cx_exec_ctx::Fd{};
        continue;
      }
      todo.push_back({key, nullptr});
      args.emplace_back(pa, pb, rows, (int)ra.first, (int)rb.first, (int)radix_b);
    }
  if (todo.empty()) return CX_OK;
  unsigned* flags = nullptr;
  CX_CUDA(cudaMalloc(&flags, todo.size() * sizeof(unsigned)));
  int rc = CX_OK;
  if (cudaMemsetAsync(flags, 0, todo.size() * sizeof(unsigned), s) != cudaSuccess) rc = fail(CX_E_CUDA, "fd check: memset");
  for (size_t i = 0; i < todo.size() && rc == CX_OK; ++i) {
    const auto& t = args[i];
    if (cudaMalloc(&todo[i].tab, (size_t)std::get<5>(t) * sizeof(int)) != cudaSuccess) { rc = fail(CX_E_CUDA, "fd check: cudaMalloc"); break; }
    rc = cx_internal::fd_check_launch(std::get<0>(t), std::get<1>(t), std::get<2>(t), std::get<3>(t), std::get<4>(t),
                                      std::get<5>(t), todo[i].tab, flags + i, s);
  }
  std::vector<unsigned> host(todo.size(), 1u);
  if (rc == CX_OK && cudaMemcpyAsync(host.data(), flags, todo.size() * sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = fail(CX_E_CUDA, "fd check: copy");
  if (rc == CX_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(CX_E_CUDA, "fd check: sync");
  cudaFree(flags);
  for (size_t i = 0; i < todo.size(); ++i) {
    cx_exec_ctx::Fd f;
    f.holds = rc == CX_OK && host[i] == 0u && todo[i].tab;
    if (f.holds) f.tab = todo[i].tab;
    else if (todo[i].tab) cudaFree(todo[i].tab);
    if (rc == CX_OK) c->fds[todo[i].key] = f;
  }
  return rc;
}

constexpr uint64_t kCubeMaxCells = 1ULL << 24;
constexpr uint64_t kCubeMaxGlobalBytes = 8ULL << 30;
constexpr uint64_t kCubeSmemBudget = 96 * 1024;
constexpr uint64_t kCubeCellsPerChunk = 16384;
constexpr uint64_t kDimSmemBudget = 96 * 1024;
constexpr int64_t kDimGlobalKeys = 1LL << 26;  // keys of a dimension whose words may live in global memory

bool plan_cubes(const LaunchPlan& lp, const cx_exec_ctx* c, const int* shapes, int nq, CubePlan& cp) {
  const int nshapes = (int)lp.sshapes.size();
  if (!lp.cube || (int)lp.cshapes.size() != nshapes) { cp.why = "program has no cube path"; return false; }
  std::vector<char>& used = cp.used;
  used.assign(nshapes, 0);
  for (int q = 0; q < nq; ++q)
    if (shapes[q] >= 0 && shapes[q] < nshapes) used[shapes[q]] = 1;
  for (const auto& at : lp.cattrs) {
    auto it = c->ranges.find(at.col);
    if (it == c->ranges.end()) { cp.why = "no registered range for " + at.col; return false; }
    const int64_t lo = it->second.first, hi = it->second.second;
    if (lo < INT32_MIN || hi > INT32_MAX || hi - lo + 1 > 65536) { cp.why = "range of " + at.col + " exceeds 65,536 values"; return false; }
    cp.lo.push_back((int)lo);
    cp.radix.push_back((int)(hi - lo + 1));
  }
  // Dimension attributes determined by another attribute of their dimension
  // (checked functional dependencies): the attribute with the most values is
  // kept first, and an attribute that a kept one determines takes no part in
  // the cells of a shape that also reads its source.
  const int na = (int)lp.cattrs.size();
  std::vector<int> src(na, -1), kept, by_radix(na);
  cp.fdtab.assign(na, nullptr);
  for (int a = 0; a < na; ++a) by_radix[a] = a;
  std::stable_sort(by_radix.begin(), by_radix.end(), [&](int x, int y) { return cp.radix[x] > cp.radix[y]; });
  for (int a : by_radix) {
    if (lp.cattrs[a].dim >= 0)
      for (int b : kept) {
        if (lp.cattrs[b].dim != lp.cattrs[a].dim) continue;
        std::string key;
        const int *pa = nullptr, *pb = nullptr;
        long long rows = 0;
        if (!fd_key(lp, c, a, b, &key, &pa, &pb, &rows)) continue;
        auto it = c->fds.find(key);
        if (it == c->fds.end() || !it->second.holds) continue;
        src[a] = b;
        cp.fdtab[a] = it->second.tab;
        break;
      }
    if (src[a] < 0) kept.push_back(a);
  }
  cp.cells.assign(nshapes, 0);
  cp.goff.assign(nshapes, 0);
  cp.stride.assign(nshapes, std::vector<int>(CX_MAX_SATTRS, 0));
  cp.fdsrc.assign(nshapes, std::vector<int>(CX_MAX_SATTRS, -1));
  cp.smem_off.assign(nshapes, -1);
  // Every shape's cells and strides, used by the batch or not, so that the
  // layout (and the scan compiled for it) stays the same from batch to batch;
  // global cubes only for the shapes the batch uses.
  uint64_t g = 0, maxcells = 0;
  for (int s = 0; s < nshapes; ++s) {
    const auto& sh = lp.cshapes[s];
    for (size_t j = 0; j < sh.attrs.size(); ++j) {
      const int b = src[sh.attrs[j]];
      if (b < 0) continue;
      for (size_t k = 0; k < sh.attrs.size(); ++k)
        if (sh.attrs[k] == b) cp.fdsrc[s][j] = (int)k;
    }
    uint64_t cells = 1;
    for (size_t j = sh.attrs.size(); j-- > 0 && cells <= kCubeMaxCells;) {
      if (cp.fdsrc[s][j] >= 0) continue;  // stride 0: the source attribute's offset decides it
      cp.stride[s][j] = (int)cells;
      cells *= (uint64_t)cp.radix[sh.attrs[j]];
    }
    if (cells > kCubeMaxCells) {
      if (used[s]) { cp.why = "a shape's cube exceeds 16,777,216 cells"; return false; }
      std::fill(cp.stride[s].begin(), cp.stride[s].end(), 0);
      continue;  // cells 0: never placed, never updated (no query of the shape)
    }
    cp.cells[s] = cells;
    if (!used[s]) continue;
    cp.goff[s] = g;
    g = align256(g + cells * (uint64_t)(sh.nsums + 1) * 8);
    maxcells = std::max(maxcells, cells);
  }
  if (g > std::min(kCubeMaxGlobalBytes, c->cube_cap)) { cp.why = "the batch's cubes exceed the context's cube budget"; return false; }
  cp.gbytes = g;
  // Shared-memory copies for the smallest cubes first, within the per-CTA budget.
  std::vector<int> order;
  for (int s = 0; s < nshapes; ++s)
    if (cp.cells[s]) order.push_back(s);
  std::sort(order.begin(), order.end(), [&](int x, int y) { return cp.cells[x] < cp.cells[y]; });
  uint64_t words = 0;
  for (int s : order) {
    // Per SUM aggregate a low and a high 32-bit word per cell, then a 32-bit row count.
    const uint64_t w = (cp.cells[s] * (uint64_t)(2 * lp.cshapes[s].nsums + 1) + 1) / 2;
    if ((words + w) * 8 > kCubeSmemBudget) continue;
    cp.smem_off[s] = (int)words;
    words += w;
  }
  cp.smem_words = words;
  cp.chunks = (int)std::max<uint64_t>(1, std::min<uint64_t>(4096, (maxcells + kCubeCellsPerChunk - 1) / kCubeCellsPerChunk));
  // Dimensions whose compact words (present bit, one bit per shape, the
  // attribute offsets) fit in 32 bits and whose key ranges, one word per key,
  // fit the budget together.
  const int nd = (int)lp.cdims.size();
  cp.dsm.assign(CX_MAX_HTS, -1);
  cp.dgl.assign(CX_MAX_HTS, 0);
  cp.desz.assign(CX_MAX_HTS, 0);
  cp.dbase.assign(CX_MAX_HTS, 0);
  cp.dlen.assign(CX_MAX_HTS, 0);
  cp.fsh.assign(CX_MAX_HTS * 4, 0);
  cp.fmk.assign(CX_MAX_HTS * 4, 0);
  cp.dcomp_off.assign(CX_MAX_HTS, 0);
  cp.dcomp_bytes.assign(CX_MAX_HTS, 0);
  std::vector<std::pair<uint64_t, int>> cand;
  for (int d = 0; d < nd && d < CX_MAX_HTS; ++d) {
    const auto& cd = lp.cdims[d];
    auto rp = c->ranges.find(cd.pk);
    if (rp == c->ranges.end()) continue;
    const int64_t klo = rp->second.first, kn = rp->second.second - rp->second.first + 1;
    if (klo < INT32_MIN || rp->second.second > INT32_MAX || kn <= 0 || kn > kDimGlobalKeys) continue;
    int bits = 1 + nshapes;
    int fw[4] = {0, 0, 0, 0};
    for (size_t a = 0; a < lp.cattrs.size(); ++a) {
      if (lp.cattrs[a].dim != d) continue;
      int w = 1;
      while ((1LL << w) < (long long)cp.radix[a]) ++w;
      fw[lp.cattrs[a].field] = w;
    }
    for (int f = 0; f < 4; ++f) {
      if (!fw[f]) continue;
      cp.fsh[d * 4 + f] = bits;
      cp.fmk[d * 4 + f] = (int)((1u << fw[f]) - 1u);
      bits += fw[f];
    }
    if (bits > 32) continue;
    cp.desz[d] = bits <= 8 ? 1 : bits <= 16 ? 2 : 4;
    cp.dbase[d] = (int)klo;
    cp.dlen[d] = (int)kn;
    cp.dcomp_bytes[d] = ((uint64_t)kn * (uint64_t)cp.desz[d] + 15) & ~15ULL;
    cand.emplace_back(cp.dcomp_bytes[d], d);
  }
  std::sort(cand.begin(), cand.end());
  uint64_t dbytes = 0;
  // Smallest first into shared memory; the rest keep their words in global
  // memory (one 1-4 byte gather per row instead of a 16-byte entry).
  for (const auto& cd : cand) {
    if (dbytes + cd.first > kDimSmemBudget) { cp.dgl[cd.second] = 1; continue; }
    cp.dsm[cd.second] = (int)dbytes;
    dbytes += cd.first;
  }
  cp.dsm_bytes = dbytes;
  cp.on = true;
  return true;
}

// The kernel arguments of a cube layout (`scratch` null: no buffers, for a
// compile of the layout ahead of its first batch).
void fill_cube_args(CxArgs& a, const CubePlan& cp, int nshapes, char* scratch, uint64_t cube_off) {
  for (size_t id = 0; id < cp.lo.size(); ++id) { a.cube_lo[id] = cp.lo[id]; a.cube_radix[id] = cp.radix[id]; }
  for (size_t id = 0; id < cp.fdtab.size(); ++id) a.cube_fdtab[id] = cp.fdtab[id];
  for (int s = 0; s < nshapes && s < CX_MAX_SHAPES; ++s) {
    for (int j = 0; j < CX_MAX_SATTRS; ++j) {
      a.cube_stride[s * CX_MAX_SATTRS + j] = cp.stride[s][j];
      a.cube_fdsrc[s * CX_MAX_SATTRS + j] = cp.fdsrc[s][j];
    }
    a.cube_g[s] = scratch && cp.used[s] && cp.cells[s] ? (unsigned long long*)(scratch + cube_off + cp.goff[s]) : nullptr;
    a.cube_cells[s] = (long long)cp.cells[s];
    a.cube_smem[s] = cp.smem_off[s];
  }
  a.cube_smem_words = (int)cp.smem_words;
  a.cube_chunks = cp.chunks;
  for (int d = 0; d < CX_MAX_HTS; ++d) {
    a.cube_dsm[d] = cp.dsm[d];
    a.cube_dgl[d] = cp.dgl[d];
    a.cube_desz[d] = cp.desz[d];
    a.cube_dbase[d] = cp.dbase[d];
    a.cube_dlen[d] = cp.dlen[d];
    a.cube_dcomp[d] = scratch && cp.dcomp_bytes[d] ? (unsigned char*)(scratch + cp.dcomp_off[d]) : nullptr;
    for (int f = 0; f < 4; ++f) { a.cube_fsh[d * 4 + f] = cp.fsh[d * 4 + f]; a.cube_fmk[d * 4 + f] = cp.fmk[d * 4 + f]; }
  }
  a.cube_dsm_bytes = (int)cp.dsm_bytes;
}


}  // namespace

// ============================================================ internal ===
namespace cx_internal {

void ctx_copy_tables(const cx_exec_ctx* src, cx_exec_ctx* dst) {
  dst->buffers = src->buffers;
  dst->nulls = src->nulls;
  dst->rows = src->rows;
  dst->ranges = src->ranges;
}

bool ctx_column_range(const cx_exec_ctx* c, const std::string& name, int64_t* lo, int64_t* hi) {
  auto it = c->ranges.find(name);
  if (it == c->ranges.end()) return false;
  *lo = it->second.first;
  *hi = it->second.second;
  return true;
}

uint64_t ctx_scratch_bytes(const cx_exec_ctx* c) { return c->own_scratch_bytes; }

void ctx_set_cube_cap(cx_exec_ctx* c, uint64_t bytes) { c->cube_cap = bytes; }

int ensure_cube_dependencies(const cx_module* m, cx_exec_ctx* c, cudaStream_t s) {
  return m ? ensure_cube_fds(m->lp, c, s) : CX_OK;
}

int prepare_cube_layout(cx_module* m, cx_exec_ctx* c, cudaStream_t s) {
  if (!m || !c || !m->lp.cube) return CX_OK;
  int rc = ensure_cube_fds(m->lp, c, s);
  if (rc) return rc;
  std::vector<int> all(m->lp.sshapes.size());
  for (size_t i = 0; i < all.size(); ++i) all[i] = (int)i;
  CubePlan cp;
  if (!plan_cubes(m->lp, c, all.data(), (int)all.size(), cp)) return CX_OK;  // batches will take the mask path
  size_t ki = 0;
  while (ki < m->lp.kernels.size() && m->lp.kernels[ki].kind != "cubescan") ++ki;
  if (ki == m->lp.kernels.size()) return CX_OK;
  int dev = 0;
  CX_CUDA(cudaGetDevice(&dev));
  CxArgs a;
  memset(&a, 0, sizeof a);
  fill_cube_args(a, cp, (int)m->lp.sshapes.size(), nullptr, 0);
  CUfunction fn = nullptr;
  return cube_spec_function(m, dev, a, m->lp.kernels[ki].name, 227 * 1024, &fn);
}

int set_error(int code, const std::string& msg) { return fail(code, "%s", msg.c_str()); }

uint64_t module_fact_rows(const cx_module* m, const cx_exec_ctx* c) {
  if (!m || !c || m->lp.tables.empty()) return 0;
  auto it = c->rows.find(m->lp.tables[0]);
  return it == c->rows.end() ? 0 : it->second;
}

void module_retain(cx_module* m) {
  if (m) m->refs.fetch_add(1);
}

cx::Tuning to_tuning(const cx_tuning* tuning) {
  cx::Tuning t;
  if (tuning) {
    t.block_threads = tuning->block_threads;
    t.items_per_thread = tuning->items_per_thread;
    t.stages = tuning->stages;
    t.ctas_per_sm = tuning->ctas_per_sm;
    t.group_placement = tuning->group_placement;
    t.smem_group_budget = tuning->smem_group_budget;
    t.bitmap_budget = tuning->bitmap_budget;
    t.group_merge = tuning->group_merge;
    t.producer_warps = tuning->producer_warps;
    t.parametric = tuning->parametric;
    t.prefetch = tuning->prefetch;
    t.wait_limit_us = tuning->wait_limit_us;
    t.debug_stall = tuning->debug_stall;
    t.compact = tuning->compact;
    t.table_budget = tuning->table_budget;
    t.cube = tuning->cube;
  }
  return t;
}

uint64_t grown_scratch(uint64_t own, uint64_t need) { return own >= need ? own : need + need / 2; }

uint64_t shared_scratch_need(const cx_module* m, const cx_exec_ctx* c, const int* shapes, int nq) {
  const LaunchPlan& lp = m->lp;
  CubePlan cp;
  const bool cube = c && plan_cubes(lp, c, shapes, nq, cp);
  uint64_t off = 0;
  for (const auto& h : lp.hts) {
    if (!(cube && h.slot >= 0 && h.slot < CX_MAX_HTS && cp.desz[h.slot] > 0)) off = align256(off + h.words * 4);
    auto it = lp.dat_words.find(h.slot);
    if (!cube && it != lp.dat_words.end()) off = align256(off + it->second * 4);
  }
  for (int i = 0; i < nq; ++i) {
    if (shapes[i] < 0 || shapes[i] >= (int)lp.sshapes.size()) continue;
    const auto& sh = lp.sshapes[shapes[i]];
    if (sh.grouped) off = align256(off + ((sh.groups + 31) / 32) * 4);
  }
  if (cube) {
    off = align256(off + cp.gbytes);
    for (int d = 0; d < CX_MAX_HTS; ++d) off = align256(off + cp.dcomp_bytes[d]);
  }
  const int maxq = cube ? std::max(nq, 1) : std::max(1, std::min(lp.shared_maxq, 256));
  const int npass = (nq + maxq - 1) / maxq;
  int maxp = lp.shared_maxp;
  if (cube) {
    int np = 0;
    for (int i = 0; i < nq; ++i)
      if (shapes[i] >= 0 && shapes[i] < (int)lp.sshapes.size()) np += lp.sshapes[shapes[i]].nlits;
    maxp = std::max(maxp, np);
  }
  const uint64_t pass_bytes = align256((uint64_t)maxq * sizeof(CxSQ) + (uint64_t)std::max(maxp, 1) * 4);
  off += (uint64_t)std::max(npass, 1) * pass_bytes;
  return align256(off + 16);
}

}  // namespace cx_internal

// ================================================================== C ABI ===
extern "C" {

int cx_abi_version(void) { return CX_ABI_VERSION; }
const char* cx_last_error(void) { return g_last_error.c_str(); }

void cx_tuning_default(cx_tuning* t) {
  if (!t) return;
  cx::Tuning d;
  t->block_threads = d.block_threads;
  t->items_per_thread = d.items_per_thread;
  t->stages = d.stages;
  t->ctas_per_sm = d.ctas_per_sm;
  t->group_placement = d.group_placement;
  t->smem_group_budget = d.smem_group_budget;
  t->bitmap_budget = d.bitmap_budget;
  t->group_merge = d.group_merge;
  t->producer_warps = d.producer_warps;
  t->parametric = d.parametric;
  t->prefetch = d.prefetch;
  t->wait_limit_us = d.wait_limit_us;
  t->debug_stall = d.debug_stall;
  t->compact = d.compact;
  t->table_budget = d.table_budget;
  t->cube = d.cube;
}

int cx_codegen(const char* plan, size_t plan_len, const cx_tuning* tuning, char* out, size_t out_cap, size_t* out_len) {
  if (!plan) return fail(CX_E_INVALID, "cx_codegen: plan is NULL");
  try {
    auto p = cx::parse_plan(std::string(plan, plan_len));
    const cx::Tuning t = cx_internal::to_tuning(tuning);
    const std::string s = cx::generate_cuda(*p, t);
    if (out_len) *out_len = s.size();
    if (out && out_cap) {
      const size_t n = s.size() < out_cap - 1 ? s.size() : out_cap - 1;
      memcpy(out, s.data(), n);
      out[n] = '\0';
      if (n < s.size()) return fail(CX_E_CAPACITY, "cx_codegen: output buffer too small (%zu < %zu)", out_cap, s.size() + 1);
    }
    return CX_OK;
  } catch (const std::exception& e) {
    return fail(CX_E_INVALID, "%s", e.what());
  }
}

int cx_compile(const char* src, size_t src_len, const char* key, cx_module** out, char* log, size_t log_cap) {
  if (!src || !out) return fail(CX_E_INVALID, "cx_compile: NULL argument");
  if (log && log_cap) log[0] = '\0';
  std::string source(src, src_len);
  // A program from the reference's code generator (SYCL launch skeleton) is
  // translated to this library's skeleton first.
  if (cx_internal::is_visitor_program(source)) {
    try {
      source = cx_internal::translate_visitor_program(source);
    } catch (const std::exception& e) {
      return fail(CX_E_INVALID, "cx_compile: %s", e.what());
    }
  }
  const size_t h = std::hash<std::string>{}(source);
  std::string ck = key ? std::string(key) : std::string();
  if (ck.empty()) ck = "anon_" + std::to_string(h);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(ck);
    if (it != g_cache.end() && it->second->src_hash == h) {
      it->second->refs.fetch_add(1);
      *out = it->second;
      return CX_OK;
    }
  }
  auto m = std::make_unique<cx_module>();
  static std::atomic<uint64_t> next_uid{1};
  m->key = ck;
  m->src_hash = h;
  m->uid = next_uid.fetch_add(1);
  std::string perr;
  if (!parse_launch_plan(source, m->lp, perr)) return fail(CX_E_INVALID, "cx_compile: %s", perr.c_str());
  m->sl = scratch_layout(m->lp);
  if (m->lp.cube) m->source = source;

  nvrtcProgram prog;
  const char* headers[] = {kCxEmbeddedCrystalHeader, kCxEmbeddedArgsHeader};
  const char* names[] = {"crystal_sm100.cuh", "cx_args.h"};
  nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "cx_query.cu", 2, headers, names);
  if (r != NVRTC_SUCCESS) return fail(CX_E_COMPILE, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};
  r = nvrtcCompileProgram(prog, 4, opts);
  size_t lsz = 0;
  nvrtcGetProgramLogSize(prog, &lsz);
  std::string plog(lsz, '\0');
  if (lsz) nvrtcGetProgramLog(prog, &plog[0]);
  if (log && log_cap) {
    const size_t n = plog.size() < log_cap - 1 ? plog.size() : log_cap - 1;
    memcpy(log, plog.data(), n);
    log[n] = '\0';
  }
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return fail(CX_E_COMPILE, "NVRTC compile failed: %s\n%.1500s", nvrtcGetErrorString(r), plog.c_str());
  }
  size_t csz = 0;
  nvrtcGetCUBINSize(prog, &csz);
  m->cubin.resize(csz);
  nvrtcGetCUBIN(prog, m->cubin.data());
  nvrtcDestroyProgram(&prog);

  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto it = g_cache.find(ck);
  if (it != g_cache.end()) {
    // Same key, different source: the newer program replaces the cache entry;
    // holders of the old module keep it alive through their references.
    if (it->second->refs.fetch_sub(1) == 1) {
      cx_module* old = it->second;
      for (auto& kv : old->per_device)
        if (kv.second.mod && driver().ok) driver().ModuleUnload(kv.second.mod);
      for (auto& sp : old->cube_specs)
        for (auto& kv : sp.second)
          if (kv.second.mod && driver().ok) driver().ModuleUnload(kv.second.mod);
      delete old;
    }
    g_cache.erase(it);
  }
  cx_module* raw = m.release();
  raw->refs.store(2);  // one for the cache, one for the caller
  g_cache[ck] = raw;
  *out = raw;
  return CX_OK;
}

int cx_module_release(cx_module* m) {
  if (!m) return CX_OK;
  if (m->refs.fetch_sub(1) == 1) {
    for (auto& kv : m->per_device)
      if (kv.second.mod && driver().ok) driver().ModuleUnload(kv.second.mod);
    for (auto& sp : m->cube_specs)
      for (auto& kv : sp.second)
        if (kv.second.mod && driver().ok) driver().ModuleUnload(kv.second.mod);
    delete m;
  }
  return CX_OK;
}

int cx_module_result_info(const cx_module* m, cx_result_info* info) {
  if (!m || !info) return fail(CX_E_INVALID, "cx_module_result_info: NULL argument");
  const LaunchPlan& lp = m->lp;
  info->groups = lp.groups;
  info->storage_ts = (uint32_t)lp.storage_ts;
  info->visible_ts = (uint32_t)lp.visible_ts;
  info->result_words = lp.result_words;
  info->validity_words = (lp.result_words + 63) / 64;
  info->finalized = lp.finalize ? 1 : 0;
  info->final_words = lp.finalize ? lp.groups * (uint64_t)lp.visible_ts : lp.result_words;
  info->sparse = lp.sparse;
  return CX_OK;
}

cx_exec_ctx* cx_ctx_create(void) { return new (std::nothrow) cx_exec_ctx(); }

void cx_ctx_destroy(cx_exec_ctx* c) {
  if (!c) return;
  if (c->pending && c->ev[3]) cudaEventSynchronize(c->ev[3]);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->own_scratch) cudaFree(c->own_scratch);
  if (c->host_err) cudaFreeHost(c->host_err);
  if (c->host_stage) cudaFreeHost(c->host_stage);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  for (auto& kv : c->fds)
    if (kv.second.tab) cudaFree(kv.second.tab);
  delete c;
}

int cx_ctx_set_buffer(cx_exec_ctx* c, const char* name, const void* p, uint64_t elems) {
  if (!c || !name) return fail(CX_E_INVALID, "cx_ctx_set_buffer: NULL argument");
  c->buffers[name] = {p, elems};
  return CX_OK;
}

int cx_ctx_set_null_bitmap(cx_exec_ctx* c, const char* name, const uint64_t* p, uint64_t words) {
  if (!c || !name) return fail(CX_E_INVALID, "cx_ctx_set_null_bitmap: NULL argument");
  c->nulls[name] = {p, words};
  return CX_OK;
}

int cx_ctx_set_table_rows(cx_exec_ctx* c, const char* table, uint64_t rows) {
  if (!c || !table) return fail(CX_E_INVALID, "cx_ctx_set_table_rows: NULL argument");
  if (rows > (1ULL << 40)) return fail(CX_E_INVALID, "cx_ctx_set_table_rows: %llu rows is out of range", (unsigned long long)rows);
  c->rows[table] = rows;
  return CX_OK;
}

int cx_ctx_set_result(cx_exec_ctx* c, uint64_t* r, uint64_t rw, uint64_t* v, uint64_t vw) {
  if (!c) return fail(CX_E_INVALID, "cx_ctx_set_result: NULL context");
  c->result = r;
  c->result_words = rw;
  c->validity = v;
  c->validity_words = vw;
  return CX_OK;
}

int cx_ctx_set_scratch(cx_exec_ctx* c, void* p, uint64_t bytes) {
  if (!c) return fail(CX_E_INVALID, "cx_ctx_set_scratch: NULL context");
  if (p && ((uintptr_t)p & 255)) return fail(CX_E_INVALID, "cx_ctx_set_scratch: scratch must be 256-byte aligned");
  c->user_scratch = p;
  c->user_scratch_bytes = p ? bytes : 0;
  return CX_OK;
}

int cx_ctx_set_sm_count(cx_exec_ctx* c, int sms) {
  if (!c || sms < 0) return fail(CX_E_INVALID, "cx_ctx_set_sm_count: bad argument");
  c->sm_override = sms;
  return CX_OK;
}

int cx_ctx_set_column_range(cx_exec_ctx* c, const char* name, int64_t lo, int64_t hi) {
  if (!c || !name || lo > hi) return fail(CX_E_INVALID, "cx_ctx_set_column_range: bad argument");
  c->ranges[name] = {lo, hi};
  return CX_OK;
}

int cx_module_scratch_bytes(const cx_module* m, const cx_exec_ctx* c, uint64_t* bytes) {
  if (!m || !bytes) return fail(CX_E_INVALID, "cx_module_scratch_bytes: NULL argument");
  *bytes = m->sl.total;
  if ((!m->lp.mht_table.empty() || m->lp.rows_sized) && c) {
    std::vector<long long> rows(m->lp.tables.size(), 0);
    for (size_t t = 0; t < m->lp.tables.size(); ++t) {
      auto it = c->rows.find(m->lp.tables[t]);
      if (it == c->rows.end()) return fail(CX_E_MISSING, "cx_module_scratch_bytes: row count of table %s is not set", m->lp.tables[t].c_str());
      rows[t] = (long long)it->second;
    }
    *bytes = scratch_layout(m->lp, &rows).total + mht_payload_bytes(m->lp, rows);
  }
  return CX_OK;
}

int cx_execute(cx_module* m, cx_exec_ctx* c, void* stream_v) { return cx_execute_params(m, c, nullptr, 0, stream_v); }

int cx_execute_params(cx_module* m, cx_exec_ctx* c, const int32_t* params, int nparams, void* stream_v) {
  if (!m || !c) return fail(CX_E_INVALID, "cx_execute: NULL argument");
  const LaunchPlan& lp = m->lp;
  if (lp.shared) return fail(CX_E_INVALID, "cx_execute: a shared-scan program runs through cx_shared_execute");
  cudaStream_t stream = (cudaStream_t)stream_v;

  // Resolve tables, columns and result buffers before touching the GPU.
  CxArgs a;
  memset(&a, 0, sizeof a);
  const int want = lp.nparams < 0 ? 0 : lp.nparams;
  if (nparams != want || (nparams > 0 && !params))
    return fail(CX_E_INVALID, "cx_execute: the module takes %d literal parameters, %d given", want, nparams);
  for (int k = 0; k < nparams; ++k) a.lits[k] = params[k];
  std::vector<long long> rows(lp.tables.size(), 0);
  for (size_t t = 0; t < lp.tables.size(); ++t) {
    auto it = c->rows.find(lp.tables[t]);
    if (it == c->rows.end()) return fail(CX_E_MISSING, "cx_execute: row count of table %s is not set", lp.tables[t].c_str());
    rows[t] = (long long)it->second;
    a.rows[t] = rows[t];
  }
  for (const auto& col : lp.cols) {
    auto it = c->buffers.find(col.name);
    if (it == c->buffers.end() || (!it->second.first && rows[col.table] > 0))
      return fail(CX_E_MISSING, "cx_execute: buffer %s is not in the execution context", col.name.c_str());
    if (it->second.second < (uint64_t)rows[col.table])
      return fail(CX_E_CAPACITY, "cx_execute: buffer %s holds %llu rows, table has %lld", col.name.c_str(),
                  (unsigned long long)it->second.second, rows[col.table]);
    a.col[col.slot] = (const int*)it->second.first;
  }
  for (const auto& nl : lp.nulls) {
    auto it = c->nulls.find(nl.second);
    if (it == c->nulls.end()) continue;  // no bitmap registered: every row valid (getNullBitmap -> nullptr)
    int table = 0;
    for (const auto& col : lp.cols)
      if (col.slot == nl.first) table = col.table;
    if (it->second.second < ((uint64_t)rows[table] + 63) / 64)
      return fail(CX_E_CAPACITY, "cx_execute: validity of %s is shorter than its table", nl.second.c_str());
    a.nul[nl.first] = (const unsigned long long*)it->second.first;
  }
  const uint64_t vwords = (lp.result_words + 63) / 64;
  if (!c->result || c->result_words < lp.result_words)
    return fail(CX_E_CAPACITY, "cx_execute: result buffer holds %llu words, query needs %llu",
                (unsigned long long)c->result_words, (unsigned long long)lp.result_words);
  if (!c->validity || c->validity_words < vwords)
    return fail(CX_E_CAPACITY, "cx_execute: validity buffer holds %llu words, query needs %llu",
                (unsigned long long)c->validity_words, (unsigned long long)vwords);
  a.result = (unsigned long long*)c->result;
  a.result_validity = (unsigned long long*)c->validity;

  int dev = 0;
  CX_CUDA(cudaGetDevice(&dev));
  int rc = ensure_ctx_device(c, dev);
  if (rc) return rc;
  cx_module::Loaded* L = nullptr;
  rc = load_on_device(m, dev, &L);
  if (rc) return rc;

  // Scratch: the plan's layout (hash tables sized by row counts where the plan
  // says so), then the MHT row-id payloads.
  const ScratchLayout sl = lp.rows_sized ? scratch_layout(lp, &rows) : m->sl;
  const uint64_t need = sl.total + mht_payload_bytes(lp, rows);
  char* scratch = nullptr;
  if (c->user_scratch) {
    if (c->user_scratch_bytes < need)
      return fail(CX_E_CAPACITY, "cx_execute: caller scratch holds %llu bytes, query needs %llu",
                  (unsigned long long)c->user_scratch_bytes, (unsigned long long)need);
    scratch = (char*)c->user_scratch;
  } else {
    if (c->own_scratch_bytes < need) {
      if (c->own_scratch) {
        if (c->pending) cudaEventSynchronize(c->ev[3]);
        cudaFree(c->own_scratch);
        c->own_scratch = nullptr;
        c->own_scratch_bytes = 0;
      }
      const uint64_t grow = need + need / 2;  // 1.5x high-water, as DynamicDeviceBuffer
      CX_CUDA(cudaMalloc(&c->own_scratch, grow));
      c->own_scratch_bytes = grow;
    }
    scratch = (char*)c->own_scratch;
  }
  for (size_t i = 0; i < lp.hts.size(); ++i) {
    a.ht[lp.hts[i].slot] = (int*)(scratch + sl.ht_off[i]);
    if (lp.htv_words.count(lp.hts[i].slot)) a.htv[lp.hts[i].slot] = (unsigned int*)(scratch + sl.htv_off[i]);
    if (lp.bm_words.count(lp.hts[i].slot)) a.bm[lp.hts[i].slot] = (unsigned int*)(scratch + sl.bm_off[i]);
  }
  a.touched = (unsigned int*)(scratch + sl.touched_off);
  a.finalize_tmp = (unsigned long long*)(scratch + sl.fin_off);
  a.err = (unsigned int*)(scratch + sl.err_off);
  {
    uint64_t off = sl.total;
    for (const auto& kv : lp.mht_table) {
      a.mpay[kv.first] = (int*)(scratch + off);
      off += mht_slot_bytes(lp, kv.first, rows[kv.second]);
    }
  }

  int sms = c->sm_override;
  if (sms <= 0) CX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  Driver& d = driver();
  int launches = 0, scan_grid = 0;
  void* kargs[] = {&a};
  auto launch = [&](size_t ki, unsigned grid) -> int {
    const KernelSpec& k = lp.kernels[ki];
    if (grid == 0) return CX_OK;
    CUresult r = d.LaunchKernel(L->fns[ki], grid, 1, 1, k.block, 1, 1, (unsigned)k.smem, (CUstream)stream, kargs, nullptr);
    if (r != CUDA_SUCCESS) return drv_fail(r, k.name.c_str());
    ++launches;
    return CX_OK;
  };

  CX_CUDA(cudaEventRecord(c->ev[0], stream));
  CX_CUDA(cudaMemsetAsync(scratch, 0, sl.total, stream));
  CX_CUDA(cudaMemsetAsync(c->result, 0, lp.result_words * 8, stream));
  CX_CUDA(cudaMemsetAsync(c->validity, 0, vwords * 8, stream));
  size_t ki = 0;
  // Phase 1: slot initialisation and hash-table builds.
  for (; ki < lp.kernels.size() && lp.kernels[ki].kind != "scan" && lp.kernels[ki].kind != "tilescan"; ++ki) {
    const KernelSpec& k = lp.kernels[ki];
    unsigned grid = 0;
    if (k.kind == "groups") grid = (unsigned)((lp.groups + k.block - 1) / k.block);
    else if (k.kind == "fixed") grid = (unsigned)k.table;
    else if (k.kind == "build") {
      const long long tiles = (rows[k.table] + k.tile - 1) / k.tile;
      grid = (unsigned)std::min<long long>(tiles, (long long)sms * 16);
    } else if (k.kind == "tiles") {
      // One CTA per tile of the table (a translated nd_range kernel).
      grid = (unsigned)((rows[k.table] + k.tile - 1) / k.tile);
    }
    if ((rc = launch(ki, grid))) return rc;
  }
  CX_CUDA(cudaEventRecord(c->ev[1], stream));
  // Phase 2: the fused scan.
  if (ki < lp.kernels.size() && lp.kernels[ki].kind == "tilescan") {
    const KernelSpec& k = lp.kernels[ki];
    const long long tiles = (rows[k.table] + k.tile - 1) / k.tile;
    if (tiles > 0x7fffffffLL) return fail(CX_E_CAPACITY, "cx_execute: %lld tiles exceed one grid", tiles);
    scan_grid = (int)tiles;
    if ((rc = launch(ki, (unsigned)tiles))) return rc;
    ++ki;
  } else if (ki < lp.kernels.size()) {
    const KernelSpec& k = lp.kernels[ki];
    const long long tiles = (rows[0] + k.tile - 1) / k.tile;
    const long long warps = std::max(1, k.block / 32);
    const int per_sm = std::max(1, std::min(k.ctas_per_sm, L->occupancy[ki]));
    const long long grid = std::min<long long>((tiles + warps - 1) / warps, (long long)sms * per_sm);
    scan_grid = (int)grid;
    if ((rc = launch(ki, (unsigned)grid))) return rc;
    ++ki;
  }
  CX_CUDA(cudaEventRecord(c->ev[2], stream));
  // Phase 3: epilogues.
  for (; ki < lp.kernels.size(); ++ki) {
    const KernelSpec& k = lp.kernels[ki];
    unsigned grid = (unsigned)((lp.groups + k.block - 1) / k.block);
    if ((rc = launch(ki, grid))) return rc;
  }
  if (lp.finalize) {
    const uint64_t vis = lp.fin_groups * (uint64_t)lp.fin_vts;
    CX_CUDA(cudaMemcpyAsync(c->result, a.finalize_tmp, vis * 8, cudaMemcpyDeviceToDevice, stream));
    CX_CUDA(cudaMemcpyAsync(c->validity, a.finalize_tmp + vis, ((vis + 63) / 64) * 8, cudaMemcpyDeviceToDevice, stream));
  }
  CX_CUDA(cudaMemcpyAsync(c->host_err, a.err, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
  CX_CUDA(cudaEventRecord(c->ev[3], stream));
  c->pending = true;
  c->timing = cx_timing{};
  c->timing.scan_grid = scan_grid;
  c->timing.gpu_launches = launches;
  return CX_OK;
}


int cx_plan_literals(const char* plan, size_t plan_len, int64_t* out, int cap, int* n) {
  if (!plan || !n) return fail(CX_E_INVALID, "cx_plan_literals: NULL argument");
  try {
    auto p = cx::parse_plan(std::string(plan, plan_len));
    std::vector<const cx::Expr*> lits;
    cx::collect_literals(*p, lits);
    *n = (int)lits.size();
    if (out)
      for (int i = 0; i < (int)lits.size() && i < cap; ++i) out[i] = lits[i]->ival;
    if (out && cap < (int)lits.size()) return fail(CX_E_CAPACITY, "cx_plan_literals: %d literals, capacity %d", (int)lits.size(), cap);
    return CX_OK;
  } catch (const std::exception& e) {
    return fail(CX_E_INVALID, "%s", e.what());
  }
}

int cx_shared_codegen(const char* const* plans, const size_t* lens, int nshapes, const cx_tuning* tuning, char* out,
                      size_t out_cap, size_t* out_len) {
  if (!plans || !lens || nshapes <= 0) return fail(CX_E_INVALID, "cx_shared_codegen: no shapes");
  try {
    std::vector<std::unique_ptr<cx::Plan>> owned;
    std::vector<const cx::Plan*> shapes;
    for (int i = 0; i < nshapes; ++i) {
      owned.push_back(cx::parse_plan(std::string(plans[i], lens[i])));
      shapes.push_back(owned.back().get());
    }
    cx::Tuning t = cx_internal::to_tuning(tuning);
    if (!tuning) {
      // Shared scans default to one 32-warp CTA per SM, one row per thread
      // and a 3-deep staging ring.
      t.block_threads = 1024;
      t.items_per_thread = 1;
      t.stages = 3;
      t.ctas_per_sm = 1;
    }
    const std::string src = cx::generate_shared_cuda(shapes, t);
    if (out_len) *out_len = src.size();
    if (out && out_cap) {
      const size_t n = src.size() < out_cap - 1 ? src.size() : out_cap - 1;
      memcpy(out, src.data(), n);
      out[n] = '\0';
      if (n < src.size()) return fail(CX_E_CAPACITY, "cx_shared_codegen: output buffer too small");
    }
    return CX_OK;
  } catch (const std::exception& e) {
    return fail(CX_E_INVALID, "%s", e.what());
  }
}

int cx_shared_execute(cx_module* m, cx_exec_ctx* c, const cx_shared_query* queries, int nq, const int32_t* params,
                      int nparams, void* stream_v) {
  return cx_shared_execute_rows(m, c, queries, nq, params, nparams, 0, UINT64_MAX, nullptr, stream_v);
}

int cx_shared_execute_rows(cx_module* m, cx_exec_ctx* c, const cx_shared_query* queries, int nq, const int32_t* params,
                           int nparams, uint64_t row0, uint64_t nrows, const uint8_t* keep, void* stream_v) {
  if (!m || !c || (!queries && nq > 0) || nq < 0 || nparams < 0 || (nparams > 0 && !params))
    return fail(CX_E_INVALID, "cx_shared_execute: bad argument");
  const LaunchPlan& lp = m->lp;
  if (!lp.shared) return fail(CX_E_INVALID, "cx_shared_execute: not a shared-scan program");
  if (nq > 256 || nparams > 4096) return fail(CX_E_CAPACITY, "cx_shared_execute: batch of %d queries / %d parameters exceeds 256 / 4096", nq, nparams);
  cudaStream_t stream = (cudaStream_t)stream_v;
  const int nshapes = (int)lp.sshapes.size();

  CxArgs a;
  memset(&a, 0, sizeof a);
  std::vector<long long> rows(lp.tables.size(), 0);
  for (size_t t = 0; t < lp.tables.size(); ++t) {
    auto it = c->rows.find(lp.tables[t]);
    if (it == c->rows.end()) return fail(CX_E_MISSING, "cx_shared_execute: row count of table %s is not set", lp.tables[t].c_str());
    rows[t] = (long long)it->second;
    a.rows[t] = rows[t];
  }
  // The fact-table rows this launch scans: [row0, row0 + nrows), clipped to the table.
  const uint64_t fact_rows = lp.tables.empty() ? 0 : (uint64_t)rows[0];
  if (row0 > fact_rows) return fail(CX_E_INVALID, "cx_shared_execute: row range starts past the fact table");
  const uint64_t range_rows = std::min<uint64_t>(nrows, fact_rows - row0);
  if (!lp.tables.empty()) a.rows[0] = (long long)range_rows;
  for (const auto& col : lp.cols) {
    auto it = c->buffers.find(col.name);
    if (it == c->buffers.end() || (!it->second.first && rows[col.table] > 0))
      return fail(CX_E_MISSING, "cx_shared_execute: buffer %s is not in the execution context", col.name.c_str());
    if (it->second.second < (uint64_t)rows[col.table])
      return fail(CX_E_CAPACITY, "cx_shared_execute: buffer %s is shorter than its table", col.name.c_str());
    a.col[col.slot] = (const int*)it->second.first + (col.table == 0 ? row0 : 0);
  }
  // Filter-table windows from the registered column ranges.
  for (const auto& fc : lp.fcols) {
    auto it = c->ranges.find(fc.second);
    a.fbase[fc.first] = 0;
    a.fwin[fc.first] = 0;
    if (it == c->ranges.end()) continue;
    const int64_t lo = std::max<int64_t>(it->second.first, INT32_MIN);
    const int64_t hi = std::min<int64_t>(it->second.second, INT32_MAX);
    if (lo > hi) continue;
    a.fbase[fc.first] = (int)lo;
    a.fwin[fc.first] = (int)std::min<int64_t>(256, hi - lo + 1);
  }
  // Queries grouped by shape; validate every query before touching the GPU.
  std::vector<int> order;
  for (int s = 0; s < nshapes; ++s)
    for (int q = 0; q < nq; ++q)
      if (queries[q].shape == s) order.push_back(q);
  if ((int)order.size() != nq) return fail(CX_E_INVALID, "cx_shared_execute: a query names a shape outside 0..%d", nshapes - 1);
  for (int i = 0; i < nq; ++i) {
    const cx_shared_query& q = queries[order[i]];
    const auto& sh = lp.sshapes[q.shape];
    const uint64_t need = sh.groups * (uint64_t)sh.ts;
    if (!q.result || q.result_words < need || !q.validity || q.validity_words < (need + 63) / 64)
      return fail(CX_E_CAPACITY, "cx_shared_execute: query %d result buffers are smaller than its shape needs (%llu words)", order[i], (unsigned long long)need);
    if (q.param_off < 0 || q.param_off + sh.nlits > nparams)
      return fail(CX_E_INVALID, "cx_shared_execute: query %d parameters fall outside the parameter array", order[i]);
  }
  // The aggregate-cube path answers the whole batch in one pass when the
  // registered ranges allow; otherwise passes of at most maxq queries run the
  // per-query mask kernels.  Each pass gets its own descriptors and a
  // compacted parameter array.
  CubePlan cp;
  std::vector<int> qshapes(nq);
  for (int i = 0; i < nq; ++i) qshapes[i] = queries[i].shape;
  if (lp.cube) {
    const int frc = ensure_cube_fds(lp, c, stream);
    if (frc) return frc;
  }
  const bool cube = plan_cubes(lp, c, qshapes.data(), nq, cp);
  const int maxq = cube ? std::max(nq, 1) : std::max(1, std::min(lp.shared_maxq, 256));
  const int npass = (nq + maxq - 1) / maxq;
  std::vector<int> pass_params(std::max(npass, 1), 0);
  int maxp = lp.shared_maxp;
  for (int ps = 0; ps < npass; ++ps) {
    int np = 0;
    for (int i = ps * maxq; i < std::min(nq, (ps + 1) * maxq); ++i) np += lp.sshapes[queries[order[i]].shape].nlits;
    if (!cube && np > lp.shared_maxp) return fail(CX_E_CAPACITY, "cx_shared_execute: %d parameters in one pass exceed %d", np, lp.shared_maxp);
    pass_params[ps] = np;
    maxp = std::max(maxp, np);
  }

  // Scratch: dimension slot entries (zeroed per pass), touched bits per grouped
  // query, per-pass descriptors and parameters, error word.
  uint64_t off = 0;
  std::vector<uint64_t> dkm_off, dat_off;
  // The cube path needs no int4 entries for dimensions kept as compact words,
  // and no extra-attribute arrays at all (those serve the mask path).
  auto compact_dim = [&](int slot) { return cube && slot >= 0 && slot < CX_MAX_HTS && cp.desz[slot] > 0; };
  for (const auto& h : lp.hts) {
    dkm_off.push_back(off);
    if (!compact_dim(h.slot)) off = align256(off + h.words * 4);
    auto it = lp.dat_words.find(h.slot);
    dat_off.push_back(off);
    if (!cube && it != lp.dat_words.end()) off = align256(off + it->second * 4);
  }
  if (cube)
    for (int d = 0; d < CX_MAX_HTS; ++d)
      if (cp.dcomp_bytes[d]) { cp.dcomp_off[d] = off; off = align256(off + cp.dcomp_bytes[d]); }
  const uint64_t dim_end = off;
  std::vector<uint64_t> touch_off(nq, 0);
  for (int i = 0; i < nq; ++i) {
    const auto& sh = lp.sshapes[queries[order[i]].shape];
    if (sh.grouped) { touch_off[i] = off; off = align256(off + ((sh.groups + 31) / 32) * 4); }
  }
  const uint64_t touch_end = off;
  const uint64_t cube_off = off;
  if (cube) off = align256(off + cp.gbytes);
  const size_t desc_bytes = (size_t)maxq * sizeof(CxSQ), par_bytes = (size_t)std::max(maxp, 1) * 4;
  const size_t pass_bytes = align256(desc_bytes + par_bytes);
  const uint64_t pass_off = off; off += (uint64_t)std::max(npass, 1) * pass_bytes;
  const uint64_t err_off = off; off = align256(off + 16);
  const uint64_t total = off;

  int dev = 0;
  CX_CUDA(cudaGetDevice(&dev));
  int rc = ensure_ctx_device(c, dev);
  if (rc) return rc;
  cx_module::Loaded* L = nullptr;
  rc = load_on_device(m, dev, &L);
  if (rc) return rc;
  if (c->pending) { CX_CUDA(cudaEventSynchronize(c->ev[3])); c->pending = false; }

  char* scratch = nullptr;
  if (c->user_scratch) {
    if (c->user_scratch_bytes < total) return fail(CX_E_CAPACITY, "cx_shared_execute: caller scratch too small (%llu < %llu)", (unsigned long long)c->user_scratch_bytes, (unsigned long long)total);
    scratch = (char*)c->user_scratch;
  } else {
    if (c->own_scratch_bytes < total) {
      if (c->own_scratch) { cudaFree(c->own_scratch); c->own_scratch = nullptr; c->own_scratch_bytes = 0; }
      const uint64_t grow = total + total / 2;
      CX_CUDA(cudaMalloc(&c->own_scratch, grow));
      c->own_scratch_bytes = grow;
    }
    scratch = (char*)c->own_scratch;
  }
  for (size_t i = 0; i < lp.hts.size(); ++i) {
    a.ht[lp.hts[i].slot] = compact_dim(lp.hts[i].slot) ? nullptr : (int*)(scratch + dkm_off[i]);
    if (!cube && lp.dat_words.count(lp.hts[i].slot)) a.dat[lp.hts[i].slot] = (int*)(scratch + dat_off[i]);
  }
  a.err = (unsigned int*)(scratch + err_off);

  // Host staging of every pass's descriptors and parameters (pinned; the
  // previous batch's copies finished before the wait above).
  const size_t stage_bytes = (size_t)std::max(npass, 1) * pass_bytes;
  if (c->host_stage_bytes < stage_bytes) {
    if (c->host_stage) cudaFreeHost(c->host_stage);
    c->host_stage = nullptr;
    c->host_stage_bytes = 0;
    CX_CUDA(cudaMallocHost(&c->host_stage, stage_bytes * 2));
    c->host_stage_bytes = stage_bytes * 2;
  }

  size_t scan_ki = 0;
  const char* scan_kind = cube ? "cubescan" : "sharedscan";
  while (scan_ki < lp.kernels.size() && lp.kernels[scan_ki].kind != scan_kind) ++scan_ki;
  if (scan_ki == lp.kernels.size()) return fail(CX_E_INVALID, "cx_shared_execute: program has no %s kernel", scan_kind);
  const KernelSpec& sk = lp.kernels[scan_ki];
  // Shared-memory group tables go into the slack the scan's own residency
  // leaves, so they never cost a resident CTA.
  const int by_threads = std::max(1, 2048 / std::max(sk.block, 1));
  const size_t qb_max = (size_t)lp.shared_qb_bytes * (size_t)std::min(nq, maxq) + 16;
  const int resident = std::max(1, std::min({sk.ctas_per_sm, by_threads, (int)(233472 / (sk.smem + qb_max + 1024))}));
  const size_t smem_cap = std::min<size_t>(200 * 1024, 233472 / resident - 1024);

  int sms = c->sm_override;
  if (sms <= 0) CX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  Driver& d = driver();

  // Plan every pass on the host: descriptors and parameters into the pinned
  // staging, kernel arguments, grids and shared-memory sizes.
  struct Pass {
    CxArgs args;
    int qn = 0, nparams = 0;
    size_t extra_smem = 0;
    unsigned scan_grid = 0;
    char* hstage = nullptr;
    CUfunction scan_fn = nullptr;  // the generic scan kernel, or its build for the batch's cube layout
  };
  std::vector<Pass> passes(npass);
  for (int ps = 0; ps < npass; ++ps) {
    Pass& P = passes[ps];
    const int q0 = ps * maxq, qn = std::min(nq, q0 + maxq) - q0;
    char* hstage = (char*)c->host_stage + (size_t)ps * pass_bytes;
    CxSQ* hsq = (CxSQ*)hstage;
    int* hpar = (int*)(hstage + desc_bytes);
    int poff = 0;
    uint64_t tab_words = 0, bit_words = 0;
    const size_t qb_bytes = cube ? 0 : ((size_t)lp.shared_qb_bytes * (size_t)qn + 15) & ~(size_t)15;
    for (int j = 0; j < qn; ++j) {
      const cx_shared_query& q = queries[order[q0 + j]];
      const auto& sh = lp.sshapes[q.shape];
      hsq[j].result = (unsigned long long*)q.result;
      hsq[j].validity = (unsigned long long*)q.validity;
      hsq[j].touched = sh.grouped ? (unsigned int*)(scratch + touch_off[q0 + j]) : nullptr;
      hsq[j].shape = q.shape;
      hsq[j].param_off = poff;
      if (sh.nlits) memcpy(hpar + poff, params + q.param_off, (size_t)sh.nlits * 4);
      poff += sh.nlits;
      hsq[j].smem_acc = -1;
      hsq[j].smem_bits = 0;
      hsq[j].keep = keep ? (keep[order[q0 + j]] ? 1 : 0) : 0;
      if (cube || !sh.smem_ok) continue;
      const uint64_t tw = tab_words + sh.groups * (uint64_t)sh.naggs;
      const uint64_t bw = bit_words + sh.tw * (uint64_t)(1 + sh.nseen);
      if (sk.smem + qb_bytes + tw * 8 + bw * 4 + 64 > smem_cap) continue;
      hsq[j].smem_acc = (int)tab_words;
      hsq[j].smem_bits = (int)bit_words;
      tab_words = tw;
      bit_words = bw;
    }
    a.sq = (const CxSQ*)(scratch + pass_off + (uint64_t)ps * pass_bytes);
    a.sparams = (const int*)(scratch + pass_off + (uint64_t)ps * pass_bytes + desc_bytes);
    a.sq_total = qn;
    a.nparams = poff;
    a.smem_tab_words = (int)tab_words;
    a.smem_bit_words = (int)bit_words;
    for (int s = 0; s < CX_MAX_SHAPES; ++s) { a.sq_first[s] = 0; a.sq_num[s] = 0; }
    for (int j = 0; j < qn; ++j) {
      const int s = hsq[j].shape;
      if (s < CX_MAX_SHAPES) { if (a.sq_num[s] == 0) a.sq_first[s] = j; ++a.sq_num[s]; }
    }
    if (cube) fill_cube_args(a, cp, nshapes, scratch, cube_off);
    P.args = a;
    P.qn = qn;
    P.nparams = poff;
    P.hstage = hstage;
    P.extra_smem = cube ? (size_t)cp.dsm_bytes + (size_t)cp.smem_words * 8 : qb_bytes + (size_t)tab_words * 8 + (size_t)bit_words * 4 + 16;
    P.scan_fn = L->fns[scan_ki];
    if (cube) {
      CUfunction spec = nullptr;
      cube_spec_function(m, dev, P.args, sk.name, 227 * 1024, &spec);
      if (spec) P.scan_fn = spec;
    }
    int occ = 1;
    CUresult orr = d.Occupancy(&occ, P.scan_fn, sk.block, sk.smem + P.extra_smem);
    if (orr != CUDA_SUCCESS) return drv_fail(orr, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) return fail(CX_E_CAPACITY, "cx_shared_execute: shared scan cannot be resident with %zu bytes of shared memory", sk.smem + P.extra_smem);
    const long long tiles = (rows[0] + sk.tile - 1) / sk.tile;
    const int per_sm = std::max(1, std::min(sk.ctas_per_sm, occ));
    P.scan_grid = (unsigned)std::min<long long>(tiles, (long long)sms * per_sm);
  }

  // Enqueues the whole batch on `s`: one fixed sequence per pass shape, so a
  // captured graph of it replays for every batch with the same pass shapes.
  int launches = 0;
  auto enqueue = [&](cudaStream_t s, bool capturing) -> int {
    launches = 0;
    // Inside a capture only an external record becomes a graph node that
    // records the timing event.
    auto rec = [&](cudaEvent_t e) {
      return capturing ? cudaEventRecordWithFlags(e, s, cudaEventRecordExternal) : cudaEventRecord(e, s);
    };
    auto launch = [&](size_t ki, unsigned grid, size_t extra, CxArgs* args, CUfunction fn = nullptr) -> int {
      const KernelSpec& k = lp.kernels[ki];
      if (grid == 0) return CX_OK;
      void* kp[] = {args};
      CUresult r = d.LaunchKernel(fn ? fn : L->fns[ki], grid, 1, 1, k.block, 1, 1, (unsigned)(k.smem + extra), (CUstream)s, kp, nullptr);
      if (r != CUDA_SUCCESS) return drv_fail(r, k.name.c_str());
      ++launches;
      return CX_OK;
    };
    CX_CUDA(rec(c->ev[0]));
    CX_CUDA(cudaMemsetAsync(scratch + err_off, 0, 16, s));
    for (int ps = 0; ps < npass; ++ps) {
      Pass& P = passes[ps];
      CX_CUDA(cudaMemcpyAsync((void*)P.args.sq, P.hstage, (size_t)P.qn * sizeof(CxSQ), cudaMemcpyHostToDevice, s));
      if (P.nparams)
        CX_CUDA(cudaMemcpyAsync((void*)P.args.sparams, P.hstage + desc_bytes, (size_t)P.nparams * 4, cudaMemcpyHostToDevice, s));
      CX_CUDA(cudaMemsetAsync(scratch, 0, dim_end, s));
      if (cube && cp.gbytes) CX_CUDA(cudaMemsetAsync(scratch + cube_off, 0, cp.gbytes, s));
      // Before the scan: result zeroing and the path's dimension indexes; after
      // it: the cube answers (cube path) and the group-key epilogue.
      for (size_t ki = 0; ki < scan_ki; ++ki) {
        const KernelSpec& k = lp.kernels[ki];
        unsigned grid;
        if (k.kind == "zero") grid = (unsigned)P.qn;
        else if (k.kind == (cube ? "cubeidx" : "build"))
          grid = (unsigned)std::min<long long>((rows[k.table] + k.tile - 1) / k.tile, (long long)sms * 16);
        else continue;
        int r = launch(ki, grid, 0, &P.args);
        if (r) return r;
      }
      if (ps == 0) CX_CUDA(rec(c->ev[1]));
      int r = launch(scan_ki, P.scan_grid, P.extra_smem, &P.args, P.scan_fn);
      if (r) return r;
      if (ps == npass - 1) CX_CUDA(rec(c->ev[2]));
      for (size_t ki = scan_ki + 1; ki < lp.kernels.size(); ++ki) {
        const KernelSpec& k = lp.kernels[ki];
        unsigned grid;
        if (k.kind == "queries") grid = (unsigned)P.qn;
        else if (cube && k.kind == "cubeans") grid = (unsigned)(P.qn * cp.chunks);
        else continue;
        if ((r = launch(ki, grid, 0, &P.args))) return r;
      }
    }
    if (npass == 0) {
      CX_CUDA(rec(c->ev[1]));
      CX_CUDA(rec(c->ev[2]));
    }
    CX_CUDA(cudaMemcpyAsync(c->host_err, scratch + err_off, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    CX_CUDA(rec(c->ev[3]));
    return CX_OK;
  };

  int graph_mode = 0;
  if (c->graph_replay && npass > 0) {
    // Everything a captured graph bakes in: module, buffers, staging, and per
    // pass the kernel arguments, grids, shared memory and copy sizes.
    std::vector<unsigned char> sig;
    auto put = [&](const void* p, size_t n) { sig.insert(sig.end(), (const unsigned char*)p, (const unsigned char*)p + n); };
    // The module by its unique id, not its address: a module freed and a new
    // one allocated at the same address must not replay the old graph.
    const void* ids[] = {scratch, c->host_stage, c->host_err};
    put(ids, sizeof ids);
    put(&m->uid, sizeof m->uid);
    const uint64_t sizes[] = {dim_end, err_off, (uint64_t)npass, (uint64_t)sms, (uint64_t)cube, cube_off, cp.gbytes};
    put(sizes, sizeof sizes);
    for (const Pass& P : passes) {
      put(&P.args, sizeof(CxArgs));
      const uint64_t v[] = {(uint64_t)P.qn, (uint64_t)P.nparams, P.extra_smem, P.scan_grid, (uint64_t)(P.hstage - (char*)c->host_stage)};
      put(v, sizeof v);
    }
    if (!(c->gexec && sig == c->gsig)) {
      if (!c->cap_stream) CX_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
      CX_CUDA(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
      const int er = enqueue(c->cap_stream, true);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(c->cap_stream, &g);
      if (er) { if (g) cudaGraphDestroy(g); return er; }
      if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return fail(CX_E_CUDA, "cx_shared_execute: graph capture: %s", cudaGetErrorString(ce)); }
      bool updated = false;
      if (c->gexec) {
        cudaGraphExecUpdateResultInfo info;
        updated = cudaGraphExecUpdate(c->gexec, g, &info) == cudaSuccess;
        if (!updated) { cudaGetLastError(); cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
      }
      if (!updated) {
        const cudaError_t ie = cudaGraphInstantiate(&c->gexec, g, 0);
        if (ie != cudaSuccess) { cudaGraphDestroy(g); c->gexec = nullptr; return fail(CX_E_CUDA, "cx_shared_execute: graph instantiate: %s", cudaGetErrorString(ie)); }
      }
      cudaGraphDestroy(g);
      c->gsig = std::move(sig);
      c->graph_launches = launches;
      graph_mode = 2;
    } else {
      graph_mode = 1;
    }
    CX_CUDA(cudaGraphLaunch(c->gexec, stream));
    launches = c->graph_launches;
  } else {
    const int er = enqueue(stream, false);
    if (er) return er;
  }
  c->pending = true;
  c->timing = cx_timing{};
  c->timing.scan_grid = npass ? (int)passes.back().scan_grid : 0;
  c->timing.gpu_launches = launches;
  c->timing.graph = graph_mode;
  c->timing.mode = cube ? 1 : 0;
  return CX_OK;
}

int cx_ctx_set_graph_replay(cx_exec_ctx* c, int enable) {
  if (!c) return fail(CX_E_INVALID, "cx_ctx_set_graph_replay: NULL context");
  c->graph_replay = enable != 0;
  return CX_OK;
}

int cx_ctx_sync(cx_exec_ctx* c) {
  if (!c) return fail(CX_E_INVALID, "cx_ctx_sync: NULL context");
  if (!c->pending) return CX_OK;
  CX_CUDA(cudaEventSynchronize(c->ev[3]));
  c->pending = false;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  c->timing.build_ms = ms;
  cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
  c->timing.scan_ms = ms;
  cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]);
  c->timing.post_ms = ms;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[3]);
  c->timing.total_ms = ms;
  c->kernel_err = *c->host_err;
  if (c->kernel_err) return fail(CX_E_KERNEL, "kernel raised error code %u", c->kernel_err);
  return CX_OK;
}

int cx_ctx_timing(const cx_exec_ctx* c, cx_timing* t) {
  if (!c || !t) return fail(CX_E_INVALID, "cx_ctx_timing: NULL argument");
  *t = c->timing;
  return CX_OK;
}

int cx_ctx_kernel_error(const cx_exec_ctx* c, uint32_t* code) {
  if (!c || !code) return fail(CX_E_INVALID, "cx_ctx_kernel_error: NULL argument");
  *code = c->kernel_err;
  return CX_OK;
}

}  // extern "C"
