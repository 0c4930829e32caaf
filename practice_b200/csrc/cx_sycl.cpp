// cx_sycl.cpp -- takes the program the reference's code generator emits
// (JITOperatorVisitor::generateCode, src/core/visitor.cpp:4771-4878: a SYCL
// translation unit whose `extern "C" void execute_query(db::ExecutionContext*)`
// binds buffers by name, zeroes hash tables and the result, and submits one
// nd_range kernel per hash-table build plus the fused fact scan) and rewrites
// its launch skeleton into a CUDA program for this library: the same kernel
// bodies -- the crystal primitive calls, the emitted predicate and aggregate
// code -- become `extern "C" __global__` kernels over one `const CxArgs a`,
// compiled by NVRTC for sm_100a against crystal_sm100.cuh, and the host part
// becomes the `/*@cx-launch ... @*/` plan the generic executor runs.  So
// ICompiler::compile can hand cx_compile the visitor's text unchanged.
//
// Mapping of the skeleton:
//   ctx->getBuffer<int>("d_c")             -> column slot of "d_c" (table by the
//                                              column's first letter, as
//                                              include/crystal/utils.h getTableName)
//   getScratchIntBuffer("d_x_hash_table", K*N | K*X_LEN)
//                                           -> hash table slot of K*N words, or
//                                              K x the row count of table X
//   q.memset(ht | d_result, 0, ...)         -> the executor zeroes every hash table
//                                              and the result before the kernels
//   q.submit(... parallel_for<class K>(nd_range((X_LEN + TILE-1)/TILE * BT, BT), body))
//                                           -> kernel K, one CTA of BT threads per
//                                              TILE rows of table X
//   X_LEN (utils.h's SF10 constants)        -> the context's row count of table X
//   it.get_local_linear_id() / get_group_linear_id() / get_group_range(0)
//                                           -> threadIdx.x / blockIdx.x / gridDim.x
//   sycl::reduce_over_group(it.get_group(), v, plus|minimum|maximum<ull>{})
//                                           -> cx::group_reduce_u64 (every thread
//                                              gets the CTA's result)
//   ctx->tuple_size_ = T; memset(d_result, 0, W * 8)
//                                           -> result of W words, tuples of T
// Programs that need the host in the middle (dense result materialisation
// with a host prefix sum, multi-value hash tables sized by a read-back,
// projections, ORDER BY / LIMIT) are refused with a message; cx_codegen,
// cx_finalize and the plan builder cover those.
#include <cctype>
#include <cstring>
#include <map>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/crystal_b200.h"
#include "cx_args.h"
#include "cx_internal.h"

namespace {

struct Kernel {
  std::string name, table, body;
  bool scan = false;
};

struct Program {
  int block_threads = 0, items_per_thread = 0;
  std::vector<std::string> tables;             // slot order; LINEORDER first
  std::vector<std::pair<std::string, int>> cols;  // buffer name, table slot
  std::vector<std::pair<std::string, std::string>> nulls;  // variable, column buffer name
  struct Ht { std::string name; unsigned long long mult = 1, words = 0; int table = -1; };
  std::vector<Ht> hts;
  std::vector<Kernel> kernels;
  unsigned long long result_words = 0;
  int tuple_size = 0;
};

[[noreturn]] void refuse(const std::string& why) { throw std::runtime_error("visitor program: " + why); }

// The reference's table of each LEN macro (include/crystal/utils.h).
std::string table_of_len(const std::string& macro) {
  if (macro == "LO_LEN") return "LINEORDER";
  if (macro == "P_LEN") return "PART";
  if (macro == "S_LEN") return "SUPPLIER";
  if (macro == "C_LEN") return "CUSTOMER";
  if (macro == "D_LEN") return "DDATE";
  refuse("unknown row-count macro " + macro);
}

// The table of a column buffer "d_<column>" by the column's first letter
// (getTableName, include/crystal/utils.h).
std::string table_of_column(const std::string& buffer) {
  const std::string c = buffer.substr(2);
  switch (c.empty() ? '?' : c[0]) {
    case 'l': return "LINEORDER";
    case 's': return "SUPPLIER";
    case 'c': return "CUSTOMER";
    case 'p': return "PART";
    case 'd': return "DDATE";
  }
  refuse("cannot tell the table of column buffer " + buffer);
}

int table_slot(Program& p, const std::string& t) {
  for (size_t i = 0; i < p.tables.size(); ++i)
    if (p.tables[i] == t) return (int)i;
  p.tables.push_back(t);
  return (int)p.tables.size() - 1;
}

// Index just past the bracket that closes the one at `open`.
size_t match(const std::string& s, size_t open) {
  const char o = s[open], c = o == '(' ? ')' : o == '{' ? '}' : o == '[' ? ']' : '>';
  int depth = 0;
  for (size_t i = open; i < s.size(); ++i) {
    if (s[i] == '"') {  // skip string literals
      for (++i; i < s.size() && s[i] != '"'; ++i)
        if (s[i] == '\\') ++i;
      continue;
    }
    if (s[i] == o) ++depth;
    else if (s[i] == c && --depth == 0) return i + 1;
  }
  refuse("unbalanced brackets");
}

std::string trim(const std::string& s) {
  size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b])) ++b;
  while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
  return s.substr(b, e - b);
}

// "K*N", "K*X_LEN", "N" or "X_LEN" -> (multiplier, constant words or table)
void parse_size(Program& p, const std::string& expr, Program::Ht& h) {
  static const std::regex re(R"re(^\s*(?:(\d+)\s*\*\s*)?(\d+|[A-Z]+_LEN)\s*$)re");
  std::smatch m;
  if (!std::regex_match(expr, m, re)) refuse("hash table size '" + expr + "'");
  h.mult = m[1].matched ? std::stoull(m[1]) : 1ULL;
  const std::string v = m[2];
  if (std::isdigit((unsigned char)v[0])) h.words = h.mult * std::stoull(v);
  else h.table = table_slot(p, table_of_len(v));
}

// Rewrites `sycl::reduce_over_group(it.get_group(), X, sycl::OP<unsigned long long>{})`.
std::string rewrite_reductions(const std::string& body) {
  static const std::string key = "sycl::reduce_over_group(";
  std::string out;
  size_t pos = 0;
  for (;;) {
    const size_t at = body.find(key, pos);
    if (at == std::string::npos) break;
    out += body.substr(pos, at - pos);
    const size_t open = at + key.size() - 1;
    const size_t end = match(body, open);
    const std::string inner = body.substr(open + 1, end - open - 2);
    // Split the three arguments at top-level commas.
    std::vector<std::string> args;
    int depth = 0;
    size_t start = 0;
    for (size_t i = 0; i < inner.size(); ++i) {
      const char ch = inner[i];
      if (ch == '(' || ch == '{' || ch == '[' || ch == '<') ++depth;
      else if (ch == ')' || ch == '}' || ch == ']' || ch == '>') --depth;
      else if (ch == ',' && depth == 0) {
        args.push_back(trim(inner.substr(start, i - start)));
        start = i + 1;
      }
    }
    args.push_back(trim(inner.substr(start)));
    if (args.size() != 3 || args[0] != "it.get_group()") refuse("reduce_over_group form '" + inner + "'");
    int op = -1;
    if (args[2] == "sycl::plus<unsigned long long>{}") op = 0;
    else if (args[2] == "sycl::minimum<unsigned long long>{}") op = 1;
    else if (args[2] == "sycl::maximum<unsigned long long>{}") op = 2;
    else refuse("reduction operator " + args[2]);
    out += "cx::group_reduce_u64<BLOCK_THREADS, " + std::to_string(op) + ">(" + args[1] + ", cx_red)";
    pos = end;
  }
  out += body.substr(pos);
  return out;
}

std::string replace_all(std::string s, const std::string& from, const std::string& to) {
  for (size_t at = s.find(from); at != std::string::npos; at = s.find(from, at + to.size())) s.replace(at, from.size(), to);
  return s;
}

Kernel parse_submit(Program& p, const std::string& sub) {
  static const std::regex name_re(R"re(h\.parallel_for<class\s+(\w+)>\s*\(\s*sycl::nd_range<1>\s*\()re");
  std::smatch m;
  if (!std::regex_search(sub, m, name_re))
    refuse("a q.submit that is not an nd_range kernel (host-side steps between kernels are not translated)");
  Kernel k;
  k.name = m[1];
  const std::string pre = sub.substr(0, (size_t)m.position(0));
  static const std::regex tiles_re(R"re(int\s+num_tiles\s*=\s*\(\s*([A-Z]+_LEN)\s*\+\s*TILE_SIZE\s*-\s*1\s*\)\s*/\s*TILE_SIZE\s*;)re");
  std::smatch tm;
  if (!std::regex_search(pre, tm, tiles_re)) refuse("kernel " + k.name + " is not a tile loop over a table");
  k.table = table_of_len(tm[1]);
  table_slot(p, k.table);
  // nd_range(global, local): num_tiles * BLOCK_THREADS work-items in groups of BLOCK_THREADS.
  const size_t open = (size_t)(m.position(0) + m.length(0)) - 1;
  const size_t close = match(sub, open);
  const std::string range = trim(sub.substr(open + 1, close - open - 2));
  const bool direct = std::regex_match(range, std::regex(R"re(num_tiles\s*\*\s*BLOCK_THREADS\s*,\s*BLOCK_THREADS)re"));
  const bool named = std::regex_match(range, std::regex(R"re(global\s*,\s*local)re")) &&
                     std::regex_search(pre, std::regex(R"re(size_t\s+local\s*=\s*BLOCK_THREADS\s*;)re")) &&
                     std::regex_search(pre, std::regex(R"re(size_t\s+global\s*=\s*num_tiles\s*\*\s*BLOCK_THREADS\s*;)re"));
  if (!direct && !named) refuse("kernel " + k.name + " launch range '" + range + "'");
  static const std::regex lam_re(R"re(\[=\]\s*\(\s*sycl::nd_item<1>\s+it\s*\)\s*\{)re");
  std::smatch lm;
  const std::string rest = sub.substr(close);
  if (!std::regex_search(rest, lm, lam_re)) refuse("kernel " + k.name + " has no nd_item lambda");
  const size_t bopen = close + (size_t)(lm.position(0) + lm.length(0)) - 1;
  const size_t bend = match(sub, bopen);
  std::string body = sub.substr(bopen + 1, bend - bopen - 2);
  body = rewrite_reductions(body);
  body = replace_all(body, "it.get_local_linear_id()", "(int)threadIdx.x");
  body = replace_all(body, "it.get_group_linear_id()", "(int)blockIdx.x");
  body = replace_all(body, "it.get_group_range(0)", "(int)gridDim.x");
  if (body.find("sycl::") != std::string::npos || std::regex_search(body, std::regex(R"re(\bit\.)re")))
    refuse("kernel " + k.name + " uses a SYCL construct outside the translated set");
  k.body = body;
  k.scan = k.table == "LINEORDER" && k.name.rfind("Scan_", 0) == 0;
  return k;
}

Program parse(const std::string& src) {
  Program p;
  p.tables.push_back("LINEORDER");
  std::smatch m;
  if (!std::regex_search(src, m, std::regex(R"re(constexpr\s+int\s+BLOCK_THREADS\s*=\s*(\d+)\s*;)re")))
    refuse("no BLOCK_THREADS");
  p.block_threads = std::stoi(m[1]);
  if (!std::regex_search(src, m, std::regex(R"re(constexpr\s+int\s+ITEMS_PER_THREAD\s*=\s*(\d+)\s*;)re")))
    refuse("no ITEMS_PER_THREAD");
  p.items_per_thread = std::stoi(m[1]);
  if (p.block_threads <= 0 || p.block_threads > 1024 || p.block_threads % 32 || p.items_per_thread <= 0 ||
      p.items_per_thread > 64)
    refuse("launch shape out of range");
  const std::string sig = "extern \"C\" void execute_query(db::ExecutionContext* ctx)";
  const size_t at = src.find(sig);
  if (at == std::string::npos) refuse("no execute_query entry point");
  const size_t open = src.find('{', at + sig.size());
  const size_t end = match(src, open);
  const std::string body = src.substr(open + 1, end - open - 2);

  static const std::regex col_re(R"re(^int\*\s+(\w+)\s*=\s*ctx->getBuffer<int>\(\s*"(\w+)"\s*\)$)re");
  static const std::regex ht_re(
      R"re(^int\*\s+(\w+)\s*=\s*ctx->config_\.reuse_scratch_buffers\s*\?\s*ctx->getScratchIntBuffer\(\s*"(\w+)"\s*,\s*static_cast<size_t>\((.+)\)\)\s*:\s*sycl::malloc_device<int>\((.+),\s*q\)$)re");
  static const std::regex null_re(R"re(^uint64_t\*\s+(\w+)\s*=\s*ctx->getNullBitmap\(\s*"(\w+)"\s*\)$)re");
  static const std::regex memset_re(R"re(^q\.memset\(\s*(\w+)\s*,\s*0\s*,\s*(.+)\)$)re");
  static const std::regex result_re(R"re(^\(?\s*(\d+)\s*\)?\s*\*\s*sizeof\(unsigned long long\)$)re");
  static const std::regex ts_re(R"re(^ctx->tuple_size_\s*=\s*(\d+)$)re");
  static const std::regex dense_re(R"re(^ctx->result_is_dense_\s*=\s*(true|false)$)re");
  static const std::regex ignore_re(
      R"re(^(auto\s+__crystal_generated_(start|end)\s*=.*|sycl::queue&\s+q\s*=\s*\*\(ctx->q_\)|unsigned long long\*\s+d_result\s*=\s*ctx->getResultPointer\(\)|uint64_t\*\s+d_result_validity\s*=\s*ctx->getResultValidityPointer\(\)|ctx->result_row_count_\s*=\s*0|ctx->expected_result_validity_words_\s*=\s*0|q\.wait\(\)|if\s*\(!ctx->config_\.reuse_scratch_buffers\)\s*sycl::free\(\w+,\s*q\)|ctx->timing_\.\w+\s*=.*)$)re");

  size_t pos = 0;
  while (pos < body.size()) {
    while (pos < body.size() && std::isspace((unsigned char)body[pos])) ++pos;
    if (pos >= body.size()) break;
    if (body.compare(pos, 9, "q.submit(") == 0) {
      const size_t e = match(body, pos + 8);
      const size_t lam = body.find('{', pos);
      p.kernels.push_back(parse_submit(p, body.substr(lam, e - lam)));
      pos = e;
      while (pos < body.size() && (std::isspace((unsigned char)body[pos]) || body[pos] == ';')) ++pos;
      continue;
    }
    if (body[pos] == '{') refuse("a host-side block between kernels (dense result materialisation?)");
    // One statement up to its ';' at bracket depth 0.
    size_t i = pos;
    int depth = 0;
    for (; i < body.size(); ++i) {
      const char ch = body[i];
      if (ch == '"') {
        for (++i; i < body.size() && body[i] != '"'; ++i)
          if (body[i] == '\\') ++i;
        continue;
      }
      if (ch == '(' || ch == '{' || ch == '[') ++depth;
      else if (ch == ')' || ch == '}' || ch == ']') --depth;
      else if (ch == ';' && depth == 0) break;
    }
    std::string st = trim(body.substr(pos, i - pos));
    st = std::regex_replace(st, std::regex(R"re(\s+)re"), " ");
    pos = i + 1;
    std::smatch sm;
    if (std::regex_match(st, sm, col_re)) {
      if (sm[1] != sm[2]) refuse("column variable " + std::string(sm[1]) + " bound to " + std::string(sm[2]));
      p.cols.emplace_back(sm[2], table_slot(p, table_of_column(sm[2])));
    } else if (std::regex_match(st, sm, null_re)) {
      p.nulls.emplace_back(sm[1], sm[2]);
    } else if (std::regex_match(st, sm, ht_re)) {
      if (sm[1] != sm[2] || trim(sm[3]) != trim(sm[4])) refuse("hash table binding " + st);
      Program::Ht h;
      h.name = sm[1];
      parse_size(p, sm[3], h);
      p.hts.push_back(h);
    } else if (std::regex_match(st, sm, memset_re)) {
      const std::string target = sm[1];
      std::smatch rm;
      const std::string bytes = trim(sm[2]);
      if (target == "d_result") {
        if (!std::regex_match(bytes, rm, result_re)) refuse("result memset " + st);
        p.result_words = std::stoull(rm[1]);
      } else {
        bool known = false;
        for (const auto& h : p.hts) known = known || h.name == target;
        if (!known) refuse("memset of an unknown buffer " + target);
      }
    } else if (std::regex_match(st, sm, ts_re)) {
      p.tuple_size = std::stoi(sm[1]);
    } else if (std::regex_match(st, sm, dense_re)) {
      if (sm[1] == "true") refuse("dense result materialisation");
    } else if (std::regex_match(st, ignore_re)) {
      // timing, queue and cleanup statements: the executor owns these
    } else {
      refuse("statement not translated: " + st.substr(0, 120));
    }
  }
  for (const auto& n : p.nulls) {
    bool bound = false;
    for (const auto& c : p.cols) bound = bound || c.first == n.second;
    if (!bound) refuse("validity of " + n.second + " without its column");
  }
  if (p.kernels.empty()) refuse("no kernels");
  if (p.result_words == 0 || p.tuple_size <= 0 || p.result_words % (unsigned long long)p.tuple_size)
    refuse("result size / tuple size");
  int scans = 0;
  for (const auto& k : p.kernels) scans += k.scan;
  if (scans != 1 || !p.kernels.back().scan) refuse("expected the fact scan as the last kernel");
  if (p.tables.size() > CX_MAX_TABLES || p.cols.size() > CX_MAX_COLS || p.hts.size() > CX_MAX_HTS)
    refuse("more tables, columns or hash tables than the argument block holds");
  return p;
}

std::string emit(const Program& p) {
  std::ostringstream o;
  const int tile = p.block_threads * p.items_per_thread;
  bool validity = false;
  for (const auto& k : p.kernels) validity = validity || k.body.find("d_result_validity") != std::string::npos;
  o << "/*@cx-launch\nv 1\n";
  for (size_t t = 0; t < p.tables.size(); ++t) o << "table " << t << " " << p.tables[t] << "\n";
  for (size_t c = 0; c < p.cols.size(); ++c) o << "col " << c << " " << p.cols[c].first << " " << p.cols[c].second << "\n";
  for (const auto& n : p.nulls)
    for (size_t c = 0; c < p.cols.size(); ++c)
      if (p.cols[c].first == n.second) o << "null " << c << " " << n.second << "\n";
  for (size_t h = 0; h < p.hts.size(); ++h) {
    if (p.hts[h].table >= 0) o << "htrows " << h << " " << p.hts[h].name << " " << p.hts[h].mult << " " << p.hts[h].table << "\n";
    else o << "ht " << h << " " << p.hts[h].name << " " << p.hts[h].words << "\n";
  }
  const unsigned long long groups = p.result_words / (unsigned long long)p.tuple_size;
  o << "result " << p.result_words << " " << groups << " " << p.tuple_size << " " << p.tuple_size << " "
    << (validity ? 0 : 1) << "\n";
  for (const auto& k : p.kernels) {
    int tslot = 0;
    for (size_t t = 0; t < p.tables.size(); ++t)
      if (p.tables[t] == k.table) tslot = (int)t;
    o << "kernel " << k.name << " " << (k.scan ? "tilescan" : "tiles") << " " << tslot << " " << p.block_threads << " "
      << tile << "\n";
  }
  o << "@*/\n";
  o << "// Translated from the reference code generator's SYCL program: the kernel bodies\n"
       "// are its own, the launch skeleton is this library's.\n";
  o << "#include \"cx_args.h\"\n#include \"crystal_sm100.cuh\"\n\n";
  o << "constexpr int BLOCK_THREADS = " << p.block_threads << ";\n";
  o << "constexpr int ITEMS_PER_THREAD = " << p.items_per_thread << ";\n";
  o << "constexpr int TILE_SIZE = BLOCK_THREADS * ITEMS_PER_THREAD;\n\n";
  // Row counts the reference bakes in as macros come from the context.
  static const char* macros[][2] = {{"LO_LEN", "LINEORDER"}, {"P_LEN", "PART"}, {"S_LEN", "SUPPLIER"},
                                    {"C_LEN", "CUSTOMER"}, {"D_LEN", "DDATE"}};
  for (const auto& mc : macros) {
    int slot = -1;
    for (size_t t = 0; t < p.tables.size(); ++t)
      if (p.tables[t] == mc[1]) slot = (int)t;
    if (slot >= 0) o << "#define " << mc[0] << " ((int)a.rows[" << slot << "])\n";
  }
  o << "\n";
  for (const auto& k : p.kernels) {
    o << "extern \"C\" __global__ void __launch_bounds__(" << p.block_threads << ") " << k.name << "(const CxArgs a) {\n";
    o << "  __shared__ unsigned long long cx_red[BLOCK_THREADS / 32 + 1]; (void)cx_red;\n";
    for (size_t c = 0; c < p.cols.size(); ++c)
      o << "  int* " << p.cols[c].first << " = const_cast<int*>(a.col[" << c << "]); (void)" << p.cols[c].first << ";\n";
    for (const auto& n : p.nulls)
      for (size_t c = 0; c < p.cols.size(); ++c)
        if (p.cols[c].first == n.second)
          o << "  uint64_t* " << n.first << " = (uint64_t*)a.nul[" << c << "]; (void)" << n.first << ";\n";
    for (size_t h = 0; h < p.hts.size(); ++h) o << "  int* " << p.hts[h].name << " = a.ht[" << h << "]; (void)" << p.hts[h].name << ";\n";
    o << "  unsigned long long* d_result = a.result; (void)d_result;\n";
    o << "  uint64_t* d_result_validity = (uint64_t*)a.result_validity; (void)d_result_validity;\n";
    o << "  {" << k.body << "}\n}\n\n";
  }
  return o.str();
}

}  // namespace

namespace cx_internal {

bool is_visitor_program(const std::string& src) {
  return src.find("/*@cx-launch") == std::string::npos &&
         src.find("extern \"C\" void execute_query(db::ExecutionContext* ctx)") != std::string::npos;
}

std::string translate_visitor_program(const std::string& src) { return emit(parse(src)); }

}  // namespace cx_internal

extern "C" int cx_translate_visitor(const char* src, size_t src_len, char* out, size_t out_cap, size_t* out_len) {
  if (!src) return cx_internal::set_error(CX_E_INVALID, "cx_translate_visitor: source is NULL");
  try {
    const std::string t = cx_internal::translate_visitor_program(std::string(src, src_len));
    if (out_len) *out_len = t.size();
    if (out && out_cap) {
      const size_t n = t.size() < out_cap - 1 ? t.size() : out_cap - 1;
      memcpy(out, t.data(), n);
      out[n] = '\0';
      if (n < t.size()) return cx_internal::set_error(CX_E_CAPACITY, "cx_translate_visitor: output buffer too small");
    }
    return CX_OK;
  } catch (const std::exception& e) {
    return cx_internal::set_error(CX_E_INVALID, e.what());
  }
}
