// cx_codegen.cpp -- emits one CUDA C++ translation unit per plan.
//
// Structure of the emitted unit (the CUDA counterpart of the program the
// reference's generateCode prints, src/core/visitor.cpp:4771-4878):
//   1. a launch plan comment the executor reads (buffers, tables, kernels);
//   2. `init_aggregate_slots` when a MIN aggregate needs ~0 slots (:2474-2503);
//   3. one `build_hashtable_<dim>` kernel per join (:4206-4290);
//   4. the fused fact-scan kernel `Scan_<FACT>` (:1657-1751): persistent CTAs,
//      fact-column tiles staged into shared memory by TMA bulk copies, the
//      reference's primitive calls per tile, and block-private aggregation;
//   5. `group_keys_epilogue` when groups are aggregated in global memory;
//   6. `finalize_aggregate_slots` for AVG (:2505-2586).
// Expression strings follow the reference's three translators:
// expressionValidExpr / expressionValueNoEmit (:890-991) for predicates and
// CASE, translateMathExprPush (:1947-2010) for aggregate inputs, and the
// Horner perfect hash of generatePerfectHash (:2056-2127).
#include "cx_codegen.h"

#include "cx_args.h"

#include <algorithm>
#include <cctype>
#include <functional>
#include <map>
#include <set>
#include <cstring>
#include <cctype>
#include <sstream>

namespace cx {

namespace {

bool lit_true(const std::string& v) { return v == "1" || v == "true" || v == "(1)" || v == "(true)"; }
bool lit_false(const std::string& v) { return v == "0" || v == "false" || v == "(0)" || v == "(false)"; }

// Eager mode: conjunctions and disjunctions are emitted as `&` / `|` over
// operands converted to bool, so the generated code evaluates every operand
// and needs no branch per short-circuit.  Only for expressions whose operands
// are safe to evaluate whatever the others' values (registers, literals,
// parameters and the total db::safe_* functions): the fact-filter conditions.
thread_local bool g_eager = false;
struct EagerScope {
  bool prev;
  EagerScope() : prev(g_eager) { g_eager = true; }
  ~EagerScope() { g_eager = prev; }
};
std::string eager_term(const std::string& t) { return "(bool)(" + t + ")"; }

std::string and_terms(const std::vector<std::string>& terms) {
  std::string out;
  int n = 0;
  for (const auto& t : terms) {
    if (t.empty() || lit_true(t)) continue;
    if (!out.empty()) out += g_eager ? " & " : " && ";
    out += g_eager ? eager_term(t) : t;
    ++n;
  }
  if (out.empty()) return "1";
  return g_eager && n > 1 ? "(" + out + ")" : out;
}
std::string b_and(const std::string& a, const std::string& b) {
  if (lit_false(a) || lit_false(b)) return "0";
  if (lit_true(a)) return b;
  if (lit_true(b)) return a;
  if (g_eager) return "(" + eager_term(a) + " & " + eager_term(b) + ")";
  return "(" + a + " && " + b + ")";
}
std::string b_or(const std::string& a, const std::string& b) {
  if (lit_true(a) || lit_true(b)) return "1";
  if (lit_false(a)) return b;
  if (lit_false(b)) return a;
  if (g_eager) return "(" + eager_term(a) + " | " + eager_term(b) + ")";
  return "(" + a + " || " + b + ")";
}
std::string b_not(const std::string& a) {
  if (lit_true(a)) return "0";
  if (lit_false(a)) return "1";
  return "(!(" + a + "))";
}

const char* safe_fn(Op op) {
  switch (op) {
    case Op::Add: return "db::safe_add";
    case Op::Sub: return "db::safe_sub";
    case Op::Mul: return "db::safe_mul";
    case Op::Div: return "db::safe_div";
    case Op::Eq: return "db::safe_eq";
    case Op::Ne: return "db::safe_neq";
    case Op::Lt: return "db::safe_lt";
    case Op::Le: return "db::safe_lte";
    case Op::Gt: return "db::safe_gt";
    case Op::Ge: return "db::safe_gte";
    default: return "?";
  }
}
const char* pred_suffix(Op op) {
  switch (op) {
    case Op::Eq: return "Eq";
    case Op::Ne: return "NEq";
    case Op::Lt: return "LT";
    case Op::Le: return "LTE";
    case Op::Gt: return "GT";
    case Op::Ge: return "GTE";
    default: return "Eq";
  }
}

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

struct Emitter {
  const Plan& p;
  const Tuning& tu;
  std::ostringstream meta;  // launch plan lines
  std::ostringstream src;   // kernels

  std::map<std::string, int> col_slot;  // column -> CxArgs.col slot
  std::vector<std::string> col_order;
  std::map<std::string, int> ht_slot;   // dimension -> CxArgs.ht slot
  std::set<std::string> ptable;          // joins whose scan keeps a payload table in shared memory
  std::set<std::string> payload_valid;  // payload columns that carry validity (PHT_2V)

  // Per-kernel register state.
  std::set<std::string> loaded;         // register arrays holding a column
  std::set<std::string> valid_regs;     // columns with a <col>_valid register

  // Shared-scan mode: integer literals become per-query parameters P[k]
  // (or hoisted registers P<k> when param_regs is set).
  const std::map<const Expr*, int>* lit_index = nullptr;
  bool param_regs = false;
  int nparams = -1;  // plain parametric kernels: literals read from CxArgs.lits

  std::string param_decl() const {
    return nparams >= 0 ? "  const int* __restrict__ P = a.lits; (void)P;\n" : "";
  }

  Emitter(const Plan& plan, const Tuning& t) : p(plan), tu(t) {}

  std::string int_lit(const Expr* e) const {
    if (lit_index) {
      auto it = lit_index->find(e);
      if (it != lit_index->end())
        return param_regs ? "P" + std::to_string(it->second) : "P[" + std::to_string(it->second) + "]";
    }
    return std::to_string(e->ival);
  }

  bool nullable(const std::string& c) const { return p.nullable.count(c) != 0; }

  int slot_of(const std::string& c) {
    auto it = col_slot.find(c);
    if (it != col_slot.end()) return it->second;
    const int s = (int)col_order.size();
    if (s >= 40) throw PlanError("too many columns for one query");
    col_slot[c] = s;
    col_order.push_back(c);
    return s;
  }

  // ---------------------------------------------------------- expressions --
  // Column spelling override (shared-scan kernels read columns from
  // shared-memory tiles or dimension rows rather than register arrays).
  std::map<std::string, std::string> col_expr;
  std::string reg(const std::string& c) const {
    auto it = col_expr.find(c);
    return it != col_expr.end() ? it->second : c + "[i]";
  }

  std::string valid_of(const Expr* e) const {
    if (!e) return "1";
    switch (e->op) {
      case Op::Null: return "0";
      case Op::Star: case Op::Int: case Op::IsNull: case Op::NotNull: return "1";
      case Op::Col: return valid_regs.count(e->name) ? e->name + "_valid[i]" : "1";
      case Op::Not: return valid_of(e->kids[0].get());
      case Op::And: {
        const std::string lv = valid_of(e->kids[0].get()), rv = valid_of(e->kids[1].get());
        const std::string l = value_of(e->kids[0].get()), r = value_of(e->kids[1].get());
        return b_or(b_or(and_terms({lv, b_not(l)}), and_terms({rv, b_not(r)})), and_terms({lv, rv}));
      }
      case Op::Or: {
        const std::string lv = valid_of(e->kids[0].get()), rv = valid_of(e->kids[1].get());
        const std::string l = value_of(e->kids[0].get()), r = value_of(e->kids[1].get());
        return b_or(b_or(and_terms({lv, l}), and_terms({rv, r})), and_terms({lv, rv}));
      }
      case Op::Case: {
        const std::string cv = valid_of(e->kids[0].get()), c = value_of(e->kids[0].get());
        const std::string then_sel = and_terms({cv, c});
        const std::string else_sel = b_not(then_sel);
        return b_or(and_terms({then_sel, valid_of(e->kids[1].get())}), and_terms({else_sel, valid_of(e->kids[2].get())}));
      }
      default:  // arithmetic and comparisons: both operands known
        return and_terms({valid_of(e->kids[0].get()), valid_of(e->kids[1].get())});
    }
  }

  std::string value_of(const Expr* e) const {
    if (!e) return "0";
    switch (e->op) {
      case Op::Col: return reg(e->name);
      case Op::Int: return int_lit(e);
      case Op::Null: return "0";
      case Op::Star: return "1";
      case Op::IsNull:
      case Op::NotNull: {
        const std::string v = valid_of(e->kids[0].get());
        if (lit_true(v)) return e->op == Op::IsNull ? "0" : "1";
        if (lit_false(v)) return e->op == Op::IsNull ? "1" : "0";
        return e->op == Op::IsNull ? "(!(" + v + "))" : "(" + v + ")";
      }
      case Op::Not: return b_not(value_of(e->kids[0].get()));
      case Op::And: return b_and(value_of(e->kids[0].get()), value_of(e->kids[1].get()));
      case Op::Or: return b_or(value_of(e->kids[0].get()), value_of(e->kids[1].get()));
      case Op::Case: {
        const std::string sel = and_terms({valid_of(e->kids[0].get()), value_of(e->kids[0].get())});
        return "((" + sel + ") ? (" + value_of(e->kids[1].get()) + ") : (" + value_of(e->kids[2].get()) + "))";
      }
      default:
        return std::string(safe_fn(e->op)) + "(" + value_of(e->kids[0].get()) + ", " + value_of(e->kids[1].get()) + ")";
    }
  }

  // Aggregate input: only the leftmost leaf is widened to u64 (reference
  // translateMathExprPush), so right operands keep their C types.
  std::string math_push(const Expr* e, bool cast) const {
    if (!e) return "0";
    switch (e->op) {
      case Op::Col: return cast ? "(unsigned long long)" + reg(e->name) : reg(e->name);
      case Op::Int: return int_lit(e);
      case Op::Star: return cast ? "(unsigned long long)1" : "1";
      case Op::Null: return "0";
      case Op::Add: case Op::Sub: case Op::Mul: {
        const char* op = e->op == Op::Add ? " + " : e->op == Op::Sub ? " - " : " * ";
        return "(" + math_push(e->kids[0].get(), cast) + op + math_push(e->kids[1].get(), false) + ")";
      }
      case Op::Div:
        return "cx_mdiv(" + math_push(e->kids[0].get(), cast) + ", " + math_push(e->kids[1].get(), false) + ")";
      case Op::IsNull: case Op::NotNull: {
        const std::string v = value_of(e);
        return cast ? "(unsigned long long)" + v : v;
      }
      default: {
        const std::string v = value_of(e);
        return cast ? "(unsigned long long)(" + v + ")" : v;
      }
    }
  }

  void collect(const Expr* e, std::vector<std::string>& out) const {
    if (!e) return;
    if (e->op == Op::Col && std::find(out.begin(), out.end(), e->name) == out.end()) out.push_back(e->name);
    for (const auto& k : e->kids) collect(k.get(), out);
  }

  // ---------------------------------------------------------------- loads --
  // `tile_ptr(col)` names the pointer to the current tile of a column.
  std::function<std::string(const std::string&)> tile_ptr;

  void ensure_loaded(std::ostream& o, const std::string& c, const std::string& ind) {
    if (loaded.count(c)) return;
    loaded.insert(c);
    o << ind << "BlockLoad<int, BLOCK_THREADS, ITEMS_PER_THREAD>(" << tile_ptr(c)
      << ", tid, tile_offset, " << c << ", num_tile_items);\n";
    if (nullable(c)) {
      valid_regs.insert(c);
      o << ind << "BlockLoadValidity<BLOCK_THREADS, ITEMS_PER_THREAD>(n_" << c << ", tid, tile_offset, " << c
        << "_valid, num_tile_items);\n";
    }
  }

  void load_expr_cols(std::ostream& o, const Expr* e, const std::string& ind) {
    std::vector<std::string> cols;
    collect(e, cols);
    for (const auto& c : cols)
      if (!loaded.count(c)) ensure_loaded(o, c, ind);
  }

  // A filter step: AND-chains of non-nullable `column op literal` leaves use
  // the BlockPredA* primitives (the reference fast path, visitor.cpp:1838-1880);
  // every other leaf is evaluated under three-valued logic, keeping a row only
  // when the predicate is known TRUE.
  void emit_filter(std::ostream& o, const Expr* e, const std::string& ind) {
    if (e->op == Op::And) {
      emit_filter(o, e->kids[0].get(), ind);
      emit_filter(o, e->kids[1].get(), ind);
      return;
    }
    load_expr_cols(o, e, ind);
    if (is_compare(e->op) && e->kids[0]->op == Op::Col && e->kids[1]->op == Op::Int &&
        !valid_regs.count(e->kids[0]->name) && e->kids[1]->ival >= -2147483647LL && e->kids[1]->ival <= 2147483647LL) {
      o << ind << "BlockPredA" << pred_suffix(e->op) << "<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, "
        << e->kids[0]->name << ", flags, " << int_lit(e->kids[1].get()) << ", num_tile_items);\n";
      return;
    }
    std::string cond;
    {
      EagerScope eager;  // the whole condition evaluated without branches
      cond = and_terms({valid_of(e), value_of(e)});
    }
    if (lit_true(cond)) return;
    o << ind << "#pragma unroll\n"
      << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n"
      << ind << "  flags[i] = (tid + BLOCK_THREADS * i < num_tile_items) ? ((int)(flags[i] != 0) & (int)(bool)(" << cond
      << ")) : flags[i];\n"
      << ind << "}\n";
  }

  std::string ht_name(const std::string& dim) const { return "d_" + lower(dim) + "_hash_table"; }

  // ---------------------------------------------------------------- meta --
  void declare_cols(std::ostream& o, const std::vector<std::string>& cols, const std::string& ind) {
    for (const auto& c : cols) {
      const int s = slot_of(c);
      o << ind << "const int* __restrict__ d_" << c << " = a.col[" << s << "];\n";
      if (nullable(c)) o << ind << "const uint64_t* n_" << c << " = (const uint64_t*)a.nul[" << s << "];\n";
    }
  }
  void declare_regs(std::ostream& o, const std::vector<std::string>& cols, const std::string& ind) {
    for (const auto& c : cols) {
      o << ind << "int " << c << "[ITEMS_PER_THREAD];\n";
      if (nullable(c) || payload_valid.count(c)) o << ind << "int " << c << "_valid[ITEMS_PER_THREAD];\n";
    }
  }

  // ------------------------------------------------------------- builds ---
  // Multi-value hash table scratch (ints, one `ht` slot): the directory
  // [key, offset, count] per slot at 0, then counts, offsets, write cursors
  // and the per-4096-slot block sums of the offset scan.
  static long long mht_blocks(const Join& j) { return (j.len + 4095) / 4096; }
  static long long mht_words(const Join& j) { return 6 * j.len + mht_blocks(j) + 1; }
  // The MHT payload holds, per entry, the build row id and a copy of every
  // build column the probe publishes (and its validity where nullable), each
  // in its own array of build-table length: a probe reads the values directly
  // instead of first loading the row id and then gathering by it.
  int mht_arrays(const Join& j) const {
    int n = 1;
    for (const auto& g : j.gathers) n += nullable(g) ? 2 : 1;
    return n;
  }
  // Array index of gathered column g (and of its validity, + 1).
  int mht_array_of(const Join& j, const std::string& g) const {
    int n = 1;
    for (const auto& c : j.gathers) {
      if (c == g) return n;
      n += nullable(c) ? 2 : 1;
    }
    throw PlanError("column " + g + " is not gathered by the join on " + j.dim);
  }
  // Loads of the published columns of MHT entry `pos` (an expression).
  void emit_mht_gathers(std::ostream& o, const Join& j, const std::string& pos, const std::string& ind) {
    const std::string d = lower(j.dim);
    for (const auto& g : j.gathers) {
      const int k = mht_array_of(j, g);
      o << ind << g << "[i] = mpay_" << d << "[" << k << "LL * mst_" << d << " + " << pos << "];\n";
      if (nullable(g)) o << ind << g << "_valid[i] = mpay_" << d << "[" << k + 1 << "LL * mst_" << d << " + " << pos << "];\n";
    }
  }

  // Build-side prologue shared by the PHT and MHT build kernels: the tile loop
  // over the dimension, its filter and the key's validity.
  void build_prologue(std::ostream& o, const Join& j, const std::vector<std::string>& cols, int t) {
    o << "  constexpr int BLOCK_THREADS = 128, ITEMS_PER_THREAD = 4, TILE_SIZE = 512;\n";
    o << "  const int tid = threadIdx.x;\n";
    o << "  const long long n_rows = a.rows[" << t << "];\n";
    declare_cols(o, cols, "  ");
    o << "  for (long long tile = blockIdx.x; tile * TILE_SIZE < n_rows; tile += gridDim.x) {\n";
    o << "    const long long tile_offset = tile * TILE_SIZE;\n";
    o << "    const int num_tile_items = (int)(n_rows - tile_offset < TILE_SIZE ? n_rows - tile_offset : TILE_SIZE);\n";
    o << "    int flags[ITEMS_PER_THREAD];\n";
    declare_regs(o, cols, "    ");
    o << "    InitFlags<BLOCK_THREADS, ITEMS_PER_THREAD>(flags);\n";
    if (j.filter) emit_filter(o, j.filter.get(), "    ");
    ensure_loaded(o, j.pk, "    ");
    if (nullable(j.pk))
      o << "    BlockApplyValidityAnd<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, flags, " << j.pk << "_valid, num_tile_items);\n";
  }

  // MHT build (emitMHTBuildKernels, visitor.cpp:4295-4464): count per slot,
  // a three-kernel exclusive scan of the counts, then the write of build row
  // ids.  The payload array is sized by the dimension's rows, so nothing is
  // read back to the host between the passes.  A slot that receives two
  // distinct keys raises ERR_DIM_COLLISION (the count pass stores each row's
  // key, the write pass checks it before the directory is rewritten).
  void emit_mht_build(const Join& j) {
    const int t = p.table_slot(j.dim);
    const int h = ht_slot.at(j.dim);
    const long long L = j.len, NB = mht_blocks(j);
    const std::string d = lower(j.dim);
    std::vector<std::string> cols;
    if (j.filter) collect(j.filter.get(), cols);
    if (std::find(cols.begin(), cols.end(), j.pk) == cols.end()) cols.push_back(j.pk);
    const std::string Ls = std::to_string(L) + "LL";
    auto views = [&](std::ostream& o) {
      o << "  int* ht_dir = a.ht[" << h << "]; (void)ht_dir;\n";
      o << "  int* mht_counts = ht_dir + 3 * " << Ls << "; (void)mht_counts;\n";
      o << "  int* mht_offsets = ht_dir + 4 * " << Ls << "; (void)mht_offsets;\n";
      o << "  int* mht_wpos = ht_dir + 5 * " << Ls << "; (void)mht_wpos;\n";
      o << "  int* mht_bsum = ht_dir + 6 * " << Ls << "; (void)mht_bsum;\n";
    };
    auto key_loop = [&](std::ostream& o, const std::string& body) {
      o << "    #pragma unroll\n    for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
      o << "      if (flags[i] && tid + BLOCK_THREADS * i < num_tile_items) {\n";
      o << "        const int s_ = cx_detail::pht_slot<int>(" << j.pk << "[i], " << L << ", " << j.keymin << ");\n";
      o << "        if (s_ >= 0) " << body << "\n";
      o << "      }\n    }\n";
    };

    // Pass 1: count.
    {
      const std::string kname = "mht_count_" + d;
      meta << "kernel " << kname << " build " << t << " 128 512\n";
      loaded.clear();
      valid_regs.clear();
      tile_ptr = [](const std::string& c) { return "d_" + c + " + tile_offset"; };
      std::ostringstream& o = src;
      o << "extern \"C\" __global__ void __launch_bounds__(128) " << kname << "(const CxArgs a) {\n";
      o << param_decl();
      views(o);
      build_prologue(o, j, cols, t);
      o << "    BlockBuildMHT_Count<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << j.pk << ", flags, mht_counts, " << L
        << ", " << j.keymin << ", num_tile_items);\n";
      key_loop(o, "ht_dir[3LL * s_] = " + j.pk + "[i];");
      o << "  }\n}\n\n";
    }
    // Pass 2: per-block sums of 4096 counts.
    {
      const std::string kname = "mht_blocksum_" + d;
      meta << "kernel " << kname << " fixed " << NB << " 256 0\n";
      src << "extern \"C\" __global__ void __launch_bounds__(256) " << kname << "(const CxArgs a) {\n";
      views(src);
      src << "  __shared__ unsigned long long red[8];\n";
      src << "  const long long base = (long long)blockIdx.x * 4096LL;\n";
      src << "  unsigned long long s = 0;\n";
      src << "  for (int k = threadIdx.x; k < 4096; k += 256) {\n";
      src << "    const long long x = base + k;\n";
      src << "    if (x < " << Ls << ") s += (unsigned long long)mht_counts[x];\n";
      src << "  }\n";
      src << "  s = cx::block_sum_u64<256>(s, red);\n";
      src << "  if (threadIdx.x == 0) mht_bsum[blockIdx.x] = (int)s;\n";
      src << "}\n\n";
    }
    // Pass 3: exclusive scan of the block sums (one CTA).
    {
      const std::string kname = "mht_blockscan_" + d;
      meta << "kernel " << kname << " fixed 1 1024 0\n";
      src << "extern \"C\" __global__ void __launch_bounds__(1024) " << kname << "(const CxArgs a) {\n";
      views(src);
      src << "  __shared__ long long sc[33];\n";
      src << "  long long carry = 0;\n";
      src << "  for (long long b0 = 0; b0 < " << NB << "LL; b0 += 1024) {\n";
      src << "    const long long b = b0 + threadIdx.x;\n";
      src << "    const long long v = b < " << NB << "LL ? (long long)mht_bsum[b] : 0LL;\n";
      src << "    long long tot = 0;\n";
      src << "    const long long ex = cx::block_exclusive_scan_i64<1024>(v, sc, &tot);\n";
      src << "    if (b < " << NB << "LL) mht_bsum[b] = (int)(carry + ex);\n";
      src << "    carry += tot;\n";
      src << "  }\n";
      src << "}\n\n";
    }
    // Pass 4: slot offsets = block base + scan within the block.
    {
      const std::string kname = "mht_offsets_" + d;
      meta << "kernel " << kname << " fixed " << NB << " 256 0\n";
      src << "extern \"C\" __global__ void __launch_bounds__(256) " << kname << "(const CxArgs a) {\n";
      views(src);
      src << "  __shared__ long long sc[9];\n";
      src << "  const long long base = (long long)blockIdx.x * 4096LL + (long long)threadIdx.x * 16;\n";
      src << "  int v[16];\n";
      src << "  long long loc = 0;\n";
      src << "  #pragma unroll\n  for (int k = 0; k < 16; ++k) {\n";
      src << "    v[k] = base + k < " << Ls << " ? mht_counts[base + k] : 0;\n";
      src << "    loc += v[k];\n";
      src << "  }\n";
      src << "  long long tot = 0;\n";
      src << "  long long run = (long long)mht_bsum[blockIdx.x] + cx::block_exclusive_scan_i64<256>(loc, sc, &tot);\n";
      src << "  #pragma unroll\n  for (int k = 0; k < 16; ++k) {\n";
      src << "    if (base + k < " << Ls << ") mht_offsets[base + k] = (int)run;\n";
      src << "    run += v[k];\n";
      src << "  }\n";
      src << "}\n\n";
    }
    // Pass 5: write row ids and the directory.
    {
      const std::string kname = "mht_write_" + d;
      meta << "kernel " << kname << " build " << t << " 128 512\n";
      loaded.clear();
      valid_regs.clear();
      tile_ptr = [](const std::string& c) { return "d_" + c + " + tile_offset"; };
      std::ostringstream& o = src;
      o << "extern \"C\" __global__ void __launch_bounds__(128) " << kname << "(const CxArgs a) {\n";
      o << param_decl();
      views(o);
      o << "  int* mht_payload = a.mpay[" << h << "];\n";
      o << "  const long long mst_ = a.rows[" << t << "]; (void)mst_;\n";
      std::vector<std::string> wcols = cols;
      for (const auto& g : j.gathers)
        if (std::find(wcols.begin(), wcols.end(), g) == wcols.end()) wcols.push_back(g);
      build_prologue(o, j, wcols, t);
      for (const auto& g : j.gathers) ensure_loaded(o, g, "    ");
      o << "    int row_ids[ITEMS_PER_THREAD];\n";
      o << "    BlockMakeRowIds<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, (int)tile_offset, row_ids, num_tile_items);\n";
      key_loop(o, "{ if (((volatile int*)ht_dir)[3LL * s_] != " + j.pk + "[i]) cx::raise(a.err, cx::ERR_DIM_COLLISION); }");
      // BlockBuildMHT_Write (include/crystal/join.h) places each row id at
      // its slot's next position; the published columns go to the same
      // position of their own arrays.
      o << "    #pragma unroll\n    for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
      o << "      if (!flags[i] || tid + BLOCK_THREADS * i >= num_tile_items) continue;\n";
      o << "      const int s_ = cx_detail::pht_slot<int>(" << j.pk << "[i], " << L << ", " << j.keymin << ");\n";
      o << "      if (s_ < 0) continue;\n";
      o << "      const long long pos_ = (long long)mht_offsets[s_] + atomicAdd(&mht_wpos[s_], 1);\n";
      o << "      mht_payload[pos_] = row_ids[i];\n";
      for (const auto& g : j.gathers) {
        const int k = mht_array_of(j, g);
        o << "      mht_payload[" << k << "LL * mst_ + pos_] = " << g << "[i];\n";
        if (nullable(g)) o << "      mht_payload[" << k + 1 << "LL * mst_ + pos_] = " << g << "_valid[i];\n";
      }
      o << "      ht_dir[3LL * s_ + 0] = " << j.pk << "[i];\n";
      o << "      ht_dir[3LL * s_ + 1] = mht_offsets[s_];\n";
      o << "      ht_dir[3LL * s_ + 2] = mht_counts[s_];\n";
      o << "    }\n";
      o << "  }\n}\n\n";
    }
  }

  void emit_build(const Join& j) {
    if (j.multi) return emit_mht_build(j);
    const int t = p.table_slot(j.dim);
    const int h = ht_slot.at(j.dim);
    std::vector<std::string> cols;
    if (j.filter) collect(j.filter.get(), cols);
    for (const std::string& c : {j.pk, j.payload})
      if (!c.empty() && std::find(cols.begin(), cols.end(), c) == cols.end()) cols.push_back(c);
    const bool v2 = !j.payload.empty();
    const bool v2v = v2 && payload_valid.count(j.payload);
    const std::string kname = "build_hashtable_" + lower(j.dim);
    meta << "kernel " << kname << " build " << t << " 128 512\n";

    loaded.clear();
    valid_regs.clear();
    tile_ptr = [](const std::string& c) { return "d_" + c + " + tile_offset"; };
    std::ostringstream& o = src;
    o << "extern \"C\" __global__ void __launch_bounds__(128) " << kname << "(const CxArgs a) {\n";
    o << param_decl();
    o << "  int* " << ht_name(j.dim) << " = a.ht[" << h << "];\n";
    if (v2v) o << "  unsigned int* " << ht_name(j.dim) << "_valid = a.htv[" << h << "];\n";
    build_prologue(o, j, cols, t);
    if (!v2) {
      o << "    BlockBuildSelectivePHT_1<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << j.pk << ", flags, "
        << ht_name(j.dim) << ", " << j.len << ", " << j.keymin << ", num_tile_items);\n";
    } else {
      ensure_loaded(o, j.payload, "    ");
      if (v2v) {
        o << "    BlockBuildSelectivePHT_2V<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << j.pk << ", "
          << j.payload << ", " << j.payload << "_valid, flags, " << ht_name(j.dim) << ", " << ht_name(j.dim)
          << "_valid, " << j.len << ", " << j.keymin << ", num_tile_items);\n";
      } else {
        o << "    BlockBuildSelectivePHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << j.pk << ", "
          << j.payload << ", flags, " << ht_name(j.dim) << ", " << j.len << ", " << j.keymin << ", num_tile_items);\n";
      }
    }
    o << "  }\n}\n\n";
  }

  // Exact-membership bitmap of a built PHT: bit h is set when slot h holds
  // the key key_min + h, i.e. when a probe of that in-window key hits.
  static bool exact_window_ok(const Join& j) {
    return j.keymin >= -2147483648LL && j.keymin + j.len - 1 <= 2147483647LL;
  }
  // Joins whose payload's catalog range fits a byte get a payload table
  // instead (one byte per slot, see BlockProbeExactTable), in join order while
  // the tables fit `table_budget` bytes of shared memory.
  bool table_candidate(const Join& j) const {
    return !j.multi && !j.expands() && exact_window_ok(j) && !j.payload.empty() && !payload_valid.count(j.payload) &&
           j.prange_card >= 1 && j.prange_card <= 254;
  }
  void choose_tables() {
    unsigned long long used = 0;
    for (const auto& s : p.steps) {
      if (s.kind != Step::JoinStep || !table_candidate(s.join)) continue;
      const unsigned long long bytes = (((unsigned long long)s.join.len + 3) / 4 * 4 + 15) & ~15ULL;
      if (used + bytes > (unsigned long long)std::max(0, tu.table_budget)) continue;
      ptable.insert(s.join.dim);
      used += bytes;
    }
  }
  void emit_payload_table(const Join& j) {
    const int h = ht_slot.at(j.dim);
    const long long words = (j.len + 3) / 4;
    const std::string kname = "occupancy_" + lower(j.dim);
    meta << "kernel " << kname << " fixed " << (words + 255) / 256 << " 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) " << kname << "(const CxArgs a) {\n";
    src << param_decl();
    src << "  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n";
    src << "  if (w >= " << words << "LL) return;\n";
    src << "  const int* ht = a.ht[" << h << "];\n";
    src << "  unsigned bytes = 0u;\n";
    src << "  for (int b = 0; b < 4; ++b) {\n";
    src << "    const long long slot = w * 4 + b;\n";
    src << "    unsigned v = 0xFFu;\n";
    src << "    if (slot < " << j.len << "LL && ht[slot * 2] == (int)(" << j.keymin << "LL + slot)) {\n";
    src << "      const long long pv = (long long)ht[slot * 2 + 1] - (" << j.prange_min << "LL);\n";
    src << "      v = (pv >= 0 && pv < " << j.prange_card << "LL) ? (unsigned)pv : 0xFEu;\n";
    src << "    }\n";
    src << "    bytes |= v << (8 * b);\n";
    src << "  }\n";
    src << "  a.bm[" << h << "][w] = bytes;\n";
    src << "}\n\n";
  }
  void emit_occupancy(const Join& j) {
    if (j.multi) return;
    if (ptable.count(j.dim)) return emit_payload_table(j);
    const int h = ht_slot.at(j.dim);
    const long long words = (j.len + 31) / 32;
    const std::string kname = "occupancy_" + lower(j.dim);
    meta << "kernel " << kname << " fixed " << (words + 255) / 256 << " 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) " << kname << "(const CxArgs a) {\n";
    src << param_decl();
    src << "  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n";
    src << "  if (w >= " << words << "LL) return;\n";
    src << "  const int* ht = a.ht[" << h << "];\n";
    src << "  unsigned bits = 0u;\n";
    src << "  for (int b = 0; b < 32; ++b) {\n";
    src << "    const long long slot = w * 32 + b;\n";
    src << "    if (slot < " << j.len << "LL && ht[slot" << (j.payload.empty() ? "" : " * 2") << "] == (int)(" << j.keymin
        << "LL + slot)) bits |= 1u << b;\n";
    src << "  }\n";
    src << "  a.bm[" << h << "][w] = bits;\n";
    src << "}\n\n";
  }

  // --------------------------------------------------------- group hash ---
  std::string group_term(size_t k) const {
    const GroupKey& g = p.groups[k];
    const std::string v = value_of(g.expr.get());
    if (!g.nullable) return "(" + v + " - " + std::to_string(g.min) + ")";
    return "((" + valid_of(g.expr.get()) + ") ? (" + v + " - " + std::to_string(g.min) + " + 1) : 0)";
  }
  long long eff_card(size_t k) const { return p.groups[k].card + (p.groups[k].nullable ? 1 : 0); }
  // Storage slot of an unconditional COUNT(*) aggregate (-1 if none).
  int count_star_slot() const {
    for (size_t k = 0; k < p.aggs.size(); ++k)
      if (p.aggs[k].fn == AggFn::Count && p.aggs[k].arg && p.aggs[k].arg->op == Op::Star) return (int)(p.groups.size() + k);
    return -1;
  }
  unsigned long long total_groups() const {
    unsigned long long t = 1;
    for (size_t k = 0; k < p.groups.size(); ++k) t *= (unsigned long long)eff_card(k);
    return t;
  }

  // Canonical key values of group `gvar` (decoded from the perfect hash).
  void emit_key_store(std::ostream& o, const std::string& gvar, const std::string& ind) {
    const int ts = p.storage_ts();
    o << ind << "long long rem = " << gvar << ";\n";
    for (size_t kk = p.groups.size(); kk-- > 0;) {
      o << ind << "const long long gd" << kk << " = rem % " << eff_card(kk) << "LL; rem /= " << eff_card(kk) << "LL;\n";
    }
    o << ind << "(void)rem;\n";
    for (size_t k = 0; k < p.groups.size(); ++k) {
      const GroupKey& g = p.groups[k];
      const std::string slot = "(unsigned long long)" + gvar + " * " + std::to_string(ts) + "ULL + " + std::to_string(k);
      if (g.nullable) {
        o << ind << "d_result[" << slot << "] = (gd" << k << " == 0) ? 0ULL : (unsigned long long)(gd" << k << " - 1 + "
          << g.min << "LL);\n";
        if (!p.sparse) o << ind << "if (gd" << k << " != 0) db::atomic_set_valid_bit(d_result_validity, " << slot << ");\n";
      } else {
        o << ind << "d_result[" << slot << "] = (unsigned long long)(gd" << k << " + " << g.min << "LL);\n";
        if (!p.sparse) o << ind << "db::atomic_set_valid_bit(d_result_validity, " << slot << ");\n";
      }
    }
  }

  // ----------------------------------------------------------------- scan --
  void emit_scan() {
    const int CTA = tu.block_threads, IPT = tu.items_per_thread;
    if (CTA % 32 || CTA < 32 || CTA > 1024 || IPT < 1 || IPT > 16) throw PlanError("bad block shape");
    const int NW = CTA / 32;
    const int WT = 32 * IPT;  // rows of one warp tile
    const std::string fact = p.tables[0].name;

    // Fact columns the pipeline reads, in first-use order.
    std::vector<std::string> fact_cols;
    auto add_fact = [&](const Expr* e) {
      std::vector<std::string> cs;
      collect(e, cs);
      for (const auto& c : cs)
        if (p.table_of_col.at(c) == 0 && std::find(fact_cols.begin(), fact_cols.end(), c) == fact_cols.end())
          fact_cols.push_back(c);
    };
    std::vector<std::string> payload_cols;
    for (const auto& s : p.steps) {
      if (s.kind == Step::Filter) add_fact(s.filter.get());
      else {
        for (const auto& fk : s.join.fks)
          if (std::find(fact_cols.begin(), fact_cols.end(), fk) == fact_cols.end()) fact_cols.push_back(fk);
        if (!s.join.payload.empty()) payload_cols.push_back(s.join.payload);
      }
    }
    for (const auto& g : p.groups) add_fact(g.expr.get());
    for (const auto& ag : p.aggs) add_fact(ag.arg.get());
    // The first join that can emit a row more than once (an OR over several
    // fact keys or an MHT) switches the rest of the pipeline to item mode.
    std::vector<std::string> gather_cols;
    size_t xs = p.steps.size();
    for (size_t k = 0; k < p.steps.size(); ++k) {
      const Step& s = p.steps[k];
      if (s.kind != Step::JoinStep) continue;
      for (const auto& g : s.join.gathers) gather_cols.push_back(g);
      if (s.join.expands() && xs == p.steps.size()) xs = k;
    }
    const bool expanding = xs < p.steps.size();

    const int NSC = (int)fact_cols.size();
    const int STAGES = (NSC == 0) ? 0 : std::max(0, tu.stages);
    const bool grouped = !p.groups.empty();
    const unsigned long long G = total_groups();
    const int TS = p.storage_ts();
    const int NA = (int)p.aggs.size();
    int n_avg = 0;
    for (const auto& ag : p.aggs) n_avg += ag.fn == AggFn::Avg;
    const int NACC = NA + n_avg;                 // accumulator words per group
    std::vector<int> seen_idx(NA, -1);           // SUM/MIN/MAX track "any valid input"
    std::vector<int> avg_idx(NA, -1);            // accumulator word of an AVG's hidden count
    int NSEEN = 0;
    for (int k = 0, ai = 0; k < NA; ++k) {
      const AggFn f = p.aggs[k].fn;
      if (f == AggFn::Sum || f == AggFn::Min || f == AggFn::Max) seen_idx[k] = NSEEN++;
      if (f == AggFn::Avg) avg_idx[k] = NA + ai++;
    }
    const int NSEEN_T = p.sparse ? 0 : NSEEN;    // seen bitmaps actually kept
    const unsigned long long TW = (G + 31) / 32; // words of one group bitmap

    // Shared memory: per-warp staging rings, per-warp mbarriers, reduction
    // scratch, then the group tables (one per CTA, or one per warp when the
    // group domain is small enough to replicate).
    const unsigned long long warp_stage_ints = (unsigned long long)STAGES * NSC * WT;
    unsigned long long off = (unsigned long long)NW * warp_stage_ints * 4;
    const unsigned long long bars_off = off; off += (unsigned long long)NW * std::max(STAGES, 1) * 8;
    const unsigned long long red_off = off; off += (unsigned long long)NW * 8;
    // Join membership bitmaps kept in shared memory (in join order, while they fit the budget).
    // Payload tables (one byte per slot: membership and payload) take the
    // joins choose_tables picked; the others get bitmaps while they fit.
    struct SBm {
      std::string dim, fk; int h; long long len, keymin; unsigned long long words, off; bool pair, table;
      long long vmin;
    };
    std::vector<SBm> sbms;
    {
      unsigned long long used = 0;
      for (const auto& s : p.steps) {
        if (s.kind != Step::JoinStep || s.join.expands() || !exact_window_ok(s.join)) continue;
        const bool table = ptable.count(s.join.dim) > 0;
        const unsigned long long words = (unsigned long long)(table ? (s.join.len + 3) / 4 : (s.join.len + 31) / 32);
        const unsigned long long bytes = ((words * 4) + 15) & ~15ULL;
        if (!table && used + bytes > (unsigned long long)std::max(0, tu.bitmap_budget)) continue;
        off = (off + 15) & ~15ULL;
        sbms.push_back({s.join.dim, s.join.fks[0], ht_slot.at(s.join.dim), s.join.len, s.join.keymin, words, off,
                        !s.join.payload.empty(), table, s.join.prange_min});
        off += bytes;
        if (!table) used += bytes;
      }
    }
    bool smem_groups = false;
    // Tiny group domains accumulate in registers for the whole kernel and are
    // reduced across the CTA once at the end (the reference's local group
    // reduce for <= 64 groups, visitor.cpp:2901-2982, without per-tile atomics).
    // Tiny domains live per thread: in shared-memory slots ([word][thread],
    // conflict-free; one load-add-store per update) when they fit the group
    // budget, else in registers selected by a compare chain over the groups.
    const bool tiny = grouped && G <= 32 && G * NACC <= 16;
    const bool lane_groups = tiny && (tu.group_placement == 4 ||
                                      (tu.group_placement == 0 &&
                                       G * NACC * 8ULL * CTA <= (unsigned long long)std::max(0, tu.smem_group_budget)));
    const bool reg_groups = tiny && !lane_groups && (tu.group_placement == 0 || tu.group_placement == 3);
    int REP = 1;
    unsigned long long acc_off = 0, touch_off = 0, seen_off = 0;
    unsigned long long lacc_off = 0;
    if (lane_groups) {
      lacc_off = (off + 15) & ~15ULL;
      off = lacc_off + G * NACC * 8ULL * CTA;
    }
    if (grouped && !reg_groups && !lane_groups) {
      const unsigned long long one = G * NACC * 8 + TW * 4 * (1 + NSEEN_T);
      if (tu.group_placement == 1) smem_groups = true;
      else if (tu.group_placement == 2) smem_groups = false;
      else smem_groups = one <= (unsigned long long)tu.smem_group_budget;
      if (smem_groups) {
        if (G <= 256 && one * NW <= (unsigned long long)tu.smem_group_budget) REP = NW;
        acc_off = (off + 15) & ~15ULL; off = acc_off + (unsigned long long)REP * G * NACC * 8;
        touch_off = off; off += (unsigned long long)REP * TW * 4;
        seen_off = off; off += (unsigned long long)REP * NSEEN_T * TW * 4;
      }
    }
    // Warp compaction of qualifying rows (grouped, non-expanding plans with
    // every fact column vector-loaded at the tile start): after the cheap
    // membership tests (exact join bitmaps, filters over fact columns) each
    // warp appends its qualifying rows' values to a per-warp queue in shared
    // memory and runs the rest of the pipeline -- payload fetches, remaining
    // probes and filters, the group update -- on 32 queued rows at a time with
    // every lane busy, instead of on mostly idle lanes of every tile.
    const bool vec_pf_all = STAGES == 0 && NSC > 0 && (IPT == 1 || IPT == 2 || IPT % 4 == 0) && tu.prefetch > 0;
    const bool compact = tu.compact > 0 && !expanding && grouped && vec_pf_all;
    // Queued rows run the rest of the pipeline 32 x DB at a time (compact = 2:
    // two batches' gathers in flight together, half the drains).
    const int DB = compact ? std::max(1, std::min(2, tu.compact)) : 1;
    std::set<std::string> exact_set;
    for (const auto& b : sbms) exact_set.insert(b.dim);
    auto fact_only = [&](const Expr* e) {
      std::vector<std::string> cs;
      collect(e, cs);
      for (const auto& c : cs)
        if (p.table_of_col.at(c) != 0) return false;
      return true;
    };
    std::vector<std::string> qcols;  // fact columns (and validity) the queued rows carry
    auto add_q = [&](const std::string& c) {
      if (p.table_of_col.at(c) == 0 && std::find(qcols.begin(), qcols.end(), c) == qcols.end()) qcols.push_back(c);
    };
    if (compact) {
      for (const auto& s : p.steps) {
        if (s.kind == Step::Filter) {
          if (!fact_only(s.filter.get())) {
            std::vector<std::string> cs;
            collect(s.filter.get(), cs);
            for (const auto& c : cs) add_q(c);
          }
        } else if (!exact_set.count(s.join.dim) || !s.join.payload.empty()) {
          add_q(s.join.fks[0]);
        }
      }
      for (const auto& g : p.groups) {
        std::vector<std::string> cs;
        collect(g.expr.get(), cs);
        for (const auto& c : cs) add_q(c);
      }
      for (const auto& ag : p.aggs) {
        std::vector<std::string> cs;
        collect(ag.arg.get(), cs);
        for (const auto& c : cs) add_q(c);
      }
    }
    int NQ = 0;
    for (const auto& c : qcols) NQ += 1 + (nullable(c) ? 1 : 0);
    const int QCAP = 32 * (IPT + DB);
    unsigned long long q_off = 0;
    if (compact && NQ > 0) {
      q_off = (off + 15) & ~15ULL;
      off = q_off + (unsigned long long)NW * NQ * QCAP * 4;
    }
    const unsigned long long smem_total = (off + 127) & ~127ULL;
    if (smem_total > 227 * 1024) throw PlanError("scan kernel shared memory exceeds 227 KB; lower stages or items per thread");
    const unsigned wait_limit = (unsigned)std::min(60000000, std::max(1, tu.wait_limit_us));

    const std::string kname = "Scan_" + fact;
    meta << "kernel " << kname << " scan 0 " << CTA << " " << WT << " " << smem_total << " " << tu.ctas_per_sm << "\n";
    if (grouped && !smem_groups && !reg_groups && !lane_groups) meta << "touched " << TW << "\n";

    std::vector<std::string> reg_cols = fact_cols;
    for (const auto& c : payload_cols) reg_cols.push_back(c);
    for (const auto& c : gather_cols) reg_cols.push_back(c);

    loaded.clear();
    valid_regs.clear();
    tile_ptr = [](const std::string& c) { return "t_" + c; };

    std::ostringstream& o = src;
    o << "// Warp-tiled persistent scan: every warp owns a TMA staging ring and\n"
         "// walks its own sequence of " << WT << "-row tiles; the main loop has no\n"
         "// CTA-wide barrier, so independent warps hide probe latency.\n";
    o << "extern \"C\" __global__ void __launch_bounds__(" << CTA << ") " << kname << "(const CxArgs a) {\n";
    o << param_decl();
    o << "  constexpr int BLOCK_THREADS = 32, ITEMS_PER_THREAD = " << IPT << ", TILE_SIZE = " << WT << ";\n";
    o << "  constexpr int NWARP = " << NW << ", NSTAGE = " << STAGES << ", NSC = " << NSC << ";\n";
    o << "  extern __shared__ __align__(1024) unsigned char cx_smem[];\n";
    if (tu.debug_stall)
      o << "  { cx::debug_stall((unsigned long long*)cx_smem, a.err, " << wait_limit << "u); return; }\n";
    o << "  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    o << "  const int tid = lane;\n";
    o << "  int* stage_buf = (int*)cx_smem + (long long)warp * " << warp_stage_ints << "LL; (void)stage_buf;\n";
    o << "  unsigned long long* bars = (unsigned long long*)(cx_smem + " << bars_off << ") + warp * "
      << std::max(STAGES, 1) << "; (void)bars;\n";
    o << "  unsigned long long* red = (unsigned long long*)(cx_smem + " << red_off << "); (void)red;\n";
    o << "  const long long n_rows = a.rows[0];\n";
    o << "  const long long num_tiles = (n_rows + TILE_SIZE - 1) / TILE_SIZE;\n";
    o << "  const long long full_tiles = n_rows / TILE_SIZE;\n";
    o << "  const long long gwarp = (long long)blockIdx.x * NWARP + warp;\n";
    o << "  const long long nwarps = (long long)gridDim.x * NWARP;\n";
    o << "  unsigned long long* d_result = a.result; (void)d_result;\n";
    o << "  uint64_t* d_result_validity = (uint64_t*)a.result_validity; (void)d_result_validity;\n";
    declare_cols(o, fact_cols, "  ");
    declare_cols(o, gather_cols, "  ");
    for (const auto& s : p.steps) {
      if (s.kind != Step::JoinStep) continue;
      const int h = ht_slot.at(s.join.dim);
      o << "  const int* " << ht_name(s.join.dim) << " = a.ht[" << h << "];\n";
      if (s.join.multi) {
        o << "  const int* mpay_" << lower(s.join.dim) << " = a.mpay[" << h << "];\n";
        o << "  const long long mst_" << lower(s.join.dim) << " = a.rows[" << p.table_slot(s.join.dim) << "];\n";
      }
      if (!s.join.payload.empty() && payload_valid.count(s.join.payload))
        o << "  const unsigned int* " << ht_name(s.join.dim) << "_valid = a.htv[" << h << "];\n";
    }

    // Aggregate state.
    if (!grouped) {
      for (int k = 0; k < NA; ++k) {
        o << "  unsigned long long acc_" << k << " = " << (p.aggs[k].fn == AggFn::Min ? "~0ULL" : "0ULL") << ";\n";
        if (seen_idx[k] >= 0) o << "  unsigned long long seen_" << k << " = 0ULL;\n";
        if (p.aggs[k].fn == AggFn::Avg) o << "  unsigned long long cnt_" << k << " = 0ULL;\n";
      }
    } else if (lane_groups) {
      o << "  unsigned long long* s_lacc = (unsigned long long*)(cx_smem + " << lacc_off << ");\n";
      for (unsigned long long w = 0; w < G * NACC; ++w) {
        const int k = (int)(w % NACC);
        o << "  s_lacc[" << w * CTA << "ULL + threadIdx.x] = " << (k < NA && p.aggs[k].fn == AggFn::Min ? "~0ULL" : "0ULL")
          << ";\n";
      }
      o << "  unsigned rtouch = 0u;\n";
      for (int k = 0; k < NA; ++k)
        if (seen_idx[k] >= 0 && NSEEN_T > 0) o << "  unsigned rseen_" << k << " = 0u;\n";
    } else if (reg_groups) {
      o << "  unsigned long long racc[" << G * NACC << "];\n";
      o << "  #pragma unroll\n  for (int r = 0; r < " << G * NACC << "; ++r) racc[r] = 0ULL;\n";
      for (int k = 0; k < NA; ++k)
        if (p.aggs[k].fn == AggFn::Min)
          o << "  #pragma unroll\n  for (int g = 0; g < " << G << "; ++g) racc[g * " << NACC << " + " << k << "] = ~0ULL;\n";
      o << "  unsigned rtouch = 0u;\n";
      for (int k = 0; k < NA; ++k)
        if (seen_idx[k] >= 0 && NSEEN_T > 0) o << "  unsigned rseen_" << k << " = 0u;\n";
    } else if (smem_groups) {
      o << "  unsigned long long* s_acc_all = (unsigned long long*)(cx_smem + " << acc_off << ");\n";
      o << "  unsigned int* s_touch_all = (unsigned int*)(cx_smem + " << touch_off << ");\n";
      o << "  unsigned int* s_seen_all = (unsigned int*)(cx_smem + " << seen_off << "); (void)s_seen_all;\n";
      o << "  unsigned long long* s_acc = s_acc_all + " << (REP > 1 ? "(long long)warp * " + std::to_string(G * NACC) + "LL" : "0") << ";\n";
      o << "  unsigned int* s_touch = s_touch_all + " << (REP > 1 ? "(long long)warp * " + std::to_string(TW) + "LL" : "0") << ";\n";
      o << "  unsigned int* s_seen = s_seen_all + " << (REP > 1 ? "(long long)warp * " + std::to_string(NSEEN_T * TW) + "LL" : "0") << "; (void)s_seen;\n";
      std::string init = "0ULL";
      {
        std::string cond;
        for (int k = 0; k < NA; ++k)
          if (p.aggs[k].fn == AggFn::Min) cond += (cond.empty() ? "" : " || ") + std::string("s == ") + std::to_string(k);
        if (!cond.empty()) init = "(" + cond + ") ? ~0ULL : 0ULL";
      }
      o << "  for (long long w = threadIdx.x; w < " << (unsigned long long)REP * G * NACC << "LL; w += " << CTA << ") {\n";
      o << "    const int s = (int)(w % " << NACC << "); (void)s;\n";
      o << "    s_acc_all[w] = " << init << ";\n";
      o << "  }\n";
      o << "  for (long long w = threadIdx.x; w < " << (unsigned long long)REP * TW * (1 + NSEEN_T) << "LL; w += " << CTA
        << ") s_touch_all[w] = 0u;\n";
    } else {
      o << "  unsigned int* g_touch = a.touched;\n";
    }

    // Join membership bitmaps: global -> shared once per CTA.
    for (const auto& b : sbms) {
      o << "  unsigned int* s_bm_" << lower(b.dim) << " = (unsigned int*)(cx_smem + " << b.off << ");\n";
      o << "  for (long long w = threadIdx.x; w < " << b.words << "LL; w += " << CTA << ") s_bm_" << lower(b.dim)
        << "[w] = a.bm[" << b.h << "][w];\n";
    }

    // Per-warp TMA staging rings.
    if (STAGES > 0) {
      o << "  bool staged_ok = true;\n";
      for (const auto& c : fact_cols) o << "  staged_ok = staged_ok && ((((unsigned long long)d_" << c << ") & 15ULL) == 0ULL);\n";
      o << "  unsigned long long l2_policy = 0;\n";
      o << "  if (lane == 0) {\n";
      o << "    for (int s = 0; s < NSTAGE; ++s) cx::mbar_init(&bars[s], 1);\n";
      o << "    cx::fence_mbar_init();\n";
      o << "    l2_policy = cx::l2_evict_first_policy();\n";
      o << "  }\n";
      o << "#define CX_ISSUE(TILE_, STAGE_) do { \\\n";
      o << "    cx::mbar_expect_tx(&bars[(STAGE_)], " << (unsigned long long)NSC * WT * 4 << "u); \\\n";
      for (int c = 0; c < NSC; ++c)
        o << "    cx::bulk_g2s(stage_buf + ((STAGE_) * NSC + " << c << ") * TILE_SIZE, d_" << fact_cols[c]
          << " + (TILE_) * TILE_SIZE, " << WT * 4 << "u, &bars[(STAGE_)], l2_policy); \\\n";
      o << "  } while (0)\n";
    }
    o << "  __syncthreads();\n";
    if (STAGES > 0) {
      o << "  if (lane == 0 && staged_ok) {\n";
      o << "    for (int k = 0; k < NSTAGE; ++k) {\n";
      o << "      const long long t = gwarp + (long long)k * nwarps;\n";
      o << "      if (t < full_tiles) CX_ISSUE(t, k);\n";
      o << "    }\n";
      o << "  }\n";
    }

    // Unstaged scans: every fact column of a full warp tile is read with
    // vector loads (vector-striped rows) one tile ahead, so the next tile's
    // loads are in flight while this one probes and aggregates.
    const bool vec_pf = STAGES == 0 && NSC > 0 && (IPT == 1 || IPT == 2 || IPT % 4 == 0) && tu.prefetch > 0;
    const bool ahead = vec_pf && tu.prefetch == 2;
    const bool l2_ahead = vec_pf && tu.prefetch == 3;
    if (vec_pf) {
      o << "  bool vec_ok = true;\n";
      for (const auto& c : fact_cols) o << "  vec_ok = vec_ok && ((((unsigned long long)d_" << c << ") & 15ULL) == 0ULL);\n";
    }
    if (ahead) {
      for (const auto& c : fact_cols) o << "  int pf_" << c << "[ITEMS_PER_THREAD];\n";
      o << "  if (vec_ok && gwarp < full_tiles) {\n";
      for (const auto& c : fact_cols)
        o << "    WarpLoadTileV<ITEMS_PER_THREAD>(d_" << c << " + gwarp * TILE_SIZE, lane, pf_" << c << ");\n";
      o << "  }\n";
    }
    o << "  long long k_iter = 0;\n";
    o << "  bool aborted = false; (void)aborted;\n";
    if (compact) {
      o << "  int* q_base = (int*)(cx_smem + " << q_off << ") + (long long)warp * " << NQ * QCAP << "LL; (void)q_base;\n";
      o << "  int q_n = 0;  // rows waiting in this warp's queue (warp-uniform)\n";
      o << "  for (long long t = gwarp; ; t += nwarps, ++k_iter) {\n";
      o << "   const bool live_ = t < num_tiles;\n";
      o << "   if (live_) {\n";
    } else {
      o << "  for (long long t = gwarp; t < num_tiles; t += nwarps, ++k_iter) {\n";
    }
    o << "    const long long tile_offset = t * TILE_SIZE;\n";
    o << "    const int num_tile_items = (int)(n_rows - tile_offset < TILE_SIZE ? n_rows - tile_offset : TILE_SIZE);\n";
    if (STAGES > 0) {
      o << "    const int stage = (int)(k_iter % NSTAGE);\n";
      o << "    const bool staged = staged_ok && t < full_tiles;\n";
      o << "    bool timed_out = false;\n";
      o << "    if (staged) timed_out = !cx::mbar_wait_bounded(&bars[stage], (unsigned)((k_iter / NSTAGE) & 1), " << wait_limit << "u);\n";
      o << "    if (__any_sync(0xffffffffu, timed_out)) { if (lane == 0) cx::raise(a.err, cx::ERR_WAIT_TIMEOUT); aborted = true; break; }\n";
      for (int c = 0; c < NSC; ++c)
        o << "    const int* t_" << fact_cols[c] << " = staged ? stage_buf + (stage * NSC + " << c << ") * TILE_SIZE : d_"
          << fact_cols[c] << " + tile_offset;\n";
    } else {
      for (int c = 0; c < NSC; ++c)
        o << "    const int* t_" << fact_cols[c] << " = d_" << fact_cols[c] << " + tile_offset;\n";
    }
    o << "    int flags[ITEMS_PER_THREAD];\n";
    declare_regs(o, reg_cols, "    ");
    o << "    InitFlags<BLOCK_THREADS, ITEMS_PER_THREAD>(flags);\n";
    if (vec_pf) {
      o << "    if (vec_ok && t < full_tiles) {\n";
      if (l2_ahead) {
        // The warp's next tile into L2 while this one is processed: its loads
        // then wait on L2, not DRAM (no registers held for it).
        o << "      if (lane == 0 && t + nwarps < full_tiles) {\n";
        for (const auto& c : fact_cols)
          o << "        cx::l2_prefetch_bulk(d_" << c << " + (t + nwarps) * TILE_SIZE, TILE_SIZE * 4u);\n";
        o << "      }\n";
      }
      if (ahead) {
        o << "      #pragma unroll\n      for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
        for (const auto& c : fact_cols) o << "        " << c << "[i] = pf_" << c << "[i];\n";
        o << "      }\n";
        o << "      if (t + nwarps < full_tiles) {\n";
        for (const auto& c : fact_cols)
          o << "        WarpLoadTileV<ITEMS_PER_THREAD>(d_" << c << " + (t + nwarps) * TILE_SIZE, lane, pf_" << c << ");\n";
        o << "      }\n";
      } else {
        for (const auto& c : fact_cols)
          o << "      WarpLoadTileV<ITEMS_PER_THREAD>(d_" << c << " + tile_offset, lane, " << c << ");\n";
      }
      for (const auto& c : fact_cols)
        if (nullable(c)) o << "      WarpLoadValidityV<ITEMS_PER_THREAD>(n_" << c << ", lane, tile_offset, " << c << "_valid);\n";
      o << "    } else {\n";
      for (const auto& c : fact_cols) {
        o << "      BlockLoad<int, BLOCK_THREADS, ITEMS_PER_THREAD>(t_" << c << ", tid, tile_offset, " << c << ", num_tile_items);\n";
        if (nullable(c))
          o << "      BlockLoadValidity<BLOCK_THREADS, ITEMS_PER_THREAD>(n_" << c << ", tid, tile_offset, " << c
            << "_valid, num_tile_items);\n";
      }
      o << "    }\n";
      for (const auto& c : fact_cols) {
        loaded.insert(c);
        if (nullable(c)) valid_regs.insert(c);
      }
    }

    // Pipeline body: the reference's primitive calls, one warp tile at a time.
    const std::string ind = "    ";
    // Membership of every join with a shared-memory exact bitmap first: those
    // joins need no table access at all for in-window keys, and the payload
    // loads and L2 probes below only run for rows that qualify on all of them.
    std::set<std::string> exact_dims;
    for (const auto& b : sbms) {
      ensure_loaded(o, b.fk, ind);
      if (valid_regs.count(b.fk))
        o << ind << "BlockApplyValidityAnd<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, flags, " << b.fk << "_valid, num_tile_items);\n";
      if (b.table)
        o << ind << "BlockProbeExactTable<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << b.fk
          << ", flags, (const unsigned char*)s_bm_" << lower(b.dim) << ", " << ht_name(b.dim) << ", " << b.len << ", "
          << b.keymin << ", num_tile_items);\n";
      else
        o << ind << "BlockProbeExactBitmap<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << b.fk << ", flags, s_bm_"
          << lower(b.dim) << ", " << ht_name(b.dim) << ", " << (b.pair ? 1 : 0) << ", " << b.len << ", " << b.keymin
          << ", num_tile_items);\n";
      exact_dims.insert(b.dim);
    }
    // The steps after the membership tests, in plan order (with compaction:
    // the ones that run on queued rows).
    auto emit_steps = [&](std::ostream& o, const std::string& ind, bool post) {
    for (size_t k = 0; k < xs; ++k) {
      const Step& s = p.steps[k];
      if (s.kind == Step::Filter) {
        const bool early = fact_only(s.filter.get());
        if (!compact || early != post) emit_filter(o, s.filter.get(), ind);
        continue;
      }
      if (compact && !post) continue;
      const Join& j = s.join;
      const std::string& fk = j.fks[0];
      if (exact_dims.count(j.dim) && j.payload.empty()) continue;
      ensure_loaded(o, fk, ind);
      if (exact_dims.count(j.dim)) {
        // Membership is settled; fetch the payload of qualifying rows.
        if (j.payload.empty()) continue;
        if (payload_valid.count(j.payload)) {
          o << ind << "BlockFetchPayloadPHT_2V<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", " << j.payload
            << ", " << j.payload << "_valid, flags, " << ht_name(j.dim) << ", " << ht_name(j.dim) << "_valid, " << j.len
            << ", " << j.keymin << ", num_tile_items);\n";
          valid_regs.insert(j.payload);
        } else if (ptable.count(j.dim)) {
          o << ind << "BlockFetchPayloadTable<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", " << j.payload
            << ", flags, (const unsigned char*)s_bm_" << lower(j.dim) << ", " << ht_name(j.dim) << ", " << j.len << ", "
            << j.keymin << ", (int)(" << j.prange_min << "LL), num_tile_items);\n";
        } else {
          o << ind << "BlockFetchPayloadPHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", " << j.payload
            << ", flags, " << ht_name(j.dim) << ", " << j.len << ", " << j.keymin << ", num_tile_items);\n";
        }
        loaded.insert(j.payload);
        continue;
      }
      if (valid_regs.count(fk))
        o << ind << "BlockApplyValidityAnd<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, flags, " << fk << "_valid, num_tile_items);\n";
      if (j.payload.empty()) {
        o << ind << "BlockProbeAndPHT_1<int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", flags, " << ht_name(j.dim)
          << ", " << j.len << ", " << j.keymin << ", num_tile_items);\n";
      } else if (payload_valid.count(j.payload)) {
        o << ind << "BlockProbeAndPHT_2V<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", " << j.payload
          << ", " << j.payload << "_valid, flags, " << ht_name(j.dim) << ", " << ht_name(j.dim) << "_valid, " << j.len
          << ", " << j.keymin << ", num_tile_items);\n";
        loaded.insert(j.payload);
        valid_regs.insert(j.payload);
      } else {
        o << ind << "BlockProbeAndPHT_2<int, int, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, " << fk << ", " << j.payload
          << ", flags, " << ht_name(j.dim) << ", " << j.len << ", " << j.keymin << ", num_tile_items);\n";
        loaded.insert(j.payload);
      }
    }
    };
    emit_steps(o, ind, false);
    // Per-row aggregate updates shared by the vector and the item-mode paths.
    // Ungrouped: thread-private accumulators.
    auto scalar_update = [&](const std::string& ii) {
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const std::string v = ag.arg->op == Op::Star ? "1" : valid_of(ag.arg.get());
        const std::string x = ag.fn == AggFn::Count ? "1ULL" : math_push(ag.arg.get(), true);
        switch (ag.fn) {
          case AggFn::Count: o << ii << "if (" << v << ") acc_" << k << " += 1ULL;\n"; break;
          case AggFn::Sum: o << ii << "if (" << v << ") { acc_" << k << " += " << x << "; seen_" << k << " += 1ULL; }\n"; break;
          case AggFn::Avg: o << ii << "if (" << v << ") { acc_" << k << " += " << x << "; cnt_" << k << " += 1ULL; }\n"; break;
          case AggFn::Min:
            o << ii << "if (" << v << ") { const unsigned long long x_ = " << x << "; if (x_ < acc_" << k << ") acc_" << k
              << " = x_; seen_" << k << " += 1ULL; }\n";
            break;
          case AggFn::Max:
            o << ii << "if (" << v << ") { const unsigned long long x_ = " << x << "; if (x_ > acc_" << k << ") acc_" << k
              << " = x_; seen_" << k << " += 1ULL; }\n";
            break;
        }
      }
    };
    // Grouped: the perfect-hash group of the row in `hash`.
    auto group_hash = [&](const std::string& ii) {
      std::string horner, dom;
      for (size_t k = 0; k < p.groups.size(); ++k) {
        o << ii << "const int gt" << k << " = " << group_term(k) << ";\n";
        horner = horner.empty() ? "gt0" : "(" + horner + " * " + std::to_string(eff_card(k)) + " + gt" + std::to_string(k) + ")";
        dom += (dom.empty() ? "" : " && ") + std::string("(unsigned)gt") + std::to_string(k) + " < " +
               std::to_string(eff_card(k)) + "u";
      }
      // Keys inside their domains give a Horner value below G, where the
      // reference's `% G` is the identity; only an out-of-domain key pays for it.
      o << ii << "int hash = " << horner << ";\n";
      o << ii << "if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
    };
    // Tiny group domains: register accumulators selected by a compare chain.
    auto reg_update = [&](const std::string& ii) {
      o << ii << "rtouch |= 1u << hash;\n";
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const std::string v = ag.arg->op == Op::Star ? "1" : valid_of(ag.arg.get());
        const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + math_push(ag.arg.get(), true) + ")";
        o << ii << "if (" << v << ") {\n";
        o << ii << "  const unsigned long long x_ = " << x << ";\n";
        o << ii << "  #pragma unroll\n" << ii << "  for (int g = 0; g < " << G << "; ++g) if (hash == g) {\n";
        const std::string r = "racc[g * " + std::to_string(NACC) + " + " + std::to_string(k) + "]";
        if (ag.fn == AggFn::Min) o << ii << "    if (x_ < " << r << ") " << r << " = x_;\n";
        else if (ag.fn == AggFn::Max) o << ii << "    if (x_ > " << r << ") " << r << " = x_;\n";
        else o << ii << "    " << r << " += x_;\n";
        if (ag.fn == AggFn::Avg) o << ii << "    racc[g * " << NACC << " + " << avg_idx[k] << "] += 1ULL;\n";
        o << ii << "  }\n";
        if (seen_idx[k] >= 0 && NSEEN_T > 0) o << ii << "  rseen_" << k << " |= 1u << hash;\n";
        o << ii << "}\n";
      }
    };
    auto lane_update = [&](const std::string& ii) {
      o << ii << "rtouch |= 1u << hash;\n";
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const std::string v = ag.arg->op == Op::Star ? "1" : valid_of(ag.arg.get());
        const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + math_push(ag.arg.get(), true) + ")";
        const std::string r = "s_lacc[((unsigned)hash * " + std::to_string(NACC) + "u + " + std::to_string(k) + "u) * " +
                              std::to_string(CTA) + "u + threadIdx.x]";
        o << ii << "if (" << v << ") {\n";
        o << ii << "  const unsigned long long x_ = " << x << ";\n";
        if (ag.fn == AggFn::Min) o << ii << "  if (x_ < " << r << ") " << r << " = x_;\n";
        else if (ag.fn == AggFn::Max) o << ii << "  if (x_ > " << r << ") " << r << " = x_;\n";
        else o << ii << "  " << r << " += x_;\n";
        if (ag.fn == AggFn::Avg)
          o << ii << "  s_lacc[((unsigned)hash * " << NACC << "u + " << avg_idx[k] << "u) * " << CTA << "u + threadIdx.x] += 1ULL;\n";
        if (seen_idx[k] >= 0 && NSEEN_T > 0) o << ii << "  rseen_" << k << " |= 1u << hash;\n";
        o << ii << "}\n";
      }
    };
    // Item mode, larger domains: one atomic update per row into the shared or
    // global group table (no warp merging: lanes run different expansions).
    auto atomic_update = [&](const std::string& ii) {
      const std::string bit = "(1u << (hash & 31))";
      if (smem_groups) o << ii << "atomicOr(&s_touch[hash >> 5], " << bit << ");\n";
      else if (count_star_slot() < 0) o << ii << "atomicOr(&g_touch[hash >> 5], " << bit << ");\n";
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const int slot = (int)p.groups.size() + k;
        const std::string v = ag.arg->op == Op::Star ? "1" : valid_of(ag.arg.get());
        const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + math_push(ag.arg.get(), true) + ")";
        const std::string row = "(unsigned long long)hash * " + std::to_string(TS) + "ULL";
        const std::string acc = smem_groups ? "s_acc[(long long)hash * " + std::to_string(NACC) + " + " + std::to_string(k) + "]"
                                            : "d_result[" + row + " + " + std::to_string(slot) + "]";
        o << ii << "if (" << v << ") {\n";
        o << ii << "  const unsigned long long x_ = " << x << ";\n";
        if (ag.fn == AggFn::Min) o << ii << "  atomicMin(&" << acc << ", x_);\n";
        else if (ag.fn == AggFn::Max) o << ii << "  atomicMax(&" << acc << ", x_);\n";
        else o << ii << "  atomicAdd(&" << acc << ", x_);\n";
        if (seen_idx[k] >= 0 && NSEEN_T > 0) {
          if (smem_groups)
            o << ii << "  atomicOr(&s_seen[" << (unsigned long long)seen_idx[k] * TW << "ULL + (hash >> 5)], " << bit << ");\n";
          else
            o << ii << "  db::atomic_set_valid_bit(d_result_validity, " << row << " + " << slot << ");\n";
        }
        if (ag.fn == AggFn::Avg) {
          if (smem_groups) o << ii << "  atomicAdd(&s_acc[(long long)hash * " << NACC << " + " << avg_idx[k] << "], 1ULL);\n";
          else o << ii << "  atomicAdd(&d_result[" << row << " + " << p.hidden_count_slot(k) << "], 1ULL);\n";
        }
        o << ii << "}\n";
        if (ag.fn == AggFn::Count && !p.sparse && !smem_groups)
          o << ii << "db::atomic_set_valid_bit(d_result_validity, " << row << " + " << slot << ");\n";
      }
    };
    auto item_consume = [&](const std::string& ii) {
      if (!grouped) return scalar_update(ii);
      o << ii << "{\n";
      group_hash(ii + "  ");
      o << ii << "  if ((unsigned)hash < " << G << "u) {\n";
      if (reg_groups) reg_update(ii + "    ");
      else if (lane_groups) lane_update(ii + "    ");
      else atomic_update(ii + "    ");
      o << ii << "  }\n" << ii << "}\n";
    };
    // Steps from k on for item i (consumeHashJoinVector's OR-join branches and
    // MHT expansion loop, visitor.cpp:4587-4730; later joins probe in item
    // mode like consumeHashJoinItem).  A fact key equal to an earlier valid key
    // of the same row is skipped, so one dimension row is never counted twice.
    std::function<void(size_t, const std::string&)> item_steps = [&](size_t k, const std::string& ii) {
      if (k == p.steps.size()) return item_consume(ii);
      const Step& s = p.steps[k];
      if (s.kind == Step::Filter) {
        o << ii << "if (" << and_terms({valid_of(s.filter.get()), value_of(s.filter.get())}) << ") {\n";
        item_steps(k + 1, ii + "  ");
        o << ii << "}\n";
        return;
      }
      const Join& j = s.join;
      const std::string K = std::to_string(k), ht = ht_name(j.dim);
      for (size_t f = 0; f < j.fks.size(); ++f) {
        const std::string& fk = j.fks[f];
        std::vector<std::string> terms{valid_regs.count(fk) ? fk + "_valid[i]" : "1"};
        for (size_t q = 0; q < f; ++q) {
          const std::string& pf = j.fks[q];
          const std::string pv = valid_regs.count(pf) ? pf + "_valid[i]" : "1";
          terms.push_back(lit_true(pv) ? fk + "[i] != " + pf + "[i]" : "(!(" + pv + ") || " + fk + "[i] != " + pf + "[i])");
        }
        o << ii << "if (" << and_terms(terms) << ") {\n";
        const std::string i2 = ii + "  ";
        if (j.multi) {
          const std::string off = "off" + K, cnt = "cnt" + K, fl = "fl" + K, jj = "j" + K, rid = "rid" + K;
          o << i2 << "int " << off << " = 0, " << cnt << " = 0, " << fl << " = 1;\n";
          o << i2 << "ProbeMultiHT<int>(" << fk << "[i], " << off << ", " << cnt << ", " << fl << ", " << ht << ", " << j.len
            << ", " << j.keymin << ");\n";
          o << i2 << "for (int " << jj << " = 0; " << jj << " < " << cnt << "; ++" << jj << ") {\n";
          (void)rid;
          emit_mht_gathers(o, j, "(long long)" + off + " + " + jj, i2 + "  ");
          item_steps(k + 1, i2 + "  ");
          o << i2 << "}\n";
        } else {
          const std::string hs = "h" + K + "_" + std::to_string(f);
          o << i2 << "const int " << hs << " = cx_detail::pht_slot<int>(" << fk << "[i], " << j.len << ", " << j.keymin << ");\n";
          if (j.payload.empty()) {
            o << i2 << "if (" << hs << " >= 0 && " << ht << "[" << hs << "] == " << fk << "[i]) {\n";
          } else {
            o << i2 << "if (" << hs << " >= 0 && " << ht << "[2LL * " << hs << "] == " << fk << "[i]) {\n";
            o << i2 << "  " << j.payload << "[i] = " << ht << "[2LL * " << hs << " + 1];\n";
            if (payload_valid.count(j.payload))
              o << i2 << "  " << j.payload << "_valid[i] = (int)((" << ht << "_valid[" << hs << " >> 5] >> (" << hs
                << " & 31)) & 1u);\n";
          }
          item_steps(k + 1, i2 + "  ");
          o << i2 << "}\n";
        }
        o << ii << "}\n";
      }
    };

    // Group update of one item under the flag `act_init`: lanes with the same
    // group merge their values (one match) and the lowest applies them -- or,
    // with per-warp tables and direct merging, every active lane applies its
    // own.  All lanes of the warp execute it (it ballots).
    auto merged_update = [&](const std::string& ind, const std::string& act_init) {
      o << ind << "{\n";
      o << ind << "  bool act = " << act_init << ";\n";
      o << ind << "  int hash = 0;\n";
      o << ind << "  if (act) {\n";
      std::string horner, dom;
      for (size_t k = 0; k < p.groups.size(); ++k) {
        o << ind << "    const int gt" << k << " = " << group_term(k) << ";\n";
        horner = horner.empty() ? "gt0" : "(" + horner + " * " + std::to_string(eff_card(k)) + " + gt" + std::to_string(k) + ")";
        dom += (dom.empty() ? "" : " && ") + std::string("(unsigned)gt") + std::to_string(k) + " < " +
               std::to_string(eff_card(k)) + "u";
      }
      o << ind << "    hash = " << horner << ";\n";
      o << ind << "    if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
      o << ind << "    if ((unsigned)hash >= " << G << "u) act = false;\n";
      o << ind << "  }\n";
      // Warp-uniform skip when no lane of the warp aggregates this item; else
      // lanes with the same group merge their updates (one match per item) and
      // the lowest lane applies them -- or, with per-warp tables and direct
      // merging, every active lane applies its own update.
      const bool direct = tu.group_merge == 2 || (tu.group_merge == 0 && smem_groups && REP > 1);
      o << ind << "  const unsigned amask = __ballot_sync(0xffffffffu, act);\n";
      o << ind << "  if (amask != 0u) {\n";
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const std::string v = ag.arg->op == Op::Star ? "1" : valid_of(ag.arg.get());
        const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + math_push(ag.arg.get(), true) + ")";
        o << ind << "  bool v" << k << " = act && (" << v << ");\n";
        o << ind << "  unsigned long long x" << k << " = v" << k << " ? " << x << " : "
          << (ag.fn == AggFn::Min ? "~0ULL" : "0ULL") << ";\n";
      }
      o << ind << "  if (act) {\n";
      if (direct) o << ind << "    const unsigned peers = 1u << lane;\n";
      else o << ind << "    const unsigned peers = __popc(amask) == 1 ? amask : __match_any_sync(amask, (unsigned)hash);\n";
      o << ind << "    const int leader = __ffs(peers) - 1;\n";
      o << ind << "    if (__popc(peers) > 1) {\n";
      for (int k = 0; k < NA; ++k) {
        const AggFn f = p.aggs[k].fn;
        o << ind << "      { unsigned long long r_ = 0" << (f == AggFn::Min ? "xffffffffffffffffULL" : "ULL") << ";\n";
        o << ind << "        for (unsigned m = peers; m; m &= m - 1) {\n";
        o << ind << "          const unsigned long long y_ = __shfl_sync(peers, x" << k << ", __ffs(m) - 1);\n";
        if (f == AggFn::Min) o << ind << "          r_ = y_ < r_ ? y_ : r_;\n";
        else if (f == AggFn::Max) o << ind << "          r_ = y_ > r_ ? y_ : r_;\n";
        else o << ind << "          r_ += y_;\n";
        o << ind << "        }\n";
        o << ind << "        x" << k << " = r_; }\n";
        if (f == AggFn::Avg || (seen_idx[k] >= 0 && NSEEN_T > 0))
          o << ind << "      v" << k << " = __ballot_sync(peers, v" << k << ") != 0u;\n";
      }
      o << ind << "    }\n";
      o << ind << "    if (lane == leader) {\n";
      const std::string bit = "(1u << (hash & 31))";
      if (smem_groups) o << ind << "      atomicOr(&s_touch[hash >> 5], " << bit << ");\n";
      else if (count_star_slot() < 0) o << ind << "      atomicOr(&g_touch[hash >> 5], " << bit << ");\n";
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const int slot = (int)p.groups.size() + k;
        const std::string acc = smem_groups ? "s_acc[(long long)hash * " + std::to_string(NACC) + " + " + std::to_string(k) + "]"
                                            : "d_result[(unsigned long long)hash * " + std::to_string(TS) + "ULL + " +
                                                  std::to_string(slot) + "]";
        if (ag.fn == AggFn::Min) o << ind << "      if (v" << k << ") atomicMin(&" << acc << ", x" << k << ");\n";
        else if (ag.fn == AggFn::Max) o << ind << "      if (v" << k << ") atomicMax(&" << acc << ", x" << k << ");\n";
        else o << ind << "      if (x" << k << ") atomicAdd(&" << acc << ", x" << k << ");\n";
        if (seen_idx[k] >= 0 && NSEEN_T > 0) {
          if (smem_groups)
            o << ind << "      if (v" << k << ") atomicOr(&s_seen[" << (unsigned long long)seen_idx[k] * TW << "ULL + (hash >> 5)], " << bit << ");\n";
          else
            o << ind << "      if (v" << k << ") db::atomic_set_valid_bit(d_result_validity, (unsigned long long)hash * " << TS << "ULL + " << slot << ");\n";
        }
        if (ag.fn == AggFn::Count && !p.sparse && !smem_groups)
          o << ind << "      db::atomic_set_valid_bit(d_result_validity, (unsigned long long)hash * " << TS << "ULL + " << slot << ");\n";
      }
      o << ind << "    }\n";
      for (int k = 0; k < NA; ++k) {
        if (p.aggs[k].fn != AggFn::Avg) continue;
        const std::string cacc = smem_groups ? "s_acc[(long long)hash * " + std::to_string(NACC) + " + " + std::to_string(avg_idx[k]) + "]"
                                             : "d_result[(unsigned long long)hash * " + std::to_string(TS) + "ULL + " +
                                                   std::to_string(p.hidden_count_slot(k)) + "]";
        o << ind << "    { const unsigned c_ = __popc(__ballot_sync(peers, act && (" << (p.aggs[k].arg->op == Op::Star ? std::string("1") : valid_of(p.aggs[k].arg.get())) << ")));\n";
        o << ind << "      if (lane == leader && c_) atomicAdd(&" << cacc << ", (unsigned long long)c_); }\n";
      }
      o << ind << "  }\n";
      o << ind << "  }\n";
      o << ind << "}\n";
    };
    if (expanding) {
      // Columns the expansion publishes are written inside the item loop;
      // every fact column the rest of the pipeline reads is loaded once here.
      for (size_t k = xs; k < p.steps.size(); ++k) {
        const Step& s = p.steps[k];
        if (s.kind != Step::JoinStep) continue;
        for (const auto& c : s.join.gathers) {
          loaded.insert(c);
          if (nullable(c)) valid_regs.insert(c);
        }
        if (!s.join.payload.empty()) {
          loaded.insert(s.join.payload);
          if (payload_valid.count(s.join.payload)) valid_regs.insert(s.join.payload);
        }
      }
      for (size_t k = xs; k < p.steps.size(); ++k) {
        const Step& s = p.steps[k];
        if (s.kind == Step::Filter) load_expr_cols(o, s.filter.get(), ind);
        else for (const auto& fk : s.join.fks) ensure_loaded(o, fk, ind);
      }
    }
    if (!compact) {
      for (const auto& g : p.groups) load_expr_cols(o, g.expr.get(), ind);
      for (const auto& ag : p.aggs) load_expr_cols(o, ag.arg.get(), ind);
    }

    // With group_merge = 1, one expanding join feeding a shared-memory or
    // global group table runs as a warp-uniform loop (every lane takes its
    // next match each round): the later steps become a per-lane predicate and
    // equal groups merge across the warp before the atomics, as in the vector
    // path.  Otherwise (the default; measured no slower) every expanded row
    // updates on its own (item_steps).
    int n_expanding = 0;
    for (const auto& s : p.steps)
      if (s.kind == Step::JoinStep && s.join.expands()) ++n_expanding;
    const bool uniform_expand =
        expanding && n_expanding == 1 && grouped && !reg_groups && !lane_groups && tu.group_merge == 1;
    auto uniform_tail = [&](const std::string& ii) {
      for (size_t k = xs + 1; k < p.steps.size(); ++k) {
        const Step& s = p.steps[k];
        if (s.kind == Step::Filter) {
          o << ii << "act_ = act_ && (" << and_terms({valid_of(s.filter.get()), value_of(s.filter.get())}) << ");\n";
          continue;
        }
        const Join& j = s.join;
        const std::string& fk = j.fks[0];
        const std::string ht = ht_name(j.dim), hs = "h" + std::to_string(k) + "_";
        const std::string fkv = valid_regs.count(fk) ? fk + "_valid[i]" : "1";
        o << ii << "if (act_) {\n";
        o << ii << "  const int " << hs << " = cx_detail::pht_slot<int>(" << fk << "[i], " << j.len << ", " << j.keymin << ");\n";
        if (j.payload.empty()) {
          o << ii << "  if (!((" << fkv << ") && " << hs << " >= 0 && " << ht << "[" << hs << "] == " << fk << "[i])) act_ = false;\n";
        } else {
          o << ii << "  if ((" << fkv << ") && " << hs << " >= 0 && " << ht << "[2LL * " << hs << "] == " << fk << "[i]) {\n";
          o << ii << "    " << j.payload << "[i] = " << ht << "[2LL * " << hs << " + 1];\n";
          if (payload_valid.count(j.payload))
            o << ii << "    " << j.payload << "_valid[i] = (int)((" << ht << "_valid[" << hs << " >> 5] >> (" << hs << " & 31)) & 1u);\n";
          o << ii << "  } else {\n" << ii << "    act_ = false;\n" << ii << "  }\n";
        }
        o << ii << "}\n";
      }
      merged_update(ii, "act_");
    };
    auto uniform_expansion = [&](const std::string& ii) {
      const Join& j = p.steps[xs].join;
      const std::string ht = ht_name(j.dim);
      o << ii << "#pragma unroll\n" << ii << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
      o << ii << "  const bool base_ = flags[i] && (tid + BLOCK_THREADS * i < num_tile_items);\n";
      for (size_t f = 0; f < j.fks.size(); ++f) {
        const std::string& fk = j.fks[f];
        std::vector<std::string> terms{"base_", valid_regs.count(fk) ? fk + "_valid[i]" : "1"};
        for (size_t q = 0; q < f; ++q) {
          const std::string& pf = j.fks[q];
          const std::string pv = valid_regs.count(pf) ? pf + "_valid[i]" : "1";
          terms.push_back(lit_true(pv) ? fk + "[i] != " + pf + "[i]" : "(!(" + pv + ") || " + fk + "[i] != " + pf + "[i])");
        }
        const std::string i2 = ii + "  ";
        o << i2 << "{\n";
        o << i2 << "  const bool br_ = " << and_terms(terms) << ";\n";
        if (j.multi) {
          o << i2 << "  int off_ = 0, cnt_ = 0;\n";
          o << i2 << "  if (br_) { int fl_ = 1; ProbeMultiHT<int>(" << fk << "[i], off_, cnt_, fl_, " << ht << ", " << j.len << ", "
            << j.keymin << "); }\n";
          o << i2 << "  for (int j_ = 0; __any_sync(0xffffffffu, j_ < cnt_); ++j_) {\n";
          o << i2 << "    bool act_ = j_ < cnt_;\n";
          o << i2 << "    if (act_) {\n";
          emit_mht_gathers(o, j, "(long long)off_ + j_", i2 + "      ");
          o << i2 << "    }\n";
          uniform_tail(i2 + "    ");
          o << i2 << "  }\n";
        } else {
          o << i2 << "  bool act_ = br_;\n";
          o << i2 << "  if (act_) {\n";
          o << i2 << "    const int hx_ = cx_detail::pht_slot<int>(" << fk << "[i], " << j.len << ", " << j.keymin << ");\n";
          if (j.payload.empty()) {
            o << i2 << "    if (!(hx_ >= 0 && " << ht << "[hx_] == " << fk << "[i])) act_ = false;\n";
          } else {
            o << i2 << "    if (hx_ >= 0 && " << ht << "[2LL * hx_] == " << fk << "[i]) {\n";
            o << i2 << "      " << j.payload << "[i] = " << ht << "[2LL * hx_ + 1];\n";
            if (payload_valid.count(j.payload))
              o << i2 << "      " << j.payload << "_valid[i] = (int)((" << ht << "_valid[hx_ >> 5] >> (hx_ & 31)) & 1u);\n";
            o << i2 << "    } else {\n" << i2 << "      act_ = false;\n" << i2 << "    }\n";
          }
          o << i2 << "  }\n";
          uniform_tail(i2 + "  ");
        }
        o << i2 << "}\n";
      }
      o << ii << "}\n";
    };

    // Aggregate consume.
    auto emit_consume = [&](const std::string& ind) {
      if (uniform_expand) {
        uniform_expansion(ind);
      } else if (expanding) {
        o << ind << "#pragma unroll\n" << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
        o << ind << "  if (flags[i] && (tid + BLOCK_THREADS * i < num_tile_items)) {\n";
        item_steps(xs, ind + "    ");
        o << ind << "  }\n" << ind << "}\n";
      } else if (!grouped) {
        o << ind << "#pragma unroll\n" << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
        o << ind << "  if (flags[i] && (tid + BLOCK_THREADS * i < num_tile_items)) {\n";
        scalar_update(ind + "    ");
        o << ind << "  }\n" << ind << "}\n";
      } else if (reg_groups || lane_groups) {
        o << ind << "#pragma unroll\n" << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
        o << ind << "  if (flags[i] && (tid + BLOCK_THREADS * i < num_tile_items)) {\n";
        group_hash(ind + "    ");
        o << ind << "    if ((unsigned)hash < " << G << "u) {\n";
        if (reg_groups) reg_update(ind + "      ");
        else lane_update(ind + "      ");
        o << ind << "    }\n";
        o << ind << "  }\n";
        o << ind << "}\n";
      } else {
        o << ind << "#pragma unroll\n" << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
        merged_update(ind + "  ", "flags[i] && (tid + BLOCK_THREADS * i < num_tile_items)");
        o << ind << "}\n";
      }

    };
    if (!compact) {
      emit_consume(ind);
    } else {
      // Append this tile's qualifying rows to the warp's queue.
      o << ind << "#pragma unroll\n" << ind << "for (int i = 0; i < ITEMS_PER_THREAD; ++i) {\n";
      o << ind << "  const bool f_ = flags[i] && (tid + BLOCK_THREADS * i < num_tile_items);\n";
      o << ind << "  const unsigned m_ = __ballot_sync(0xffffffffu, f_);\n";
      // Every lane computes its slot (at most q_n + 31, inside the queue);
      // only qualifying lanes store, by predicated stores without a branch.
      o << ind << "  const int p_ = q_n + __popc(m_ & ((1u << lane) - 1u));\n";
      {
        int qi = 0;
        for (const auto& c : qcols) {
          o << ind << "  cx::st_shared_if(f_, &q_base[" << qi++ * QCAP << " + p_], " << c << "[i]);\n";
          if (nullable(c)) o << ind << "  cx::st_shared_if(f_, &q_base[" << qi++ * QCAP << " + p_], " << c << "_valid[i]);\n";
        }
      }
      o << ind << "  q_n += __popc(m_);\n";
      o << ind << "}\n";
      o << "   }\n";  // live_
      // Run the rest of the pipeline on 32 queued rows at a time (the last,
      // partial batch once the warp has no tiles left).
      o << "   while (q_n >= " << 32 * DB << " || (!live_ && q_n > 0)) {\n";
      o << "    const int cnt_ = q_n < " << 32 * DB << " ? q_n : " << 32 * DB << ";\n";
      o << "    __syncwarp();\n";
      o << "    {\n";
      o << "    constexpr int ITEMS_PER_THREAD = " << DB << ";\n";
      o << "    const int num_tile_items = cnt_;\n";
      o << "    int flags[" << DB << "];\n";
      for (int j = 0; j < DB; ++j) o << "    flags[" << j << "] = lane + " << 32 * j << " < cnt_ ? 1 : 0;\n";
      std::vector<std::string> dregs = qcols;
      for (const auto& c : payload_cols) dregs.push_back(c);
      declare_regs(o, dregs, "    ");
      const std::set<std::string> saved_loaded = loaded, saved_valid = valid_regs;
      loaded.clear();
      valid_regs.clear();
      {
        int qi = 0;
        for (const auto& c : qcols) {
          for (int j = 0; j < DB; ++j) o << "    " << c << "[" << j << "] = q_base[" << qi * QCAP + 32 * j << " + lane];\n";
          ++qi;
          loaded.insert(c);
          if (nullable(c)) {
            for (int j = 0; j < DB; ++j) o << "    " << c << "_valid[" << j << "] = q_base[" << qi * QCAP + 32 * j << " + lane];\n";
            ++qi;
            valid_regs.insert(c);
          }
        }
      }
      emit_steps(o, "    ", true);
      emit_consume("    ");
      loaded = saved_loaded;
      valid_regs = saved_valid;
      o << "    }\n";
      o << "    __syncwarp();\n";
      // Move the rows left over to the queue's front.
      o << "    const int rest_ = q_n - cnt_;\n";
      o << "    for (int b_ = 0; b_ < rest_; b_ += 32) {\n";
      o << "      const int e_ = b_ + lane;\n";
      o << "      int v_[" << std::max(NQ, 1) << "];\n";
      o << "      if (e_ < rest_) {\n";
      for (int qi = 0; qi < NQ; ++qi) o << "        v_[" << qi << "] = q_base[" << qi * QCAP << " + cnt_ + e_];\n";
      o << "      }\n";
      o << "      __syncwarp();\n";
      o << "      if (e_ < rest_) {\n";
      for (int qi = 0; qi < NQ; ++qi) o << "        q_base[" << qi * QCAP << " + e_] = v_[" << qi << "];\n";
      o << "      }\n";
      o << "      __syncwarp();\n";
      o << "    }\n";
      o << "    q_n = rest_;\n";
      o << "   }\n";
      o << "   if (!live_) break;\n";
    }

    if (STAGES > 0) {
      o << "    __syncwarp();\n";
      o << "    if (lane == 0 && staged_ok) {\n";
      o << "      const long long t2 = t + (long long)NSTAGE * nwarps;\n";
      o << "      if (t2 < full_tiles) CX_ISSUE(t2, stage);\n";
      o << "    }\n";
    }
    o << "  }\n";
    if (STAGES > 0)
      o << "  if (aborted && lane == 0 && staged_ok) cx::drain_stages(bars, NSTAGE, k_iter, gwarp, nwarps, full_tiles, "
        << wait_limit << "u);\n";

    // Flush block-private state.
    if (!grouped) {
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        o << "  {\n";
        if (ag.fn == AggFn::Min) {
          o << "    const unsigned long long r_ = cx::block_min_u64<" << CTA << ">(acc_" << k << ", red);\n";
          o << "    if (threadIdx.x == 0) db::atomic_min_ull(d_result[" << k << "], r_);\n";
        } else if (ag.fn == AggFn::Max) {
          o << "    const unsigned long long r_ = cx::block_max_u64<" << CTA << ">(acc_" << k << ", red);\n";
          o << "    if (threadIdx.x == 0) db::atomic_max_ull(d_result[" << k << "], r_);\n";
        } else {
          o << "    const unsigned long long r_ = cx::block_sum_u64<" << CTA << ">(acc_" << k << ", red);\n";
          o << "    if (threadIdx.x == 0) db::atomic_add_ull(d_result[" << k << "], r_);\n";
        }
        if (ag.fn == AggFn::Count) o << "    if (threadIdx.x == 0) db::atomic_set_valid_bit(d_result_validity, " << k << ");\n";
        if (seen_idx[k] >= 0) {
          o << "    const unsigned long long s_ = cx::block_sum_u64<" << CTA << ">(seen_" << k << ", red);\n";
          o << "    if (threadIdx.x == 0 && s_ != 0ULL) db::atomic_set_valid_bit(d_result_validity, " << k << ");\n";
        }
        if (ag.fn == AggFn::Avg) {
          o << "    const unsigned long long c_ = cx::block_sum_u64<" << CTA << ">(cnt_" << k << ", red);\n";
          o << "    if (threadIdx.x == 0) db::atomic_add_ull(d_result[" << p.hidden_count_slot(k) << "], c_);\n";
        }
        o << "  }\n";
      }
    } else if (reg_groups || lane_groups) {
      o << "  const unsigned touch_all = cx::block_or_u32<" << CTA << ">(rtouch, red);\n";
      for (int k = 0; k < NA; ++k)
        if (seen_idx[k] >= 0 && NSEEN_T > 0)
          o << "  const unsigned seen_all_" << k << " = cx::block_or_u32<" << CTA << ">(rseen_" << k << ", red);\n";
      o << "  #pragma unroll 1\n  for (int g = 0; g < " << G << "; ++g) {\n";
      o << "    unsigned long long v_[" << NACC << "];\n";
      o << "    #pragma unroll\n    for (int k = 0; k < " << NACC << "; ++k) {\n";
      o << "      unsigned long long x_ = 0ULL;\n";
      if (lane_groups)
        o << "      x_ = s_lacc[((unsigned)g * " << NACC << "u + (unsigned)k) * " << CTA << "u + threadIdx.x];\n";
      else
        o << "      #pragma unroll\n      for (int h = 0; h < " << G << "; ++h) if (h == g) x_ = racc[h * " << NACC << " + k];\n";
      o << "      v_[k] = x_;\n";
      o << "    }\n";
      for (int k = 0; k < NACC; ++k) {
        const bool is_min = k < NA && p.aggs[k].fn == AggFn::Min;
        const bool is_max = k < NA && p.aggs[k].fn == AggFn::Max;
        if (is_min) o << "    v_[" << k << "] = cx::block_min_u64<" << CTA << ">(v_[" << k << "], red);\n";
        else if (is_max) o << "    v_[" << k << "] = cx::block_max_u64<" << CTA << ">(v_[" << k << "], red);\n";
        else o << "    v_[" << k << "] = cx::block_sum_u64<" << CTA << ">(v_[" << k << "], red);\n";
      }
      o << "    if (threadIdx.x == 0 && ((touch_all >> g) & 1u)) {\n";
      emit_key_store(o, "g", "      ");
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const int slot = (int)p.groups.size() + k;
        const std::string ix = "(unsigned long long)g * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
        if (ag.fn == AggFn::Min) o << "      if (v_[" << k << "] != ~0ULL) atomicMin(&d_result[" << ix << "], v_[" << k << "]);\n";
        else if (ag.fn == AggFn::Max) o << "      if (v_[" << k << "] != 0ULL) atomicMax(&d_result[" << ix << "], v_[" << k << "]);\n";
        else o << "      if (v_[" << k << "] != 0ULL) atomicAdd(&d_result[" << ix << "], v_[" << k << "]);\n";
        if (!p.sparse) {
          if (ag.fn == AggFn::Count) o << "      db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
          if (seen_idx[k] >= 0) o << "      if ((seen_all_" << k << " >> g) & 1u) db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
        }
        if (ag.fn == AggFn::Avg)
          o << "      if (v_[" << avg_idx[k] << "] != 0ULL) atomicAdd(&d_result[(unsigned long long)g * " << TS << "ULL + " << p.hidden_count_slot(k) << "], v_[" << avg_idx[k] << "]);\n";
      }
      o << "    }\n";
      o << "  }\n";
    } else if (smem_groups) {
      o << "  __syncthreads();\n";
      o << "  for (long long g = threadIdx.x; g < " << G << "LL; g += " << CTA << ") {\n";
      o << "    unsigned touched_ = 0u;\n";
      o << "    for (int r = 0; r < " << REP << "; ++r) touched_ |= (s_touch_all[(long long)r * " << TW << "LL + (g >> 5)] >> (g & 31)) & 1u;\n";
      o << "    if (!touched_) continue;\n";
      emit_key_store(o, "g", "    ");
      for (int k = 0; k < NA; ++k) {
        const Agg& ag = p.aggs[k];
        const int slot = (int)p.groups.size() + k;
        const std::string dst = "d_result[(unsigned long long)g * " + std::to_string(TS) + "ULL + " + std::to_string(slot) + "]";
        const std::string vb = "(unsigned long long)g * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
        o << "    { unsigned long long v_ = " << (ag.fn == AggFn::Min ? "~0ULL" : "0ULL") << "; unsigned seen_ = 0u; (void)seen_;\n";
        o << "      for (int r = 0; r < " << REP << "; ++r) {\n";
        o << "        const unsigned long long y_ = s_acc_all[((long long)r * " << G << "LL + g) * " << NACC << " + " << k << "];\n";
        if (ag.fn == AggFn::Min) o << "        v_ = y_ < v_ ? y_ : v_;\n";
        else if (ag.fn == AggFn::Max) o << "        v_ = y_ > v_ ? y_ : v_;\n";
        else o << "        v_ += y_;\n";
        if (seen_idx[k] >= 0 && NSEEN_T > 0)
          o << "        seen_ |= (s_seen_all[(long long)r * " << (unsigned long long)NSEEN_T * TW << "LL + " << (unsigned long long)seen_idx[k] * TW
            << "LL + (g >> 5)] >> (g & 31)) & 1u;\n";
        o << "      }\n";
        if (ag.fn == AggFn::Min) o << "      if (v_ != ~0ULL) atomicMin(&" << dst << ", v_);\n";
        else if (ag.fn == AggFn::Max) o << "      if (v_ != 0ULL) atomicMax(&" << dst << ", v_);\n";
        else o << "      if (v_ != 0ULL) atomicAdd(&" << dst << ", v_);\n";
        if (!p.sparse) {
          if (ag.fn == AggFn::Count) o << "      db::atomic_set_valid_bit(d_result_validity, " << vb << ");\n";
          if (seen_idx[k] >= 0) o << "      if (seen_) db::atomic_set_valid_bit(d_result_validity, " << vb << ");\n";
        }
        if (ag.fn == AggFn::Avg) {
          o << "      unsigned long long c_ = 0ULL;\n";
          o << "      for (int r = 0; r < " << REP << "; ++r) c_ += s_acc_all[((long long)r * " << G << "LL + g) * " << NACC << " + " << avg_idx[k] << "];\n";
          o << "      if (c_ != 0ULL) atomicAdd(&d_result[(unsigned long long)g * " << TS << "ULL + " << p.hidden_count_slot(k) << "], c_);\n";
        }
        o << "    }\n";
      }
      o << "  }\n";
    }
    o << "}\n";
    if (STAGES > 0) o << "#undef CX_ISSUE\n";
    o << "\n";

    if (grouped && !smem_groups && !reg_groups && !lane_groups) {
      meta << "kernel group_keys_epilogue groups 0 256 0\n";
      o << "extern \"C\" __global__ void __launch_bounds__(256) group_keys_epilogue(const CxArgs a) {\n";
      o << "  unsigned long long* d_result = a.result;\n";
      o << "  uint64_t* d_result_validity = (uint64_t*)a.result_validity; (void)d_result_validity;\n";
      o << "  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n";
      o << "  if (g >= " << G << "LL) return;\n";
      // A COUNT(*) slot is non-zero exactly for the groups some row reached, so
      // plans with one keep no touched bits in global memory.
      if (count_star_slot() >= 0)
        o << "  if (d_result[(unsigned long long)g * " << p.storage_ts() << "ULL + " << count_star_slot() << "] == 0ULL) return;\n";
      else
        o << "  if (!((a.touched[g >> 5] >> (g & 31)) & 1u)) return;\n";
      emit_key_store(o, "g", "  ");
      o << "}\n\n";
    }
  }

  // ------------------------------------------------------- aux kernels ---
  void emit_init_min() {
    const unsigned long long G = total_groups();
    const int TS = p.storage_ts();
    meta << "kernel init_aggregate_slots groups 0 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) init_aggregate_slots(const CxArgs a) {\n";
    src << "  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n";
    src << "  if (g >= " << G << "LL) return;\n";
    src << "  const unsigned long long base = (unsigned long long)g * " << TS << "ULL;\n";
    for (size_t k = 0; k < p.aggs.size(); ++k)
      if (p.aggs[k].fn == AggFn::Min) src << "  a.result[base + " << p.groups.size() + k << "] = ~0ULL;\n";
    src << "}\n\n";
  }

  void emit_finalize() {
    const unsigned long long G = total_groups();
    const int TS = p.storage_ts(), VTS = p.visible_ts();
    const bool scalar = p.groups.empty();
    meta << "finalize " << G << " " << VTS << "\n";
    meta << "kernel finalize_aggregate_slots groups 0 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) finalize_aggregate_slots(const CxArgs a) {\n";
    src << "  const unsigned long long* d_result = a.result;\n";
    src << "  const uint64_t* d_result_validity = (const uint64_t*)a.result_validity;\n";
    src << "  unsigned long long* d_visible_result = a.finalize_tmp;\n";
    src << "  uint64_t* d_visible_validity = (uint64_t*)(a.finalize_tmp + " << G * VTS << "ULL);\n";
    src << "  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;\n";
    src << "  if (g >= " << G << "LL) return;\n";
    src << "  const unsigned long long src = (unsigned long long)g * " << TS << "ULL, dst = (unsigned long long)g * " << VTS << "ULL;\n";
    int slot = 0;
    for (size_t k = 0; k < p.groups.size(); ++k, ++slot) {
      src << "  d_visible_result[dst + " << slot << "] = d_result[src + " << slot << "];\n";
      src << "  if (db::bitmap_valid_at(d_result_validity, src + " << slot << ")) db::atomic_set_valid_bit(d_visible_validity, dst + " << slot << ");\n";
    }
    for (size_t k = 0; k < p.aggs.size(); ++k, ++slot) {
      const Agg& ag = p.aggs[k];
      const std::string s = std::to_string(slot);
      if (ag.fn == AggFn::Count) {
        src << "  d_visible_result[dst + " << s << "] = d_result[src + " << s << "];\n";
        if (scalar) src << "  db::atomic_set_valid_bit(d_visible_validity, dst + " << s << ");\n";
        else src << "  if (d_result[src + " << s << "] != 0ULL) db::atomic_set_valid_bit(d_visible_validity, dst + " << s << ");\n";
      } else if (ag.fn == AggFn::Avg) {
        const int cs = p.hidden_count_slot(k);
        src << "  { const unsigned long long cnt_ = d_result[src + " << cs << "];\n";
        src << "    if (cnt_ != 0ULL) {\n";
        src << "      const double avg_ = (double)d_result[src + " << s << "] / (double)cnt_;\n";
        src << "      d_visible_result[dst + " << s << "] = db::bit_cast_double_to_ull(avg_);\n";
        src << "      db::atomic_set_valid_bit(d_visible_validity, dst + " << s << ");\n";
        src << "    } }\n";
      } else {
        if (ag.fn == AggFn::Min)
          src << "  d_visible_result[dst + " << s << "] = (d_result[src + " << s << "] == ~0ULL) ? 0ULL : d_result[src + " << s << "];\n";
        else
          src << "  d_visible_result[dst + " << s << "] = d_result[src + " << s << "];\n";
        src << "  if (db::bitmap_valid_at(d_result_validity, src + " << s << ")) db::atomic_set_valid_bit(d_visible_validity, dst + " << s << ");\n";
      }
    }
    src << "}\n\n";
  }

  std::string run() {
    // Payload columns that keep their validity through the hash table.
    for (const auto& s : p.steps)
      if (s.kind == Step::JoinStep && !s.join.payload.empty() && nullable(s.join.payload))
        payload_valid.insert(s.join.payload);

    meta << "v 1\n";
    if (nparams >= 0) meta << "params " << nparams << "\n";
    for (size_t t = 0; t < p.tables.size(); ++t) meta << "table " << t << " " << p.tables[t].name << "\n";
    choose_tables();
    int h = 0;
    for (const auto& s : p.steps) {
      if (s.kind != Step::JoinStep) continue;
      ht_slot[s.join.dim] = h;
      if (s.join.multi) {
        meta << "ht " << h << " " << ht_name(s.join.dim) << " " << mht_words(s.join) << "\n";
        meta << "mht " << h << " " << p.table_slot(s.join.dim) << " " << mht_arrays(s.join) << "\n";
        ++h;
        continue;
      }
      const long long words = 2 * s.join.len;  // 2 x len, as the reference allocates (visitor.cpp:4216-4218)
      meta << "ht " << h << " " << ht_name(s.join.dim) << " " << words << "\n";
      if (!s.join.payload.empty() && payload_valid.count(s.join.payload))
        meta << "htv " << h << " " << (s.join.len + 31) / 32 << "\n";
      meta << "bm " << h << " " << (ptable.count(s.join.dim) ? (s.join.len + 3) / 4 : (s.join.len + 31) / 32) << "\n";
      ++h;
    }
    if (h > CX_MAX_HTS_) throw PlanError("too many joins");
    const unsigned long long G = total_groups();
    meta << "result " << G * p.storage_ts() << " " << G << " " << p.storage_ts() << " " << p.visible_ts() << " "
         << (p.sparse ? 1 : 0) << "\n";

    if (p.has_min()) emit_init_min();
    for (const auto& s : p.steps)
      if (s.kind == Step::JoinStep) emit_build(s.join);
    for (const auto& s : p.steps)
      if (s.kind == Step::JoinStep) emit_occupancy(s.join);  // exact membership bitmaps
    emit_scan();
    if (p.hidden_count_slots() > 0) emit_finalize();

    for (size_t s = 0; s < col_order.size(); ++s) {
      meta << "col " << s << " d_" << col_order[s] << " " << p.table_of_col.at(col_order[s]) << "\n";
      if (nullable(col_order[s])) meta << "null " << s << " d_" << col_order[s] << "\n";
    }

    std::ostringstream out;
    out << "/*@cx-launch\n" << meta.str() << "@*/\n";
    out << "// Generated by crystal-b200 for sm_100a.\n";
    out << "#include \"cx_args.h\"\n#include \"crystal_sm100.cuh\"\n\n";
    out << "template <typename A, typename B>\n"
           "__device__ __forceinline__ auto cx_mdiv(A x, B y) -> decltype(x / y) {\n"
           "  return (y == 0) ? (decltype(x / y))0 : x / y;\n}\n\n";
    out << src.str();
    return out.str();
  }

  static constexpr int CX_MAX_HTS_ = 8;
};

std::string generate_cuda_impl(const Plan& plan, const Tuning& tuning) {
  Emitter e(plan, tuning);
  std::map<const Expr*, int> lm;
  if (tuning.parametric) {
    std::vector<const Expr*> lits;
    collect_literals(plan, lits);
    if (lits.size() > 64) throw PlanError("more than 64 literals in a parametric kernel");
    for (size_t k = 0; k < lits.size(); ++k) {
      if (lits[k]->ival < -2147483647LL || lits[k]->ival > 2147483647LL) throw PlanError("literal outside int32");
      lm[lits[k]] = (int)k;
    }
    e.lit_index = &lm;
    e.nparams = (int)lits.size();
  }
  return e.run();
}

// ============================================================ shared scan ===
// One persistent kernel answers a batch of up to 64 queries of several plan
// shapes in one pass over the fact table.  Every query's predicates collapse
// into one 64-bit query mask per fact row (bit q set: the row passes query q),
// in the manner of the CJOIN shared star-join operator (Candea, Polyzotis,
// Vingralek, VLDB 2009):
//  * index_<dim> kernels store, at the PHT slot HASH(key, len, key_min) of each
//    dimension row, {key, mask_lo, mask_hi, attr0} and up to three more payload
//    attributes.  Mask bit q is set when query q does not join the dimension or
//    the row passes the query's dimension filter -- the condition under which
//    the reference's filtered PHT would hold that key (join.h:124-253, 7-120).
//    Keys must occupy distinct slots (checked while indexing) and foreign keys
//    must be non-zero (checked by the engine before it forms a batch).
//  * single-column fact filters become per-CTA lookup tables over a window of
//    FW values of the column, starting at the column minimum the host
//    registered; values outside the window, and every other filter, are
//    evaluated per query for the rows still in the mask.
//  * warps then take (query, row slice) units and aggregate the rows whose bit
//    is set, four rows per lane, with partial aggregates in registers, a
//    per-query shared-memory table or global atomics.

void lits_of(const Expr* e, std::vector<const Expr*>& out) {
  if (!e) return;
  if (e->op == Op::Int) out.push_back(e);
  for (const auto& k : e->kids) lits_of(k.get(), out);
}

// Top-level AND terms of a filter.  Shared shapes have no nullable columns, so
// two-valued logic holds and the terms can be evaluated separately.
void conjuncts_of(const Expr* e, std::vector<const Expr*>& out) {
  if (!e) return;
  if (e->op == Op::And) {
    conjuncts_of(e->kids[0].get(), out);
    conjuncts_of(e->kids[1].get(), out);
    return;
  }
  out.push_back(e);
}

void cols_of(const Expr* e, std::vector<std::string>& out) {
  if (!e) return;
  if (e->op == Op::Col && std::find(out.begin(), out.end(), e->name) == out.end()) out.push_back(e->name);
  for (const auto& k : e->kids) cols_of(k.get(), out);
}

struct SharedGen {
  static constexpr int MAXQ = 64;       // queries per launch (two 32-bit mask words)
  static constexpr int FW = 256;        // values per fact filter table
  static constexpr int MAX_FCOLS = 8;   // fact columns with filter tables
  static constexpr int MAX_ATTRS = 4;   // payload attributes per dimension

  const std::vector<const Plan*>& shapes;
  const Tuning& tu;
  std::ostringstream meta, src;
  std::string fact;
  std::vector<std::string> tables;
  std::vector<std::string> fact_cols;   // staged fact columns
  struct Dim {
    std::string name, pk, fk;
    long long len = 0, keymin = 0;
    std::vector<std::string> attrs;     // payload attributes; attrs[0] rides in the key entry
    std::vector<std::string> fcols;     // dimension columns read by join filters
    int slot = 0, table = 0;
  };
  std::vector<Dim> dims;
  std::map<std::string, int> attr_dim;  // payload attribute -> dimension index
  std::map<std::string, int> col_slot;
  std::vector<std::pair<std::string, int>> col_order;
  std::vector<std::map<const Expr*, int>> lit_maps;
  int max_lits = 0, max_scalar_aggs = 0;
  struct Preds {
    std::map<int, std::vector<const Expr*>> joins;   // dimension -> its filters (null: join only)
    std::map<int, std::vector<const Expr*>> pushed;  // filter-table column -> conjuncts on it
    std::vector<const Expr*> resid;                  // conjuncts evaluated per row and query
  };
  std::vector<Preds> preds;
  std::vector<std::string> fcols;       // fact columns with filter tables

  SharedGen(const std::vector<const Plan*>& s, const Tuning& t) : shapes(s), tu(t) {}

  int table_slot(const std::string& t) {
    for (size_t i = 0; i < tables.size(); ++i)
      if (tables[i] == t) return (int)i;
    tables.push_back(t);
    return (int)tables.size() - 1;
  }
  int slot_of(const std::string& c, int table) {
    auto it = col_slot.find(c);
    if (it != col_slot.end()) return it->second;
    const int s = (int)col_order.size();
    if (s >= CX_MAX_COLS_) throw PlanError("too many columns in a shared batch");
    col_slot[c] = s;
    col_order.push_back({c, table});
    return s;
  }
  int dim_index(const std::string& n) const {
    for (size_t i = 0; i < dims.size(); ++i)
      if (dims[i].name == n) return (int)i;
    return -1;
  }
  void add_fact(const std::string& c) {
    if (std::find(fact_cols.begin(), fact_cols.end(), c) == fact_cols.end()) fact_cols.push_back(c);
  }
  // Columns of a row-level expression: fact columns are staged, any other
  // column must be a payload attribute of a dimension the shape joins.
  void need_row_cols(const Plan& p, const Expr* e) {
    std::vector<std::string> cs;
    cols_of(e, cs);
    for (const auto& c : cs) {
      if (p.table_of_col.at(c) == 0) add_fact(c);
      else if (!attr_dim.count(c)) throw PlanError("column " + c + " is neither a fact column nor a join payload");
    }
  }

  void collect() {
    if (shapes.empty() || shapes.size() > CX_MAX_SHAPES_) throw PlanError("shared batch needs 1..16 shapes");
    fact = shapes[0]->tables[0].name;
    table_slot(fact);
    preds.resize(shapes.size());
    for (size_t si = 0; si < shapes.size(); ++si) {
      const Plan& p = *shapes[si];
      if (p.tables[0].name != fact) throw PlanError("shared batch mixes fact tables");
      std::function<void(const Expr*)> no_null = [&](const Expr* x) {
        if (!x) return;
        if (x->op == Op::Col && p.nullable.count(x->name)) throw PlanError("nullable column " + x->name + " is not shareable");
        for (const auto& k : x->kids) no_null(k.get());
      };
      std::map<const Expr*, int> lm;
      std::vector<const Expr*> lits;
      collect_literals(p, lits);
      for (size_t k = 0; k < lits.size(); ++k) {
        if (lits[k]->ival < -2147483647LL || lits[k]->ival > 2147483647LL) throw PlanError("literal outside int32");
        lm[lits[k]] = (int)k;
      }
      max_lits = std::max(max_lits, (int)lits.size());
      if (p.groups.empty()) max_scalar_aggs = std::max(max_scalar_aggs, (int)p.aggs.size());
      lit_maps.push_back(lm);
      // Joins first: their payloads are the attributes later expressions read.
      for (const auto& s : p.steps) {
        if (s.kind != Step::JoinStep) continue;
        const Join& j = s.join;
        if (j.fks.size() != 1) throw PlanError("OR-joins are not shareable");
        if (j.multi) throw PlanError("multi-value hash joins are not shareable");
        int di = dim_index(j.dim);
        if (di < 0) {
          dims.push_back(Dim());
          Dim& d = dims.back();
          d.name = j.dim;
          d.pk = j.pk;
          d.fk = j.fks[0];
          d.len = j.len;
          d.keymin = j.keymin;
          d.slot = (int)dims.size() - 1;
          d.table = table_slot(j.dim);
          di = d.slot;
        } else {
          const Dim& d = dims[di];
          if (d.pk != j.pk || d.fk != j.fks[0] || d.len != j.len || d.keymin != j.keymin)
            throw PlanError("shapes join " + j.dim + " differently");
        }
        Dim& d = dims[di];
        if (p.nullable.count(j.fks[0]) || p.nullable.count(j.pk)) throw PlanError("nullable join key is not shareable");
        if (d.len <= 0 || d.len > (1LL << 30)) throw PlanError("dimension " + j.dim + " has an unusable slot count");
        add_fact(j.fks[0]);
        no_null(j.filter.get());
        std::vector<std::string> fc;
        cols_of(j.filter.get(), fc);
        for (const auto& c : fc) {
          if (p.table_of_col.at(c) != p.table_slot(j.dim)) throw PlanError("join filter of " + j.dim + " reads " + c);
          if (std::find(d.fcols.begin(), d.fcols.end(), c) == d.fcols.end()) d.fcols.push_back(c);
        }
        preds[si].joins[di].push_back(j.filter.get());
        if (!j.payload.empty()) {
          if (p.nullable.count(j.payload)) throw PlanError("nullable dimension column " + j.payload + " is not shareable");
          auto it = attr_dim.find(j.payload);
          if (it != attr_dim.end() && it->second != di) throw PlanError("payload " + j.payload + " of two dimensions");
          if (std::find(d.attrs.begin(), d.attrs.end(), j.payload) == d.attrs.end()) d.attrs.push_back(j.payload);
          attr_dim[j.payload] = di;
          if ((int)d.attrs.size() > MAX_ATTRS) throw PlanError("more than 4 payload attributes of " + j.dim + " in one shared batch");
        }
      }
      for (const auto& s : p.steps) {
        if (s.kind != Step::Filter) continue;
        no_null(s.filter.get());
        std::vector<const Expr*> cj;
        conjuncts_of(s.filter.get(), cj);
        for (const Expr* c : cj) {
          std::vector<std::string> cs;
          cols_of(c, cs);
          need_row_cols(p, c);
          // A conjunct over payload attributes of one joined dimension is a
          // predicate on the dimension row: it joins that dimension's mask.
          int dd = -1;
          bool dim_only = !cs.empty();
          for (const auto& cc : cs) {
            auto it = attr_dim.find(cc);
            if (p.table_of_col.at(cc) == 0 || it == attr_dim.end() || (dd >= 0 && dd != it->second)) { dim_only = false; break; }
            dd = it->second;
          }
          if (dim_only && preds[si].joins.count(dd)) {
            preds[si].joins[dd].push_back(c);
            for (const auto& cc : cs)
              if (std::find(dims[dd].fcols.begin(), dims[dd].fcols.end(), cc) == dims[dd].fcols.end()) dims[dd].fcols.push_back(cc);
            continue;
          }
          if (cs.size() == 1 && p.table_of_col.at(cs[0]) == 0) {
            auto it = std::find(fcols.begin(), fcols.end(), cs[0]);
            int k = (int)(it - fcols.begin());
            if (it == fcols.end()) {
              if ((int)fcols.size() < MAX_FCOLS) { fcols.push_back(cs[0]); k = (int)fcols.size() - 1; }
              else k = -1;
            }
            if (k >= 0) { preds[si].pushed[k].push_back(c); continue; }
          }
          preds[si].resid.push_back(c);
        }
      }
      for (const auto& a : p.aggs) {
        if (a.fn != AggFn::Count && a.fn != AggFn::Sum) throw PlanError("shared scans support COUNT and SUM");
        no_null(a.arg.get());
        need_row_cols(p, a.arg.get());
      }
      for (const auto& g : p.groups) {
        if (g.nullable) throw PlanError("nullable group key is not shareable");
        no_null(g.expr.get());
        need_row_cols(p, g.expr.get());
      }
    }
    if ((int)dims.size() > CX_MAX_HTS_) throw PlanError("too many dimensions in a shared batch");
    if (dims.size() > 32) throw PlanError("too many dimensions in a shared batch");
  }

  std::string conj_and(Emitter& e, const std::vector<const Expr*>& cs) const {
    std::string out;
    for (const Expr* c : cs) {
      if (!c) continue;
      const std::string t = and_terms({e.valid_of(c), e.value_of(c)});
      if (lit_true(t)) continue;
      out += (out.empty() ? "" : " && ") + std::string("(") + t + ")";
    }
    return out.empty() ? "true" : out;
  }

  // Per pass: zeroes every query's result words, validity words and touched
  // bits (one block per query), so a pass has the same launches whatever its
  // queries' buffers are.
  void emit_zero() {
    meta << "kernel shared_zero zero 0 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) shared_zero(const CxArgs a) {\n";
    src << "  const int q = blockIdx.x;\n";
    src << "  if (q >= a.sq_total) return;\n";
    src << "  const CxSQ Q = a.sq[q];\n";
    src << "  long long nw = 0, nt = 0;\n";
    src << "  switch (Q.shape) {\n";
    for (size_t si = 0; si < shapes.size(); ++si) {
      const Plan& p = *shapes[si];
      Emitter e(p, tu);
      const unsigned long long G = e.total_groups();
      src << "    case " << si << ": nw = " << G * (unsigned long long)p.storage_ts() << "LL; nt = "
          << (p.groups.empty() ? 0ULL : (G + 31) / 32) << "LL; break;\n";
    }
    src << "    default: break;\n";
    src << "  }\n";
    src << "  const long long nv = (nw + 63) / 64;\n";
    src << "  if (!Q.keep) {  // a query continuing over a later row range keeps its result\n";
    src << "    for (long long i = threadIdx.x; i < nw; i += blockDim.x) Q.result[i] = 0ULL;\n";
    src << "    for (long long i = threadIdx.x; i < nv; i += blockDim.x) Q.validity[i] = 0ULL;\n";
    src << "  }\n";
    src << "  if (Q.touched)\n";
    src << "    for (long long i = threadIdx.x; i < nt; i += blockDim.x) Q.touched[i] = 0u;\n";
    src << "}\n\n";
  }

  // Per batch: slot entries of one dimension with the batch's query masks.
  void emit_index(const Dim& d, int di) {
    const std::string k = "index_" + lower(d.name);
    meta << "kernel " << k << " build " << d.table << " 256 1024\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) " << k << "(const CxArgs a) {\n";
    src << "  __shared__ int s_shape[" << MAXQ << "], s_poff[" << MAXQ << "];\n";
    src << "  const int nq = a.sq_total < " << MAXQ << " ? a.sq_total : " << MAXQ << ";\n";
    src << "  for (int q = threadIdx.x; q < nq; q += blockDim.x) { s_shape[q] = a.sq[q].shape; s_poff[q] = a.sq[q].param_off; }\n";
    src << "  __syncthreads();\n";
    src << "  const long long n = a.rows[" << d.table << "];\n";
    src << "  int4* dkm = (int4*)a.ht[" << d.slot << "];\n";
    if (d.attrs.size() > 1) src << "  int4* dat = (int4*)a.dat[" << d.slot << "];\n";
    src << "  const int* __restrict__ key = a.col[" << slot_of(d.pk, d.table) << "];\n";
    for (size_t i = 0; i < d.attrs.size(); ++i)
      src << "  const int* __restrict__ at" << i << " = a.col[" << slot_of(d.attrs[i], d.table) << "];\n";
    for (const auto& c : d.fcols) src << "  const int* __restrict__ F_" << c << " = a.col[" << slot_of(c, d.table) << "];\n";
    src << "  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {\n";
    src << "    const int k = key[r];\n";
    src << "    if (k == 0) continue;\n";
    src << "    const int h = (int)HASH(k, " << d.len << ", " << d.keymin << ");\n";
    src << "    if ((unsigned)h >= " << d.len << "u) continue;\n";
    src << "    if (atomicCAS(&dkm[h].x, 0, k) != 0) { cx::raise(a.err, cx::ERR_DIM_COLLISION); continue; }\n";
    src << "    unsigned long long m = 0ULL;\n";
    src << "    for (int q = 0; q < nq; ++q) {\n";
    src << "      const int* P = a.sparams + s_poff[q]; (void)P;\n";
    src << "      bool pass = true;\n";
    src << "      switch (s_shape[q]) {\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      auto it = preds[s].joins.find(di);
      if (it == preds[s].joins.end()) continue;
      Emitter e(*shapes[s], tu);
      e.lit_index = &lit_maps[s];
      for (const auto& c : d.fcols) e.col_expr[c] = "F_" + c + "[r]";
      const std::string f = conj_and(e, it->second);
      if (f == "true") continue;
      src << "        case " << s << ": pass = " << f << "; break;\n";
    }
    src << "        default: break;\n";
    src << "      }\n";
    src << "      if (pass) m |= 1ULL << q;\n";
    src << "    }\n";
    src << "    dkm[h] = make_int4(k, (int)(unsigned)m, (int)(unsigned)(m >> 32), " << (d.attrs.empty() ? "0" : "at0[r]") << ");\n";
    if (d.attrs.size() > 1) {
      src << "    dat[h] = make_int4(";
      for (size_t i = 1; i < 4; ++i) src << (i > 1 ? ", " : "") << (i < d.attrs.size() ? "at" + std::to_string(i) + "[r]" : "0");
      src << ", 0);\n";
    }
    src << "  }\n}\n\n";
  }

  // ------------------------------------------------------ aggregate cubes --
  // The queries of one shape differ only in their literals.  When every column
  // that a shape's predicates and GROUP BY keys read has a small value range,
  // one pass adds each fact row's aggregate values into one cell per shape --
  // the cell indexed by those columns' values, dimension columns taken from the
  // row the join finds -- and each query is answered afterwards from the cells
  // its own predicates accept (CUBE-style shared aggregation; integer sums in
  // any order give the same words).  The per-row work then no longer grows with
  // the number of queries.  Value ranges are registered on the execution
  // context, so the program keeps the per-query mask kernels beside the cube
  // kernels and the runtime picks one path per batch.
  struct CAttr { int dim; int field; std::string col; };  // dim < 0: a fact column
  std::vector<CAttr> cattrs;
  std::map<std::string, int> cattr_id;
  std::vector<std::vector<int>> sh_attrs;  // per shape: its attributes in cell order (last varies fastest)
  std::vector<int> dim_fields;             // 16-bit attribute fields used per dimension entry
  std::string cube_why;                    // why the batch has no cube path ("" = it has one)
  static constexpr int MAX_CATTRS = 32, MAX_SATTRS = 8;

  void collect_cube() {
    dim_fields.assign(dims.size(), 0);
    sh_attrs.assign(shapes.size(), {});
    auto add = [&](const Plan& p, const std::string& c, std::vector<int>& mine) -> bool {
      int id;
      auto it = cattr_id.find(c);
      if (it != cattr_id.end()) {
        id = it->second;
      } else {
        CAttr at{-1, 0, c};
        const int ts = p.table_of_col.at(c);
        if (ts != 0) {
          const int di = dim_index(p.tables[ts].name);
          if (di < 0) { cube_why = "column " + c + " is not of a joined dimension"; return false; }
          if (dim_fields[di] >= 4) { cube_why = "more than four cube attributes of " + dims[di].name; return false; }
          at.dim = di;
          at.field = dim_fields[di]++;
        }
        if ((int)cattrs.size() >= MAX_CATTRS) { cube_why = "more than 32 cube attributes"; return false; }
        id = (int)cattrs.size();
        cattrs.push_back(at);
        cattr_id[c] = id;
      }
      if (std::find(mine.begin(), mine.end(), id) == mine.end()) mine.push_back(id);
      return true;
    };
    for (size_t si = 0; si < shapes.size(); ++si) {
      const Plan& p = *shapes[si];
      for (const auto& ag : p.aggs) {
        std::vector<const Expr*> ls;
        lits_of(ag.arg.get(), ls);
        if (!ls.empty()) { cube_why = "an aggregate reads a literal"; return; }
        std::vector<std::string> cs;
        cols_of(ag.arg.get(), cs);
        for (const auto& c : cs)
          if (p.table_of_col.at(c) != 0) { cube_why = "an aggregate reads dimension column " + c; return; }
      }
      std::vector<std::string> cs;
      for (const auto& st : p.steps) cols_of(st.kind == Step::Filter ? st.filter.get() : st.join.filter.get(), cs);
      for (const auto& g : p.groups) cols_of(g.expr.get(), cs);
      for (const auto& c : cs)
        if (!add(p, c, sh_attrs[si])) return;
      if ((int)sh_attrs[si].size() > MAX_SATTRS) { cube_why = "a shape reads more than 8 cube attributes"; return; }
    }
  }

  // Bit c of colmask[s]: shape s reads staged fact column c.
  std::vector<unsigned long long> shape_colmasks() const {
    std::vector<unsigned long long> colmask(shapes.size(), 0ULL);
    for (size_t si = 0; si < shapes.size(); ++si) {
      const Plan& p = *shapes[si];
      std::vector<std::string> cs;
      for (const auto& st : p.steps) {
        if (st.kind == Step::Filter) cols_of(st.filter.get(), cs);
        else cs.push_back(st.join.fks[0]);
      }
      for (const auto& g : p.groups) cols_of(g.expr.get(), cs);
      for (const auto& ag : p.aggs) cols_of(ag.arg.get(), cs);
      for (const auto& c : cs) {
        auto it = std::find(fact_cols.begin(), fact_cols.end(), c);
        if (it != fact_cols.end() && it - fact_cols.begin() < 64) colmask[si] |= 1ULL << (it - fact_cols.begin());
      }
    }
    return colmask;
  }

  int sum_aggs(const Plan& p) const {
    int n = 0;
    for (const auto& ag : p.aggs) n += ag.fn == AggFn::Sum;
    return n;
  }

  // Per batch: each dimension row's entry at its slot -- key, the shapes one of
  // whose queries its join filter passes (shapes that do not join the
  // dimension always set), and its cube attributes as 16-bit offsets from the
  // registered range minimum.
  void emit_cube_index(const Dim& d, int di) {
    const std::string k = "cube_index_" + lower(d.name);
    meta << "kernel " << k << " cubeidx " << d.table << " 256 1024\n";
    std::ostringstream& o = src;
    o << "extern \"C\" __global__ void __launch_bounds__(256) " << k << "(const CxArgs a) {\n";
    o << "  const long long n = a.rows[" << d.table << "];\n";
    o << "  int4* ent = (int4*)a.ht[" << d.slot << "];\n";
    o << "  const int* __restrict__ key = a.col[" << slot_of(d.pk, d.table) << "];\n";
    std::set<std::string> decl;
    auto declare = [&](const std::string& c) {
      if (decl.insert(c).second) o << "  const int* __restrict__ F_" << c << " = a.col[" << slot_of(c, d.table) << "];\n";
    };
    for (const auto& c : d.fcols) declare(c);
    for (const auto& at : cattrs)
      if (at.dim == di) declare(at.col);
    unsigned nj = 0;
    for (size_t s = 0; s < shapes.size(); ++s)
      if (!preds[s].joins.count(di)) nj |= 1u << s;
    o << "  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {\n";
    o << "    const int k = key[r];\n";
    o << "    if (k == 0) continue;\n";
    o << "    const int h = (int)HASH(k, " << d.len << ", " << d.keymin << ");\n";
    o << "    if ((unsigned)h >= " << d.len << "u) continue;\n";
    o << "    unsigned f_[4] = {0u, 0u, 0u, 0u};\n";
    o << "    bool bad_ = false;\n";
    for (size_t id = 0; id < cattrs.size(); ++id) {
      if (cattrs[id].dim != di) continue;
      o << "    { const unsigned x_ = (unsigned)(F_" << cattrs[id].col << "[r] - a.cube_lo[" << id << "]);\n";
      o << "      if (x_ >= (unsigned)a.cube_radix[" << id << "]) bad_ = true; else f_[" << cattrs[id].field << "] = x_; }\n";
    }
    o << "    if (bad_) { cx::raise(a.err, cx::ERR_CUBE_RANGE); continue; }\n";
    o << "    unsigned rel = " << nj << "u;\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      auto it = preds[s].joins.find(di);
      if (it == preds[s].joins.end()) continue;
      Emitter e(*shapes[s], tu);
      e.lit_index = &lit_maps[s];
      for (const auto& c : d.fcols) e.col_expr[c] = "F_" + c + "[r]";
      const std::string f = conj_and(e, it->second);
      if (f == "true") {
        o << "    if (a.sq_num[" << s << "] > 0) rel |= " << (1u << s) << "u;\n";
        continue;
      }
      o << "    for (int q = a.sq_first[" << s << "]; q < a.sq_first[" << s << "] + a.sq_num[" << s << "]; ++q) {\n";
      o << "      const int* P = a.sparams + a.sq[q].param_off; (void)P;\n";
      o << "      if (" << f << ") { rel |= " << (1u << s) << "u; break; }\n";
      o << "    }\n";
    }
    // A dimension kept as compact words: its word at key - key range minimum
    // (set with a 32-bit atomic OR on the word's 4-byte container, so a second
    // row with the same key is seen by its present bit), and no int4 entry.
    o << "    if (a.cube_desz[" << di << "] > 0) {\n";
    o << "      const unsigned o_ = (unsigned)k - (unsigned)a.cube_dbase[" << di << "];\n";
    o << "      if (o_ >= (unsigned)a.cube_dlen[" << di << "]) { cx::raise(a.err, cx::ERR_CUBE_RANGE); continue; }\n";
    o << "      unsigned w_ = 1u | (rel << 1);\n";
    o << "      #pragma unroll\n";
    o << "      for (int j = 0; j < 4; ++j) w_ |= f_[j] << a.cube_fsh[" << di * 4 << " + j];\n";
    o << "      unsigned* cw_ = (unsigned*)a.cube_dcomp[" << di << "];\n";
    o << "      const int es_ = a.cube_desz[" << di << "];\n";
    o << "      const unsigned sh_ = es_ == 1 ? (o_ & 3u) * 8u : es_ == 2 ? (o_ & 1u) * 16u : 0u;\n";
    o << "      const unsigned wi_ = es_ == 1 ? (o_ >> 2) : es_ == 2 ? (o_ >> 1) : o_;\n";
    o << "      const unsigned old_ = atomicOr(&cw_[wi_], w_ << sh_);\n";
    o << "      if ((old_ >> sh_) & 1u) cx::raise(a.err, cx::ERR_DIM_COLLISION);\n";
    o << "      continue;\n";
    o << "    }\n";
    o << "    if (atomicCAS(&ent[h].x, 0, k) != 0) { cx::raise(a.err, cx::ERR_DIM_COLLISION); continue; }\n";
    o << "    ent[h] = make_int4(k, (int)rel, (int)(f_[0] | (f_[1] << 16)), (int)(f_[2] | (f_[3] << 16)));\n";
    o << "  }\n}\n\n";
  }

  // One pass over the fact rows: warp tiles of 32 x IPT rows read with vector
  // loads; per row the shapes it may belong to (fact filter tables and the
  // dimension entries, a superset of what any query of the shape accepts),
  // then per such shape one cell update -- shared-memory cubes per CTA, merged
  // into the global cube at the end, or global atomics for large cubes.
  void emit_cube_scan() {
    // Few CTAs per SM, so each SM holds few copies of the shared-memory cubes
    // and dimension words: two or four rows per lane in one 1024-thread CTA (64
    // registers; compact dimension words keep four rows' state in them), one
    // in two 768-thread CTAs (40 registers, 48 warps).
    const int IPT = std::max(1, std::min(4, tu.cube)), VW = IPT >= 4 ? 4 : IPT;
    const int CTA = IPT >= 2 ? 1024 : 768;
    const int min_blocks = IPT == 1 ? 2 : 1;
    if (IPT == 3) throw PlanError("cube scans take 1, 2 or 4 rows per lane");
    const int NFC = (int)fcols.size();
    const unsigned long long fr_bytes = ((unsigned long long)NFC * FW * 4 + 15) & ~15ULL;
    const std::string kname = "CubeScan_" + fact;
    meta << "kernel " << kname << " cubescan 0 " << CTA << " " << 32 * IPT << " " << fr_bytes << " " << min_blocks << "\n";
    std::ostringstream o;
    o << "extern \"C\" __global__ void __launch_bounds__(" << CTA << ", " << min_blocks << ") " << kname << "(const CxArgs a) {\n";
    o << "  constexpr int IPT = " << IPT << ", VW = " << VW << ", TROWS = " << 32 * IPT << ";\n";
    o << "  extern __shared__ __align__(16) unsigned char cx_smem[];\n";
    o << "  unsigned* s_fr = (unsigned*)cx_smem; (void)s_fr;\n";
    o << "  unsigned char* s_dim = cx_smem + " << fr_bytes << "; (void)s_dim;\n";
    o << "  unsigned long long* s_cube = (unsigned long long*)(cx_smem + " << fr_bytes << " + a.cube_dsm_bytes);\n";
    o << "  const int lane = threadIdx.x & 31;\n";
    o << "  for (int w = threadIdx.x; w < a.cube_smem_words; w += " << CTA << ") s_cube[w] = 0ULL;\n";
    // Compact dimension words into shared memory (16-byte copies; the arrays are padded to 16 bytes).
    for (size_t di = 0; di < dims.size(); ++di) {
      o << "  if (a.cube_dsm[" << di << "] >= 0) {\n";
      o << "    const uint4* src_ = (const uint4*)a.cube_dcomp[" << di << "];\n";
      o << "    uint4* dst_ = (uint4*)(s_dim + a.cube_dsm[" << di << "]);\n";
      o << "    const int n16_ = (int)(((long long)a.cube_dlen[" << di << "] * a.cube_desz[" << di << "] + 15) / 16);\n";
      o << "    for (int w = threadIdx.x; w < n16_; w += " << CTA << ") dst_[w] = src_[w];\n";
      o << "  }\n";
    }
    o << "  unsigned live = 0u;\n";
    for (size_t s = 0; s < shapes.size(); ++s) o << "  if (a.sq_num[" << s << "] > 0) live |= " << (1u << s) << "u;\n";
    // Filter tables: bit s of s_fr[k * FW + v] clears when no query of shape s
    // accepts the value fbase[k] + v on filter column k.
    if (NFC) {
      o << "  for (int v = threadIdx.x; v < " << NFC * FW << "; v += " << CTA << ") {\n";
      o << "    const int k_ = v / " << FW << ";\n";
      o << "    const int fv_ = (int)((unsigned)a.fbase[k_] + (unsigned)(v - k_ * " << FW << "));\n";
      o << "    unsigned m = ~0u;\n";
      for (size_t s = 0; s < shapes.size(); ++s) {
        Emitter e(*shapes[s], tu);
        e.lit_index = &lit_maps[s];
        for (const auto& kv : preds[s].pushed) {
          e.col_expr.clear();
          e.col_expr[fcols[kv.first]] = "fv_";
          o << "    if (k_ == " << kv.first << " && a.sq_num[" << s << "] > 0) {\n";
          o << "      bool any_ = false;\n";
          o << "      for (int q = a.sq_first[" << s << "]; q < a.sq_first[" << s << "] + a.sq_num[" << s << "] && !any_; ++q) {\n";
          o << "        const int* P = a.sparams + a.sq[q].param_off; (void)P;\n";
          o << "        any_ = " << conj_and(e, kv.second) << ";\n";
          o << "      }\n";
          o << "      if (!any_) m &= ~" << (1u << s) << "u;\n";
          o << "    }\n";
        }
      }
      o << "    s_fr[v] = m;\n";
      o << "  }\n";
    }
    o << "  __syncthreads();\n";
    for (const auto& c : fact_cols) o << "  const int* __restrict__ d_" << c << " = a.col[" << slot_of(c, 0) << "];\n";
    for (const Dim& d : dims) o << "  const int4* __restrict__ ci_" << lower(d.name) << " = (const int4*)a.ht[" << d.slot << "];\n";
    for (int k = 0; k < NFC; ++k) o << "  const unsigned fb" << k << " = (unsigned)a.fbase[" << k << "], fw" << k << " = (unsigned)a.fwin[" << k << "];\n";
    o << "  bool vec_ok = true;\n";
    for (const auto& c : fact_cols) o << "  vec_ok = vec_ok && ((((unsigned long long)d_" << c << ") & 15ULL) == 0ULL);\n";
    // Fact columns the batch's shapes read (columns of shapes without queries are not loaded).
    if (fact_cols.size() > 64) throw PlanError("more than 64 fact columns in a shared batch");
    const std::vector<unsigned long long> colmask = shape_colmasks();
    o << "  unsigned long long need = 0ULL;\n";
    for (size_t s = 0; s < shapes.size(); ++s) o << "  if (a.sq_num[" << s << "] > 0) need |= " << colmask[s] << "ULL;\n";
    o << "  const long long n = a.rows[0];\n";
    o << "  const long long ntiles = (n + TROWS - 1) / TROWS;\n";
    o << "  const long long nw = ((long long)gridDim.x * " << CTA << ") >> 5;\n";
    o << "  bool bad_ = false;\n";
    o << "  for (long long t = ((long long)blockIdx.x * " << CTA << " + threadIdx.x) >> 5; t < ntiles; t += nw) {\n";
    o << "    const long long base = t * TROWS;\n";
    o << "    const int nt = (int)(n - base < TROWS ? n - base : TROWS);\n";
    for (const auto& c : fact_cols) o << "    int c_" << c << "[IPT];\n";
    o << "    if (nt == TROWS && vec_ok) {\n";
    for (size_t k = 0; k < fact_cols.size(); ++k) {
      const std::string& c = fact_cols[k];
      o << "      if ((need >> " << k << ") & 1ULL) WarpLoadTileV<IPT>(d_" << c << " + base, lane, c_" << c << ");\n";
      o << "      else { \n        #pragma unroll\n        for (int i = 0; i < IPT; ++i) c_" << c << "[i] = 0;\n      }\n";
    }
    o << "    } else {\n";
    o << "      #pragma unroll\n";
    o << "      for (int i = 0; i < IPT; ++i) {\n";
    o << "        const int r = (i / VW) * 32 * VW + lane * VW + (i % VW);\n";
    for (size_t k = 0; k < fact_cols.size(); ++k)
      o << "        c_" << fact_cols[k] << "[i] = (r < nt && ((need >> " << k << ") & 1ULL)) ? d_" << fact_cols[k] << "[base + r] : 0;\n";
    o << "      }\n";
    o << "    }\n";
    // Shapes each row may belong to after the fact filter tables.
    o << "    unsigned rel_[IPT];\n";
    o << "    #pragma unroll\n";
    o << "    for (int i = 0; i < IPT; ++i) {\n";
    o << "      const int r = (i / VW) * 32 * VW + lane * VW + (i % VW);\n";
    o << "      unsigned m = r < nt ? live : 0u;\n";
    for (int k = 0; k < NFC; ++k)
      o << "      { const unsigned d_ = (unsigned)c_" << fcols[k] << "[i] - fb" << k << "; if (d_ < fw" << k << ") m &= s_fr[" << k * FW << " + d_]; }\n";
    o << "      rel_[i] = m;\n";
    o << "    }\n";
    std::vector<unsigned> joiners(dims.size(), 0u);
    for (size_t s = 0; s < shapes.size(); ++s)
      for (const auto& kv : preds[s].joins) joiners[kv.first] |= 1u << s;
    const unsigned all_shapes = (1u << shapes.size()) - 1u;
    // Dimensions kept in shared memory first: their compact words cost no
    // gather, and the shapes they rule out skip the other dimensions' gathers.
    // Dimension by dimension over the lane's rows, so the rows' lookups are
    // independent instructions in flight together.
    for (size_t di = 0; di < dims.size(); ++di) o << "    unsigned w" << di << "_[IPT];\n";
    for (size_t di = 0; di < dims.size(); ++di) {
      const Dim& d = dims[di];
      o << "    if (a.cube_dsm[" << di << "] >= 0) {\n";
      o << "      const unsigned char* sd_ = s_dim + a.cube_dsm[" << di << "];\n";
      o << "      const int es_ = a.cube_desz[" << di << "];\n";
      o << "      #pragma unroll\n";
      o << "      for (int i = 0; i < IPT; ++i) {\n";
      // 32-bit wrap-around: o_ < dlen exactly when the key lies in [dbase, dbase + dlen).
      o << "        const unsigned o_ = (unsigned)c_" << d.fk << "[i] - (unsigned)a.cube_dbase[" << di << "];\n";
      o << "        w" << di << "_[i] = ((rel_[i] & " << joiners[di] << "u) && o_ < (unsigned)a.cube_dlen[" << di
        << "]) ? (es_ == 1 ? (unsigned)sd_[o_] : es_ == 2 ? (unsigned)((const unsigned short*)sd_)[o_] : ((const unsigned*)sd_)[o_]) : 0u;\n";
      o << "      }\n";
      o << "      #pragma unroll\n";
      // A word's shape bits are set for the shapes that do not join the
      // dimension; an absent key's word is 0 (no shape bits): OR-ing in the
      // non-joining shapes gives both cases without testing the present bit.
      o << "      for (int i = 0; i < IPT; ++i) rel_[i] &= (w" << di << "_[i] >> 1) | " << (~joiners[di] & all_shapes) << "u;\n";
      o << "    } else {\n";
      o << "      #pragma unroll\n";
      o << "      for (int i = 0; i < IPT; ++i) w" << di << "_[i] = 0u;\n";
      o << "    }\n";
    }
    // The other dimensions: their compact words gathered from global memory
    // (one word per key, no key check), or else their int4 entries; every
    // gather of the tile's rows in flight together.
    for (size_t di = 0; di < dims.size(); ++di) o << "    int4 e" << di << "_[IPT];\n";
    o << "    #pragma unroll\n";
    o << "    for (int i = 0; i < IPT; ++i) {\n";
    for (size_t di = 0; di < dims.size(); ++di) {
      const Dim& d = dims[di];
      const char* ldw = d.len * 16 <= (1LL << 20) ? "__ldg" : "__ldcg";
      o << "      if (a.cube_dsm[" << di << "] < 0 && a.cube_dgl[" << di << "] && (rel_[i] & " << joiners[di] << "u)) {\n";
      o << "        const unsigned o_ = (unsigned)c_" << d.fk << "[i] - (unsigned)a.cube_dbase[" << di << "];\n";
      o << "        if (o_ < (unsigned)a.cube_dlen[" << di << "]) {\n";
      o << "          const unsigned char* gd_ = a.cube_dcomp[" << di << "];\n";
      o << "          const int es_ = a.cube_desz[" << di << "];\n";
      o << "          w" << di << "_[i] = es_ == 1 ? (unsigned)" << ldw << "(gd_ + o_) : es_ == 2 ? (unsigned)" << ldw
        << "((const unsigned short*)gd_ + o_) : " << ldw << "((const unsigned*)gd_ + o_);\n";
      o << "        }\n";
      o << "      }\n";
      o << "      e" << di << "_[i] = make_int4(0, 0, 0, 0);\n";
      o << "      if (a.cube_dsm[" << di << "] < 0 && !a.cube_dgl[" << di << "] && (rel_[i] & " << joiners[di] << "u)) {\n";
      o << "        const int h_ = cx_detail::pht_slot<int>(c_" << d.fk << "[i], " << d.len << ", " << d.keymin << ");\n";
      // Entries of a small dimension stay in L1; a large dimension's entries
      // bypass it (L2 only), so its random gathers do not evict the small ones.
      const char* ld = d.len * 16 <= (1LL << 20) ? "__ldg" : "__ldcg";
      o << "        if (h_ >= 0) e" << di << "_[i] = " << ld << "(&ci_" << lower(d.name) << "[h_]);\n";
      o << "      }\n";
    }
    o << "    }\n";
    o << "    #pragma unroll\n";
    o << "    for (int i = 0; i < IPT; ++i) {\n";
    o << "      unsigned m = rel_[i];\n";
    for (size_t di = 0; di < dims.size(); ++di) {
      const Dim& d = dims[di];
      o << "      if (a.cube_dsm[" << di << "] < 0 && a.cube_dgl[" << di << "]) m &= (w" << di << "_[i] >> 1) | "
        << (~joiners[di] & all_shapes) << "u;\n";
      o << "      if (a.cube_dsm[" << di << "] < 0 && !a.cube_dgl[" << di << "]) {\n";
      o << "        const int4 g_ = e" << di << "_[i];\n";
      o << "        const bool hit_ = g_.x != 0 && g_.x == c_" << d.fk << "[i];\n";
      o << "        m &= hit_ ? (unsigned)g_.y : " << (~joiners[di] & all_shapes) << "u;\n";
      o << "      }\n";
    }
    o << "      if (m == 0u) continue;\n";
    const char* fld[4] = {"((unsigned)g_.z & 0xFFFFu)", "((unsigned)g_.z >> 16)", "((unsigned)g_.w & 0xFFFFu)", "((unsigned)g_.w >> 16)"};
    // The row's cell in every shape's cube (plain arithmetic, no branches),
    // then the low-word atomics of all its shared-memory cubes issued
    // together, then the carries, counts and global-cube updates: the
    // atomics' round trips overlap instead of following one another.
    std::vector<std::vector<std::string>> xs(shapes.size());
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      Emitter e(p, tu);
      for (const auto& c : fact_cols) e.col_expr[c] = "c_" + c + "[i]";
      for (const auto& ag : p.aggs)
        if (ag.fn == AggFn::Sum) xs[s].push_back("(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")");
      o << "      unsigned cl" << s << "_ = 0u;\n";
      o << "      bool h" << s << "_;\n";
      o << "      {\n";
      o << "        bool in_ = true;\n";
      for (size_t j = 0; j < sh_attrs[s].size(); ++j) {
        const int id = sh_attrs[s][j];
        const CAttr& at = cattrs[id];
        const std::string stride = "(unsigned)a.cube_stride[" + std::to_string(s * MAX_SATTRS + j) + "]";
        if (at.dim < 0) {
          o << "        { const unsigned x_ = (unsigned)(c_" << at.col << "[i] - a.cube_lo[" << id << "]);\n";
          o << "          in_ = in_ && x_ < (unsigned)a.cube_radix[" << id << "];\n";
          o << "          cl" << s << "_ += x_ * " << stride << "; }\n";
        } else {
          const std::string fi = std::to_string(at.dim * 4 + at.field);
          o << "        { const int4 g_ = e" << at.dim << "_[i];\n";
          o << "          const unsigned f_ = (a.cube_dsm[" << at.dim << "] >= 0 || a.cube_dgl[" << at.dim << "]) ? ((w" << at.dim << "_[i] >> a.cube_fsh[" << fi
            << "]) & (unsigned)a.cube_fmk[" << fi << "]) : " << fld[at.field] << ";\n";
          o << "          cl" << s << "_ += f_ * " << stride << "; }\n";
        }
      }
      // A value outside its attribute's range is reported once per thread
      // after the scan; the row updates nothing.
      o << "        const bool b_ = ((m >> " << s << ") & 1u) != 0u;\n";
      o << "        bad_ = bad_ || (b_ && !in_);\n";
      o << "        h" << s << "_ = b_ && in_;\n";
      o << "      }\n";
    }
    // Shared-memory cubes keep each sum as two 32-bit words (low word first,
    // the carry of its add going into the high word) and a 32-bit row count:
    // every update is a native 32-bit shared-memory atomic.
    for (size_t s = 0; s < shapes.size(); ++s) {
      for (size_t k = 0; k < xs[s].size(); ++k) {
        o << "      unsigned long long x" << s << "_" << k << " = 0ULL;\n";
        o << "      unsigned o" << s << "_" << k << " = 0u;\n";
      }
      o << "      if (a.cube_smem[" << s << "] >= 0) {\n";
      o << "        unsigned* cs_ = (unsigned*)(s_cube + a.cube_smem[" << s << "]);\n";
      o << "        const unsigned nc_ = (unsigned)a.cube_cells[" << s << "];\n";
      for (size_t k = 0; k < xs[s].size(); ++k) {
        o << "        x" << s << "_" << k << " = " << xs[s][k] << ";\n";
        o << "        o" << s << "_" << k << " = h" << s << "_ ? atomicAdd(&cs_[" << 2 * k << "u * nc_ + cl" << s << "_], (unsigned)x" << s << "_" << k << ") : 0u;\n";
      }
      o << "      }\n";
    }
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      const int NS = (int)xs[s].size();
      const bool counts = (int)p.aggs.size() > NS;
      o << "      if (h" << s << "_) {\n";
      o << "        if (a.cube_smem[" << s << "] >= 0) {\n";
      o << "          unsigned* cs_ = (unsigned*)(s_cube + a.cube_smem[" << s << "]);\n";
      o << "          const unsigned nc_ = (unsigned)a.cube_cells[" << s << "];\n";
      for (int k = 0; k < NS; ++k) {
        const std::string x = "x" + std::to_string(s) + "_" + std::to_string(k), ov = "o" + std::to_string(s) + "_" + std::to_string(k);
        o << "          { const unsigned lo_ = (unsigned)" << x << ";\n";
        o << "            const unsigned hi_ = (unsigned)(" << x << " >> 32) + (" << ov << " + lo_ < " << ov << " ? 1u : 0u);\n";
        o << "            if (hi_) atomicAdd(&cs_[" << 2 * k + 1 << "u * nc_ + cl" << s << "_], hi_); }\n";
      }
      // A shape without COUNT aggregates needs only whether a cell has rows:
      // a plain store of 1 instead of an atomic count.
      if (counts) o << "          atomicAdd(&cs_[" << 2 * NS << "u * nc_ + cl" << s << "_], 1u);\n";
      else o << "          cs_[" << 2 * NS << "u * nc_ + cl" << s << "_] = 1u;\n";
      o << "        } else {\n";
      o << "          unsigned long long* cg_ = a.cube_g[" << s << "];\n";
      o << "          const unsigned long long nc_ = (unsigned long long)a.cube_cells[" << s << "];\n";
      for (int k = 0; k < NS; ++k)
        o << "          { const unsigned long long x_ = " << xs[s][k] << "; if (x_) atomicAdd(&cg_[" << k << "ULL * nc_ + cl" << s << "_], x_); }\n";
      if (counts) o << "          atomicAdd(&cg_[" << NS << "ULL * nc_ + cl" << s << "_], 1ULL);\n";
      else o << "          cg_[" << NS << "ULL * nc_ + cl" << s << "_] = 1ULL;\n";
      o << "        }\n";
      o << "      }\n";
    }
    o << "    }\n";
    o << "  }\n";
    o << "  if (bad_) cx::raise(a.err, cx::ERR_CUBE_RANGE);\n";
    // Shared-memory cubes into the global cubes.
    o << "  __syncthreads();\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const int NS = sum_aggs(*shapes[s]);
      o << "  if (a.cube_smem[" << s << "] >= 0 && a.sq_num[" << s << "] > 0) {\n";
      o << "    const unsigned* cs_ = (const unsigned*)(s_cube + a.cube_smem[" << s << "]);\n";
      o << "    const unsigned nc_ = (unsigned)a.cube_cells[" << s << "];\n";
      o << "    unsigned long long* cg_ = a.cube_g[" << s << "];\n";
      o << "    for (unsigned c = threadIdx.x; c < nc_; c += " << CTA << ") {\n";
      o << "      const unsigned n_ = cs_[" << 2 * NS << "u * nc_ + c];\n";
      o << "      if (!n_) continue;\n";
      if ((int)shapes[s]->aggs.size() > NS) o << "      atomicAdd(&cg_[" << NS << "ULL * nc_ + c], (unsigned long long)n_);\n";
      else o << "      cg_[" << NS << "ULL * nc_ + c] = 1ULL;\n";
      for (int k = 0; k < NS; ++k)
        o << "      { const unsigned long long v_ = ((unsigned long long)cs_[" << 2 * k + 1 << "u * nc_ + c] << 32) | cs_["
          << 2 * k << "u * nc_ + c]; if (v_) atomicAdd(&cg_[" << k << "ULL * nc_ + c], v_); }\n";
      o << "    }\n";
      o << "  }\n";
    }
    o << "}\n\n";
    // The batch's cube layout (dimension words, strides, cube offsets and
    // sizes, attribute ranges) is read through CXS_* macros: by default the
    // kernel arguments, while the runtime recompiles this region once per
    // layout with the values as constants (-DCXS_SPEC), which folds the
    // layout's branches and multiplications away.
    std::string body = o.str();
    static const std::pair<const char*, const char*> hooks[] = {
        {"a.cube_dsm_bytes", "CXS_DSMB"}, {"a.cube_dsm[", "CXS_DSM"}, {"a.cube_desz[", "CXS_DESZ"},
        {"a.cube_dbase[", "CXS_DBASE"}, {"a.cube_dlen[", "CXS_DLEN"}, {"a.cube_fsh[", "CXS_FSH"},
        {"a.cube_fmk[", "CXS_FMK"}, {"a.cube_stride[", "CXS_STRIDE"}, {"a.cube_smem[", "CXS_SMEM"},
        {"a.cube_cells[", "CXS_CELLS"}, {"a.cube_lo[", "CXS_LO"}, {"a.cube_radix[", "CXS_RADIX"}, {"a.cube_dgl[", "CXS_DGL"},
        {"a.cube_smem_words", "CXS_SMEMW"}};
    std::set<std::string> used;
    std::string out;
    for (size_t i = 0; i < body.size();) {
      bool hit = false;
      for (const auto& h : hooks) {
        const size_t n = strlen(h.first);
        if (body.compare(i, n, h.first) != 0) continue;
        if (h.first[n - 1] == '[') {
          const size_t close = body.find(']', i + n);
          const std::string idx = body.substr(i + n, close - i - n);
          bool digits = !idx.empty();
          for (char ch : idx) digits = digits && isdigit((unsigned char)ch);
          if (!digits) continue;  // a run-time index stays an argument read
          const std::string name = std::string(h.second) + "_" + idx;
          used.insert(std::string(h.first) + idx + "]|" + name);
          out += name;
          i = close + 1;
        } else {
          used.insert(std::string(h.first) + "|" + h.second);
          out += h.second;
          i += n;
        }
        hit = true;
        break;
      }
      if (!hit) out += body[i++];
    }
    src << "//@cx-cube-begin\n#ifndef CXS_SPEC\n";
    for (const auto& u : used) {
      const size_t bar = u.find('|');
      src << "#define " << u.substr(bar + 1) << " (" << u.substr(0, bar) << ")\n";
    }
    src << "#endif\n" << out << "//@cx-cube-end\n";
  }

  // Per query: the cells of its shape's cube that its predicates accept, added
  // into its result the way the per-query path adds rows (touched bits,
  // validity), each block taking one chunk of the cells.
  void emit_cube_answer() {
    meta << "kernel cube_answer cubeans 0 256 0\n";
    std::ostringstream& o = src;
    o << "extern \"C\" __global__ void __launch_bounds__(256) cube_answer(const CxArgs a) {\n";
    o << "  const int nch = a.cube_chunks > 0 ? a.cube_chunks : 1;\n";
    o << "  const int q = blockIdx.x / nch, ch = blockIdx.x - q * nch;\n";
    o << "  if (q >= a.sq_total) return;\n";
    o << "  const CxSQ Q = a.sq[q];\n";
    o << "  const int* P = a.sparams + Q.param_off; (void)P;\n";
    o << "  unsigned long long* d_result = Q.result; (void)d_result;\n";
    o << "  uint64_t* d_result_validity = (uint64_t*)Q.validity; (void)d_result_validity;\n";
    o << "  unsigned int* g_touch = Q.touched; (void)g_touch;\n";
    o << "  switch (Q.shape) {\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      Emitter e(p, tu);
      e.lit_index = &lit_maps[s];
      for (int id : sh_attrs[s]) e.col_expr[cattrs[id].col] = "v_" + cattrs[id].col;
      const int NS = sum_aggs(p);
      o << "    case " << s << ": {\n";
      if (p.groups.empty()) {
        for (size_t k = 0; k < p.aggs.size(); ++k)
          if (p.aggs[k].fn == AggFn::Count)
            o << "      if (ch == 0 && threadIdx.x == 0) db::atomic_set_valid_bit(d_result_validity, " << k << ");\n";
      }
      o << "      const unsigned long long* cg_ = a.cube_g[" << s << "];\n";
      o << "      const long long nc_ = a.cube_cells[" << s << "];\n";
      o << "      const long long per_ = (nc_ + nch - 1) / nch, c0_ = (long long)ch * per_;\n";
      o << "      const long long c1_ = c0_ + per_ < nc_ ? c0_ + per_ : nc_;\n";
      o << "      for (long long c = c0_ + threadIdx.x; c < c1_; c += blockDim.x) {\n";
      o << "        const unsigned long long n_ = cg_[" << NS << "ULL * (unsigned long long)nc_ + c];\n";
      o << "        if (!n_) continue;\n";
      o << "        const unsigned cu_ = (unsigned)c;\n";
      // Value offsets from the cell index; an attribute with a functional
      // source (stride 0) reads its offset from the source's through its table.
      const size_t NAT = sh_attrs[s].size();
      for (size_t j = 0; j < NAT; ++j) {
        const int id = sh_attrs[s][j];
        const std::string st = "a.cube_stride[" + std::to_string(s * MAX_SATTRS + j) + "]";
        o << "        int x" << j << "_ = " << st << " > 0 ? (int)((cu_ / (unsigned)" << st << ") % (unsigned)a.cube_radix[" << id << "]) : 0;\n";
      }
      for (size_t j = 0; j < NAT; ++j) {
        const int id = sh_attrs[s][j];
        o << "        switch (a.cube_fdsrc[" << s * MAX_SATTRS + j << "]) {\n";
        for (size_t k = 0; k < NAT; ++k)
          if (k != j) o << "          case " << k << ": x" << j << "_ = a.cube_fdtab[" << id << "][x" << k << "_]; break;\n";
        o << "          default: break;\n";
        o << "        }\n";
      }
      for (size_t j = 0; j < NAT; ++j) {
        const int id = sh_attrs[s][j];
        o << "        const int v_" << cattrs[id].col << " = x" << j << "_ + a.cube_lo[" << id << "];\n";
      }
      std::vector<const Expr*> all;
      for (const auto& st : p.steps) all.push_back(st.kind == Step::Filter ? st.filter.get() : st.join.filter.get());
      o << "        if (!(" << conj_and(e, all) << ")) continue;\n";
      if (p.groups.empty()) {
        int ks = 0;
        for (size_t k = 0; k < p.aggs.size(); ++k) {
          if (p.aggs[k].fn == AggFn::Count) {
            o << "        atomicAdd(&d_result[" << k << "], n_);\n";
          } else {
            o << "        { const unsigned long long v_ = cg_[" << ks << "ULL * (unsigned long long)nc_ + c]; if (v_) atomicAdd(&d_result[" << k << "], v_); }\n";
            o << "        db::atomic_set_valid_bit(d_result_validity, " << k << ");\n";
            ++ks;
          }
        }
      } else {
        const unsigned long long G = e.total_groups();
        const int TS = p.storage_ts();
        std::string horner, dom;
        for (size_t k = 0; k < p.groups.size(); ++k) {
          o << "        const int gt" << k << " = " << e.group_term(k) << ";\n";
          horner = horner.empty() ? "gt0" : "(" + horner + " * " + std::to_string(e.eff_card(k)) + " + gt" + std::to_string(k) + ")";
          dom += (dom.empty() ? "" : " && ") + std::string("(unsigned)gt") + std::to_string(k) + " < " + std::to_string(e.eff_card(k)) + "u";
        }
        o << "        int hash = " << horner << ";\n";
        o << "        if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
        o << "        if ((unsigned)hash >= " << G << "u) continue;\n";
        o << "        atomicOr(&g_touch[hash >> 5], 1u << (hash & 31));\n";
        int ks = 0;
        for (size_t k = 0; k < p.aggs.size(); ++k) {
          const std::string ix = "(unsigned long long)hash * " + std::to_string(TS) + "ULL + " + std::to_string(p.groups.size() + k);
          if (p.aggs[k].fn == AggFn::Count) {
            o << "        atomicAdd(&d_result[" << ix << "], n_);\n";
          } else {
            o << "        { const unsigned long long v_ = cg_[" << ks << "ULL * (unsigned long long)nc_ + c]; if (v_) atomicAdd(&d_result[" << ix << "], v_); }\n";
            ++ks;
          }
          if (!p.sparse) o << "        db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
        }
      }
      o << "      }\n";
      o << "      break; }\n";
    }
    o << "    default: break;\n";
    o << "  }\n";
    o << "}\n\n";
  }

  std::string run() {
    collect();
    if (tu.cube > 0) collect_cube();
    else cube_why = "cube path switched off";
    meta << "v 1\nshared " << MAXQ << " " << MAXQ * std::max(1, max_lits) << "\n";
    for (const Dim& d : dims) {
      meta << "ht " << d.slot << " dkm_" << lower(d.name) << " " << d.len * 4 << "\n";
      if (d.attrs.size() > 1) meta << "dat " << d.slot << " " << d.len * 4 << "\n";
    }
    for (size_t k = 0; k < fcols.size(); ++k) meta << "fcol " << k << " d_" << fcols[k] << "\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      Emitter e(p, tu);
      const unsigned long long G = e.total_groups();
      const int NA = (int)p.aggs.size();
      int nseen = 0;
      for (const auto& ag : p.aggs) nseen += (ag.fn == AggFn::Sum && !p.sparse);
      const bool smem_ok = !p.groups.empty() && G * NA * 8 <= 4096ULL;
      meta << "sshape " << s << " " << G << " " << p.storage_ts() << " " << (p.groups.empty() ? 0 : 1)
           << " " << (p.sparse ? 1 : 0) << " " << lit_maps[s].size() << " " << (smem_ok ? 1 : 0) << " " << NA << " "
           << (G + 31) / 32 << " " << nseen << "\n";
    }
    if (cube_why.empty()) {
      meta << "cube " << cattrs.size() << "\n";
      for (size_t id = 0; id < cattrs.size(); ++id)
        meta << "cattr " << id << " " << cattrs[id].dim << " " << cattrs[id].field << " d_" << cattrs[id].col << "\n";
      for (size_t s = 0; s < shapes.size(); ++s) {
        meta << "cshape " << s << " " << sum_aggs(*shapes[s]) << " " << sh_attrs[s].size();
        for (int id : sh_attrs[s]) meta << " " << id;
        meta << "\n";
      }
      for (size_t di = 0; di < dims.size(); ++di)
        meta << "cdim " << di << " " << dims[di].table << " " << dims[di].len << " " << dims[di].keymin << " d_"
             << dims[di].fk << " d_" << dims[di].pk << "\n";
    }
    emit_zero();
    for (size_t di = 0; di < dims.size(); ++di) emit_index(dims[di], (int)di);
    if (cube_why.empty())
      for (size_t di = 0; di < dims.size(); ++di) emit_cube_index(dims[di], (int)di);
    emit_scan();
    if (cube_why.empty()) {
      emit_cube_scan();
      emit_cube_answer();
    }
    emit_keys();
    for (size_t i = 0; i < tables.size(); ++i) meta << "table " << i << " " << tables[i] << "\n";
    for (size_t i = 0; i < col_order.size(); ++i)
      meta << "col " << i << " d_" << col_order[i].first << " " << col_order[i].second << "\n";
    std::ostringstream out;
    out << "/*@cx-launch\n" << meta.str() << "@*/\n";
    out << "// Generated by crystal-b200 for sm_100a (shared scan).\n";
    out << "#include \"cx_args.h\"\n#include \"crystal_sm100.cuh\"\n\n";
    out << "template <typename A, typename B>\n"
           "__device__ __forceinline__ auto cx_mdiv(A x, B y) -> decltype(x / y) {\n"
           "  return (y == 0) ? (decltype(x / y))0 : x / y;\n}\n";
    out << "//@cx-prelude-end\n\n";
    out << src.str();
    return out.str();
  }

  // CTA-tiled shared scan.  Per tile of TR = block x items rows: thread 0
  // stages the union of fact columns by TMA bulk copies; every thread builds
  // the query masks of its rows (filter tables, one gather per dimension,
  // residual filters) and stores them with the payload attributes in shared
  // memory; then warps take (query, row slice) units and aggregate the rows
  // whose mask bit is set.
  void emit_scan() {
    const int CTA = tu.block_threads, IPT = tu.items_per_thread;
    if (CTA % 32 || CTA < 64 || CTA > 1024 || IPT < 1 || IPT > 16) throw PlanError("bad block shape");
    const int NW = CTA / 32, TR = CTA * IPT;
    if (NW < 3) throw PlanError("shared scan needs at least 3 warps (staging, masks, aggregation)");
    // Warp roles: warp 0 stages tiles, NPW warps build masks, the rest aggregate.
    const int NPW = tu.producer_warps > 0 ? std::min(tu.producer_warps, NW - 2) : std::max(1, (NW - 1) * 3 / 8);
    const int NCW = NW - 1 - NPW;
    const int NSC = (int)fact_cols.size();
    int STAGES = std::max(2, tu.stages);
    const int MAXP = MAXQ * std::max(1, max_lits);
    const int NACC = std::max(1, max_scalar_aggs) * 2;  // (sum, count) per scalar aggregate
    const int NFC = (int)fcols.size();
    int nattr = 0;
    std::map<std::string, int> attr_slot;
    for (const Dim& d : dims)
      for (const auto& at : d.attrs) attr_slot[at] = nattr++;
    // Shapes with a small group domain and literal-free group keys get per-group
    // row bitmaps (plus one word of out-of-domain rows) built with the masks.
    std::vector<int> gm_base(shapes.size(), -1);
    int gm_words = 0;
    for (size_t si = 0; si < shapes.size(); ++si) {
      const Plan& p = *shapes[si];
      if (p.groups.empty() || tu.group_merge == 2) continue;
      Emitter e(p, tu);
      const unsigned long long G = e.total_groups();
      std::vector<const Expr*> gl;
      for (const auto& g : p.groups) lits_of(g.expr.get(), gl);
      if (G <= 31 && G * p.aggs.size() <= 16 && gl.empty()) {
        gm_base[si] = gm_words;
        gm_words += (int)G + 1;
      }
    }
    // Fewer stages when the ring would not leave room for the rest.
    while (STAGES > 2 && (unsigned long long)STAGES * ((unsigned long long)(NSC + nattr) * TR * 4 + (MAXQ + gm_words) * (TR / 32) * 4) > 160 * 1024) --STAGES;
    unsigned long long off = 0;
    const int NB = TR / 32;  // 32-row blocks per tile
    // Row stride of a query's (or a group's) block words: one word of padding,
    // so the 32 lanes of a mask warp, each storing the word of its own query
    // for the same block, hit 32 different banks.
    const int NBS = NB + 1;
    // Per stage: the fact columns, the payload attributes and the per-query row bitmaps of one tile.
    const unsigned long long stage_off = off; off += (unsigned long long)STAGES * NSC * TR * 4;
    const unsigned long long attr_off = off; off += (unsigned long long)STAGES * nattr * TR * 4;
    const unsigned long long gm_off = off; off += (unsigned long long)STAGES * gm_words * NBS * 4;
    const unsigned long long bars_off = off; off += (unsigned long long)STAGES * 3 * 8 + 16;
    off = (off + 15) & ~15ULL;
    const unsigned long long par_off = off; off += (unsigned long long)MAXP * 4;
    off = (off + 15) & ~15ULL;
    const unsigned long long acc_off = off; off += (unsigned long long)MAXQ * NACC * 8;
    const unsigned long long sq_off = off; off += ((unsigned long long)MAXQ * sizeof(CxSQ) + 15) & ~15ULL;
    const unsigned long long fm_off = off; off += (unsigned long long)NFC * FW * 8;
    const unsigned long long nj_off = off; off += (unsigned long long)(dims.size() + 4) * 8;
    off = (off + 15) & ~15ULL;
    // The per-query row bitmaps (STAGES x NB words per query of the pass) and
    // the group tables follow the fixed part; the host sizes both per pass.
    const unsigned long long qb_off = (off + 15) & ~15ULL;
    const unsigned long long smem_total = qb_off;
    if (smem_total + (unsigned long long)MAXQ * STAGES * NBS * 4 > 200 * 1024)
      throw PlanError("shared scan shared memory exceeds 200 KB before group tables");
    meta << "sqb " << STAGES * NBS * 4 << "\n";
    const unsigned wait_limit = (unsigned)std::min(60000000, std::max(1, tu.wait_limit_us));
    const std::string kname = "SharedScan_" + fact;
    meta << "kernel " << kname << " sharedscan 0 " << CTA << " " << TR << " " << smem_total << " " << tu.ctas_per_sm << "\n";

    std::ostringstream& o = src;
    // At least 32 resident warps per SM: registers are capped at 64.
    o << "extern \"C\" __global__ void __launch_bounds__(" << CTA << ", " << std::max(1, 1024 / CTA) << ") " << kname << "(const CxArgs a) {\n";
    o << "  constexpr int TR = " << TR << ", NSTAGE = " << STAGES << ", NSC = " << NSC << ", NPW = " << NPW << ", NCW = " << NCW << ";\n";
    o << "  extern __shared__ __align__(1024) unsigned char cx_smem[];\n";
    if (tu.debug_stall)
      o << "  { cx::debug_stall((unsigned long long*)cx_smem, a.err, " << wait_limit << "u); return; }\n";
    o << "  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n";
    o << "  int* stage_buf = (int*)(cx_smem + " << stage_off << ");\n";
    o << "  int* s_attr = (int*)(cx_smem + " << attr_off << "); (void)s_attr;\n";
    o << "  unsigned* s_qb = (unsigned*)(cx_smem + " << qb_off << ");  // [stage][query][32-row block] row bitmaps\n";
    o << "  const int nq_ = a.sq_total < " << MAXQ << " ? a.sq_total : " << MAXQ << ";\n";
    o << "  unsigned* s_gm = (unsigned*)(cx_smem + " << gm_off << "); (void)s_gm;  // [stage][shape group][32-row block]\n";
    o << "  unsigned long long* bar_full = (unsigned long long*)(cx_smem + " << bars_off << ");   // tile staged\n";
    o << "  unsigned long long* bar_ready = bar_full + NSTAGE;   // masks built\n";
    o << "  unsigned long long* bar_empty = bar_full + 2 * NSTAGE;  // aggregation done\n";
    o << "  volatile int* s_abort = (volatile int*)(bar_full + 3 * NSTAGE);\n";
    o << "  int* s_nissued = (int*)(bar_full + 3 * NSTAGE) + 1;\n";
    o << "  int* s_params = (int*)(cx_smem + " << par_off << ");\n";
    o << "  unsigned long long* s_qacc = (unsigned long long*)(cx_smem + " << acc_off << ");\n";
    o << "  CxSQ* s_sq = (CxSQ*)(cx_smem + " << sq_off << ");\n";
    o << "  unsigned long long* s_fm = (unsigned long long*)(cx_smem + " << fm_off << "); (void)s_fm;\n";
    o << "  unsigned long long* s_nj = (unsigned long long*)(cx_smem + " << nj_off << ");\n";
    o << "  unsigned long long* s_tab = (unsigned long long*)(cx_smem + " << qb_off << " + ((NSTAGE * nq_ * " << NBS * 4 << " + 15) & ~15)); (void)s_tab;\n";
    o << "  unsigned int* s_bits = (unsigned int*)(s_tab + a.smem_tab_words); (void)s_bits;\n";
    o << "  const int nq = a.sq_total < " << MAXQ << " ? a.sq_total : " << MAXQ << ";\n";
    o << "  const long long n_rows = a.rows[0];\n";
    o << "  const long long num_tiles = (n_rows + TR - 1) / TR;\n";
    o << "  const long long full_tiles = n_rows / TR;\n";
    o << "  for (int w = threadIdx.x; w < nq; w += " << CTA << ") s_sq[w] = a.sq[w];\n";
    o << "  for (int w = threadIdx.x; w < a.nparams && w < " << MAXP << "; w += " << CTA << ") s_params[w] = a.sparams[w];\n";
    o << "  for (int w = threadIdx.x; w < " << MAXQ * NACC << "; w += " << CTA << ") s_qacc[w] = 0ULL;\n";
    o << "  for (int w = threadIdx.x; w < a.smem_tab_words; w += " << CTA << ") s_tab[w] = 0ULL;\n";
    o << "  for (int w = threadIdx.x; w < a.smem_bit_words; w += " << CTA << ") s_bits[w] = 0u;\n";
    o << "  __syncthreads();\n";
    // Filter tables: bit q of s_fm[k * FW + v] clears when query q's conjuncts
    // on filter column k reject the value fbase[k] + v.
    if (NFC) {
      o << "  for (int v = threadIdx.x; v < " << NFC * FW << "; v += " << CTA << ") {\n";
      o << "    const int k_ = v / " << FW << ";\n";
      o << "    const int fv_ = (int)((unsigned)a.fbase[k_] + (unsigned)(v - k_ * " << FW << "));\n";
      o << "    unsigned long long m = ~0ULL;\n";
      o << "    for (int q = 0; q < nq; ++q) {\n";
      o << "      const int* P = s_params + s_sq[q].param_off; (void)P;\n";
      o << "      bool pass = true;\n";
      o << "      switch (s_sq[q].shape) {\n";
      for (size_t s = 0; s < shapes.size(); ++s) {
        if (preds[s].pushed.empty()) continue;
        Emitter e(*shapes[s], tu);
        e.lit_index = &lit_maps[s];
        o << "        case " << s << ":\n";
        for (const auto& kv : preds[s].pushed) {
          e.col_expr.clear();
          e.col_expr[fcols[kv.first]] = "fv_";
          o << "          if (k_ == " << kv.first << ") pass = " << conj_and(e, kv.second) << ";\n";
        }
        o << "          break;\n";
      }
      o << "        default: break;\n";
      o << "      }\n";
      o << "      if (!pass) m &= ~(1ULL << q);\n";
      o << "    }\n";
      o << "    s_fm[v] = m;\n";
      o << "  }\n";
    }
    // Fact columns each shape reads (bits over the staged columns).
    if (NSC > 64) throw PlanError("more than 64 fact columns in a shared batch");
    const std::vector<unsigned long long> colmask = shape_colmasks();
    // Masks of the queries that skip each dimension, that carry residual
    // filters, that have filter-table conjuncts, and of the whole batch; and
    // the fact columns the batch reads.
    {
      std::vector<unsigned> joins(shapes.size(), 0u);
      std::vector<int> has_res(shapes.size(), 0), has_push(shapes.size(), 0);
      for (size_t s = 0; s < shapes.size(); ++s) {
        for (const auto& kv : preds[s].joins) joins[s] |= 1u << kv.first;
        has_res[s] = !preds[s].resid.empty();
        has_push[s] = !preds[s].pushed.empty();
      }
      o << "  if (threadIdx.x < " << dims.size() + 4 << ") {\n";
      o << "    const int t_ = threadIdx.x;\n";
      o << "    unsigned long long m = 0ULL;\n";
      o << "    for (int q = 0; q < nq; ++q) {\n";
      o << "      unsigned j_ = 0u; int r_ = 0, p_ = 0; unsigned long long c_ = 0ULL;\n";
      o << "      switch (s_sq[q].shape) {\n";
      for (size_t s = 0; s < shapes.size(); ++s)
        o << "        case " << s << ": j_ = " << joins[s] << "u; r_ = " << has_res[s] << "; p_ = " << has_push[s]
          << "; c_ = " << colmask[s] << "ULL; break;\n";
      o << "        default: break;\n";
      o << "      }\n";
      o << "      bool b_ = false;\n";
      o << "      if (t_ < " << dims.size() << ") b_ = !((j_ >> t_) & 1u);\n";
      o << "      else if (t_ == " << dims.size() << ") b_ = r_ != 0;\n";
      o << "      else if (t_ == " << dims.size() + 1 << ") b_ = p_ != 0;\n";
      o << "      else b_ = true;\n";
      o << "      if (t_ == " << dims.size() + 3 << ") m |= c_;\n";
      o << "      else if (b_) m |= 1ULL << q;\n";
      o << "    }\n";
      o << "    s_nj[t_] = m;\n";
      o << "  }\n";
    }
    for (const auto& c : fact_cols) o << "  const int* __restrict__ d_" << c << " = a.col[" << slot_of(c, 0) << "];\n";
    for (const Dim& d : dims) {
      o << "  const int4* __restrict__ dkm_" << lower(d.name) << " = (const int4*)a.ht[" << d.slot << "];\n";
      if (d.attrs.size() > 1) o << "  const int4* __restrict__ dat_" << lower(d.name) << " = (const int4*)a.dat[" << d.slot << "];\n";
    }
    for (int k = 0; k < NFC; ++k) o << "  const unsigned fb" << k << " = (unsigned)a.fbase[" << k << "], fw" << k << " = (unsigned)a.fwin[" << k << "];\n";
    o << "  bool staged_ok = true;\n";
    for (const auto& c : fact_cols) o << "  staged_ok = staged_ok && ((((unsigned long long)d_" << c << ") & 15ULL) == 0ULL);\n";
    o << "  unsigned long long l2_policy = 0;\n";
    o << "  if (threadIdx.x == 0) {\n";
    o << "    for (int s = 0; s < NSTAGE; ++s) {\n";
    o << "      cx::mbar_init(&bar_full[s], 1);\n";
    o << "      cx::mbar_init(&bar_ready[s], NPW);\n";
    o << "      cx::mbar_init(&bar_empty[s], NCW);\n";
    o << "    }\n";
    o << "    *s_abort = 0;\n";
    o << "    *s_nissued = 0;\n";
    o << "    cx::fence_mbar_init();\n";
    o << "    l2_policy = cx::l2_evict_first_policy();\n";
    o << "  }\n";
    // Only the columns the batch's shapes read are staged.
    o << "#define CX_ISSUE(TILE_, STAGE_) do { \\\n";
    o << "    cx::mbar_expect_tx(&bar_full[(STAGE_)], stage_tx); \\\n";
    for (int c = 0; c < NSC; ++c)
      o << "    if ((m_cols >> " << c << ") & 1ULL) cx::bulk_g2s(stage_buf + ((STAGE_) * NSC + " << c << ") * TR, d_" << fact_cols[c]
        << " + (TILE_) * TR, " << TR * 4 << "u, &bar_full[(STAGE_)], l2_policy); \\\n";
    o << "  } while (0)\n";
    o << "  __syncthreads();\n";
    o << "  const unsigned long long m_res = s_nj[" << dims.size() << "], m_push = s_nj[" << dims.size() + 1
      << "], m_all = s_nj[" << dims.size() + 2 << "];\n";
    o << "  (void)m_res; (void)m_push;\n";
    o << "  const unsigned long long m_cols = s_nj[" << dims.size() + 3 << "];\n";
    o << "  const unsigned stage_tx = (unsigned)__popcll(m_cols) * (unsigned)(TR * 4);\n";
    o << "  (void)stage_tx;\n";
    // Enough (query, slice) units to occupy the aggregation warps, but no
    // slice under 8 blocks: a small batch leaves warps idle rather than pay a
    // flush per sliver.
    o << "  const int slices = nq > 0 ? max(1, min((NCW + nq - 1) / nq, " << std::max(1, NB / 8) << ")) : 1;\n";
    o << "  const int units = nq * slices;\n";
    const std::string LIM = std::to_string(wait_limit) + "u";
    // Per-tile views of one stage.
    auto tile_ptrs = [&](const std::string& ind) {
      o << ind << "const long long tile_offset = t * TR;\n";
      o << ind << "const int n_tile = (int)(n_rows - tile_offset < TR ? n_rows - tile_offset : TR);\n";
      o << ind << "const int nblk = (n_tile + 31) >> 5;\n";
      o << ind << "int* tile = stage_buf + s * NSC * TR;\n";
      for (int c = 0; c < NSC; ++c) o << ind << "const int* S_" << fact_cols[c] << " = tile + " << c << " * TR;\n";
      for (const Dim& d : dims)
        for (const auto& at : d.attrs)
          o << ind << "int* S_" << at << " = s_attr + (s * " << nattr << " + " << attr_slot[at] << ") * TR;\n";
      o << ind << "unsigned* s_qb_t = s_qb + s * nq * " << NBS << ";\n";
      o << ind << "unsigned* s_gm_t = s_gm + s * " << gm_words * NBS << "; (void)s_gm_t;\n";
    };
    // Staging warp: refills a stage once the aggregation warps released it.
    o << "  if (warp == 0) {\n";
    o << "    if (lane == 0) {\n";
    o << "      long long k = 0;\n";
    o << "      for (long long t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {\n";
    o << "        const int s = (int)(k % NSTAGE);\n";
    o << "        if (k >= NSTAGE && !cx::mbar_wait_bounded(&bar_empty[s], (unsigned)(((k / NSTAGE) - 1) & 1), " << LIM << ")) {\n";
    o << "          cx::raise(a.err, cx::ERR_WAIT_TIMEOUT);\n";
    o << "          *s_abort = 1;\n";
    o << "          break;\n";
    o << "        }\n";
    o << "        if (*s_abort) break;\n";
    o << "        cx::fence_proxy_async_smem();\n";
    o << "        if (staged_ok && t < full_tiles) CX_ISSUE(t, s); else cx::mbar_arrive(&bar_full[s]);\n";
    o << "        *s_nissued = (int)(k + 1);\n";
    o << "      }\n";
    o << "    }\n";
    // Mask warps.
    o << "  } else if (warp <= NPW) {\n";
    o << "    const int pw = warp - 1;\n";
    o << "    long long k = 0;\n";
    o << "    for (long long t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {\n";
    o << "      const int s = (int)(k % NSTAGE);\n";
    o << "      const bool ok_ = cx::mbar_wait_bounded(&bar_full[s], (unsigned)((k / NSTAGE) & 1), " << LIM << ");\n";
    o << "      if (__any_sync(0xffffffffu, !ok_)) { if (lane == 0) { cx::raise(a.err, cx::ERR_WAIT_TIMEOUT); *s_abort = 1; } break; }\n";
    o << "      if (__any_sync(0xffffffffu, *s_abort != 0)) break;\n";
    tile_ptrs("      ");
    o << "      const bool staged = staged_ok && t < full_tiles;\n";
    // Phase A: query masks of the tile's rows, RB rows per thread with every
    // dimension gather of those rows in flight together.
    const int RB = dims.size() <= 2 ? std::min(IPT, 2) : 1;  // 64 registers hold 8 gathered entries
    o << "    for (int b0_ = pw; b0_ < nblk; b0_ += " << NPW * RB << ") {\n";
    // Ragged last tile (or unaligned columns): each mask warp loads the rows of its own blocks.
    o << "      if (!staged) {\n";
    o << "        for (int j = 0; j < " << RB << "; ++j) {\n";
    o << "          const int r = ((b0_ + j * NPW) << 5) + lane;\n";
    o << "          if (r >= n_tile) continue;\n";
    for (int c = 0; c < NSC; ++c) o << "          tile[" << c << " * TR + r] = d_" << fact_cols[c] << "[tile_offset + r];\n";
    o << "        }\n";
    o << "        __syncwarp();\n";
    o << "      }\n";
    o << "      unsigned long long mk_[" << RB << "];\n";
    o << "      bool ow_[" << RB << "];\n";
    o << "      #pragma unroll\n";
    o << "      for (int j = 0; j < " << RB << "; ++j) {\n";
    o << "        const int i = ((b0_ + j * NPW) << 5) + lane;\n";
    o << "        mk_[j] = 0ULL;\n";
    o << "        ow_[j] = false;\n";
    o << "        if (i < n_tile) {\n";
    o << "          unsigned long long m = m_all;\n";
    for (int k = 0; k < NFC; ++k) {
      const int ck = (int)(std::find(fact_cols.begin(), fact_cols.end(), fcols[k]) - fact_cols.begin());
      o << "          if ((m_cols >> " << ck << ") & 1ULL) { const unsigned d_ = (unsigned)S_" << fcols[k] << "[i] - fb" << k << ";\n";
      o << "            if (d_ < fw" << k << ") m &= s_fm[" << k * FW << " + d_]; else ow_[j] = true; }\n";
    }
    o << "          mk_[j] = m;\n";
    o << "        }\n";
    o << "      }\n";
    for (size_t di = 0; di < dims.size(); ++di) o << "      int4 g" << di << "_[" << RB << "];\n";
    for (size_t di = 0; di < dims.size(); ++di) o << "      int k" << di << "_[" << RB << "];\n";
    o << "      #pragma unroll\n";
    o << "      for (int j = 0; j < " << RB << "; ++j) {\n";
    o << "        const int i = ((b0_ + j * NPW) << 5) + lane;\n";
    o << "        const bool live_ = i < n_tile && mk_[j] != 0ULL;\n";
    for (size_t di = 0; di < dims.size(); ++di) {
      const Dim& d = dims[di];
      o << "        {\n";
      o << "          g" << di << "_[j] = make_int4(0, 0, 0, 0);\n";
      o << "          const int fk_ = live_ ? S_" << d.fk << "[i] : 0;\n";
      o << "          k" << di << "_[j] = fk_;\n";
      o << "          const int h_ = cx_detail::pht_slot<int>(fk_, " << d.len << ", " << d.keymin << ");\n";
      o << "          if (live_ && h_ >= 0) g" << di << "_[j] = __ldg(&dkm_" << lower(d.name) << "[h_]);\n";
      o << "        }\n";
    }
    o << "      }\n";
    o << "      #pragma unroll\n";
    o << "      for (int j = 0; j < " << RB << "; ++j) {\n";
    o << "        const int i = ((b0_ + j * NPW) << 5) + lane;\n";
    o << "        if (b0_ + j * NPW >= nblk) break;  // warp-uniform: a block is one warp's 32 rows\n";
    o << "        unsigned long long m = mk_[j];\n";
    o << "        const bool oow = ow_[j]; (void)oow;\n";
    o << "        if (m != 0ULL) {\n";
    const char* comp[] = {"x", "y", "z"};
    for (size_t di = 0; di < dims.size(); ++di) {
      const Dim& d = dims[di];
      const std::string dn = lower(d.name);
      o << "          {\n";
      o << "            const int4 g_ = g" << di << "_[j];\n";
      o << "            const bool hit_ = g_.x != 0 && g_.x == k" << di << "_[j];\n";
      o << "            m &= hit_ ? (((unsigned long long)(unsigned)g_.z << 32) | (unsigned)g_.y) : s_nj[" << di << "];\n";
      if (!d.attrs.empty()) o << "            S_" << d.attrs[0] << "[i] = g_.w;\n";
      if (d.attrs.size() > 1) {
        o << "            int4 a_ = make_int4(0, 0, 0, 0);\n";
        o << "            if (hit_) a_ = __ldg(&dat_" << dn << "[cx_detail::pht_slot<int>(k" << di << "_[j], " << d.len << ", " << d.keymin << ")]);\n";
        for (size_t k = 1; k < d.attrs.size(); ++k) o << "            S_" << d.attrs[k] << "[i] = a_." << comp[k - 1] << ";\n";
      }
      o << "          }\n";
    }
    // Residual filters (and filter-table conjuncts of values outside the window).
    bool any_slow = false;
    for (size_t s = 0; s < shapes.size(); ++s) any_slow = any_slow || !preds[s].resid.empty() || !preds[s].pushed.empty();
    if (any_slow) {
      o << "        unsigned long long r_ = m & (m_res | (oow ? m_push : 0ULL));\n";
      o << "        while (r_) {\n";
      o << "          const int q = __ffsll((long long)r_) - 1;\n";
      o << "          r_ &= r_ - 1ULL;\n";
      o << "          const int* P = s_params + s_sq[q].param_off; (void)P;\n";
      o << "          bool pass = true;\n";
      o << "          switch (s_sq[q].shape) {\n";
      for (size_t s = 0; s < shapes.size(); ++s) {
        if (preds[s].resid.empty() && preds[s].pushed.empty()) continue;
        Emitter e(*shapes[s], tu);
        e.lit_index = &lit_maps[s];
        for (const auto& c : fact_cols) e.col_expr[c] = "S_" + c + "[i]";
        for (const auto& kv : attr_slot) e.col_expr[kv.first] = "S_" + kv.first + "[i]";
        std::vector<const Expr*> all_pushed;
        for (const auto& kv : preds[s].pushed) all_pushed.insert(all_pushed.end(), kv.second.begin(), kv.second.end());
        o << "            case " << s << ": pass = (" << conj_and(e, preds[s].resid) << ") && (!oow || (" << conj_and(e, all_pushed) << ")); break;\n";
      }
      o << "            default: break;\n";
      o << "          }\n";
      o << "          if (!pass) m &= ~(1ULL << q);\n";
      o << "        }\n";
    }
    o << "        }\n";
    o << "        const int blk_ = i >> 5;\n";
    for (size_t si = 0; si < shapes.size(); ++si) {
      if (gm_base[si] < 0) continue;
      const Plan& p = *shapes[si];
      Emitter e(p, tu);
      for (const auto& c : fact_cols) e.col_expr[c] = "S_" + c + "[i]";
      for (const auto& kv : attr_slot) e.col_expr[kv.first] = "S_" + kv.first + "[i]";
      const unsigned long long G = e.total_groups();
      std::string horner, dom;
      o << "        {  // group rows of shape " << si << "\n";
      o << "          int h_ = " << G << ";\n";
      o << "          bool bad_ = false;\n";
      o << "          if (m != 0ULL) {\n";
      for (size_t k = 0; k < p.groups.size(); ++k) {
        o << "            const int gt" << k << " = " << e.group_term(k) << ";\n";
        horner = horner.empty() ? "gt0" : "(" + horner + " * " + std::to_string(e.eff_card(k)) + " + gt" + std::to_string(k) + ")";
        dom += (dom.empty() ? "" : " && ") + std::string("(unsigned)gt") + std::to_string(k) + " < " + std::to_string(e.eff_card(k)) + "u";
      }
      o << "            bad_ = !(" << dom << ");\n";
      o << "            const int hash = bad_ ? (" << horner << ") % " << G << " : (" << horner << ");\n";
      o << "            h_ = (unsigned)hash < " << G << "u ? hash : " << G << ";\n";
      o << "          }\n";
      // One match over the lanes gives every group's row word at once: the
      // block's words are cleared, then the lowest lane of each group writes
      // its group's word (the same lane writes the out-of-domain word).
      const std::string gm_at = "s_gm_t[(" + std::to_string(gm_base[si]) + " + ";
      o << "          if (lane <= " << G << ") " << gm_at << "lane) * " << NBS << " + blk_] = 0u;\n";
      o << "          __syncwarp();\n";
      o << "          const unsigned peers_ = __match_any_sync(0xffffffffu, h_);\n";
      o << "          if (h_ < " << G << " && lane == __ffs(peers_) - 1) " << gm_at << "h_) * " << NBS << " + blk_] = peers_;\n";
      o << "          const unsigned bb_ = __ballot_sync(0xffffffffu, bad_);\n";
      o << "          if (lane == " << G << ") " << gm_at << G << ") * " << NBS << " + blk_] = bb_;\n";
      o << "        }\n";
    }
    // Transpose the warp's 32 row masks into one word per query.
    o << "        const unsigned wl_ = cx::warp_transpose32((unsigned)m, lane);\n";
    o << "        if (lane < nq) s_qb_t[lane * " << NBS << " + blk_] = wl_;\n";
    o << "        if (nq > 32) {\n";
    o << "          const unsigned wh_ = cx::warp_transpose32((unsigned)(m >> 32), lane);\n";
    o << "          if (lane + 32 < nq) s_qb_t[(lane + 32) * " << NBS << " + blk_] = wh_;\n";
    o << "        }\n";
    o << "      }\n";
    o << "    }\n";
    o << "    __syncwarp();\n";
    o << "    if (lane == 0) cx::mbar_arrive(&bar_ready[s]);\n";
    o << "    }\n";
    // Aggregation warps: query units aggregate the rows whose bit is set.
    o << "  } else {\n";
    o << "    const int cw = warp - 1 - NPW;\n";
    o << "    long long k = 0;\n";
    o << "    for (long long t = blockIdx.x; t < num_tiles; t += gridDim.x, ++k) {\n";
    o << "      const int s = (int)(k % NSTAGE);\n";
    o << "      const bool ok_ = cx::mbar_wait_bounded(&bar_ready[s], (unsigned)((k / NSTAGE) & 1), " << LIM << ");\n";
    o << "      if (__any_sync(0xffffffffu, !ok_)) { if (lane == 0) { cx::raise(a.err, cx::ERR_WAIT_TIMEOUT); *s_abort = 1; } break; }\n";
    o << "      if (__any_sync(0xffffffffu, *s_abort != 0)) break;\n";
    tile_ptrs("      ");
    o << "    for (int u = cw; u < units; u += NCW) {\n";
    o << "      const int q_ = u / slices, sl_ = u - q_ * slices;\n";
    o << "      const int perb_ = (nblk + slices - 1) / slices;\n";
    o << "      const int blo_ = sl_ * perb_, bhi_ = blo_ + perb_ < nblk ? blo_ + perb_ : nblk;\n";
    // Fewer blocks than lanes: lanes share a block, each taking a bit range of its word.
    o << "      const int lpb_ = perb_ >= 32 ? 1 : perb_ >= 16 ? 2 : perb_ >= 8 ? 4 : perb_ >= 4 ? 8 : perb_ >= 2 ? 16 : 32;\n";
    o << "      const int bw_ = 32 / lpb_, sub_ = lane % lpb_;\n";
    o << "      const unsigned bm_ = (bw_ == 32 ? 0xffffffffu : ((1u << bw_) - 1u)) << (sub_ * bw_);\n";
    o << "      const CxSQ& Q = s_sq[q_];\n";
    o << "      const int* P = s_params + Q.param_off; (void)P;\n";
    o << "      const unsigned* qw_ = s_qb_t + q_ * " << NBS << ";\n";
    o << "      switch (Q.shape) {\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      Emitter e(p, tu);
      e.lit_index = &lit_maps[s];
      const std::string ind = "          ";
      o << "      case " << s << ": {\n";
      const int NA = (int)p.aggs.size();
      const int TS = p.storage_ts();
      std::vector<std::string> need;
      for (const auto& g : p.groups) cols_of(g.expr.get(), need);
      for (const auto& ag : p.aggs) cols_of(ag.arg.get(), need);
      // Parameters of group and aggregate expressions in registers.
      {
        std::vector<const Expr*> ls;
        for (const auto& g : p.groups) lits_of(g.expr.get(), ls);
        for (const auto& ag : p.aggs) lits_of(ag.arg.get(), ls);
        std::set<int> ks;
        for (const Expr* l : ls) ks.insert(lit_maps[s].at(l));
        for (int k : ks) o << ind << "const int P" << k << " = P[" << k << "];\n";
      }
      e.param_regs = true;
      for (const auto& c : need) e.col_expr[c] = "S_" + c + "[i]";
      // Each lane walks the set bits of its 32-row blocks.
      std::string loop_open = ind + "for (int b_ = blo_ + lane / lpb_; b_ < bhi_; b_ += 32 / lpb_) {\n";
      loop_open += ind + "  unsigned w_ = qw_[b_] & bm_;\n";
      loop_open += ind + "  while (w_) {\n";
      loop_open += ind + "  const int i = (b_ << 5) + __ffs(w_) - 1;\n";
      loop_open += ind + "  w_ &= w_ - 1u;\n";
      const std::string loop_close = ind + "  }\n" + ind + "}\n";
      if (p.groups.empty()) {
        for (int k = 0; k < NA; ++k) o << ind << "unsigned long long s" << k << "_ = 0ULL, c" << k << "_ = 0ULL;\n";
        o << loop_open;
        for (int k = 0; k < NA; ++k) {
          const Agg& ag = p.aggs[k];
          const std::string x = ag.fn == AggFn::Count ? "1ULL" : e.math_push(ag.arg.get(), true);
          o << ind << "  s" << k << "_ += " << x << "; c" << k << "_ += 1ULL;\n";
        }
        o << loop_close;
        for (int k = 0; k < NA; ++k) {
          o << ind << "if (__any_sync(0xffffffffu, c" << k << "_ != 0ULL)) {\n";
          o << ind << "  for (int o_ = 16; o_ > 0; o_ >>= 1) { s" << k << "_ += __shfl_xor_sync(0xffffffffu, s" << k << "_, o_); c" << k << "_ += __shfl_xor_sync(0xffffffffu, c" << k << "_, o_); }\n";
          o << ind << "  if (lane == 0) { atomicAdd(&s_qacc[(long long)q_ * " << NACC << " + " << 2 * k << "], s" << k << "_); atomicAdd(&s_qacc[(long long)q_ * " << NACC << " + " << 2 * k + 1 << "], c" << k << "_); }\n";
          o << ind << "}\n";
        }
      } else {
        const unsigned long long G = e.total_groups();
        const unsigned long long TWq = (G + 31) / 32;
        std::string horner, dom;
        std::ostringstream terms;
        for (size_t k = 0; k < p.groups.size(); ++k) {
          terms << ind << "  const int gt" << k << " = " << e.group_term(k) << ";\n";
          horner = horner.empty() ? "gt0" : "(" + horner + " * " + std::to_string(e.eff_card(k)) + " + gt" + std::to_string(k) + ")";
          dom += (dom.empty() ? "" : " && ") + std::string("(unsigned)gt") + std::to_string(k) + " < " + std::to_string(e.eff_card(k)) + "u";
        }
        o << ind << "unsigned long long* d_result = Q.result; (void)d_result;\n";
        o << ind << "uint64_t* d_result_validity = (uint64_t*)Q.validity; (void)d_result_validity;\n";
        o << ind << "unsigned int* g_touch = Q.touched; (void)g_touch;\n";
        o << ind << "unsigned long long* qtab = Q.smem_acc >= 0 ? s_tab + Q.smem_acc : nullptr; (void)qtab;\n";
        o << ind << "unsigned int* qbits = s_bits + (Q.smem_acc >= 0 ? Q.smem_bits : 0); (void)qbits;\n";
        // Flush of a unit's register partials: one reduce-scatter of all G x NA
        // values; the lanes that end up holding a total apply it.
        auto tiny_flush = [&]() {
          int P2 = 1;
          while (P2 < (int)(G * NA)) P2 <<= 1;
          o << ind << "ttouch = __reduce_or_sync(0xffffffffu, ttouch);\n";
          for (int k = 0; k < NA; ++k)
            if (!p.sparse && p.aggs[k].fn == AggFn::Sum) o << ind << "tseen" << k << " = __reduce_or_sync(0xffffffffu, tseen" << k << ");\n";
          o << ind << "if (ttouch) {\n";
          o << ind << "  unsigned long long rv_[" << P2 << "];\n";
          o << ind << "  #pragma unroll\n" << ind << "  for (int r = 0; r < " << P2 << "; ++r) rv_[r] = r < " << G * NA << " ? tacc[r < " << G * NA << " ? r : 0] : 0ULL;\n";
          o << ind << "  const int ri_ = cx::warp_reduce_scatter_u64<" << P2 << ">(rv_, lane);\n";
          o << ind << "  const int g = ri_ / " << NA << ", k_ = ri_ - g * " << NA << "; (void)k_;\n";
          o << ind << "  if ((lane & " << (32 / P2 - 1) << ") == 0 && ri_ < " << G * NA << " && ((ttouch >> g) & 1u)) {\n";
          o << ind << "    const unsigned long long s_ = rv_[0];\n";
          int sk = 0;
          for (int k = 0; k < NA; ++k) {
            const int slot = (int)p.groups.size() + k;
            const std::string ix = "(unsigned long long)g * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
            o << ind << "    if (k_ == " << k << ") {\n";
            o << ind << "      if (qtab) { if (s_) atomicAdd(&qtab[ri_], s_); }\n";
            o << ind << "      else if (s_) atomicAdd(&d_result[" << ix << "], s_);\n";
            if (!p.sparse) {
              if (p.aggs[k].fn == AggFn::Count) o << ind << "      if (!qtab) db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
              else {
                o << ind << "      if ((tseen" << k << " >> g) & 1u) { if (qtab) atomicOr(&qbits[" << TWq * (1 + sk) << "ULL + (g >> 5)], 1u << (g & 31)); else db::atomic_set_valid_bit(d_result_validity, " << ix << "); }\n";
                ++sk;
              }
            }
            o << ind << "    }\n";
          }
          o << ind << "  }\n";
          o << ind << "  if (lane == 0) { if (qtab) atomicOr(&qbits[0], ttouch); else atomicOr(&g_touch[0], ttouch); }\n";
          o << ind << "}\n";
        };
        if (gm_base[s] >= 0) {
          // Group row bitmaps: per block and group, the query's rows of that
          // group; COUNT is a popcount, SUM walks the rows.
          o << ind << "unsigned long long tacc[" << G * NA << "];\n";
          o << ind << "#pragma unroll\n" << ind << "for (int r = 0; r < " << G * NA << "; ++r) tacc[r] = 0ULL;\n";
          o << ind << "unsigned ttouch = 0u;\n";
          o << ind << "const unsigned* gm_ = s_gm_t + " << gm_base[s] << " * " << NBS << ";\n";
          o << ind << "for (int b_ = blo_ + lane / lpb_; b_ < bhi_; b_ += 32 / lpb_) {\n";
          o << ind << "  const unsigned w_ = qw_[b_] & bm_;\n";
          o << ind << "  if (!w_) continue;\n";
          o << ind << "  if (w_ & gm_[" << G << " * " << NBS << " + b_]) cx::raise(a.err, cx::ERR_GROUP_DOMAIN);\n";
          o << ind << "  #pragma unroll\n";
          o << ind << "  for (int g = 0; g < " << G << "; ++g) {\n";
          o << ind << "    unsigned wg_ = w_ & gm_[g * " << NBS << " + b_];\n";
          o << ind << "    if (!wg_) continue;\n";
          o << ind << "    ttouch |= 1u << g;\n";
          bool any_sum = false;
          for (int k = 0; k < NA; ++k) {
            if (p.aggs[k].fn == AggFn::Count) o << ind << "    tacc[g * " << NA << " + " << k << "] += (unsigned long long)__popc(wg_);\n";
            else any_sum = true;
          }
          if (any_sum) {
            o << ind << "    while (wg_) {\n";
            o << ind << "      const int i = (b_ << 5) + __ffs(wg_) - 1;\n";
            o << ind << "      wg_ &= wg_ - 1u;\n";
            for (int k = 0; k < NA; ++k)
              if (p.aggs[k].fn == AggFn::Sum)
                o << ind << "      tacc[g * " << NA << " + " << k << "] += (unsigned long long)(" << e.math_push(p.aggs[k].arg.get(), true) << ");\n";
            o << ind << "    }\n";
          }
          o << ind << "  }\n";
          o << ind << "}\n";
          // No nullable columns in a shared shape: a SUM is valid wherever its group was touched.
          for (int k = 0; k < NA; ++k)
            if (!p.sparse && p.aggs[k].fn == AggFn::Sum) o << ind << "unsigned tseen" << k << " = ttouch;\n";
          tiny_flush();
        } else {
        const bool tiny = G <= 32 && G * (unsigned long long)NA <= 16;
        if (tiny && tu.group_merge == 2) {
          // Queries with a shared-memory table add straight into it; the
          // touched / seen bits collect in registers until the unit ends.
          o << ind << "if (qtab) {\n";
          o << ind << "unsigned ttouch = 0u;\n";
          for (int k = 0; k < NA; ++k)
            if (!p.sparse && p.aggs[k].fn == AggFn::Sum) o << ind << "unsigned tseen" << k << " = 0u;\n";
          o << loop_open;
          o << terms.str();
          o << ind << "  int hash = " << horner << ";\n";
          o << ind << "  if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
          o << ind << "  if ((unsigned)hash >= " << G << "u) continue;\n";
          o << ind << "  ttouch |= 1u << hash;\n";
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")";
            o << ind << "  { const unsigned long long x_ = " << x << "; if (x_) atomicAdd(&qtab[hash * " << NA << " + " << k << "], x_); }\n";
            if (!p.sparse && ag.fn == AggFn::Sum) o << ind << "  tseen" << k << " |= 1u << hash;\n";
          }
          o << loop_close;
          o << ind << "ttouch = __reduce_or_sync(0xffffffffu, ttouch);\n";
          int sk = 0;
          for (int k = 0; k < NA; ++k)
            if (!p.sparse && p.aggs[k].fn == AggFn::Sum) {
              o << ind << "tseen" << k << " = __reduce_or_sync(0xffffffffu, tseen" << k << ");\n";
              o << ind << "if (lane == 0 && tseen" << k << ") atomicOr(&qbits[" << TWq * (1 + sk) << "], tseen" << k << ");\n";
              ++sk;
            }
          o << ind << "if (lane == 0 && ttouch) atomicOr(&qbits[0], ttouch);\n";
          o << ind << "} else {\n";
        }
        if (tiny) {
          o << ind << "unsigned long long tacc[" << G * NA << "];\n";
          o << ind << "#pragma unroll\n" << ind << "for (int r = 0; r < " << G * NA << "; ++r) tacc[r] = 0ULL;\n";
          o << ind << "unsigned ttouch = 0u;\n";
          for (int k = 0; k < NA; ++k)
            if (!p.sparse && p.aggs[k].fn == AggFn::Sum) o << ind << "unsigned tseen" << k << " = 0u;\n";
        }
        if (tiny) {
          o << loop_open;
          o << terms.str();
          o << ind << "  int hash = " << horner << ";\n";
          o << ind << "  if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
          o << ind << "  if ((unsigned)hash >= " << G << "u) continue;\n";
          o << ind << "  ttouch |= 1u << hash;\n";
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")";
            o << ind << "  { const unsigned long long x_ = " << x << ";\n";
            o << ind << "    #pragma unroll\n" << ind << "    for (int g = 0; g < " << G << "; ++g) if (hash == g) tacc[g * " << NA << " + " << k << "] += x_;\n";
            if (!p.sparse && ag.fn == AggFn::Sum) o << ind << "    tseen" << k << " |= 1u << hash;\n";
            o << ind << "  }\n";
          }
          o << loop_close;
          tiny_flush();
          if (tu.group_merge == 2) o << ind << "}\n";
        } else if (tu.group_merge == 2 || tu.group_merge == 3) {
          // Direct per-row updates: shared-memory table when the query has one, else global atomics.
          o << loop_open;
          o << terms.str();
          o << ind << "  int hash = " << horner << ";\n";
          o << ind << "  if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
          o << ind << "  if ((unsigned)hash >= " << G << "u) continue;\n";
          o << ind << "  if (qtab) {\n";
          o << ind << "    atomicOr(&qbits[hash >> 5], 1u << (hash & 31));\n";
          int sk = 0;
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")";
            o << ind << "    { const unsigned long long x_ = " << x << "; if (x_) atomicAdd(&qtab[(long long)hash * " << NA << " + " << k << "], x_);";
            if (!p.sparse && ag.fn == AggFn::Sum) { o << " atomicOr(&qbits[" << TWq * (1 + sk) << "ULL + (hash >> 5)], 1u << (hash & 31));"; ++sk; }
            o << " }\n";
          }
          o << ind << "  } else {\n";
          o << ind << "    atomicOr(&g_touch[hash >> 5], 1u << (hash & 31));\n";
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const int slot = (int)p.groups.size() + k;
            const std::string ix = "(unsigned long long)hash * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
            const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")";
            o << ind << "    { const unsigned long long x_ = " << x << "; if (x_) atomicAdd(&d_result[" << ix << "], x_);";
            if (!p.sparse && ag.fn == AggFn::Sum) o << " db::atomic_set_valid_bit(d_result_validity, " << ix << ");";
            o << " }\n";
            if (!p.sparse && ag.fn == AggFn::Count) o << ind << "    db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
          }
          o << ind << "  }\n";
          o << loop_close;
        } else {
          // Larger domains: one row per lane per round in a warp-uniform loop;
          // lanes that hit the same group merge their values (one
          // `__match_any_sync`) so the table sees one atomic per distinct
          // group, not one per row -- a query's few live groups would
          // otherwise serialise the warp's atomics.
          o << ind << "int b_ = blo_ + lane / lpb_;\n";
          o << ind << "unsigned w_ = b_ < bhi_ ? (qw_[b_] & bm_) : 0u;\n";
          o << ind << "for (;;) {\n";
          o << ind << "  while (w_ == 0u && b_ < bhi_) { b_ += 32 / lpb_; w_ = b_ < bhi_ ? (qw_[b_] & bm_) : 0u; }\n";
          o << ind << "  if (!__any_sync(0xffffffffu, w_ != 0u)) break;\n";
          o << ind << "  int hash = -1;\n";
          for (int k = 0; k < NA; ++k) o << ind << "  unsigned long long x" << k << "_ = 0ULL;\n";
          o << ind << "  if (w_ != 0u) {\n";
          o << ind << "  const int i = (b_ << 5) + __ffs(w_) - 1;\n";
          o << ind << "  w_ &= w_ - 1u;\n";
          o << terms.str();
          o << ind << "  hash = " << horner << ";\n";
          o << ind << "  if (!(" << dom << ")) { cx::raise(a.err, cx::ERR_GROUP_DOMAIN); hash = hash % " << G << "; }\n";
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const std::string x = ag.fn == AggFn::Count ? "1ULL" : "(unsigned long long)(" + e.math_push(ag.arg.get(), true) + ")";
            o << ind << "  x" << k << "_ = " << x << ";\n";
          }
          o << ind << "  }\n";
          o << ind << "  const bool ok_ = (unsigned)hash < " << G << "u;\n";
          o << ind << "  const unsigned okm_ = __ballot_sync(0xffffffffu, ok_);\n";
          o << ind << "  if (ok_) {\n";
          o << ind << "    const unsigned peers_ = __match_any_sync(okm_, hash);\n";
          o << ind << "    if (__popc(peers_) > 1) {\n";
          for (int k = 0; k < NA; ++k) {
            o << ind << "      { unsigned long long r_ = 0ULL;\n";
            o << ind << "        for (unsigned m_ = peers_; m_; m_ &= m_ - 1u) r_ += __shfl_sync(peers_, x" << k << "_, __ffs(m_) - 1);\n";
            o << ind << "        x" << k << "_ = r_; }\n";
          }
          o << ind << "    }\n";
          o << ind << "    if (lane == __ffs(peers_) - 1) {\n";
          o << ind << "      if (qtab) {\n";
          o << ind << "        atomicOr(&qbits[hash >> 5], 1u << (hash & 31));\n";
          int sk = 0;
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            o << ind << "        if (x" << k << "_) atomicAdd(&qtab[(long long)hash * " << NA << " + " << k << "], x" << k << "_);\n";
            if (!p.sparse && ag.fn == AggFn::Sum) { o << ind << "        atomicOr(&qbits[" << TWq * (1 + sk) << "ULL + (hash >> 5)], 1u << (hash & 31));\n"; ++sk; }
          }
          o << ind << "      } else {\n";
          o << ind << "        atomicOr(&g_touch[hash >> 5], 1u << (hash & 31));\n";
          for (int k = 0; k < NA; ++k) {
            const Agg& ag = p.aggs[k];
            const int slot = (int)p.groups.size() + k;
            const std::string ix = "(unsigned long long)hash * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
            o << ind << "        if (x" << k << "_) atomicAdd(&d_result[" << ix << "], x" << k << "_);\n";
            if (!p.sparse && (ag.fn == AggFn::Sum || ag.fn == AggFn::Count))
              o << ind << "        db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
          }
          o << ind << "      }\n";
          o << ind << "    }\n";
          o << ind << "  }\n";
          o << ind << "}\n";
        }
        }
      }
      o << "        break; }\n";
    }
    o << "        default: break;\n";
    o << "      }\n";
    o << "    }\n";
    o << "    __syncwarp();\n";
    o << "    if (lane == 0) cx::mbar_arrive(&bar_empty[s]);\n";
    o << "    }\n";
    o << "  }\n";
    o << "  __syncthreads();\n";
    // After a timeout: wait (bounded) for the copies still in flight, then leave.
    o << "  if (*s_abort) {\n";
    o << "    if (threadIdx.x == 0 && staged_ok) {\n";
    o << "      const int ni = *s_nissued;\n";
    o << "      for (int kk = ni - NSTAGE < 0 ? 0 : ni - NSTAGE; kk < ni; ++kk)\n";
    o << "        if ((long long)blockIdx.x + (long long)kk * gridDim.x < full_tiles)\n";
    o << "          (void)cx::mbar_wait_bounded(&bar_full[kk % NSTAGE], (unsigned)((kk / NSTAGE) & 1), cx::drain_limit_us(" << LIM << "));\n";
    o << "    }\n";
    o << "    return;\n";
    o << "  }\n";
    o << "  for (int q = threadIdx.x; q < nq; q += " << CTA << ") {\n";
    o << "    const CxSQ& Q = s_sq[q];\n";
    o << "    switch (Q.shape) {\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      if (!p.groups.empty()) continue;
      o << "      case " << s << ": {\n";
      for (size_t k = 0; k < p.aggs.size(); ++k) {
        o << "        { const unsigned long long s_ = s_qacc[(long long)q * " << NACC << " + " << 2 * k << "], c_ = s_qacc[(long long)q * " << NACC << " + " << 2 * k + 1 << "];\n";
        o << "          if (s_) atomicAdd(&Q.result[" << k << "], s_);\n";
        if (p.aggs[k].fn == AggFn::Count) o << "          db::atomic_set_valid_bit((uint64_t*)Q.validity, " << k << ");\n";
        else o << "          if (c_) db::atomic_set_valid_bit((uint64_t*)Q.validity, " << k << ");\n";
        o << "        }\n";
      }
      o << "        break; }\n";
    }
    o << "      default: break;\n";
    o << "    }\n";
    o << "  }\n";
    // Grouped queries with shared-memory tables: one flush per CTA.
    o << "  for (int q = 0; q < nq; ++q) {\n";
    o << "    const CxSQ& Q = s_sq[q];\n";
    o << "    if (Q.smem_acc < 0) continue;\n";
    o << "    unsigned long long* d_result = Q.result; (void)d_result;\n";
    o << "    uint64_t* d_result_validity = (uint64_t*)Q.validity; (void)d_result_validity;\n";
    o << "    const unsigned long long* qtab = s_tab + Q.smem_acc;\n";
    o << "    const unsigned int* qbits = s_bits + Q.smem_bits;\n";
    o << "    switch (Q.shape) {\n";
    for (size_t s2 = 0; s2 < shapes.size(); ++s2) {
      const Plan& p = *shapes[s2];
      if (p.groups.empty()) continue;
      Emitter e(p, tu);
      const unsigned long long G = e.total_groups();
      const int NA = (int)p.aggs.size();
      if (G * (unsigned long long)NA * 8 > 4096ULL) continue;
      const unsigned long long TWq = (G + 31) / 32;
      const int TS = p.storage_ts();
      o << "      case " << s2 << ":\n";
      o << "        for (long long g = threadIdx.x; g < " << G << "LL; g += " << CTA << ") {\n";
      o << "          if (!((qbits[g >> 5] >> (g & 31)) & 1u)) continue;\n";
      e.emit_key_store(o, "g", "          ");
      int sk = 0;
      for (int k = 0; k < NA; ++k) {
        const int slot = (int)p.groups.size() + k;
        const std::string ix = "(unsigned long long)g * " + std::to_string(TS) + "ULL + " + std::to_string(slot);
        o << "          { const unsigned long long v_ = qtab[g * " << NA << " + " << k << "];\n";
        o << "            if (v_) atomicAdd(&d_result[" << ix << "], v_);\n";
        if (!p.sparse) {
          if (p.aggs[k].fn == AggFn::Count) o << "            db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
          else {
            o << "            if ((qbits[" << TWq * (1 + sk) << "ULL + (g >> 5)] >> (g & 31)) & 1u) db::atomic_set_valid_bit(d_result_validity, " << ix << ");\n";
            ++sk;
          }
        }
        o << "          }\n";
      }
      o << "        }\n        break;\n";
    }
    o << "      default: break;\n";
    o << "    }\n";
    o << "  }\n";
    o << "}\n";
    o << "#undef CX_ISSUE\n\n";
  }

  void emit_keys() {
    meta << "kernel shared_keys_epilogue queries 0 256 0\n";
    src << "extern \"C\" __global__ void __launch_bounds__(256) shared_keys_epilogue(const CxArgs a) {\n";
    src << "  const int q = blockIdx.x;\n";
    src << "  if (q >= a.sq_total) return;\n";
    src << "  const CxSQ Q = a.sq[q];\n";
    src << "  unsigned long long* d_result = Q.result; (void)d_result;\n";
    src << "  uint64_t* d_result_validity = (uint64_t*)Q.validity; (void)d_result_validity;\n";
    src << "  switch (Q.shape) {\n";
    for (size_t s = 0; s < shapes.size(); ++s) {
      const Plan& p = *shapes[s];
      if (p.groups.empty()) continue;
      Emitter e(p, tu);
      src << "    case " << s << ":\n";
      src << "      for (long long g = threadIdx.x; g < " << e.total_groups() << "LL; g += blockDim.x) {\n";
      src << "        if (!((Q.touched[g >> 5] >> (g & 31)) & 1u)) continue;\n";
      e.emit_key_store(src, "g", "        ");
      src << "      }\n      break;\n";
    }
    src << "    default: break;\n  }\n}\n\n";
  }

  static constexpr int CX_MAX_COLS_ = 40;
  static constexpr int CX_MAX_HTS_ = 8;
  static constexpr size_t CX_MAX_SHAPES_ = 16;
};

}  // namespace

std::string generate_cuda(const Plan& plan, const Tuning& tuning) {
  // Payload tables are an optimisation: when they leave the scan without the
  // shared memory its other parts need, smaller table budgets are tried down
  // to none before the launch shape is refused.
  Tuning t = tuning;
  for (;;) {
    try {
      return generate_cuda_impl(plan, t);
    } catch (const PlanError& e) {
      if (t.table_budget <= 0 || std::string(e.what()).find("shared memory exceeds") == std::string::npos) throw;
      t.table_budget = t.table_budget >= 16384 ? t.table_budget / 2 : 0;
    }
  }
}

void collect_literals(const Plan& p, std::vector<const Expr*>& out) {
  for (const auto& s : p.steps) {
    if (s.kind == Step::Filter) lits_of(s.filter.get(), out);
    else lits_of(s.join.filter.get(), out);
  }
  for (const auto& g : p.groups) lits_of(g.expr.get(), out);
  for (const auto& a : p.aggs) lits_of(a.arg.get(), out);
}

std::string generate_shared_cuda(const std::vector<const Plan*>& shapes, const Tuning& tuning) {
  SharedGen g(shapes, tuning);
  return g.run();
}

bool shared_shape_ok(const Plan& plan, std::string* why) {
  std::vector<const Plan*> one{&plan};
  Tuning t;
  SharedGen g(one, t);
  try {
    g.collect();
  } catch (const PlanError& e) {
    if (why) *why = e.what();
    return false;
  }
  return true;
}

}  // namespace cx
