// cx_plan.cpp -- S-expression reader and validation for star-join plans.
#include "cx_plan.h"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <set>

namespace cx {

namespace {

struct Node {
  bool atom = false;
  std::string text;
  std::vector<Node> items;
};

class Reader {
 public:
  explicit Reader(const std::string& s) : s_(s) {}
  Node read() {
    skip();
    Node n = read_node();
    skip();
    if (pos_ != s_.size()) fail("trailing text after plan");
    return n;
  }

 private:
  const std::string& s_;
  size_t pos_ = 0;

  [[noreturn]] void fail(const std::string& m) {
    throw PlanError("plan parse error at offset " + std::to_string(pos_) + ": " + m);
  }
  void skip() {
    while (pos_ < s_.size()) {
      if (std::isspace((unsigned char)s_[pos_])) {
        ++pos_;
      } else if (s_[pos_] == ';') {
        while (pos_ < s_.size() && s_[pos_] != '\n') ++pos_;
      } else {
        break;
      }
    }
  }
  Node read_node() {
    skip();
    if (pos_ >= s_.size()) fail("unexpected end of plan");
    Node n;
    if (s_[pos_] == '(') {
      ++pos_;
      for (;;) {
        skip();
        if (pos_ >= s_.size()) fail("missing ')'");
        if (s_[pos_] == ')') { ++pos_; break; }
        n.items.push_back(read_node());
      }
      return n;
    }
    if (s_[pos_] == ')') fail("unexpected ')'");
    n.atom = true;
    while (pos_ < s_.size() && !std::isspace((unsigned char)s_[pos_]) && s_[pos_] != '(' && s_[pos_] != ')')
      n.text.push_back(s_[pos_++]);
    return n;
  }
};

const std::string& head(const Node& n) {
  static const std::string empty;
  if (n.atom || n.items.empty() || !n.items[0].atom) return empty;
  return n.items[0].text;
}

long long to_int(const Node& n, const char* what) {
  if (!n.atom) throw PlanError(std::string("expected integer for ") + what);
  char* end = nullptr;
  errno = 0;
  long long v = std::strtoll(n.text.c_str(), &end, 10);
  if (errno != 0 || end == n.text.c_str() || *end != '\0')
    throw PlanError(std::string("bad integer '") + n.text + "' for " + what);
  return v;
}

const std::string& to_name(const Node& n, const char* what) {
  if (!n.atom) throw PlanError(std::string("expected name for ") + what);
  return n.text;
}

// Column names become identifiers of the generated kernels (one register
// array per column, plus names derived from it), so a name must be a C
// identifier that is not a C++ keyword, a CUDA built-in, a name of this
// library's primitives, or one of the generated code's own identifiers
// (fixed names, and numbered temporaries such as gt3 or x5_).
void check_column_name(const std::string& c) {
  static const std::set<std::string> reserved = {
      // C++ keywords
      "alignas", "alignof", "and", "and_eq", "asm", "auto", "bitand", "bitor", "bool", "break", "case", "catch",
      "char", "char8_t", "char16_t", "char32_t", "class", "compl", "concept", "const", "consteval", "constexpr",
      "constinit", "const_cast", "continue", "co_await", "co_return", "co_yield", "decltype", "default", "delete",
      "do", "double", "dynamic_cast", "else", "enum", "explicit", "export", "extern", "false", "float", "for",
      "friend", "goto", "if", "inline", "int", "long", "mutable", "namespace", "new", "noexcept", "not", "not_eq",
      "nullptr", "operator", "or", "or_eq", "private", "protected", "public", "register", "reinterpret_cast",
      "requires", "return", "short", "signed", "sizeof", "static", "static_assert", "static_cast", "struct",
      "switch", "template", "this", "thread_local", "throw", "true", "try", "typedef", "typeid", "typename",
      "union", "unsigned", "using", "virtual", "void", "volatile", "wchar_t", "while", "xor", "xor_eq",
      // CUDA built-ins and types, namespaces and primitives of the generated code
      "threadIdx", "blockIdx", "blockDim", "gridDim", "warpSize", "int2", "int4", "uint2", "uint4", "int32_t",
      "int64_t", "uint32_t", "uint64_t", "size_t", "std", "db", "cx", "cx_detail", "HASH", "CxArgs", "InitFlags",
      "InitFlagsZero", "ColumnValidAt", "ProbePHT_1", "ProbePHT_2", "ProbeMultiHT", "GreaterThan", "LessThan",
      "GreaterThanEq", "LessThanEq", "Equal", "NotEqual", "PromoteType", "Promoted",
      // fixed identifiers of the generated kernels
      "BLOCK_THREADS", "IPT", "ITEMS_PER_THREAD", "NWARP", "NSTAGE", "NSC", "TILE_SIZE", "TROWS", "VW", "TR",
      "aborted", "act", "amask", "any_", "avg_", "bad_", "bar_empty", "bar_full", "bar_ready", "bars", "base",
      "bb_", "bits", "blk_", "blo_", "bm_", "bw_", "carry", "cg_", "cnt_", "cs_", "cu_", "cw", "cw_", "cx_smem",
      "d_", "d_result", "d_result_validity", "d_visible_result", "d_visible_validity", "dkm", "dst_", "ent",
      "es_", "ex", "f_", "fk_", "flags", "full_tiles", "fv_", "g_touch", "gd_", "gm_", "gwarp", "hash", "hi_",
      "hit_", "ht", "ht_dir", "in_", "k_iter", "key", "kk", "l2_policy", "lane", "leader", "live", "live_", "lo_",
      "loc", "lpb_", "m_", "m_cols", "m_res", "mht_bsum", "mht_counts", "mht_offsets", "mht_payload", "mht_wpos",
      "mk_", "mst_", "n16_", "n_", "n_rows", "n_tile", "nblk", "nc_", "nch", "need", "ni", "nq", "nq_", "nt",
      "ntiles", "num_tile_items", "num_tiles", "nv", "nw", "nwarps", "o_", "ok_", "okm_", "old_", "oow", "ow_",
      "p_", "pass", "peers", "peers_", "per_", "perb_", "pos_", "pw", "q_", "q_base", "q_n", "qbits", "qtab",
      "qw_", "r_", "red", "rel", "rel_", "rem", "rest_", "ri_", "row_ids", "rtouch", "run", "rv_", "s_", "s_abort",
      "s_acc", "s_acc_all", "s_attr", "s_bits", "s_cube", "s_dim", "s_fm", "s_fr", "s_gm", "s_gm_t", "s_lacc",
      "s_nissued", "s_nj", "s_params", "s_qacc", "s_qb", "s_qb_t", "s_seen", "s_seen_all", "s_shape", "s_tab",
      "s_touch", "s_touch_all", "sc", "sd_", "seen_", "sh_", "slices", "slot", "src", "src_", "stage",
      "stage_buf", "stage_tx", "staged", "staged_ok", "t_", "tacc", "tid", "tile", "tile_offset", "timed_out",
      "tot", "touch_all", "touched_", "ttouch", "units", "v_", "vec_ok", "w_", "wg_", "wh_", "wi_", "wl_", "x_",
      "y_"};
  auto bad = [&](const char* why) {
    throw PlanError("column name '" + c + "' " + why + "; rename the column");
  };
  if (c.empty() || !(std::isalpha((unsigned char)c[0]) || c[0] == '_')) bad("is not a C identifier");
  for (char ch : c)
    if (!(std::isalnum((unsigned char)ch) || ch == '_')) bad("is not a C identifier");
  if (c.size() == 1) bad("is a one-letter name, which the generated kernels use");
  if (c[0] == '_' && (c.size() < 2 || c[1] == '_' || std::isupper((unsigned char)c[1]))) bad("is a reserved identifier");
  if (reserved.count(c)) bad("collides with an identifier of the generated kernels");
  auto prefixed = [&](const char* pre) {
    const size_t n = std::strlen(pre);
    return c.size() > n && c.compare(0, n, pre) == 0 && std::isupper((unsigned char)c[n]);
  };
  if (prefixed("Block") || prefixed("Warp") || prefixed("atomic") || c.compare(0, 3, "cx_") == 0 ||
      c.compare(0, 3, "CX_") == 0 || c.compare(0, 2, "__") == 0)
    bad("collides with this library's primitives");
  // Numbered temporaries: a short stem, digits, optionally _digits and a trailing underscore.
  static const char* stems[] = {"gt", "gd", "x", "v", "h", "k", "e", "w", "g", "cl", "o", "j", "b", "s", "at",
                                "off", "acc_", "seen_", "t", "c", "l", "fb", "fw", "m", "p", "r", "q", "y", "z"};
  for (const char* st : stems) {
    const size_t n = std::strlen(st);
    if (c.size() <= n || c.compare(0, n, st) != 0 || !std::isdigit((unsigned char)c[n])) continue;
    size_t i = n;
    while (i < c.size() && std::isdigit((unsigned char)c[i])) ++i;
    if (i < c.size() && c[i] == '_') {
      ++i;
      while (i < c.size() && std::isdigit((unsigned char)c[i])) ++i;
    }
    if (i == c.size()) bad("has the form of a numbered temporary of the generated kernels");
  }
}

// (key value) lookup inside a list node.
const Node* field(const Node& n, const std::string& key) {
  for (size_t i = 1; i < n.items.size(); ++i)
    if (head(n.items[i]) == key) return &n.items[i];
  return nullptr;
}

struct OpName {
  const char* name;
  Op op;
  int arity;
};
const OpName kOps[] = {
    {"add", Op::Add, 2}, {"sub", Op::Sub, 2}, {"mul", Op::Mul, 2}, {"div", Op::Div, 2},
    {"eq", Op::Eq, 2},   {"ne", Op::Ne, 2},   {"lt", Op::Lt, 2},   {"le", Op::Le, 2},
    {"gt", Op::Gt, 2},   {"ge", Op::Ge, 2},   {"and", Op::And, 2}, {"or", Op::Or, 2},
    {"not", Op::Not, 1}, {"isnull", Op::IsNull, 1}, {"notnull", Op::NotNull, 1},
    {"case", Op::Case, 3},
};

std::unique_ptr<Expr> to_expr(const Node& n) {
  const std::string& h = head(n);
  auto e = std::make_unique<Expr>();
  if (h == "col") {
    if (n.items.size() != 2) throw PlanError("(col NAME) takes one name");
    e->op = Op::Col;
    e->name = to_name(n.items[1], "col");
    return e;
  }
  if (h == "int") {
    if (n.items.size() != 2) throw PlanError("(int N) takes one integer");
    e->op = Op::Int;
    e->ival = to_int(n.items[1], "int literal");
    return e;
  }
  if (h == "null") { e->op = Op::Null; return e; }
  if (h == "star") { e->op = Op::Star; return e; }
  for (const auto& o : kOps) {
    if (h == o.name) {
      if ((int)n.items.size() != o.arity + 1)
        throw PlanError(std::string("(") + o.name + " ...) takes " + std::to_string(o.arity) + " operands");
      e->op = o.op;
      for (int k = 1; k <= o.arity; ++k) e->kids.push_back(to_expr(n.items[k]));
      return e;
    }
  }
  throw PlanError("unknown expression '" + (h.empty() ? std::string("<atom>") : h) + "'");
}

void collect_cols(const Expr* e, std::vector<std::string>& out) {
  if (!e) return;
  if (e->op == Op::Col) out.push_back(e->name);
  for (const auto& k : e->kids) collect_cols(k.get(), out);
}

}  // namespace

bool is_arith(Op op) { return op == Op::Add || op == Op::Sub || op == Op::Mul || op == Op::Div; }
bool is_compare(Op op) {
  return op == Op::Eq || op == Op::Ne || op == Op::Lt || op == Op::Le || op == Op::Gt || op == Op::Ge;
}
const char* op_name(Op op) {
  for (const auto& o : kOps)
    if (o.op == op) return o.name;
  switch (op) {
    case Op::Col: return "col";
    case Op::Int: return "int";
    case Op::Null: return "null";
    case Op::Star: return "star";
    default: return "?";
  }
}

int Plan::table_slot(const std::string& t) const {
  for (size_t i = 0; i < tables.size(); ++i)
    if (tables[i].name == t) return (int)i;
  return -1;
}

unsigned long long Plan::group_count() const {
  unsigned long long g = 1;
  for (const auto& k : groups) g *= (unsigned long long)k.card;
  return g;
}

int Plan::hidden_count_slots() const {
  int n = 0;
  for (const auto& a : aggs) n += (a.fn == AggFn::Avg);
  return n;
}

int Plan::storage_ts() const {
  const int s = (int)(groups.size() + aggs.size()) + hidden_count_slots();
  return s == 0 ? 1 : s;
}

int Plan::hidden_count_slot(size_t agg_idx) const {
  if (agg_idx >= aggs.size() || aggs[agg_idx].fn != AggFn::Avg) return -1;
  int slot = visible_ts();
  for (size_t i = 0; i < agg_idx; ++i) slot += (aggs[i].fn == AggFn::Avg);
  return slot;
}

bool Plan::has_min() const {
  for (const auto& a : aggs)
    if (a.fn == AggFn::Min) return true;
  return false;
}

std::unique_ptr<Plan> parse_plan(const std::string& text) {
  Reader rd(text);
  Node root = rd.read();
  if (head(root) != "query") throw PlanError("plan must start with (query ...)");
  auto p = std::make_unique<Plan>();
  bool have_agg = false;

  for (size_t i = 1; i < root.items.size(); ++i) {
    const Node& n = root.items[i];
    const std::string& h = head(n);
    if (h == "table") {
      Table t;
      if (n.items.size() < 3) throw PlanError("(table NAME [fact] (cols ...))");
      t.name = to_name(n.items[1], "table");
      for (size_t k = 2; k < n.items.size(); ++k) {
        if (n.items[k].atom && n.items[k].text == "fact") t.fact = true;
        else if (head(n.items[k]) == "cols")
          for (size_t c = 1; c < n.items[k].items.size(); ++c) {
            t.cols.push_back(to_name(n.items[k].items[c], "cols"));
            check_column_name(t.cols.back());
          }
        else throw PlanError("unexpected item in (table " + t.name + " ...)");
      }
      if (p->table_slot(t.name) >= 0) throw PlanError("table declared twice: " + t.name);
      if (t.fact && !p->tables.empty() && p->tables[0].fact) throw PlanError("two fact tables");
      if (t.fact) p->tables.insert(p->tables.begin(), std::move(t));
      else p->tables.push_back(std::move(t));
    } else if (h == "nullable") {
      for (size_t k = 1; k < n.items.size(); ++k) p->nullable.insert(to_name(n.items[k], "nullable"));
    } else if (h == "filter") {
      if (have_agg) throw PlanError("filter after aggregate is not part of the scan pipeline");
      if (n.items.size() != 2) throw PlanError("(filter EXPR)");
      Step s;
      s.kind = Step::Filter;
      s.filter = to_expr(n.items[1]);
      p->steps.push_back(std::move(s));
    } else if (h == "join") {
      if (have_agg) throw PlanError("join after aggregate");
      Step s;
      s.kind = Step::JoinStep;
      Join& j = s.join;
      j.dim = to_name(n.items.at(1), "join table");
      const Node* pk = field(n, "pk");
      const Node* fk = field(n, "fk");
      const Node* len = field(n, "len");
      const Node* km = field(n, "keymin");
      if (!pk || pk->items.size() != 2 || !fk || fk->items.size() < 2 || !len || !km)
        throw PlanError("(join DIM (pk C) (fk C...) (len N) (keymin N) ...) is incomplete for " + j.dim);
      j.pk = to_name(pk->items[1], "pk");
      for (size_t k = 1; k < fk->items.size(); ++k) j.fks.push_back(to_name(fk->items[k], "fk"));
      j.len = to_int(len->items.at(1), "len");
      j.keymin = to_int(km->items.at(1), "keymin");
      if (const Node* f = field(n, "filter")) j.filter = to_expr(f->items.at(1));
      if (const Node* mu = field(n, "multi")) j.multi = to_int(mu->items.at(1), "multi") != 0;
      if (const Node* pl = field(n, "payload")) {
        if (pl->items.size() < 2) throw PlanError("(payload C ...) names no column for " + j.dim);
        if (j.multi) {
          for (size_t k = 1; k < pl->items.size(); ++k) j.gathers.push_back(to_name(pl->items[k], "payload"));
        } else {
          if (pl->items.size() != 2) throw PlanError("a perfect-hash join publishes one payload column: " + j.dim);
          j.payload = to_name(pl->items[1], "payload");
        }
      }
      if (const Node* pr = field(n, "prange")) {
        if (pr->items.size() != 3) throw PlanError("(prange MIN CARD) for " + j.dim);
        j.prange_min = to_int(pr->items[1], "prange");
        j.prange_card = to_int(pr->items[2], "prange");
        if (j.prange_card < 0 || j.prange_min < -2147483648LL || j.prange_min > 2147483647LL)
          throw PlanError("prange out of range for " + j.dim);
      }
      if (j.len <= 0 || j.len > (1LL << 30)) throw PlanError("join len out of range for " + j.dim);
      if (j.fks.size() > 4) throw PlanError("an OR-join takes at most 4 fact keys: " + j.dim);
      if (j.gathers.size() > 8) throw PlanError("an MHT join publishes at most 8 columns: " + j.dim);
      p->steps.push_back(std::move(s));
    } else if (h == "aggregate") {
      if (have_agg) throw PlanError("two aggregates");
      have_agg = true;
      for (size_t k = 1; k < n.items.size(); ++k) {
        const Node& a = n.items[k];
        const std::string& ah = head(a);
        if (ah == "group") {
          GroupKey g;
          g.expr = to_expr(a.items.at(1));
          const Node* mn = field(a, "min");
          const Node* cd = field(a, "card");
          const Node* nl = field(a, "nullable");
          if (!mn || !cd) throw PlanError("(group EXPR (min N) (card N) [(nullable 0|1)])");
          g.min = to_int(mn->items.at(1), "group min");
          g.card = to_int(cd->items.at(1), "group card");
          g.nullable = nl ? to_int(nl->items.at(1), "nullable") != 0 : false;
          if (g.card <= 0) throw PlanError("group card must be positive");
          if (g.expr->op != Op::Col && g.expr->op != Op::Case)
            throw PlanError("GROUP BY expression is not supported by perfect hash codegen: " +
                            std::string(op_name(g.expr->op)));
          p->groups.push_back(std::move(g));
        } else if (ah == "sparse") {
          p->sparse = to_int(a.items.at(1), "sparse") != 0;
        } else {
          Agg g;
          if (ah == "count") g.fn = AggFn::Count;
          else if (ah == "sum") g.fn = AggFn::Sum;
          else if (ah == "min") g.fn = AggFn::Min;
          else if (ah == "max") g.fn = AggFn::Max;
          else if (ah == "avg") g.fn = AggFn::Avg;
          else throw PlanError("unknown aggregate '" + ah + "'");
          if (a.items.size() != 2) throw PlanError("aggregate takes one argument");
          g.arg = to_expr(a.items[1]);
          if (g.arg->op == Op::Star && g.fn != AggFn::Count)
            throw PlanError("only COUNT accepts '*'");
          p->aggs.push_back(std::move(g));
        }
      }
      if (p->aggs.empty()) throw PlanError("aggregate needs at least one aggregate function");
    } else {
      throw PlanError("unknown plan item '" + h + "'");
    }
  }

  if (!have_agg) throw PlanError("plan has no aggregate (projection plans are not on this path)");
  if (p->tables.empty() || !p->tables[0].fact) throw PlanError("plan declares no fact table");
  if ((int)p->tables.size() > 8) throw PlanError("too many tables");
  for (size_t t = 0; t < p->tables.size(); ++t)
    for (const auto& c : p->tables[t].cols) {
      if (p->table_of_col.count(c)) throw PlanError("column declared twice: " + c);
      p->table_of_col[c] = (int)t;
    }

  // Column/table consistency: fact-side expressions may reference fact columns
  // and the payloads of joins already probed; build-side filters only their
  // own dimension.
  std::set<std::string> visible;
  for (const auto& c : p->tables[0].cols) visible.insert(c);
  auto check = [&](const Expr* e, const std::set<std::string>& allowed, const std::string& where) {
    std::vector<std::string> cols;
    collect_cols(e, cols);
    for (const auto& c : cols) {
      if (!p->table_of_col.count(c)) throw PlanError("unknown column '" + c + "' in " + where);
      if (!allowed.count(c)) throw PlanError("column '" + c + "' is not available in " + where);
    }
  };
  std::set<std::string> seen_dims;
  for (auto& s : p->steps) {
    if (s.kind == Step::Filter) {
      check(s.filter.get(), visible, "fact-side filter");
      continue;
    }
    Join& j = s.join;
    const int dt = p->table_slot(j.dim);
    if (dt <= 0) throw PlanError("join dimension '" + j.dim + "' is not a declared dimension table");
    if (seen_dims.count(j.dim)) throw PlanError("dimension joined twice: " + j.dim);
    seen_dims.insert(j.dim);
    std::set<std::string> dimcols(p->tables[dt].cols.begin(), p->tables[dt].cols.end());
    if (!dimcols.count(j.pk)) throw PlanError("pk '" + j.pk + "' is not a column of " + j.dim);
    for (size_t k = 0; k < j.fks.size(); ++k) {
      const std::string& fk = j.fks[k];
      if (!visible.count(fk) || p->table_of_col[fk] != 0) throw PlanError("fk '" + fk + "' is not a fact column");
      for (size_t q = 0; q < k; ++q)
        if (j.fks[q] == fk) throw PlanError("fk '" + fk + "' listed twice in the OR-join with " + j.dim);
    }
    if (j.filter) check(j.filter.get(), dimcols, "build filter of " + j.dim);
    if (!j.payload.empty()) {
      if (!dimcols.count(j.payload) || j.payload == j.pk) throw PlanError("bad payload column for " + j.dim);
      visible.insert(j.payload);
    }
    for (const auto& c : j.gathers) {
      if (!dimcols.count(c)) throw PlanError("payload '" + c + "' is not a column of " + j.dim);
      if (std::count(j.gathers.begin(), j.gathers.end(), c) != 1) throw PlanError("payload '" + c + "' listed twice");
      visible.insert(c);
    }
  }
  for (const auto& g : p->groups) check(g.expr.get(), visible, "GROUP BY");
  for (const auto& a : p->aggs) check(a.arg.get(), visible, "aggregate");
  if (p->group_count() > (1ULL << 31)) throw PlanError("group domain too large for a perfect hash");
  {
    // A column X_valid would share its name with the validity register of a column X.
    std::set<std::string> all;
    for (const auto& t : p->tables) all.insert(t.cols.begin(), t.cols.end());
    for (const auto& c : all)
      if (c.size() > 6 && c.compare(c.size() - 6, 6, "_valid") == 0 && all.count(c.substr(0, c.size() - 6)))
        throw PlanError("column name '" + c + "' collides with the validity register of column '" +
                        c.substr(0, c.size() - 6) + "'; rename the column");
  }
  return p;
}

}  // namespace cx
