// cx_plan.h -- the star-join pipeline plan the code generator consumes.
//
// A plan is the reference's optimised operator tree for the hot path, flattened
// into the order the push-model visitor walks it (src/core/visitor.cpp:1657-1751,
// produceHashJoin :4466-4528): one fact-table scan, then the filters and hash
// joins met on the way up, then one aggregate.  Join build parameters (hash
// table length, key minimum, payload column) are the values
// JITOperatorVisitor::computeBuildInfo derives (visitor.cpp:3864-4016); GROUP BY
// domains are the catalog statistics generatePerfectHash reads (:2056-2127).
//
// Text form (an S-expression, written by the Python plan builder):
//   (query
//     (table LINEORDER fact (cols lo_orderdate lo_discount ...))
//     (table DDATE (cols d_datekey d_year))
//     (nullable lo_revenue c_city)
//     (filter EXPR)
//     (join DDATE (pk d_datekey) (fk lo_orderdate) (len 61131) (keymin 19920101)
//           (filter EXPR) (payload d_year))
//     (join CUSTOMER (pk c_custkey) (fk lo_custkey) (len N) (keymin N) (multi 1)
//           (payload c_city c_nation))
//     (join DDATE (pk d_datekey) (fk lo_orderdate lo_commitdate) ...)
//     (aggregate (group EXPR (min 1992) (card 7) (nullable 0)) ... (sum EXPR) (count (star))
//                (sparse 0)))
// EXPR: (col NAME) (int N) (null) (star) (add|sub|mul|div E E)
//       (eq|ne|lt|le|gt|ge E E) (and E E) (or E E) (not E) (isnull E) (notnull E)
//       (case COND THEN ELSE)
#pragma once

#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

namespace cx {

struct PlanError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

enum class Op {
  Col, Int, Null, Star,
  Add, Sub, Mul, Div,
  Eq, Ne, Lt, Le, Gt, Ge,
  And, Or, Not, IsNull, NotNull,
  Case
};

struct Expr {
  Op op = Op::Int;
  std::string name;   // Col
  long long ival = 0; // Int
  std::vector<std::unique_ptr<Expr>> kids;
};

bool is_arith(Op op);
bool is_compare(Op op);
const char* op_name(Op op);

struct Table {
  std::string name;
  bool fact = false;
  std::vector<std::string> cols;
};

struct Join {
  std::string dim;                 // dimension table
  std::string pk;                  // build key column
  std::vector<std::string> fks;    // probe key column(s); >1 is the OR-join form
  long long len = 0;               // PHT slots (HASH modulus)
  long long keymin = 0;            // HASH offset
  std::unique_ptr<Expr> filter;    // build-side predicate, may be null
  std::string payload;             // PHT_2 payload column; empty => PHT_1 (or MHT)
  // Catalog range of the payload's values (min, distinct count; card 0 =
  // unknown): a small range lets the scan keep membership and payload of
  // every slot in one byte of shared memory.
  long long prange_min = 0, prange_card = 0;
  // Multi-value hash table (non-unique build key, visitor.cpp:3947-3968): the
  // directory maps a key to the build row ids that carry it and every match
  // expands the probe row; `gathers` are the build columns read by row id.
  bool multi = false;
  std::vector<std::string> gathers;
  // A join whose probe can emit a row more than once: an MHT, or an OR over
  // several fact keys (each distinct key probes, visitor.cpp:4566-4640).
  bool expands() const { return multi || fks.size() > 1; }
};

struct Step {
  enum Kind { Filter, JoinStep } kind = Filter;
  std::unique_ptr<Expr> filter;
  Join join;
};

struct GroupKey {
  std::unique_ptr<Expr> expr;
  long long min = 0;
  long long card = 1;
  bool nullable = false;
};

enum class AggFn { Count, Sum, Min, Max, Avg };

struct Agg {
  AggFn fn = AggFn::Count;
  std::unique_ptr<Expr> arg;  // Star for COUNT(*)
};

struct Plan {
  std::vector<Table> tables;            // tables[0] is the fact table
  std::set<std::string> nullable;       // catalog-nullable columns
  std::vector<Step> steps;              // pipeline order from the scan upwards
  std::vector<GroupKey> groups;
  std::vector<Agg> aggs;
  bool sparse = false;                  // fast sparse output (no validity bits)

  // Derived.
  std::map<std::string, int> table_of_col;  // column -> table slot
  int table_slot(const std::string& t) const;
  unsigned long long group_count() const;    // product of group cards (1 if none)
  int visible_ts() const { return (int)(groups.size() + aggs.size()); }
  int hidden_count_slots() const;
  int storage_ts() const;
  int hidden_count_slot(size_t agg_idx) const;  // -1 if the aggregate has none
  bool has_min() const;
};

// Parses and validates a plan; throws PlanError with a readable message.
std::unique_ptr<Plan> parse_plan(const std::string& text);

}  // namespace cx
