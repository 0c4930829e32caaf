// emit_visitor.cpp -- runs the reference's own code generator (JITOperatorVisitor
// from src/core/visitor.cpp, after the Optimizer of src/core/optimizer_rules.cpp)
// on hand-built operator trees of the measured query shapes and prints the
// SYCL programs it emits.  TEST INFRASTRUCTURE ONLY: the output is committed as
// golden fixtures under tests/golden/visitor/ (tests/golden/make_visitor_golden.py)
// and checked by the tests that feed it to cx_compile / cx_execute.
//
// The reference builds these trees from SQL with its QueryTranslator
// (src/core/translator.cpp), which needs the hsql parser that is not vendored
// here; the trees below are what the translator produces for each query before
// optimisation: a FilterNode holding every WHERE conjunct above a left-deep
// chain of HashJoinNodes (build side first, as test/test_optimizer.cpp:110-137
// builds them), under an AggregateNode.  The catalog carries the synthetic
// schema's row counts and column statistics (key ranges, dense attribute
// domains), as the catalog cache would after loading that data.
//
// Usage: emit_visitor <query> ; queries: q11 q31 q31_nullable t0 t1 t2 t3
#include <iostream>
#include <memory>
#include <string>

#include "core/optimizer_rules.h"
#include "core/visitor.h"

namespace db {
// The accept() one-liners live in src/core/translator.cpp beside the SQL
// translator; they are restated here so the visitor links without hsql.
void ColumnRefExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void LiteralIntExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void LiteralFloatExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void LiteralNullExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void BinaryExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void CaseWhenExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void StarExpr::accept(ExprVisitor& v) const { v.visit(*this); }
void TableScanNode::accept(OperatorVisitor& v) const { v.visit(*this); }
void FilterNode::accept(OperatorVisitor& v) const { v.visit(*this); }
void HashJoinNode::accept(OperatorVisitor& v) const { v.visit(*this); }
void AggregateNode::accept(OperatorVisitor& v) const { v.visit(*this); }
void ProjectionNode::accept(OperatorVisitor& v) const { v.visit(*this); }
void SortLimitNode::accept(OperatorVisitor& v) const { v.visit(*this); }
}  // namespace db

using namespace db;

namespace {

using Expr = std::unique_ptr<ExprNode>;
using Op = std::unique_ptr<OperatorNode>;

const char* table_of(const std::string& col) {
  switch (col[0]) {
    case 'l': return "LINEORDER";
    case 'c': return "CUSTOMER";
    case 's': return "SUPPLIER";
    case 'p': return "PART";
    default: return "DDATE";
  }
}

Expr col(const char* c) { return std::make_unique<ColumnRefExpr>(c, table_of(c)); }
Expr lit(long v) { return std::make_unique<LiteralIntExpr>(v); }
Expr bin(ExprType t, Expr a, Expr b) { return std::make_unique<BinaryExpr>(t, std::move(a), std::move(b)); }
Expr eq(const char* c, long v) { return bin(ExprType::OP_EQ, col(c), lit(v)); }
Expr ge(const char* c, long v) { return bin(ExprType::OP_GTE, col(c), lit(v)); }
Expr le(const char* c, long v) { return bin(ExprType::OP_LTE, col(c), lit(v)); }
Expr lt(const char* c, long v) { return bin(ExprType::OP_LT, col(c), lit(v)); }
Expr gt(const char* c, long v) { return bin(ExprType::OP_GT, col(c), lit(v)); }
Expr and_(Expr a, Expr b) { return bin(ExprType::OP_AND, std::move(a), std::move(b)); }
Expr or_(Expr a, Expr b) { return bin(ExprType::OP_OR, std::move(a), std::move(b)); }
Expr is_null(const char* c) { return bin(ExprType::OP_IS_NULL, col(c), nullptr); }
Expr not_null(const char* c) { return bin(ExprType::OP_IS_NOT_NULL, col(c), nullptr); }

// Joins `dim` (build side) to `probe` on fk = pk.
Op join(const char* fk, const char* pk, Op probe) {
  auto j = std::make_unique<HashJoinNode>(bin(ExprType::OP_EQ, col(fk), col(pk)));
  j->addChild(std::make_unique<TableScanNode>(table_of(pk)));
  j->addChild(std::move(probe));
  return j;
}

Op scan() { return std::make_unique<TableScanNode>("LINEORDER"); }

Op filtered(Expr pred, Op in) {
  auto f = std::make_unique<FilterNode>(std::move(pred));
  f->addChild(std::move(in));
  return f;
}

std::shared_ptr<Catalog> catalog(long fact_rows, bool nullable) {
  auto cat = std::make_shared<Catalog>();
  TableMetadata lo("LINEORDER", {"lo_orderdate", "lo_custkey", "lo_suppkey", "lo_partkey", "lo_quantity",
                                 "lo_discount", "lo_extendedprice", "lo_revenue", "lo_supplycost"},
                   fact_rows, true);
  if (nullable) lo.setColumnNullable("lo_revenue");
  cat->pushTableMetadata(lo);
  TableMetadata d("DDATE", {"d_datekey", "d_year", "d_month", "d_weeknum"}, 2556, false);
  d.setColumnStats("d_datekey", {19920101, 19981230, 2556});
  d.setColumnPrimaryKey("d_datekey");
  d.setColumnStats("d_year", {1992, 1998, 7});
  d.setColumnStats("d_month", {1, 12, 12});
  cat->pushTableMetadata(d);
  for (const char* t : {"CUSTOMER", "SUPPLIER"}) {
    const bool c = t[0] == 'C';
    const long n = c ? 300000 : 20000;
    const std::string p = c ? "c_" : "s_";
    TableMetadata m(t, {p + (c ? "custkey" : "suppkey"), p + "region", p + "nation", p + "city"}, n, false);
    m.setColumnStats(p + (c ? "custkey" : "suppkey"), {1, n, (uint64_t)n});
    m.setColumnPrimaryKey(p + (c ? "custkey" : "suppkey"));
    m.setColumnStats(p + "region", {0, 4, 5});
    m.setColumnStats(p + "nation", {0, 24, 25});
    m.setColumnStats(p + "city", {0, 249, 250});
    if (c && nullable) m.setColumnNullable("c_city");
    cat->pushTableMetadata(m);
  }
  TableMetadata p("PART", {"p_partkey", "p_mfgr", "p_category", "p_brand1"}, 200000, false);
  p.setColumnStats("p_partkey", {1, 200000, 200000});
  p.setColumnPrimaryKey("p_partkey");
  p.setColumnStats("p_mfgr", {0, 4, 5});
  p.setColumnStats("p_category", {0, 24, 25});
  p.setColumnStats("p_brand1", {0, 999, 1000});
  cat->pushTableMetadata(p);
  return cat;
}

std::unique_ptr<AggregateNode> aggregate(Op in) {
  auto a = std::make_unique<AggregateNode>();
  a->addChild(std::move(in));
  return a;
}

// The query shapes, with the literals the tests use (tests/test_visitor_dropin.py).
std::unique_ptr<AggregateNode> build(const std::string& q) {
  if (q == "q11") {  // SSB Q1.1 shape
    auto a = aggregate(filtered(and_(and_(and_(eq("d_year", 1995), ge("lo_discount", 2)), le("lo_discount", 4)),
                                     lt("lo_quantity", 30)),
                                join("lo_orderdate", "d_datekey", scan())));
    a->aggregates.emplace_back("SUM", bin(ExprType::OP_MUL, col("lo_extendedprice"), col("lo_discount")));
    return a;
  }
  if (q == "q31" || q == "q31_nullable") {  // SSB Q3.1 shape (and its nullable variant)
    const bool nul = q == "q31_nullable";
    const long r = nul ? 1 : 2, y0 = nul ? 1993 : 1992, y1 = nul ? 1998 : 1997;
    Expr pred = and_(and_(and_(eq("c_region", r), eq("s_region", r)), ge("d_year", y0)), le("d_year", y1));
    if (nul)
      pred = and_(and_(and_(std::move(pred), or_(ge("lo_revenue", 2000000), is_null("lo_revenue"))),
                       or_(bin(ExprType::OP_NOT, gt("lo_revenue", 9500000), nullptr), is_null("lo_revenue"))),
                  or_(not_null("c_city"), not_null("lo_revenue")));
    auto a = aggregate(filtered(std::move(pred),
                                join("lo_orderdate", "d_datekey",
                                     join("lo_suppkey", "s_suppkey", join("lo_custkey", "c_custkey", scan())))));
    if (nul) {
      a->group_by_exprs.push_back(col("c_city"));
      a->group_by_exprs.push_back(col("d_year"));
      a->aggregates.emplace_back("COUNT", std::make_unique<StarExpr>());
      a->aggregates.emplace_back("COUNT", col("lo_revenue"));
      a->aggregates.emplace_back("SUM", col("lo_revenue"));
    } else {
      a->group_by_exprs.push_back(col("c_nation"));
      a->group_by_exprs.push_back(col("s_nation"));
      a->group_by_exprs.push_back(col("d_year"));
      a->aggregates.emplace_back("SUM", col("lo_revenue"));
    }
    return a;
  }
  if (q == "t0") {  // ranges + scalar SUM
    auto a = aggregate(filtered(and_(and_(and_(ge("lo_quantity", 5), le("lo_quantity", 35)), ge("lo_discount", 3)),
                                     le("lo_discount", 5)),
                                scan()));
    a->aggregates.emplace_back("SUM", bin(ExprType::OP_MUL, col("lo_revenue"), col("lo_discount")));
    return a;
  }
  if (q == "t1") {  // date join + GROUP BY year
    auto a = aggregate(filtered(and_(and_(lt("lo_quantity", 25), ge("d_year", 1993)), le("d_year", 1996)),
                                join("lo_orderdate", "d_datekey", scan())));
    a->group_by_exprs.push_back(col("d_year"));
    a->aggregates.emplace_back("SUM", col("lo_revenue"));
    return a;
  }
  if (q == "t2") {  // three joins + GROUP BY (nation, year)
    auto a = aggregate(filtered(and_(and_(and_(eq("c_region", 3), eq("s_region", 1)), ge("d_year", 1994)),
                                     le("d_year", 1998)),
                                join("lo_orderdate", "d_datekey",
                                     join("lo_suppkey", "s_suppkey", join("lo_custkey", "c_custkey", scan())))));
    a->group_by_exprs.push_back(col("c_nation"));
    a->group_by_exprs.push_back(col("d_year"));
    a->aggregates.emplace_back("SUM", col("lo_revenue"));
    return a;
  }
  if (q == "t3") {  // four joins + GROUP BY (brand, year)
    auto a = aggregate(filtered(and_(and_(eq("p_category", 7), eq("s_region", 2)), le("c_region", 3)),
                                join("lo_orderdate", "d_datekey",
                                     join("lo_custkey", "c_custkey",
                                          join("lo_suppkey", "s_suppkey",
                                               join("lo_partkey", "p_partkey", scan()))))));
    a->group_by_exprs.push_back(col("p_brand1"));
    a->group_by_exprs.push_back(col("d_year"));
    a->aggregates.emplace_back("SUM", bin(ExprType::OP_SUB, col("lo_revenue"), col("lo_supplycost")));
    return a;
  }
  return nullptr;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: emit_visitor <q11|q31|q31_nullable|t0|t1|t2|t3> [fact_rows]\n";
    return 2;
  }
  const std::string q = argv[1];
  const long rows = argc > 2 ? std::stol(argv[2]) : 60000000;
  auto agg = build(q);
  if (!agg) {
    std::cerr << "unknown query " << q << "\n";
    return 2;
  }
  auto cat = catalog(rows, q == "q31_nullable");
  std::unique_ptr<OperatorNode> tree = std::move(agg);
  Optimizer opt;
  tree = opt.optimize(std::move(tree));
  JITContext ctx;
  JITOperatorVisitor v(ctx, *cat);
  tree->accept(v);
  std::cout << v.generateCode();
  return 0;
}
