// ref_harness.cpp -- runs star-join queries on the host with the reference's
// OWN crystal primitives (include/crystal/load.h, pred.h, join.h and
// include/core/inline_math.h, compiled unmodified from the reference tree) in
// the kernel structure the reference's visitor emits
// (src/core/visitor.cpp:1657-1751, 4206-4290, 3017-3195): per 512-row tile,
// 128 work-items x 4 items, build kernels first, then one fused scan with
// BlockLoad / BlockPred* / BlockProbeAndPHT_* and the aggregate.  Work-groups
// run in parallel with OpenMP; the work-items of one group run in sequence and
// the group reduction (reduce_over_group) is their sum.  Atomics map to
// std::atomic_ref through the shim in oracle/ref/sycl/sycl.hpp.
//
// This is the "reference" kind of CPU baseline and a second, independent check
// of the oracle restatement.  Test/bench infrastructure only.
//
// Query shapes: AND-chains of `column op literal` filters on the fact table
// and on each dimension, PHT_1/PHT_2 joins, GROUP BY over payload or fact
// columns, SUM/COUNT of a column, a product or a difference of two columns.
// One join may expand rows: an OR over two fact keys (visitor.cpp:4587-4640,
// vector probes per key with duplicate keys skipped) or a multi-value hash
// table (count / prefix sum / write build, :4295-4464, and the row-expanding
// ProbeMultiHT loop, :4672-4730, whose payload is the build row id used to
// read one build column); joins after it probe in item mode (ProbePHT_1/2,
// :4741-4790).
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

#include "crystal/load.h"
#include "crystal/pred.h"
#include "crystal/join.h"
#include "core/inline_math.h"

namespace {

constexpr int BT = 128;
constexpr int IPT = 4;
constexpr int TILE = BT * IPT;

}  // namespace

extern "C" {

struct RefPred {
  int col;  // column index
  int op;   // 0 eq 1 ne 2 lt 3 le 4 gt 5 ge
  int lit;
};

struct RefJoin {
  int fk;          // fact column index
  int pk;          // dimension key column index
  int payload;     // dimension payload column index, -1 for PHT_1
  int len;         // HASH modulus
  int keymin;      // HASH offset
  int dim_rows;
  int npred;
  RefPred preds[8];
  int fk2;         // second fact key of an OR-join, -1 for none
  int multi;       // 1: multi-value hash table; `payload` is read through the row id
};

struct RefOperand {
  int kind;  // 0 fact column, 1 payload of join `idx`
  int idx;
};

struct RefGroup {
  RefOperand v;
  int min;
  int card;
};

struct RefAgg {
  int fn;    // 0 count(*), 1 sum
  int form;  // 0 a, 1 a*b, 2 a-b
  RefOperand a, b;
};

struct RefQuery {
  int npred;
  RefPred preds[8];
  int njoin;
  RefJoin joins[4];
  int ngroup;
  RefGroup groups[4];
  int nagg;
  RefAgg aggs[4];
};

}  // extern "C"

namespace {

// BlockPred / BlockPredA<op>: the first fact predicate sets flags, the rest AND
// into them (visitor.cpp:1852-1867, first_flag = false keeps the scan mask).
void apply_pred(int tid, int (&items)[IPT], int (&flags)[IPT], const RefPred& p, int n, bool first) {
  if (first) {
    switch (p.op) {
      case 0: BlockPredEq<int, BT, IPT>(tid, items, flags, p.lit, n); break;
      case 1: BlockPredNEq<int, BT, IPT>(tid, items, flags, p.lit, n); break;
      case 2: BlockPredLT<int, BT, IPT>(tid, items, flags, p.lit, n); break;
      case 3: BlockPredLTE<int, BT, IPT>(tid, items, flags, p.lit, n); break;
      case 4: BlockPredGT<int, BT, IPT>(tid, items, flags, p.lit, n); break;
      default: BlockPredGTE<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    }
    return;
  }
  switch (p.op) {
    case 0: BlockPredAEq<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    case 1: BlockPredANEq<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    case 2: BlockPredALT<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    case 3: BlockPredALTE<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    case 4: BlockPredAGT<int, BT, IPT>(tid, items, flags, p.lit, n); break;
    default: BlockPredAGTE<int, BT, IPT>(tid, items, flags, p.lit, n); break;
  }
}

struct ThreadRegs {
  int flags[IPT];
  int items[IPT];
  int payload[4][IPT];
};

int operand(const ThreadRegs& r, const RefOperand& o, int i, int (*fact_items)[IPT]) {
  return o.kind == 0 ? fact_items[o.idx][i] : r.payload[o.idx][i];
}

}  // namespace

extern "C" int ref_run(const RefQuery* q, const int32_t* const* cols, long long n_fact, uint64_t* result,
                       long long result_words, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  std::memset(result, 0, (size_t)result_words * sizeof(uint64_t));

  // Build kernels (emitPHTBuildKernel): dimension filter, then PHT_1 / PHT_2.
  std::vector<std::vector<int>> hts(q->njoin);
  std::vector<std::vector<int>> mpay(q->njoin);
  int ej = -1;  // the expanding join, if any
  for (int j = 0; j < q->njoin; ++j)
    if (q->joins[j].multi || q->joins[j].fk2 >= 0) ej = j;
  for (int j = 0; j < q->njoin; ++j) {
    const RefJoin& J = q->joins[j];
    if (J.multi) {
      // emitMHTBuildKernels: count, exclusive prefix sum, write.
      hts[j].assign(3 * (size_t)J.len, 0);
      std::vector<int> counts(J.len, 0), offsets(J.len, 0), wpos(J.len, 0);
      mpay[j].assign(J.dim_rows > 0 ? J.dim_rows : 1, 0);
      const int tiles = (J.dim_rows + TILE - 1) / TILE;
      for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
          long long run = 0;
          for (int h = 0; h < J.len; ++h) { offsets[h] = (int)run; run += counts[h]; }
        }
#pragma omp parallel for schedule(static)
        for (int t = 0; t < tiles; ++t) {
          const int tile_offset = t * TILE;
          const int n = (t == tiles - 1) ? J.dim_rows - tile_offset : TILE;
          for (int tid = 0; tid < BT; ++tid) {
            int items[IPT], items2[IPT], flags[IPT];
            InitFlags<BT, IPT>(flags);
            for (int k = 0; k < J.npred; ++k) {
              BlockLoad<int, BT, IPT>(const_cast<int*>(cols[J.preds[k].col]) + tile_offset, tid, tile_offset, items, n);
              apply_pred(tid, items, flags, J.preds[k], n, k == 0);
            }
            BlockLoad<int, BT, IPT>(const_cast<int*>(cols[J.pk]) + tile_offset, tid, tile_offset, items, n);
            if (pass == 0) {
              BlockBuildMHT_Count<int, BT, IPT>(tid, items, flags, counts.data(), J.len, J.keymin, n);
            } else {
              BlockMakeRowIds<BT, IPT>(tid, tile_offset, items2, n);
              BlockBuildMHT_Write<int, int, BT, IPT>(tid, items, items2, flags, hts[j].data(), offsets.data(),
                                                     wpos.data(), counts.data(), mpay[j].data(), J.len, J.keymin, n);
            }
          }
        }
      }
      continue;
    }
    hts[j].assign(2 * (size_t)J.len, 0);
    int* ht = hts[j].data();
    const int tiles = (J.dim_rows + TILE - 1) / TILE;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < tiles; ++t) {
      const int tile_offset = t * TILE;
      const int n = (t == tiles - 1) ? J.dim_rows - tile_offset : TILE;
      for (int tid = 0; tid < BT; ++tid) {
        int items[IPT], items2[IPT], flags[IPT];
        InitFlags<BT, IPT>(flags);
        for (int k = 0; k < J.npred; ++k) {
          BlockLoad<int, BT, IPT>(const_cast<int*>(cols[J.preds[k].col]) + tile_offset, tid, tile_offset, items, n);
          apply_pred(tid, items, flags, J.preds[k], n, k == 0);
        }
        BlockLoad<int, BT, IPT>(const_cast<int*>(cols[J.pk]) + tile_offset, tid, tile_offset, items, n);
        if (J.payload < 0) {
          BlockBuildSelectivePHT_1<int, BT, IPT>(tid, items, flags, ht, J.len, J.keymin, n);
        } else {
          BlockLoad<int, BT, IPT>(const_cast<int*>(cols[J.payload]) + tile_offset, tid, tile_offset, items2, n);
          BlockBuildSelectivePHT_2<int, int, BT, IPT>(tid, items, items2, flags, ht, J.len, J.keymin, n);
        }
      }
    }
  }

  // The fused scan (produceTableScan / consume*Vector).
  long long G = 1;
  for (int g = 0; g < q->ngroup; ++g) G *= q->groups[g].card;
  const int ts = q->ngroup + q->nagg;
  const long long tiles = (n_fact + TILE - 1) / TILE;
  // fact columns referenced anywhere get a register array per work-item
  int used[64] = {0};
  int nused = 0;
  auto use = [&](int c) {
    for (int k = 0; k < nused; ++k)
      if (used[k] == c) return;
    used[nused++] = c;
  };
  for (int k = 0; k < q->npred; ++k) use(q->preds[k].col);
  for (int j = 0; j < q->njoin; ++j) {
    use(q->joins[j].fk);
    if (q->joins[j].fk2 >= 0) use(q->joins[j].fk2);
  }
  for (int g = 0; g < q->ngroup; ++g)
    if (q->groups[g].v.kind == 0) use(q->groups[g].v.idx);
  for (int a = 0; a < q->nagg; ++a) {
    if (q->aggs[a].fn == 0) continue;
    if (q->aggs[a].a.kind == 0) use(q->aggs[a].a.idx);
    if (q->aggs[a].form && q->aggs[a].b.kind == 0) use(q->aggs[a].b.idx);
  }

#pragma omp parallel for schedule(static)
  for (long long t = 0; t < tiles; ++t) {
    const int tile_offset = (int)(t * TILE);
    const int n = (t == tiles - 1) ? (int)(n_fact - t * TILE) : TILE;
    unsigned long long group_sum[4] = {0, 0, 0, 0};
    for (int tid = 0; tid < BT; ++tid) {
      ThreadRegs r;
      int fact_items[64][IPT];
      InitFlags<BT, IPT>(r.flags);
      for (int k = 0; k < nused; ++k)
        BlockLoad<int, BT, IPT>(const_cast<int*>(cols[used[k]]) + tile_offset, tid, tile_offset, fact_items[used[k]], n);
      for (int k = 0; k < q->npred; ++k)
        apply_pred(tid, fact_items[q->preds[k].col], r.flags, q->preds[k], n, false);
      // Aggregate of one qualifying item (consumeAggregate, vector or item mode).
      auto consume_item = [&](ThreadRegs& rr, int i) {
        if (q->ngroup == 0) {
          for (int a = 0; a < q->nagg; ++a) {
            const RefAgg& A = q->aggs[a];
            unsigned long long v = 1ULL;
            if (A.fn == 1) {
              const int x = operand(rr, A.a, i, fact_items);
              if (A.form == 0) v = (unsigned long long)x;
              else if (A.form == 1) v = (unsigned long long)x * operand(rr, A.b, i, fact_items);
              else v = (unsigned long long)x - operand(rr, A.b, i, fact_items);
            }
            group_sum[a] += v;  // per-work-item locals, summed = reduce_over_group
          }
          return;
        }
        int hash = 0;
        for (int g = 0; g < q->ngroup; ++g) {
          const int term = operand(rr, q->groups[g].v, i, fact_items) - q->groups[g].min;
          hash = g == 0 ? term : hash * q->groups[g].card + term;
        }
        hash = (int)(hash % G);
        const long long out = (long long)hash * ts;
        for (int g = 0; g < q->ngroup; ++g)
          result[out + g] = static_cast<unsigned long long>(operand(rr, q->groups[g].v, i, fact_items));
        for (int a = 0; a < q->nagg; ++a) {
          const RefAgg& A = q->aggs[a];
          unsigned long long v = 1ULL;
          if (A.fn == 1) {
            const int x = operand(rr, A.a, i, fact_items);
            if (A.form == 0) v = (unsigned long long)x;
            else if (A.form == 1) v = (unsigned long long)x * operand(rr, A.b, i, fact_items);
            else v = (unsigned long long)x - operand(rr, A.b, i, fact_items);
          }
          db::atomic_add_ull(*reinterpret_cast<unsigned long long*>(&result[out + q->ngroup + a]), v);
        }
      };
      // Joins after the expanding one, in item mode (consumeHashJoinItem).
      auto item_tail = [&](ThreadRegs& rr, int i) {
        for (int j = ej + 1; j < q->njoin; ++j) {
          const RefJoin& J = q->joins[j];
          const int key = fact_items[J.fk][i];
          const bool hit = J.payload < 0 ? ProbePHT_1<int>(key, hts[j].data(), J.len, J.keymin)
                                         : ProbePHT_2<int, int>(key, rr.payload[j][i], hts[j].data(), J.len, J.keymin);
          if (!hit) return;
        }
        consume_item(rr, i);
      };
      const int vec_joins = ej < 0 ? q->njoin : ej;
      for (int j = 0; j < vec_joins; ++j) {
        const RefJoin& J = q->joins[j];
        if (J.payload < 0)
          BlockProbeAndPHT_1<int, BT, IPT>(tid, fact_items[J.fk], r.flags, hts[j].data(), J.len, J.keymin, n);
        else
          BlockProbeAndPHT_2<int, int, BT, IPT>(tid, fact_items[J.fk], r.payload[j], r.flags, hts[j].data(), J.len,
                                                J.keymin, n);
      }
      if (ej < 0) {
        for (int i = 0; i < IPT; ++i)
          if (r.flags[i] && (tid + BT * i < n)) consume_item(r, i);
        continue;
      }
      const RefJoin& E = q->joins[ej];
      const int nfk = E.fk2 >= 0 ? 2 : 1;
      if (!E.multi) {
        // OR-join on a PHT: one vector probe per fact key, a key equal to an
        // earlier one skipped, the rest of the pipeline consumed per key.
        int base[IPT];
        for (int i = 0; i < IPT; ++i) base[i] = r.flags[i];
        for (int f = 0; f < nfk; ++f) {
          const int fcol = f == 0 ? E.fk : E.fk2;
          for (int i = 0; i < IPT; ++i) {
            r.flags[i] = base[i];
            if (f == 1 && (tid + BT * i < n)) r.flags[i] = r.flags[i] && db::safe_neq(fact_items[E.fk2][i], fact_items[E.fk][i]);
          }
          if (E.payload < 0)
            BlockProbeAndPHT_1<int, BT, IPT>(tid, fact_items[fcol], r.flags, hts[ej].data(), E.len, E.keymin, n);
          else
            BlockProbeAndPHT_2<int, int, BT, IPT>(tid, fact_items[fcol], r.payload[ej], r.flags, hts[ej].data(), E.len,
                                                  E.keymin, n);
          for (int i = 0; i < IPT; ++i)
            if (r.flags[i] && (tid + BT * i < n)) item_tail(r, i);
        }
        continue;
      }
      // MHT: row-expanding probe per item and fact key.
      for (int i = 0; i < IPT; ++i) {
        for (int f = 0; f < nfk; ++f) {
          const int fcol = f == 0 ? E.fk : E.fk2;
          int branch_flag = r.flags[i] && (tid + BT * i < n);
          if (f == 1) branch_flag = branch_flag && db::safe_neq(fact_items[E.fk2][i], fact_items[E.fk][i]);
          if (!branch_flag) continue;
          int offset = 0, count = 0;
          ProbeMultiHT(fact_items[fcol][i], offset, count, branch_flag, hts[ej].data(), E.len, E.keymin);
          for (int jj = 0; jj < count; ++jj) {
            const int rid = mpay[ej][offset + jj];
            if (E.payload >= 0) r.payload[ej][i] = cols[E.payload][rid];
            item_tail(r, i);
          }
        }
      }
    }
    if (q->ngroup == 0)
      for (int a = 0; a < q->nagg; ++a)
        db::atomic_add_ull(*reinterpret_cast<unsigned long long*>(&result[a]), group_sum[a]);
  }
  return 0;
}

extern "C" int ref_max_threads(void) { return omp_get_max_threads(); }
