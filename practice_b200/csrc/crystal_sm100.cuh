// crystal_sm100.cuh -- Crystal block primitives for NVIDIA B200 (sm_100a).
//
// This header is the device-side operator API that generated query kernels
// instantiate.  Every public template keeps the name, template parameters and
// argument order of the reference's SYCL primitives so that code emitted by the
// reference's push-model visitor compiles against it unchanged:
//
//   include/crystal/load.h:6-123   BlockLoad*, BlockGather, BlockMakeRowIds,
//                                  ColumnValidAt, BlockLoadValidity,
//                                  BlockGatherValidity, BlockApplyValidityAnd
//   include/crystal/pred.h:5-445   predicate functors, InitFlags*, BlockPred*,
//                                  BlockApplyMask*, *_Cols
//   include/crystal/join.h:3-363   HASH, BlockProbe*PHT_1/2, BlockBuild*PHT_1/2,
//                                  ProbePHT_1/2, ProbeMultiHT, BlockBuildMHT_*
//   include/core/inline_math.h     db::safe_*, db::atomic_*, validity helpers
//
// Semantics follow the reference with three deliberate, documented changes that
// only matter on inputs where the reference is undefined:
//   * hash slots outside [0, ht_len) are treated as a probe miss / skipped build
//     instead of an out-of-bounds access (reference: negative HASH when a key is
//     below key_min);
//   * integer division by zero yields 0 (reference: undefined behaviour);
//   * the PHT_2 payload store happens only when the slot holds the row's key
//     after the CAS (reference join.h:205,227 stores it unconditionally; the two
//     agree whenever build keys are unique, which the PHT path requires).
//
// The header compiles under NVRTC (no standard headers) and under nvcc.
#pragma once

#if defined(__CUDACC_RTC__)
typedef unsigned long long uint64_t;
typedef long long int64_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef decltype(sizeof(0)) size_t;
#else
#include <cstddef>
#include <cstdint>
#endif

#ifndef CX_DEVICE
#define CX_DEVICE __device__ __forceinline__
#endif

// Perfect-hash slot of a dense key (join.h:3).
#define HASH(X, Y, Z) ((X - Z) % Y)

namespace cx_detail {

// Calls fn(i) for every item slot i of this thread; `guarded` restricts to the
// slots whose striped row (i*BT + tid) lies inside the tile.
template <int BT, int IPT, typename Fn>
CX_DEVICE void for_items(size_t tid, int num_items, bool guarded, Fn fn) {
  if (!guarded) {
#pragma unroll
    for (int i = 0; i < IPT; ++i) fn(i);
  } else {
#pragma unroll
    for (int i = 0; i < IPT; ++i)
      if (i * BT + (int)tid < num_items) fn(i);
  }
}

template <int BT, int IPT>
CX_DEVICE bool tile_is_full(int num_items) { return BT * IPT == num_items; }

// Slot of `key` in a perfect hash table of `len` slots, or -1 when the slot
// would fall outside the table.  A key inside [key_min, key_min + len) is its
// own offset (HASH's modulo is the identity there), so the division runs only
// for keys outside that window.
template <typename K>
CX_DEVICE int pht_slot(K key, int len, K key_min) {
  const K d = key - key_min;
  if (d >= K(0) && d < K(len)) return (int)d;
  const int h = (int)HASH(key, len, key_min);
  return ((unsigned)h < (unsigned)len) ? h : -1;
}

}  // namespace cx_detail

// ------------------------------------------------------------------ loads ---
// Striped tile layout: thread tid owns rows tid, tid+BT, ..., tid+(IPT-1)*BT.
// `block_iter` may point at global memory or at a shared-memory staging buffer.

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockLoadDirect(const T* block_iter, size_t tid, T (&items)[ITEMS_PER_THREAD]) {
  const T* p = block_iter + tid;
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, 0, false,
      [&](int i) { items[i] = p[i * BLOCK_THREADS]; });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockLoadDirect(const T* block_iter, size_t tid, T (&items)[ITEMS_PER_THREAD], int num_items) {
  const T* p = block_iter + tid;
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true,
      [&](int i) { items[i] = p[i * BLOCK_THREADS]; });
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockLoad(const T* input, size_t tid, int tile_offset, int (&items)[ITEMS_PER_THREAD], int num_items) {
  (void)tile_offset;
  if (cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items))
    BlockLoadDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(input, tid, items);
  else
    BlockLoadDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(input, tid, items, num_items);
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockGather(const T* input, int tid, int (&row_ids)[ITEMS_PER_THREAD],
                           int (&flags)[ITEMS_PER_THREAD], T (&items)[ITEMS_PER_THREAD], int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (flags[i]) items[i] = input[row_ids[i]];
  });
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockMakeRowIds(int tid, int tile_offset, int (&row_ids)[ITEMS_PER_THREAD], int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true,
      [&](int i) { row_ids[i] = tile_offset + tid + i * BLOCK_THREADS; });
}

// --------------------------------------------------------------- validity ---
// Bit r of a uint64 word array is 1 when row r is valid (load.h:72-76).

CX_DEVICE int ColumnValidAt(const uint64_t* null_bitmap, long long row_id) {
  if (null_bitmap == nullptr) return 1;
  return (int)((null_bitmap[row_id >> 6] >> (row_id & 63)) & 1ULL);
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockLoadValidity(const uint64_t* null_bitmap, int tid, long long tile_offset,
                                 int (&valid)[ITEMS_PER_THREAD], int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    const int local = i * BLOCK_THREADS + tid;
    valid[i] = (local < num_items) ? ColumnValidAt(null_bitmap, tile_offset + local) : 0;
  }
}

// Vector-striped tile layout (full warp tiles of 32 x IPT rows, no
// reference counterpart): with VW = min(IPT, 4), item i of a lane holds row
// (i / VW) * 32 * VW + lane * VW + i % VW, so each lane reads VW consecutive
// rows with one vector load and a warp covers a contiguous segment per load.
// Rows are loaded with the streaming cache hint (read once).
template <int IPT>
CX_DEVICE void WarpLoadTileV(const int* tile, int lane, int (&items)[IPT]) {
  constexpr int VW = IPT >= 4 ? 4 : IPT;
  static_assert(IPT % VW == 0, "items per thread must be 1, 2 or a multiple of 4");
#pragma unroll
  for (int v = 0; v < IPT / VW; ++v) {
    const int* p = tile + v * 32 * VW + lane * VW;
    if constexpr (VW == 4) {
      asm("ld.global.cs.v4.s32 {%0, %1, %2, %3}, [%4];"
          : "=r"(items[4 * v]), "=r"(items[4 * v + 1]), "=r"(items[4 * v + 2]), "=r"(items[4 * v + 3])
          : "l"(p));
    } else if constexpr (VW == 2) {
      asm("ld.global.cs.v2.s32 {%0, %1}, [%2];" : "=r"(items[2 * v]), "=r"(items[2 * v + 1]) : "l"(p));
    } else {
      asm("ld.global.cs.s32 %0, [%1];" : "=r"(items[v]) : "l"(p));
    }
  }
}
// Validity bits in the same vector-striped layout.
template <int IPT>
CX_DEVICE void WarpLoadValidityV(const uint64_t* null_bitmap, int lane, long long tile_offset, int (&valid)[IPT]) {
  constexpr int VW = IPT >= 4 ? 4 : IPT;
  static_assert(IPT % VW == 0 && 64 % VW == 0, "items per thread must be 1, 2 or a multiple of 4");
  if (null_bitmap == nullptr) {
#pragma unroll
    for (int i = 0; i < IPT; ++i) valid[i] = 1;
    return;
  }
  // A lane's VW rows start at a multiple of VW (tile_offset is a multiple of
  // 32 * IPT), so they share one word: one load per vector, not per row.
#pragma unroll
  for (int j = 0; j < IPT / VW; ++j) {
    const long long base = tile_offset + (long long)j * 32 * VW + lane * VW;
    const uint64_t bits = null_bitmap[base >> 6] >> (base & 63);
#pragma unroll
    for (int k = 0; k < VW; ++k) valid[j * VW + k] = (int)((bits >> k) & 1ULL);
  }
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockGatherValidity(const uint64_t* null_bitmap, int tid, int (&row_ids)[ITEMS_PER_THREAD],
                                   int (&flags)[ITEMS_PER_THREAD], int (&valid)[ITEMS_PER_THREAD], int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    const bool live = flags[i] && (i * BLOCK_THREADS + tid < num_items);
    valid[i] = live ? ColumnValidAt(null_bitmap, row_ids[i]) : 0;
  }
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockApplyValidityAnd(int tid, int (&flags)[ITEMS_PER_THREAD], int (&valid)[ITEMS_PER_THREAD],
                                     int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true,
      [&](int i) { flags[i] = flags[i] && valid[i]; });
}

// ------------------------------------------------------------- predicates ---

template <typename T> struct GreaterThan {
  T _compare;
  CX_DEVICE GreaterThan(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v > _compare; }
};
template <typename T> struct LessThan {
  T _compare;
  CX_DEVICE LessThan(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v < _compare; }
};
template <typename T> struct GreaterThanEq {
  T _compare;
  CX_DEVICE GreaterThanEq(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v >= _compare; }
};
template <typename T> struct LessThanEq {
  T _compare;
  CX_DEVICE LessThanEq(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v <= _compare; }
};
template <typename T> struct Equal {
  T _compare;
  CX_DEVICE Equal(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v == _compare; }
};
template <typename T> struct NotEqual {
  T _compare;
  CX_DEVICE NotEqual(T c) : _compare(c) {}
  CX_DEVICE bool operator()(const T& v) const { return v != _compare; }
};

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void InitFlags(int (&flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) flags[i] = 1;
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void InitFlagsZero(int (&flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) flags[i] = 0;
}

namespace cx_detail {
// Combine mode of a predicate with the incoming flag: set, AND, OR.
enum class Comb { Set, And, Or };
template <Comb C> CX_DEVICE int combine(int flag, bool p) {
  if (C == Comb::Set) return p ? 1 : 0;
  if (C == Comb::And) return (flag && p) ? 1 : 0;
  return (flag || p) ? 1 : 0;
}
template <Comb C, typename T, typename P, int BT, int IPT>
CX_DEVICE void pred_apply(size_t tid, T (&items)[IPT], int (&flags)[IPT], P pred, int num_items, bool guarded) {
  for_items<BT, IPT>(tid, num_items, guarded, [&](int i) { flags[i] = combine<C>(flags[i], pred(items[i])); });
}
template <Comb C, typename T, typename P, int BT, int IPT>
CX_DEVICE void pred_dispatch(size_t tid, T (&items)[IPT], int (&flags)[IPT], P pred, int num_items) {
  pred_apply<C, T, P, BT, IPT>(tid, items, flags, pred, num_items, !tile_is_full<BT, IPT>(num_items));
}
}  // namespace cx_detail

template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred) {
  cx_detail::pred_apply<cx_detail::Comb::Set, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, 0, false);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_apply<cx_detail::Comb::Set, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items, true);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPred(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_dispatch<cx_detail::Comb::Set, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredAndDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred) {
  cx_detail::pred_apply<cx_detail::Comb::And, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, 0, false);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredAndDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_apply<cx_detail::Comb::And, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items, true);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredAnd(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_dispatch<cx_detail::Comb::And, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredOrDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred) {
  cx_detail::pred_apply<cx_detail::Comb::Or, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, 0, false);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredOrDirect(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_apply<cx_detail::Comb::Or, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items, true);
}
template <typename T, typename Predicate, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockPredOr(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], Predicate pred, int num_items) {
  cx_detail::pred_dispatch<cx_detail::Comb::Or, T, Predicate, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, pred, num_items);
}

// Literal comparisons: BlockPred<Op> sets, BlockPredA<Op> ANDs, BlockPredO<Op>
// (BlockPredOr<Op> for Eq/NEq) ORs into flags (pred.h:153-260).
#define CX_LITERAL_PRED(NAME, FUNCTOR, DISPATCH)                                                     \
  template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                     \
  CX_DEVICE void NAME(size_t tid, T (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],      \
                      T compare, int num_items) {                                                    \
    DISPATCH<T, FUNCTOR<T>, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, FUNCTOR<T>(compare), \
                                                             num_items);                             \
  }
CX_LITERAL_PRED(BlockPredLT, LessThan, BlockPred)
CX_LITERAL_PRED(BlockPredALT, LessThan, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOLT, LessThan, BlockPredOr)
CX_LITERAL_PRED(BlockPredGT, GreaterThan, BlockPred)
CX_LITERAL_PRED(BlockPredAGT, GreaterThan, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOGT, GreaterThan, BlockPredOr)
CX_LITERAL_PRED(BlockPredLTE, LessThanEq, BlockPred)
CX_LITERAL_PRED(BlockPredALTE, LessThanEq, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOLTE, LessThanEq, BlockPredOr)
CX_LITERAL_PRED(BlockPredGTE, GreaterThanEq, BlockPred)
CX_LITERAL_PRED(BlockPredAGTE, GreaterThanEq, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOGTE, GreaterThanEq, BlockPredOr)
CX_LITERAL_PRED(BlockPredEq, Equal, BlockPred)
CX_LITERAL_PRED(BlockPredAEq, Equal, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOrEq, Equal, BlockPredOr)
CX_LITERAL_PRED(BlockPredNEq, NotEqual, BlockPred)
CX_LITERAL_PRED(BlockPredANEq, NotEqual, BlockPredAnd)
CX_LITERAL_PRED(BlockPredOrNEq, NotEqual, BlockPredOr)
#undef CX_LITERAL_PRED

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockApplyMaskOr(size_t tid, int (&target_mask)[ITEMS_PER_THREAD], int (&source_mask)[ITEMS_PER_THREAD]) {
  (void)tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) target_mask[i] = (target_mask[i] || source_mask[i]) ? 1 : 0;
}

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockApplyMaskAnd(size_t tid, int (&target_mask)[ITEMS_PER_THREAD], int (&source_mask)[ITEMS_PER_THREAD]) {
  (void)tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) target_mask[i] = (target_mask[i] && source_mask[i]) ? 1 : 0;
}

// Column-vs-column comparisons (pred.h:264-445); always guarded by the tile size.
#define CX_COLS_PRED(NAME, COMB, OP)                                                                   \
  template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                       \
  CX_DEVICE void NAME(size_t tid, T (&items1)[ITEMS_PER_THREAD], T (&items2)[ITEMS_PER_THREAD],        \
                      int (&flags)[ITEMS_PER_THREAD], int num_items) {                                 \
    cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {           \
      flags[i] = cx_detail::combine<cx_detail::Comb::COMB>(flags[i], items1[i] OP items2[i]);          \
    });                                                                                                \
  }
CX_COLS_PRED(BlockPredEq_Cols, Set, ==)
CX_COLS_PRED(BlockPredAEq_Cols, And, ==)
CX_COLS_PRED(BlockPredOrEq_Cols, Or, ==)
CX_COLS_PRED(BlockPredNEq_Cols, Set, !=)
CX_COLS_PRED(BlockPredANEq_Cols, And, !=)
CX_COLS_PRED(BlockPredOrNEq_Cols, Or, !=)
CX_COLS_PRED(BlockPredLT_Cols, Set, <)
CX_COLS_PRED(BlockPredALT_Cols, And, <)
CX_COLS_PRED(BlockPredOrLT_Cols, Or, <)
CX_COLS_PRED(BlockPredLTE_Cols, Set, <=)
CX_COLS_PRED(BlockPredALTE_Cols, And, <=)
CX_COLS_PRED(BlockPredOrLTE_Cols, Or, <=)
CX_COLS_PRED(BlockPredGT_Cols, Set, >)
CX_COLS_PRED(BlockPredAGT_Cols, And, >)
CX_COLS_PRED(BlockPredOrGT_Cols, Or, >)
CX_COLS_PRED(BlockPredGTE_Cols, Set, >=)
CX_COLS_PRED(BlockPredAGTE_Cols, And, >=)
CX_COLS_PRED(BlockPredOrGTE_Cols, Or, >=)
#undef CX_COLS_PRED

// ------------------------------------------------- perfect hash tables (PHT) ---
// PHT_1 stores keys only: ht[slot] = key.  PHT_2 stores pairs:
// ht[2*slot] = key, ht[2*slot+1] = payload.  Empty slots hold 0, so build keys
// must be non-zero (join.h:140-141).

namespace cx_detail {
template <typename K, typename V, int BT, int IPT, bool PAIR>
CX_DEVICE void pht_probe(int tid, K (&items)[IPT], V* res, int (&flags)[IPT], const K* ht, int ht_len, K key_min,
                         int num_items, bool guarded) {
  const bool pair8 = PAIR && sizeof(K) == 4 && (reinterpret_cast<unsigned long long>(ht) & 7ULL) == 0ULL;
  for_items<BT, IPT>(tid, num_items, guarded, [&](int i) {
    if (!flags[i]) return;
    const int h = pht_slot<K>(items[i], ht_len, key_min);
    if (h < 0) { flags[i] = 0; return; }
    if (PAIR) {
      K k, v;
      if (pair8) {
        // Key and payload of a slot are adjacent: one 8-byte load.
        const int2 kv = *reinterpret_cast<const int2*>(ht + ((long long)h << 1));
        k = (K)kv.x;
        v = (K)kv.y;
      } else {
        k = ht[(long long)h << 1];
        v = ht[((long long)h << 1) + 1];
      }
      if (k == items[i]) res[i] = static_cast<V>(v);
      else flags[i] = 0;
    } else {
      flags[i] = (ht[h] == items[i]) ? 1 : 0;
    }
  });
}
template <typename K, typename V, int BT, int IPT, bool PAIR>
CX_DEVICE void pht_build(int tid, K (&keys)[IPT], V* vals, int (&flags)[IPT], K* ht, int ht_len, K key_min,
                         int num_items, bool guarded) {
  for_items<BT, IPT>(tid, num_items, guarded, [&](int i) {
    if (!flags[i]) return;
    const int h = pht_slot<K>(keys[i], ht_len, key_min);
    if (h < 0) return;
    if (PAIR) {
      const K prev = atomicCAS(&ht[(long long)h << 1], K(0), keys[i]);
      if (prev == K(0) || prev == keys[i]) ht[((long long)h << 1) + 1] = static_cast<K>(vals[i]);
    } else {
      atomicCAS(&ht[h], K(0), keys[i]);
    }
  });
}
}  // namespace cx_detail

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                        const K* ht, int ht_len, K key_mins) {
  cx_detail::pht_probe<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(tid, items, (K*)nullptr, flags, ht, ht_len, key_mins, 0, false);
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                        const K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_probe<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(tid, items, (K*)nullptr, flags, ht, ht_len, key_mins, num_items, true);
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                  const K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_probe<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(
      tid, items, (K*)nullptr, flags, ht, ht_len, key_mins, num_items,
      !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items));
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                  const K* ht, int ht_len, int num_items) {
  BlockProbeAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeDirectAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                        int (&flags)[ITEMS_PER_THREAD], const K* ht, int ht_len, K key_mins) {
  cx_detail::pht_probe<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(tid, items, res, flags, ht, ht_len, key_mins, 0, false);
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeDirectAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                        int (&flags)[ITEMS_PER_THREAD], const K* ht, int ht_len, K key_mins,
                                        int num_items) {
  cx_detail::pht_probe<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(tid, items, res, flags, ht, ht_len, key_mins, num_items, true);
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                  int (&flags)[ITEMS_PER_THREAD], const K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_probe<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(
      tid, items, res, flags, ht, ht_len, key_mins, num_items,
      !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items));
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                  int (&flags)[ITEMS_PER_THREAD], const K* ht, int ht_len, int num_items) {
  BlockProbeAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, items, res, flags, ht, ht_len, K(0), num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildDirectSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                              K* ht, int ht_len, K key_mins) {
  cx_detail::pht_build<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(tid, keys, (K*)nullptr, flags, ht, ht_len, key_mins, 0, false);
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildDirectSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                              K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_build<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(tid, keys, (K*)nullptr, flags, ht, ht_len, key_mins, num_items, true);
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                        K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_build<K, K, BLOCK_THREADS, ITEMS_PER_THREAD, false>(
      tid, keys, (K*)nullptr, flags, ht, ht_len, key_mins, num_items,
      !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items));
}
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                        K* ht, int ht_len, int num_items) {
  BlockBuildSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, keys, flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                              int (&flags)[ITEMS_PER_THREAD], K* ht, int ht_len, K key_mins) {
  cx_detail::pht_build<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(tid, keys, res, flags, ht, ht_len, key_mins, 0, false);
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                              int (&flags)[ITEMS_PER_THREAD], K* ht, int ht_len, K key_mins,
                                              int num_items) {
  cx_detail::pht_build<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(tid, keys, res, flags, ht, ht_len, key_mins, num_items, true);
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                        int (&flags)[ITEMS_PER_THREAD], K* ht, int ht_len, K key_mins, int num_items) {
  cx_detail::pht_build<K, V, BLOCK_THREADS, ITEMS_PER_THREAD, true>(
      tid, keys, res, flags, ht, ht_len, key_mins, num_items,
      !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items));
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                        int (&flags)[ITEMS_PER_THREAD], K* ht, int ht_len, int num_items) {
  BlockBuildSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(tid, keys, res, flags, ht, ht_len, K(0), num_items);
}

// Validity-carrying PHT_2 extension.  The reference stores a dimension payload
// without its NULL bit, so a NULL payload column cannot form a NULL group.
// These variants keep one validity bit per slot in `ht_valid` (len bits).  They
// have no counterpart in the reference API.
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildSelectivePHT_2V(int tid, K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                         int (&res_valid)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], K* ht,
                                         unsigned int* ht_valid, int ht_len, K key_mins, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (!flags[i]) return;
    const int h = cx_detail::pht_slot<K>(keys[i], ht_len, key_mins);
    if (h < 0) return;
    const K prev = atomicCAS(&ht[(long long)h << 1], K(0), keys[i]);
    if (prev == K(0) || prev == keys[i]) {
      ht[((long long)h << 1) + 1] = static_cast<K>(res[i]);
      if (res_valid[i]) atomicOr(&ht_valid[h >> 5], 1u << (h & 31));
    }
  });
}
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeAndPHT_2V(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                   int (&res_valid)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD], const K* ht,
                                   const unsigned int* ht_valid, int ht_len, K key_mins, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (!flags[i]) return;
    const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_mins);
    if (h < 0 || ht[(long long)h << 1] != items[i]) { flags[i] = 0; return; }
    res[i] = static_cast<V>(ht[((long long)h << 1) + 1]);
    res_valid[i] = (int)((ht_valid[h >> 5] >> (h & 31)) & 1u);
  });
}

// Membership pre-filter from a slot-occupancy bitmap (bit h = slot h of the
// PHT holds a key), typically copied into shared memory.  Clears the flag of
// every item whose slot is empty or out of range; a key of 0 keeps its flag on
// an empty slot because the PHT probe matches 0 against the empty sentinel
// (join.h:7-41).  Exact: a following BlockProbeAndPHT_* confirms the key.  No
// counterpart in the reference API.
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeBitmapAnd(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                   const unsigned int* bitmap, int ht_len, K key_mins, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items), [&](int i) {
    if (!flags[i]) return;
    const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_mins);
    if (h < 0) { flags[i] = 0; return; }
    const bool occupied = (bitmap[h >> 5] >> (h & 31)) & 1u;
    flags[i] = (occupied || items[i] == K(0)) ? 1 : 0;
  });
}

// Exact membership from a slot bitmap in which bit h is set when slot h of a
// finished PHT holds the key key_min + h.  For a key inside the window
// [key_min, key_min + len) that bit is the probe's answer (HASH maps the key
// to slot key - key_min), so no table access is needed; a key outside the
// window falls back to the full probe of `ht` (`pair` = 1 for [key, payload]
// slots).  Clears the flag of every item that misses.  The in-window test is
// branch-free (an outside key reads bit 0 of word 0 and masks it off); the
// items with an outside key and a set flag are probed afterwards, behind one
// branch per call instead of one per item.  No counterpart in the reference
// API.
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeExactBitmap(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                     const unsigned int* bitmap, const K* ht, int pair, int ht_len, K key_min,
                                     int num_items) {
  static_assert(ITEMS_PER_THREAD <= 32, "one bit per item");
  const bool guarded = !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items);
  unsigned outside = 0u;  // bit i: item i's key lies outside the window and its flag is set
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    const bool live = !guarded || i * BLOCK_THREADS + tid < num_items;
    const K d = items[i] - key_min;
    const bool in = sizeof(K) == 4 ? (unsigned)d < (unsigned)ht_len : (d >= K(0) && d < K(ht_len));
    const unsigned o = in ? (unsigned)d : 0u;
    const int hit = (int)((bitmap[o >> 5] >> (o & 31u)) & 1u) & (int)in;
    const int f = (int)(flags[i] != 0);
    outside |= (unsigned)(live && !in && f) << i;
    flags[i] = live ? (f & hit) : flags[i];
  }
  if (outside) {
#pragma unroll
    for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
      if (!((outside >> i) & 1u)) continue;
      const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_min);
      flags[i] = (h >= 0 && ht[(long long)h << pair] == items[i]) ? 1 : 0;
    }
  }
}

// Exact membership from a payload table in shared memory: byte h is 0xFF when
// slot h does not hold the key key_min + h, else the slot's payload minus its
// catalog minimum, or 0xFE for a payload outside the catalog range.  Keys
// outside the table's window probe the PHT (pair layout).
template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockProbeExactTable(int tid, K (&items)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                    const unsigned char* table, const K* ht, int ht_len, K key_min, int num_items) {
  const bool guarded = !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items);
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (guarded && i * BLOCK_THREADS + tid >= num_items) continue;
    const K d = items[i] - key_min;
    int hit;
    if (sizeof(K) == 4 ? (unsigned)d < (unsigned)ht_len : (d >= K(0) && d < K(ht_len))) {
      hit = table[(unsigned)d] != 0xFFu;
    } else {
      hit = 0;
      if (flags[i]) {
        const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_min);
        hit = (h >= 0 && ht[(long long)h << 1] == items[i]) ? 1 : 0;
      }
    }
    flags[i] = (int)(flags[i] != 0) & hit;
  }
}

// The payload of every flagged item from the same table (membership already
// known): its catalog minimum plus the byte, or the PHT's payload where the
// byte is 0xFE or the key lies outside the window.
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockFetchPayloadTable(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                      int (&flags)[ITEMS_PER_THREAD], const unsigned char* table, const K* ht,
                                      int ht_len, K key_min, V value_min, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(
      tid, num_items, !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items), [&](int i) {
        if (!flags[i]) return;
        const K d = items[i] - key_min;
        const unsigned b = (sizeof(K) == 4 ? (unsigned)d < (unsigned)ht_len : (d >= K(0) && d < K(ht_len)))
                               ? (unsigned)table[(unsigned)d]
                               : 0xFEu;
        if (b < 0xFEu) {
          res[i] = value_min + static_cast<V>(b);
        } else {
          const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_min);
          if (h >= 0) res[i] = static_cast<V>(ht[((long long)h << 1) + 1]);
        }
      });
}

// PHT_2 payload of every flagged item whose membership is already known (the
// slot of its key holds the key): one table load per qualifying row.
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockFetchPayloadPHT_2(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                      int (&flags)[ITEMS_PER_THREAD], const K* ht, int ht_len, K key_min,
                                      int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(
      tid, num_items, !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items), [&](int i) {
        if (!flags[i]) return;
        const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_min);
        if (h >= 0) res[i] = static_cast<V>(ht[((long long)h << 1) + 1]);
      });
}
// The same with the payload's validity bit (PHT_2V tables).
template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockFetchPayloadPHT_2V(int tid, K (&items)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                       int (&res_valid)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                       const K* ht, const unsigned int* ht_valid, int ht_len, K key_min,
                                       int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(
      tid, num_items, !cx_detail::tile_is_full<BLOCK_THREADS, ITEMS_PER_THREAD>(num_items), [&](int i) {
        if (!flags[i]) return;
        const int h = cx_detail::pht_slot<K>(items[i], ht_len, key_min);
        if (h < 0) return;
        res[i] = static_cast<V>(ht[((long long)h << 1) + 1]);
        res_valid[i] = (int)((ht_valid[h >> 5] >> (h & 31)) & 1u);
      });
}

// Push-model thread-local probes (join.h:258-274).
template <typename K>
CX_DEVICE bool ProbePHT_1(K key, const K* ht, int ht_len, K key_mins) {
  const int h = cx_detail::pht_slot<K>(key, ht_len, key_mins);
  return h >= 0 && ht[h] == key;
}
template <typename K, typename V>
CX_DEVICE bool ProbePHT_2(K key, V& res, const K* ht, int ht_len, K key_mins) {
  const int h = cx_detail::pht_slot<K>(key, ht_len, key_mins);
  if (h < 0 || ht[(long long)h << 1] != key) return false;
  res = static_cast<V>(ht[((long long)h << 1) + 1]);
  return true;
}

// ------------------------------------------- multi-value hash tables (MHT) ---
// Directory entry per slot: [key, offset, count] (join.h:276-363).

template <typename K>
CX_DEVICE void ProbeMultiHT(K key, int& offset, int& count, int& flag, const K* ht_dir, int ht_len, K key_mins) {
  count = 0;
  if (!flag) return;
  const int h = cx_detail::pht_slot<K>(key, ht_len, key_mins);
  const K* e = (h >= 0) ? ht_dir + 3LL * h : nullptr;
  if (e && e[0] == key && e[2] > 0) {
    offset = e[1];
    count = e[2];
  } else {
    flag = 0;
  }
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildMHT_Count(int tid, K (&keys)[ITEMS_PER_THREAD], int (&flags)[ITEMS_PER_THREAD],
                                   int* d_counts, int ht_len, K key_mins, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (!flags[i]) return;
    const int h = cx_detail::pht_slot<K>(keys[i], ht_len, key_mins);
    if (h >= 0) atomicAdd(&d_counts[h], 1);
  });
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
CX_DEVICE void BlockBuildMHT_Write(int tid, K (&keys)[ITEMS_PER_THREAD], V (&vals)[ITEMS_PER_THREAD],
                                   int (&flags)[ITEMS_PER_THREAD], int* ht_dir, int* d_offsets, int* d_write_pos,
                                   int* d_counts, int* payload, int ht_len, K key_mins, int num_items) {
  cx_detail::for_items<BLOCK_THREADS, ITEMS_PER_THREAD>(tid, num_items, true, [&](int i) {
    if (!flags[i]) return;
    const int h = cx_detail::pht_slot<K>(keys[i], ht_len, key_mins);
    if (h < 0) return;
    const int pos = d_offsets[h] + atomicAdd(&d_write_pos[h], 1);
    payload[pos] = (int)vals[i];
    ht_dir[3LL * h + 0] = (int)keys[i];
    ht_dir[3LL * h + 1] = d_offsets[h];
    ht_dir[3LL * h + 2] = d_counts[h];
  });
}

// ---------------------------------------------------------- inline math ---
namespace db {

// Promotion used by predicate arithmetic (inline_math.h:8-13).
template <typename T> struct PromoteType { using type = T; };
template <> struct PromoteType<int> { using type = long long; };
template <> struct PromoteType<unsigned int> { using type = unsigned long long; };
template <> struct PromoteType<float> { using type = double; };

template <typename A, typename B>
struct Promoted {
  using PA = typename PromoteType<A>::type;
  using PB = typename PromoteType<B>::type;
  using type = decltype(PA() + PB());
};

template <typename A, typename B>
CX_DEVICE auto safe_add(A a, B b) { using C = typename Promoted<A, B>::type; return (C)a + (C)b; }
template <typename A, typename B>
CX_DEVICE auto safe_sub(A a, B b) { using C = typename Promoted<A, B>::type; return (C)a - (C)b; }
template <typename A, typename B>
CX_DEVICE auto safe_mul(A a, B b) { using C = typename Promoted<A, B>::type; return (C)a * (C)b; }
template <typename A, typename B>
CX_DEVICE auto safe_div(A a, B b) {
  using C = typename Promoted<A, B>::type;
  return ((C)b == (C)0) ? (C)0 : (C)a / (C)b;
}

#define CX_SAFE_CMP(NAME, OP)                                                         \
  template <typename A, typename B>                                                   \
  CX_DEVICE int NAME(A a, B b) {                                                      \
    using C = typename Promoted<A, B>::type;                                          \
    return ((C)a OP (C)b) ? 1 : 0;                                                    \
  }
CX_SAFE_CMP(safe_lt, <)
CX_SAFE_CMP(safe_gt, >)
CX_SAFE_CMP(safe_lte, <=)
CX_SAFE_CMP(safe_gte, >=)
CX_SAFE_CMP(safe_eq, ==)
CX_SAFE_CMP(safe_neq, !=)
#undef CX_SAFE_CMP

CX_DEVICE unsigned long long bit_cast_double_to_ull(double v) { return (unsigned long long)__double_as_longlong(v); }
CX_DEVICE double bit_cast_ull_to_double(unsigned long long v) { return __longlong_as_double((long long)v); }

// Relaxed device-scope 64-bit atomics on global or shared memory.
CX_DEVICE unsigned long long atomic_fetch_add_ull(unsigned long long& t, unsigned long long v) { return atomicAdd(&t, v); }
CX_DEVICE void atomic_add_ull(unsigned long long& t, unsigned long long v) { atomicAdd(&t, v); }
CX_DEVICE void atomic_min_ull(unsigned long long& t, unsigned long long v) { atomicMin(&t, v); }
CX_DEVICE void atomic_max_ull(unsigned long long& t, unsigned long long v) { atomicMax(&t, v); }

CX_DEVICE void atomic_set_valid_bit(uint64_t* bitmap, unsigned long long bit) {
  if (bitmap == nullptr) return;
  atomicOr((unsigned long long*)&bitmap[bit >> 6], 1ULL << (bit & 63ULL));
}
CX_DEVICE int bitmap_valid_at(const uint64_t* bitmap, unsigned long long bit) {
  if (bitmap == nullptr) return 1;
  return (int)((bitmap[bit >> 6] >> (bit & 63ULL)) & 1ULL);
}

}  // namespace db

// ================================================================ sm_100a ===
// Runtime pieces the generated kernels use around the primitives: TMA bulk
// staging of fact-column tiles into shared memory, bounded mbarrier waits,
// warp-aggregated group updates and block reductions.

namespace cx {

// Error codes a kernel can raise in its error word (first writer wins).
enum : unsigned int {
  ERR_NONE = 0,
  ERR_WAIT_TIMEOUT = 1,      // an mbarrier wait exceeded its time limit
  ERR_GROUP_DOMAIN = 2,      // a GROUP BY key fell outside its catalog domain
  ERR_SCRATCH = 3,           // scratch too small for the requested table
  ERR_DIM_COLLISION = 4,     // two distinct dimension keys share a slot of a shared-scan
                             // index or of a multi-value hash table
  ERR_CUBE_RANGE = 5,        // a value outside the registered range of a cube attribute
};

CX_DEVICE void raise(unsigned int* err, unsigned int code) {
  if (err) atomicCAS(err, 0u, code);
}

CX_DEVICE unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

CX_DEVICE void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
CX_DEVICE void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
CX_DEVICE void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

CX_DEVICE void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

CX_DEVICE void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

CX_DEVICE bool mbar_try_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: the thread sleeps in the barrier until the
// phase completes or about `ns` nanoseconds pass, instead of spinning.
CX_DEVICE bool mbar_try_wait_sleep(unsigned long long* bar, unsigned phase, unsigned ns) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase), "r"(ns)
      : "memory");
  return ok != 0;
}

// Nanoseconds of the GPU's global timer.
CX_DEVICE unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for phase `phase` of `bar`; gives up once `limit_us` microseconds
// (global timer) have passed.  Returns false on timeout so the caller can
// record an error and leave.  After a few quick polls each poll sleeps in the
// barrier (up to 2 us), so waiting warps leave their issue slots to the warps
// that work.
CX_DEVICE bool mbar_wait_bounded(unsigned long long* bar, unsigned phase, unsigned limit_us) {
#pragma unroll 1
  for (int it = 0; it < 8; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  const unsigned long long t0 = global_ns();
  const unsigned long long lim = (unsigned long long)limit_us * 1000ULL;
#pragma unroll 1
  while (true) {
    if (mbar_try_wait_sleep(bar, phase, 2000u)) return true;
    if (global_ns() - t0 > lim) return false;
  }
}

// Test hook of the bounded-wait error path: every thread of the CTA waits on
// a barrier that nothing arrives at, so the wait runs out after `limit_us`
// and thread 0 records ERR_WAIT_TIMEOUT.  Called first thing in a kernel, with
// no copy in flight; the caller returns right after it.
CX_DEVICE void debug_stall(unsigned long long* bar, unsigned int* err, unsigned limit_us);

// Limit of the waits that collect a CTA's own bulk copies after another wait
// gave up: never shorter than 200 ms, far above the few microseconds a copy
// in flight needs to land, so no copy lands in shared memory after the CTA
// has exited whatever limit the caller chose.
CX_DEVICE unsigned drain_limit_us(unsigned limit_us) { return limit_us > 200000u ? limit_us : 200000u; }

// After a staging wait gave up, waits (bounded) for the copies this warp still
// has in flight -- local iterations k_iter .. k_iter+nstage-1 of its tile
// sequence first, first+stride, ... -- so no bulk copy lands in shared memory
// after the CTA has exited.  Cold path, kept out of line.
static __device__ __noinline__ void drain_stages(unsigned long long* bars, int nstage, long long k_iter,
                                                 long long first, long long stride, long long full_tiles,
                                                 unsigned limit);

// L2 policy that marks streamed fact bytes evict-first so dimension hash tables
// stay resident in L2.
CX_DEVICE unsigned long long l2_evict_first_policy() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// One bulk (non-tensor) TMA copy global -> this CTA's shared memory, completing
// on `bar`.  Both addresses 16-byte aligned, bytes a multiple of 16.  No
// multicast.
CX_DEVICE void bulk_g2s(void* smem_dst, const void* gmem_src, unsigned bytes, unsigned long long* bar,
                        unsigned long long policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// Store of one 32-bit word to shared memory under a predicate: a lane whose
// predicate is false issues nothing, and no branch is needed around the store.
// `addr` must point into shared memory (it is converted to a shared-window
// address); it is not accessed when `pred` is false.
CX_DEVICE void st_shared_if(bool pred, int* addr, int v) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(addr);
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p st.shared.b32 [%0], %1;\n\t}" ::"r"(a), "r"(v),
      "r"((unsigned)pred)
      : "memory");
}

// Bulk prefetch of `bytes` of global memory into L2 (no destination, no
// completion to wait for): a warp asks for its next tile's columns a tile ahead
// at no register cost.  Address 16-byte aligned, bytes a multiple of 16, the
// range inside the buffer.
CX_DEVICE void l2_prefetch_bulk(const void* gmem_src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gmem_src), "r"(bytes) : "memory");
}

CX_DEVICE void debug_stall(unsigned long long* bar, unsigned int* err, unsigned limit_us) {
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (!mbar_wait_bounded(bar, 0u, limit_us) && threadIdx.x == 0) raise(err, ERR_WAIT_TIMEOUT);
}

static __device__ __noinline__ void drain_stages(unsigned long long* bars, int nstage, long long k_iter,
                                                 long long first, long long stride, long long full_tiles,
                                                 unsigned limit) {
  for (int j = 0; j < nstage; ++j) {
    const long long kk = k_iter + j;
    const long long tt = first + kk * stride;
    if (tt < full_tiles) (void)mbar_wait_bounded(&bars[kk % nstage], (unsigned)((kk / nstage) & 1), drain_limit_us(limit));
  }
}

// Exclusive prefix sum of a 64-bit value over the CTA (every thread gets the
// sum of the values of lower-numbered threads); `*total` receives the CTA sum
// in every thread.  `scratch` holds BT/32 + 1 words.
template <int BT>
CX_DEVICE long long block_exclusive_scan_i64(long long v, long long* scratch, long long* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  __syncthreads();
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int w = 0; w < BT / 32; ++w) {
      const long long t = scratch[w];
      scratch[w] = run;
      run += t;
    }
    scratch[BT / 32] = run;
  }
  __syncthreads();
  *total = scratch[BT / 32];
  return scratch[warp] + inc - v;
}

// Sum of a 64-bit value over the CTA; the result is valid in thread 0.
template <int BT>
CX_DEVICE unsigned long long block_sum_u64(unsigned long long v, unsigned long long* scratch /* BT/32 */) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  unsigned long long s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) s += scratch[w];
  return s;
}
template <int BT>
CX_DEVICE unsigned long long block_min_u64(unsigned long long v, unsigned long long* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long u = __shfl_down_sync(0xffffffffu, v, o);
    v = u < v ? u : v;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  unsigned long long s = ~0ULL;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) s = scratch[w] < s ? scratch[w] : s;
  return s;
}
template <int BT>
CX_DEVICE unsigned long long block_max_u64(unsigned long long v, unsigned long long* scratch) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long u = __shfl_down_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  unsigned long long s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) s = scratch[w] > s ? scratch[w] : s;
  return s;
}

// The reference's sycl::reduce_over_group over one work-group of BT threads
// (OP 0 sum, 1 minimum, 2 maximum of unsigned 64-bit values): every thread
// receives the CTA's result.  `scratch` holds BT/32 + 1 words; every thread
// of the CTA must make the call.
template <int BT, int OP>
CX_DEVICE unsigned long long group_reduce_u64(unsigned long long v, unsigned long long* scratch) {
  const unsigned long long r = OP == 0 ? block_sum_u64<BT>(v, scratch)
                               : OP == 1 ? block_min_u64<BT>(v, scratch)
                                         : block_max_u64<BT>(v, scratch);
  __syncthreads();
  if (threadIdx.x == 0) scratch[BT / 32] = r;
  __syncthreads();
  return scratch[BT / 32];
}

// Bitwise OR of a 32-bit value over the CTA; the result is valid in thread 0.
template <int BT>
CX_DEVICE unsigned block_or_u32(unsigned v, unsigned long long* scratch) {
  v = __reduce_or_sync(0xffffffffu, v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  unsigned s = 0u;
  if (threadIdx.x == 0)
    for (int w = 0; w < BT / 32; ++w) s |= (unsigned)scratch[w];
  return s;
}

// Warp-aggregated update of a group table.  Every lane of the warp must call
// this (inactive lanes pass active=false).  Lanes that target the same group
// are merged with __match_any_sync and a shuffle reduction; one lane per
// distinct group then applies `apply(group, sum)`.
template <typename Apply>
CX_DEVICE void warp_group_add(bool active, int group, unsigned long long v, Apply apply) {
  const unsigned key = active ? (unsigned)group : 0xffffffffu;
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  if (!active) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  unsigned long long sum = 0;
  for (unsigned m = peers; m; m &= m - 1) {
    const int src = __ffs(m) - 1;
    const unsigned long long x = __shfl_sync(peers, v, src);
    sum += x;
  }
  if (lane == leader) apply(group, sum);
}

// 32x32 bit-matrix transpose across a warp: lane r passes row r; lane c gets
// column c (bit r of the result = bit c of lane r's row).  Five exchange
// steps swap the off-diagonal blocks of 16, 8, 4, 2 and 1 bits (the
// recursive block transpose of Hacker's Delight 7-3, one row per lane).
// Every lane of the warp must call it.
CX_DEVICE unsigned warp_transpose32(unsigned x, int lane) {
  const unsigned masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int j = 16 >> s;
    const unsigned m = masks[s];
    const unsigned y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~m) | ((y >> j) & m)) : ((x & m) | ((y << j) & ~m));
  }
  return x;
}

// Warp reduce-scatter of P (a power of two <= 32) per-lane u64 values.  Each
// exchange step halves the values a lane carries: the lane keeps the half its
// lane bit selects and adds the partner's copy of it; once one value is left
// the remaining steps are a plain butterfly.  Returns the value index whose
// warp total the lane then holds in v[0]; lanes with (lane & (32 / P - 1)) == 0
// hold each index exactly once.  Every lane of the warp must call it.
template <int P>
CX_DEVICE int warp_reduce_scatter_u64(unsigned long long (&v)[P], int lane) {
  static_assert(P >= 1 && P <= 32 && (P & (P - 1)) == 0, "P must be a power of two <= 32");
  int idx = 0;
  int cnt = P;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    if (cnt > 1) {
      const int h = cnt / 2;
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < h; ++k) {
        const unsigned long long send = up ? v[k] : v[k + h];
        const unsigned long long keep = up ? v[k + h] : v[k];
        v[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
      if (up) idx += h;
      cnt = h;
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    }
  }
  return idx;
}


}  // namespace cx

