// cx_finalize.cu -- aggregate result finalisation on the device.
//
// The reference's generated post-processing turns the group table into
// columnar result rows (AggregateDenseCount / AggregateDenseWrite,
// src/core/visitor.cpp:2589-2697: a group is present when its visible tuple
// has a validity bit or a non-zero word; a scalar aggregate always yields one
// row; rows in group order), then orders and cuts them (SortLimit*,
// src/core/visitor.cpp:307-581: each key compared in the column's result type,
// a valid value before NULL, ties broken by row index; then LIMIT).  Here the
// row offsets come from a device prefix sum (the reference copies counts to
// the host), and ORDER BY sorts row indices with a bitonic network: inside one
// CTA's shared memory up to 2048 rows, else in global memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "../../include/crystal_b200.h"
#include "cx_internal.h"

namespace {

int ffail(int code, const char* msg) { return cx_internal::set_error(code, msg); }

int fcuda(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  return cx_internal::set_error(CX_E_CUDA, buf);
}

constexpr int kMaxCols = 32;
constexpr int kMaxKeys = 8;
constexpr int kBlock = 256;
constexpr unsigned long long kPerBlock = 2048;  // groups per block of the count / write passes
constexpr unsigned kInvalid = 0xffffffffu;

struct FinDesc {
  unsigned long long groups;
  unsigned ts, cols;
  int sparse, scalar;
  unsigned char type[kMaxCols];      // CX_COL_INT64 / UINT64 / FLOAT64
  unsigned char nullable[kMaxCols];
  int nkeys;
  int key_col[kMaxKeys];
  int key_desc[kMaxKeys];
};

__device__ __forceinline__ bool bit_at(const unsigned long long* v, unsigned long long i) {
  return (v[i >> 6] >> (i & 63)) & 1ULL;
}

__device__ __forceinline__ bool present(const unsigned long long* __restrict__ src,
                                        const unsigned long long* __restrict__ val, const FinDesc& d,
                                        unsigned long long g) {
  if (d.scalar) return true;
  const unsigned long long base = g * d.ts;
  if (d.sparse) {
    for (unsigned c = 0; c < d.ts; ++c)
      if (src[base + c] != 0ULL) return true;
    return false;
  }
  for (unsigned c = 0; c < d.cols; ++c)
    if ((val && bit_at(val, base + c)) || src[base + c] != 0ULL) return true;
  return false;
}

// Pass 1: present groups per block of kPerBlock groups.
__global__ void __launch_bounds__(kBlock) fin_count(const unsigned long long* __restrict__ src,
                                                    const unsigned long long* __restrict__ val, const FinDesc d,
                                                    unsigned long long* __restrict__ counts) {
  const unsigned long long g0 = (unsigned long long)blockIdx.x * kPerBlock;
  unsigned long long cnt = 0;
  for (unsigned long long g = g0 + threadIdx.x; g < g0 + kPerBlock && g < d.groups; g += kBlock)
    cnt += present(src, val, d, g);
  __shared__ unsigned long long part[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < kBlock / 32; ++w) s += part[w];
    counts[blockIdx.x] = s;
  }
}

// Pass 2: exclusive prefix of the block counts (one CTA) and the row total.
__global__ void __launch_bounds__(1024) fin_scan(unsigned long long* counts, unsigned long long nblocks,
                                                 unsigned long long* total) {
  __shared__ unsigned long long carry;
  __shared__ unsigned long long wsum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long b = 0; b < nblocks; b += 1024) {
    const unsigned long long i = b + threadIdx.x;
    const unsigned long long v = i < nblocks ? counts[i] : 0ULL;
    unsigned long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long w = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const unsigned long long incl = x + (warp > 0 ? wsum[warp - 1] : 0ULL);
    if (i < nblocks) counts[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Pass 3: present groups become rows, column by column, in group order.
__global__ void __launch_bounds__(kBlock) fin_write(const unsigned long long* __restrict__ src,
                                                    const unsigned long long* __restrict__ val, const FinDesc d,
                                                    const unsigned long long* __restrict__ offsets,
                                                    unsigned long long* __restrict__ cols, unsigned long long* vcols,
                                                    unsigned long long row_cap) {
  const unsigned long long g0 = (unsigned long long)blockIdx.x * kPerBlock;
  const unsigned long long vw = (row_cap + 63) / 64;
  __shared__ unsigned long long warp_tot[kBlock / 32];
  __shared__ unsigned long long base_s;
  if (threadIdx.x == 0) base_s = offsets[blockIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long chunk = g0; chunk < g0 + kPerBlock && chunk < d.groups; chunk += kBlock) {
    const unsigned long long g = chunk + threadIdx.x;
    const bool p = g < d.groups && g < g0 + kPerBlock && present(src, val, d, g);
    const unsigned ballot = __ballot_sync(0xffffffffu, p);
    if (lane == 0) warp_tot[warp] = __popc(ballot);
    __syncthreads();
    unsigned long long row = base_s;
    for (int w = 0; w < warp; ++w) row += warp_tot[w];
    row += __popc(ballot & ((1u << lane) - 1u));
    if (p && row < row_cap) {
      const unsigned long long base = g * d.ts;
      for (unsigned c = 0; c < d.cols; ++c) {
        cols[c * row_cap + row] = src[base + c];
        const bool valid = d.sparse || !d.nullable[c] || (val && bit_at(val, base + c));
        if (valid) atomicOr(&vcols[c * vw + (row >> 6)], 1ULL << (row & 63));
      }
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < kBlock / 32; ++w) base_s += warp_tot[w];
    __syncthreads();
  }
}

// True when row `r` orders before row `l` (the reference's comparator).
__device__ __forceinline__ bool right_before_left(const unsigned long long* __restrict__ cols,
                                                  const unsigned long long* __restrict__ vcols, const FinDesc& d,
                                                  unsigned long long row_cap, unsigned l, unsigned r) {
  if (r == l) return false;
  if (r == kInvalid) return false;
  if (l == kInvalid) return true;
  const unsigned long long vw = (row_cap + 63) / 64;
  for (int k = 0; k < d.nkeys; ++k) {
    const int c = d.key_col[k];
    if (d.nullable[c]) {
      const bool lv = bit_at(vcols + (unsigned long long)c * vw, l), rv = bit_at(vcols + (unsigned long long)c * vw, r);
      if (lv != rv) return rv;
      if (!lv) continue;
    }
    const unsigned long long a = cols[(unsigned long long)c * row_cap + l], b = cols[(unsigned long long)c * row_cap + r];
    bool lt, gt;  // right < left, left < right
    if (d.type[c] == CX_COL_INT64) {
      lt = (long long)b < (long long)a;
      gt = (long long)a < (long long)b;
    } else if (d.type[c] == CX_COL_FLOAT64) {
      lt = __longlong_as_double((long long)b) < __longlong_as_double((long long)a);
      gt = __longlong_as_double((long long)a) < __longlong_as_double((long long)b);
    } else {
      lt = b < a;
      gt = a < b;
    }
    if (lt) return !d.key_desc[k];
    if (gt) return d.key_desc[k] != 0;
  }
  return r < l;
}

// Bitonic network over row indices in one CTA (n <= 2048, a power of two).
__global__ void __launch_bounds__(1024) fin_sort_small(const unsigned long long* __restrict__ cols,
                                                       const unsigned long long* __restrict__ vcols, const FinDesc d,
                                                       unsigned long long row_cap, unsigned long long rows, unsigned n,
                                                       unsigned* __restrict__ idx) {
  __shared__ unsigned s[2048];
  for (unsigned i = threadIdx.x; i < n; i += blockDim.x) s[i] = i < rows ? i : kInvalid;
  __syncthreads();
  for (unsigned k = 2; k <= n; k <<= 1) {
    for (unsigned j = k >> 1; j > 0; j >>= 1) {
      for (unsigned i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned x = i ^ j;
        if (x > i) {
          const unsigned l = s[i], r = s[x];
          const bool rb = right_before_left(cols, vcols, d, row_cap, l, r);
          const bool lb = l != r && !rb;
          if ((i & k) == 0 ? rb : lb) { s[i] = r; s[x] = l; }
        }
      }
      __syncthreads();
    }
  }
  for (unsigned i = threadIdx.x; i < n; i += blockDim.x) idx[i] = s[i];
}

__global__ void fin_sort_init(unsigned* idx, unsigned long long rows, unsigned long long n) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    idx[i] = i < rows ? (unsigned)i : kInvalid;
}

// One compare-exchange step (k, j) of the global bitonic network.
__global__ void fin_sort_step(const unsigned long long* __restrict__ cols, const unsigned long long* __restrict__ vcols,
                              const FinDesc d, unsigned long long row_cap, unsigned* idx, unsigned long long n,
                              unsigned long long k, unsigned long long j) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long x = i ^ j;
    if (x <= i) continue;
    const unsigned l = idx[i], r = idx[x];
    const bool rb = right_before_left(cols, vcols, d, row_cap, l, r);
    const bool lb = l != r && !rb;
    if ((i & k) == 0 ? rb : lb) { idx[i] = r; idx[x] = l; }
  }
}

// Reorders the first `out` sorted rows into temporary columns.
__global__ void fin_gather(const unsigned long long* __restrict__ cols, const unsigned long long* __restrict__ vcols,
                           const FinDesc d, unsigned long long row_cap, const unsigned* __restrict__ idx,
                           unsigned long long out, unsigned long long* __restrict__ tcols,
                           unsigned long long* __restrict__ tv) {
  const unsigned long long vw = (row_cap + 63) / 64;
  for (unsigned long long o = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; o < out;
       o += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned src = idx[o];
    for (unsigned c = 0; c < d.cols; ++c) {
      tcols[c * row_cap + o] = cols[c * row_cap + src];
      if (bit_at(vcols + c * vw, src)) atomicOr(&tv[c * vw + (o >> 6)], 1ULL << (o & 63));
    }
  }
}

unsigned grid_for(unsigned long long n) {
  unsigned long long g = (n + 255) / 256;
  if (g > 148ULL * 32) g = 148ULL * 32;
  return g == 0 ? 1 : (unsigned)g;
}

}  // namespace

extern "C" int cx_finalize(const uint64_t* dev_result, const uint64_t* dev_validity, const cx_result_layout* layout,
                           const cx_sort_key* keys, int nkeys, uint64_t limit, uint64_t* dev_columns,
                           uint64_t* dev_col_validity, uint64_t row_cap, uint64_t* rows_out, void* stream_v) {
  if (!dev_result || !layout || !dev_columns || !dev_col_validity || !rows_out || nkeys < 0 || (nkeys > 0 && !keys))
    return ffail(CX_E_INVALID, "cx_finalize: bad argument");
  if (layout->columns == 0 || layout->columns > (uint32_t)kMaxCols || layout->tuple_size < layout->columns ||
      nkeys > kMaxKeys)
    return ffail(CX_E_INVALID, "cx_finalize: 1..32 visible columns within the tuple, at most 8 sort keys");
  if (!layout->sparse && !dev_validity && !layout->scalar)
    return ffail(CX_E_INVALID, "cx_finalize: a dense result needs its validity words");
  FinDesc d{};
  d.groups = layout->scalar ? (layout->groups ? 1ULL : 0ULL) : layout->groups;
  d.ts = layout->tuple_size;
  d.cols = layout->columns;
  d.sparse = layout->sparse;
  d.scalar = layout->scalar;
  for (uint32_t c = 0; c < d.cols; ++c) {
    d.type[c] = layout->column_type ? layout->column_type[c] : (unsigned char)CX_COL_UINT64;
    d.nullable[c] = layout->column_nullable ? layout->column_nullable[c] : 0;
    if (d.type[c] > CX_COL_FLOAT64) return ffail(CX_E_INVALID, "cx_finalize: unknown column type");
  }
  d.nkeys = nkeys;
  for (int k = 0; k < nkeys; ++k) {
    if (keys[k].column < 0 || (uint32_t)keys[k].column >= d.cols) return ffail(CX_E_INVALID, "cx_finalize: sort key outside the columns");
    d.key_col[k] = keys[k].column;
    d.key_desc[k] = keys[k].descending != 0;
  }
  if (row_cap < d.groups) return ffail(CX_E_CAPACITY, "cx_finalize: the row capacity is below the group count");
  if (row_cap > 0xfffffffeULL) return ffail(CX_E_CAPACITY, "cx_finalize: more than 2^32-2 rows");
  cudaStream_t s = (cudaStream_t)stream_v;
  const unsigned long long vw = (row_cap + 63) / 64;
  const unsigned long long* src = (const unsigned long long*)dev_result;
  const unsigned long long* val = (const unsigned long long*)dev_validity;
  unsigned long long* cols = (unsigned long long*)dev_columns;
  unsigned long long* vcols = (unsigned long long*)dev_col_validity;
  cudaError_t e = cudaMemsetAsync(vcols, 0, d.cols * vw * 8, s);
  if (e != cudaSuccess) return fcuda(e, "cudaMemsetAsync");
  const unsigned long long nblocks = (d.groups + kPerBlock - 1) / kPerBlock;
  unsigned long long rows = 0;
  if (nblocks) {
    unsigned long long* tmp = nullptr;  // block counts + the total
    if ((e = cudaMallocAsync((void**)&tmp, (nblocks + 1) * 8, s)) != cudaSuccess) return fcuda(e, "cudaMallocAsync");
    fin_count<<<(unsigned)nblocks, kBlock, 0, s>>>(src, val, d, tmp);
    fin_scan<<<1, 1024, 0, s>>>(tmp, nblocks, tmp + nblocks);
    fin_write<<<(unsigned)nblocks, kBlock, 0, s>>>(src, val, d, tmp, cols, vcols, row_cap);
    e = cudaMemcpyAsync(&rows, tmp + nblocks, 8, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(tmp, s);
    if (e != cudaSuccess) return fcuda(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fcuda(e, "cudaStreamSynchronize");
  }
  const unsigned long long out = rows < limit ? rows : limit;
  if (nkeys > 0 && rows > 1) {
    unsigned long long n = 1;
    while (n < rows) n <<= 1;
    unsigned* idx = nullptr;
    unsigned long long* tcols = nullptr;
    if ((e = cudaMallocAsync((void**)&idx, n * 4, s)) != cudaSuccess) return fcuda(e, "cudaMallocAsync");
    if ((e = cudaMallocAsync((void**)&tcols, (d.cols * row_cap + d.cols * vw) * 8, s)) != cudaSuccess) {
      cudaFreeAsync(idx, s);
      return fcuda(e, "cudaMallocAsync");
    }
    unsigned long long* tv = tcols + d.cols * row_cap;
    if (n <= 2048) {
      fin_sort_small<<<1, 1024, 0, s>>>(cols, vcols, d, row_cap, rows, (unsigned)n, idx);
    } else {
      fin_sort_init<<<grid_for(n), 256, 0, s>>>(idx, rows, n);
      for (unsigned long long k = 2; k <= n; k <<= 1)
        for (unsigned long long j = k >> 1; j > 0; j >>= 1)
          fin_sort_step<<<grid_for(n), 256, 0, s>>>(cols, vcols, d, row_cap, idx, n, k, j);
    }
    cudaMemsetAsync(tv, 0, d.cols * vw * 8, s);
    fin_gather<<<grid_for(out), 256, 0, s>>>(cols, vcols, d, row_cap, idx, out, tcols, tv);
    for (unsigned c = 0; c < d.cols; ++c) {
      if (out) cudaMemcpyAsync(cols + c * row_cap, tcols + c * row_cap, out * 8, cudaMemcpyDeviceToDevice, s);
    }
    cudaMemcpyAsync(vcols, tv, d.cols * vw * 8, cudaMemcpyDeviceToDevice, s);
    cudaFreeAsync(tcols, s);
    cudaFreeAsync(idx, s);
  } else if (out < rows) {
    // LIMIT without ORDER BY keeps the first rows; clear validity past them.
    for (unsigned c = 0; c < d.cols; ++c) {
      const unsigned long long first_word = (out + 63) / 64;
      if (out & 63) {
        const unsigned long long keep = (1ULL << (out & 63)) - 1ULL;
        unsigned long long w = 0;
        e = cudaMemcpyAsync(&w, vcols + c * vw + out / 64, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fcuda(e, "cudaMemcpyAsync");
        w &= keep;
        cudaMemcpyAsync(vcols + c * vw + out / 64, &w, 8, cudaMemcpyHostToDevice, s);
        cudaStreamSynchronize(s);
      }
      if (first_word < vw) cudaMemsetAsync(vcols + c * vw + first_word, 0, (vw - first_word) * 8, s);
    }
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return fcuda(e, "cx_finalize launch");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fcuda(e, "cudaStreamSynchronize");
  *rows_out = out;
  return CX_OK;
}
