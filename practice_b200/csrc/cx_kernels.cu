// cx_kernels.cu -- statically compiled (nvcc, sm_100a) kernels of the runtime:
// sparse-result compaction and the seeded synthetic column generator.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/crystal_b200.h"
#include "cx_internal.h"
#include "cx_rng.h"

namespace {

// Every failure is recorded as the calling thread's cx_last_error().
int cuda_fail(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  return cx_internal::set_error(CX_E_CUDA, buf);
}

int invalid(const char* what) { return cx_internal::set_error(CX_E_INVALID, what); }

constexpr int kCompactBlock = 256;
constexpr int kCompactPerBlock = 2048;  // groups per block

// Pass 1: number of present groups (any non-zero slot) per block of groups.
__global__ void __launch_bounds__(kCompactBlock)
compact_count(const unsigned long long* __restrict__ src, unsigned long long groups, unsigned ts,
              unsigned long long* __restrict__ block_counts) {
  const unsigned long long g0 = (unsigned long long)blockIdx.x * kCompactPerBlock;
  unsigned long long cnt = 0;
  for (unsigned long long g = g0 + threadIdx.x; g < g0 + kCompactPerBlock && g < groups; g += kCompactBlock) {
    bool present = false;
    for (unsigned c = 0; c < ts && !present; ++c) present = src[g * ts + c] != 0ULL;
    cnt += present;
  }
  __shared__ unsigned long long part[kCompactBlock / 32];
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long s = 0;
    for (int w = 0; w < kCompactBlock / 32; ++w) s += part[w];
    block_counts[blockIdx.x] = s;
  }
}

// Pass 2: exclusive prefix over block counts (one block, sequential chunks).
__global__ void __launch_bounds__(1024)
compact_scan(unsigned long long* counts, unsigned long long nblocks, unsigned long long* total) {
  __shared__ unsigned long long carry;
  __shared__ unsigned long long warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (unsigned long long base = 0; base < nblocks; base += 1024) {
    const unsigned long long i = base + threadIdx.x;
    const unsigned long long v = i < nblocks ? counts[i] : 0ULL;
    unsigned long long x = v;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long w = warp_sums[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long incl = x + (warp > 0 ? warp_sums[warp - 1] : 0ULL);
    if (i < nblocks) counts[i] = carry + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Pass 3: write present tuples in group order.
__global__ void __launch_bounds__(kCompactBlock)
compact_write(const unsigned long long* __restrict__ src, unsigned long long groups, unsigned ts,
              const unsigned long long* __restrict__ offsets, unsigned long long* __restrict__ dst) {
  const unsigned long long g0 = (unsigned long long)blockIdx.x * kCompactPerBlock;
  __shared__ unsigned long long warp_tot[kCompactBlock / 32];
  __shared__ unsigned long long base_s;
  if (threadIdx.x == 0) base_s = offsets[blockIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (unsigned long long chunk = g0; chunk < g0 + kCompactPerBlock && chunk < groups; chunk += kCompactBlock) {
    const unsigned long long g = chunk + threadIdx.x;
    bool present = false;
    if (g < groups && g < g0 + kCompactPerBlock)
      for (unsigned c = 0; c < ts && !present; ++c) present = src[g * ts + c] != 0ULL;
    const unsigned ballot = __ballot_sync(0xffffffffu, present);
    if (lane == 0) warp_tot[warp] = __popc(ballot);
    __syncthreads();
    unsigned long long before = base_s;
    for (int w = 0; w < warp; ++w) before += warp_tot[w];
    before += __popc(ballot & ((1u << lane) - 1u));
    if (present)
      for (unsigned c = 0; c < ts; ++c) dst[before * ts + c] = src[g * ts + c];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < kCompactBlock / 32; ++w) base_s += warp_tot[w];
    __syncthreads();
  }
}

__global__ void gen_uniform_kernel(unsigned long long stream, unsigned long long seed, long long lo, unsigned long long span,
                                   unsigned long long row0, unsigned long long rows, int* __restrict__ out) {
  const unsigned long long key = cx_rng_stream_key(seed, stream);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (unsigned long long)gridDim.x * blockDim.x)
    out[i] = (int)(lo + (long long)cx_rng_below(cx_rng_hash(key, row0 + i), span));
}

__global__ void gen_datekey_kernel(unsigned long long stream, unsigned long long seed, unsigned days,
                                   unsigned long long row0, unsigned long long rows, int* __restrict__ out) {
  const unsigned long long key = cx_rng_stream_key(seed, stream);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned d = (unsigned)cx_rng_below(cx_rng_hash(key, row0 + i), days);
    out[i] = cx_datekey_of_day(d);
  }
}

__global__ void gen_validity_kernel(unsigned long long stream, unsigned long long seed, unsigned long long rows,
                                    unsigned permille, unsigned long long* __restrict__ out) {
  const unsigned long long key = cx_rng_stream_key(seed, stream);
  const unsigned long long words = (rows + 63) / 64;
  for (unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; w < words;
       w += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long bits = 0;
    for (int b = 0; b < 64; ++b) {
      const unsigned long long r = w * 64 + b;
      if (r >= rows) break;
      const bool is_null = cx_rng_below(cx_rng_hash(key, r), 1000) < permille;
      if (!is_null) bits |= 1ULL << b;
    }
    out[w] = bits;
  }
}

unsigned grid_for(unsigned long long n, unsigned block) {
  unsigned long long g = (n + block - 1) / block;
  if (g > 148ULL * 32) g = 148ULL * 32;
  return g == 0 ? 1 : (unsigned)g;
}

}  // namespace

extern "C" int cx_compact_sparse(const uint64_t* src, uint64_t groups, uint32_t ts, uint64_t* dst, uint64_t* dev_count,
                                 void* stream_v) {
  if (!src || !dst || !dev_count || ts == 0) return invalid("cx_compact_sparse: null buffer or zero tuple size");
  cudaStream_t s = (cudaStream_t)stream_v;
  const unsigned long long nblocks = (groups + kCompactPerBlock - 1) / kCompactPerBlock;
  if (nblocks == 0) {
    cudaError_t e = cudaMemsetAsync(dev_count, 0, 8, s);
    return e == cudaSuccess ? CX_OK : cuda_fail(e, "cudaMemsetAsync");
  }
  unsigned long long* counts = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&counts, nblocks * 8, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync");
  compact_count<<<(unsigned)nblocks, kCompactBlock, 0, s>>>((const unsigned long long*)src, groups, ts, counts);
  compact_scan<<<1, 1024, 0, s>>>(counts, nblocks, (unsigned long long*)dev_count);
  compact_write<<<(unsigned)nblocks, kCompactBlock, 0, s>>>((const unsigned long long*)src, groups, ts, counts,
                                                            (unsigned long long*)dst);
  e = cudaGetLastError();
  cudaFreeAsync(counts, s);
  return e == cudaSuccess ? CX_OK : cuda_fail(e, "compaction launch");
}

// ------------------------------------------------ no-allocation compaction ---
// Some callers cannot let this library allocate device memory: a serving loop
// that has reserved the whole HBM budget for admitted queries (an allocation
// here could fail or silently break its accounting), and engines whose memory
// guard must see every device byte before a query runs.  For them the block
// counts of the compaction live in this fixed file-scope array instead of a
// cudaMallocAsync buffer.  It holds kNoAllocMaxBlocks counts (128 KiB), so one
// call compacts at most kNoAllocMaxBlocks * kCompactPerBlock group tuples; every
// GPU that loads the library keeps the array until the process exits.
constexpr unsigned long long kNoAllocMaxBlocks = 16384;
static __device__ __align__(256) unsigned long long g_noalloc_block_counts[kNoAllocMaxBlocks];

namespace {
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[256] = {};  // last resolved device address of the array, per device ordinal
}  // namespace

extern "C" int cx_compact_sparse_noalloc(const uint64_t* src, uint64_t groups, uint32_t ts, uint64_t* dst,
                                         uint64_t* dev_count, void* stream_v) {
  if (!src || !dst || !dev_count || ts == 0)
    return invalid("cx_compact_sparse_noalloc: null buffer or zero tuple size");
  const unsigned long long nblocks = (groups + kCompactPerBlock - 1) / kCompactPerBlock;
  if (nblocks > kNoAllocMaxBlocks) {
    char buf[256];
    snprintf(buf, sizeof buf, "cx_compact_sparse_noalloc: %llu groups exceed the fixed maximum of %llu groups per call",
             (unsigned long long)groups, kNoAllocMaxBlocks * kCompactPerBlock);
    return cx_internal::set_error(CX_E_CAPACITY, buf);
  }
  cudaStream_t s = (cudaStream_t)stream_v;
  if (nblocks == 0) {
    cudaError_t e = cudaMemsetAsync(dev_count, 0, 8, s);
    return e == cudaSuccess ? CX_OK : cuda_fail(e, "cudaMemsetAsync");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 256) return invalid("cx_compact_sparse_noalloc: device ordinal out of range");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamIsCapturing");
  unsigned long long* counts = nullptr;
  {
    // The host-side symbol is not a device address: resolve the array's
    // address in the current device's context.  Outside stream capture it is
    // resolved on every call, so a context re-created after cudaDeviceReset
    // (or another context made current) gets its own address; inside capture
    // the address resolved by an earlier call on this device is used, so the
    // first call on a device must come before any capture.
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (cap == cudaStreamCaptureStatusNone) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_block_counts);
      if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
      g_noalloc_ptr[dev] = (unsigned long long*)p;
    } else if (!g_noalloc_ptr[dev]) {
      return cx_internal::set_error(CX_E_INVALID,
                                    "cx_compact_sparse_noalloc: the first call on a device must come before stream capture");
    }
    counts = g_noalloc_ptr[dev];
  }
  // compact_count writes every one of the nblocks counts, so the array needs
  // no clearing between calls.
  compact_count<<<(unsigned)nblocks, kCompactBlock, 0, s>>>((const unsigned long long*)src, groups, ts, counts);
  compact_scan<<<1, 1024, 0, s>>>(counts, nblocks, (unsigned long long*)dev_count);
  compact_write<<<(unsigned)nblocks, kCompactBlock, 0, s>>>((const unsigned long long*)src, groups, ts, counts,
                                                            (unsigned long long*)dst);
  e = cudaGetLastError();
  return e == cudaSuccess ? CX_OK : cuda_fail(e, "compaction launch");
}

extern "C" int cx_gen_uniform(uint64_t stream, uint64_t seed, int64_t lo, int64_t hi, uint64_t row0, uint64_t rows,
                              int32_t* out, void* cuda_stream) {
  if (!out || hi < lo || lo < INT32_MIN || hi > INT32_MAX) return invalid("cx_gen_uniform: null output or bad range");
  if (rows == 0) return CX_OK;
  gen_uniform_kernel<<<grid_for(rows, 256), 256, 0, (cudaStream_t)cuda_stream>>>(
      stream, seed, lo, (unsigned long long)(hi - lo + 1), row0, rows, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CX_OK : cuda_fail(e, "gen_uniform");
}

extern "C" int cx_gen_datekey(uint64_t stream, uint64_t seed, uint32_t days, uint64_t row0, uint64_t rows, int32_t* out,
                              void* cuda_stream) {
  if (!out || days == 0 || days > 36500) return invalid("cx_gen_datekey: null output or bad day count");
  if (rows == 0) return CX_OK;
  gen_datekey_kernel<<<grid_for(rows, 256), 256, 0, (cudaStream_t)cuda_stream>>>(stream, seed, days, row0, rows, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CX_OK : cuda_fail(e, "gen_datekey");
}

extern "C" int cx_gen_validity(uint64_t stream, uint64_t seed, uint64_t rows, uint32_t null_permille, uint64_t* out,
                               void* cuda_stream) {
  if (!out || null_permille > 1000) return invalid("cx_gen_validity: null output or permille above 1000");
  if (rows == 0) return CX_OK;
  gen_validity_kernel<<<grid_for((rows + 63) / 64, 256), 256, 0, (cudaStream_t)cuda_stream>>>(
      stream, seed, rows, null_permille, (unsigned long long*)out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CX_OK : cuda_fail(e, "gen_validity");
}

// ------------------------------------------------- functional dependencies --
// Whether column B of a dimension determines column A (every row with the
// same B value has the same A value): each row claims tab[B - lo_b] for its
// A offset; a second, different offset sets the flag.  `tab` (radix_b ints)
// must hold -1 before the launch; afterwards it maps each B offset that
// occurs to its A offset.
namespace {

__global__ void __launch_bounds__(256)
fd_check(const int* __restrict__ a, const int* __restrict__ b, long long n, int lo_a, int lo_b, unsigned radix_b,
         int* __restrict__ tab, unsigned* __restrict__ flag) {
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    const unsigned bo = (unsigned)(b[r] - lo_b);
    const int ao = a[r] - lo_a;
    if (bo >= radix_b) { atomicOr(flag, 1u); continue; }
    const int old = atomicCAS(&tab[bo], -1, ao);
    if (old != -1 && old != ao) atomicOr(flag, 1u);
  }
}

}  // namespace

namespace cx_internal {

int fd_check_launch(const int* a, const int* b, long long n, int lo_a, int lo_b, int radix_b, int* tab, unsigned* flag,
                    cudaStream_t s) {
  if (!a || !b || !tab || !flag || n < 0 || radix_b <= 0) return invalid("fd_check: bad argument");
  cudaError_t e = cudaMemsetAsync(tab, 0xFF, (size_t)radix_b * sizeof(int), s);
  if (e != cudaSuccess) return cuda_fail(e, "fd_check: memset");
  if (n == 0) return CX_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long blocks = std::min<long long>((n + 255) / 256, (long long)sms * 8);
  fd_check<<<(unsigned)blocks, 256, 0, s>>>(a, b, n, lo_a, lo_b, (unsigned)radix_b, tab, flag);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fd_check");
  return CX_OK;
}

}  // namespace cx_internal
