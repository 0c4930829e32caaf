// cx_rng.h -- counter-based generator shared by the device column generator
// and its host twins (practice_b200/datagen.py restates it in numpy).
//
// value(row) = lo + below(hash(key(seed, stream), row), hi - lo + 1), where
// hash is two rounds of the splitmix64 finaliser and below(h, n) keeps the high
// 32 bits of h scaled to [0, n) (multiply-shift).  Dates are yyyymmdd keys of
// consecutive days from 1992-01-01 (SSB's date dimension range).
#pragma once

#if defined(__CUDACC__)
#define CX_HD __host__ __device__ __forceinline__
#else
#define CX_HD inline
#endif

CX_HD unsigned long long cx_splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

CX_HD unsigned long long cx_rng_stream_key(unsigned long long seed, unsigned long long stream) {
  return cx_splitmix64(seed ^ cx_splitmix64(stream * 0xD6E8FEB86659FD93ULL + 1ULL));
}

CX_HD unsigned long long cx_rng_hash(unsigned long long key, unsigned long long row) {
  return cx_splitmix64(key + row * 0x9E3779B97F4A7C15ULL);
}

CX_HD unsigned long long cx_rng_below(unsigned long long h, unsigned long long n) {
  return ((h >> 32) * n) >> 32;
}

// yyyymmdd of day `d` after 1992-01-01 (proleptic Gregorian; days-from-civil
// inverse over the 400-year era, integer only).
CX_HD int cx_datekey_of_day(unsigned d) {
  const long long z = 8035LL + (long long)d + 719468LL;  // 8035 = days 1970-01-01 .. 1992-01-01
  const long long era = z / 146097;
  const long long doe = z - era * 146097;
  const long long yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  long long y = yoe + era * 400;
  const long long doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  const long long mp = (5 * doy + 2) / 153;
  const long long dd = doy - (153 * mp + 2) / 5 + 1;
  const long long mm = mp < 10 ? mp + 3 : mp - 9;
  if (mm <= 2) ++y;
  return (int)(y * 10000 + mm * 100 + dd);
}
