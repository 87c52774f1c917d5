// Word-sized modular arithmetic for 60-bit NTT primes (device and host).
//
// Shoup products for fixed multipliers (twiddles, CRT constants):
//   w' = floor(w * 2^64 / p),  x*w mod p = x*w - hi64(x*w')*p  in [0, 2p).
// Barrett reduction of 128-bit values with mu = floor(2^128 / p), exact
// after at most two conditional subtractions.  Every routine returns the
// exact residue / quotient, so results do not depend on how an intermediate
// was reduced.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CUHE_HD __host__ __device__ __forceinline__
#else
#define CUHE_HD inline
#endif

namespace cuhe {
namespace bfv {

using u64 = uint64_t;
using u128 = unsigned __int128;

struct Prime {
  u64 p;
  u64 mu_hi, mu_lo;  // floor(2^128 / p)
};

CUHE_HD u64 mulhi(u64 a, u64 b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return u64((u128(a) * b) >> 64);
#endif
}

// x*w mod p in [0, 2p) for any x < 2^64, w < p, wq = floor(w*2^64/p)
CUHE_HD u64 shoup_lazy(u64 x, u64 w, u64 wq, u64 p) { return x * w - mulhi(x, wq) * p; }
CUHE_HD u64 shoup(u64 x, u64 w, u64 wq, u64 p) {
  u64 r = shoup_lazy(x, w, wq, p);
  return r >= p ? r - p : r;
}

// floor(x / 2^128 * mu) estimate of floor(x / p), correct within 2 below.
CUHE_HD u64 barrett_quotient(u64 hi, u64 lo, const Prime& m) {
  const u128 p00 = u128(lo) * m.mu_lo;
  const u128 p01 = u128(lo) * m.mu_hi;
  const u128 p10 = u128(hi) * m.mu_lo;
  const u128 middle = (p00 >> 64) + u64(p01) + u64(p10);
  return hi * m.mu_hi + u64(p01 >> 64) + u64(p10 >> 64) + u64(middle >> 64);
}

// exact x mod p for any 128-bit x
CUHE_HD u64 reduce128(u128 x, const Prime& m) {
  const u64 lo = u64(x), hi = u64(x >> 64);
  u64 q = barrett_quotient(hi, lo, m);
  u64 r = lo - q * m.p;
  while (r >= m.p) r -= m.p;
  return r;
}

// exact (floor(x/p), x mod p) when floor(x/p) < 2^64
CUHE_HD void divide128(u128 x, const Prime& m, u64* quotient, u64* remainder) {
  const u64 lo = u64(x), hi = u64(x >> 64);
  u64 q = barrett_quotient(hi, lo, m);
  u64 r = lo - q * m.p;
  while (r >= m.p) { r -= m.p; ++q; }
  *quotient = q;
  *remainder = r;
}

// exact floor(y * 2^64 / p) for y < p
CUHE_HD u64 fraction64(u64 y, const Prime& m) {
  u64 q = barrett_quotient(y, 0, m);
  u64 r = u64(0) - q * m.p;
  while (r >= m.p) { r -= m.p; ++q; }
  return q;
}

CUHE_HD u64 mulmod(u64 a, u64 b, const Prime& m) { return reduce128(u128(a) * b, m); }
CUHE_HD u64 addmod(u64 a, u64 b, u64 p) {
  u64 s = a + b;
  return s >= p ? s - p : s;
}
CUHE_HD u64 submod(u64 a, u64 b, u64 p) { return a >= b ? a - b : a + p - b; }

}  // namespace bfv
}  // namespace cuhe
