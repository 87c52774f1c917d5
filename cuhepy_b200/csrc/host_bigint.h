// Small host-side multi-precision helpers used only to derive Montgomery
// constants when a Paillier context is created (R mod N, R^2 mod N, N^-1 mod
// 2^32, ...).  Little-endian 32-bit limbs; nothing here is on a hot path.
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

namespace cuhe {
namespace host {

using Limbs = std::vector<uint32_t>;

inline int cmp(const Limbs& a, const Limbs& b) {
  for (size_t i = a.size(); i-- > 0;) {
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  }
  return 0;
}

// a -= b (same length), returns borrow
inline uint32_t sub_in_place(Limbs& a, const Limbs& b) {
  uint64_t borrow = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    uint64_t d = uint64_t(a[i]) - b[i] - borrow;
    a[i] = uint32_t(d);
    borrow = (d >> 63) & 1u;
  }
  return uint32_t(borrow);
}

// a += b (same length), returns carry
inline uint32_t add_in_place(Limbs& a, const Limbs& b) {
  uint64_t carry = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    uint64_t s = uint64_t(a[i]) + b[i] + carry;
    a[i] = uint32_t(s);
    carry = s >> 32;
  }
  return uint32_t(carry);
}

// x = 2x mod m for x < m (m occupies the same number of limbs as x)
inline void double_mod(Limbs& x, const Limbs& m) {
  uint32_t top = x.back() >> 31;
  for (size_t i = x.size(); i-- > 1;) x[i] = (x[i] << 1) | (x[i - 1] >> 31);
  x[0] <<= 1;
  if (top || cmp(x, m) >= 0) sub_in_place(x, m);
}

// x * 2^shift mod m, for x < m
inline Limbs shift_mod(Limbs x, size_t shift, const Limbs& m) {
  for (size_t i = 0; i < shift; ++i) double_mod(x, m);
  return x;
}

// full product of a and b, truncated / zero-extended to `words` limbs
inline Limbs mul(const Limbs& a, const Limbs& b, size_t words) {
  Limbs r(words, 0u);
  for (size_t i = 0; i < a.size() && i < words; ++i) {
    uint64_t carry = 0;
    for (size_t j = 0; j < b.size() && i + j < words; ++j) {
      uint64_t t = uint64_t(a[i]) * b[j] + r[i + j] + carry;
      r[i + j] = uint32_t(t);
      carry = t >> 32;
    }
    for (size_t k = i + b.size(); carry && k < words; ++k) {
      uint64_t t = uint64_t(r[k]) + carry;
      r[k] = uint32_t(t);
      carry = t >> 32;
    }
  }
  return r;
}

// m^-1 mod 2^32 for odd m0 (Newton iteration)
inline uint32_t inv32(uint32_t m0) {
  uint32_t x = 1u;
  for (int i = 0; i < 5; ++i) x *= 2u - m0 * x;
  return x;
}

inline Limbs resized(const uint32_t* src, size_t src_words, size_t words) {
  Limbs r(words, 0u);
  std::memcpy(r.data(), src, sizeof(uint32_t) * (src_words < words ? src_words : words));
  return r;
}

inline bool fits(const uint32_t* src, size_t src_words, size_t words) {
  for (size_t i = words; i < src_words; ++i)
    if (src[i]) return false;
  return true;
}

inline size_t bit_length(const Limbs& x) {
  for (size_t i = x.size(); i-- > 0;) {
    if (x[i]) return i * 32 + (32 - __builtin_clz(x[i]));
  }
  return 0;
}

inline bool is_zero(const Limbs& x) {
  for (uint32_t w : x)
    if (w) return false;
  return true;
}

// x >>= 1 with `top` shifted into the most significant bit
inline void shr1(Limbs& x, uint32_t top = 0u) {
  for (size_t i = 0; i + 1 < x.size(); ++i) x[i] = (x[i] >> 1) | (x[i + 1] << 31);
  x.back() = (x.back() >> 1) | (top << 31);
}

// x = x / 2 mod m for x < m, m odd (same limb count)
inline void half_mod(Limbs& x, const Limbs& m) {
  if (x[0] & 1u) {
    const uint32_t carry = add_in_place(x, m);
    shr1(x, carry);
  } else {
    shr1(x);
  }
}

// x = x - y mod m for x, y < m
inline void sub_mod(Limbs& x, const Limbs& y, const Limbs& m) {
  if (sub_in_place(x, y)) add_in_place(x, m);
}

// x mod m (bitwise long division; m nonzero).  Result has m's limb count.
inline Limbs mod_reduce(const Limbs& x, const Limbs& m) {
  Limbs r(m.size(), 0u);
  for (size_t i = bit_length(x); i-- > 0;) {
    const uint32_t top = r.back() >> 31;
    for (size_t k = r.size(); k-- > 1;) r[k] = (r[k] << 1) | (r[k - 1] >> 31);
    r[0] = (r[0] << 1) | ((x[i / 32] >> (i % 32)) & 1u);
    if (top || cmp(r, m) >= 0) sub_in_place(r, m);
  }
  return r;
}

// a^-1 mod m for odd m and 0 < a < m (binary extended Euclid).  Returns false
// when gcd(a, m) != 1.  All values have m's limb count.
inline bool mod_inverse_odd(const Limbs& a, const Limbs& m, Limbs* out) {
  const size_t w = m.size();
  Limbs one(w, 0u);
  one[0] = 1u;
  Limbs u = a, v = m, x1 = one, x2(w, 0u);
  if (is_zero(u) || !(m[0] & 1u)) return false;
  while (cmp(u, one) != 0 && cmp(v, one) != 0) {
    if (is_zero(u) || is_zero(v)) return false;
    while (!(u[0] & 1u)) { shr1(u); half_mod(x1, m); }
    while (!(v[0] & 1u)) { shr1(v); half_mod(x2, m); }
    if (cmp(u, v) >= 0) {
      sub_in_place(u, v);
      sub_mod(x1, x2, m);
    } else {
      sub_in_place(v, u);
      sub_mod(x2, x1, m);
    }
  }
  *out = cmp(u, one) == 0 ? x1 : x2;
  return true;
}

// Left-to-right sliding-window schedule for a fixed exponent.  Each op is
// (squarings << 16) | (odd-power table index + 1); the first op only loads
// its table entry.  Table entry t holds base^(2t+1).
inline std::vector<int32_t> window_schedule(const Limbs& e, int window) {
  std::vector<int32_t> ops;
  const size_t bits = bit_length(e);
  if (bits == 0) return ops;
  auto bit = [&](long i) -> int { return (e[size_t(i) / 32] >> (size_t(i) % 32)) & 1u; };
  long i = long(bits) - 1;
  int pending = 0;
  bool first = true;
  while (i >= 0) {
    if (!bit(i)) { ++pending; --i; continue; }
    long lo = i - window + 1;
    if (lo < 0) lo = 0;
    while (!bit(lo)) ++lo;
    int value = 0;
    for (long j = i; j >= lo; --j) value = (value << 1) | bit(j);
    const int width = int(i - lo + 1);
    if (first) {
      ops.push_back(int32_t((value - 1) / 2 + 1));
      first = false;
    } else {
      ops.push_back(int32_t(((pending + width) << 16) | ((value - 1) / 2 + 1)));
    }
    pending = 0;
    i = lo - 1;
  }
  if (pending) ops.push_back(int32_t(pending << 16));
  return ops;
}

}  // namespace host
}  // namespace cuhe
