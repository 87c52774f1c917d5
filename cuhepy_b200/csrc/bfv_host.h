// Host-side construction of a BFV residue ring: the auxiliary 60-bit NTT
// primes, negacyclic NTT twiddles, and the exact RNS conversion constants of
// the tensor scale-and-round.  Follows the parameter rules of the reference
// Ring / RNSScale / ResidueArithmetic classes (src/cuhepy/bfv/_cpu_ext/
// rns_ntt.h:317-374, rns_scale.h:59-81,156-173, bfv_residue.h:20-27); all
// arithmetic here is this file's own multiword code.
#pragma once
#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "bfv_arith.cuh"

namespace cuhe {
namespace bfv {
namespace host {

// ---- unsigned multiword integers (little-endian u64 limbs) -----------------
struct Big {
  std::vector<u64> w;
  Big() {}
  explicit Big(u64 v) { if (v) w.push_back(v); }
  void trim() { while (!w.empty() && w.back() == 0) w.pop_back(); }
  bool zero() const { return w.empty(); }
  size_t bits() const {
    if (w.empty()) return 0;
    return (w.size() - 1) * 64 + (64 - __builtin_clzll(w.back()));
  }
};

inline int cmp(const Big& a, const Big& b) {
  if (a.w.size() != b.w.size()) return a.w.size() < b.w.size() ? -1 : 1;
  for (size_t i = a.w.size(); i-- > 0;)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}

inline Big add(const Big& a, const Big& b) {
  Big r;
  r.w.resize(std::max(a.w.size(), b.w.size()) + 1, 0);
  u128 c = 0;
  for (size_t i = 0; i < r.w.size(); ++i) {
    c += (i < a.w.size() ? a.w[i] : 0);
    c += (i < b.w.size() ? b.w[i] : 0);
    r.w[i] = u64(c);
    c >>= 64;
  }
  r.trim();
  return r;
}

inline Big sub(const Big& a, const Big& b) {  // a >= b
  Big r;
  r.w.resize(a.w.size(), 0);
  u64 borrow = 0;
  for (size_t i = 0; i < a.w.size(); ++i) {
    u64 bi = i < b.w.size() ? b.w[i] : 0;
    u128 d = u128(a.w[i]) - bi - borrow;
    r.w[i] = u64(d);
    borrow = (d >> 64) ? 1 : 0;
  }
  r.trim();
  return r;
}

inline Big mul_small(const Big& a, u64 m) {
  Big r;
  r.w.resize(a.w.size() + 1, 0);
  u128 c = 0;
  for (size_t i = 0; i < a.w.size(); ++i) {
    c += u128(a.w[i]) * m;
    r.w[i] = u64(c);
    c >>= 64;
  }
  r.w[a.w.size()] = u64(c);
  r.trim();
  return r;
}

inline Big mul(const Big& a, const Big& b) {
  Big r;
  r.w.assign(a.w.size() + b.w.size() + 1, 0);
  for (size_t i = 0; i < a.w.size(); ++i) {
    u128 c = 0;
    for (size_t j = 0; j < b.w.size(); ++j) {
      c += u128(a.w[i]) * b.w[j] + r.w[i + j];
      r.w[i + j] = u64(c);
      c >>= 64;
    }
    size_t k = i + b.w.size();
    while (c) {
      c += r.w[k];
      r.w[k++] = u64(c);
      c >>= 64;
    }
  }
  r.trim();
  return r;
}

inline u64 mod_small(const Big& a, u64 m) {
  u128 r = 0;
  for (size_t i = a.w.size(); i-- > 0;) r = ((r << 64) | a.w[i]) % m;
  return u64(r);
}

inline Big div_small(const Big& a, u64 m, u64* rem = nullptr) {
  Big q;
  q.w.assign(a.w.size(), 0);
  u128 r = 0;
  for (size_t i = a.w.size(); i-- > 0;) {
    r = (r << 64) | a.w[i];
    q.w[i] = u64(r / m);
    r %= m;
  }
  q.trim();
  if (rem) *rem = u64(r);
  return q;
}

inline Big shl(const Big& a, size_t bits) {
  Big r;
  size_t words = bits / 64, s = bits % 64;
  r.w.assign(a.w.size() + words + 1, 0);
  for (size_t i = 0; i < a.w.size(); ++i) {
    r.w[i + words] |= a.w[i] << s;
    if (s) r.w[i + words + 1] |= a.w[i] >> (64 - s);
  }
  r.trim();
  return r;
}

// floor(a / b) by binary long division (setup only)
inline Big div(const Big& a, const Big& b) {
  if (b.zero()) throw std::invalid_argument("division by zero");
  if (cmp(a, b) < 0) return Big();
  Big q, r;
  const size_t nb = a.bits();
  q.w.assign((nb + 63) / 64, 0);
  for (size_t i = nb; i-- > 0;) {
    r = shl(r, 1);
    if ((a.w[i / 64] >> (i % 64)) & 1) {
      if (r.w.empty()) r.w.push_back(0);
      r.w[0] |= 1;
    }
    if (cmp(r, b) >= 0) {
      r = sub(r, b);
      q.w[i / 64] |= u64(1) << (i % 64);
    }
  }
  q.trim();
  return q;
}

inline Big from_hex(const std::string& s) {
  Big r;
  for (char ch : s) {
    int v;
    if (ch >= '0' && ch <= '9') v = ch - '0';
    else if (ch >= 'a' && ch <= 'f') v = ch - 'a' + 10;
    else if (ch >= 'A' && ch <= 'F') v = ch - 'A' + 10;
    else throw std::invalid_argument("invalid hexadecimal digit");
    r = shl(r, 4);
    if (v) {
      if (r.w.empty()) r.w.push_back(0);
      r.w[0] |= u64(v);
    }
  }
  r.trim();
  return r;
}

// ---- word primes ------------------------------------------------------------
inline u64 powmod(u64 b, u64 e, u64 m) {
  u64 r = 1 % m;
  b %= m;
  while (e) {
    if (e & 1) r = u64(u128(r) * b % m);
    b = u64(u128(b) * b % m);
    e >>= 1;
  }
  return r;
}

// deterministic Miller-Rabin for 64-bit inputs
inline bool is_prime64(u64 n) {
  if (n < 2) return false;
  for (u64 p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    if (n % p == 0) return n == p;
  }
  u64 d = n - 1;
  int s = 0;
  while ((d & 1) == 0) { d >>= 1; ++s; }
  for (u64 a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    u64 x = powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool composite = true;
    for (int r = 1; r < s; ++r) {
      x = u64(u128(x) * x % n);
      if (x == n - 1) { composite = false; break; }
    }
    if (composite) return false;
  }
  return true;
}

inline Prime make_prime(u64 p) {
  Prime m;
  m.p = p;
  const u128 mu = ~u128(0) / p;  // == floor(2^128 / p) for odd p
  m.mu_hi = u64(mu >> 64);
  m.mu_lo = u64(mu);
  return m;
}

inline u64 shoup_quotient(u64 w, u64 p) { return u64((u128(w) << 64) / p); }

inline unsigned log2_exact(size_t n) {
  unsigned l = 0;
  while ((size_t(1) << l) < n) ++l;
  return l;
}

inline size_t bitrev(size_t x, unsigned bits) {
  size_t r = 0;
  for (unsigned i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}

// Negacyclic NTT tables for one prime: psi is the smallest-candidate primitive
// 2N-th root (candidate^((p-1)/2N) whose N-th power is -1).
struct NTTTable {
  u64 psi = 0;
  std::vector<u64> fwd, fwd_q;   // psi^bitrev(i) and Shoup quotients, i < N
  std::vector<u64> inv, inv_q;   // psi^-bitrev(i)
  u64 n_inv = 0, n_inv_q = 0;    // N^-1
  u64 last = 0, last_q = 0;      // psi^-bitrev(1) * N^-1
};

inline NTTTable build_ntt(size_t n, u64 p) {
  NTTTable t;
  for (u64 c = 2;; ++c) {
    u64 root = powmod(c, (p - 1) / (2 * n), p);
    if (powmod(root, n, p) == p - 1) { t.psi = root; break; }
  }
  const unsigned logn = log2_exact(n);
  const u64 psi_inv = powmod(t.psi, p - 2, p);
  std::vector<u64> pw(n, 1), ipw(n, 1);
  for (size_t i = 1; i < n; ++i) {
    pw[i] = u64(u128(pw[i - 1]) * t.psi % p);
    ipw[i] = u64(u128(ipw[i - 1]) * psi_inv % p);
  }
  t.fwd.resize(n); t.fwd_q.resize(n); t.inv.resize(n); t.inv_q.resize(n);
  for (size_t i = 0; i < n; ++i) {
    const size_t r = bitrev(i, logn);
    t.fwd[i] = pw[r];
    t.inv[i] = ipw[r];
    t.fwd_q[i] = shoup_quotient(t.fwd[i], p);
    t.inv_q[i] = shoup_quotient(t.inv[i], p);
  }
  t.n_inv = powmod(u64(n) % p, p - 2, p);
  t.n_inv_q = shoup_quotient(t.n_inv, p);
  t.last = u64(u128(t.inv[1]) * t.n_inv % p);
  t.last_q = shoup_quotient(t.last, p);
  return t;
}

// Exact RNS base conversion constants (base primes -> target primes).
struct ExactBase {
  std::vector<size_t> base, target;          // prime indices
  Big product;                               // M
  std::vector<u64> inv, inv_q;               // (M/p_j)^-1 mod p_j (Shoup)
  std::vector<std::vector<u64>> partial_mod_target;  // [k][j] (M/p_j) mod p_k
  std::vector<u64> product_mod_target, product_mod_target_q;  // M mod p_k (Shoup)
  std::vector<std::vector<u64>> partial_words;  // M/p_j as fixed words
  std::vector<u64> product_words;
};

constexpr int kCrtWords = 18;

inline std::vector<u64> to_words(const Big& v) {
  if (v.w.size() > size_t(kCrtWords)) throw std::invalid_argument("CRT constant exceeds the fixed-word bound");
  std::vector<u64> out(kCrtWords, 0);
  std::copy(v.w.begin(), v.w.end(), out.begin());
  return out;
}

inline ExactBase build_base(const std::vector<u64>& primes, size_t start, size_t count, size_t tstart,
                            size_t tcount) {
  ExactBase b;
  for (size_t j = 0; j < count; ++j) b.base.push_back(start + j);
  for (size_t k = 0; k < tcount; ++k) b.target.push_back(tstart + k);
  b.product = Big(1);
  for (size_t j = 0; j < count; ++j) b.product = mul_small(b.product, primes[start + j]);
  b.product_words = to_words(b.product);
  b.partial_mod_target.assign(tcount, std::vector<u64>(count));
  for (size_t j = 0; j < count; ++j) {
    const u64 p = primes[start + j];
    Big partial = div_small(b.product, p);
    b.partial_words.push_back(to_words(partial));
    const u64 inv = powmod(mod_small(partial, p), p - 2, p);
    b.inv.push_back(inv);
    b.inv_q.push_back(shoup_quotient(inv, p));
    for (size_t k = 0; k < tcount; ++k) b.partial_mod_target[k][j] = mod_small(partial, primes[tstart + k]);
  }
  for (size_t k = 0; k < tcount; ++k) {
    const u64 p = primes[tstart + k];
    const u64 v = mod_small(b.product, p);
    b.product_mod_target.push_back(v);
    b.product_mod_target_q.push_back(shoup_quotient(v, p));
  }
  return b;
}

// Complete residue-ring plan.
struct RingPlan {
  size_t n = 0;
  unsigned logn = 0;
  Big q;
  unsigned q_bits = 0;
  size_t coefficient_bytes = 0;
  unsigned digit_bits = 0;
  size_t digits = 0;
  std::vector<u64> primes;          // all auxiliary primes (K of them)
  size_t residue_count = 0;         // L: Q = product of the first L primes
  size_t tensor_count = 0;          // primes used by the exact tensor product
  std::vector<NTTTable> ntt;
  std::vector<std::vector<u64>> garner_inv, garner_inv_q;  // [j][k<j] p_k^-1 mod p_j
  bool has_scale = false;
  ExactBase q_to_b, b_to_q;
  std::vector<u64> inv_q_mod_b, inv_q_mod_b_q;  // Q^-1 mod B primes
};

inline size_t prime_count_for(const std::vector<u64>& primes, const Big& bound) {
  Big product(1), twice = mul_small(bound, 2);
  for (size_t c = 1; c <= primes.size(); ++c) {
    product = mul_small(product, primes[c - 1]);
    if (cmp(product, twice) > 0) return c;
  }
  throw std::invalid_argument("Insufficient auxiliary CRT modulus for exact reconstruction");
}

inline RingPlan build_ring(size_t n, const Big& q, unsigned bits, bool residue = true) {
  RingPlan r;
  const size_t qb = q.bits();
  if (n < 8 || n > 32768 || (n & (n - 1)) || cmp(q, Big(3)) < 0 || qb > 512 || bits < 1 || bits > qb)
    throw std::invalid_argument("Invalid native BFV ring parameters");
  r.n = n;
  r.logn = log2_exact(n);
  r.q = q;
  r.q_bits = unsigned(qb);
  r.coefficient_bytes = (qb + 7) / 8;
  r.digit_bits = bits;
  r.digits = (qb + bits - 1) / bits;
  const Big qm1 = sub(q, Big(1));
  // |gadget dot product| <= N*D*(2^b-1)*(q-1); BFV cross term <= 2N(q-1)^2
  const Big switch_bound = mul(mul_small(mul_small(Big(u64(n)), u64(r.digits)), 1), mul(sub(shl(Big(1), bits), Big(1)), qm1));
  const Big tensor_bound = mul_small(mul(qm1, qm1), u64(2 * n));
  const Big needed = mul_small(cmp(switch_bound, tensor_bound) > 0 ? switch_bound : tensor_bound, 2);
  Big product(1);
  u64 prime = (u64(1) << 60) - 2 * n + 1;
  while (cmp(product, needed) <= 0) {
    while (!is_prime64(prime)) {
      if (prime <= (u64(1) << 59)) throw std::invalid_argument("No suitable 60-bit auxiliary prime");
      prime -= 2 * n;
    }
    r.primes.push_back(prime);
    product = mul_small(product, prime);
    prime -= 2 * n;
  }
  // Q must be the product of the first L primes
  Big prefix(1);
  for (size_t c = 1; c <= r.primes.size(); ++c) {
    prefix = mul_small(prefix, r.primes[c - 1]);
    if (cmp(prefix, q) == 0) r.residue_count = c;
  }
  if (residue && (!r.residue_count || r.residue_count > 8))
    throw std::invalid_argument("Residue backend requires Q to be a product of the first 60-bit NTT primes");
  if (!residue) r.residue_count = 0;
  r.tensor_count = prime_count_for(r.primes, tensor_bound);
  for (u64 p : r.primes) r.ntt.push_back(build_ntt(n, p));
  // Garner constants: over the residue primes, or over every auxiliary
  // prime of a native (prime q) ring, whose results are composed from up to
  // all of them
  const size_t garner = residue ? r.residue_count : r.primes.size();
  r.garner_inv.assign(garner, {});
  r.garner_inv_q.assign(garner, {});
  for (size_t j = 0; j < garner; ++j) {
    const u64 p = r.primes[j];
    for (size_t k = 0; k < j; ++k) {
      const u64 inv = powmod(r.primes[k] % p, p - 2, p);
      r.garner_inv[j].push_back(inv);
      r.garner_inv_q[j].push_back(shoup_quotient(inv, p));
    }
  }
  return r;
}

// RNSScale constants (rns_scale.h:156-173); throws like the reference.
inline void build_scale(RingPlan& r, u64 t) {
  const size_t L = r.residue_count, K = r.tensor_count;
  if (K <= L) throw std::invalid_argument("Invalid exact RNS conversion bases");
  if (L > 17 || K - L > 17) throw std::invalid_argument("Invalid exact RNS conversion bases");
  r.q_to_b = build_base(r.primes, 0, L, L, K - L);
  r.b_to_q = build_base(r.primes, L, K - L, 0, L);
  if (t < 2 || t >= (u64(1) << 60) || cmp(Big(t), r.q) >= 0 || cmp(r.q_to_b.product, r.q) != 0 || L > 8)
    throw std::invalid_argument("Invalid RNS scale parameters");
  const Big qm1 = sub(r.q, Big(1));
  const Big quotient_bound = add(div(mul_small(mul(qm1, qm1), u64(2 * r.n)), r.q), Big(1));
  if (cmp(r.b_to_q.product, mul_small(quotient_bound, 2)) <= 0)
    throw std::invalid_argument("RNS quotient basis is too small for exact signed scaling");
  r.inv_q_mod_b.clear();
  r.inv_q_mod_b_q.clear();
  for (size_t j = L; j < K; ++j) {
    const u64 p = r.primes[j];
    const u64 inv = powmod(mod_small(r.q, p), p - 2, p);
    r.inv_q_mod_b.push_back(inv);
    r.inv_q_mod_b_q.push_back(shoup_quotient(inv, p));
  }
  r.has_scale = true;
}

}  // namespace host
}  // namespace bfv
}  // namespace cuhe
