// Minimal mpz_class / gmp_randclass over the C API in gmp.h, written from the
// GMP manual's description of the C++ interface (eager evaluation instead of
// expression templates; '/' and '%' truncate like gmpxx, '>>' floors).
//
// TEST INFRASTRUCTURE ONLY: lets the reference's C++ BFV sources build
// against the system libgmp.so.10 for the checker under oracle/_ref.
#ifndef CUHE_ORACLE_GMPXX_SHIM_H
#define CUHE_ORACLE_GMPXX_SHIM_H

#include <cstdlib>
#include <cstring>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "gmp.h"

class mpz_class {
 public:
  mpz_t mp;

  template <class T>
  using if_int = std::enable_if_t<std::is_integral_v<T> && !std::is_same_v<T, bool>, int>;

  mpz_class() { mpz_init(mp); }
  mpz_class(const mpz_class& o) { mpz_init_set(mp, o.mp); }
  mpz_class(mpz_class&& o) noexcept { mpz_init(mp); mpz_swap(mp, o.mp); }
  template <class T, if_int<T> = 0>
  mpz_class(T x) {
    if constexpr (std::is_signed_v<T>) mpz_init_set_si(mp, long(x));
    else mpz_init_set_ui(mp, (unsigned long)(x));
  }
  explicit mpz_class(mpz_srcptr z) { mpz_init_set(mp, z); }
  explicit mpz_class(const char* s, int base = 0) {
    if (mpz_init_set_str(mp, s, base) != 0) {
      mpz_clear(mp);
      throw std::invalid_argument("mpz_set_str");
    }
  }
  explicit mpz_class(const std::string& s, int base = 0) : mpz_class(s.c_str(), base) {}
  ~mpz_class() { mpz_clear(mp); }

  mpz_class& operator=(const mpz_class& o) { if (this != &o) mpz_set(mp, o.mp); return *this; }
  mpz_class& operator=(mpz_class&& o) noexcept { mpz_swap(mp, o.mp); return *this; }
  template <class T, if_int<T> = 0>
  mpz_class& operator=(T x) {
    if constexpr (std::is_signed_v<T>) mpz_set_si(mp, long(x));
    else mpz_set_ui(mp, (unsigned long)(x));
    return *this;
  }

  mpz_ptr get_mpz_t() { return mp; }
  mpz_srcptr get_mpz_t() const { return mp; }
  int set_str(const char* s, int base) { return mpz_set_str(mp, s, base); }
  int set_str(const std::string& s, int base) { return mpz_set_str(mp, s.c_str(), base); }
  std::string get_str(int base = 10) const {
    char* raw = mpz_get_str(nullptr, base, mp);
    std::string s(raw);
    void (*freefunc)(void*, size_t) = nullptr;
    mp_get_memory_functions(nullptr, nullptr, &freefunc);
    freefunc(raw, std::strlen(raw) + 1);
    return s;
  }
  unsigned long get_ui() const { return mpz_get_ui(mp); }
  long get_si() const { return mpz_get_si(mp); }
  bool fits_ulong_p() const { return mpz_fits_ulong_p(mp) != 0; }
  bool fits_slong_p() const { return mpz_fits_slong_p(mp) != 0; }

  mpz_class& operator+=(const mpz_class& o) { mpz_add(mp, mp, o.mp); return *this; }
  mpz_class& operator-=(const mpz_class& o) { mpz_sub(mp, mp, o.mp); return *this; }
  mpz_class& operator*=(const mpz_class& o) { mpz_mul(mp, mp, o.mp); return *this; }
  mpz_class& operator/=(const mpz_class& o) { mpz_tdiv_q(mp, mp, o.mp); return *this; }
  mpz_class& operator%=(const mpz_class& o) { mpz_tdiv_r(mp, mp, o.mp); return *this; }
  template <class T, if_int<T> = 0> mpz_class& operator+=(T o) { return *this += mpz_class(o); }
  template <class T, if_int<T> = 0> mpz_class& operator-=(T o) { return *this -= mpz_class(o); }
  template <class T, if_int<T> = 0> mpz_class& operator*=(T o) { return *this *= mpz_class(o); }
  template <class T, if_int<T> = 0> mpz_class& operator/=(T o) { return *this /= mpz_class(o); }
  template <class T, if_int<T> = 0> mpz_class& operator%=(T o) { return *this %= mpz_class(o); }
  template <class T, if_int<T> = 0> mpz_class& operator<<=(T bits) { mpz_mul_2exp(mp, mp, mp_bitcnt_t(bits)); return *this; }
  template <class T, if_int<T> = 0> mpz_class& operator>>=(T bits) { mpz_fdiv_q_2exp(mp, mp, mp_bitcnt_t(bits)); return *this; }
  mpz_class& operator++() { mpz_add_ui(mp, mp, 1); return *this; }
  mpz_class& operator--() { mpz_sub_ui(mp, mp, 1); return *this; }
};

inline mpz_class operator-(const mpz_class& a) { mpz_class r; mpz_neg(r.mp, a.mp); return r; }
inline mpz_class operator+(const mpz_class& a) { return a; }

#define CUHE_MPZ_BINARY(op, fn)                                                                    \
  inline mpz_class operator op(const mpz_class& a, const mpz_class& b) { mpz_class r; fn(r.mp, a.mp, b.mp); return r; } \
  template <class T, mpz_class::if_int<T> = 0>                                                    \
  inline mpz_class operator op(const mpz_class& a, T b) { return a op mpz_class(b); }              \
  template <class T, mpz_class::if_int<T> = 0>                                                    \
  inline mpz_class operator op(T a, const mpz_class& b) { return mpz_class(a) op b; }
CUHE_MPZ_BINARY(+, mpz_add)
CUHE_MPZ_BINARY(-, mpz_sub)
CUHE_MPZ_BINARY(*, mpz_mul)
CUHE_MPZ_BINARY(/, mpz_tdiv_q)
CUHE_MPZ_BINARY(%, mpz_tdiv_r)
#undef CUHE_MPZ_BINARY

template <class T, mpz_class::if_int<T> = 0>
inline mpz_class operator<<(const mpz_class& a, T bits) { mpz_class r; mpz_mul_2exp(r.mp, a.mp, mp_bitcnt_t(bits)); return r; }
template <class T, mpz_class::if_int<T> = 0>
inline mpz_class operator>>(const mpz_class& a, T bits) { mpz_class r; mpz_fdiv_q_2exp(r.mp, a.mp, mp_bitcnt_t(bits)); return r; }

inline int cuhe_mpz_cmp(const mpz_class& a, const mpz_class& b) { return mpz_cmp(a.mp, b.mp); }
#define CUHE_MPZ_COMPARE(op)                                                                                   \
  inline bool operator op(const mpz_class& a, const mpz_class& b) { return cuhe_mpz_cmp(a, b) op 0; }           \
  template <class T, mpz_class::if_int<T> = 0>                                                                 \
  inline bool operator op(const mpz_class& a, T b) { return cuhe_mpz_cmp(a, mpz_class(b)) op 0; }              \
  template <class T, mpz_class::if_int<T> = 0>                                                                 \
  inline bool operator op(T a, const mpz_class& b) { return cuhe_mpz_cmp(mpz_class(a), b) op 0; }
CUHE_MPZ_COMPARE(==)
CUHE_MPZ_COMPARE(!=)
CUHE_MPZ_COMPARE(<)
CUHE_MPZ_COMPARE(<=)
CUHE_MPZ_COMPARE(>)
CUHE_MPZ_COMPARE(>=)
#undef CUHE_MPZ_COMPARE

inline std::ostream& operator<<(std::ostream& os, const mpz_class& v) { return os << v.get_str(10); }

class gmp_randclass {
 public:
  explicit gmp_randclass(void (*init)(gmp_randstate_t)) {
    std::memset(state_, 0, sizeof(state_));
    init(state_);
  }
  ~gmp_randclass() { gmp_randclear(state_); }
  gmp_randclass(const gmp_randclass&) = delete;
  gmp_randclass& operator=(const gmp_randclass&) = delete;
  void seed(unsigned long s) { gmp_randseed_ui(state_, s); }
  mpz_class get_z_bits(mp_bitcnt_t bits) { mpz_class r; mpz_urandomb(r.mp, state_, bits); return r; }
  mpz_class get_z_range(const mpz_class& bound) { mpz_class r; mpz_urandomm(r.mp, state_, bound.mp); return r; }

 private:
  gmp_randstate_t state_;
};

#endif
