// Warp-cooperative Montgomery arithmetic on the FP64 pipe, for sm_100a.
//
// The integer multiply pipe (fmaheavy) is the bound of the 32-bit-limb CIOS
// in bigint_group.cuh: every 32x32 word product costs a mad.lo and a mad.hi.
// The FP64 pipe is a separate unit with the same lane rate on B200, and one
// 52x52-bit product (2.6x the bits of a word product) costs three FP64
// instructions there:
//
//   h = fma_rz(x, y, 2^104)           bits(h) = 0x467 << 52 | floor(xy / 2^52)
//   s = h - (2^104 + 2^52)            (floor(xy / 2^52) - 1) * 2^52, exact
//   l = fma_rz(x, y, -s)              bits(l) = 0x433 << 52 | (xy mod 2^52)
//
// (x, y integers below 2^52 held exactly as doubles; every rounding above is
// exact or toward zero by construction.)  The raw bit patterns of h and l are
// "bias + value" integers; they are summed in 64-bit integer accumulators on
// the ALU pipe and the biases, whose counts are fixed by the schedule, are
// removed where a value is needed.  This is the double-precision technique
// of Emmart, Zheng and Weems ("Faster modular exponentiation using double
// precision floating point arithmetic on the GPU", ARITH 2018), written here
// as a warp-cooperative CIOS for this library's lane groups.  The word
// products of m = acc_0 (-M^-1) mod 2^52 stay on the integer pipe.
//
// A value below M < 2^(52K) is K limbs of 52 bits spread over a group of TPI
// lanes, lane g owning limbs [gL, gL+L), L = K/TPI, as doubles.  One CIOS
// step per limb b_i of the second operand (read from shared memory):
// acc += a*b_i; m = acc_0 * (-M^-1) mod 2^52 (computed by the group's lane
// 0 and broadcast); acc += m*M; acc shifts down one limb.  Each 64-bit
// accumulator receives at most four 52-bit values per step for at most K
// steps, so no normalisation is needed inside the loop; the column leaving
// at position 0 passes its exact carry (acc_0 >> 52) to the next one, and a
// lane's top-position high halves move to its upper neighbour at the shift.
#pragma once
#include <cstdint>

namespace cuhe52 {

constexpr int kBits = 52;
constexpr uint64_t kMask = (1ull << 52) - 1;
constexpr double kTwo52 = 4503599627370496.0;                       // 2^52
constexpr double kTwo104 = 20282409603651670423947251286016.0;      // 2^104
constexpr double kTwo104p52 = 20282409603651674927546878656512.0;   // 2^104 + 2^52
constexpr uint64_t kHiBias = 0x4670000000000000ull;                 // bits of 2^104
constexpr uint64_t kLoBias = 0x4330000000000000ull;                 // bits of 2^52

// Raw (bias + value) halves of the 104-bit product of x, y < 2^52.
__device__ __forceinline__ void mul52(double x, double y, uint64_t& hi, uint64_t& lo) {
  const double h = __fma_rz(x, y, kTwo104);
  const double s = __dsub_rn(h, kTwo104p52);
  const double l = __fma_rz(x, y, -s);
  hi = static_cast<uint64_t>(__double_as_longlong(h));
  lo = static_cast<uint64_t>(__double_as_longlong(l));
}

// An integer below 2^52 as an exact double, and back.
__device__ __forceinline__ double to_f64(uint64_t v) {
  return __dsub_rn(__longlong_as_double(static_cast<long long>(v | kLoBias)), kTwo52);
}
__device__ __forceinline__ uint64_t to_u64(double d) {
  return static_cast<uint64_t>(__double_as_longlong(__dadd_rn(d, kTwo52))) & kMask;
}

__device__ __forceinline__ uint64_t shfl_down64(uint32_t mask, uint64_t v, int delta, int width) {
  const uint32_t lo = __shfl_down_sync(mask, static_cast<uint32_t>(v), delta, width);
  const uint32_t hi = __shfl_down_sync(mask, static_cast<uint32_t>(v >> 32), delta, width);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_up64(uint32_t mask, uint64_t v, int delta, int width) {
  const uint32_t lo = __shfl_up_sync(mask, static_cast<uint32_t>(v), delta, width);
  const uint32_t hi = __shfl_up_sync(mask, static_cast<uint32_t>(v >> 32), delta, width);
  return (static_cast<uint64_t>(hi) << 32) | lo;
}
__device__ __forceinline__ double shfl_f64(uint32_t mask, double v, int src, int width) {
  const long long b = __double_as_longlong(v);
  const uint32_t lo = __shfl_sync(mask, static_cast<uint32_t>(b), src, width);
  const uint32_t hi = __shfl_sync(mask, static_cast<uint32_t>(static_cast<unsigned long long>(b) >> 32), src, width);
  return __longlong_as_double(static_cast<long long>((static_cast<uint64_t>(hi) << 32) | lo));
}

template <int K, int TPI>
struct Group52 {
  static_assert(TPI >= 2 && TPI <= 32 && (TPI & (TPI - 1)) == 0, "TPI must be a power of two <= 32");
  static_assert(K % TPI == 0, "K must be a multiple of TPI");
  static constexpr int L = K / TPI;
  // bias sums: a position in 1..K-1 receives per step two low and two high
  // halves, position 0 two low halves, the top pending position two high.
  static constexpr uint64_t kStep = 2ull * kLoBias + 2ull * kHiBias;

  uint32_t mask;
  int gl;
  int base_lane;

  __device__ __forceinline__ Group52() {
    const int lane = threadIdx.x & 31;
    gl = lane & (TPI - 1);
    base_lane = lane & ~(TPI - 1);
    mask = (TPI == 32) ? 0xffffffffu : (((1u << TPI) - 1u) << base_lane);
  }

  // acc (raw) += a * b over K steps; b: K doubles in shared memory.
  // On return acc holds positions gL..gL+L-1 of the result (columns K.. of
  // the full sum) with the bias of each position still included.
  //
  // The critical path of a step is acc_0 -> m -> m*M.  m is formed on the
  // integer pipe (a 64-bit multiply, low 52 bits; the FP64 pipe is the busy
  // one here) and broadcast as an integer, and the products a * b_(i+1) of
  // the next step, which do not depend on m, are issued while it is formed.
  // Steps run in unrolled blocks of U (a multiple of 2 and of L): the shift
  // of the accumulator is a rotation of register names (logical position k
  // is register (k + s) mod L in step s of a block) and the two product
  // buffers alternate by step parity, so neither costs a move.
  static constexpr int U = (L % 2 == 0) ? L : 2 * L;
  static_assert(K % U == 0, "K must be a multiple of the unrolled block");

  __device__ __forceinline__ void cios(uint64_t (&acc)[L], const double (&a)[L], const double* __restrict__ b,
                                       const double (&n)[L], uint64_t ninv) const {
    uint64_t off = kLoBias;  // bias of column i at position 0 when m_i is taken
    uint64_t hab[2][L], lab[2][L];
    {
      const double b0 = b[0];
#pragma unroll
      for (int k = 0; k < L; ++k) mul52(a[k], b0, hab[0][k], lab[0][k]);
    }
#pragma unroll 1
    for (int i0 = 0; i0 < K; i0 += U) {
#pragma unroll
      for (int s = 0; s < U; ++s) {
        const int i = i0 + s;
        const int cur = s & 1, nxt = cur ^ 1;
        uint64_t& a0 = acc[s % L];  // logical position 0
        a0 += lab[cur][0];
        // m = (acc_0 mod 2^52) * (-M^-1) mod 2^52 by lane 0, broadcast
        const uint64_t mi = ((a0 - off) * ninv) & kMask;
        const uint32_t mlo = __shfl_sync(mask, static_cast<uint32_t>(mi), 0, TPI);
        const uint32_t mhi = __shfl_sync(mask, static_cast<uint32_t>(mi >> 32), 0, TPI);
        // the next step's a * b_(i+1) (independent of m)
        const double bn = b[i + 1 < K ? i + 1 : i];
#pragma unroll
        for (int k = 0; k < L; ++k) mul52(a[k], bn, hab[nxt][k], lab[nxt][k]);
        const double m = to_f64((static_cast<uint64_t>(mhi) << 32) | mlo);
        uint64_t hnm[L], lnm[L];
#pragma unroll
        for (int k = 0; k < L; ++k) mul52(n[k], m, hnm[k], lnm[k]);
        a0 += lnm[0];
#pragma unroll
        for (int k = 1; k < L; ++k) {
          uint64_t& ak = acc[(k + s) % L];
          ak = ak + lab[cur][k] + hab[cur][k - 1];
          ak = ak + lnm[k] + hnm[k - 1];
        }
        const uint64_t pend = hab[cur][L - 1] + hnm[L - 1];
        // column i leaves: its exact value is a multiple of 2^52
        const uint64_t carry = (a0 - off - kLoBias) >> kBits;
        uint64_t next = shfl_down64(mask, a0, 1, TPI);
        if (gl == TPI - 1) next = 0;
        a0 = next + pend;                           // becomes logical position L - 1
        if (gl == 0) acc[(s + 1) % L] += carry;      // the new logical position 0
        off += kStep;
      }
    }
  }

  // Remove the biases of the K result positions, normalise to 52-bit limbs
  // and reduce T < 2M into [0, M).  r receives the canonical limbs.
  __device__ __forceinline__ void finalize(double (&r)[L], uint64_t (&acc)[L], const double (&n)[L]) const {
    uint64_t t[L];
#pragma unroll
    for (int k = 0; k < L; ++k) {
      // final column K + p at position p: 2 high halves at position K (the
      // pending one) plus (K - 1 - p) steps at positions K-1 .. p+1
      const uint64_t p = uint64_t(gl * L + k);
      t[k] = acc[k] - (2ull * kHiBias + (uint64_t(K) - 1ull - p) * kStep);
    }
    // carries: within the lane, then across lanes until none remain
    uint64_t cin = 0;
#pragma unroll
    for (int k = 0; k < L; ++k) {
      t[k] += cin;
      cin = t[k] >> kBits;
      t[k] &= kMask;
    }
    for (int guard = 0; guard < TPI + 1; ++guard) {
      uint64_t in = shfl_up64(mask, cin, 1, TPI);
      if (gl == 0) in = 0;
      cin = 0;
#pragma unroll
      for (int k = 0; k < L; ++k) {
        t[k] += in;
        in = t[k] >> kBits;
        t[k] &= kMask;
      }
      cin = (gl == TPI - 1) ? 0 : in;
      if (!__any_sync(mask, cin != 0)) break;
    }
    // d = t - M with lane-local borrow, then cross-lane borrow lookahead
    uint64_t d[L];
    uint64_t borrow = 0;
    uint64_t zero = 0;
#pragma unroll
    for (int k = 0; k < L; ++k) {
      const uint64_t nk = to_u64(n[k]);
      const uint64_t v = t[k] - nk - borrow;  // wraps when negative
      borrow = v >> 63;
      d[k] = v & kMask;
      zero |= d[k];
    }
    const uint32_t gb = __ballot_sync(mask, borrow != 0);
    const uint32_t pb = __ballot_sync(mask, zero == 0);
    const uint64_t lanes = (TPI == 32) ? 0xffffffffull : ((1ull << TPI) - 1ull);
    const uint64_t G = (uint64_t(gb) >> base_lane) & lanes;
    const uint64_t P = (uint64_t(pb) >> base_lane) & lanes;
    const uint64_t S = G + (G | P);
    const uint64_t cin_b = S ^ G ^ (G | P);
    const bool out_borrow = (S >> TPI) & 1ull;
    if ((cin_b >> gl) & 1ull) {
      uint64_t b2 = 1;
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const uint64_t v = d[k] - b2;
        b2 = v >> 63;
        d[k] = v & kMask;
      }
    }
    // T >= M exactly when the subtraction does not borrow out of the top
    const bool ge = !out_borrow;
#pragma unroll
    for (int k = 0; k < L; ++k) r[k] = to_f64(ge ? d[k] : t[k]);
  }

  // r = a * b * 2^(-52K) mod M.  a: registers (< M), b: shared memory (< M).
  __device__ __forceinline__ void mont_mul(double (&r)[L], const double (&a)[L], const double* __restrict__ b,
                                           const double (&n)[L], uint64_t ninv) const {
    uint64_t acc[L];
#pragma unroll
    for (int k = 0; k < L; ++k) acc[k] = 0;
    cios(acc, a, b, n, ninv);
    finalize(r, acc, n);
  }

  // r = (init + a * b) * 2^(-52K) mod M, init < 2^(52K) in canonical limbs.
  __device__ __forceinline__ void mont_mul_acc(double (&r)[L], const double (&init)[L], const double (&a)[L],
                                               const double* __restrict__ b, const double (&n)[L],
                                               uint64_t ninv) const {
    uint64_t acc[L];
#pragma unroll
    for (int k = 0; k < L; ++k) acc[k] = to_u64(init[k]);
    cios(acc, a, b, n, ninv);
    finalize(r, acc, n);
  }

  __device__ __forceinline__ void publish(double* buf, const double (&x)[L]) const {
    __syncwarp(mask);
#pragma unroll
    for (int k = 0; k < L; ++k) buf[gl * L + k] = x[k];
    __syncwarp(mask);
  }
};

}  // namespace cuhe52
