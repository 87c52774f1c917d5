// Warp-cooperative multi-precision Montgomery arithmetic for sm_100a.
//
// A big integer of K 32-bit limbs (little-endian) is spread over a group of
// TPI consecutive lanes of one warp: lane g of the group owns limbs
// [g*L, g*L+L), L = K/TPI.  Montgomery multiplication is CIOS (coarsely
// integrated operand scanning): for every word b_i of the second operand the
// group adds a*b_i and m*N (m = t_0 * (-N^-1) mod 2^32, broadcast by a
// shuffle), then shifts the accumulator down one word (a second shuffle moves
// each lane's lowest word to its lower neighbour).  Carries out of a lane's
// top limb stay in a two-word "pending" register and enter the next lane at
// the shift, so no warp-wide carry propagation happens inside the loop.
// Multiply-accumulate chains are PTX mad.lo.cc / madc.hi.cc sequences.
//
// The second operand b is read from shared memory as 16-byte broadcasts;
// results are canonical (< N) after a carry-lookahead conditional
// subtraction that resolves cross-lane borrows with two ballots.
#pragma once
#include <cstdint>

namespace cuhe {

// ---- single PTX instructions; consecutive volatile asm keeps the carry flag
__device__ __forceinline__ uint32_t add_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t addc_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t addc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("addc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t sub_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t subc_cc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t subc(uint32_t a, uint32_t b) {
  uint32_t r; asm volatile("subc.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b)); return r; }
__device__ __forceinline__ uint32_t madlo_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ uint32_t madloc_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ uint32_t madhic_cc(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r; asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }

// Lane-group context.  `mask` names exactly the TPI lanes of this group so
// that groups of one warp may follow different control flow.
template <int K, int TPI>
struct Group {
  static_assert(TPI >= 2 && TPI <= 32 && (TPI & (TPI - 1)) == 0, "TPI must be a power of two <= 32");
  static_assert(K % TPI == 0, "K must be a multiple of TPI");
  static constexpr int L = K / TPI;
  static_assert(L % 4 == 0, "each lane must own a multiple of four limbs");

  uint32_t mask;   // lanes of this group within the warp
  int gl;          // lane index within the group
  int base_lane;   // warp lane of group lane 0

  __device__ __forceinline__ Group() {
    const int lane = threadIdx.x & 31;
    gl = lane & (TPI - 1);
    base_lane = lane & ~(TPI - 1);
    mask = (TPI == 32) ? 0xffffffffu : (((1u << TPI) - 1u) << base_lane);
  }

  // ---- global / shared memory movement (each lane moves its L limbs) ----
  __device__ __forceinline__ void load(uint32_t (&x)[L], const uint32_t* __restrict__ src) const {
    const uint4* p = reinterpret_cast<const uint4*>(src + gl * L);
#pragma unroll
    for (int j = 0; j < L / 4; ++j) {
      uint4 v = p[j];
      x[4 * j] = v.x; x[4 * j + 1] = v.y; x[4 * j + 2] = v.z; x[4 * j + 3] = v.w;
    }
  }
  __device__ __forceinline__ void load_ro(uint32_t (&x)[L], const uint32_t* __restrict__ src) const {
    const uint4* p = reinterpret_cast<const uint4*>(src + gl * L);
#pragma unroll
    for (int j = 0; j < L / 4; ++j) {
      uint4 v = __ldg(p + j);
      x[4 * j] = v.x; x[4 * j + 1] = v.y; x[4 * j + 2] = v.z; x[4 * j + 3] = v.w;
    }
  }
  __device__ __forceinline__ void store(uint32_t* __restrict__ dst, const uint32_t (&x)[L]) const {
    uint4* p = reinterpret_cast<uint4*>(dst + gl * L);
#pragma unroll
    for (int j = 0; j < L / 4; ++j) p[j] = make_uint4(x[4 * j], x[4 * j + 1], x[4 * j + 2], x[4 * j + 3]);
  }
  // Publish x to a shared buffer read by the whole group (b operand).
  __device__ __forceinline__ void publish(uint32_t* buf, const uint32_t (&x)[L]) const {
    __syncwarp(mask);
    store(buf, x);
    __syncwarp(mask);
  }

  // ---- acc[0..L) , (c1:c0) += a[0..L) * b  (two interleaved carry chains) ----
  __device__ __forceinline__ static void mac_row(uint32_t (&acc)[L], uint32_t& c0, uint32_t& c1,
                                                 const uint32_t (&a)[L], uint32_t b) {
    acc[0] = madlo_cc(a[0], b, acc[0]);
    acc[1] = madhic_cc(a[0], b, acc[1]);
#pragma unroll
    for (int j = 2; j < L; j += 2) {
      acc[j] = madloc_cc(a[j], b, acc[j]);
      acc[j + 1] = madhic_cc(a[j], b, acc[j + 1]);
    }
    c0 = addc_cc(c0, 0u);
    c1 = addc(c1, 0u);
    acc[1] = madlo_cc(a[1], b, acc[1]);
#pragma unroll
    for (int j = 1; j < L - 2; j += 2) {
      acc[j + 1] = madhic_cc(a[j], b, acc[j + 1]);
      acc[j + 2] = madloc_cc(a[j + 2], b, acc[j + 2]);
    }
    c0 = madhic_cc(a[L - 1], b, c0);
    c1 = addc(c1, 0u);
  }

  // One CIOS word step: acc = (acc + a*bi + m*N) / 2^32.
  __device__ __forceinline__ void step(uint32_t (&acc)[L], uint32_t& c0, uint32_t& c1,
                                       const uint32_t (&a)[L], const uint32_t (&n)[L],
                                       uint32_t bi, uint32_t ninv) const {
    mac_row(acc, c0, c1, a, bi);
    const uint32_t m = __shfl_sync(mask, acc[0] * ninv, 0, TPI);
    mac_row(acc, c0, c1, n, m);
    uint32_t next = __shfl_down_sync(mask, acc[0], 1, TPI);
    if (gl == TPI - 1) next = 0u;
#pragma unroll
    for (int j = 0; j < L - 1; ++j) acc[j] = acc[j + 1];
    acc[L - 1] = add_cc(next, c0);
    c0 = addc(c1, 0u);
    c1 = 0u;
  }

  // Carry-lookahead over the group: given this lane's generate/propagate
  // flags, return the carry (or borrow) entering this lane; *out receives the
  // carry leaving the top lane.
  __device__ __forceinline__ bool lookahead(bool generate, bool propagate, bool* out) const {
    const uint32_t gb = __ballot_sync(mask, generate);
    const uint32_t pb = __ballot_sync(mask, propagate);
    const uint64_t lanes = (TPI == 32) ? 0xffffffffull : ((1ull << TPI) - 1ull);
    const uint64_t G = (uint64_t(gb) >> base_lane) & lanes;
    const uint64_t P = (uint64_t(pb) >> base_lane) & lanes;
    const uint64_t S = G + (G | P);
    const uint64_t cin = S ^ G ^ (G | P);
    if (out) *out = (S >> TPI) & 1ull;
    return (cin >> gl) & 1ull;
  }

  // Resolve pending inter-lane carries of (acc, c0) and reduce the value
  // T < 2N into [0, N).
  __device__ __forceinline__ void finalize(uint32_t (&r)[L], uint32_t (&acc)[L], uint32_t c0,
                                           const uint32_t (&n)[L]) const {
    uint32_t top = 0u;
    if (gl == TPI - 1) { top = c0; c0 = 0u; }
    // pending carries are tiny (< 4); one pass almost always settles them
    for (int guard = 0; guard < TPI; ++guard) {
      uint32_t cin = __shfl_up_sync(mask, c0, 1, TPI);
      if (gl == 0) cin = 0u;
      acc[0] = add_cc(acc[0], cin);
#pragma unroll
      for (int j = 1; j < L; ++j) acc[j] = addc_cc(acc[j], 0u);
      const uint32_t carry = addc(0u, 0u);
      if (gl == TPI - 1) { top += carry; c0 = 0u; } else { c0 = carry; }
      if (!__any_sync(mask, c0 != 0u)) break;
    }
    // d = acc - N with lane-local borrow, then cross-lane borrow lookahead
    uint32_t d[L];
    d[0] = sub_cc(acc[0], n[0]);
#pragma unroll
    for (int j = 1; j < L; ++j) d[j] = subc_cc(acc[j], n[j]);
    const uint32_t borrow = subc(0u, 0u) & 1u;
    uint32_t zero = d[0];
#pragma unroll
    for (int j = 1; j < L; ++j) zero |= d[j];
    bool group_borrow = false;
    const bool bin = lookahead(borrow != 0u, zero == 0u, &group_borrow);
    if (bin) {
      d[0] = sub_cc(d[0], 1u);
#pragma unroll
      for (int j = 1; j < L; ++j) d[j] = subc_cc(d[j], 0u);
      (void)subc(0u, 0u);
    }
    // T >= N  <=>  top >= final borrow (both known to the top lane)
    const bool ge = __shfl_sync(mask, (int)(top >= (uint32_t)group_borrow), TPI - 1, TPI) != 0;
#pragma unroll
    for (int j = 0; j < L; ++j) r[j] = ge ? d[j] : acc[j];
  }

  // The K CIOS word steps of one Montgomery product, b read from shared memory.
  __device__ __forceinline__ void cios(uint32_t (&acc)[L], uint32_t& c0, uint32_t& c1, const uint32_t (&a)[L],
                                       const uint32_t* __restrict__ b, const uint32_t (&n)[L],
                                       uint32_t ninv) const {
#pragma unroll 1
    for (int base = 0; base < K; base += L) {
#pragma unroll
      for (int q = 0; q < L; q += 4) {
        const uint4 bw = *reinterpret_cast<const uint4*>(b + base + q);
        step(acc, c0, c1, a, n, bw.x, ninv);
        step(acc, c0, c1, a, n, bw.y, ninv);
        step(acc, c0, c1, a, n, bw.z, ninv);
        step(acc, c0, c1, a, n, bw.w, ninv);
      }
    }
  }

  // r = a * b * 2^(-32K) mod N.  a: registers (< N), b: shared memory (< N).
  __device__ __forceinline__ void mont_mul(uint32_t (&r)[L], const uint32_t (&a)[L],
                                           const uint32_t* __restrict__ b, const uint32_t (&n)[L],
                                           uint32_t ninv) const {
    uint32_t acc[L];
#pragma unroll
    for (int j = 0; j < L; ++j) acc[j] = 0u;
    uint32_t c0 = 0u, c1 = 0u;
    cios(acc, c0, c1, a, b, n, ninv);
    finalize(r, acc, c0, n);
  }

  // r = (init + a * b) * 2^(-32K) mod N with the accumulator started at
  // init.  Valid for init < 2^(32K), a < 2^(32K), b < N: the CIOS value stays
  // below 2N, which finalize reduces.
  __device__ __forceinline__ void mont_mul_acc(uint32_t (&r)[L], const uint32_t (&init)[L],
                                               const uint32_t (&a)[L], const uint32_t* __restrict__ b,
                                               const uint32_t (&n)[L], uint32_t ninv) const {
    uint32_t acc[L];
#pragma unroll
    for (int j = 0; j < L; ++j) acc[j] = init[j];
    uint32_t c0 = 0u, c1 = 0u;
    cios(acc, c0, c1, a, b, n, ninv);
    finalize(r, acc, c0, n);
  }

  // Exact division helper: steps of the same shape as Montgomery reduction
  // with modulus M' = 2^(32K) - M and multiplier minv = M^-1 mod 2^32.  Each
  // step removes one low word of y - q*M and emits quotient word q_i; after
  // `words` steps q holds y / M for any y divisible by M with y/M < 2^(32*words).
  __device__ __forceinline__ void exact_div(uint32_t (&q)[L], uint32_t (&acc)[L],
                                            const uint32_t (&mneg)[L], uint32_t minv, int words) const {
#pragma unroll
    for (int j = 0; j < L; ++j) q[j] = 0u;
    uint32_t c0 = 0u, c1 = 0u;
    uint32_t zero[L];
#pragma unroll
    for (int j = 0; j < L; ++j) zero[j] = 0u;
#pragma unroll 1
    for (int base = 0; base < words; base += L) {
#pragma unroll
      for (int s = 0; s < L; ++s) {
        const uint32_t m = __shfl_sync(mask, acc[0] * minv, 0, TPI);
        if (base / L == gl) q[s] = m;
        mac_row(acc, c0, c1, mneg, m);
        uint32_t next = __shfl_down_sync(mask, acc[0], 1, TPI);
        if (gl == TPI - 1) next = 0u;
#pragma unroll
        for (int j = 0; j < L - 1; ++j) acc[j] = acc[j + 1];
        acc[L - 1] = add_cc(next, c0);
        c0 = addc(c1, 0u);
        c1 = 0u;
      }
    }
  }

  // Is x < bound?  (x, bound canonical K-limb values held by the group.)
  __device__ __forceinline__ bool less_than(const uint32_t (&x)[L], const uint32_t (&bound)[L]) const {
    uint32_t d = sub_cc(x[0], bound[0]);
    uint32_t zero = d;
#pragma unroll
    for (int j = 1; j < L; ++j) { d = subc_cc(x[j], bound[j]); zero |= d; }
    const uint32_t borrow = subc(0u, 0u) & 1u;
    bool out = false;
    (void)lookahead(borrow != 0u, zero == 0u, &out);
    return __shfl_sync(mask, (int)out, 0, TPI) != 0;
  }

  __device__ __forceinline__ bool is_zero(const uint32_t (&x)[L]) const {
    uint32_t z = 0u;
#pragma unroll
    for (int j = 0; j < L; ++j) z |= x[j];
    return !__any_sync(mask, z != 0u);
  }
};

}  // namespace cuhe
