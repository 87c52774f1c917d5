// BFV residue-ring kernels for sm_100a.
//
// Layout in HBM: residues are u64 planes [poly][prime][N] in coefficient or
// NTT (bit-reversed) order; composed integers are [poly][N][W] little-endian
// u64 words (W = ceil(bits(Q)/64)).  The negacyclic NTT of one N-point plane
// runs inside one CTA in shared memory (N <= 16384).
#pragma once
#include <cstdint>

#include "bfv_arith.cuh"

namespace cuhe {
namespace bfv {

constexpr int kMaxPrimes = 18;
constexpr int kMaxResidue = 8;
constexpr int kCrtWordsDev = 18;
constexpr int kMaxWords = 8;  // composed coefficient words (Q <= 512 bits)

struct BaseDev {
  int start, count, tstart, tcount;
  u64 inv[kMaxPrimes], inv_q[kMaxPrimes];
  u64 partial_mod_target[kMaxPrimes][kMaxPrimes];  // [k][j]
  u64 product_mod_target[kMaxPrimes], product_mod_target_q[kMaxPrimes];
  u64 partial_words[kMaxPrimes][kCrtWordsDev];
  u64 product_words[kCrtWordsDev];
};

// Native rings: constants of the first `count` auxiliary primes (P their
// product) for reducing a centred CRT integer mod q without composing it
// (k_native_reduce, mode 0); R2 = 2^128.
struct NativeCrt {
  u64 inv[kMaxPrimes], inv_q[kMaxPrimes];  // (P / p_j)^-1 mod p_j and its Shoup quotient
  u64 c[kMaxPrimes][kMaxWords];            // (P / p_j) R2 mod q
  u64 pq[kMaxWords];                       // P R2 mod q
  u64 cq[kMaxWords + 1];                   // count q
};

// Native rings, plaintext modulus t: constants of the scale-and-round over
// the tensor primes (P their product).  With t P / p_j = A_j q + B_j and
// t P = A_P q + B_P: a = (A mod q) 2^128 mod q, f = floor(B 2^128 / q).
struct NativeScale {
  u64 a[kMaxPrimes][kMaxWords];
  u64 ap[kMaxWords];
  u64 f[kMaxPrimes][2];
  u64 fp[2];
};

struct RingDev {
  int n, logn, primes, residue, tensor, digits, digit_bits, words;
  const NativeCrt* crt;  // native rings: [count - 1] for count = 1 .. primes; else null
  u64 q_ninv;            // -q^-1 mod 2^64 (native rings)
  int has_nscale;        // nscale valid (native ring with t set, q of at least 68 bits)
  NativeScale nscale;
  Prime prime[kMaxPrimes];
  // twiddles as (w, floor(w 2^64 / p)) pairs, one 16-byte load each
  const ulonglong2* fwd2[kMaxPrimes];
  const ulonglong2* inv2[kMaxPrimes];
  u64 n_inv[kMaxPrimes], n_inv_q[kMaxPrimes], last[kMaxPrimes], last_q[kMaxPrimes];
  u64 garner[kMaxPrimes][kMaxPrimes], garner_q[kMaxPrimes][kMaxPrimes];
  u64 q_words[kMaxWords];       // Q
  u64 pow64_mod[kMaxPrimes][kMaxWords];  // 2^(64i) mod p_j
  // exact scale-and-round (valid when has_scale)
  int has_scale;
  u64 t;
  BaseDev q_to_b, b_to_q;
  u64 inv_q_mod_b[kMaxPrimes], inv_q_mod_b_q[kMaxPrimes];
  u64 t_mod[kMaxPrimes], t_mod_q[kMaxPrimes];  // t mod p_j (Shoup)
};

// ---- negacyclic NTT of one plane in shared memory ---------------------------
// Shared-memory planes are padded by one u64 every 16 elements so that the
// stride-1 radix-16 blocks of the last passes do not all hit one bank.
__device__ __forceinline__ int sp(int i) { return i + (i >> 4); }
__host__ __device__ constexpr size_t plane_smem_words(int n) { return size_t(n) + size_t(n) / 16 + 16; }

// Forward (decimation in frequency, psi^bitrev twiddles, bit-reversed output)
// as passes of up to four radix-2 stages held in registers: a block of E = 2^P
// elements at stride `stride` runs stages s0 .. s0+P-1 without touching shared
// memory.  Stage s has 2^s groups of gap N/2^(s+1); inside a block the group
// of element k at stage s0+t is G*2^t + (k >> (P-t)).
// kHalf: the plane is half `half` (0 or 1) of a transform of twice its
// length whose first stage has already run; its stage s is the full
// transform's stage s + 1, whose twiddles for this half start at m (2 + half)
// instead of m.
// Lazy bounds (every ring prime is below 2^60, so 16p < 2^64): a pass takes
// values below 16p, its first stage brings u below 8p with one conditional
// subtraction, and each stage adds less than 2p (the Shoup product is below
// 2p for any 64-bit input), so after at most four stages the values are
// below 16p again.  Only the first stage of a pass corrects u; `last` then
// reduces the outputs to [0, p).
__device__ __forceinline__ u64 reduce_below_16p(u64 v, u64 p) {
  v = v >= 8 * p ? v - 8 * p : v;
  v = v >= 4 * p ? v - 4 * p : v;
  v = v >= 2 * p ? v - 2 * p : v;
  return v >= p ? v - p : v;
}

template <int P, bool kHalf = false>
__device__ __forceinline__ void ntt_forward_pass(u64* a, int s0, int logn, const ulonglong2* __restrict__ w2,
                                                 u64 p, bool last, int half_id = 0) {
  static_assert(P >= 1 && P <= 4, "at most four stages per pass keep values below 16p");
  constexpr int E = 1 << P;
  const int n = 1 << logn;
  const u64 two_p = 2 * p, eight_p = 8 * p;
  const int g = n >> (s0 + 1);
  const int stride = g >> (P - 1);
  const int log_stride = (logn - s0 - 1) - (P - 1);
  const int nblocks = n >> P;
  for (int blk = threadIdx.x; blk < nblocks; blk += blockDim.x) {
    const int G = blk >> log_stride, jj = blk & (stride - 1);
    const int base = G * 2 * g + jj;
    u64 x[E];
#pragma unroll
    for (int k = 0; k < E; ++k) x[k] = a[sp(base + k * stride)];
#pragma unroll
    for (int t = 0; t < P; ++t) {
      const int half = E >> (t + 1);
      const int m = 1 << (s0 + t);
#pragma unroll
      for (int k = 0; k < E; ++k) {
        if (k & half) continue;
        const int idx = (kHalf ? m * (2 + half_id) : m) + (G << t) + (k >> (P - t));
        const ulonglong2 tw = __ldg(w2 + idx);
        const u64 root = tw.x, rq = tw.y;
        u64 u = x[k];
        if (t == 0 && u >= eight_p) u -= eight_p;
        const u64 v = shoup_lazy(x[k + half], root, rq, p);
        x[k] = u + v;
        x[k + half] = u + two_p - v;
      }
    }
#pragma unroll
    for (int k = 0; k < E; ++k) a[sp(base + k * stride)] = last ? reduce_below_16p(x[k], p) : x[k];
  }
}

// Inverse (decimation in time) passes: stage u has gap 2^u and N/2^(u+1)
// groups; the final stage (gap N/2) folds in 1/N and the inverse twist.
template <int P, bool kHalf = false, bool kFinal = false>
__device__ __forceinline__ void ntt_inverse_pass(u64* a, int u0, int logn, const ulonglong2* __restrict__ w2,
                                                 u64 p, u64 n_inv, u64 n_inv_q, u64 last_w, u64 last_q,
                                                 int half_id = 0) {
  constexpr int E = 1 << P;
  const int n = 1 << logn;
  const u64 two_p = 2 * p;
  const int stride = 1 << u0;
  const int nblocks = n >> P;
  for (int blk = threadIdx.x; blk < nblocks; blk += blockDim.x) {
    const int G = blk >> u0, jj = blk & (stride - 1);
    const int base = (G << (u0 + P)) + jj;
    u64 x[E];
#pragma unroll
    for (int k = 0; k < E; ++k) x[k] = a[sp(base + k * stride)];
#pragma unroll
    for (int t = 0; t < P; ++t) {
      const int half = 1 << t;
      const int stage = u0 + t;
      const bool final_stage = kFinal && t == P - 1;  // kFinal: this pass ends at stage logn - 1
      const int m = n >> (stage + 1);
#pragma unroll
      for (int k = 0; k < E; ++k) {
        if (k & half) continue;
        const u64 u = x[k], v = x[k + half];
        if (final_stage) {
          x[k] = shoup(u + v, n_inv, n_inv_q, p);
          x[k + half] = shoup(u + two_p - v, last_w, last_q, p);
        } else {
          const int idx = m + (G << (P - t - 1)) + (k >> (t + 1));
          const ulonglong2 tw = __ldg(w2 + (kHalf ? idx + m * (1 + half_id) : idx));
          const u64 root = tw.x, rq = tw.y;
          const u64 s = u + v;
          x[k] = s >= two_p ? s - two_p : s;
          x[k + half] = shoup_lazy(u + two_p - v, root, rq, p);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < E; ++k) a[sp(base + k * stride)] = x[k];
  }
}

// Whole transforms over a padded shared-memory plane (all threads of the CTA).
// max_p (1..4) caps the stages per register pass (radix 2^max_p).
// kHalf: the plane is half `half_id` of a transform of length 2^(logn + 1)
// (logn = R.logn - 1): forward after that transform's first stage, inverse
// before its last (whose 1/N and twist the caller applies).
// canonical = false leaves the outputs below 16p (for callers that only
// multiply them by Shoup products).
template <bool kHalf = false>
__device__ __forceinline__ void ntt_forward_fast(u64* a, const RingDev& R, int j, int max_p = 4, int half_id = 0,
                                                 bool canonical = true) {
  const int logn = kHalf ? R.logn - 1 : R.logn;
  const u64 p = R.prime[j].p;
  const ulonglong2* w2 = R.fwd2[j];
  for (int s0 = 0; s0 < logn; s0 += max_p) {
    const int P = logn - s0 < max_p ? logn - s0 : max_p;
    const bool last = canonical && s0 + P == logn;
    switch (P) {
      case 4: ntt_forward_pass<4, kHalf>(a, s0, logn, w2, p, last, half_id); break;
      case 3: ntt_forward_pass<3, kHalf>(a, s0, logn, w2, p, last, half_id); break;
      case 2: ntt_forward_pass<2, kHalf>(a, s0, logn, w2, p, last, half_id); break;
      default: ntt_forward_pass<1, kHalf>(a, s0, logn, w2, p, last, half_id); break;
    }
    __syncthreads();
  }
}

// The first `stages` stages of the forward transform (outputs below 16p);
// the caller applies the rest.
__device__ __forceinline__ void ntt_forward_stages(u64* a, const RingDev& R, int j, int max_p, int stages) {
  const int logn = R.logn;
  const u64 p = R.prime[j].p;
  const ulonglong2* w2 = R.fwd2[j];
  for (int s0 = 0; s0 < stages; s0 += max_p) {
    const int P = stages - s0 < max_p ? stages - s0 : max_p;
    switch (P) {
      case 4: ntt_forward_pass<4, false>(a, s0, logn, w2, p, false, 0); break;
      case 3: ntt_forward_pass<3, false>(a, s0, logn, w2, p, false, 0); break;
      case 2: ntt_forward_pass<2, false>(a, s0, logn, w2, p, false, 0); break;
      default: ntt_forward_pass<1, false>(a, s0, logn, w2, p, false, 0); break;
    }
    __syncthreads();
  }
}

template <bool kHalf = false>
__device__ __forceinline__ void ntt_inverse_fast(u64* a, const RingDev& R, int j, int max_p = 4, int half_id = 0) {
  const int logn = kHalf ? R.logn - 1 : R.logn;
  const u64 p = R.prime[j].p;
  const ulonglong2* w2 = R.inv2[j];
  for (int u0 = 0; u0 < logn; u0 += max_p) {
    const int P = logn - u0 < max_p ? logn - u0 : max_p;
    const int key = P * 2 + (!kHalf && u0 + P == logn ? 1 : 0);
#define CUHE_INV_PASS(PP, F) \
  ntt_inverse_pass<PP, kHalf, F>(a, u0, logn, w2, p, R.n_inv[j], R.n_inv_q[j], R.last[j], R.last_q[j], half_id)
    switch (key) {
      case 9: CUHE_INV_PASS(4, true); break;
      case 8: CUHE_INV_PASS(4, false); break;
      case 7: CUHE_INV_PASS(3, true); break;
      case 6: CUHE_INV_PASS(3, false); break;
      case 5: CUHE_INV_PASS(2, true); break;
      case 4: CUHE_INV_PASS(2, false); break;
      case 3: CUHE_INV_PASS(1, true); break;
      default: CUHE_INV_PASS(1, false); break;
    }
#undef CUHE_INV_PASS
    __syncthreads();
  }
}

// The inverse transform from stage `first` on (the caller applied the
// earlier ones; inputs below 2p), including the final 1/N and twist.
__device__ __forceinline__ void ntt_inverse_from(u64* a, const RingDev& R, int j, int max_p, int first) {
  const int logn = R.logn;
  const u64 p = R.prime[j].p;
  const ulonglong2* w2 = R.inv2[j];
  for (int u0 = first; u0 < logn; u0 += max_p) {
    const int P = logn - u0 < max_p ? logn - u0 : max_p;
    const int key = P * 2 + (u0 + P == logn ? 1 : 0);
#define CUHE_INV_PASS(PP, F) \
  ntt_inverse_pass<PP, false, F>(a, u0, logn, w2, p, R.n_inv[j], R.n_inv_q[j], R.last[j], R.last_q[j], 0)
    switch (key) {
      case 9: CUHE_INV_PASS(4, true); break;
      case 8: CUHE_INV_PASS(4, false); break;
      case 7: CUHE_INV_PASS(3, true); break;
      case 6: CUHE_INV_PASS(3, false); break;
      case 5: CUHE_INV_PASS(2, true); break;
      case 4: CUHE_INV_PASS(2, false); break;
      case 3: CUHE_INV_PASS(1, true); break;
      default: CUHE_INV_PASS(1, false); break;
    }
#undef CUHE_INV_PASS
    __syncthreads();
  }
}

// The inverse transform's first stage (gap 1) on the pair (x0, x1) =
// coefficients (2b, 2b + 1), inputs below 2p, outputs below 2p.
__device__ __forceinline__ void inverse_stage0(u64& x0, u64& x1, const ulonglong2* __restrict__ w2, int half_n,
                                               int b, u64 p) {
  const ulonglong2 tw = __ldg(w2 + half_n + b);
  const u64 two_p = 2 * p, u = x0, v = x1;
  const u64 s = u + v;
  x0 = s >= two_p ? s - two_p : s;
  x1 = shoup_lazy(u + two_p - v, tw.x, tw.y, p);
}

// Batched transform: plane b of `data` (stride n) uses prime prime_of(b).
// prime = (b / prime_block) % prime_mod + prime_base.  MAXP bounds the
// register pass width at compile time: radix-8 passes fit 64 registers, so
// the <3> kernel runs 1024-thread CTAs; the <4> kernel (radix 16) needs more
// registers per thread and runs smaller CTAs.
template <int MAXP>
__device__ __forceinline__ void ntt_plane(u64* data, const RingDev* __restrict__ ring, int prime_base, int prime_mod,
                                          int prime_block, int inverse, int max_p) {
  extern __shared__ __align__(16) u64 s_plane[];
  const RingDev& R = *ring;
  const int n = R.n;
  long long b = blockIdx.x;
  const long long group = (long long)prime_mod * prime_block;
  if (prime_mod > 1 && gridDim.x % group == 0) {
    // prime-major order: CTAs launched together transform planes of the
    // same prime, so they share its twiddle table in L1 / L2 (a bijection:
    // slot s, index k -> ((k / block) * mod + s) * block + k % block)
    const long long per_slot = gridDim.x / prime_mod;
    const long long slot = b / per_slot, k = b % per_slot;
    b = ((k / prime_block) * prime_mod + slot) * prime_block + k % prime_block;
  }
  const int j = prime_base + int((b / prime_block) % prime_mod);
  u64* plane = data + b * n;
  const u64 p = R.prime[j].p;
  max_p = max_p < MAXP ? max_p : MAXP;
  // 16-byte global accesses when the plane allows them (pairs 2i, 2i + 1
  // never straddle a padding gap of sp, which falls every 16 words).  When
  // the stages leave a single one over (log2 N = 1 mod max_p), the gap-1
  // stage runs on those pairs in registers: the forward transform's last
  // before the store, the inverse transform's first after the load.
  const bool wide = (reinterpret_cast<uintptr_t>(plane) & 15) == 0;
  const bool pairs = wide && R.logn % max_p == 1 && R.logn > 1;
  const int half_n = n / 2;
  if (wide) {
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(plane);
    for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
      const ulonglong2 v = src[i];
      u64 x0 = v.x, x1 = v.y;
      if (pairs && inverse) inverse_stage0(x0, x1, R.inv2[j], half_n, i, p);
      s_plane[sp(2 * i)] = x0;
      s_plane[sp(2 * i) + 1] = x1;
    }
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_plane[sp(i)] = plane[i];
  }
  __syncthreads();
  if (inverse) {
    if (pairs) ntt_inverse_from(s_plane, R, j, max_p, 1);
    else ntt_inverse_fast(s_plane, R, j, max_p);
  } else {
    if (pairs) ntt_forward_stages(s_plane, R, j, max_p, R.logn - 1);
    else ntt_forward_fast(s_plane, R, j, max_p);
  }
  if (wide) {
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(plane);
    const ulonglong2* w2 = R.fwd2[j];
    const u64 two_p = 2 * p;
    for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
      const int at = sp(2 * i);
      u64 x0 = s_plane[at], x1 = s_plane[at + 1];
      if (pairs && !inverse) {
        // the last forward stage: gap 1, twiddle (N/2 + i), canonical outputs
        // (inputs below 16p: u is brought below 8p, the outputs are below 10p)
        const ulonglong2 tw = __ldg(w2 + half_n + i);
        if (x0 >= 8 * p) x0 -= 8 * p;
        const u64 v = shoup_lazy(x1, tw.x, tw.y, p);
        x1 = reduce_below_16p(x0 + two_p - v, p);
        x0 = reduce_below_16p(x0 + v, p);
      }
      dst[i] = make_ulonglong2(x0, x1);
    }
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) plane[i] = s_plane[sp(i)];
  }
}

__global__ void k_ntt(u64* data, const RingDev* __restrict__ ring, int prime_base, int prime_mod, int prime_block,
                      int inverse, int max_p = 4) {
  ntt_plane<4>(data, ring, prime_base, prime_mod, prime_block, inverse, max_p);
}

__global__ void __launch_bounds__(1024, 1)
k_ntt8(u64* data, const RingDev* __restrict__ ring, int prime_base, int prime_mod, int prime_block, int inverse,
       int max_p = 3) {
  ntt_plane<3>(data, ring, prime_base, prime_mod, prime_block, inverse, max_p);
}

// ---- transforms of N = 32768 (a plane exceeds one CTA's shared memory) ------
// The first forward stage (gap N/2, one twiddle) and the last inverse stage
// (1/N and the twist) pair the two halves of a plane and run as elementwise
// kernels on global memory; every other stage stays within a half, which a
// CTA transforms in shared memory (k_ntt_half).  Planes follow launch_ntt's
// prime mapping: prime = (b / prime_block) % prime_mod + prime_base.
__device__ __forceinline__ int plane_prime(long long b, int prime_base, int prime_mod, int prime_block) {
  return prime_base + int((b / prime_block) % prime_mod);
}

// forward stage 0 (inputs canonical; outputs below 4p, within the passes' 16p)
// or, with kInverse, the final inverse stage (inputs below 2p, outputs
// canonical); one thread per pair (i, i + N/2)
template <bool kInverse>
__global__ void k_ntt_cross(u64* __restrict__ data, long long planes, const RingDev* __restrict__ ring, int prime_base,
                            int prime_mod, int prime_block) {
  const RingDev& R = *ring;
  const int hn = R.n >> 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= planes * hn) return;
  const long long b = idx / hn;
  const int i = int(idx % hn);
  const int j = plane_prime(b, prime_base, prime_mod, prime_block);
  const u64 p = R.prime[j].p, two_p = 2 * p;
  u64* a = data + b * R.n;
  const u64 u = a[i], v = a[i + hn];
  if (kInverse) {
    a[i] = shoup(u + v, R.n_inv[j], R.n_inv_q[j], p);
    a[i + hn] = shoup(u + two_p - v, R.last[j], R.last_q[j], p);
  } else {
    const ulonglong2 tw = __ldg(R.fwd2[j] + 1);  // stage 0: one group
    const u64 w = shoup_lazy(v, tw.x, tw.y, p);
    a[i] = u + w;
    a[i + hn] = u + two_p - w;
  }
}

// stages 1 .. logN - 1 (forward) or 0 .. logN - 2 (inverse) of one half:
// CTA b transforms half (b & 1) of plane b >> 1
template <bool kInverse>
__global__ void __launch_bounds__(1024, 1)
k_ntt_half(u64* __restrict__ data, const RingDev* __restrict__ ring, int prime_base, int prime_mod, int prime_block) {
  extern __shared__ __align__(16) u64 s_plane[];
  const RingDev& R = *ring;
  const int hn = R.n >> 1;
  const long long b = blockIdx.x >> 1;
  const int h = int(blockIdx.x & 1);
  const int j = plane_prime(b, prime_base, prime_mod, prime_block);
  u64* a = data + b * R.n + (long long)h * hn;
  for (int i = threadIdx.x; i < hn; i += blockDim.x) s_plane[sp(i)] = a[i];
  __syncthreads();
  if (kInverse) ntt_inverse_fast<true>(s_plane, R, j, 3, h);
  else ntt_forward_fast<true>(s_plane, R, j, 3, h);
  for (int i = threadIdx.x; i < hn; i += blockDim.x) a[i] = s_plane[sp(i)];
}

// ---- wire unpacking ---------------------------------------------------------
__device__ __forceinline__ u64 load_word_bytes(const uint8_t* data, long long nbytes, long long offset) {
  u64 r = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const long long at = offset + k;
    if (at < nbytes) r |= u64(data[at]) << (8 * k);
  }
  return r;
}

// words[poly][i][W] from `bits`-bit packed little-endian coefficients; each
// coefficient must be < Q (status bit 1 otherwise).
__global__ void k_unpack(const uint8_t* __restrict__ wire, long long poly_bytes, int bits, int polys,
                         u64* __restrict__ words, const RingDev* __restrict__ ring, int* status) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)polys * R.n;
  if (idx >= total) return;
  const long long poly = idx / R.n;
  const long long i = idx % R.n;
  const uint8_t* src = wire + poly * poly_bytes;
  const long long bit0 = i * bits;
  const long long off = (bit0 / 64) * 8;
  const int sh = int(bit0 % 64);
  const int W = R.words;
  const int nw = (bits + 63) / 64;
  u64 v[kMaxWords];
#pragma unroll
  for (int k = 0; k < kMaxWords; ++k) v[k] = 0;
  for (int k = 0; k < nw; ++k) {
    u64 x = load_word_bytes(src, poly_bytes, off + 8 * k) >> sh;
    if (sh) x |= load_word_bytes(src, poly_bytes, off + 8 * k + 8) << (64 - sh);
    v[k] = x;
  }
  if (bits % 64) v[nw - 1] &= (u64(1) << (bits % 64)) - 1;
  // v < Q ?
  bool less = false, decided = false;
  for (int k = W - 1; k >= 0 && !decided; --k) {
    if (v[k] != R.q_words[k]) { less = v[k] < R.q_words[k]; decided = true; }
  }
  if (!less) atomicOr(status, 1);
  u64* dst = words + idx * W;
  for (int k = 0; k < W; ++k) dst[k] = v[k];
}

// value mod p_j of a composed W-word integer (Horner over 64-bit words)
__device__ __forceinline__ u64 words_mod(const u64* v, int W, const RingDev& R, int j) {
  u128 acc = 0;
  for (int k = 0; k < W; ++k) acc += u128(v[k]) * R.pow64_mod[j][k];
  return reduce128(acc, R.prime[j]);
}

// out[poly][j][i] = words[poly][i] mod p_j for j < primes_out
__global__ void k_words_to_residues(const u64* __restrict__ words, long long polys, int primes_out,
                                    u64* __restrict__ out, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  const u64* w = words + idx * R.words;
  for (int j = 0; j < primes_out; ++j) out[(poly * primes_out + j) * R.n + i] = words_mod(w, R.words, R, j);
}

// residues[t][c][j][i] of (query - tile) mod Q for c in {0,1}, j < primes_out.
__global__ void k_diff_residues(const u64* __restrict__ query_words, const u64* __restrict__ tile_words,
                                int tiles, int primes_out, u64* __restrict__ out, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_tile = 2LL * R.n;
  if (idx >= tiles * per_tile) return;
  const long long t = idx / per_tile;
  const int c = int((idx % per_tile) / R.n);
  const int i = int(idx % R.n);
  const int W = R.words;
  const u64* a = query_words + ((long long)c * R.n + i) * W;
  const u64* b = tile_words + ((t * 2 + c) * R.n + i) * W;
  u64 d[kMaxWords];
  u64 borrow = 0;
  for (int k = 0; k < W; ++k) {
    const u128 x = u128(a[k]) - b[k] - borrow;
    d[k] = u64(x);
    borrow = u64(x >> 64) ? 1 : 0;
  }
  if (borrow) {
    u64 carry = 0;
    for (int k = 0; k < W; ++k) {
      const u128 s = u128(d[k]) + R.q_words[k] + carry;
      d[k] = u64(s);
      carry = u64(s >> 64);
    }
  }
  for (int j = 0; j < primes_out; ++j)
    out[((t * 2 + c) * primes_out + j) * R.n + i] = words_mod(d, W, R, j);
}

// NTT-domain tensor of (x0, x1) and (y0, y1): out = (x0 y0, x0 y1 + x1 y0, x1 y1).
__global__ void k_tensor(const u64* __restrict__ x, const u64* __restrict__ y, int polys, int primes,
                         u64* __restrict__ out, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)primes * R.n;
  if (idx >= polys * per) return;
  const long long t = idx / per;
  const int j = int((idx % per) / R.n);
  const int i = int(idx % R.n);
  const Prime& m = R.prime[j];
  const u64 a0 = x[((t * 2 + 0) * primes + j) * R.n + i], a1 = x[((t * 2 + 1) * primes + j) * R.n + i];
  const u64 b0 = y[((t * 2 + 0) * primes + j) * R.n + i], b1 = y[((t * 2 + 1) * primes + j) * R.n + i];
  out[((t * 3 + 0) * primes + j) * R.n + i] = reduce128(u128(a0) * b0, m);
  out[((t * 3 + 1) * primes + j) * R.n + i] = reduce128(u128(a0) * b1 + u128(a1) * b0, m);
  out[((t * 3 + 2) * primes + j) * R.n + i] = reduce128(u128(a1) * b1, m);
}

// NTT-domain square of (x0, x1): out = (x0^2, 2 x0 x1, x1^2) per prime.
__global__ void k_tensor_square(const u64* __restrict__ x, int tiles, int primes, u64* __restrict__ out,
                                const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_tile = (long long)primes * R.n;
  if (idx >= tiles * per_tile) return;
  const long long t = idx / per_tile;
  const int j = int((idx % per_tile) / R.n);
  const int i = int(idx % R.n);
  const Prime& m = R.prime[j];
  const u64 a = x[((t * 2 + 0) * primes + j) * R.n + i];
  const u64 b = x[((t * 2 + 1) * primes + j) * R.n + i];
  const u128 ab = u128(a) * b;
  out[((t * 3 + 0) * primes + j) * R.n + i] = reduce128(u128(a) * a, m);
  // x0*x1 + x1*x0 (< 2^121, exact in 128 bits)
  out[((t * 3 + 1) * primes + j) * R.n + i] = reduce128(ab + ab, m);
  out[((t * 3 + 2) * primes + j) * R.n + i] = reduce128(u128(b) * b, m);
}

// ---- exact RNS scale-and-round (round(t z / Q) mod Q from z mod P) -----------
__device__ __forceinline__ void words_addmul(u64 (&v)[kCrtWordsDev], const u64* src, u64 m) {
  u128 c = 0;
#pragma unroll 1
  for (int i = 0; i < kCrtWordsDev; ++i) {
    c += u128(src[i]) * m + v[i];
    v[i] = u64(c);
    c >>= 64;
  }
}

__device__ __forceinline__ bool words_ge(const u64 (&a)[kCrtWordsDev], const u64 (&b)[kCrtWordsDev]) {
  for (int i = kCrtWordsDev - 1; i >= 0; --i)
    if (a[i] != b[i]) return a[i] > b[i];
  return true;
}

struct Normalized {
  u64 terms[kMaxPrimes];
  u64 alpha;
};

// A = sum terms_j M_j, theta = A/M; alpha = floor(theta) or round(theta),
// certified by a fixed-point interval with an exact multiword fallback.
__device__ __forceinline__ void normalize(const BaseDev& B, const RingDev& R, const u64* residues, bool centered,
                                          Normalized& out) {
  u128 frac = 0;
  for (int j = 0; j < B.count; ++j) {
    const Prime& m = R.prime[B.start + j];
    out.terms[j] = shoup(residues[j], B.inv[j], B.inv_q[j], m.p);
    frac += fraction64(out.terms[j], m);
  }
  const u128 bias = centered ? (u128(1) << 63) : 0;
  out.alpha = u64((frac + bias) >> 64);
  if (out.alpha != u64((frac + u128(B.count) + bias) >> 64)) {
    u64 sum[kCrtWordsDev], rhs[kCrtWordsDev];
    for (int i = 0; i < kCrtWordsDev; ++i) sum[i] = rhs[i] = 0;
    for (int j = 0; j < B.count; ++j) words_addmul(sum, B.partial_words[j], out.terms[j]);
    if (centered) {
      u64 twice[kCrtWordsDev];
      for (int i = 0; i < kCrtWordsDev; ++i) twice[i] = 0;
      words_addmul(twice, sum, 2);
      words_addmul(rhs, B.product_words, 2 * out.alpha + 1);
      if (words_ge(twice, rhs)) ++out.alpha;
    } else {
      words_addmul(rhs, B.product_words, out.alpha + 1);
      if (words_ge(sum, rhs)) ++out.alpha;
    }
  }
}

__device__ __forceinline__ void convert(const BaseDev& B, const RingDev& R, const Normalized& v, u64* out) {
  for (int k = 0; k < B.tcount; ++k) {
    const Prime& m = R.prime[B.tstart + k];
    u128 s = 0;
    for (int j = 0; j < B.count; ++j) s += u128(v.terms[j]) * B.partial_mod_target[k][j];
    const u64 residue = reduce128(s, m);
    const u64 corr = shoup(v.alpha, B.product_mod_target[k], B.product_mod_target_q[k], m.p);
    out[k] = submod(residue, corr, m.p);
  }
}

// round(t r / M) for r = A - alpha M (the canonical lift)
__device__ __forceinline__ u64 round_fraction(const BaseDev& B, const RingDev& R, const Normalized& v, u64 t) {
  u64 whole = 0;
  u128 frac = 0;
  for (int j = 0; j < B.count; ++j) {
    const Prime& m = R.prime[B.start + j];
    u64 q, r;
    divide128(u128(t) * v.terms[j], m, &q, &r);
    whole += q;
    frac += fraction64(r, m);
  }
  const u128 half = u128(1) << 63;
  u64 rounded = whole + u64((frac + half) >> 64);
  if (((frac + half) >> 64) != ((frac + u128(B.count) + half) >> 64)) {
    u64 sum[kCrtWordsDev], lhs[kCrtWordsDev], rhs[kCrtWordsDev];
    for (int i = 0; i < kCrtWordsDev; ++i) sum[i] = lhs[i] = rhs[i] = 0;
    for (int j = 0; j < B.count; ++j) words_addmul(sum, B.partial_words[j], v.terms[j]);
    words_addmul(lhs, sum, 2 * t);
    words_addmul(rhs, B.product_words, 2 * rounded + 1);
    if (words_ge(lhs, rhs)) ++rounded;
  }
  return rounded - t * v.alpha;
}

// tensor[poly][K][N] (coefficient domain, residues of the signed product z)
// -> out[poly][L][N] = round(t z / Q) mod Q, per coefficient.
__global__ void k_rns_scale(const u64* __restrict__ tensor, long long polys, u64* __restrict__ out,
                            const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  const int L = R.residue, K = R.tensor;
  const u64* z = tensor + poly * K * R.n + i;
  u64 rem[kMaxPrimes], quot[kMaxPrimes], rb[kMaxPrimes], kq[kMaxPrimes];
  for (int j = 0; j < L; ++j) rem[j] = z[j * R.n];
  Normalized nq;
  normalize(R.q_to_b, R, rem, false, nq);
  convert(R.q_to_b, R, nq, rb);
  const u64 rounded = round_fraction(R.q_to_b, R, nq, R.t);
  for (int j = 0; j < K - L; ++j) {
    const u64 p = R.prime[L + j].p;
    const u64 residue = submod(z[(L + j) * R.n], rb[j], p);
    quot[j] = shoup(residue, R.inv_q_mod_b[j], R.inv_q_mod_b_q[j], p);
  }
  Normalized nb;
  normalize(R.b_to_q, R, quot, true, nb);
  convert(R.b_to_q, R, nb, kq);
  for (int j = 0; j < L; ++j) {
    const u64 p = R.prime[j].p;
    const u64 r = rounded >= p ? rounded - p : rounded;
    const u64 c = shoup(kq[j], R.t_mod[j], R.t_mod_q[j], p) + r;
    out[(poly * L + j) * R.n + i] = c >= p ? c - p : c;
  }
}

// ---- key switching ------------------------------------------------------------
// One key-switch job: out_k = base_k + [k == 0] sigma_g(x0) + KS(sigma_g(x1))_k,
// with sigma_g the Galois automorphism X -> X^g (g = 1: identity).
struct SwitchOp {
  const u64* base;   // [2][L][N] or null
  const u64* x0;     // [L][N] or null
  const u64* words;  // composed sigma_g(x1): [N][W]
  const u64* key;    // [D][2][L][N] NTT domain
  const u64* key_q;  // Shoup quotients floor(key * 2^64 / p), same layout
  u64* out;          // [2][L][N]
  unsigned g_inv;    // inverse of g mod 2N (gather for x0)
  unsigned pad;
  // [L][N] NTT-domain plaintext or null: the output is multiplied by it
  // (k_keyswitch_tm only).  out may alias base and x0: each CTA reads its
  // prime's planes of them whole before it writes that prime's output.
  const u64* mask = nullptr;
};

struct ComposeOp {
  const u64* x1;  // [L][N] coefficient residues
  u64* words;     // [N][W] output
  unsigned g;
  unsigned pad;
};

// Garner: canonical integer in [0, Q) of each coefficient, written to the
// position of X^g (negated when the exponent wraps past N).  kL: the ring's
// residue count as a compile-time constant (its words then equal kL: 60-bit
// primes), which keeps the digits and words in registers; 0 = any.
template <int kL>
__global__ void k_compose(const ComposeOp* __restrict__ ops, const RingDev* __restrict__ ring) {
  constexpr int kD = kL ? kL : kMaxResidue, kWw = kL ? kL : kMaxWords;
  const RingDev& R = *ring;
  const ComposeOp op = ops[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.n) return;
  const int L = kL ? kL : R.residue, W = kL ? kL : R.words;
  u64 digit[kD];
#pragma unroll
  for (int j = 0; j < kD; ++j) {
    if (j >= L) break;
    const u64 p = R.prime[j].p;
    u64 value = op.x1[(long long)j * R.n + i];
#pragma unroll
    for (int k = 0; k < kD; ++k) {
      if (k >= j) break;
      const u64 d = digit[k] >= p ? digit[k] - p : digit[k];
      value = shoup(value + p - d, R.garner[j][k], R.garner_q[j][k], p);
    }
    digit[j] = value;
  }
  // Horner over the mixed radix; every partial value is below the product
  // of the primes used so far, so W words always hold it
  u64 w[kWw];
#pragma unroll
  for (int k = 0; k < kWw; ++k) w[k] = 0;
  w[0] = digit[L - 1];
#pragma unroll
  for (int jj = kD - 1; jj > 0; --jj) {
    if (jj > L - 1) continue;
    u64 carry = digit[jj - 1];
    const u64 p = R.prime[jj - 1].p;
#pragma unroll
    for (int k = 0; k < kWw; ++k) {
      if (k >= W) break;
      const u128 prod = u128(w[k]) * p + carry;
      w[k] = u64(prod);
      carry = u64(prod >> 64);
    }
  }
  const unsigned at = unsigned((unsigned long long)i * op.g % (2u * unsigned(R.n)));
  const int dst = int(at % unsigned(R.n));
  bool nonzero = false;
#pragma unroll
  for (int k = 0; k < kWw; ++k)
    if (k < W) nonzero |= w[k] != 0;
  if (at >= unsigned(R.n) && nonzero) {
    u64 borrow = 0;
#pragma unroll
    for (int k = 0; k < kWw; ++k) {
      if (k >= W) break;
      const u128 x = u128(R.q_words[k]) - w[k] - borrow;
      w[k] = u64(x);
      borrow = u64(x >> 64) ? 1 : 0;
    }
  }
  u64* o = op.words + (long long)dst * W;
#pragma unroll
  for (int k = 0; k < kWw; ++k)
    if (k < W) o[k] = w[k];
}

// digit d of a composed integer, reduced mod p_j
__device__ __forceinline__ u64 gadget_digit(const u64* w, int W, int d, const RingDev& R, int j) {
  const int bits = R.digit_bits;
  const int start = d * bits;
  const Prime& m = R.prime[j];
  if (bits <= 64) {
    const int limb = start / 64, off = start % 64;
    u64 v = limb < W ? (w[limb] >> off) : 0;
    if (off && limb + 1 < W) v |= w[limb + 1] << (64 - off);
    if (bits < 64) v &= (u64(1) << bits) - 1;
    if (bits <= 60) return v >= m.p ? v - m.p : v;
    return v % m.p;
  }
  // wide digit: Horner over 64-bit chunks from the top of [start, start+bits)
  u64 r = 0;
  int remaining = bits;
  while (remaining > 0) {
    const int take = remaining > 64 ? 64 : remaining;
    const int lo = start + remaining - take;
    const int limb = lo / 64, off = lo % 64;
    u64 v = limb < W ? (w[limb] >> off) : 0;
    if (off && limb + 1 < W) v |= w[limb + 1] << (64 - off);
    if (take < 64) v &= (u64(1) << take) - 1;
    const u128 shifted = take == 64 ? (u128(r) << 64) : (u128(r) << take);
    r = reduce128(shifted + v, m);
    remaining -= take;
  }
  return r;
}

// ---- tensor memory (TMEM) as accumulator storage ------------------------------
// Each SM has 512 TMEM columns x 128 lanes of 32 bits.  A CTA allocates
// columns with tcgen05.alloc (one warp; the address lands in shared memory),
// and warp w may access lanes 32 (w % 4) .. 32 (w % 4) + 31 only.  The
// 32x32b shapes move one lane per thread: thread t of the warp reads or
// writes 16 consecutive columns of lane 32 (w % 4) + t.
__device__ __forceinline__ uint32_t smem_addr_u32(const void* ptr) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(ptr));
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_addr_u32(dst)), "r"(cols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// load 16 columns of this thread's lane; the registers are valid on return
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
               "tcgen05.wait::ld.sync.aligned;"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]) : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
               :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]) : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// The fused key switch.  CTA per (op, prime j < L): the D forward NTTs of
// the op's gadget digits mod p_j, their products with the key in the NTT
// domain (Shoup, precomputed quotients) accumulated over the digits, two
// inverse NTTs, and the epilogue additions (base, the permuted x0).  The
// accumulators live in TMEM: shared memory holds only the plane (70 KB at
// N = 8192), so two 512-thread CTAs (64 registers each) are resident per SM
// and one CTA's global loads and barriers overlap the other's butterflies.  Thread t owns
// coefficients i = t + 512 k (k < kCoef) and keeps (acc0, acc1) of each as
// four 32-bit columns: 4 kCoef columns per thread, lanes by warp quarter, 4
// warps per quarter -> 16 kCoef columns per CTA.  N <= 8192 (kCoef = 16):
// 256 columns, 512 for the two CTAs of an SM (the whole TMEM); N = 16384
// (kCoef = 32, a 139 KB plane, one CTA per SM): 512 columns.  A further
// co-resident CTA would wait in tcgen05.alloc until another deallocates.
// Every tcgen05 instruction is executed by whole warps (the coefficient
// guard i < n covers only the arithmetic), and no thread leaves before the
// final dealloc.
template <int MAXP, int kCoef = 16>
__global__ void __launch_bounds__(512, kCoef == 16 ? 2 : 1)
k_keyswitch_tm(const SwitchOp* __restrict__ ops, const RingDev* __restrict__ ring) {
  static_assert(kCoef == 16 || kCoef == 32, "16 or 32 coefficients per thread");
  constexpr int kThreads = 512, kChunks = kCoef / 4, kCols = 16 * kCoef;  // 4 coefficients per chunk
  extern __shared__ __align__(16) u64 s_plane[];
  __shared__ uint32_t s_tmem;
  const RingDev& R = *ring;
  const SwitchOp op = ops[blockIdx.x];
  const int j = blockIdx.y;
  const int n = R.n, L = R.residue, W = R.words;
  const u64 p = R.prime[j].p, two_p = 2 * p;
  const int warp = int(threadIdx.x >> 5);
  if (warp == 0) {
    tmem_alloc(&s_tmem, kCols);
    tmem_relinquish();
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tbase = s_tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t((warp >> 2) * 4 * kCoef);
  // When the forward transform's last pass would be a single stage (log2 N
  // = 1 mod MAXP), that stage runs in the product loop instead: thread t
  // takes coefficient pairs (2b, 2b + 1), b = t + kThreads k, applies the
  // stage's butterfly in registers and reads the key pairs as 16-byte
  // loads.  Column group kk of chunk c then holds coefficient
  // 2 (t + kThreads (2c + kk / 2)) + kk % 2 (else t + kThreads (4c + kk)).
  const bool pairs = R.logn % MAXP == 1 && R.logn > 1;
  auto coef = [&](int c, int kk) {
    return pairs ? 2 * (int(threadIdx.x) + (c * 2 + (kk >> 1)) * kThreads) + (kk & 1)
                 : int(threadIdx.x) + (c * 4 + kk) * kThreads;
  };
  const ulonglong2* w2 = R.fwd2[j];
  const int half_n = n >> 1;
  // each digit adds a key product below 2p: with at most eight digits the
  // sums stay below 16p and are reduced once, at the last digit
  const bool lazy_sum = R.digits <= 8;
  for (int d = 0; d < R.digits; ++d) {
    const int start = d * R.digit_bits, limb = start / 64, off = start % 64;
    if (R.digit_bits <= 63) {
      // digits below 2^63 < 16p enter the lazy transform unreduced; the
      // words of four coefficients are loaded before any is used
      const u64 dmask = (u64(1) << R.digit_bits) - 1;
      const bool two = off && off + R.digit_bits > 64 && limb + 1 < W;
      for (int i0 = int(threadIdx.x); i0 < n; i0 += 4 * kThreads) {
        u64 w0[4], w1[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + u * kThreads;
          const u64* w = op.words + (long long)i * W;
          w0[u] = i < n && limb < W ? w[limb] : 0;
          w1[u] = i < n && two ? w[limb + 1] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + u * kThreads;
          u64 v = w0[u] >> off;
          if (two) v |= w1[u] << (64 - off);
          if (i < n) s_plane[sp(i)] = v & dmask;
        }
      }
    } else {
      for (int i = threadIdx.x; i < n; i += kThreads)
        s_plane[sp(i)] = gadget_digit(op.words + (long long)i * W, W, d, R, j);
    }
    __syncthreads();
    // the digit transforms feed only the Shoup key products: no canonical pass
    if (pairs) ntt_forward_stages(s_plane, R, j, MAXP, R.logn - 1);
    else ntt_forward_fast(s_plane, R, j, MAXP, 0, false);
    const long long k0o = ((long long)(d * 2 + 0) * L + j) * n, k1o = ((long long)(d * 2 + 1) * L + j) * n;
    const bool last = d + 1 == R.digits;
#pragma unroll 1
    for (int c = 0; c < kChunks; ++c) {
      uint32_t acc[16];
      if (d > 0) {
        tmem_ld16(tbase + uint32_t(c * 16), acc);
      } else {
#pragma unroll
        for (int k = 0; k < 16; ++k) acc[k] = 0;
      }
      if (pairs) {
#pragma unroll
        for (int kp = 0; kp < 2; ++kp) {
          const int b = int(threadIdx.x) + (c * 2 + kp) * kThreads;
          if (b < half_n) {
            // the last forward stage: gap 1, twiddle (N/2 + b); the outputs
            // (below 10p) only enter Shoup products, so they stay unreduced
            u64 u = s_plane[sp(2 * b)];
            const u64 x1 = s_plane[sp(2 * b + 1)];
            const ulonglong2 tw = __ldg(w2 + half_n + b);
            if (u >= 8 * p) u -= 8 * p;
            const u64 v = shoup_lazy(x1, tw.x, tw.y, p);
            const u64 y[2] = {u + v, u + two_p - v};
            // one key component at a time keeps fewer registers live
            u64 out0[2];
#pragma unroll
            for (int comp = 0; comp < 2; ++comp) {
              const long long ko = comp ? k1o : k0o;
              const ulonglong2 kv = __ldg(reinterpret_cast<const ulonglong2*>(op.key + ko) + b);
              const ulonglong2 kq = __ldg(reinterpret_cast<const ulonglong2*>(op.key_q + ko) + b);
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int col = 4 * (2 * kp + e) + 2 * comp;
                u64 a = shoup_lazy(y[e], e ? kv.y : kv.x, e ? kq.y : kq.x, p);
                a += u64(acc[col]) | (u64(acc[col + 1]) << 32);
                if (!lazy_sum) a = a >= two_p ? a - two_p : a;
                if (last) a = lazy_sum ? reduce_below_16p(a, p) : a >= p ? a - p : a;
                if (comp == 0) out0[e] = a;
                acc[col] = uint32_t(a);
                acc[col + 1] = uint32_t(a >> 32);
              }
            }
            if (last && !op.mask) {
              // component 0 transforms first, its first inverse stage here
              inverse_stage0(out0[0], out0[1], R.inv2[j], half_n, b, p);
              s_plane[sp(2 * b)] = out0[0];
              s_plane[sp(2 * b + 1)] = out0[1];
            }
          }
        }
      } else {
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const int i = int(threadIdx.x) + (c * 4 + kk) * kThreads;
          if (i < n) {
            const u64 v = s_plane[sp(i)];
            u64 a0 = shoup_lazy(v, __ldg(op.key + k0o + i), __ldg(op.key_q + k0o + i), p);
            u64 a1 = shoup_lazy(v, __ldg(op.key + k1o + i), __ldg(op.key_q + k1o + i), p);
            a0 += u64(acc[4 * kk]) | (u64(acc[4 * kk + 1]) << 32);
            a1 += u64(acc[4 * kk + 2]) | (u64(acc[4 * kk + 3]) << 32);
            if (!lazy_sum) {
              a0 = a0 >= two_p ? a0 - two_p : a0;
              a1 = a1 >= two_p ? a1 - two_p : a1;
            }
            if (last) {
              a0 = lazy_sum ? reduce_below_16p(a0, p) : a0 >= p ? a0 - p : a0;
              a1 = lazy_sum ? reduce_below_16p(a1, p) : a1 >= p ? a1 - p : a1;
              s_plane[sp(i)] = a0;  // component 0 transforms first
            }
            acc[4 * kk] = uint32_t(a0);
            acc[4 * kk + 1] = uint32_t(a0 >> 32);
            acc[4 * kk + 2] = uint32_t(a1);
            acc[4 * kk + 3] = uint32_t(a1 >> 32);
          }
        }
      }
      tmem_st16(tbase + uint32_t(c * 16), acc);
    }
    tmem_wait_st();
    __syncthreads();
  }
  if (op.mask) {
    // masked output: NTT(out) = acc + NTT(base + sigma(x0)) exactly, so each
    // component transforms its addends forward, adds the accumulator, takes
    // the product with the mask and transforms back once
    const Prime& pr = R.prime[j];
    const u64* m = op.mask + (long long)j * n;
    for (int comp = 0; comp < 2; ++comp) {
      const u64* base = op.base ? op.base + ((long long)comp * L + j) * n : nullptr;
      for (int i = threadIdx.x; i < n; i += kThreads) {
        u64 v = base ? base[i] : 0;
        if (comp == 0 && op.x0) {
          const unsigned sidx = unsigned((unsigned long long)i * op.g_inv % (2u * unsigned(n)));
          u64 x = sidx < unsigned(n) ? op.x0[(long long)j * n + sidx] : op.x0[(long long)j * n + (sidx - n)];
          if (sidx >= unsigned(n) && x) x = p - x;
          v = addmod(v, x, p);
        }
        s_plane[sp(i)] = v;
      }
      __syncthreads();
      ntt_forward_fast(s_plane, R, j, MAXP);
#pragma unroll 1
      for (int c = 0; c < kChunks; ++c) {
        uint32_t acc[16];
        tmem_ld16(tbase + uint32_t(c * 16), acc);
        auto masked = [&](int kk, int i) {
          const u64 a0 = u64(acc[4 * kk]) | (u64(acc[4 * kk + 1]) << 32);
          const u64 a1 = u64(acc[4 * kk + 2]) | (u64(acc[4 * kk + 3]) << 32);
          const u64 a = comp == 0 ? a0 : a1;  // static register indices
          return reduce128(u128(addmod(s_plane[sp(i)], a, p)) * m[i], pr);
        };
        if (pairs) {
#pragma unroll
          for (int kp = 0; kp < 2; ++kp) {
            const int b = int(threadIdx.x) + (c * 2 + kp) * kThreads;
            if (b < half_n) {
              u64 x0 = masked(2 * kp, 2 * b), x1 = masked(2 * kp + 1, 2 * b + 1);
              inverse_stage0(x0, x1, R.inv2[j], half_n, b, p);
              s_plane[sp(2 * b)] = x0;
              s_plane[sp(2 * b + 1)] = x1;
            }
          }
        } else {
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const int i = coef(c, kk);
            if (i < n) s_plane[sp(i)] = masked(kk, i);
          }
        }
      }
      __syncthreads();
      if (pairs) ntt_inverse_from(s_plane, R, j, MAXP, 1);
      else ntt_inverse_fast(s_plane, R, j, MAXP);
      u64* out = op.out + ((long long)comp * L + j) * n;
      for (int i = threadIdx.x; i < n; i += kThreads) out[i] = s_plane[sp(i)];
      __syncthreads();
    }
  } else {
    for (int comp = 0; comp < 2; ++comp) {
      if (comp == 1) {
#pragma unroll 1
        for (int c = 0; c < kChunks; ++c) {
          uint32_t acc[16];
          tmem_ld16(tbase + uint32_t(c * 16), acc);
          if (pairs) {
#pragma unroll
            for (int kp = 0; kp < 2; ++kp) {
              const int b = int(threadIdx.x) + (c * 2 + kp) * kThreads;
              if (b < half_n) {
                u64 x0 = u64(acc[8 * kp + 2]) | (u64(acc[8 * kp + 3]) << 32);
                u64 x1 = u64(acc[8 * kp + 6]) | (u64(acc[8 * kp + 7]) << 32);
                inverse_stage0(x0, x1, R.inv2[j], half_n, b, p);
                s_plane[sp(2 * b)] = x0;
                s_plane[sp(2 * b + 1)] = x1;
              }
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
              const int i = coef(c, kk);
              if (i < n) s_plane[sp(i)] = u64(acc[4 * kk + 2]) | (u64(acc[4 * kk + 3]) << 32);
            }
          }
        }
        __syncthreads();
      }
      if (pairs) ntt_inverse_from(s_plane, R, j, MAXP, 1);
      else ntt_inverse_fast(s_plane, R, j, MAXP);
      u64* out = op.out + ((long long)comp * L + j) * n;
      const u64* base = op.base ? op.base + ((long long)comp * L + j) * n : nullptr;
      for (int i = threadIdx.x; i < n; i += kThreads) {
        u64 v = s_plane[sp(i)];
        if (base) v = addmod(v, base[i], p);
        if (comp == 0 && op.x0) {
          const unsigned sidx = unsigned((unsigned long long)i * op.g_inv % (2u * unsigned(n)));
          u64 x = sidx < unsigned(n) ? op.x0[(long long)j * n + sidx] : op.x0[(long long)j * n + (sidx - n)];
          if (sidx >= unsigned(n) && x) x = p - x;
          v = addmod(v, x, p);
        }
        out[i] = v;
      }
      __syncthreads();
    }
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(s_tmem, kCols);
}

// ---- unfused key switch (N = 32768) --------------------------------------------
// digits[op][prime][d][N] = digit d of op's composed words, mod the prime
__global__ void k_ks_digits(const SwitchOp* __restrict__ ops, int L, u64* __restrict__ digits,
                            const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.n) return;
  const int plane = blockIdx.y;  // (op * L + j) * D + d
  const int d = plane % R.digits, j = (plane / R.digits) % L, op = plane / (R.digits * L);
  const SwitchOp& o = ops[op];
  digits[(long long)plane * R.n + i] = gadget_digit(o.words + (long long)i * R.words, R.words, d, R, j);
}

// acc[op][c][prime][N] = sum_d digits[op][prime][d] * key[d][c][prime] (NTT domain)
__global__ void k_ks_mac(const SwitchOp* __restrict__ ops, int L, const u64* __restrict__ digits,
                         u64* __restrict__ acc, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.n) return;
  const int plane = blockIdx.y;  // (op * 2 + c) * L + j
  const int j = plane % L, c = (plane / L) % 2, op = plane / (2 * L);
  const SwitchOp& o = ops[op];
  const u64 p = R.prime[j].p;
  u64 sum = 0;
  for (int d = 0; d < R.digits; ++d) {
    const u64 v = digits[(((long long)op * L + j) * R.digits + d) * R.n + i];
    const long long ko = ((long long)(d * 2 + c) * L + j) * R.n + i;
    sum = addmod(sum, shoup(v, __ldg(o.key + ko), __ldg(o.key_q + ko), p), p);
  }
  acc[(long long)plane * R.n + i] = sum;
}

// out = acc + base + [c == 0] sigma(x0), as k_keyswitch's epilogue
__global__ void k_ks_finish(const SwitchOp* __restrict__ ops, int L, const u64* __restrict__ acc,
                            const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const int n = R.n;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int plane = blockIdx.y;  // (op * 2 + c) * L + j
  const int j = plane % L, c = (plane / L) % 2, op = plane / (2 * L);
  const SwitchOp& o = ops[op];
  const u64 p = R.prime[j].p;
  u64 v = acc[(long long)plane * n + i];
  if (o.base) v = addmod(v, o.base[((long long)c * L + j) * n + i], p);
  if (c == 0 && o.x0) {
    const unsigned sidx = unsigned((unsigned long long)i * o.g_inv % (2u * unsigned(n)));
    u64 x = sidx < unsigned(n) ? o.x0[(long long)j * n + sidx] : o.x0[(long long)j * n + (sidx - n)];
    if (sidx >= unsigned(n) && x) x = p - x;
    v = addmod(v, x, p);
  }
  o.out[((long long)c * L + j) * n + i] = v;
}

// ---- elementwise ------------------------------------------------------------------
// data[b][j][N] *= plain[j][N] (NTT domain), j = plane % L
__global__ void k_mul_plain(u64* __restrict__ data, long long planes, int L, const u64* __restrict__ plain,
                            const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= planes * R.n) return;
  const long long plane = idx / R.n;
  const int i = int(idx % R.n);
  const int j = int(plane % L);
  data[idx] = reduce128(u128(data[idx]) * plain[(long long)j * R.n + i], R.prime[j]);
}

// ---- native rings: coefficients are integers mod a prime q ----------------------
// (rns_ntt.h:394-513, bfv_server.h:123-151 of the reference).  Products are
// exact integers recovered by Garner from enough auxiliary primes, then
// reduced mod q or scaled; the multiword division is Knuth's algorithm D on
// 32-bit limbs.  Exact products fit kNarrowWords words up to 8 auxiliary
// primes (moduli up to about 220 bits); larger moduli use the wide variant.
constexpr int kNarrowWords = kMaxWords;
constexpr int kWideWords = 18;  // 18 primes x 60 bits

// u (nu limbs) = quo (nu - nv + 1 limbs) * v (nv limbs, top limb nonzero) + rem (nv limbs)
template <int LIMBS>
__device__ __forceinline__ void divmod_limbs(const uint32_t* u, int nu, const uint32_t* v, int nv, uint32_t* quo,
                                             uint32_t* rem) {
  if (nu < nv) {
    for (int i = 0; i < nv; ++i) rem[i] = i < nu ? u[i] : 0u;
    return;
  }
  if (nv == 1) {
    u64 r = 0;
    for (int i = nu - 1; i >= 0; --i) {
      const u64 cur = (r << 32) | u[i];
      quo[i] = uint32_t(cur / v[0]);
      r = cur % v[0];
    }
    rem[0] = uint32_t(r);
    return;
  }
  const int sh = __clz(v[nv - 1]);
  uint32_t vn[LIMBS], un[LIMBS + 1];
  for (int i = nv - 1; i > 0; --i) vn[i] = sh ? (v[i] << sh) | (v[i - 1] >> (32 - sh)) : v[i];
  vn[0] = v[0] << sh;
  un[nu] = sh ? u[nu - 1] >> (32 - sh) : 0u;
  for (int i = nu - 1; i > 0; --i) un[i] = sh ? (u[i] << sh) | (u[i - 1] >> (32 - sh)) : u[i];
  un[0] = u[0] << sh;
  for (int j = nu - nv; j >= 0; --j) {
    const u64 num = (u64(un[j + nv]) << 32) | un[j + nv - 1];
    u64 qhat = num / vn[nv - 1];
    u64 rhat = num % vn[nv - 1];
    while (qhat >> 32 || qhat * vn[nv - 2] > ((rhat << 32) | un[j + nv - 2])) {
      --qhat;
      rhat += vn[nv - 1];
      if (rhat >> 32) break;
    }
    long long borrow = 0;
    for (int i = 0; i < nv; ++i) {
      const u64 prod = qhat * vn[i];
      const long long t = (long long)un[i + j] - borrow - (long long)(prod & 0xffffffffu);
      un[i + j] = uint32_t(t);
      borrow = (long long)(prod >> 32) - (t >> 32);
    }
    const long long t = (long long)un[j + nv] - borrow;
    un[j + nv] = uint32_t(t);
    quo[j] = uint32_t(qhat);
    if (t < 0) {
      --quo[j];
      u64 carry = 0;
      for (int i = 0; i < nv; ++i) {
        const u64 sum = u64(un[i + j]) + vn[i] + carry;
        un[i + j] = uint32_t(sum);
        carry = sum >> 32;
      }
      un[j + nv] += uint32_t(carry);
    }
  }
  for (int i = 0; i < nv; ++i) rem[i] = sh ? (un[i] >> sh) | (un[i + 1] << (32 - sh)) : un[i];
}

// significant 32-bit limbs of W words (at least one)
__device__ __forceinline__ int words_to_limbs(const u64* w, int W, uint32_t* l) {
  int n = 0;
  for (int k = 0; k < W; ++k) {
    l[2 * k] = uint32_t(w[k]);
    l[2 * k + 1] = uint32_t(w[k] >> 32);
  }
  n = 2 * W;
  while (n > 1 && l[n - 1] == 0) --n;
  return n;
}

// Garner composition of `count` residues (stride apart) into the centred
// integer x in (-P/2, P/2), P = prod p_j (the reference's decode:
// value %= product; if value > half, value -= product).  Writes |x| as words,
// sets *negative, returns the number of words written.
//
// The mixed-radix digits d_j (x mod P = d_0 + p_0 (d_1 + p_1 (d_2 + ...)))
// decide the sign without composing P: as every p_j is odd, x mod P exceeds
// (P - 1) / 2 exactly when (d_{c-1}, ..., d_0) exceeds ((p_{c-1} - 1) / 2,
// ..., (p_0 - 1) / 2) lexicographically.  The digits of P - x are then
// (p_j - 1 - d_j) plus one, carried upward.
template <int MAXW>
__device__ __forceinline__ int garner_words(const u64* res, long long stride, int count, const RingDev& R,
                                            u64 (&w)[MAXW], bool* negative) {
  u64 digit[kMaxPrimes];
  for (int j = 0; j < count; ++j) {
    const u64 p = R.prime[j].p;
    u64 value = res[(long long)j * stride];
    for (int k = 0; k < j; ++k) {
      const u64 d = digit[k] >= p ? digit[k] - p : digit[k];
      value = shoup(value + p - d, R.garner[j][k], R.garner_q[j][k], p);
    }
    digit[j] = value;
  }
  bool neg = false;
  for (int j = count - 1; j >= 0; --j) {
    const u64 half = (R.prime[j].p - 1) >> 1;
    if (digit[j] != half) {
      neg = digit[j] > half;
      break;
    }
  }
  if (neg) {
    u64 carry = 1;
    for (int j = 0; j < count; ++j) {
      const u64 p = R.prime[j].p;
      u64 e = p - 1 - digit[j] + carry;
      carry = e == p ? 1 : 0;
      digit[j] = carry ? 0 : e;
    }
  }
  *negative = neg;
  for (int k = 0; k < MAXW; ++k) w[k] = 0;
  w[0] = digit[count - 1];
  int used = 1;
  for (int j = count - 1; j > 0; --j) {
    u64 carry = digit[j - 1];
    const u64 p = R.prime[j - 1].p;
    for (int k = 0; k < used; ++k) {
      const u128 prod = u128(w[k]) * p + carry;
      w[k] = u64(prod);
      carry = u64(prod >> 64);
    }
    if (carry && used < MAXW) w[used++] = carry;
  }
  return used;
}

// res: [polys][count][N] coefficient residues of exact integers x with
// |x| < prod p_j / 2 (negacyclic products are signed).  mode 0: out = x mod q;
// mode 1: out = floor((2 t x + q) / (2 q)) mod q, the signed BFV
// scale-and-round of rns_ntt.h:500-510 (floor division).  out: [polys][N][W]
// words.  MAXW: words of |x| (at least ceil(60 count / 64)).
//
// For x = -m < 0: x mod q = (q - m mod q) mod q, and
// floor((q - 2 t m) / (2 q)) = -floor((2 t m + q - 1) / (2 q)).
// One coefficient: residues at res[j * stride] (j < count) -> out[0 .. W).
template <int MAXW>
__device__ __forceinline__ void native_reduce_one(const u64* __restrict__ res, long long stride, int count,
                                               u64* __restrict__ o, int mode, u64 t, const RingDev& R) {
  const int W = R.words;
  constexpr int kLimbs = 2 * MAXW + 4;
  u64 x[MAXW];
  bool neg = false;
  int xw = garner_words<MAXW>(res, stride, count, R, x, &neg);
  uint32_t ql[kLimbs], xl[kLimbs], quo[kLimbs], rem[kLimbs];
  const int qn = words_to_limbs(R.q_words, W, ql);
  if (mode == 1) {
    // y = 2 t |x| + q (- 1 when x < 0), then its quotient by 2 q
    u64 y[MAXW + 2];
    const int yw = (xw + 1 > W ? xw + 1 : W) + 1;
    u64 carry = 0;
    for (int k = 0; k < yw; ++k) {
      const u128 prod = u128(k < xw ? x[k] : 0) * (2 * t) + carry;
      y[k] = u64(prod);
      carry = u64(prod >> 64);
    }
    u64 c2 = 0;
    for (int k = 0; k < yw; ++k) {
      const u128 sum = u128(y[k]) + (k < W ? R.q_words[k] : 0) + c2;
      y[k] = u64(sum);
      c2 = u64(sum >> 64);
    }
    if (neg)
      for (int k = 0; k < yw; ++k)
        if (y[k]--) break;  // y >= q >= 1: the borrow stops inside y
    uint32_t yl[2 * (MAXW + 2)], dl[kLimbs];
    const int yn = words_to_limbs(y, yw, yl);
    u64 q2[kMaxWords + 1];
    u64 c3 = 0;
    for (int k = 0; k < W; ++k) {
      q2[k] = (R.q_words[k] << 1) | c3;
      c3 = R.q_words[k] >> 63;
    }
    q2[W] = c3;
    const int dn = words_to_limbs(q2, W + 1, dl);
    for (int k = 0; k < kLimbs; ++k) quo[k] = 0;
    divmod_limbs<kLimbs>(yl, yn, dl, dn, quo, rem);
    const int qlen = yn >= dn ? yn - dn + 1 : 1;
    if (yn < dn) quo[0] = 0;
    for (int k = 0; k < qlen; ++k) xl[k] = quo[k];
    int xn = qlen;
    while (xn > 1 && xl[xn - 1] == 0) --xn;
    divmod_limbs<kLimbs>(xl, xn, ql, qn, quo, rem);
  } else {
    const int xn = words_to_limbs(x, xw, xl);
    divmod_limbs<kLimbs>(xl, xn, ql, qn, quo, rem);
  }
  u64 r[kMaxWords];
  bool nonzero = false;
  for (int k = 0; k < W; ++k) {
    const uint32_t lo = 2 * k < qn ? rem[2 * k] : 0u, hi = 2 * k + 1 < qn ? rem[2 * k + 1] : 0u;
    r[k] = u64(lo) | (u64(hi) << 32);
    nonzero |= r[k] != 0;
  }
  if (neg && nonzero) {  // r <- q - r
    u64 borrow = 0;
    for (int k = 0; k < W; ++k) {
      const u128 d = u128(R.q_words[k]) - r[k] - borrow;
      r[k] = u64(d);
      borrow = u64(d >> 64) ? 1 : 0;
    }
  }
  for (int k = 0; k < W; ++k) o[k] = r[k];
}

template <int MAXW>
__global__ void k_native_reduce(const u64* __restrict__ res, long long polys, int count, u64* __restrict__ out,
                                int mode, u64 t, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  native_reduce_one<MAXW>(res + poly * count * R.n + i, R.n, count, out + (poly * R.n + i) * R.words, mode, t, R);
}

// A rotation of word ciphertexts (k_native_permute / k_native_finish and the
// finishing form of k_native_mod_q): in = (c0, c1), perm = (sigma(c0),
// sigma(c1)), out = (sigma(c0) + KS_0, KS_1) [+ in, accumulating], ks = the
// switched words; all [2][N][W].
struct NativeOp {
  const u64* in;
  u64* perm;
  u64* out;
  const u64* ks;
};

__device__ __forceinline__ void words_add_modq(const u64* x, const u64* y, u64* o, const RingDev& R);

// The rotation's last step for coefficient i of component c = poly % 2 of
// ops[poly / 2], given the switched value v (k_native_finish for one
// coefficient).
template <int kW, bool kAccumulate>
__device__ __forceinline__ void native_finish_one(const NativeOp* __restrict__ ops, long long poly, int i,
                                                  const u64 (&v)[kW], const RingDev& R) {
  const NativeOp op = ops[poly >> 1];
  const int c = int(poly & 1);
  const long long off = ((long long)c * R.n + i) * kW;
  u64 t[kW];
  if (c == 0) {
    words_add_modq(v, op.perm + off, t, R);
  } else {
#pragma unroll
    for (int k = 0; k < kW; ++k) t[k] = v[k];
  }
  if (kAccumulate) {
    words_add_modq(t, op.in + off, op.out + off, R);
  } else {
#pragma unroll
    for (int k = 0; k < kW; ++k) op.out[off + k] = t[k];
  }
}

// Mode-0 reduction straight from the residues, after the reference's
// certified CRT (rns_ntt.h:422-469): with y_j = r_j (P / p_j)^-1 mod p_j and
// theta = sum y_j / p_j, the centred integer is x = sum y_j (P / p_j) - v P
// with v = round(theta), so x = sum y_j c_j - v pq (mod q) for c_j = P / p_j
// mod q, pq = P mod q.  theta is summed in 64-bit fixed point (each term
// within 2 units of the last place below its true value); when a rounding
// boundary falls inside that error interval the coefficient is decoded
// exactly instead (native_reduce_one).  Otherwise A = sum y_j c'_j + count q
// - v pq' (c', pq' carry an extra factor 2^128) lies in [0, 2^65 q), and two
// Montgomery word steps give A 2^-128 mod q = x mod q in [0, 2q).  kW = the
// ring's words, a compile-time constant so that A stays in registers.
// kFinish (1, 2 accumulating): poly 2k + c of res is component c of the key
// switch of ops[k], and the reduced value is finished as k_native_finish
// does (+ sigma(c0) for c = 0, + in when accumulating) into ops[k].out
// instead of being written to out.
template <int kW, int MAXW, int kFinish = 0>
__global__ void k_native_mod_q(const u64* __restrict__ res, long long polys, int count, u64* __restrict__ out,
                               const RingDev* __restrict__ ring, const NativeOp* __restrict__ ops = nullptr) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  const u64* z = res + poly * count * R.n + i;
  u64 fin[kW];  // kFinish: the reduced value, finished below
  u64* o = kFinish ? fin : out + (poly * R.n + i) * kW;
  const NativeCrt& C = R.crt[count - 1];
  u64 a[kW + 2];
#pragma unroll
  for (int k = 0; k < kW + 2; ++k) a[k] = k <= kW ? C.cq[k] : 0;
  u128 theta = 0;
  for (int j = 0; j < count; ++j) {
    const Prime& m = R.prime[j];
    const u64 y = shoup(z[(long long)j * R.n], C.inv[j], C.inv_q[j], m.p);
    theta += u128(y * m.mu_hi + mulhi(y, m.mu_lo));  // floor(y mu / 2^64), mu = floor(2^128 / p)
    u64 carry = 0;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
      const u128 sum = u128(C.c[j][k]) * y + a[k] + carry;
      a[k] = u64(sum);
      carry = u64(sum >> 64);
    }
    const u128 s1 = u128(a[kW]) + carry;
    a[kW] = u64(s1);
    a[kW + 1] += u64(s1 >> 64);
  }
  const u128 half = u128(1) << 63;
  const u64 v = u64((theta + half) >> 64);
  if (v != u64((theta + u128(2 * count) + half) >> 64)) {
    native_reduce_one<MAXW>(z, R.n, count, o, 0, 0, R);
    if (kFinish) native_finish_one<kW, kFinish == 2>(ops, poly, i, fin, R);
    return;
  }
  u64 borrow = 0;  // a -= v pq (stays >= 0: v <= count and pq < q)
#pragma unroll
  for (int k = 0; k < kW + 2; ++k) {
    const u128 prod = k < kW ? u128(C.pq[k]) * v + borrow : u128(borrow);
    const u64 lo = u64(prod);
    borrow = u64(prod >> 64) + (a[k] < lo ? 1 : 0);
    a[k] -= lo;
  }
#pragma unroll
  for (int step = 0; step < 2; ++step) {  // a <- (a + m q) / 2^64
    const u64 mq = a[0] * R.q_ninv;
    u64 carry = 0;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
      const u128 sum = u128(R.q_words[k]) * mq + a[k] + carry;
      a[k] = u64(sum);
      carry = u64(sum >> 64);
    }
    const u128 s1 = u128(a[kW]) + carry;
    a[kW] = u64(s1);
    a[kW + 1] += u64(s1 >> 64);
#pragma unroll
    for (int k = 0; k < kW + 1; ++k) a[k] = a[k + 1];
    a[kW + 1] = 0;
  }
  // a < 2q (a[kW] may hold the top bit): subtract q once if a >= q
  bool ge = a[kW] != 0;
  bool decided = ge;
#pragma unroll
  for (int k = kW - 1; k >= 0; --k)
    if (!decided && a[k] != R.q_words[k]) {
      ge = a[k] > R.q_words[k];
      decided = true;
    }
  if (!decided) ge = true;  // a == q
  if (ge) {
    u64 b = 0;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
      const u128 d = u128(a[k]) - R.q_words[k] - b;
      a[k] = u64(d);
      b = u64(d >> 64) ? 1 : 0;
    }
  }
#pragma unroll
  for (int k = 0; k < kW; ++k) o[k] = a[k];
  if (kFinish) native_finish_one<kW, kFinish == 2>(ops, poly, i, fin, R);
}

// Mode-1 (scale-and-round) reduction from the residues of the tensor primes:
// with x = sum y_j (P / p_j) - v P as in k_native_mod_q,
//   floor((2 t x + q) / (2 q)) = I + floor(E / q + 1/2),
//   I = sum y_j A_j - v A_P,  E = sum y_j B_j - v B_P,
// so the result mod q is (I mod q) + round(E / q), the first by the same
// Montgomery finish as k_native_mod_q and the second from 128-bit fixed-point
// fractions f = B / q (error below 2^-60 in all).  A rounding boundary inside
// the error interval, or q below 2^68 (then |round(E / q)| may reach q),
// sends the coefficient to the exact path.
template <int kW, int MAXW>
__global__ void k_native_scale(const u64* __restrict__ res, long long polys, int count, u64* __restrict__ out, u64 t,
                               const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  const u64* z = res + poly * count * R.n + i;
  u64* o = out + (poly * R.n + i) * kW;
  const NativeCrt& C = R.crt[count - 1];
  const NativeScale& S = R.nscale;
  u64 a[kW + 2];
#pragma unroll
  for (int k = 0; k < kW + 2; ++k) a[k] = k <= kW ? C.cq[k] : 0;
  u64 e[4] = {0, 0, 0, 0};  // sum y_j f_j - v f_P: two's complement, 128 fraction bits
  u128 theta = 0;
  for (int j = 0; j < count; ++j) {
    const Prime& m = R.prime[j];
    const u64 y = shoup(z[(long long)j * R.n], C.inv[j], C.inv_q[j], m.p);
    theta += u128(y * m.mu_hi + mulhi(y, m.mu_lo));
    u64 carry = 0;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
      const u128 sum = u128(S.a[j][k]) * y + a[k] + carry;
      a[k] = u64(sum);
      carry = u64(sum >> 64);
    }
    const u128 s1 = u128(a[kW]) + carry;
    a[kW] = u64(s1);
    a[kW + 1] += u64(s1 >> 64);
    const u128 p0 = u128(S.f[j][0]) * y + e[0];
    e[0] = u64(p0);
    const u128 p1 = u128(S.f[j][1]) * y + e[1] + u64(p0 >> 64);
    e[1] = u64(p1);
    const u128 p2 = u128(e[2]) + u64(p1 >> 64);
    e[2] = u64(p2);
    e[3] += u64(p2 >> 64);
  }
  const u128 half = u128(1) << 63;
  const u64 v = u64((theta + half) >> 64);
  if (v != u64((theta + u128(2 * count) + half) >> 64) || !R.has_nscale) {
    native_reduce_one<MAXW>(z, R.n, count, o, 1, t, R);
    return;
  }
  {
    u64 borrow = 0;  // a -= v A_P
#pragma unroll
    for (int k = 0; k < kW + 2; ++k) {
      const u128 prod = k < kW ? u128(S.ap[k]) * v + borrow : u128(borrow);
      const u64 lo = u64(prod);
      borrow = u64(prod >> 64) + (a[k] < lo ? 1 : 0);
      a[k] -= lo;
    }
  }
  {
    u64 borrow = 0;  // e -= v f_P
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const u128 prod = k < 2 ? u128(S.fp[k]) * v + borrow : u128(borrow);
      const u64 lo = u64(prod);
      borrow = u64(prod >> 64) + (e[k] < lo ? 1 : 0);
      e[k] -= lo;
    }
  }
  // r = floor(E / q + 1/2): E 2^128 / q lies in (e - 32, e + 2^66), so r is
  // certain when the top 128 bits of e - 32 + 2^127 and e + 2^66 + 2^127
  // agree (256-bit two's complement)
  u64 rlo[2], rhi[2];
  {
    u64 w[4] = {e[0], e[1], e[2], e[3]};
    u64 c = w[0] < 32 ? 1 : 0;
    w[0] -= 32;
    for (int k = 1; k < 4; ++k) {
      const u64 before = w[k];
      w[k] -= c;
      c = (c && before == 0) ? 1 : 0;
    }
    const u128 h1 = u128(w[1]) + (u64(1) << 63);
    w[1] = u64(h1);
    const u128 h2 = u128(w[2]) + u64(h1 >> 64);
    w[2] = u64(h2);
    w[3] += u64(h2 >> 64);
    rlo[0] = w[2];
    rlo[1] = w[3];
  }
  {
    u64 w[4] = {e[0], e[1], e[2], e[3]};
    const u128 h1 = u128(w[1]) + 4 + (u64(1) << 63);  // 2^66 + 2^127 in word 1
    w[1] = u64(h1);
    const u128 h2 = u128(w[2]) + u64(h1 >> 64);
    w[2] = u64(h2);
    w[3] += u64(h2 >> 64);
    rhi[0] = w[2];
    rhi[1] = w[3];
  }
  if (rlo[0] != rhi[0] || rlo[1] != rhi[1]) {
    native_reduce_one<MAXW>(z, R.n, count, o, 1, t, R);
    return;
  }
  // I mod q by two Montgomery word steps (a < 2^65 q)
#pragma unroll
  for (int step = 0; step < 2; ++step) {
    const u64 mq = a[0] * R.q_ninv;
    u64 carry = 0;
#pragma unroll
    for (int k = 0; k < kW; ++k) {
      const u128 sum = u128(R.q_words[k]) * mq + a[k] + carry;
      a[k] = u64(sum);
      carry = u64(sum >> 64);
    }
    const u128 s1 = u128(a[kW]) + carry;
    a[kW] = u64(s1);
    a[kW + 1] += u64(s1 >> 64);
#pragma unroll
    for (int k = 0; k < kW + 1; ++k) a[k] = a[k + 1];
    a[kW + 1] = 0;
  }
  // add r (signed 128-bit, |r| < 2^67 <= q): a in [0, 2q) -> a + r in (-q, 3q)
  const bool rneg = (rlo[1] >> 63) != 0;
  u64 rm[2] = {rlo[0], rlo[1]};
  if (rneg) {  // |r|
    rm[0] = ~rm[0] + 1;
    rm[1] = ~rm[1] + (rm[0] == 0 ? 1 : 0);
  }
  u64 b[kW + 1];
#pragma unroll
  for (int k = 0; k < kW + 1; ++k) b[k] = a[k];
  if (!rneg) {
    u64 c = 0;
#pragma unroll
    for (int k = 0; k < kW + 1; ++k) {
      const u128 sum = u128(b[k]) + (k < 2 ? rm[k] : 0) + c;
      b[k] = u64(sum);
      c = u64(sum >> 64);
    }
  } else {
    u64 c = 0;  // b = a + q - |r| (>= 0 since |r| < q)
#pragma unroll
    for (int k = 0; k < kW + 1; ++k) {
      const u128 sum = u128(b[k]) + (k < kW ? R.q_words[k] : 0) + c;
      b[k] = u64(sum);
      c = u64(sum >> 64);
    }
    u64 br = 0;
#pragma unroll
    for (int k = 0; k < kW + 1; ++k) {
      const u128 d = u128(b[k]) - (k < 2 ? rm[k] : 0) - br;
      b[k] = u64(d);
      br = u64(d >> 64) ? 1 : 0;
    }
  }
  // b in [0, 3q): subtract q while b >= q (at most twice)
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    bool ge = b[kW] != 0;
    bool decided = ge;
#pragma unroll
    for (int k = kW - 1; k >= 0; --k)
      if (!decided && b[k] != R.q_words[k]) {
        ge = b[k] > R.q_words[k];
        decided = true;
      }
    if (!decided) ge = true;
    if (ge) {
      u64 br = 0;
#pragma unroll
      for (int k = 0; k < kW + 1; ++k) {
        const u128 d = u128(b[k]) - (k < kW ? R.q_words[k] : 0) - br;
        b[k] = u64(d);
        br = u64(d >> 64) ? 1 : 0;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kW; ++k) o[k] = b[k];
}

// out = a +- b mod q over `units` polys of words; poly u of a / b / out
// starts at u * stride coefficients (stride 0 repeats one poly).
__global__ void k_words_addsub(const u64* __restrict__ a, long long a_stride, const u64* __restrict__ b,
                               long long b_stride, u64* __restrict__ out, long long out_stride, long long units,
                               int subtract, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= units * R.n) return;
  const long long u = idx / R.n;
  const int i = int(idx % R.n);
  const int W = R.words;
  const u64* x = a + (u * a_stride + i) * W;
  const u64* y = b + (u * b_stride + i) * W;
  u64 r[kMaxWords];
  if (subtract) {
    u64 borrow = 0;
    for (int k = 0; k < W; ++k) {
      const u128 d = u128(x[k]) - y[k] - borrow;
      r[k] = u64(d);
      borrow = u64(d >> 64) ? 1 : 0;
    }
    if (borrow) {
      u64 carry = 0;
      for (int k = 0; k < W; ++k) {
        const u128 sum = u128(r[k]) + R.q_words[k] + carry;
        r[k] = u64(sum);
        carry = u64(sum >> 64);
      }
    }
  } else {
    u64 carry = 0;
    for (int k = 0; k < W; ++k) {
      const u128 sum = u128(x[k]) + y[k] + carry;
      r[k] = u64(sum);
      carry = u64(sum >> 64);
    }
    // subtract q when the sum is at least q (a carry out means it is)
    bool ge = carry != 0;
    if (!ge) {
      ge = true;
      for (int k = W - 1; k >= 0; --k)
        if (r[k] != R.q_words[k]) { ge = r[k] > R.q_words[k]; break; }
    }
    if (ge) {
      u64 borrow = 0;
      for (int k = 0; k < W; ++k) {
        const u128 d = u128(r[k]) - R.q_words[k] - borrow;
        r[k] = u64(d);
        borrow = u64(d >> 64) ? 1 : 0;
      }
    }
  }
  u64* o = out + (u * out_stride + i) * W;
  for (int k = 0; k < W; ++k) o[k] = r[k];
}

// Per-ciphertext descriptors of the native rotate / add steps (two word polys
// each): permute writes perm = sigma_g(in); finish writes out = (ks0 + perm0,
// ks1); add writes out = in + perm.
__device__ __forceinline__ void words_add_modq(const u64* x, const u64* y, u64* o, const RingDev& R) {
  const int W = R.words;
  u64 r[kMaxWords];
  u64 carry = 0;
  for (int k = 0; k < W; ++k) {
    const u128 sum = u128(x[k]) + y[k] + carry;
    r[k] = u64(sum);
    carry = u64(sum >> 64);
  }
  bool ge = carry != 0;
  if (!ge) {
    ge = true;
    for (int k = W - 1; k >= 0; --k)
      if (r[k] != R.q_words[k]) { ge = r[k] > R.q_words[k]; break; }
  }
  if (ge) {
    u64 borrow = 0;
    for (int k = 0; k < W; ++k) {
      const u128 d = u128(r[k]) - R.q_words[k] - borrow;
      r[k] = u64(d);
      borrow = u64(d >> 64) ? 1 : 0;
    }
  }
  for (int k = 0; k < W; ++k) o[k] = r[k];
}

// perm = sigma_g(in) on words mod q: coefficient i moves to g i mod 2N,
// negated when that wraps past N (rns_ntt.h:656-664).
// grid: (blocks over 2N coefficients, ops)
__global__ void k_native_permute(const NativeOp* __restrict__ ops, unsigned g, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const NativeOp op = ops[blockIdx.y];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * R.n) return;
  const int c = idx / R.n, i = idx % R.n, W = R.words;
  const unsigned at = unsigned((unsigned long long)i * g % (2u * unsigned(R.n)));
  const u64* x = op.in + ((long long)c * R.n + i) * W;
  u64* o = op.perm + ((long long)c * R.n + (at % unsigned(R.n))) * W;
  bool nonzero = false;
  for (int k = 0; k < W; ++k) nonzero |= x[k] != 0;
  if (at >= unsigned(R.n) && nonzero) {
    u64 borrow = 0;
    for (int k = 0; k < W; ++k) {
      const u128 d = u128(R.q_words[k]) - x[k] - borrow;
      o[k] = u64(d);
      borrow = u64(d >> 64) ? 1 : 0;
    }
  } else {
    for (int k = 0; k < W; ++k) o[k] = x[k];
  }
}

// out = (ks_0 + perm_0, ks_1); with kAccumulate, out = in + that (the
// rotation added into its input: out may be in, each thread reading its
// words before writing them)
template <bool kAccumulate>
__global__ void k_native_finish(const NativeOp* __restrict__ ops, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const NativeOp op = ops[blockIdx.y];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * R.n) return;
  const int W = R.words;
  const long long off = (long long)idx * W;
  if (!kAccumulate) {
    if (idx < R.n) {
      words_add_modq(op.ks + off, op.perm + off, op.out + off, R);
    } else {
      for (int k = 0; k < W; ++k) op.out[off + k] = op.ks[off + k];
    }
    return;
  }
  u64 t[kMaxWords];
  if (idx < R.n) {
    words_add_modq(op.ks + off, op.perm + off, t, R);
    words_add_modq(t, op.in + off, op.out + off, R);
  } else {
    words_add_modq(op.ks + off, op.in + off, op.out + off, R);
  }
}

__global__ void k_native_add(const NativeOp* __restrict__ ops, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const NativeOp op = ops[blockIdx.y];
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 2 * R.n) return;
  const long long off = (long long)idx * R.words;
  words_add_modq(op.in + off, op.perm + off, op.out + off, R);
}

// ---- client-side encryption (bfv/scheme.py:371-394, 426-444) -------------------
// Batch encoding: plane c position perm[j] receives slot j of plaintext c, so
// that the inverse negacyclic NTT mod t of the plane is the encoded
// polynomial (slot j is the value at the evaluation point of order[j]).
__global__ void k_scatter_slots(const uint32_t* __restrict__ slots, const int32_t* __restrict__ perm,
                                long long count, int n, uint32_t t, u64* __restrict__ planes, int* status) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= count * n) return;
  const long long c = idx / n;
  const int j = int(idx % n);
  const uint32_t v = slots[idx];
  if (v >= t) {
    atomicOr(status, 1);
    return;
  }
  planes[c * n + perm[j]] = v;
}

// ---- client noise from a ChaCha20 keystream (RFC 8439 block function) ----------
// State: the constant "expand 32-byte k", the key (8 little-endian words), a
// 32-bit block counter and the nonce (3 words); 20 rounds (10 column +
// diagonal double rounds) of the quarter round, then the input added back.
__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
__device__ __forceinline__ void chacha_quarter(uint32_t& a, uint32_t& b, uint32_t& c, uint32_t& d) {
  a += b; d ^= a; d = rotl32(d, 16);
  c += d; b ^= c; b = rotl32(b, 12);
  a += b; d ^= a; d = rotl32(d, 8);
  c += d; b ^= c; b = rotl32(b, 7);
}
__device__ __forceinline__ void chacha20_block(const uint32_t (&key)[8], uint32_t counter, const uint32_t (&nonce)[3],
                                               uint32_t (&out)[16]) {
  uint32_t x[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                    key[4],      key[5],      key[6],      key[7],      counter, nonce[0], nonce[1], nonce[2]};
  uint32_t s[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) s[k] = x[k];
#pragma unroll 1
  for (int r = 0; r < 10; ++r) {
    chacha_quarter(x[0], x[4], x[8], x[12]);
    chacha_quarter(x[1], x[5], x[9], x[13]);
    chacha_quarter(x[2], x[6], x[10], x[14]);
    chacha_quarter(x[3], x[7], x[11], x[15]);
    chacha_quarter(x[0], x[5], x[10], x[15]);
    chacha_quarter(x[1], x[6], x[11], x[12]);
    chacha_quarter(x[2], x[7], x[8], x[13]);
    chacha_quarter(x[3], x[4], x[9], x[14]);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) out[k] = x[k] + s[k];
}

struct NoiseKey {
  uint32_t key[8];
  uint32_t nonce[3];
  uint32_t eta;              // e = popcount of an eta-bit word minus another's
  uint64_t first_ct;         // ciphertext index of the batch's first row
  uint32_t blocks_per_ct;    // e blocks, then u blocks
  uint32_t e_blocks;
};

// One thread per 64-byte keystream block of ciphertext (first_ct + row):
// counter = (first_ct + row) * blocks_per_ct + b.  Blocks [0, e_blocks)
// give e: words of 4 bytes (eta <= 31) or 8 bytes, in pairs, pair v giving
// e[row][v / N][v % N] = popcount(w0 & mask) - popcount(w1 & mask).  The
// remaining N / 8 blocks give u: 8 bytes per coefficient, u = (first byte
// below 255) % 3 - 1; eight bytes of 255 (probability 2^-64) set *status.
__global__ void k_keyed_noise(NoiseKey nk, long long rows, int n, int8_t* __restrict__ u, int8_t* __restrict__ e,
                              int* __restrict__ status) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * nk.blocks_per_ct) return;
  const long long row = idx / nk.blocks_per_ct;
  const uint32_t b = uint32_t(idx % nk.blocks_per_ct);
  uint32_t w[16];
  chacha20_block(nk.key, uint32_t((nk.first_ct + row) * nk.blocks_per_ct + b), nk.nonce, w);
  if (b < nk.e_blocks) {
    int8_t* er = e + row * 2 * n;
    if (nk.eta <= 31) {
      const uint32_t mask = (1u << nk.eta) - 1u;
#pragma unroll
      for (int v = 0; v < 8; ++v)
        er[b * 8 + v] = int8_t(__popc(w[2 * v] & mask) - __popc(w[2 * v + 1] & mask));
    } else {
      const uint64_t mask = (uint64_t(1) << nk.eta) - 1u;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const uint64_t w0 = uint64_t(w[4 * v]) | (uint64_t(w[4 * v + 1]) << 32);
        const uint64_t w1 = uint64_t(w[4 * v + 2]) | (uint64_t(w[4 * v + 3]) << 32);
        er[b * 4 + v] = int8_t(__popcll(w0 & mask) - __popcll(w1 & mask));
      }
    }
    return;
  }
  int8_t* ur = u + row * n;
  const uint32_t ub = b - nk.e_blocks;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    int chosen = -1;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const uint32_t byte = (w[2 * v + (k >> 2)] >> (8 * (k & 3))) & 0xffu;
      if (chosen < 0 && byte < 255u) chosen = int(byte);
    }
    if (chosen < 0) {
      atomicOr(status, 2);
      chosen = 1;
    }
    ur[ub * 8 + v] = int8_t(chosen % 3 - 1);
  }
}

// out[poly][j][i] = v mod p_j for signed small v (u, e): residues mod the
// first L primes.
__global__ void k_small_residues(const int8_t* __restrict__ v, long long polys, int L, u64* __restrict__ out,
                                 const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= polys * R.n) return;
  const long long poly = idx / R.n;
  const int i = int(idx % R.n);
  const int x = v[idx];
  for (int j = 0; j < L; ++j) {
    const u64 p = R.prime[j].p;
    out[(poly * L + j) * R.n + i] = x >= 0 ? u64(x) : p - u64(-x);
  }
}

// prod[c][comp][j][i] = u_ntt[c][j][i] * pk_ntt[comp][j][i] mod p_j
__global__ void k_mul_public(const u64* __restrict__ u_ntt, const u64* __restrict__ pk_ntt, long long count, int L,
                             u64* __restrict__ prod, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = 2LL * L * R.n;
  if (idx >= count * per) return;
  const long long c = idx / per;
  const long long rest = idx % per;
  const int comp = int(rest / ((long long)L * R.n));
  const int j = int((rest / R.n) % L);
  const int i = int(rest % R.n);
  prod[idx] = mulmod(u_ntt[(c * L + j) * R.n + i], pk_ntt[((long long)comp * L + j) * R.n + i], R.prime[j]);
}

// ct[c][0] += e[c][0] + delta * m[c], ct[c][1] += e[c][1]  (mod p_j); m < t
__global__ void k_add_noise_message(u64* __restrict__ ct, const int8_t* __restrict__ e, const u64* __restrict__ m,
                                    const u64* __restrict__ delta, long long count, int L,
                                    const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = 2LL * L * R.n;
  if (idx >= count * per) return;
  const long long c = idx / per;
  const long long rest = idx % per;
  const int comp = int(rest / ((long long)L * R.n));
  const int j = int((rest / R.n) % L);
  const int i = int(rest % R.n);
  const u64 p = R.prime[j].p;
  const int x = e[(c * 2 + comp) * R.n + i];
  u64 v = addmod(ct[idx], x >= 0 ? u64(x) : p - u64(-x), p);
  if (comp == 0) v = addmod(v, mulmod(delta[j], m[c * R.n + i], R.prime[j]), p);
  ct[idx] = v;
}

// q[b][i] = floor(x[b][i] * 2^64 / p_j), j = b % L: Shoup quotients of fixed
// multipliers (compiled keys).
__global__ void k_shoup_quotients(const u64* __restrict__ x, u64* __restrict__ q, long long planes, int L,
                                  const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= planes * R.n) return;
  const int j = int((idx / R.n) % L);
  q[idx] = fraction64(x[idx], R.prime[j]);
}

// out = a + b elementwise over planes of L primes
__global__ void k_add(const u64* __restrict__ a, const u64* __restrict__ b, u64* __restrict__ out, long long planes,
                      int L, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= planes * R.n) return;
  const int j = int((idx / R.n) % L);
  out[idx] = addmod(a[idx], b[idx], R.prime[j].p);
}

// Compaction: c' = floor((2*target*c + Q) / (2Q)) mod target on composed words
// (bfv_server.h:142-151), by binary long division.
__global__ void k_compact(u64* __restrict__ words, long long coeffs, const u64* __restrict__ target_words,
                          int target_nwords, const RingDev* __restrict__ ring) {
  const RingDev& R = *ring;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= coeffs) return;
  const int W = R.words;
  constexpr int NW = 2 * kMaxWords + 2;
  u64* c = words + idx * W;
  // num = 2 * target * c + Q
  u64 num[NW], den[NW], rem[NW], quo[NW];
  for (int k = 0; k < NW; ++k) num[k] = den[k] = rem[k] = quo[k] = 0;
  for (int a = 0; a < target_nwords; ++a) {
    u128 carry = 0;
    for (int b = 0; b < W; ++b) {
      carry += u128(target_words[a]) * c[b] + num[a + b];
      num[a + b] = u64(carry);
      carry >>= 64;
    }
    for (int k = a + W; carry && k < NW; ++k) {
      carry += num[k];
      num[k] = u64(carry);
      carry >>= 64;
    }
  }
  // *2
  u64 top = 0;
  for (int k = 0; k < NW; ++k) {
    const u64 nt = num[k] >> 63;
    num[k] = (num[k] << 1) | top;
    top = nt;
  }
  u128 carry = 0;
  for (int k = 0; k < NW; ++k) {
    carry += u128(num[k]) + (k < W ? R.q_words[k] : 0);
    num[k] = u64(carry);
    carry >>= 64;
  }
  // den = 2Q
  top = 0;
  for (int k = 0; k < NW; ++k) {
    const u64 qk = k < W ? R.q_words[k] : 0;
    den[k] = (qk << 1) | top;
    top = qk >> 63;
  }
  int nbits = 0;
  for (int k = NW - 1; k >= 0; --k)
    if (num[k]) { nbits = k * 64 + 64 - __clzll(num[k]); break; }
  for (int bit = nbits - 1; bit >= 0; --bit) {
    u64 t2 = 0;
    for (int k = 0; k < NW; ++k) {
      const u64 nt = rem[k] >> 63;
      rem[k] = (rem[k] << 1) | t2;
      t2 = nt;
    }
    rem[0] |= (num[bit / 64] >> (bit % 64)) & 1;
    bool ge = true;
    for (int k = NW - 1; k >= 0; --k)
      if (rem[k] != den[k]) { ge = rem[k] > den[k]; break; }
    if (ge) {
      u64 borrow = 0;
      for (int k = 0; k < NW; ++k) {
        const u128 x = u128(rem[k]) - den[k] - borrow;
        rem[k] = u64(x);
        borrow = u64(x >> 64) ? 1 : 0;
      }
      quo[bit / 64] |= u64(1) << (bit % 64);
    }
  }
  // quotient <= target; reduce mod target (one subtraction)
  bool ge = true;
  for (int k = NW - 1; k >= 0; --k) {
    const u64 tk = k < target_nwords ? target_words[k] : 0;
    if (quo[k] != tk) { ge = quo[k] > tk; break; }
  }
  if (ge) {
    u64 borrow = 0;
    for (int k = 0; k < NW; ++k) {
      const u64 tk = k < target_nwords ? target_words[k] : 0;
      const u128 x = u128(quo[k]) - tk - borrow;
      quo[k] = u64(x);
      borrow = u64(x >> 64) ? 1 : 0;
    }
  }
  for (int k = 0; k < W; ++k) c[k] = quo[k];
}

// Pack composed words into `bits`-bit little-endian coefficients: thread per
// output 64-bit word gathers the (at most bits/64 + 2) overlapping coefficients.
__global__ void k_pack(const u64* __restrict__ words, int W, int n, int bits, int polys, u64* __restrict__ out,
                       long long out_words_per_poly) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)polys * out_words_per_poly) return;
  const long long poly = idx / out_words_per_poly;
  const long long ow = idx % out_words_per_poly;
  const long long lo_bit = ow * 64, hi_bit = lo_bit + 64;
  long long first = lo_bit / bits, last = (hi_bit - 1) / bits;
  if (last >= n) last = n - 1;
  u64 acc = 0;
  for (long long i = first; i <= last; ++i) {
    const u64* c = words + (poly * n + i) * W;
    const long long cb = i * bits;  // coefficient start bit
    // bits of coefficient overlapping [lo_bit, hi_bit)
    for (int k = 0; k < W; ++k) {
      const long long wb = cb + 64LL * k;  // global bit of c[k]'s bit 0
      if (64LL * k >= bits) break;
      u64 v = c[k];
      if (64LL * (k + 1) > bits) v &= (bits - 64 * k) >= 64 ? ~u64(0) : ((u64(1) << (bits - 64 * k)) - 1);
      const long long rel = wb - lo_bit;
      if (rel >= 64 || rel <= -64) continue;
      acc |= rel >= 0 ? (v << rel) : (v >> (-rel));
    }
  }
  out[idx] = acc;
}

}  // namespace bfv
}  // namespace cuhe
