// Paillier / Paillier-Lookup kernels for sm_100a.
//
// One instance (ciphertext) is owned by a TPI-lane group (see bigint_group.cuh);
// a 128-thread block holds 128/TPI instances.  All arithmetic mod n^2 is in the
// Montgomery domain with R = 2^(32K); arithmetic mod n uses the same K-limb
// routines with n zero-padded to K limbs.
#pragma once
#include <cstdint>
#include "bigint52.cuh"
#include "bigint_group.cuh"

namespace cuhe {

// Rows of the per-key constant block (each row K words).
enum ConstRow : int {
  C_N2 = 0,     // n^2
  C_R2 = 1,     // R^2 mod n^2
  C_ONE = 2,    // 1
  C_RM = 3,     // R mod n^2  (Montgomery form of 1)
  C_N = 4,      // n, zero-padded
  C_R2N = 5,    // R^2 mod n
  C_NNEG = 6,   // 2^(32K) - n
  C_NR = 7,     // n * R mod n^2
  C_MULTR = 8,  // (secret multiplier) * R mod n
  C_ROWS = 9
};

// Rows of the CRT constant block (each row K words).  Half rows hold the p^2
// value in words [0, K/2) and the q^2 value in words [K/2, K); R_h = 2^(16K).
enum CrtRow : int {
  CR_M = 0,    // p^2 | q^2
  CR_RM = 1,   // R_h mod p^2 | R_h mod q^2
  CR_R3 = 2,   // R_h^3 mod p^2 | R_h^3 mod q^2
  CR_H = 3,    // (q^2)^-1 R_h mod p^2 | 0
  CR_CQ = 4,   // q^2 R mod n^2 (full row)
  CR_R52 = 5,  // R52 R_h^2 mod p^2 | R52 R_h^2 mod q^2, R52 = 2^(52 K52) (FP64-pipe kernel)
  CR_ROWS = 6
};

struct CrtScalars {
  uint32_t ninv[2];   // -(p^2)^-1, -(q^2)^-1 mod 2^32
  unsigned long long ninv52[2];  // -(p^2)^-1, -(q^2)^-1 mod 2^52
};

struct KeyScalars {
  uint32_t ninv2;  // -(n^2)^-1 mod 2^32
  uint32_t ninv1;  // -n^-1 mod 2^32
  uint32_t ndiv;   // n^-1 mod 2^32 (exact division)
  uint32_t mult_is_zero;
};

// status bits written by kernels
enum StatusBits : int { ST_RANGE = 1 };

enum ExpMode : int { EXP_POW = 0, EXP_ENCRYPT = 1, EXP_DECRYPT = 2, EXP_DECODE = 3 };

constexpr int kBlockThreads = 128;

template <int K>
__host__ __device__ constexpr int inst_stride_words(int buffers) {
  return buffers * K + 4;  // +4 words shifts consecutive instances by 4 banks
}

// -- helpers shared by kernels ---------------------------------------------

template <int K, int TPI>
__device__ __forceinline__ void copy_rows_to_smem(uint32_t* dst, const uint32_t* consts, const int* rows,
                                                  int nrows) {
  for (int r = 0; r < nrows; ++r)
    for (int i = threadIdx.x; i < K; i += blockDim.x) dst[r * K + i] = consts[rows[r] * K + i];
}

// x + small (small < 2^32) over the group, with lookahead carry resolution.
template <int K, int TPI>
__device__ __forceinline__ void add_small(const Group<K, TPI>& g, uint32_t (&x)[K / TPI], uint32_t small) {
  constexpr int L = K / TPI;
  uint32_t add0 = (g.gl == 0) ? small : 0u;
  x[0] = add_cc(x[0], add0);
#pragma unroll
  for (int j = 1; j < L; ++j) x[j] = addc_cc(x[j], 0u);
  const uint32_t carry = addc(0u, 0u);
  uint32_t ones = x[0];
#pragma unroll
  for (int j = 1; j < L; ++j) ones &= x[j];
  const bool cin = g.lookahead(carry != 0u, ones == 0xffffffffu, nullptr);
  if (cin) {
    x[0] = add_cc(x[0], 1u);
#pragma unroll
    for (int j = 1; j < L; ++j) x[j] = addc_cc(x[j], 0u);
    (void)addc(0u, 0u);
  }
}

// x - y for x >= y over the group.
template <int K, int TPI>
__device__ __forceinline__ void sub_group(const Group<K, TPI>& g, uint32_t (&x)[K / TPI],
                                          const uint32_t (&y)[K / TPI]) {
  constexpr int L = K / TPI;
  x[0] = sub_cc(x[0], y[0]);
#pragma unroll
  for (int j = 1; j < L; ++j) x[j] = subc_cc(x[j], y[j]);
  const uint32_t borrow = subc(0u, 0u) & 1u;
  uint32_t zero = x[0];
#pragma unroll
  for (int j = 1; j < L; ++j) zero |= x[j];
  const bool bin = g.lookahead(borrow != 0u, zero == 0u, nullptr);
  if (bin) {
    x[0] = sub_cc(x[0], 1u);
#pragma unroll
    for (int j = 1; j < L; ++j) x[j] = subc_cc(x[j], 0u);
    (void)subc(0u, 0u);
  }
}

// x += y over the group; returns the carry out of the top lane.
template <int K, int TPI>
__device__ __forceinline__ bool add_group(const Group<K, TPI>& g, uint32_t (&x)[K / TPI],
                                          const uint32_t (&y)[K / TPI]) {
  constexpr int L = K / TPI;
  x[0] = add_cc(x[0], y[0]);
#pragma unroll
  for (int j = 1; j < L; ++j) x[j] = addc_cc(x[j], y[j]);
  const uint32_t carry = addc(0u, 0u);
  uint32_t ones = x[0];
#pragma unroll
  for (int j = 1; j < L; ++j) ones &= x[j];
  bool out = false;
  const bool cin = g.lookahead(carry != 0u, ones == 0xffffffffu, &out);
  if (cin) {
    x[0] = add_cc(x[0], 1u);
#pragma unroll
    for (int j = 1; j < L; ++j) x[j] = addc_cc(x[j], 0u);
    (void)addc(0u, 0u);
  }
  return out;
}

// x = (x - y) mod m for x, y < m over the group.
template <int K, int TPI>
__device__ __forceinline__ void sub_mod(const Group<K, TPI>& g, uint32_t (&x)[K / TPI],
                                        const uint32_t (&y)[K / TPI], const uint32_t (&m)[K / TPI]) {
  constexpr int L = K / TPI;
  x[0] = sub_cc(x[0], y[0]);
#pragma unroll
  for (int j = 1; j < L; ++j) x[j] = subc_cc(x[j], y[j]);
  const uint32_t borrow = subc(0u, 0u) & 1u;
  uint32_t zero = x[0];
#pragma unroll
  for (int j = 1; j < L; ++j) zero |= x[j];
  bool under = false;  // x < y: the group-wide borrow (same value in every lane)
  const bool bin = g.lookahead(borrow != 0u, zero == 0u, &under);
  if (bin) {
    x[0] = sub_cc(x[0], 1u);
#pragma unroll
    for (int j = 1; j < L; ++j) x[j] = subc_cc(x[j], 0u);
    (void)subc(0u, 0u);
  }
  if (under) (void)add_group<K, TPI>(g, x, m);
}

// Epilogue shared by the decrypt / decode kernels.  x = base^e mod n^2
// (canonical); writes floor((x - 1)/n) * mult mod n (EXP_DECRYPT) or the
// popcount of its even bits over pop_words words (EXP_DECODE).  Block rows:
// s_one = 1, s_r2n = R^2 mod n, s_multr = mult * R mod n.
template <int K, int TPI>
__device__ __forceinline__ void decrypt_epilogue(const Group<K, TPI>& g, uint32_t (&x)[K / TPI],
                                                 uint32_t* __restrict__ out, long long inst,
                                                 const uint32_t* __restrict__ consts, const KeyScalars& ks,
                                                 const uint32_t* s_one, const uint32_t* s_r2n,
                                                 const uint32_t* s_multr, int mode, int pop_words) {
  constexpr int L = K / TPI;
  uint32_t nn[L];
  g.load_ro(nn, consts + C_N * K);
  uint32_t res[L];
  if (g.is_zero(x)) {
    // floor(-1/n) = -1  ->  (-mult) mod n
    uint32_t multr[L], mult[L];
    g.load(multr, s_multr);
    g.mont_mul(mult, multr, s_one, nn, ks.ninv1);
#pragma unroll
    for (int j = 0; j < L; ++j) res[j] = nn[j];
    if (ks.mult_is_zero) {
#pragma unroll
      for (int j = 0; j < L; ++j) res[j] = 0u;
    } else {
      sub_group<K, TPI>(g, res, mult);
    }
  } else {
    uint32_t one[L];
#pragma unroll
    for (int j = 0; j < L; ++j) one[j] = (g.gl == 0 && j == 0) ? 1u : 0u;
    sub_group<K, TPI>(g, x, one);                 // y
    uint32_t t1[L];
    g.mont_mul(t1, x, s_one, nn, ks.ninv1);       // y R^-1 mod n
    uint32_t rem[L];
    g.mont_mul(rem, t1, s_r2n, nn, ks.ninv1);     // y mod n
    sub_group<K, TPI>(g, x, rem);                 // y - (y mod n) = q*n
    uint32_t q[L], mneg[L];
    g.load_ro(mneg, consts + C_NNEG * K);
    g.exact_div(q, x, mneg, ks.ndiv, K / 2);      // q = floor(y/n) < n
    g.mont_mul(res, q, s_multr, nn, ks.ninv1);    // q * mult mod n
  }
  if (mode == EXP_DECRYPT) {
    g.store(out + inst * K, res);
    return;
  }
  // EXP_DECODE
  int pc = 0;
#pragma unroll
  for (int j = 0; j < L; ++j)
    if (g.gl * L + j < pop_words) pc += __popc(res[j] & 0x55555555u);
#pragma unroll
  for (int off = TPI / 2; off > 0; off >>= 1) pc += __shfl_xor_sync(g.mask, pc, off, TPI);
  if (g.gl == 0) out[inst] = uint32_t(pc);
}

// ---------------------------------------------------------------------------
// Fixed-exponent modular exponentiation with per-instance bases.
//   EXP_POW     out = base^e mod n^2
//   EXP_ENCRYPT out = base^e * (1 + aux*n) mod n^2          (Paillier encrypt, g = n+1)
//   EXP_DECRYPT out = floor((base^e mod n^2 - 1)/n) * mult mod n
//   EXP_DECODE  out32 = popcount of the even bits of the EXP_DECRYPT value
// The exponent is a host-built sliding-window schedule (host_bigint.h).
// ---------------------------------------------------------------------------
// One CTA's share of a modexp launch: instances [block*IPB, block*IPB + IPB).
// Every thread of the CTA calls it (it synchronises the CTA once, after
// staging the key rows in shared memory).
template <int K, int TPI, int W>
__device__ __forceinline__ void modexp_unit(const uint32_t* __restrict__ base, const uint32_t* __restrict__ aux,
                                            int aux_words, uint32_t* __restrict__ out, long long count,
                                            const uint32_t* __restrict__ consts, const KeyScalars& ks,
                                            const int32_t* __restrict__ ops, int nops, int mode, int pop_words,
                                            int* status, long long block) {
  constexpr int L = K / TPI;
  constexpr int T = 1 << (W - 1);
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int STRIDE = inst_stride_words<K>(T + 1);
  extern __shared__ __align__(16) uint32_t smem[];
  // block rows: ONE, R2, NR, R2N, MULTR
  uint32_t* s_one = smem;
  uint32_t* s_r2 = smem + K;
  uint32_t* s_nr = smem + 2 * K;
  uint32_t* s_r2n = smem + 3 * K;
  uint32_t* s_multr = smem + 4 * K;
  {
    const int rows[5] = {C_ONE, C_R2, C_NR, C_R2N, C_MULTR};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 5);
  }
  __syncthreads();

  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = block * IPB + slot;
  if (inst >= count) return;  // whole groups leave together
  uint32_t* s_inst = smem + 5 * K + slot * STRIDE;
  uint32_t* s_x = s_inst;               // current value (b operand of squarings)
  uint32_t* s_tab = s_inst + K;         // T odd powers

  uint32_t n2[L];
  g.load_ro(n2, consts + C_N2 * K);
  uint32_t x[L], acc[L];
  g.load(x, base + inst * K);
  if (!g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  // odd-power table in Montgomery form
  g.mont_mul(acc, x, s_r2, n2, ks.ninv2);  // x*R
  g.publish(s_tab, acc);
  if (T > 1) {
    uint32_t sq[L];
    g.mont_mul(sq, acc, s_tab, n2, ks.ninv2);  // x^2 R
    g.publish(s_x, sq);
#pragma unroll 1
    for (int t = 1; t < T; ++t) {
      g.mont_mul(acc, acc, s_x, n2, ks.ninv2);
      g.publish(s_tab + t * K, acc);
    }
  }
  // exponent schedule
  if (nops == 0) {
    g.load(acc, s_tab);  // unused value, replaced below by R mod n^2
    uint32_t rm[L];
    g.load_ro(rm, consts + C_RM * K);
#pragma unroll
    for (int j = 0; j < L; ++j) acc[j] = rm[j];
  } else {
    const int first = __ldg(ops) & 0xffff;
    g.load(acc, s_tab + (first - 1) * K);
  }
  g.publish(s_x, acc);
#pragma unroll 1
  for (int o = 1; o < nops; ++o) {
    const int op = __ldg(ops + o);
    const int sq = op >> 16;
    const int idx = op & 0xffff;
#pragma unroll 1
    for (int s = 0; s < sq; ++s) {
      g.mont_mul(acc, acc, s_x, n2, ks.ninv2);
      g.publish(s_x, acc);
    }
    if (idx) {
      g.mont_mul(acc, acc, s_tab + (idx - 1) * K, n2, ks.ninv2);
      g.publish(s_x, acc);
    }
  }

  if (mode == EXP_POW) {
    g.mont_mul(x, acc, s_one, n2, ks.ninv2);
    g.store(out + inst * K, x);
    return;
  }
  if (mode == EXP_ENCRYPT) {
    uint32_t m[L];
    g.load(m, aux + inst * aux_words);  // aux_words == K (zero-padded m < n)
    uint32_t nn[L];
    g.load_ro(nn, consts + C_N * K);
    if (!g.less_than(m, nn)) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
    g.mont_mul(x, m, s_nr, n2, ks.ninv2);  // m*n (exact, < n^2)
    add_small<K, TPI>(g, x, 1u);           // 1 + m*n = g^m mod n^2
    g.publish(s_x, x);
    g.mont_mul(x, acc, s_x, n2, ks.ninv2);  // r^n * g^m
    g.store(out + inst * K, x);
    return;
  }
  // decrypt / decode
  g.mont_mul(x, acc, s_one, n2, ks.ninv2);
  decrypt_epilogue<K, TPI>(g, x, out, inst, consts, ks, s_one, s_r2n, s_multr, mode, pop_words);
}

template <int K, int TPI, int W>
__global__ void __launch_bounds__(kBlockThreads)
k_modexp(const uint32_t* __restrict__ base, const uint32_t* __restrict__ aux, int aux_words,
         uint32_t* __restrict__ out, long long count, const uint32_t* __restrict__ consts, KeyScalars ks,
         const int32_t* __restrict__ ops, int nops, int mode, int pop_words, int* status) {
  modexp_unit<K, TPI, W>(base, aux, aux_words, out, count, consts, ks, ops, nops, mode, pop_words, status,
                         (long long)blockIdx.x);
}

// One fixed-exponent exponentiation batch of a mixed launch: `count` bases of
// one key (its constant block and Montgomery scalars) raised to one exponent
// (its window schedule).  first_unit = CTA units of the tasks before it.
struct ModexpTask {
  const uint32_t* base;
  uint32_t* out;
  long long count;
  const uint32_t* consts;
  const int32_t* ops;
  long long first_unit;
  KeyScalars ks;
  int nops;
  int mode;
  const double* n52;            // k_modexp52_tasks: the key's 52-bit constants
  unsigned long long ninv52;
};

// Persistent mixed launch: CTAs take units (IPB instances of one task) from
// a global counter until every unit of every task is done, so batches of
// uneven sizes and different keys share one launch without tail waves per
// batch.  tasks[] is ordered by first_unit.
template <int K, int TPI, int W>
__global__ void __launch_bounds__(kBlockThreads)
k_modexp_tasks(const ModexpTask* __restrict__ tasks, int ntasks, long long total_units,
               unsigned long long* __restrict__ counter, int* status) {
  __shared__ long long s_unit;
  while (true) {
    if (threadIdx.x == 0) s_unit = (long long)atomicAdd(counter, 1ull);
    __syncthreads();
    const long long unit = s_unit;
    if (unit >= total_units) break;
    int lo = 0, hi = ntasks - 1;  // last task with first_unit <= unit
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].first_unit <= unit) lo = mid; else hi = mid - 1;
    }
    const ModexpTask& t = tasks[lo];
    modexp_unit<K, TPI, W>(t.base, nullptr, K, t.out, t.count, t.consts, t.ks, t.ops, t.nops, t.mode, 0, status,
                           unit - t.first_unit);
    __syncthreads();  // shared rows and tables are restaged by the next unit
  }
}

// ---------------------------------------------------------------------------
// Decrypt / decode exponentiation by the Chinese remainder theorem, for keys
// whose factorisation n = p q is known (EXP_DECRYPT / EXP_DECODE only).
//
// Each ciphertext is owned by 2*TPI consecutive lanes.  Its lower TPI lanes
// (side 0) compute x_p = c^e mod p^2 and its upper TPI lanes (side 1)
// x_q = c^e mod q^2, each a KH-word Montgomery exponentiation with
// R_h = 2^(32 KH) on its own half of the lanes, so one modular product costs
// a quarter of a K-word one.  Garner's recombination
//   h = (x_p - x_q) (q^2)^-1 mod p^2,   x = x_q + q^2 h   (< n^2, exact)
// runs on the two halves together as a K-word group, and the same epilogue
// as k_modexp follows, so the result equals the direct c^e mod n^2 path for
// every c < n^2.
// ---------------------------------------------------------------------------
template <int KH, int TPI, int W>
__global__ void __launch_bounds__(kBlockThreads)
k_modexp_crt(const uint32_t* __restrict__ base, uint32_t* __restrict__ out, long long count,
             const uint32_t* __restrict__ consts, KeyScalars ks, const uint32_t* __restrict__ crt, CrtScalars cs,
             const int32_t* __restrict__ ops, int nops, int mode, int pop_words, int* status) {
  constexpr int K = 2 * KH;
  constexpr int L = KH / TPI;
  constexpr int T = 1 << (W - 1);
  constexpr int IPB = kBlockThreads / (2 * TPI);
  constexpr int SIDE = (T + 1) * KH + 4;  // per side: x, then T odd powers; +4 words moves the banks
  extern __shared__ __align__(16) uint32_t smem[];
  // block rows: ONE, R2N, MULTR (K words each), RM, R3, H (two halves), CQ (K words)
  uint32_t* s_one = smem;
  uint32_t* s_r2n = smem + K;
  uint32_t* s_multr = smem + 2 * K;
  uint32_t* s_rm = smem + 3 * K;
  uint32_t* s_r3 = smem + 4 * K;
  uint32_t* s_h = smem + 5 * K;
  uint32_t* s_cq = smem + 6 * K;
  {
    const int rows[3] = {C_ONE, C_R2N, C_MULTR};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 3);
    const int crows[4] = {CR_RM, CR_R3, CR_H, CR_CQ};
    copy_rows_to_smem<K, TPI>(smem + 3 * K, crt, crows, 4);
  }
  __syncthreads();

  Group<K, 2 * TPI> g;   // the whole ciphertext
  Group<KH, TPI> h;      // this side's half
  const int side = (threadIdx.x / TPI) & 1;
  const int slot = threadIdx.x / (2 * TPI);
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;  // both halves leave together
  uint32_t* s_item = smem + 7 * K + slot * 2 * SIDE;
  uint32_t* s_x = s_item + side * SIDE;
  uint32_t* s_tab = s_x + KH;

  {
    uint32_t c[L], n2[L];
    g.load_ro(n2, consts + C_N2 * K);
    g.load(c, base + inst * K);
    if (!g.less_than(c, n2)) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
  }
  const uint32_t ninv = cs.ninv[side];
  uint32_t m[L], lo[L], hi[L], acc[L];
  h.load_ro(m, crt + CR_M * K + side * KH);
  h.load(lo, base + inst * K);
  h.load(hi, base + inst * K + KH);
  // c = lo + hi R_h:  (lo + hi * (R_h mod M)) R_h^-1 = c R_h^-1, then * R_h^3 R_h^-1
  h.mont_mul_acc(acc, lo, hi, s_rm + side * KH, m, ninv);
  h.mont_mul(acc, acc, s_r3 + side * KH, m, ninv);  // c R_h mod M (Montgomery form)
  h.publish(s_tab, acc);
  if (T > 1) {
    uint32_t sq[L];
    h.mont_mul(sq, acc, s_tab, m, ninv);
    h.publish(s_x, sq);
#pragma unroll 1
    for (int t = 1; t < T; ++t) {
      h.mont_mul(acc, acc, s_x, m, ninv);
      h.publish(s_tab + t * KH, acc);
    }
  }
  if (nops == 0) {
    h.load(acc, s_rm + side * KH);  // e = 0: Montgomery form of 1
  } else {
    const int first = __ldg(ops) & 0xffff;
    h.load(acc, s_tab + (first - 1) * KH);
  }
  h.publish(s_x, acc);
#pragma unroll 1
  for (int o = 1; o < nops; ++o) {
    const int op = __ldg(ops + o);
    const int sq = op >> 16;
    const int idx = op & 0xffff;
#pragma unroll 1
    for (int s = 0; s < sq; ++s) {
      h.mont_mul(acc, acc, s_x, m, ninv);
      h.publish(s_x, acc);
    }
    if (idx) {
      h.mont_mul(acc, acc, s_tab + (idx - 1) * KH, m, ninv);
      h.publish(s_x, acc);
    }
  }
  uint32_t xs[L];
  h.mont_mul(xs, acc, s_one, m, ninv);  // x_side, canonical
  __syncwarp(g.mask);
  h.store(s_x, xs);
  __syncwarp(g.mask);
  uint32_t* s_xp = s_item;
  uint32_t* s_xq = s_item + SIDE;
  if (side == 0) {
    // h = x_p (q^2)^-1 - x_q (q^2)^-1 mod p^2   (x_q may exceed p^2; x_q < R_h)
    uint32_t xq[L], v[L], u[L];
    h.load(xq, s_xq);
    h.mont_mul(v, xs, s_h, m, ninv);
    h.mont_mul(u, xq, s_h, m, ninv);
    sub_mod<KH, TPI>(h, v, u, m);
    __syncwarp(h.mask);
    h.store(s_xp, v);
  }
  __syncwarp(g.mask);
  // x = x_q + q^2 h over the whole group: side 0 lanes hold the low words
  uint32_t hv[L], xq[L], x[L];
  if (side == 0) {
    h.load(hv, s_xp);
    h.load(xq, s_xq);
  } else {
#pragma unroll
    for (int j = 0; j < L; ++j) hv[j] = xq[j] = 0u;
  }
  uint32_t n2[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.mont_mul(x, hv, s_cq, n2, ks.ninv2);  // h q^2 mod n^2 = h q^2
  (void)add_group<K, 2 * TPI>(g, x, xq);
  decrypt_epilogue<K, 2 * TPI>(g, x, out, inst, consts, ks, s_one, s_r2n, s_multr, mode, pop_words);
}

// ---------------------------------------------------------------------------
// The same CRT decrypt / decode with both exponentiations on the FP64 pipe.
//
// Per side the value mod M (p^2 or q^2, KH 32-bit words) is carried as
// K52 = 5 KH / 8 limbs of 52 bits on TPI = KH / 16 lanes (ten limbs per
// lane, sixteen 32-bit words), in the Montgomery domain of R52 = 2^(52 K52)
// (cuhe52::Group52).  Ten limbs per lane give each lane twenty independent
// products per step to cover the latency of the step's m; a 3-bit window
// keeps the table small enough for four CTAs per SM.  Entry and
// exit stay in 32-bit words: c R_h^-1 by the 32-bit reduction as in
// k_modexp_crt, then * (R52 R_h^2 mod M) gives c R52 mod M, which is
// re-cut into 52-bit limbs through shared memory; the odd-power table and
// the window schedule run as 52-bit Montgomery products; the result mod M
// is re-cut into 32-bit words and the Garner recombination and epilogue of
// k_modexp_crt follow unchanged, so the output equals k_modexp_crt's (and
// the direct kernel's) for every c < n^2.
// ---------------------------------------------------------------------------

// limb i (52 bits at 52 i) of a little-endian array of nwords 32-bit words
__device__ __forceinline__ uint64_t limb52_from_words(const uint32_t* w, int nwords, int i) {
  const int bit = 52 * i, j = bit >> 5, off = bit & 31;
  const uint64_t w0 = j < nwords ? w[j] : 0u;
  const uint64_t w1 = j + 1 < nwords ? w[j + 1] : 0u;
  const uint64_t w2 = j + 2 < nwords ? w[j + 2] : 0u;
  uint64_t v = (w0 | (w1 << 32)) >> off;
  if (off) v |= w2 << (64 - off);
  return v & cuhe52::kMask;
}

// word i (32 bits at 32 i) of an array of nlimbs 52-bit limbs
__device__ __forceinline__ uint32_t word_from_limbs52(const uint64_t* l, int nlimbs, int i) {
  const int bit = 32 * i, j = bit / 52, off = bit - 52 * j;
  const uint64_t l0 = j < nlimbs ? l[j] : 0u;
  const uint64_t l1 = j + 1 < nlimbs ? l[j + 1] : 0u;
  uint64_t v = l0 >> off;
  if (off > 20) v |= l1 << (52 - off);
  return uint32_t(v);
}

template <int KH, int W>
__global__ void __launch_bounds__(kBlockThreads, 3)
k_modexp_crt52(const uint32_t* __restrict__ base, uint32_t* __restrict__ out, long long count,
               const uint32_t* __restrict__ consts, KeyScalars ks, const uint32_t* __restrict__ crt, CrtScalars cs,
               const double* __restrict__ crt52, const int32_t* __restrict__ ops, int nops, int mode,
               int pop_words, int* status) {
  constexpr int K = 2 * KH;
  constexpr int TPI = KH / 16;     // lanes per side
  constexpr int L = 16;            // 32-bit words per lane and side
  constexpr int K52 = 5 * KH / 8;  // 52-bit limbs per side
  constexpr int L52 = K52 / TPI;   // ten
  static_assert(L52 == 10, "ten limbs per lane");
  static_assert(52 * K52 > 32 * KH + 1, "R52 must exceed 2 M");
  constexpr int T = 1 << (W - 1);
  constexpr int IPB = kBlockThreads / (2 * TPI);
  constexpr int SIDE = (T + 1) * K52 + 2;  // doubles per side: x, then T odd powers; +2 moves the banks
  extern __shared__ __align__(16) uint32_t smem[];
  // block rows: ONE, R2N, MULTR (K words each), RM, R52, H (two halves), CQ; then 1 as K52 doubles
  uint32_t* s_one = smem;
  uint32_t* s_r2n = smem + K;
  uint32_t* s_multr = smem + 2 * K;
  uint32_t* s_rm = smem + 3 * K;
  uint32_t* s_r52 = smem + 4 * K;
  uint32_t* s_h = smem + 5 * K;
  uint32_t* s_cq = smem + 6 * K;
  double* s_one52 = reinterpret_cast<double*>(smem + 7 * K);
  double* s_items = s_one52 + K52;
  {
    const int rows[3] = {C_ONE, C_R2N, C_MULTR};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 3);
    const int crows[4] = {CR_RM, CR_R52, CR_H, CR_CQ};
    copy_rows_to_smem<K, TPI>(smem + 3 * K, crt, crows, 4);
    for (int i = threadIdx.x; i < K52; i += blockDim.x) s_one52[i] = i == 0 ? 1.0 : 0.0;
  }
  __syncthreads();

  Group<K, 2 * TPI> g;            // the whole ciphertext, 32-bit words
  Group<KH, TPI> h;               // this side's half, 32-bit words
  cuhe52::Group52<K52, TPI> f;    // this side's half, 52-bit limbs
  const int side = (threadIdx.x / TPI) & 1;
  const int slot = threadIdx.x / (2 * TPI);
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;  // both halves leave together
  double* s_x = s_items + (slot * 2 + side) * SIDE;
  double* s_tab = s_x + K52;

  {
    uint32_t c[L], n2[L];
    g.load_ro(n2, consts + C_N2 * K);
    g.load(c, base + inst * K);
    if (!g.less_than(c, n2)) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
  }
  const uint32_t ninv = cs.ninv[side];
  uint32_t* s_w = reinterpret_cast<uint32_t*>(s_x);  // KH words fit in the K52 doubles of x
  {
    // c = lo + hi R_h:  (lo + hi * (R_h mod M)) R_h^-1 = c R_h^-1, then * R52 R_h^2 R_h^-1 = c R52
    uint32_t m[L], lo[L], hi[L], acc[L];
    h.load_ro(m, crt + CR_M * K + side * KH);
    h.load(lo, base + inst * K);
    h.load(hi, base + inst * K + KH);
    h.mont_mul_acc(acc, lo, hi, s_rm + side * KH, m, ninv);
    h.mont_mul(acc, acc, s_r52 + side * KH, m, ninv);
    h.publish(s_w, acc);
  }
  double x52[L52], m52[L52], acc52[L52];
  const double* cm = crt52 + side * 2 * K52;  // M, then R52 mod M
#pragma unroll
  for (int k = 0; k < L52; ++k) {
    x52[k] = cuhe52::to_f64(limb52_from_words(s_w, KH, f.gl * L52 + k));
    m52[k] = __ldg(cm + f.gl * L52 + k);
  }
  const uint64_t ninv52 = cs.ninv52[side];
  f.publish(s_tab, x52);
#pragma unroll
  for (int k = 0; k < L52; ++k) acc52[k] = x52[k];
  // Every Montgomery product of the exponentiation goes through the one
  // call site below: the unrolled product is large, and a single copy of it
  // stays in the instruction cache.  Phases: the odd-power table (x^2 to
  // s_x, then x^3 .. x^(2T-1)), the window schedule (squarings of s_x and
  // products with table entries), the final product with 1.
  enum { kTable = 0, kSchedule = 1, kFinal = 2, kDone = 3 };
  int phase = T > 1 ? kTable : kSchedule, pc = 0, o = 1, sq_left = 0, idx = 0;
  if (phase == kSchedule) pc = T;  // no table products: go straight to the schedule set-up
  double xs52[L52];
  while (phase != kDone) {
    if (phase == kTable || pc == T) {
      // (after the table) the schedule starts from its first table entry
      if (phase == kSchedule && pc == T) {
        pc = 0;
        if (nops == 0) {
#pragma unroll
          for (int k = 0; k < L52; ++k) acc52[k] = __ldg(cm + K52 + f.gl * L52 + k);  // e = 0: R52 mod M
        } else {
          const int first = __ldg(ops) & 0xffff;
          __syncwarp(f.mask);
#pragma unroll
          for (int k = 0; k < L52; ++k) acc52[k] = s_tab[(first - 1) * K52 + f.gl * L52 + k];
        }
        f.publish(s_x, acc52);
        while (sq_left == 0 && idx == 0) {
          if (o >= nops) {
            phase = kFinal;
            break;
          }
          const int op = __ldg(ops + o++);
          sq_left = op >> 16;
          idx = op & 0xffff;
        }
      }
    }
    const double* bsrc = phase == kTable   ? (pc == 0 ? s_tab : s_x)
                         : phase == kFinal ? s_one52
                         : sq_left > 0     ? s_x
                                           : s_tab + (idx - 1) * K52;
    f.mont_mul(xs52, acc52, bsrc, m52, ninv52);
    if (phase == kFinal) break;  // xs52 = x_side, canonical
    if (phase == kTable && pc == 0) {
      f.publish(s_x, xs52);  // x^2 R52; acc52 stays x
    } else {
#pragma unroll
      for (int k = 0; k < L52; ++k) acc52[k] = xs52[k];
      f.publish(phase == kTable ? s_tab + pc * K52 : s_x, acc52);
    }
    if (phase == kTable) {
      if (++pc == T) phase = kSchedule;  // pc == T: set-up at the top of the next pass
      continue;
    }
    if (sq_left > 0) --sq_left;
    else idx = 0;
    while (sq_left == 0 && idx == 0) {
      if (o >= nops) {
        phase = kFinal;
        break;
      }
      const int op = __ldg(ops + o++);
      sq_left = op >> 16;
      idx = op & 0xffff;
    }
  }
  uint64_t* s_l = reinterpret_cast<uint64_t*>(s_x);
  __syncwarp(f.mask);
#pragma unroll
  for (int k = 0; k < L52; ++k) s_l[f.gl * L52 + k] = cuhe52::to_u64(xs52[k]);
  __syncwarp(f.mask);
  uint32_t xs[L];
#pragma unroll
  for (int j = 0; j < L; ++j) xs[j] = word_from_limbs52(s_l, K52, h.gl * L + j);
  __syncwarp(g.mask);
  uint32_t* s_xp = reinterpret_cast<uint32_t*>(s_items + (slot * 2) * SIDE);
  uint32_t* s_xq = reinterpret_cast<uint32_t*>(s_items + (slot * 2 + 1) * SIDE);
  h.store(side == 0 ? s_xp : s_xq, xs);
  __syncwarp(g.mask);
  if (side == 0) {
    // h = x_p (q^2)^-1 - x_q (q^2)^-1 mod p^2   (x_q may exceed p^2; x_q < R_h)
    uint32_t m[L], xq[L], v[L], u[L];
    h.load_ro(m, crt + CR_M * K);
    h.load(xq, s_xq);
    h.mont_mul(v, xs, s_h, m, ninv);
    h.mont_mul(u, xq, s_h, m, ninv);
    sub_mod<KH, TPI>(h, v, u, m);
    __syncwarp(h.mask);
    h.store(s_xp, v);
  }
  __syncwarp(g.mask);
  // x = x_q + q^2 h over the whole group: side 0 lanes hold the low words
  uint32_t hv[L], xq[L], x[L];
  if (side == 0) {
    h.load(hv, s_xp);
    h.load(xq, s_xq);
  } else {
#pragma unroll
    for (int j = 0; j < L; ++j) hv[j] = xq[j] = 0u;
  }
  uint32_t n2[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.mont_mul(x, hv, s_cq, n2, ks.ninv2);  // h q^2 mod n^2 = h q^2
  (void)add_group<K, 2 * TPI>(g, x, xq);
  decrypt_epilogue<K, 2 * TPI>(g, x, out, inst, consts, ks, s_one, s_r2n, s_multr, mode, pop_words);
}

// ---------------------------------------------------------------------------
// The exponentiation mod n^2 itself on the FP64 pipe, for the exponents that
// need no factors (encryption's r^n, any fixed public exponent) and for
// decryption when the factors are not installed.  The value is carried as
// K52 = 5K/8 limbs of 52 bits on K/16 lanes (ten limbs per lane) in the
// Montgomery domain of R52 = 2^(52 K52), with k_modexp_crt52's product and
// schedule; entry: x R52 mod n^2 by one 32-bit Montgomery product with
// R52 R mod n^2, exit: the product with 1, re-cut into 32-bit words; then
// k_modexp's modes on 32-bit words (the factor 1 + m n of an encryption,
// the L() / popcount epilogue), so every output equals k_modexp's.
// n52: n^2 and R52 mod n^2 as K52 doubles each, then R52 R mod n^2 as K words.
// ---------------------------------------------------------------------------
template <int K, int W>
__device__ __forceinline__ void modexp52_unit(const uint32_t* __restrict__ base, const uint32_t* __restrict__ aux,
                                              int aux_words, uint32_t* __restrict__ out, long long count,
                                              const uint32_t* __restrict__ consts, const KeyScalars& ks,
                                              const double* __restrict__ n52, unsigned long long ninv52,
                                              const int32_t* __restrict__ ops, int nops, int mode, int pop_words,
                                              int* status, long long block) {
  constexpr int TPI = K / 16;      // lanes per value
  constexpr int L = 16;            // 32-bit words per lane
  constexpr int K52 = 5 * K / 8;   // 52-bit limbs
  constexpr int L52 = K52 / TPI;   // ten
  static_assert(L52 == 10, "ten limbs per lane");
  static_assert(52 * K52 > 32 * K + 1, "R52 must exceed 2 n^2");
  constexpr int T = 1 << (W - 1);
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int SLOT = (T + 1) * K52 + 2;  // doubles per value: x, then T odd powers; +2 moves the banks
  extern __shared__ __align__(16) uint32_t smem[];
  // block rows: ONE, R2, NR, R2N, MULTR, R52 R (K words each); then 1 as K52 doubles
  uint32_t* s_one = smem;
  uint32_t* s_r2 = smem + K;
  uint32_t* s_nr = smem + 2 * K;
  uint32_t* s_r2n = smem + 3 * K;
  uint32_t* s_multr = smem + 4 * K;
  uint32_t* s_r52r = smem + 5 * K;
  double* s_one52 = reinterpret_cast<double*>(smem + 6 * K);
  double* s_items = s_one52 + K52;
  {
    const int rows[5] = {C_ONE, C_R2, C_NR, C_R2N, C_MULTR};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 5);
    const uint32_t* r52r = reinterpret_cast<const uint32_t*>(n52 + 2 * K52);
    for (int i = threadIdx.x; i < K; i += blockDim.x) s_r52r[i] = r52r[i];
    for (int i = threadIdx.x; i < K52; i += blockDim.x) s_one52[i] = i == 0 ? 1.0 : 0.0;
  }
  __syncthreads();

  Group<K, TPI> g;                // the value, 32-bit words
  cuhe52::Group52<K52, TPI> f;    // the value, 52-bit limbs (same lanes)
  const int slot = threadIdx.x / TPI;
  const long long inst = block * IPB + slot;
  if (inst >= count) return;  // whole groups leave together
  double* s_x = s_items + slot * SLOT;
  double* s_tab = s_x + K52;
  uint32_t* s_w = reinterpret_cast<uint32_t*>(s_x);  // K words fit in the K52 doubles of x
  uint32_t n2[L];
  g.load_ro(n2, consts + C_N2 * K);
  {
    uint32_t x[L], xr[L];
    g.load(x, base + inst * K);
    if (!g.less_than(x, n2)) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
    g.mont_mul(xr, x, s_r52r, n2, ks.ninv2);  // x R52 mod n^2
    g.publish(s_w, xr);
  }
  double x52[L52], m52[L52], acc52[L52];
#pragma unroll
  for (int k = 0; k < L52; ++k) {
    x52[k] = cuhe52::to_f64(limb52_from_words(s_w, K, f.gl * L52 + k));
    m52[k] = __ldg(n52 + f.gl * L52 + k);
  }
  f.publish(s_tab, x52);
#pragma unroll
  for (int k = 0; k < L52; ++k) acc52[k] = x52[k];
  // One call site for every product (k_modexp_crt52): the odd-power table,
  // the window schedule, the final product with 1.
  enum { kTable = 0, kSchedule = 1, kFinal = 2 };
  int phase = T > 1 ? kTable : kSchedule, pc = 0, o = 1, sq_left = 0, idx = 0;
  if (phase == kSchedule) pc = T;
  double xs52[L52];
  while (true) {
    if (phase == kSchedule && pc == T) {
      pc = 0;
      if (nops == 0) {
#pragma unroll
        for (int k = 0; k < L52; ++k) acc52[k] = __ldg(n52 + K52 + f.gl * L52 + k);  // e = 0: R52 mod n^2
      } else {
        const int first = __ldg(ops) & 0xffff;
        __syncwarp(f.mask);
#pragma unroll
        for (int k = 0; k < L52; ++k) acc52[k] = s_tab[(first - 1) * K52 + f.gl * L52 + k];
      }
      f.publish(s_x, acc52);
      while (sq_left == 0 && idx == 0) {
        if (o >= nops) {
          phase = kFinal;
          break;
        }
        const int op = __ldg(ops + o++);
        sq_left = op >> 16;
        idx = op & 0xffff;
      }
    }
    const double* bsrc = phase == kTable   ? (pc == 0 ? s_tab : s_x)
                         : phase == kFinal ? s_one52
                         : sq_left > 0     ? s_x
                                           : s_tab + (idx - 1) * K52;
    f.mont_mul(xs52, acc52, bsrc, m52, ninv52);
    if (phase == kFinal) break;  // xs52 = x^e, canonical
    if (phase == kTable && pc == 0) {
      f.publish(s_x, xs52);  // x^2 R52; acc52 stays x
    } else {
#pragma unroll
      for (int k = 0; k < L52; ++k) acc52[k] = xs52[k];
      f.publish(phase == kTable ? s_tab + pc * K52 : s_x, acc52);
    }
    if (phase == kTable) {
      if (++pc == T) phase = kSchedule;  // pc == T: set-up at the top of the next pass
      continue;
    }
    if (sq_left > 0) --sq_left;
    else idx = 0;
    while (sq_left == 0 && idx == 0) {
      if (o >= nops) {
        phase = kFinal;
        break;
      }
      const int op = __ldg(ops + o++);
      sq_left = op >> 16;
      idx = op & 0xffff;
    }
  }
  uint64_t* s_l = reinterpret_cast<uint64_t*>(s_x);
  __syncwarp(f.mask);
#pragma unroll
  for (int k = 0; k < L52; ++k) s_l[f.gl * L52 + k] = cuhe52::to_u64(xs52[k]);
  __syncwarp(f.mask);
  uint32_t x[L];
#pragma unroll
  for (int j = 0; j < L; ++j) x[j] = word_from_limbs52(s_l, K52, g.gl * L + j);
  if (mode == EXP_POW) {
    g.store(out + inst * K, x);
    return;
  }
  if (mode == EXP_ENCRYPT) {
    uint32_t m[L], nn[L], gm[L], xr[L];
    g.load(m, aux + inst * aux_words);  // aux_words == K (zero-padded m < n)
    g.load_ro(nn, consts + C_N * K);
    if (!g.less_than(m, nn)) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
    g.mont_mul(gm, m, s_nr, n2, ks.ninv2);  // m*n (exact, < n^2)
    add_small<K, TPI>(g, gm, 1u);           // 1 + m*n = g^m mod n^2
    g.publish(s_w, gm);
    g.mont_mul(xr, x, s_r2, n2, ks.ninv2);  // r^n R
    g.mont_mul(x, xr, s_w, n2, ks.ninv2);   // r^n * g^m
    g.store(out + inst * K, x);
    return;
  }
  decrypt_epilogue<K, TPI>(g, x, out, inst, consts, ks, s_one, s_r2n, s_multr, mode, pop_words);
}

template <int K, int W>
__global__ void __launch_bounds__(kBlockThreads, 3)
k_modexp52(const uint32_t* __restrict__ base, const uint32_t* __restrict__ aux, int aux_words,
           uint32_t* __restrict__ out, long long count, const uint32_t* __restrict__ consts, KeyScalars ks,
           const double* __restrict__ n52, unsigned long long ninv52, const int32_t* __restrict__ ops, int nops,
           int mode, int pop_words, int* status) {
  modexp52_unit<K, W>(base, aux, aux_words, out, count, consts, ks, n52, ninv52, ops, nops, mode, pop_words, status,
                      blockIdx.x);
}

// The persistent mixed launch (k_modexp_tasks) on the FP64 pipe: units of
// IPB = 128 / (K/16) instances of one task.
template <int K, int W>
__global__ void __launch_bounds__(kBlockThreads, 3)
k_modexp52_tasks(const ModexpTask* __restrict__ tasks, int ntasks, long long total_units,
                 unsigned long long* __restrict__ counter, int* status) {
  __shared__ long long s_unit;
  while (true) {
    if (threadIdx.x == 0) s_unit = (long long)atomicAdd(counter, 1ull);
    __syncthreads();
    const long long unit = s_unit;
    if (unit >= total_units) break;
    int lo = 0, hi = ntasks - 1;  // last task with first_unit <= unit
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tasks[mid].first_unit <= unit) lo = mid; else hi = mid - 1;
    }
    const ModexpTask& t = tasks[lo];
    modexp52_unit<K, W>(t.base, nullptr, K, t.out, t.count, t.consts, t.ks, t.n52, t.ninv52, t.ops, t.nops, t.mode,
                        0, status, unit - t.first_unit);
    __syncthreads();  // shared rows and tables are restaged by the next unit
  }
}

// ---------------------------------------------------------------------------
// encode_hamming_server on the FP64 pipe (n^2 of 4096 / 8192 bits):
// out[q][j] = index[j] * query[q] mod n^2 as one Montgomery product of 52-bit
// limbs, the query entering in the Montgomery domain of R52
// (k_to_mont52: query R52 mod n^2, once per query) and the index value and
// the result crossing between 32-bit words and 52-bit limbs by bit
// shuffling, so each output costs one product: mont52(index, query R52) =
// index * query mod n^2, canonical, as k_mulmod_outer's.
// ---------------------------------------------------------------------------
// row: R52 R mod n^2 for plain inputs, R52 mod n^2 for inputs already in
// the 32-bit Montgomery form (x R): either way out = x R52 mod n^2.
template <int K>
__global__ void __launch_bounds__(kBlockThreads)
k_to_mont52(const uint32_t* __restrict__ in, long long count, double* __restrict__ out,
            const uint32_t* __restrict__ consts, KeyScalars ks, const uint32_t* __restrict__ row, int* status) {
  constexpr int TPI = K / 16, L = 16, K52 = 5 * K / 8, L52 = K52 / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_r52r = smem;
  for (int i = threadIdx.x; i < K; i += blockDim.x) s_r52r[i] = row[i];
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint32_t n2[L], x[L], xr[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load(x, in + inst * K);
  if (!g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  g.mont_mul(xr, x, s_r52r, n2, ks.ninv2);  // x R52 mod n^2
  uint32_t* s_w = smem + K + slot * K;
  g.publish(s_w, xr);
#pragma unroll
  for (int k = 0; k < L52; ++k)
    out[inst * K52 + g.gl * L52 + k] = cuhe52::to_f64(limb52_from_words(s_w, K, g.gl * L52 + k));
}


template <int K>
__global__ void __launch_bounds__(kBlockThreads, 3)
k_mulmod_outer52(const double* __restrict__ q52, const uint32_t* __restrict__ index, long long nx,
                 uint32_t* __restrict__ out, const uint32_t* __restrict__ consts, const double* __restrict__ n52,
                 unsigned long long ninv52, int* status) {
  constexpr int TPI = K / 16, L = 16, K52 = 5 * K / 8, L52 = K52 / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) double smd[];
  double* s_b = smd;          // the query, K52 limbs (Montgomery form)
  double* s_inst = smd + K52; // per instance K52 doubles: the index words in, the result limbs out
  const long long qi = blockIdx.y;
  for (int i = threadIdx.x; i < K52; i += blockDim.x) s_b[i] = q52[qi * K52 + i];
  __syncthreads();
  Group<K, TPI> g;
  cuhe52::Group52<K52, TPI> f;
  const int slot = threadIdx.x / TPI;
  const long long j = (long long)blockIdx.x * IPB + slot;
  if (j >= nx) return;
  uint32_t n2[L], x[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(x, index + j * K);
  if (!g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  uint32_t* s_w = reinterpret_cast<uint32_t*>(s_inst + slot * K52);
  g.publish(s_w, x);
  double a52[L52], m52[L52], r52[L52];
#pragma unroll
  for (int k = 0; k < L52; ++k) {
    a52[k] = cuhe52::to_f64(limb52_from_words(s_w, K, f.gl * L52 + k));
    m52[k] = __ldg(n52 + f.gl * L52 + k);
  }
  f.mont_mul(r52, a52, s_b, m52, ninv52);
  uint64_t* s_l = reinterpret_cast<uint64_t*>(s_inst + slot * K52);
  __syncwarp(f.mask);
#pragma unroll
  for (int k = 0; k < L52; ++k) s_l[f.gl * L52 + k] = cuhe52::to_u64(r52[k]);
  __syncwarp(f.mask);
  uint32_t w[L];
#pragma unroll
  for (int t = 0; t < L; ++t) w[t] = word_from_limbs52(s_l, K52, g.gl * L + t);
  g.store(out + (qi * nx + j) * K, w);
}

// ---------------------------------------------------------------------------
// Modular exponentiation with a per-instance exponent (fixed 4-bit windows, so
// every group of a warp follows the same schedule):
//   out[i] = base[i]^exps[i] mod n^2, exps[i] held in exp_words words.
// ---------------------------------------------------------------------------
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_modexp_var(const uint32_t* __restrict__ base, const uint32_t* __restrict__ exps, int exp_words, int windows,
             uint32_t* __restrict__ out, long long count, const uint32_t* __restrict__ consts, KeyScalars ks,
             int* status) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int T = 16;
  constexpr int STRIDE = inst_stride_words<K>(T + 1);
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_one = smem;
  uint32_t* s_r2 = smem + K;
  {
    const int rows[2] = {C_ONE, C_R2};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 2);
  }
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint32_t* s_x = smem + 2 * K + slot * STRIDE;
  uint32_t* s_tab = s_x + K;
  uint32_t n2[L], x[L], acc[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load(x, base + inst * K);
  if (!g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  g.load_ro(acc, consts + C_RM * K);
  g.publish(s_tab, acc);                   // x^0
  g.mont_mul(acc, x, s_r2, n2, ks.ninv2);  // x^1
  g.publish(s_tab + K, acc);
  g.publish(s_x, acc);
#pragma unroll 1
  for (int t = 2; t < T; ++t) {
    g.mont_mul(acc, acc, s_x, n2, ks.ninv2);
    g.publish(s_tab + t * K, acc);
  }
  const uint32_t* e = exps + inst * exp_words;
  g.load_ro(acc, consts + C_RM * K);
  g.publish(s_x, acc);
  bool started = false;
#pragma unroll 1
  for (int w = windows - 1; w >= 0; --w) {
    const int bit = 4 * w;
    const int digit = (bit / 32 < exp_words) ? int((__ldg(e + bit / 32) >> (bit % 32)) & 15u) : 0;
    if (started) {
#pragma unroll 1
      for (int s = 0; s < 4; ++s) {
        g.mont_mul(acc, acc, s_x, n2, ks.ninv2);
        g.publish(s_x, acc);
      }
    }
    if (digit) {
      g.mont_mul(acc, acc, s_tab + digit * K, n2, ks.ninv2);
      g.publish(s_x, acc);
      started = true;
    }
  }
  g.mont_mul(x, acc, s_one, n2, ks.ninv2);
  g.store(out + inst * K, x);
}

// distance[v] = sum of the chunk_num per-chunk popcounts of vector v.
__global__ void k_sum_chunks(const uint32_t* __restrict__ counts, long long vectors, int chunk_num,
                             long long* __restrict__ distance) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= vectors) return;
  long long s = 0;
  for (int c = 0; c < chunk_num; ++c) s += counts[v * chunk_num + c];
  distance[v] = s;
}

// Integer multiply-add throughput probe in the Montgomery kernels' own
// instruction mix: four independent 8-limb accumulators, each updated per
// iteration by one mad.lo.cc/madc.hi.cc row (8 word products, the shape of
// Group::mac_row) with no shuffles or memory traffic, so the probe is bound
// only by the integer multiply pipe.  Each row is 8 word products.
// FP64-pipe probe: eight independent fused multiply-add chains per thread
// (round toward zero, the form of the limb products), FP64 instructions only.
__global__ void __launch_bounds__(256) k_fp64_probe(double* sink, int iters, double seed) {
  double x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = seed + 1e-3 * double(threadIdx.x) + double(j);
  const double y = 1.0000000001, z = 1e-9;
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = __fma_rz(x[j], y, z);
  }
  double folded = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) folded += x[j];
  if (folded == 1.2345678) sink[0] = folded;
}

__global__ void __launch_bounds__(256) k_imad_chain_probe(uint32_t* sink, int iters, uint32_t seed) {
  uint32_t acc[4][8], c0[4], c1[4], a[8];
  const uint32_t b = seed * 2654435761u + blockIdx.x;
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = (seed ^ threadIdx.x) * (j + 3u) + 0x9e3779b9u;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    c0[s] = c1[s] = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[s][j] = a[j] ^ s;
  }
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int s = 0; s < 4; ++s) Group<128, 16>::mac_row(acc[s], c0[s], c1[s], a, b + s);
  }
  uint32_t folded = 0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    folded ^= c0[s] ^ c1[s];
#pragma unroll
    for (int j = 0; j < 8; ++j) folded ^= acc[s][j];
  }
  if (folded == 0x12345678u) sink[0] = folded;
}

// Integer multiply-add throughput probe in 64-bit form: every iteration
// issues one mad.wide.u32 (a full 32x32->64 word product added to a 64-bit
// accumulator) on each of eight independent accumulators.
__global__ void __launch_bounds__(256) k_imad_wide_probe(uint32_t* sink, int iters, uint32_t seed) {
  unsigned long long acc[8];
  const uint32_t b = seed * 2654435761u + blockIdx.x;
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = ((unsigned long long)(seed ^ threadIdx.x) << 7) + 977u * j + 1u;
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t lo = uint32_t(acc[j]);
      asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc[j]) : "r"(lo), "r"(b));
    }
  }
  unsigned long long folded = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) folded ^= acc[j];
  if (folded == 0x9e3779b97f4a7c15ull) sink[0] = uint32_t(folded);
}

// Integer multiply-add throughput probe: every iteration issues one
// mad.lo.u32 and one mad.hi.u32 (one 32x32->64 word product) per operand
// pair into 16 accumulators that depend only on themselves.
__global__ void __launch_bounds__(256) k_imad_probe(uint32_t* sink, int iters, uint32_t seed) {
  uint32_t lo[8], hi[8], x[8];
  const uint32_t a = seed ^ threadIdx.x, b = seed * 2654435761u + blockIdx.x;
#pragma unroll
  for (int j = 0; j < 8; ++j) { lo[j] = a + j; hi[j] = b - j; x[j] = (a * 33u) ^ (b + 7u * j); }
#pragma unroll 1
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      asm volatile("mad.lo.u32 %0, %1, %2, %0;" : "+r"(lo[j]) : "r"(x[j]), "r"(b));
      asm volatile("mad.hi.u32 %0, %1, %2, %0;" : "+r"(hi[j]) : "r"(x[j]), "r"(b));
    }
  }
  uint32_t folded = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) folded ^= lo[j] ^ hi[j];
  if (folded == 0x9e3779b9u) sink[0] = folded;
}

// ---------------------------------------------------------------------------
// Pointwise modular multiplication: out[i] = a[i] * b[i] mod n^2.
// ---------------------------------------------------------------------------
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_mulmod(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t* __restrict__ out,
         long long count, const uint32_t* __restrict__ consts, KeyScalars ks, int* status) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int STRIDE = inst_stride_words<K>(1);
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_r2 = smem;
  {
    const int rows[1] = {C_R2};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 1);
  }
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint32_t* s_b = smem + K + slot * STRIDE;
  uint32_t n2[L], x[L], y[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load(x, a + inst * K);
  g.load(y, b + inst * K);
  if (!g.less_than(x, n2) || !g.less_than(y, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  g.publish(s_b, y);
  g.mont_mul(x, x, s_b, n2, ks.ninv2);   // a b R^-1
  g.mont_mul(x, x, s_r2, n2, ks.ninv2);  // a b
  g.store(out + inst * K, x);
}

// out[q][j] = query[q] * index[j] mod n^2 with queries given in Montgomery form
// (query * R mod n^2).  One Montgomery product per output.
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_mulmod_outer(const uint32_t* __restrict__ qmont, long long nq, const uint32_t* __restrict__ index,
               long long nx, uint32_t* __restrict__ out, const uint32_t* __restrict__ consts, KeyScalars ks,
               int* status) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) uint32_t smem[];
  const long long qi = blockIdx.y;
  for (int i = threadIdx.x; i < K; i += blockDim.x) smem[i] = qmont[qi * K + i];
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long j = (long long)blockIdx.x * IPB + slot;
  if (j >= nx) return;
  uint32_t n2[L], x[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(x, index + j * K);
  if (!g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  g.mont_mul(x, x, smem, n2, ks.ninv2);
  g.store(out + (qi * nx + j) * K, x);
}

// out[i] = in[i] * R mod n^2 (to Montgomery form), or in[i] * R^-1 (from).
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_convert(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, long long count,
          const uint32_t* __restrict__ consts, KeyScalars ks, int to_mont, int* status) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) uint32_t smem[];
  {
    const int rows[1] = {to_mont ? (int)C_R2 : (int)C_ONE};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 1);
  }
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint32_t n2[L], x[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load(x, in + inst * K);
  // to_mont == 2: any x < 2^(32K) (x R mod n^2: the CIOS bound holds for any
  // first operand below R), the first half of a reduction mod n^2
  if (to_mont != 2 && !g.less_than(x, n2)) {
    if (g.gl == 0) atomicOr(status, ST_RANGE);
    return;
  }
  g.mont_mul(x, x, smem, n2, ks.ninv2);
  g.store(out + inst * K, x);
}

// Hexadecimal text <-> little-endian 32-bit limbs, one thread per limb.
// Value i is text[offsets[i], offsets[i+1]) with an optional 0x / 0X
// prefix; limb w holds the digits 8w .. 8w+7 counted from the right, digits
// beyond the K-th limb are dropped (the reference's hex_to_le_words keeps
// the low limbs), and any character that is not a hex digit sets ST_HEX.
enum : int { ST_HEX = 2 };

__device__ __forceinline__ int hex_value(char c) {
  if (c >= '0' && c <= '9') return c - '0';
  if (c >= 'a' && c <= 'f') return c - 'a' + 10;
  if (c >= 'A' && c <= 'F') return c - 'A' + 10;
  return -1;
}

__global__ void k_hex_to_limbs(const char* __restrict__ text, const long long* __restrict__ offsets, long long count,
                               int words, uint32_t* __restrict__ out, int* status) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count * words) return;
  const long long i = t / words;
  const int w = int(t - i * words);
  long long s = offsets[i];
  const long long e = offsets[i + 1];
  if (e - s >= 2 && text[s] == '0' && (text[s + 1] == 'x' || text[s + 1] == 'X')) s += 2;
  uint32_t v = 0;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const long long pos = e - 1 - 8ll * w - j;
    if (pos >= s) {
      const int d = hex_value(text[pos]);
      bad |= d < 0;
      v |= uint32_t(d < 0 ? 0 : d) << (4 * j);
    }
  }
  if (w == words - 1)
    for (long long pos = s; pos < e - 8ll * words; ++pos) bad |= hex_value(text[pos]) < 0;
  out[t] = v;
  if (bad) atomicOr(status, ST_HEX);
}

// out[i * 8 words ...]: value i as 8 * words lowercase digits, most significant first
__global__ void k_limbs_to_hex(const uint32_t* __restrict__ limbs, long long count, int words, char* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count * words) return;
  const long long i = t / words;
  const int w = int(t - i * words);
  const uint32_t v = limbs[t];
  char* o = out + i * 8ll * words + 8ll * (words - 1 - w);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t d = (v >> (4 * (7 - j))) & 15u;
    o[j] = char(d < 10 ? '0' + d : 'a' + d - 10);
  }
}

// ---------------------------------------------------------------------------
// Paillier-Lookup encryption by fixed-base table product:
//   c = prod_i G[i][digit_i(m)] * prod_k NOISE[idx_k]  mod n^2
// G and NOISE are device-resident in Montgomery form.  The plaintext digits
// come either from binary embeddings (Hamming padding "0b" per bit, read as
// MSB-first chunks of chunk_len bits) or from little-endian plaintext words.
// kWide: G is the 16-bit-digit table W[j][D] = G[2j][D mod 256] *
// G[2j+1][D / 256] (k_wide_table), one product per pair of 8-bit digits; the
// product of the same powers of g, so the ciphertext is the same.  The next
// table row is loaded while the current product runs.
// ---------------------------------------------------------------------------
constexpr int kNoiseMultiples = 14;

// 16-bit entries of row list per instance: message_chunks rounded up to even
__host__ __device__ constexpr int lookup_rows_stride(int message_chunks) { return (message_chunks + 1) & ~1; }

// The table rows of an instance's nonzero digits (one lane): 8-bit digits as
// i * 256 + d into rows16, or with kWide 16-bit digits as j * 65536 + D into
// rows32 (the same storage); returns their count.  Digits come from a binary
// embedding (Hamming padding "0b" per bit, MSB-first chunks of chunk_len
// bits) or from little-endian plaintext words.
template <bool kWide>
__device__ __forceinline__ int lookup_digit_rows(const uint8_t* __restrict__ bits, int embed_len, int chunk_len,
                                                 int chunk_num, const uint32_t* __restrict__ plain, int plain_words,
                                                 long long inst, int message_chunks, uint16_t* s_rows16) {
  uint32_t* s_rows32 = reinterpret_cast<uint32_t*>(s_rows16);
  int cnt = 0;
  int pending = 0;  // kWide: the low byte of the current 16-bit digit
  auto push = [&](int i, int d) {
    if (kWide) {
      if ((i & 1) == 0) {
        pending = d;
        if (i + 1 == message_chunks && d) s_rows32[cnt++] = uint32_t(i / 2) * 65536u + uint32_t(d);
      } else if (pending | d) {
        s_rows32[cnt++] = uint32_t(i / 2) * 65536u + uint32_t(pending + 256 * d);
      }
    } else if (d) {
      s_rows16[cnt++] = uint16_t(i * 256 + d);
    }
  };
  if (bits) {
    const long long vec = inst / chunk_num;
    const int chunk = int(inst % chunk_num);
    const int padded_total = 2 * embed_len;
    const int cbase = chunk * chunk_len;
    int avail = padded_total - cbase;
    if (avail > chunk_len) avail = chunk_len;
    if (avail < 0) avail = 0;
    const uint8_t* vb = bits + vec * embed_len;
    for (int i = 0; i < message_chunks; ++i) {
      int d = 0;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int e = 8 * i + b;  // exponent within the chunk value
        if (e < avail) {
          const int p = cbase + (avail - 1 - e);  // padded MSB-first position
          if (p & 1) d |= (vb[p >> 1] & 1) << b;
        }
      }
      push(i, d);
    }
  } else {
    const uint8_t* mb = reinterpret_cast<const uint8_t*>(plain + inst * plain_words);
    const int bytes = plain_words * 4 < message_chunks ? plain_words * 4 : message_chunks;
    for (int i = 0; i < message_chunks; ++i) push(i, i < bytes ? int(mb[i]) : 0);
  }
  return cnt;
}

template <int K, int TPI, bool kWide = false>
__global__ void __launch_bounds__(kBlockThreads)
k_lookup_encrypt(const uint8_t* __restrict__ bits, int embed_len, int chunk_len, int chunk_num,
                 const uint32_t* __restrict__ plain, int plain_words, long long count, int message_chunks,
                 const uint32_t* __restrict__ gtab, const uint32_t* __restrict__ noise, int noise_entries,
                 const uint8_t* __restrict__ noise_idx, uint32_t* __restrict__ out,
                 const uint32_t* __restrict__ consts, KeyScalars ks, int* status) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int ACC_STRIDE = inst_stride_words<K>(1);
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_one = smem;
  {
    const int rows[1] = {C_ONE};
    copy_rows_to_smem<K, TPI>(smem, consts, rows, 1);
  }
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint32_t* s_acc = smem + K + slot * ACC_STRIDE;
  // table rows of the nonzero digits: 8-bit digits as i * 256 + d (16 bits),
  // 16-bit digits as j * 65536 + D (32 bits); lookup_rows_stride(message_chunks)
  // 16-bit entries (a multiple of four bytes) a slot either way
  uint16_t* s_rows16 =
      reinterpret_cast<uint16_t*>(smem + K + IPB * ACC_STRIDE) + slot * lookup_rows_stride(message_chunks);
  uint32_t* s_rows32 = reinterpret_cast<uint32_t*>(s_rows16);
  __shared__ int s_count[IPB];

  // nonzero digits -> list of table rows (lane 0 of the group)
  if (g.gl == 0)
    s_count[slot] = lookup_digit_rows<kWide>(bits, embed_len, chunk_len, chunk_num, plain, plain_words, inst,
                                             message_chunks, s_rows16);
  __syncwarp(g.mask);
  const int cnt = s_count[slot];
  auto row_of = [&](int j) -> long long { return kWide ? (long long)s_rows32[j] : (long long)s_rows16[j]; };

  uint32_t n2[L], acc[L], a[L], nx[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(acc, consts + C_RM * K);  // Montgomery one
  g.publish(s_acc, acc);
  if (cnt > 0) g.load_ro(a, gtab + row_of(0) * K);
#pragma unroll 1
  for (int j = 0; j < cnt; ++j) {
    if (j + 1 < cnt) g.load_ro(nx, gtab + row_of(j + 1) * K);
    g.mont_mul(acc, a, s_acc, n2, ks.ninv2);
    g.publish(s_acc, acc);
#pragma unroll
    for (int k = 0; k < L; ++k) a[k] = nx[k];
  }
  const uint8_t* idx = noise_idx + inst * kNoiseMultiples;
#pragma unroll 1
  for (int k = 0; k < kNoiseMultiples; ++k) {
    const int r = idx[k];
    if (r >= noise_entries) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
    g.load_ro(a, noise + (long long)r * K);
    g.mont_mul(acc, a, s_acc, n2, ks.ninv2);
    g.publish(s_acc, acc);
  }
  g.mont_mul(a, acc, s_one, n2, ks.ninv2);
  g.store(out + inst * K, a);
}

// The 16-bit-digit table: W[j][D] = G[2j][D mod 256] * G[2j+1][D / 256]
// (Montgomery form in and out; for an odd message_chunks the last row's high
// factor is 1).  One group per entry.
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_wide_table(const uint32_t* __restrict__ gtab, int message_chunks, uint32_t* __restrict__ wide,
             const uint32_t* __restrict__ consts, KeyScalars ks) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int STRIDE = inst_stride_words<K>(1);
  extern __shared__ __align__(16) uint32_t smem[];
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;  // j * 65536 + D
  const int wide_chunks = (message_chunks + 1) / 2;
  if (inst >= (long long)wide_chunks * 65536) return;
  const int j = int(inst >> 16), D = int(inst & 65535);
  uint32_t* s_b = smem + slot * STRIDE;
  uint32_t n2[L], lo[L], hi[L], r[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(lo, gtab + ((long long)(2 * j) * 256 + (D & 255)) * K);
  if (2 * j + 1 < message_chunks) g.load_ro(hi, gtab + ((long long)(2 * j + 1) * 256 + (D >> 8)) * K);
  else g.load_ro(hi, consts + C_RM * K);
  g.publish(s_b, hi);
  g.mont_mul(r, lo, s_b, n2, ks.ninv2);
  g.store(wide + inst * K, r);
}

// The 16-bit-digit table in 52-bit limbs, R52 domain, one row j at a time:
// W[j][D] = G[2j][D mod 256] G[2j+1][D / 256] R52 mod n^2 from the 8-bit
// table (32-bit Montgomery form): one 32-bit product for the pair, one with
// R52 mod n^2 (r52w) into the R52 domain.
template <int K>
__global__ void __launch_bounds__(kBlockThreads)
k_wide_table52(const uint32_t* __restrict__ gtab, int message_chunks, int j, double* __restrict__ wide52,
               const uint32_t* __restrict__ consts, KeyScalars ks, const uint32_t* __restrict__ r52w) {
  constexpr int TPI = K / 16, L = 16, K52 = 5 * K / 8, L52 = K52 / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_r52 = smem;
  for (int i = threadIdx.x; i < K; i += blockDim.x) s_r52[i] = r52w[i];
  __syncthreads();
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const int D = blockIdx.x * IPB + slot;
  if (D >= 65536) return;
  uint32_t* s_b = smem + K + slot * K;
  uint32_t n2[L], lo[L], hi[L], p[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(lo, gtab + ((long long)(2 * j) * 256 + (D & 255)) * K);
  if (2 * j + 1 < message_chunks) g.load_ro(hi, gtab + ((long long)(2 * j + 1) * 256 + (D >> 8)) * K);
  else g.load_ro(hi, consts + C_RM * K);
  g.publish(s_b, hi);
  g.mont_mul(p, lo, s_b, n2, ks.ninv2);      // the pair, 32-bit Montgomery form
  g.mont_mul(lo, p, s_r52, n2, ks.ninv2);    // x R52 mod n^2
  g.publish(s_b, lo);
  double* o = wide52 + ((long long)j * 65536 + D) * K52;
#pragma unroll
  for (int k = 0; k < L52; ++k) o[g.gl * L52 + k] = cuhe52::to_f64(limb52_from_words(s_b, K, g.gl * L52 + k));
}

// Paillier-Lookup encryption with the 16-bit-digit table on the FP64 pipe
// (n^2 of 4096 / 8192 bits): the table and the noise entries as 52-bit limbs
// in the R52 domain, the product accumulated as in k_modexp52 (the next row
// loaded during each product), the result re-cut into words: the
// ciphertexts of k_lookup_encrypt.
template <int K>
__global__ void __launch_bounds__(kBlockThreads, 3)
k_lookup_encrypt52(const uint8_t* __restrict__ bits, int embed_len, int chunk_len, int chunk_num,
                   const uint32_t* __restrict__ plain, int plain_words, long long count, int message_chunks,
                   const double* __restrict__ wide52, const double* __restrict__ noise52, int noise_entries,
                   const uint8_t* __restrict__ noise_idx, uint32_t* __restrict__ out,
                   const double* __restrict__ n52, unsigned long long ninv52, int* status) {
  constexpr int TPI = K / 16, L = 16, K52 = 5 * K / 8, L52 = K52 / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  extern __shared__ __align__(16) double smd[];
  double* s_one52 = smd;         // 1
  double* s_accs = smd + K52;    // per instance: the accumulator (b operand), K52 + 2 doubles
  __shared__ int s_count[IPB];
  for (int i = threadIdx.x; i < K52; i += blockDim.x) s_one52[i] = i == 0 ? 1.0 : 0.0;
  __syncthreads();
  Group<K, TPI> g;
  cuhe52::Group52<K52, TPI> f;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;
  if (inst >= count) return;
  uint16_t* s_rows16 =
      reinterpret_cast<uint16_t*>(s_accs + IPB * (K52 + 2)) + slot * lookup_rows_stride(message_chunks);
  const uint32_t* s_rows32 = reinterpret_cast<const uint32_t*>(s_rows16);
  if (g.gl == 0)
    s_count[slot] = lookup_digit_rows<true>(bits, embed_len, chunk_len, chunk_num, plain, plain_words, inst,
                                            message_chunks, s_rows16);
  __syncwarp(f.mask);
  const int cnt = s_count[slot];
  double* s_b = s_accs + slot * (K52 + 2);
  double acc[L52], a[L52], nx[L52], m52[L52];
  auto load_row = [&](double (&v)[L52], const double* row) {
    const double2* r2 = reinterpret_cast<const double2*>(row + f.gl * L52);
#pragma unroll
    for (int k = 0; k < L52 / 2; ++k) {
      const double2 t = __ldg(r2 + k);
      v[2 * k] = t.x;
      v[2 * k + 1] = t.y;
    }
  };
#pragma unroll
  for (int k = 0; k < L52; ++k) {
    m52[k] = __ldg(n52 + f.gl * L52 + k);
    acc[k] = __ldg(n52 + K52 + f.gl * L52 + k);  // R52 mod n^2: one in the R52 domain
  }
  f.publish(s_b, acc);
  if (cnt > 0) load_row(a, wide52 + (long long)s_rows32[0] * K52);
#pragma unroll 1
  for (int j = 0; j < cnt; ++j) {
    if (j + 1 < cnt) load_row(nx, wide52 + (long long)s_rows32[j + 1] * K52);
    f.mont_mul(acc, a, s_b, m52, ninv52);
    f.publish(s_b, acc);
#pragma unroll
    for (int k = 0; k < L52; ++k) a[k] = nx[k];
  }
  const uint8_t* idx = noise_idx + inst * kNoiseMultiples;
#pragma unroll 1
  for (int k = 0; k < kNoiseMultiples; ++k) {
    const int r = idx[k];
    if (r >= noise_entries) {
      if (g.gl == 0) atomicOr(status, ST_RANGE);
      return;
    }
    load_row(a, noise52 + (long long)r * K52);
    f.mont_mul(acc, a, s_b, m52, ninv52);
    f.publish(s_b, acc);
  }
  double res[L52];
  f.mont_mul(res, acc, s_one52, m52, ninv52);  // canonical
  uint64_t* s_l = reinterpret_cast<uint64_t*>(s_b);
  __syncwarp(f.mask);
#pragma unroll
  for (int k = 0; k < L52; ++k) s_l[f.gl * L52 + k] = cuhe52::to_u64(res[k]);
  __syncwarp(f.mask);
  uint32_t w[L];
#pragma unroll
  for (int t = 0; t < L; ++t) w[t] = word_from_limbs52(s_l, K52, g.gl * L + t);
  g.store(out + inst * K, w);
}

// ---------------------------------------------------------------------------
// Fixed-base table construction: rows i of G = base_i^j, j = 0..255, with
// base_i = g^(2^(8i)) (all in Montgomery form).  One group per (row, chunk of
// 16 consecutive j); thread-level work is 16 sequential products.
// ---------------------------------------------------------------------------
template <int K, int TPI>
__global__ void __launch_bounds__(kBlockThreads)
k_table_rows(const uint32_t* __restrict__ bases_mont, int rows, uint32_t* __restrict__ gtab,
             const uint32_t* __restrict__ consts, KeyScalars ks) {
  constexpr int L = K / TPI;
  constexpr int IPB = kBlockThreads / TPI;
  constexpr int STRIDE = inst_stride_words<K>(2);
  extern __shared__ __align__(16) uint32_t smem[];
  Group<K, TPI> g;
  const int slot = threadIdx.x / TPI;
  const long long inst = (long long)blockIdx.x * IPB + slot;  // row * 16 + block of j
  if (inst >= (long long)rows * 16) return;
  const int row = int(inst / 16);
  const int jb = int(inst % 16);
  uint32_t* s_base = smem + slot * STRIDE;
  uint32_t* s_pow = s_base + K;
  uint32_t n2[L], b[L], p[L];
  g.load_ro(n2, consts + C_N2 * K);
  g.load_ro(b, bases_mont + (long long)row * K);
  g.publish(s_base, b);
  // p = base^(16*jb) via square-and-multiply over the 8-bit exponent
  g.load_ro(p, consts + C_RM * K);
  const int e = 16 * jb;
#pragma unroll 1
  for (int bit = 7; bit >= 0; --bit) {
    g.publish(s_pow, p);
    g.mont_mul(p, p, s_pow, n2, ks.ninv2);
    if ((e >> bit) & 1) g.mont_mul(p, p, s_base, n2, ks.ninv2);
  }
#pragma unroll 1
  for (int t = 0; t < 16; ++t) {
    g.store(gtab + ((long long)row * 256 + e + t) * K, p);
    g.mont_mul(p, p, s_base, n2, ks.ninv2);
  }
}

}  // namespace cuhe
