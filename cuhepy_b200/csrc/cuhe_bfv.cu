// C ABI of the BFV residue evaluator (see include/cuhe_bfv.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cuhe_bfv.h"
#include "../../include/cuhe_paillier.h"
#include "bfv_host.h"
#include "bfv_kernels.cuh"

using namespace cuhe::bfv;
namespace H = cuhe::bfv::host;

namespace {

thread_local std::string t_error;

int fail(int code, const std::string& msg) {
  t_error = msg;
  return code;
}

#define BFV_CUDA(call, where)                                                                 \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(CUHE_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorName(e_) + " (" +  \
                                       cudaGetErrorString(e_) + ")");                         \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Growable device workspace carved into aligned slices for one call.
// Tile batches of at least kSplitTiles tiles run as kSplitWays parts, each on
// its own stream.
constexpr int kSplitWays = 2;  // 3 and 4 parts measured the same
constexpr size_t kSplitTiles = 128;

struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  bool owned = true;  // false: a view of another arena's slice
  ~Arena() { if (base && owned) cudaFree(base); }
  cudaError_t reserve(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (base) cudaFree(base);
    base = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  bool overflow = false;
  void reset() { used = 0; overflow = false; }
  // Slices past the reserved capacity are never handed out: the call is
  // marked as overflowed and receives a null pointer, checked before launch.
  template <class T> T* take(size_t count) {
    const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (!base || used + bytes > cap) {
      overflow = true;
      return nullptr;
    }
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

// One execution lane of a ring: a stream, its device workspace and the lock
// that serialises calls on it.  Lane 0 serves every call except searches,
// which take a free lane among the active ones, so that searches issued from
// several host threads overlap on the GPU.
struct Lane {
  cudaStream_t stream = nullptr;
  Arena arena;
  std::mutex mu;
  uint8_t* host_stage = nullptr;  // pinned staging of host polynomials (grow-only)
  size_t host_cap = 0;
  cudaStream_t copy = nullptr;      // uploads overlapped with the lane's compute
  uint8_t* pin[2] = {nullptr, nullptr};  // their pinned double buffer
  size_t pin_cap[2] = {0, 0};
  u64* ks_scratch = nullptr;  // N = 32768 key switches: digit and accumulator planes (grow-only)
  size_t ks_scratch_bytes = 0;
  cudaStream_t side[kSplitWays - 1] = {};  // further compute streams of split tile batches
  ~Lane() {
    if (copy) cudaStreamSynchronize(copy);
    for (cudaStream_t st : side)
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    if (ks_scratch) cudaFree(ks_scratch);
    if (host_stage) cudaFreeHost(host_stage);
    for (uint8_t* p : pin)
      if (p) cudaFreeHost(p);
    if (copy) cudaStreamDestroy(copy);
  }
};

// Packed host polynomials of an index: one contiguous buffer, or one pointer
// per polynomial (two per tile), each poly_bytes long.
struct PolySource {
  const uint8_t* contiguous = nullptr;
  const uint8_t* const* parts = nullptr;
  size_t poly_bytes = 0;
  const uint8_t* poly(size_t k) const { return parts ? parts[k] : contiguous + k * poly_bytes; }
};

// Copy polys [first, first + count) of src into the lane's pinned staging
// buffer (several host threads for large copies) and enqueue one
// host-to-device copy to d_dst on the lane's stream.  The caller
// synchronises the stream before the lane stages again.
// Copy polys [first, first + count) of src to dst, with up to max_workers
// host threads (one per 2^shift bytes).
void copy_polys(const PolySource& src, size_t first, size_t count, uint8_t* dst, size_t max_workers,
                unsigned shift = 24) {
  const size_t bytes = count * src.poly_bytes;
  const size_t workers = std::min<size_t>(std::max<size_t>(1, bytes >> shift), max_workers);
  auto copy = [&](size_t lo, size_t hi) {
    for (size_t k = lo; k < hi; ++k) std::memcpy(dst + k * src.poly_bytes, src.poly(first + k), src.poly_bytes);
  };
  if (workers == 1) {
    copy(0, count);
    return;
  }
  std::vector<std::thread> pool;
  const size_t per = (count + workers - 1) / workers;
  for (size_t w = 0; w < workers; ++w) {
    const size_t lo = w * per, hi = std::min(count, lo + per);
    if (lo < hi) pool.emplace_back(copy, lo, hi);
  }
  for (auto& t : pool) t.join();
}

cudaError_t stage_polys(Lane& ln, const PolySource& src, size_t first, size_t count, uint8_t* d_dst) {
  const size_t bytes = count * src.poly_bytes;
  if (bytes == 0) return cudaSuccess;
  if (bytes > ln.host_cap) {
    if (ln.host_stage) cudaFreeHost(ln.host_stage);
    ln.host_stage = nullptr;
    ln.host_cap = 0;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&ln.host_stage), bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    ln.host_cap = bytes;
  }
  copy_polys(src, first, count, ln.host_stage, 8);
  return cudaMemcpyAsync(d_dst, ln.host_stage, bytes, cudaMemcpyHostToDevice, ln.stream);
}

// Index tiles per upload sub-batch of a search over a host-memory index.
constexpr size_t kPipeTiles = 256;

constexpr int kMaxLanes = 8;

#define BFV_ARENA(arena)                                                                  \
  do {                                                                                    \
    if ((arena).overflow) return fail(CUHE_OUT_OF_MEMORY, "internal workspace exhausted"); \
  } while (0)

size_t slice(size_t bytes) { return (bytes + 255) & ~size_t(255); }

}  // namespace

struct cuhe_bfv_ring {
  std::atomic<int> refs{1};
  int device = 0;
  H::RingPlan plan;
  bool residue = false, fast = false;
  unsigned kernel_level = 0;
  size_t switch_prime_count = 0;
  u64* d_tables = nullptr;
  size_t table_bytes = 0;
  NativeCrt* d_crt = nullptr;  // native rings: CRT constants per prime count
  RingDev host_dev{};
  std::map<u64, RingDev*> dev_for_t;  // t == 0: no scale constants
  struct PlainRing {             // batch encoding mod t: NTT tables and slot permutation
    RingDev* d = nullptr;
    u64* d_tables = nullptr;
    int32_t* d_perm = nullptr;
  };
  std::map<u64, PlainRing> plain_for_t;  // guarded by mu
  std::mutex mu;  // guards dev_for_t
  std::vector<std::unique_ptr<Lane>> lanes;  // kMaxLanes, created with the ring
  std::atomic<int> active_lanes{1};
  std::atomic<unsigned> next_lane{0};

  ~cuhe_bfv_ring() {
    DeviceGuard g(device);
    for (auto& ln : lanes)
      if (ln->stream) cudaStreamSynchronize(ln->stream);
    for (auto& kv : dev_for_t) cudaFree(kv.second);
    for (auto& kv : plain_for_t) {
      cudaFree(kv.second.d);
      cudaFree(kv.second.d_tables);
      cudaFree(kv.second.d_perm);
    }
    if (d_tables) cudaFree(d_tables);
    if (d_crt) cudaFree(d_crt);
    for (auto& ln : lanes)
      if (ln->stream) cudaStreamDestroy(ln->stream);
    lanes.clear();  // workspaces are freed while this device is current
  }
};

struct cuhe_bfv_key {
  std::atomic<int> refs{1};
  cuhe_bfv_ring* ring = nullptr;
  u64* d_key = nullptr;  // [D][2][L][N] NTT domain, then as many Shoup quotients
  u64* d_key_q = nullptr;
  size_t bytes = 0;
  ~cuhe_bfv_key() {
    if (d_key) {
      DeviceGuard g(ring->device);
      cudaFree(d_key);
    }
    cuhe_bfv_ring_release(ring);
  }
};

struct cuhe_bfv_server {
  std::atomic<int> refs{1};
  cuhe_bfv_ring* ring = nullptr;
  cuhe_bfv_key* relin = nullptr;
  std::map<u64, cuhe_bfv_key*> keys;
  size_t padded = 0, lanes = 0, capacity = 0;
  u64 t = 0;
  H::Big target;
  unsigned target_bits = 0;
  std::vector<u64> target_words;
  std::vector<u64> left, right;
  u64* d_full_mask = nullptr;  // [L][N] NTT domain
  u64* d_target = nullptr;
  std::map<size_t, u64*> partial_masks;
  size_t mask_primes = 0;  // primes of the prepared masks (L, or enough for N (q-1)(t-1) on native rings)
  RingDev* d_ring = nullptr;
  std::mutex mu;  // guards partial_masks and profile_ms
  double profile_ms[6] = {0, 0, 0, 0, 0, 0};
  ~cuhe_bfv_server() {
    {
      DeviceGuard g(ring->device);
      if (d_full_mask) cudaFree(d_full_mask);
      if (d_target) cudaFree(d_target);
      for (auto& kv : partial_masks) cudaFree(kv.second);
    }
    for (auto& kv : keys) cuhe_bfv_key_release(kv.second);
    cuhe_bfv_key_release(relin);
    cuhe_bfv_ring_release(ring);
  }
};

namespace {

unsigned log2u(size_t n) {
  unsigned l = 0;
  while ((size_t(1) << l) < n) ++l;
  return l;
}

// Scale constants (NativeScale) of a native ring for plaintext modulus t over
// its tensor primes.
void native_scale_constants(const H::RingPlan& P, u64 t, NativeScale& S) {
  const size_t T = P.tensor_count, W = (P.q_bits + 63) / 64;
  std::memset(&S, 0, sizeof(S));
  auto words = [&](const H::Big& a, u64* out, size_t count) {
    for (size_t k = 0; k < count; ++k) out[k] = k < a.w.size() ? a.w[k] : 0;
  };
  auto mod_q = [&](const H::Big& a) { return H::sub(a, H::mul(H::div(a, P.q), P.q)); };
  const H::Big r2 = H::shl(H::Big(1), 128);
  // num = A q + B: a = (A mod q) 2^128 mod q, f = floor(B 2^128 / q)
  auto split = [&](const H::Big& num, u64* a, u64* f) {
    const H::Big A = H::div(num, P.q);
    const H::Big B = H::sub(num, H::mul(A, P.q));
    words(mod_q(H::mul(mod_q(A), r2)), a, W);
    words(H::div(H::mul(B, r2), P.q), f, 2);
  };
  H::Big prod(1);
  for (size_t j = 0; j < T; ++j) prod = H::mul_small(prod, P.primes[j]);
  for (size_t j = 0; j < T; ++j) split(H::mul_small(H::div_small(prod, P.primes[j]), t), S.a[j], S.f[j]);
  split(H::mul_small(prod, t), S.ap, S.fp);
}

// Device copy of the ring constants; t != 0 adds the exact scale constants.
int device_ring(cuhe_bfv_ring* r, u64 t, RingDev** out) {
  std::lock_guard<std::mutex> lock(r->mu);
  auto it = r->dev_for_t.find(t);
  if (it != r->dev_for_t.end()) { *out = it->second; return CUHE_OK; }
  RingDev dev = r->host_dev;
  if (t && !r->residue && r->plan.q_bits >= 68) {
    try {
      native_scale_constants(r->plan, t, dev.nscale);
      dev.has_nscale = 1;
    } catch (const std::invalid_argument& e) {
      return fail(CUHE_INVALID_ARGUMENT, e.what());
    }
  }
  if (t && r->residue) {  // native rings scale with the CRT constants above
    H::RingPlan plan = r->plan;
    try {
      H::build_scale(plan, t);
    } catch (const std::invalid_argument& e) {
      return fail(CUHE_INVALID_ARGUMENT, e.what());
    }
    auto fill = [&](BaseDev& b, const H::ExactBase& h) {
      b.start = int(h.base.front());
      b.count = int(h.base.size());
      b.tstart = int(h.target.front());
      b.tcount = int(h.target.size());
      for (size_t j = 0; j < h.base.size(); ++j) {
        b.inv[j] = h.inv[j];
        b.inv_q[j] = h.inv_q[j];
        for (int w = 0; w < kCrtWordsDev; ++w) b.partial_words[j][w] = h.partial_words[j][size_t(w)];
      }
      for (size_t k = 0; k < h.target.size(); ++k) {
        b.product_mod_target[k] = h.product_mod_target[k];
        b.product_mod_target_q[k] = h.product_mod_target_q[k];
        for (size_t j = 0; j < h.base.size(); ++j) b.partial_mod_target[k][j] = h.partial_mod_target[k][j];
      }
      for (int w = 0; w < kCrtWordsDev; ++w) b.product_words[w] = h.product_words[size_t(w)];
    };
    fill(dev.q_to_b, plan.q_to_b);
    fill(dev.b_to_q, plan.b_to_q);
    for (size_t j = 0; j < plan.inv_q_mod_b.size(); ++j) {
      dev.inv_q_mod_b[j] = plan.inv_q_mod_b[j];
      dev.inv_q_mod_b_q[j] = plan.inv_q_mod_b_q[j];
    }
    for (size_t j = 0; j < plan.primes.size(); ++j) {
      dev.t_mod[j] = t % plan.primes[j];
      dev.t_mod_q[j] = H::shoup_quotient(dev.t_mod[j], plan.primes[j]);
    }
    dev.has_scale = 1;
    dev.t = t;
  }
  RingDev* d = nullptr;
  BFV_CUDA(cudaMalloc(&d, sizeof(RingDev)), "ring constants");
  BFV_CUDA(cudaMemcpy(d, &dev, sizeof(RingDev), cudaMemcpyHostToDevice), "ring constants");
  r->dev_for_t[t] = d;
  *out = d;
  return CUHE_OK;
}

// Batch-encoding tables for plaintext modulus t (prime, t = 1 mod 2N): the
// NTT tables of t in RingDev form (one prime) and the permutation taking
// slot j to the inverse transform's input position bitrev(order[j]), where
// order lists the evaluation points psi^(3^j) then psi^(-3^j) (the
// reference's batch layout, bfv/scheme.py:139-183).
int plain_ring(cuhe_bfv_ring* r, u64 t, cuhe_bfv_ring::PlainRing* out) {
  std::lock_guard<std::mutex> lock(r->mu);
  auto it = r->plain_for_t.find(t);
  if (it != r->plain_for_t.end()) { *out = it->second; return CUHE_OK; }
  const size_t n = r->plan.n;
  if (t < 3 || t >= (u64(1) << 32) || t % (2 * n) != 1 || !H::is_prime64(t))
    return fail(CUHE_INVALID_ARGUMENT, "plaintext modulus must be a prime below 2^32 with t = 1 mod 2N");
  const H::NTTTable tab = H::build_ntt(n, t);
  std::vector<u64> tables(4 * n);
  for (size_t i = 0; i < n; ++i) {
    tables[2 * i] = tab.fwd[i];
    tables[2 * i + 1] = tab.fwd_q[i];
    tables[2 * n + 2 * i] = tab.inv[i];
    tables[2 * n + 2 * i + 1] = tab.inv_q[i];
  }
  const unsigned logn = H::log2_exact(n);
  std::vector<int32_t> perm(n);
  u64 g = 1;
  for (size_t j = 0; j < n / 2; ++j) {
    const u64 e = g, e_neg = (2 * n - g) % (2 * n);
    perm[j] = int32_t(H::bitrev(size_t((e - 1) / 2), logn));
    perm[n / 2 + j] = int32_t(H::bitrev(size_t((e_neg - 1) / 2), logn));
    g = g * 3 % (2 * n);
  }
  RingDev dev;
  std::memset(&dev, 0, sizeof(dev));
  dev.n = int(n);
  dev.logn = int(logn);
  dev.primes = dev.residue = dev.tensor = 1;
  dev.prime[0] = H::make_prime(t);
  dev.n_inv[0] = tab.n_inv;
  dev.n_inv_q[0] = tab.n_inv_q;
  dev.last[0] = tab.last;
  dev.last_q[0] = tab.last_q;
  cuhe_bfv_ring::PlainRing pr;
  cudaError_t e = cudaMalloc(&pr.d_tables, tables.size() * 8);
  if (e == cudaSuccess) e = cudaMemcpy(pr.d_tables, tables.data(), tables.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    dev.fwd2[0] = reinterpret_cast<const ulonglong2*>(pr.d_tables);
    dev.inv2[0] = reinterpret_cast<const ulonglong2*>(pr.d_tables + 2 * n);
    e = cudaMalloc(&pr.d, sizeof(RingDev));
  }
  if (e == cudaSuccess) e = cudaMemcpy(pr.d, &dev, sizeof(RingDev), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&pr.d_perm, n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMemcpy(pr.d_perm, perm.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(pr.d);
    cudaFree(pr.d_tables);
    cudaFree(pr.d_perm);
    return fail(CUHE_CUDA_ERROR, std::string("plaintext tables: ") + cudaGetErrorString(e));
  }
  r->plain_for_t[t] = pr;
  *out = pr;
  return CUHE_OK;
}

// fixed-width little-endian coefficient bytes -> words, validated < q
int parse_polys(const cuhe_bfv_ring* r, const uint8_t* data, size_t polys, std::vector<u64>& words) {
  const auto& P = r->plan;
  const size_t n = P.n, cb = P.coefficient_bytes, W = size_t(r->host_dev.words);
  words.assign(polys * n * W, 0);
  for (size_t k = 0; k < polys * n; ++k) {
    const uint8_t* src = data + k * cb;
    u64* dst = words.data() + k * W;
    for (size_t b = 0; b < cb; ++b) dst[b / 8] |= u64(src[b]) << (8 * (b % 8));
    // compare with q
    int c = 0;
    for (size_t w = W; w-- > 0 && c == 0;) {
      const u64 qw = w < P.q.w.size() ? P.q.w[w] : 0;
      if (dst[w] != qw) c = dst[w] < qw ? -1 : 1;
    }
    if (c >= 0) return fail(CUHE_INVALID_ARGUMENT, "Noncanonical polynomial coefficient");
  }
  return CUHE_OK;
}

void words_to_bytes(const cuhe_bfv_ring* r, const std::vector<u64>& words, size_t polys, uint8_t* out) {
  const size_t n = r->plan.n, cb = r->plan.coefficient_bytes, W = size_t(r->host_dev.words);
  for (size_t k = 0; k < polys * n; ++k) {
    const u64* src = words.data() + k * W;
    for (size_t b = 0; b < cb; ++b) out[k * cb + b] = uint8_t(src[b / 8] >> (8 * (b % 8)));
  }
}

unsigned blocks_for(long long items, int threads) { return unsigned((items + threads - 1) / threads); }

size_t ntt_smem(const cuhe_bfv_ring* r) { return plane_smem_words(int(r->plan.n)) * sizeof(u64); }

// Largest CTA of an NTT launch at this radix: the radix-8 kernel k_ntt8 is
// compiled for 1024 threads; the radix-16 kernel k_ntt is bounded below 1024
// by its register use.
int ntt_max_threads(int radix_log = 4) {
  if (radix_log <= 3) return 1024;
  static int cached = 0;
  if (!cached) {
    cudaFuncAttributes attr{};
    cached = cudaFuncGetAttributes(&attr, k_ntt) == cudaSuccess ? attr.maxThreadsPerBlock / 32 * 32 : 256;
  }
  return cached;
}

// Default launch of an N-point transform: radix-8 passes, one block of eight
// per thread (at most 1024 threads).
// radix-8 CTA size: one 8-point block per thread up to 512 threads; at N =
// 8192 two 512-thread CTAs per SM (64 registers each) overlap one CTA's
// plane loads and barriers with the other's butterflies, which beats one
// 1024-thread CTA.  N = 16384 planes take a whole SM's shared memory alone.
int ntt_default_threads(size_t n) {
  return int(std::min<size_t>(n >= 16384 ? 1024 : 512, std::max<size_t>(32, n / 8)));
}

// Largest degree whose plane one CTA transforms in shared memory.
constexpr size_t kMaxPlaneN = 16384;

// Batched transforms of `planes` planes on `stream` (prime mapping of
// k_ntt8); N = 32768 runs as the cross stage plus two half-plane transforms.
// d may be a ring's or a plain ring's constants.  Shared-memory sizes are
// within the attributes set at ring creation.
cudaError_t ntt_planes(size_t n, cudaStream_t stream, RingDev* d, u64* data, long long planes, int prime_base,
                       int prime_mod, int prime_block, int inverse, int threads = 0, int radix_log = 3) {
  if (planes <= 0) return cudaSuccess;
  const size_t smem = plane_smem_words(int(std::min(n, kMaxPlaneN))) * sizeof(u64);
  if (n > kMaxPlaneN) {
    const unsigned cross = blocks_for(planes * (long long)(n / 2), 256);
    const int th = ntt_default_threads(n / 2);
    if (!inverse) {
      k_ntt_cross<false><<<cross, 256, 0, stream>>>(data, planes, d, prime_base, prime_mod, prime_block);
      k_ntt_half<false><<<unsigned(planes * 2), th, smem, stream>>>(data, d, prime_base, prime_mod, prime_block);
    } else {
      k_ntt_half<true><<<unsigned(planes * 2), th, smem, stream>>>(data, d, prime_base, prime_mod, prime_block);
      k_ntt_cross<true><<<cross, 256, 0, stream>>>(data, planes, d, prime_base, prime_mod, prime_block);
    }
    return cudaGetLastError();
  }
  if (threads == 0) threads = ntt_default_threads(n);
  if (radix_log <= 3)
    k_ntt8<<<unsigned(planes), threads, smem, stream>>>(data, d, prime_base, prime_mod, prime_block, inverse, radix_log);
  else
    k_ntt<<<unsigned(planes), threads, smem, stream>>>(data, d, prime_base, prime_mod, prime_block, inverse, radix_log);
  return cudaGetLastError();
}

cudaError_t launch_ntt(cuhe_bfv_ring* r, Lane& ln, RingDev* d, u64* data, long long planes, int prime_base, int prime_mod,
                       int prime_block, int inverse) {
  return ntt_planes(r->plan.n, ln.stream, d, data, planes, prime_base, prime_mod, prime_block, inverse);
}

// Compose ops then key-switch ops (one launch each).
// The unfused key switch over `scratch` (digit planes, NTTs, products,
// inverse NTTs, epilogue), `chunk` ops at a time: N = 32768, where no plane
// fits one CTA, and the small waves of a merge tree, where one CTA per
// (op, prime) would leave most SMs idle.
int switch_unfused(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const SwitchOp* d_sops, size_t ops, u64* scratch,
                   size_t chunk) {
  const auto& P = r->plan;
  const size_t n = P.n, L = r->residue ? P.residue_count : r->switch_prime_count, D = P.digits;
  const unsigned bx = blocks_for((long long)n, 256);
  for (size_t c0 = 0; c0 < ops; c0 += chunk) {
    const size_t cnt = std::min(chunk, ops - c0);
    u64* digits = scratch;
    u64* acc = scratch + cnt * L * D * n;
    k_ks_digits<<<dim3(bx, unsigned(cnt * L * D)), 256, 0, ln.stream>>>(d_sops + c0, int(L), digits, d);
    BFV_CUDA(ntt_planes(n, ln.stream, d, digits, (long long)(cnt * L * D), 0, int(L), int(D), 0), "digit ntt");
    k_ks_mac<<<dim3(bx, unsigned(cnt * 2 * L)), 256, 0, ln.stream>>>(d_sops + c0, int(L), digits, acc, d);
    BFV_CUDA(ntt_planes(n, ln.stream, d, acc, (long long)(cnt * 2 * L), 0, int(L), 1, 1), "switch intt");
    k_ks_finish<<<dim3(bx, unsigned(cnt * 2 * L)), 256, 0, ln.stream>>>(d_sops + c0, int(L), acc, d);
  }
  return CUHE_OK;
}

// Device bytes of the unfused key switch's scratch per op.
size_t unfused_bytes_per_op(const cuhe_bfv_ring* r) {
  const auto& P = r->plan;
  const size_t L = r->residue ? P.residue_count : r->switch_prime_count;
  return (L * P.digits + 2 * L) * P.n * sizeof(u64);
}

// Waves of at most this many (op, prime) pairs take the unfused key switch
// when the caller lends scratch.
constexpr size_t kSmallSwitchPairs = 148;

// Scratch bytes of the largest such wave.
size_t small_switch_bytes(const cuhe_bfv_ring* r) {
  const size_t L = r->residue ? r->plan.residue_count : r->switch_prime_count;
  return slice(std::max<size_t>(1, kSmallSwitchPairs / L) * unfused_bytes_per_op(r));
}

int run_switch(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const std::vector<ComposeOp>& cops, const std::vector<SwitchOp>& sops,
               ComposeOp* d_cops, SwitchOp* d_sops, Arena* small = nullptr) {
  const auto& P = r->plan;
  if (!cops.empty()) {
    BFV_CUDA(cudaMemcpyAsync(d_cops, cops.data(), cops.size() * sizeof(ComposeOp), cudaMemcpyHostToDevice, ln.stream),
             "compose ops");
    dim3 grid(blocks_for((long long)(P.n), 256), unsigned(cops.size()));
    const int L = int(P.residue_count);
    if (r->residue && r->host_dev.words == L) {
      switch (L) {
        case 1: k_compose<1><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 2: k_compose<2><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 3: k_compose<3><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 4: k_compose<4><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 5: k_compose<5><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 6: k_compose<6><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        case 7: k_compose<7><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
        default: k_compose<8><<<grid, 256, 0, ln.stream>>>(d_cops, d); break;
      }
    } else {
      k_compose<0><<<grid, 256, 0, ln.stream>>>(d_cops, d);
    }
    BFV_CUDA(cudaGetLastError(), "compose launch");
  }
  if (!sops.empty()) {
    BFV_CUDA(cudaMemcpyAsync(d_sops, sops.data(), sops.size() * sizeof(SwitchOp), cudaMemcpyHostToDevice, ln.stream),
             "switch ops");
    const size_t smem = ntt_smem(r);
    dim3 grid(unsigned(sops.size()), unsigned(r->residue ? P.residue_count : r->switch_prime_count));
    const size_t pairs = size_t(grid.x) * grid.y;
    const size_t small_need = slice(sops.size() * unfused_bytes_per_op(r));
    if (small && P.n <= kMaxPlaneN && pairs <= kSmallSwitchPairs && small->used + small_need <= small->cap) {
      // few ops: six times as many CTAs per op in the digit transforms
      u64* scratch = reinterpret_cast<u64*>(small->base + small->used);
      if (int rc = switch_unfused(r, ln, d, d_sops, sops.size(), scratch, sops.size())) return rc;
    } else if (P.n <= 8192) {
      // accumulators in tensor memory, two CTAs per SM (shared-memory size
      // within the attribute set at ring creation)
      k_keyswitch_tm<3><<<grid, 512, smem, ln.stream>>>(d_sops, d);
    } else if (P.n <= kMaxPlaneN) {
      // N = 16384: 32 coefficients per thread, the whole TMEM, one CTA per SM
      k_keyswitch_tm<3, 32><<<grid, 512, smem, ln.stream>>>(d_sops, d);
    } else {
      // N = 32768: no plane fits one CTA, so the switch runs unfused over
      // the lane's scratch, a bounded number of ops at a time
      const size_t per_op = unfused_bytes_per_op(r);
      const size_t L = r->residue ? P.residue_count : r->switch_prime_count;
      const size_t fit = std::max<size_t>(1, (size_t(768) << 20) / per_op);
      const size_t chunk = std::min({sops.size(), fit, size_t(65535) / (L * P.digits)});
      const size_t need = chunk * per_op;
      if (ln.ks_scratch_bytes < need) {
        if (ln.ks_scratch) {
          BFV_CUDA(cudaStreamSynchronize(ln.stream), "scratch drain");
          BFV_CUDA(cudaFree(ln.ks_scratch), "scratch free");
          ln.ks_scratch = nullptr;
          ln.ks_scratch_bytes = 0;
        }
        BFV_CUDA(cudaMalloc(&ln.ks_scratch, need), "key-switch scratch");
        ln.ks_scratch_bytes = need;
      }
      if (int rc = switch_unfused(r, ln, d, d_sops, sops.size(), ln.ks_scratch, chunk)) return rc;
    }
    BFV_CUDA(cudaGetLastError(), "keyswitch launch");
  }
  // op tables are reused by the next call; keep host order
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "switch synchronize");
  return CUHE_OK;
}

unsigned inverse_mod_2n(u64 g, size_t n) {
  // g odd, 2n a power of two: Newton's iteration x <- x (2 - g x) doubles
  // the correct low bits each step (1 -> 64 after six)
  u64 x = 1;
  for (int k = 0; k < 6; ++k) x *= 2 - g * x;
  return unsigned(x & (2 * u64(n) - 1));
}

// host words of a composed result (after k_compose) -> bytes
int download_words(cuhe_bfv_ring* r, Lane& ln, const u64* d_words, size_t polys, uint8_t* out) {
  std::vector<u64> words(polys * r->plan.n * size_t(r->host_dev.words));
  BFV_CUDA(cudaMemcpyAsync(words.data(), d_words, words.size() * 8, cudaMemcpyDeviceToHost, ln.stream), "download");
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "download");
  words_to_bytes(r, words, polys, out);
  return CUHE_OK;
}

// mask(count) of the Hamming server (bfv_server.h:80-99): the polynomial
// m(X) mod t with m(psi^{+-3^lane}) = 1 on the selected slots and 0 on the
// others, i.e. m_i = N^-1 * sum_{e in S} psi^(-e i) mod t.
std::vector<u64> hamming_mask(size_t n, u64 t, size_t lanes, size_t count) {
  u64 psi = 0;
  for (u64 c = 2;; ++c) {
    const u64 root = H::powmod(c, (t - 1) / (2 * n), t);
    if (H::powmod(root, n, t) == t - 1) { psi = root; break; }
  }
  const u64 psi_inv = H::powmod(psi, t - 2, t);
  std::vector<u64> exps;
  u64 g = 1;
  for (size_t lane = 0; lane < lanes; ++lane) {
    for (size_t row = 0; row < 2; ++row) {
      if (row * lanes + lane >= count) continue;
      exps.push_back(row ? 2 * n - g : g);
    }
    g = g * 3 % (2 * n);
  }
  std::vector<u64> m(n, 0);
  const u64 n_inv = H::powmod(n % t, t - 2, t);
  for (u64 e : exps) {
    const u64 step = H::powmod(psi_inv, e, t);  // psi^-e
    u64 w = 1;
    for (size_t i = 0; i < n; ++i) {
      m[i] = (m[i] + w) % t;
      w = u64(u128(w) * step % t);
    }
  }
  for (auto& v : m) v = u64(u128(v) * n_inv % t);
  return m;
}

// residues mod the first L primes of a small nonnegative polynomial, NTT'd
int upload_plain_ntt(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const std::vector<u64>& coeffs_words, u64** out,
                     size_t primes = 0) {
  const auto& P = r->plan;
  const size_t n = P.n, L = primes ? primes : P.residue_count, W = size_t(r->host_dev.words);
  u64* d_words = nullptr;
  u64* d_res = nullptr;
  BFV_CUDA(cudaMalloc(&d_words, n * W * 8), "plain alloc");
  BFV_CUDA(cudaMalloc(&d_res, L * n * 8), "plain alloc");
  BFV_CUDA(cudaMemcpyAsync(d_words, coeffs_words.data(), n * W * 8, cudaMemcpyHostToDevice, ln.stream), "plain");
  k_words_to_residues<<<blocks_for((long long)(n), 256), 256, 0, ln.stream>>>(d_words, 1, int(L), d_res, d);
  BFV_CUDA(cudaGetLastError(), "plain residues");
  BFV_CUDA(launch_ntt(r, ln, d, d_res, (long long)(L), 0, int(L), 1, 0), "plain ntt");
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "plain");
  cudaFree(d_words);
  *out = d_res;
  return CUHE_OK;
}

std::vector<u64> small_to_words(const std::vector<u64>& v, size_t W) {
  std::vector<u64> w(v.size() * W, 0);
  for (size_t i = 0; i < v.size(); ++i) w[i * W] = v[i];
  return w;
}

// Tile circuit for `ct` tiles resident as residues: tensor square of
// (query - tile) with exact scale, relinearization, the given rotations and
// the masks.  dist_out receives [ct][2][L][N] coefficient-domain residues.
struct TileArgs {
  const u64* q_words;   // [2][N][W]
  const u64* t_words;   // [ct][2][N][W]
  size_t ct;
  cuhe_bfv_key* relin;
  std::vector<u64> exps;                 // rotation exponents (1 = double)
  std::vector<cuhe_bfv_key*> keys;
  std::vector<const u64*> masks;         // per tile mask NTT [L][N]
};

int tile_circuit(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const TileArgs& a, u64* dist, double* ms) {
  const auto& P = r->plan;
  const size_t n = P.n, L = P.residue_count, T = P.tensor_count, W = size_t(r->host_dev.words);
  const size_t ct = a.ct;
  Arena& ar = ln.arena;
  u64* diff = ar.take<u64>(ct * 2 * T * n);
  u64* tens = ar.take<u64>(ct * 3 * T * n);
  u64* scaled = ar.take<u64>(ct * 3 * L * n);
  u64* words = ar.take<u64>(ct * n * W);
  u64* other = ar.take<u64>(ct * 2 * L * n);
  ComposeOp* d_cops = ar.take<ComposeOp>(ct);
  SwitchOp* d_sops = ar.take<SwitchOp>(ct);
  BFV_ARENA(ar);
  cudaEvent_t ev[5];
  for (auto& e : ev) cudaEventCreate(&e);
  cudaEventRecord(ev[0], ln.stream);
  k_diff_residues<<<blocks_for((long long)(ct * 2 * n), 256), 256, 0, ln.stream>>>(a.q_words, a.t_words, int(ct), int(T),
                                                                                    diff, d);
  BFV_CUDA(cudaGetLastError(), "diff residues");
  BFV_CUDA(launch_ntt(r, ln, d, diff, (long long)(ct * 2 * T), 0, int(T), 1, 0), "tensor ntt");
  k_tensor_square<<<blocks_for((long long)(ct * T * n), 256), 256, 0, ln.stream>>>(diff, int(ct), int(T), tens, d);
  BFV_CUDA(cudaGetLastError(), "tensor");
  BFV_CUDA(launch_ntt(r, ln, d, tens, (long long)(ct * 3 * T), 0, int(T), 1, 1), "tensor intt");
  k_rns_scale<<<blocks_for((long long)(ct * 3 * n), 128), 128, 0, ln.stream>>>(tens, (long long)(ct * 3), scaled, d);
  BFV_CUDA(cudaGetLastError(), "rns scale");
  cudaEventRecord(ev[1], ln.stream);
  // relinearize: dist = (c0, c1) + KS(c2)
  std::vector<ComposeOp> cops(ct);
  std::vector<SwitchOp> sops(ct);
  for (size_t t = 0; t < ct; ++t) {
    cops[t] = ComposeOp{scaled + (t * 3 + 2) * L * n, words + t * n * W, 1u, 0u};
    sops[t] = SwitchOp{scaled + t * 3 * L * n, nullptr, words + t * n * W, a.relin->d_key, a.relin->d_key_q,
                       dist + t * 2 * L * n, 1u, 0u};
  }
  if (int rc = run_switch(r, ln, d, cops, sops, d_cops, d_sops)) return rc;
  cudaEventRecord(ev[2], ln.stream);
  // rotations: dist += rotate(dist, g); the last one, when a key switch on
  // planes that fit one CTA, also applies the masks (its output is then
  // multiplied in the NTT domain before its single inverse transform)
  u64* cur = dist;
  u64* nxt = other;
  const bool fused_mask = !a.exps.empty() && a.exps.back() != 1 && n <= size_t(kMaxPlaneN);
  for (size_t k = 0; k < a.exps.size(); ++k) {
    const u64 g = a.exps[k];
    if (g == 1) {
      k_add<<<blocks_for((long long)(ct * 2 * L * n), 256), 256, 0, ln.stream>>>(cur, cur, nxt, (long long)(ct * 2 * L), int(L), d);
      BFV_CUDA(cudaGetLastError(), "double");
    } else {
      const unsigned ginv = inverse_mod_2n(g, n);
      const bool masked = fused_mask && k + 1 == a.exps.size();
      u64* target = masked ? cur : nxt;  // a masked switch may write in place
      for (size_t t = 0; t < ct; ++t) {
        cops[t] = ComposeOp{cur + (t * 2 + 1) * L * n, words + t * n * W, unsigned(g), 0u};
        sops[t] = SwitchOp{cur + t * 2 * L * n, cur + t * 2 * L * n, words + t * n * W, a.keys[k]->d_key,
                           a.keys[k]->d_key_q, target + t * 2 * L * n, ginv, 0u};
        if (masked) sops[t].mask = a.masks[t];
      }
      if (int rc = run_switch(r, ln, d, cops, sops, d_cops, d_sops)) return rc;
      if (masked) break;
    }
    std::swap(cur, nxt);
  }
  cudaEventRecord(ev[3], ln.stream);
  // masks in the NTT domain (unless the last rotation applied them)
  if (!fused_mask) {
    BFV_CUDA(launch_ntt(r, ln, d, cur, (long long)(ct * 2 * L), 0, int(L), 1, 0), "mask ntt");
    for (size_t t = 0; t < ct; ++t) {
      const u64* m = a.masks[t];
      size_t run = 1;
      while (t + run < ct && a.masks[t + run] == m) ++run;
      k_mul_plain<<<blocks_for((long long)(run * 2 * L * n), 256), 256, 0, ln.stream>>>(
          cur + t * 2 * L * n, (long long)(run * 2 * L), int(L), m, d);
      BFV_CUDA(cudaGetLastError(), "mask");
      t += run - 1;
    }
    BFV_CUDA(launch_ntt(r, ln, d, cur, (long long)(ct * 2 * L), 0, int(L), 1, 1), "mask intt");
  }
  if (cur != dist)
    BFV_CUDA(cudaMemcpyAsync(dist, cur, ct * 2 * L * n * 8, cudaMemcpyDeviceToDevice, ln.stream), "dist copy");
  cudaEventRecord(ev[4], ln.stream);
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "tile circuit");
  if (ms) {
    float x;
    cudaEventElapsedTime(&x, ev[0], ev[1]); ms[0] += x;
    cudaEventElapsedTime(&x, ev[1], ev[2]); ms[1] += x;
    cudaEventElapsedTime(&x, ev[2], ev[3]); ms[2] += x;
    cudaEventElapsedTime(&x, ev[3], ev[4]); ms[3] += x;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return CUHE_OK;
}

// CRT constants of the native reduction (NativeCrt) for every prime count
// 1 .. K of the ring's auxiliary primes.
std::vector<NativeCrt> native_crt_constants(const H::RingPlan& P) {
  const size_t K = P.primes.size(), W = (P.q_bits + 63) / 64;
  if (W > size_t(kMaxWords) || K > size_t(kMaxPrimes)) throw std::invalid_argument("native constants exceed limits");
  auto mod_q = [&](const H::Big& a) { return H::sub(a, H::mul(H::div(a, P.q), P.q)); };
  auto words = [&](const H::Big& a, u64* out, size_t count) {
    for (size_t k = 0; k < count; ++k) out[k] = k < a.w.size() ? a.w[k] : 0;
  };
  const H::Big r2 = H::shl(H::Big(1), 128);
  std::vector<NativeCrt> crt(K);
  H::Big prod(1);
  for (size_t c = 1; c <= K; ++c) {
    prod = H::mul_small(prod, P.primes[c - 1]);
    NativeCrt& C = crt[c - 1];
    std::memset(&C, 0, sizeof(C));
    for (size_t j = 0; j < c; ++j) {
      const u64 p = P.primes[j];
      const H::Big pj = H::div_small(prod, p);
      C.inv[j] = H::powmod(H::mod_small(pj, p), p - 2, p);
      C.inv_q[j] = H::shoup_quotient(C.inv[j], p);
      words(mod_q(H::mul(pj, r2)), C.c[j], W);
    }
    words(mod_q(H::mul(prod, r2)), C.pq, W);
    words(H::mul_small(P.q, u64(c)), C.cq, W + 1);
  }
  return crt;
}

size_t tile_arena_bytes(const cuhe_bfv_ring* r, size_t ct) {
  const auto& P = r->plan;
  const size_t n = P.n, L = P.residue_count, T = P.tensor_count, W = size_t(r->host_dev.words);
  return slice(ct * 2 * T * n * 8) + slice(ct * 3 * T * n * 8) + slice(ct * 3 * L * n * 8) + slice(ct * n * W * 8) +
         slice(ct * 2 * L * n * 8) + slice(ct * sizeof(ComposeOp)) + slice(ct * sizeof(SwitchOp));
}

// ---- native (prime q) rings: ciphertexts as words mod q --------------------------

size_t native_mask_primes(const cuhe_bfv_ring* r, u64 t) {
  // exact ct x pt product bound N (q - 1)(t - 1) (PreparedPlain, bfv_server.h:47-64)
  const auto& P = r->plan;
  const H::Big bound = H::mul_small(H::mul_small(H::sub(P.q, H::Big(1)), u64(P.n)), t - 1);
  return H::prime_count_for(P.primes, bound);
}

// finish (1, 2 accumulating; mode 0 with the certified tables only): the
// polys are the key switches of finish_ops, which are finished in the same
// pass (k_native_mod_q's epilogue) instead of being written to out.
int native_reduce(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const u64* res, size_t polys, size_t count, u64* out,
                  int mode, u64 t, const NativeOp* finish_ops = nullptr, int finish = 0) {
  if (!polys) return CUHE_OK;
  const unsigned blocks = blocks_for((long long)(polys * r->plan.n), 128);
  if (mode == 1 && r->d_crt && count == r->plan.tensor_count) {
    const bool narrow = count <= size_t(kNarrowWords);
#define CUHE_SCALE(KW)                                                                                         \
  case KW:                                                                                                     \
    if (narrow)                                                                                                \
      k_native_scale<KW, kNarrowWords><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, t, d); \
    else                                                                                                       \
      k_native_scale<KW, kWideWords><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, t, d);   \
    break;
    switch (r->host_dev.words) {
      CUHE_SCALE(1) CUHE_SCALE(2) CUHE_SCALE(3) CUHE_SCALE(4) CUHE_SCALE(5) CUHE_SCALE(6) CUHE_SCALE(7)
      default: CUHE_SCALE(8)
    }
#undef CUHE_SCALE
    BFV_CUDA(cudaGetLastError(), "native scale");
    return CUHE_OK;
  }
  if (mode == 0 && r->d_crt) {
    const bool narrow = count <= size_t(kNarrowWords);
#define CUHE_MOD_Q_F(KW, F)                                                                                 \
  if (narrow)                                                                                                   \
    k_native_mod_q<KW, kNarrowWords, F><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, d, \
                                                                       finish_ops);                             \
  else                                                                                                          \
    k_native_mod_q<KW, kWideWords, F><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, d,   \
                                                                     finish_ops);
#define CUHE_MOD_Q(KW)                  \
  case KW:                              \
    if (finish == 2) {                  \
      CUHE_MOD_Q_F(KW, 2)               \
    } else if (finish == 1) {           \
      CUHE_MOD_Q_F(KW, 1)               \
    } else {                            \
      CUHE_MOD_Q_F(KW, 0)               \
    }                                   \
    break;
    switch (r->host_dev.words) {
      CUHE_MOD_Q(1) CUHE_MOD_Q(2) CUHE_MOD_Q(3) CUHE_MOD_Q(4) CUHE_MOD_Q(5) CUHE_MOD_Q(6) CUHE_MOD_Q(7)
      default: CUHE_MOD_Q(8)
    }
#undef CUHE_MOD_Q
#undef CUHE_MOD_Q_F
    BFV_CUDA(cudaGetLastError(), "native reduce");
    return CUHE_OK;
  }
  if (finish) return fail(CUHE_INVALID_ARGUMENT, "finishing reduction needs the certified tables");
  if (count <= size_t(kNarrowWords))
    k_native_reduce<kNarrowWords><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, mode, t, d);
  else
    k_native_reduce<kWideWords><<<blocks, 128, 0, ln.stream>>>(res, (long long)polys, int(count), out, mode, t, d);
  BFV_CUDA(cudaGetLastError(), "native reduce");
  return CUHE_OK;
}

int words_addsub(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const u64* a, size_t a_stride, const u64* b,
                 size_t b_stride, u64* out, size_t out_stride, size_t units, int subtract) {
  if (!units) return CUHE_OK;
  k_words_addsub<<<blocks_for((long long)(units * r->plan.n), 256), 256, 0, ln.stream>>>(
      a, (long long)a_stride, b, (long long)b_stride, out, (long long)out_stride, (long long)units, subtract, d);
  BFV_CUDA(cudaGetLastError(), "words add/sub");
  return CUHE_OK;
}

// exact products of `polys` word polys with NTT-domain plains (`count`
// primes; masks[k] for poly k), reduced mod q into out (may alias words)
int native_mul_plain(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const u64* words, size_t polys,
                     const std::vector<const u64*>& masks, size_t count, u64* res, u64* out) {
  const size_t n = r->plan.n;
  k_words_to_residues<<<blocks_for((long long)(polys * n), 256), 256, 0, ln.stream>>>(words, (long long)polys,
                                                                                   int(count), res, d);
  BFV_CUDA(cudaGetLastError(), "residues");
  BFV_CUDA(launch_ntt(r, ln, d, res, (long long)(polys * count), 0, int(count), 1, 0), "ntt");
  for (size_t k = 0; k < polys;) {
    size_t run = 1;
    while (k + run < polys && masks[k + run] == masks[k]) ++run;
    k_mul_plain<<<blocks_for((long long)(run * count * n), 256), 256, 0, ln.stream>>>(
        res + k * count * n, (long long)(run * count), int(count), masks[k], d);
    BFV_CUDA(cudaGetLastError(), "product");
    k += run;
  }
  BFV_CUDA(launch_ntt(r, ln, d, res, (long long)(polys * count), 0, int(count), 1, 1), "intt");
  return native_reduce(r, ln, d, res, polys, count, out, 0, 0);
}

// key switches: out[k] = (key_k . digits(in[k])) mod q as two word polys
// ([ops][2][N][W]); res: [ops][2][S][N] scratch
int native_switch(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const std::vector<const u64*>& in,
                  const std::vector<const cuhe_bfv_key*>& keys, u64* res, u64* out, SwitchOp* d_sops,
                  Arena* small = nullptr, const NativeOp* finish_ops = nullptr, int finish = 0) {
  const size_t n = r->plan.n, S = r->switch_prime_count;
  std::vector<SwitchOp> sops(in.size());
  for (size_t k = 0; k < in.size(); ++k)
    sops[k] = SwitchOp{nullptr, nullptr, in[k], keys[k]->d_key, keys[k]->d_key_q, res + k * 2 * S * n, 1u, 0u};
  if (int rc = run_switch(r, ln, d, {}, sops, nullptr, d_sops, small)) return rc;
  return native_reduce(r, ln, d, res, in.size() * 2, S, out, 0, 0, finish_ops, finish);
}

// rotations of word ciphertexts by g: ops[k].out = (sigma(c0) + KS(sigma(c1))_0,
// KS(sigma(c1))_1) for ops[k].in, with ops[k].perm and ops[k].ks as
// per-ciphertext scratch (two word polys each); d_ops, res and ks_all sized
// for ops.size()
int native_rotate(cuhe_bfv_ring* r, Lane& ln, RingDev* d, std::vector<NativeOp> ops, unsigned g,
                  const cuhe_bfv_key* key, NativeOp* d_ops, u64* res, u64* ks_all, SwitchOp* d_sops,
                  Arena* small = nullptr, bool accumulate = false) {
  const size_t n = r->plan.n, W = size_t(r->host_dev.words);
  if (ops.empty()) return CUHE_OK;
  for (size_t k = 0; k < ops.size(); ++k) ops[k].ks = ks_all + k * 2 * n * W;
  BFV_CUDA(cudaMemcpyAsync(d_ops, ops.data(), ops.size() * sizeof(NativeOp), cudaMemcpyHostToDevice, ln.stream),
           "rotation ops");
  dim3 grid(blocks_for((long long)(2 * n), 256), unsigned(ops.size()));
  k_native_permute<<<grid, 256, 0, ln.stream>>>(d_ops, g, d);
  BFV_CUDA(cudaGetLastError(), "automorphism");
  std::vector<const u64*> c1(ops.size());
  std::vector<const cuhe_bfv_key*> keys(ops.size(), key);
  for (size_t k = 0; k < ops.size(); ++k) c1[k] = ops[k].perm + n * W;
  if (r->d_crt) {
    // the reduction mod q finishes the rotation in the same pass
    return native_switch(r, ln, d, c1, keys, res, ks_all, d_sops, small, d_ops, accumulate ? 2 : 1);
  }
  if (int rc = native_switch(r, ln, d, c1, keys, res, ks_all, d_sops, small)) return rc;
  if (accumulate) k_native_finish<true><<<grid, 256, 0, ln.stream>>>(d_ops, d);
  else k_native_finish<false><<<grid, 256, 0, ln.stream>>>(d_ops, d);
  BFV_CUDA(cudaGetLastError(), "rotation finish");
  return CUHE_OK;
}

int native_add_ops(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const std::vector<NativeOp>& ops, NativeOp* d_ops) {
  if (ops.empty()) return CUHE_OK;
  BFV_CUDA(cudaMemcpyAsync(d_ops, ops.data(), ops.size() * sizeof(NativeOp), cudaMemcpyHostToDevice, ln.stream),
           "add ops");
  dim3 grid(blocks_for((long long)(2 * r->plan.n), 256), unsigned(ops.size()));
  k_native_add<<<grid, 256, 0, ln.stream>>>(d_ops, d);
  BFV_CUDA(cudaGetLastError(), "add");
  return CUHE_OK;
}

// The Hamming tile circuit on word ciphertexts (distance_tile,
// rns_ntt.h:672-700): (q - t)^2 scaled, relinearised, rotated and summed,
// masked.  dist: [ct][2][N][W].
struct NativeScratch {
  u64 *diff, *dres, *tens, *words3, *ksres, *ksw, *perm, *tmp, *mres;
  SwitchOp* d_sops;
  NativeOp* d_nops;
};

size_t native_tile_bytes(const cuhe_bfv_ring* r, size_t ct, size_t mask_primes) {
  const auto& P = r->plan;
  const size_t n = P.n, T = P.tensor_count, S = r->switch_prime_count, W = size_t(r->host_dev.words);
  return slice(ct * 2 * n * W * 8) + slice(ct * 2 * T * n * 8) + slice(ct * 3 * T * n * 8) +
         slice(ct * 3 * n * W * 8) + slice(ct * 2 * S * n * 8) + 3 * slice(ct * 2 * n * W * 8) +
         slice(ct * 2 * mask_primes * n * 8) + slice(ct * sizeof(SwitchOp)) + slice(ct * sizeof(NativeOp)) + 4096;
}

int native_scratch(Arena& ar, const cuhe_bfv_ring* r, size_t ct, size_t mask_primes, NativeScratch* s) {
  const auto& P = r->plan;
  const size_t n = P.n, T = P.tensor_count, S = r->switch_prime_count, W = size_t(r->host_dev.words);
  s->diff = ar.take<u64>(ct * 2 * n * W);
  s->dres = ar.take<u64>(ct * 2 * T * n);
  s->tens = ar.take<u64>(ct * 3 * T * n);
  s->words3 = ar.take<u64>(ct * 3 * n * W);
  s->ksres = ar.take<u64>(ct * 2 * S * n);
  s->ksw = ar.take<u64>(ct * 2 * n * W);
  s->perm = ar.take<u64>(ct * 2 * n * W);
  s->tmp = ar.take<u64>(ct * 2 * n * W);
  s->mres = ar.take<u64>(ct * 2 * mask_primes * n);
  s->d_sops = ar.take<SwitchOp>(std::max<size_t>(1, ct));
  s->d_nops = ar.take<NativeOp>(std::max<size_t>(1, ct));
  BFV_ARENA(ar);
  return CUHE_OK;
}

int native_tile_circuit(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const u64* qw, const u64* tw, size_t ct, u64 t,
                        const cuhe_bfv_key* relin, const std::vector<u64>& exps,
                        const std::vector<const cuhe_bfv_key*>& keys, const std::vector<const u64*>& masks,
                        size_t mask_primes, const NativeScratch& s, u64* dist, double* ms) {
  const auto& P = r->plan;
  const size_t n = P.n, T = P.tensor_count, W = size_t(r->host_dev.words);
  cudaEvent_t ev[5];
  for (auto& e : ev) cudaEventCreate(&e);
  cudaEventRecord(ev[0], ln.stream);
  for (size_t c = 0; c < 2; ++c)
    if (int rc = words_addsub(r, ln, d, qw + c * n * W, 0, tw + c * n * W, 2 * n, s.diff + c * n * W, 2 * n, ct, 1))
      return rc;
  k_words_to_residues<<<blocks_for((long long)(ct * 2 * n), 256), 256, 0, ln.stream>>>(s.diff, (long long)(ct * 2),
                                                                                       int(T), s.dres, d);
  BFV_CUDA(cudaGetLastError(), "tensor residues");
  BFV_CUDA(launch_ntt(r, ln, d, s.dres, (long long)(ct * 2 * T), 0, int(T), 1, 0), "tensor ntt");
  k_tensor_square<<<blocks_for((long long)(ct * T * n), 256), 256, 0, ln.stream>>>(s.dres, int(ct), int(T), s.tens, d);
  BFV_CUDA(cudaGetLastError(), "tensor");
  BFV_CUDA(launch_ntt(r, ln, d, s.tens, (long long)(ct * 3 * T), 0, int(T), 1, 1), "tensor intt");
  if (int rc = native_reduce(r, ln, d, s.tens, ct * 3, T, s.words3, 1, t)) return rc;
  cudaEventRecord(ev[1], ln.stream);
  // relinearise: dist = KS(p2) + (p0, p1)
  std::vector<const u64*> p2(ct);
  std::vector<const cuhe_bfv_key*> rk(ct, relin);
  for (size_t k = 0; k < ct; ++k) p2[k] = s.words3 + (k * 3 + 2) * n * W;
  if (int rc = native_switch(r, ln, d, p2, rk, s.ksres, s.ksw, s.d_sops)) return rc;
  for (size_t c = 0; c < 2; ++c)
    if (int rc = words_addsub(r, ln, d, s.ksw + c * n * W, 2 * n, s.words3 + c * n * W, 3 * n, dist + c * n * W,
                              2 * n, ct, 0))
      return rc;
  cudaEventRecord(ev[2], ln.stream);
  // rotations: dist += rotate(dist, g)
  for (size_t e = 0; e < exps.size(); ++e) {
    if (exps[e] == 1) {
      if (int rc = words_addsub(r, ln, d, dist, n, dist, n, dist, n, ct * 2, 0)) return rc;
      continue;
    }
    // the finish adds the rotation into dist in place
    std::vector<NativeOp> ops(ct);
    for (size_t k = 0; k < ct; ++k)
      ops[k] = NativeOp{dist + k * 2 * n * W, s.perm + k * 2 * n * W, dist + k * 2 * n * W, nullptr};
    if (int rc = native_rotate(r, ln, d, ops, unsigned(exps[e]), keys[e], s.d_nops, s.ksres, s.ksw, s.d_sops,
                               nullptr, true))
      return rc;
  }
  cudaEventRecord(ev[3], ln.stream);
  std::vector<const u64*> pm(ct * 2);
  for (size_t k = 0; k < ct * 2; ++k) pm[k] = masks[k / 2];
  if (int rc = native_mul_plain(r, ln, d, dist, ct * 2, pm, mask_primes, s.mres, dist)) return rc;
  cudaEventRecord(ev[4], ln.stream);
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "native tile circuit");
  if (ms) {
    float x;
    cudaEventElapsedTime(&x, ev[0], ev[1]); ms[0] += x;
    cudaEventElapsedTime(&x, ev[1], ev[2]); ms[1] += x;
    cudaEventElapsedTime(&x, ev[2], ev[3]); ms[2] += x;
    cudaEventElapsedTime(&x, ev[3], ev[4]); ms[3] += x;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return CUHE_OK;
}

}  // namespace

extern "C" {

const char* cuhe_bfv_last_error(void) { return t_error.c_str(); }

int cuhe_bfv_create_ring(uint64_t n, const char* q_hex, uint64_t digit_bits, int fast, int residue,
                         uint64_t kernel_level, int device, cuhe_bfv_ring** out) {
  if (!out || !q_hex) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  const size_t len = std::strlen(q_hex);
  if (n > 32768 || digit_bits > 512 || kernel_level > 2)
    return fail(CUHE_INVALID_ARGUMENT, "Invalid native BFV ring parameters or kernel level");
  if (len < 1 || len > 128 || (len > 1 && q_hex[0] == '0'))
    return fail(CUHE_INVALID_ARGUMENT, "Invalid or oversized native modulus encoding");
  if (kernel_level && !residue)
    return fail(CUHE_INVALID_ARGUMENT,
                "Kernel level must be 0..2, with nonzero levels requiring the residue backend");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(CUHE_CUDA_ERROR, "no CUDA device available");
  }
  if (device < 0 || device >= count) return fail(CUHE_INVALID_ARGUMENT, "invalid device ordinal");
  auto* r = new (std::nothrow) cuhe_bfv_ring();
  if (!r) return fail(CUHE_OUT_OF_MEMORY, "ring allocation");
  try {
    const H::Big q = H::from_hex(q_hex);
    r->plan = H::build_ring(size_t(n), q, unsigned(digit_bits), residue != 0);

    if (r->plan.primes.size() > size_t(kMaxPrimes)) throw std::invalid_argument("too many auxiliary primes");
    if (!residue) {
      const H::Big qm1 = H::sub(q, H::Big(1));
      const H::Big sb = H::mul(H::mul_small(H::Big(u64(n)), u64(r->plan.digits)),
                               H::mul(H::sub(H::shl(H::Big(1), size_t(digit_bits)), H::Big(1)), qm1));
      r->switch_prime_count = H::prime_count_for(r->plan.primes, sb);
      if (r->plan.tensor_count > size_t(kMaxPrimes) || r->switch_prime_count > size_t(kMaxPrimes))
        throw std::invalid_argument("native ring needs more auxiliary primes than the B200 evaluator holds");
    } else {
      r->switch_prime_count = r->plan.residue_count;
    }
  } catch (const std::invalid_argument& e) {
    delete r;
    return fail(CUHE_INVALID_ARGUMENT, e.what());
  }
  r->device = device;
  r->residue = residue != 0;
  r->fast = fast != 0;
  r->kernel_level = unsigned(kernel_level);
  DeviceGuard guard(device);
  const auto& P = r->plan;
  const size_t K = P.primes.size(), N = P.n;
  r->table_bytes = K * 4 * N * 8;
  // per prime: forward (w, w_shoup) pairs, then inverse pairs
  std::vector<u64> tables(K * 4 * N);
  for (size_t j = 0; j < K; ++j) {
    u64* f = &tables[(j * 4 + 0) * N];
    u64* v = &tables[(j * 4 + 2) * N];
    for (size_t i = 0; i < N; ++i) {
      f[2 * i] = P.ntt[j].fwd[i];
      f[2 * i + 1] = P.ntt[j].fwd_q[i];
      v[2 * i] = P.ntt[j].inv[i];
      v[2 * i + 1] = P.ntt[j].inv_q[i];
    }
  }
  // Lane streams take the device's highest priority: a search is a chain of
  // short dependent kernels, and its blocks should be scheduled ahead of the
  // queued blocks of bulk work (Paillier batches) on default-priority streams.
  int least_priority = 0, greatest_priority = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least_priority, &greatest_priority);
  for (int k = 0; k < kMaxLanes && e == cudaSuccess; ++k) {
    r->lanes.push_back(std::make_unique<Lane>());
    e = cudaStreamCreateWithPriority(&r->lanes.back()->stream, cudaStreamNonBlocking, greatest_priority);
  }
  if (e == cudaSuccess) e = cudaMalloc(&r->d_tables, r->table_bytes);
  if (e == cudaSuccess) e = cudaMemcpy(r->d_tables, tables.data(), r->table_bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    delete r;
    return fail(CUHE_CUDA_ERROR, std::string("ring setup: ") + cudaGetErrorString(e));
  }
  RingDev& dev = r->host_dev;
  std::memset(&dev, 0, sizeof(dev));
  dev.n = int(N);
  dev.logn = int(log2u(N));
  dev.primes = int(K);
  dev.residue = int(P.residue_count);
  dev.tensor = int(P.tensor_count);
  dev.digits = int(P.digits);
  dev.digit_bits = int(P.digit_bits);
  dev.words = int((P.q_bits + 63) / 64);
  for (size_t j = 0; j < K; ++j) {
    dev.prime[j] = H::make_prime(P.primes[j]);
    dev.fwd2[j] = reinterpret_cast<const ulonglong2*>(r->d_tables + (j * 4 + 0) * N);
    dev.inv2[j] = reinterpret_cast<const ulonglong2*>(r->d_tables + (j * 4 + 2) * N);
    dev.n_inv[j] = P.ntt[j].n_inv;
    dev.n_inv_q[j] = P.ntt[j].n_inv_q;
    dev.last[j] = P.ntt[j].last;
    dev.last_q[j] = P.ntt[j].last_q;
    u64 pw = 1 % P.primes[j];
    const u64 two64 = u64((u128(1) << 64) % P.primes[j]);
    for (int w = 0; w < kMaxWords; ++w) {
      dev.pow64_mod[j][w] = pw;
      pw = u64(u128(pw) * two64 % P.primes[j]);
    }
  }
  for (size_t j = 0; j < P.garner_inv.size() && j < size_t(kMaxPrimes); ++j)
    for (size_t k = 0; k < j; ++k) {
      dev.garner[j][k] = P.garner_inv[j][k];
      dev.garner_q[j][k] = P.garner_inv_q[j][k];
    }
  // native rings: key switches run over the switch primes
  if (!r->residue) dev.residue = int(r->switch_prime_count);
  for (size_t w = 0; w < P.q.w.size() && w < size_t(kMaxWords); ++w) dev.q_words[w] = P.q.w[w];
  if (!r->residue) {
    std::vector<NativeCrt> crt;
    try {
      crt = native_crt_constants(P);
    } catch (const std::invalid_argument& ex) {
      delete r;
      return fail(CUHE_INVALID_ARGUMENT, ex.what());
    }
    cudaError_t ce = cudaMalloc(&r->d_crt, crt.size() * sizeof(NativeCrt));
    if (ce == cudaSuccess)
      ce = cudaMemcpy(r->d_crt, crt.data(), crt.size() * sizeof(NativeCrt), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) {
      delete r;
      return fail(CUHE_CUDA_ERROR, std::string("native constants: ") + cudaGetErrorString(ce));
    }
    dev.crt = r->d_crt;
    u64 inv = 1;  // q^-1 mod 2^64 by Newton's iteration (q odd)
    for (int k = 0; k < 6; ++k) inv *= 2 - P.q.w[0] * inv;
    dev.q_ninv = u64(0) - inv;
  }
  RingDev* dummy = nullptr;
  if (int rc = device_ring(r, 0, &dummy)) {
    delete r;
    return rc;
  }
  // the NTT kernels' shared-memory size for the largest supported plane,
  // once, so that later launches need no attribute call (they may run under
  // stream capture)
  e = cudaFuncSetAttribute(k_ntt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(plane_smem_words(16384) * sizeof(u64)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ntt8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(plane_smem_words(16384) * sizeof(u64)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_keyswitch_tm<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(plane_smem_words(8192) * sizeof(u64)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_keyswitch_tm<3, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(plane_smem_words(16384) * sizeof(u64)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ntt_half<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(plane_smem_words(16384) * sizeof(u64)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_ntt_half<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(plane_smem_words(16384) * sizeof(u64)));

  if (e != cudaSuccess) {
    delete r;
    return fail(CUHE_CUDA_ERROR, std::string("ring setup: ") + cudaGetErrorString(e));
  }
  *out = r;
  return CUHE_OK;
}

int cuhe_bfv_ntt(cuhe_bfv_ring* r, uint64_t* planes_dev, uint64_t planes, int primes, int inverse, int threads,
                 int radix_log, void* stream) {
  if (!r || (planes && !planes_dev)) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  const auto& P = r->plan;
  if (primes < 1 || size_t(primes) > P.primes.size())
    return fail(CUHE_INVALID_ARGUMENT, "prime count outside the ring's primes");
  if (radix_log == 0) radix_log = 3;
  if (radix_log < 1 || radix_log > 4) return fail(CUHE_INVALID_ARGUMENT, "radix_log must be 1..4");
  if (threads == 0) threads = std::min(ntt_default_threads(P.n), ntt_max_threads(radix_log));
  if (threads < 32 || threads > ntt_max_threads(radix_log) || threads % 32)
    return fail(CUHE_INVALID_ARGUMENT, "threads must be a multiple of 32 from 32 to " +
                                           std::to_string(ntt_max_threads(radix_log)) + " at this radix");
  if (planes == 0) return CUHE_OK;
  if (planes > (uint64_t(1) << 31) - 1) return fail(CUHE_INVALID_ARGUMENT, "too many planes for one launch");
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, 0, &d)) return rc;
  BFV_CUDA(ntt_planes(P.n, static_cast<cudaStream_t>(stream), d, reinterpret_cast<u64*>(planes_dev), (long long)planes,
                      0, primes, 1, inverse ? 1 : 0, threads, radix_log),
           "ntt launch");
  return CUHE_OK;
}

void cuhe_bfv_ring_release(cuhe_bfv_ring* ring) {
  if (ring && --ring->refs == 0) delete ring;
}

int cuhe_bfv_ring_info(const cuhe_bfv_ring* ring, uint64_t* primes, int capacity, int* prime_count,
                       int* switch_prime_count, int* residue_prime_count, uint64_t* table_bytes,
                       uint64_t* coefficient_bytes, int* kernel_level, int* fast) {
  if (!ring) return fail(CUHE_INVALID_ARGUMENT, "null ring");
  const auto& P = ring->plan;
  for (int i = 0; i < capacity && size_t(i) < P.primes.size(); ++i) primes[i] = P.primes[size_t(i)];
  if (prime_count) *prime_count = int(P.primes.size());
  if (switch_prime_count) *switch_prime_count = int(ring->switch_prime_count);
  if (residue_prime_count) *residue_prime_count = ring->residue ? int(P.residue_count) : 0;
  if (table_bytes) *table_bytes = ring->table_bytes;
  if (coefficient_bytes) *coefficient_bytes = P.coefficient_bytes;
  if (kernel_level) *kernel_level = int(ring->kernel_level);
  if (fast) *fast = ring->fast ? 1 : 0;
  return CUHE_OK;
}

int cuhe_bfv_compile_key(cuhe_bfv_ring* ring, const uint8_t* key_polys, uint64_t digits, cuhe_bfv_key** out) {
  if (!ring || !key_polys || !out) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  const auto& P = ring->plan;
  if (digits != P.digits) return fail(CUHE_INVALID_ARGUMENT, "Incorrect gadget digit count");
  Lane& ln = *ring->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(ring->device);
  std::vector<u64> words;
  if (int rc = parse_polys(ring, key_polys, size_t(2 * digits), words)) return rc;
  // residue rings: keys over the L primes of Q; native rings: over the switch primes
  const size_t n = P.n, L = ring->residue ? P.residue_count : ring->switch_prime_count;
  auto* key = new (std::nothrow) cuhe_bfv_key();
  if (!key) return fail(CUHE_OUT_OF_MEMORY, "key allocation");
  key->ring = ring;
  ++ring->refs;
  key->bytes = 2 * size_t(digits) * 2 * L * n * 8;  // residues + Shoup quotients
  RingDev* d = nullptr;
  int rc = device_ring(ring, 0, &d);
  u64* d_words = nullptr;
  cudaError_t e = cudaSuccess;
  if (!rc) e = cudaMalloc(&key->d_key, key->bytes);
  if (!rc && e == cudaSuccess) e = cudaMalloc(&d_words, words.size() * 8);
  if (!rc && e == cudaSuccess)
    e = cudaMemcpyAsync(d_words, words.data(), words.size() * 8, cudaMemcpyHostToDevice, ln.stream);
  if (!rc && e == cudaSuccess) {
    // layout: [digit][component][prime][N] == residues of polys in order b_0, a_0, b_1, ...
    k_words_to_residues<<<blocks_for((long long)(2 * digits * n), 256), 256, 0, ln.stream>>>(
        d_words, (long long)(2 * digits), int(L), key->d_key, d);
    e = cudaGetLastError();
  }
  if (!rc && e == cudaSuccess) e = launch_ntt(ring, ln, d, key->d_key, (long long)(2 * digits * L), 0, int(L), 1, 0);
  if (!rc && e == cudaSuccess) {
    key->d_key_q = key->d_key + size_t(digits) * 2 * L * n;
    k_shoup_quotients<<<blocks_for((long long)(2 * digits * L * n), 256), 256, 0, ln.stream>>>(
        key->d_key, key->d_key_q, (long long)(2 * digits * L), int(L), d);
    e = cudaGetLastError();
  }
  if (!rc && e == cudaSuccess) e = cudaStreamSynchronize(ln.stream);
  if (d_words) cudaFree(d_words);
  if (rc || e != cudaSuccess) {
    cuhe_bfv_key_release(key);
    return rc ? rc : fail(CUHE_CUDA_ERROR, std::string("compile_key: ") + cudaGetErrorString(e));
  }
  *out = key;
  return CUHE_OK;
}

void cuhe_bfv_key_release(cuhe_bfv_key* key) {
  if (key && --key->refs == 0) delete key;
}

uint64_t cuhe_bfv_key_bytes(const cuhe_bfv_key* key) { return key ? key->bytes : 0; }

namespace {

// upload fixed-width polys as words and residues (mod the first `primes` primes)
int upload_polys(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const uint8_t* data, size_t polys, size_t primes, u64** d_words,
                 u64** d_res) {
  std::vector<u64> words;
  if (int rc = parse_polys(r, data, polys, words)) return rc;
  const size_t n = r->plan.n;
  *d_words = ln.arena.take<u64>(words.size());
  BFV_ARENA(ln.arena);
  BFV_CUDA(cudaMemcpyAsync(*d_words, words.data(), words.size() * 8, cudaMemcpyHostToDevice, ln.stream), "upload");
  if (d_res) {
    *d_res = ln.arena.take<u64>(polys * primes * n);
    BFV_ARENA(ln.arena);
    k_words_to_residues<<<blocks_for((long long)(polys * n), 256), 256, 0, ln.stream>>>(*d_words, (long long)(polys),
                                                                                        int(primes), *d_res, d);
    BFV_CUDA(cudaGetLastError(), "residues");
  }
  BFV_CUDA(cudaStreamSynchronize(ln.stream), "upload");
  return CUHE_OK;
}

int compose_out(cuhe_bfv_ring* r, Lane& ln, RingDev* d, const u64* res, size_t polys, uint8_t* out) {
  const size_t n = r->plan.n, L = r->plan.residue_count, W = size_t(r->host_dev.words);
  u64* words = ln.arena.take<u64>(polys * n * W);
  ComposeOp* d_cops = ln.arena.take<ComposeOp>(polys);
  BFV_ARENA(ln.arena);
  std::vector<ComposeOp> cops(polys);
  for (size_t k = 0; k < polys; ++k) cops[k] = ComposeOp{res + k * L * n, words + k * n * W, 1u, 0u};
  if (int rc = run_switch(r, ln, d, cops, {}, d_cops, nullptr)) return rc;
  return download_words(r, ln, words, polys, out);
}

}  // namespace

int cuhe_bfv_apply_key(cuhe_bfv_key* key, const uint8_t* poly, uint8_t* out) {
  if (!key || !poly || !out) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  cuhe_bfv_ring* r = key->ring;
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, 0, &d)) return rc;
  const size_t n = r->plan.n, L = r->plan.residue_count, W = size_t(r->host_dev.words);
  if (!r->residue) {
    const size_t S = r->switch_prime_count;
    BFV_CUDA(ln.arena.reserve(slice(n * W * 8) * 4 + slice(2 * S * n * 8) + 4096), "workspace");
    ln.arena.reset();
    u64* words = nullptr;
    if (int rc = upload_polys(r, ln, d, poly, 1, 0, &words, nullptr)) return rc;
    u64* res = ln.arena.take<u64>(2 * S * n);
    u64* outw = ln.arena.take<u64>(2 * n * W);
    SwitchOp* d_sops = ln.arena.take<SwitchOp>(1);
    BFV_ARENA(ln.arena);
    if (int rc = native_switch(r, ln, d, {words}, {key}, res, outw, d_sops)) return rc;
    return download_words(r, ln, outw, 2, out);
  }
  BFV_CUDA(ln.arena.reserve(slice(n * W * 8) * 3 + slice(2 * L * n * 8) * 2 + 4096), "workspace");
  ln.arena.reset();
  u64* words = nullptr;
  if (int rc = upload_polys(r, ln, d, poly, 1, L, &words, nullptr)) return rc;
  u64* res = ln.arena.take<u64>(2 * L * n);
  SwitchOp* d_sops = ln.arena.take<SwitchOp>(1);
  BFV_ARENA(ln.arena);
  std::vector<SwitchOp> sops{SwitchOp{nullptr, nullptr, words, key->d_key, key->d_key_q, res, 1u, 0u}};
  if (int rc = run_switch(r, ln, d, {}, sops, nullptr, d_sops)) return rc;
  return compose_out(r, ln, d, res, 2, out);
}

int cuhe_bfv_rotate_rows(cuhe_bfv_key* key, const uint8_t* ct, uint64_t exponent, uint8_t* out) {
  if (!key || !ct || !out) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  cuhe_bfv_ring* r = key->ring;
  const size_t n = r->plan.n, L = r->plan.residue_count, W = size_t(r->host_dev.words);
  if (!(exponent & 1) || exponent >= 2 * n) return fail(CUHE_INVALID_ARGUMENT, "Invalid Galois exponent");
  if (exponent == 1) {
    std::vector<u64> words;
    if (int rc = parse_polys(r, ct, 2, words)) return rc;
    std::memcpy(out, ct, 2 * n * r->plan.coefficient_bytes);
    return CUHE_OK;
  }
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, 0, &d)) return rc;
  if (!r->residue) {
    const size_t S = r->switch_prime_count;
    BFV_CUDA(ln.arena.reserve(slice(2 * n * W * 8) * 5 + slice(2 * S * n * 8) + 8192), "workspace");
    ln.arena.reset();
    u64* words = nullptr;
    if (int rc = upload_polys(r, ln, d, ct, 2, 0, &words, nullptr)) return rc;
    u64* perm = ln.arena.take<u64>(2 * n * W);
    u64* outw = ln.arena.take<u64>(2 * n * W);
    u64* ks = ln.arena.take<u64>(2 * n * W);
    u64* res = ln.arena.take<u64>(2 * S * n);
    SwitchOp* d_sops = ln.arena.take<SwitchOp>(1);
    NativeOp* d_nops = ln.arena.take<NativeOp>(1);
    BFV_ARENA(ln.arena);
    if (int rc = native_rotate(r, ln, d, {NativeOp{words, perm, outw, nullptr}}, unsigned(exponent), key, d_nops, res,
                               ks, d_sops))
      return rc;
    return download_words(r, ln, outw, 2, out);
  }
  BFV_CUDA(ln.arena.reserve(slice(2 * n * W * 8) * 2 + slice(2 * L * n * 8) * 3 + slice(n * W * 8) + 8192), "workspace");
  ln.arena.reset();
  u64 *words = nullptr, *res = nullptr;
  if (int rc = upload_polys(r, ln, d, ct, 2, L, &words, &res)) return rc;
  u64* sw = ln.arena.take<u64>(n * W);
  u64* outres = ln.arena.take<u64>(2 * L * n);
  ComposeOp* d_cops = ln.arena.take<ComposeOp>(1);
  SwitchOp* d_sops = ln.arena.take<SwitchOp>(1);
  BFV_ARENA(ln.arena);
  std::vector<ComposeOp> cops{ComposeOp{res + L * n, sw, unsigned(exponent), 0u}};
  std::vector<SwitchOp> sops{SwitchOp{nullptr, res, sw, key->d_key, key->d_key_q, outres, inverse_mod_2n(exponent, n), 0u}};
  if (int rc = run_switch(r, ln, d, cops, sops, d_cops, d_sops)) return rc;
  return compose_out(r, ln, d, outres, 2, out);
}

int cuhe_bfv_ring_product(cuhe_bfv_ring* r, const uint8_t* lhs, const uint8_t* rhs, uint8_t* out) {
  if (!r || !lhs || !rhs || !out) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, 0, &d)) return rc;
  const size_t n = r->plan.n, W = size_t(r->host_dev.words);
  // residue rings multiply mod Q over its L primes; native rings take the
  // exact product over the tensor primes and reduce it mod q
  const size_t L = r->residue ? r->plan.residue_count : r->plan.tensor_count;
  BFV_CUDA(ln.arena.reserve(slice(n * W * 8) * 4 + slice(L * n * 8) * 3 + 8192), "workspace");
  ln.arena.reset();
  u64 *wa, *wb, *ra, *rb;
  if (int rc = upload_polys(r, ln, d, lhs, 1, L, &wa, &ra)) return rc;
  if (int rc = upload_polys(r, ln, d, rhs, 1, L, &wb, &rb)) return rc;
  BFV_CUDA(launch_ntt(r, ln, d, ra, (long long)(L), 0, int(L), 1, 0), "ntt");
  BFV_CUDA(launch_ntt(r, ln, d, rb, (long long)(L), 0, int(L), 1, 0), "ntt");
  k_mul_plain<<<blocks_for((long long)(L * n), 256), 256, 0, ln.stream>>>(ra, (long long)(L), int(L), rb, d);
  BFV_CUDA(cudaGetLastError(), "product");
  BFV_CUDA(launch_ntt(r, ln, d, ra, (long long)(L), 0, int(L), 1, 1), "intt");
  if (!r->residue) {
    u64* outw = ln.arena.take<u64>(n * W);
    BFV_ARENA(ln.arena);
    if (int rc = native_reduce(r, ln, d, ra, 1, L, outw, 0, 0)) return rc;
    return download_words(r, ln, outw, 1, out);
  }
  return compose_out(r, ln, d, ra, 1, out);
}

int cuhe_bfv_multiply(cuhe_bfv_ring* r, const uint8_t* lhs, const uint8_t* rhs, uint64_t t, uint8_t* out) {
  if (!r || !lhs || !out) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (t < 2 || t >= (u64(1) << 60) || H::cmp(H::Big(t), r->plan.q) >= 0)
    return fail(CUHE_INVALID_ARGUMENT, "Invalid plaintext modulus");
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, t, &d)) return rc;
  const size_t n = r->plan.n, L = r->plan.residue_count, T = r->plan.tensor_count, W = size_t(r->host_dev.words);
  BFV_CUDA(ln.arena.reserve(slice(2 * n * W * 8) * 2 + slice(2 * T * n * 8) * 2 + slice(3 * T * n * 8) +
                            slice(3 * L * n * 8) + slice(3 * n * W * 8) + 8192),
           "workspace");
  ln.arena.reset();
  u64 *wa, *ra, *wb = nullptr, *rb = nullptr;
  if (int rc = upload_polys(r, ln, d, lhs, 2, T, &wa, &ra)) return rc;
  if (rhs) {
    if (int rc = upload_polys(r, ln, d, rhs, 2, T, &wb, &rb)) return rc;
  }
  u64* tens = ln.arena.take<u64>(3 * T * n);
  u64* scaled = ln.arena.take<u64>(3 * L * n);
  BFV_ARENA(ln.arena);
  BFV_CUDA(launch_ntt(r, ln, d, ra, (long long)(2 * T), 0, int(T), 1, 0), "ntt");
  if (rb) BFV_CUDA(launch_ntt(r, ln, d, rb, (long long)(2 * T), 0, int(T), 1, 0), "ntt");
  k_tensor<<<blocks_for((long long)(T * n), 256), 256, 0, ln.stream>>>(ra, rb ? rb : ra, 1, int(T), tens, d);
  BFV_CUDA(cudaGetLastError(), "tensor");
  BFV_CUDA(launch_ntt(r, ln, d, tens, (long long)(3 * T), 0, int(T), 1, 1), "intt");
  if (!r->residue) {
    u64* outw = ln.arena.take<u64>(3 * n * W);
    BFV_ARENA(ln.arena);
    if (int rc = native_reduce(r, ln, d, tens, 3, T, outw, 1, t)) return rc;
    return download_words(r, ln, outw, 3, out);
  }
  k_rns_scale<<<blocks_for((long long)(3 * n), 128), 128, 0, ln.stream>>>(tens, 3, scaled, d);
  BFV_CUDA(cudaGetLastError(), "scale");
  return compose_out(r, ln, d, scaled, 3, out);
}

int cuhe_bfv_hamming_tile(cuhe_bfv_key* relin, const uint8_t* query, const uint8_t* tile, const uint64_t* exponents,
                          cuhe_bfv_key* const* keys, uint64_t rotations, const uint8_t* mask, uint64_t t,
                          uint8_t* out) {
  if (!relin || !query || !tile || !mask || !out || (rotations && (!exponents || !keys)))
    return fail(CUHE_INVALID_ARGUMENT, "null argument");
  cuhe_bfv_ring* r = relin->ring;
  const size_t n = r->plan.n, L = r->plan.residue_count, W = size_t(r->host_dev.words);
  if (t < 2 || t >= (u64(1) << 60) || H::cmp(H::Big(t), r->plan.q) >= 0)
    return fail(CUHE_INVALID_ARGUMENT, "Invalid plaintext modulus");
  for (uint64_t k = 0; k < rotations; ++k) {
    if (!(exponents[k] & 1) || exponents[k] >= 2 * n) return fail(CUHE_INVALID_ARGUMENT, "Invalid Galois exponent");
    if (!keys[k] || keys[k]->ring != r) return fail(CUHE_INVALID_ARGUMENT, "Rotation key belongs to another native ring");
  }
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, t, &d)) return rc;
  if (!r->residue) {
    // the caller's mask may be any poly below q: take its exact product over
    // the tensor primes (they cover N (q - 1)^2)
    const size_t T = r->plan.tensor_count;
    BFV_CUDA(ln.arena.reserve(native_tile_bytes(r, 1, T) + slice(2 * n * W * 8) * 3 + slice(n * W * 8) +
                              slice(T * n * 8) + 16384),
             "workspace");
    ln.arena.reset();
    u64 *qw, *tw, *mw, *mres;
    if (int rc = upload_polys(r, ln, d, query, 2, 0, &qw, nullptr)) return rc;
    if (int rc = upload_polys(r, ln, d, tile, 2, 0, &tw, nullptr)) return rc;
    if (int rc = upload_polys(r, ln, d, mask, 1, T, &mw, &mres)) return rc;
    BFV_CUDA(launch_ntt(r, ln, d, mres, (long long)(T), 0, int(T), 1, 0), "mask ntt");
    u64* dist = ln.arena.take<u64>(2 * n * W);
    NativeScratch sc;
    if (int rc = native_scratch(ln.arena, r, 1, T, &sc)) return rc;
    std::vector<u64> exps(exponents, exponents + rotations);
    std::vector<const cuhe_bfv_key*> rkeys(keys, keys + rotations);
    if (int rc = native_tile_circuit(r, ln, d, qw, tw, 1, t, relin, exps, rkeys, {mres}, T, sc, dist, nullptr))
      return rc;
    return download_words(r, ln, dist, 2, out);
  }
  BFV_CUDA(ln.arena.reserve(tile_arena_bytes(r, 1) + slice(2 * n * W * 8) * 2 + slice(n * W * 8) + slice(L * n * 8) * 2 +
                            slice(2 * L * n * 8) + slice(2 * n * W * 8) + 16384),
           "workspace");
  ln.arena.reset();
  u64 *qw, *tw, *mw, *mres;
  if (int rc = upload_polys(r, ln, d, query, 2, 0, &qw, nullptr)) return rc;
  if (int rc = upload_polys(r, ln, d, tile, 2, 0, &tw, nullptr)) return rc;
  if (int rc = upload_polys(r, ln, d, mask, 1, L, &mw, &mres)) return rc;
  BFV_CUDA(launch_ntt(r, ln, d, mres, (long long)(L), 0, int(L), 1, 0), "mask ntt");
  u64* dist = ln.arena.take<u64>(2 * L * n);
  BFV_ARENA(ln.arena);
  TileArgs a;
  a.q_words = qw;
  a.t_words = tw;
  a.ct = 1;
  a.relin = relin;
  for (uint64_t k = 0; k < rotations; ++k) {
    a.exps.push_back(exponents[k]);
    a.keys.push_back(keys[k]);
  }
  a.masks = {mres};
  if (int rc = tile_circuit(r, ln, d, a, dist, nullptr)) return rc;
  return compose_out(r, ln, d, dist, 2, out);
}

int cuhe_bfv_create_server(cuhe_bfv_key* relin, const uint64_t* exponents, cuhe_bfv_key* const* keys, uint64_t count,
                           uint64_t padded, uint64_t t, const char* target_hex, cuhe_bfv_server** out) {
  if (!relin || !out || !target_hex || (count && (!exponents || !keys)))
    return fail(CUHE_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  cuhe_bfv_ring* r = relin->ring;
  const auto& P = r->plan;
  const size_t n = P.n;
  if (t < 2 || t >= (u64(1) << 60) || H::cmp(H::Big(t), P.q) >= 0)
    return fail(CUHE_INVALID_ARGUMENT, "Invalid plaintext modulus");
  if (!padded || padded > n / 2 || (padded & (padded - 1)) || t % (2 * n) != 1 || !H::is_prime64(t))
    return fail(CUHE_INVALID_ARGUMENT, "Invalid native server layout or plaintext modulus");
  const size_t tlen = std::strlen(target_hex);
  if (tlen < 1 || tlen > (P.q_bits + 3) / 4 || (tlen > 1 && target_hex[0] == '0'))
    return fail(CUHE_INVALID_ARGUMENT, "Invalid or oversized native modulus encoding");
  H::Big target;
  try {
    target = H::from_hex(target_hex);
  } catch (const std::invalid_argument&) {
    return fail(CUHE_INVALID_ARGUMENT, "Invalid or oversized native modulus encoding");
  }
  if (H::cmp(target, H::Big(t)) <= 0 || H::cmp(target, P.q) > 0)
    return fail(CUHE_INVALID_ARGUMENT, "Invalid native response modulus");
  std::map<u64, cuhe_bfv_key*> keymap;
  for (uint64_t k = 0; k < count; ++k) {
    const u64 g = exponents[k];
    if (!(g & 1) || g >= 2 * n) return fail(CUHE_INVALID_ARGUMENT, "Invalid Galois exponent");
    if (!keys[k] || keys[k]->ring != r) return fail(CUHE_INVALID_ARGUMENT, "Rotation key belongs to another native ring");
    if (!keymap.emplace(g, keys[k]).second) return fail(CUHE_INVALID_ARGUMENT, "Duplicate rotation key");
  }
  const size_t lanes = n / (2 * padded);
  auto exponent = [&](size_t step) { return H::powmod(3, step % (n / 2), 2 * n); };
  std::vector<u64> left, right;
  for (size_t size = 1; size < padded; size *= 2) {
    left.push_back(exponent(lanes * size));
    right.push_back(exponent(n / 2 - lanes * size));
    if (!keymap.count(left.back()) || !keymap.count(right.back()))
      return fail(CUHE_INVALID_ARGUMENT, "Missing native server rotation key");
  }
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, t, &d)) return rc;
  auto* s = new (std::nothrow) cuhe_bfv_server();
  if (!s) return fail(CUHE_OUT_OF_MEMORY, "server allocation");
  s->ring = r;
  ++r->refs;
  s->relin = relin;
  ++relin->refs;
  for (auto& kv : keymap) {
    s->keys[kv.first] = kv.second;
    ++kv.second->refs;
  }
  s->padded = padded;
  s->lanes = lanes;
  s->capacity = 2 * lanes;
  s->t = t;
  s->target = target;
  s->target_bits = unsigned(target.bits());
  s->target_words = target.w;
  s->left = left;
  s->right = right;
  s->d_ring = d;
  const size_t W = size_t(r->host_dev.words);
  s->mask_primes = r->residue ? P.residue_count : native_mask_primes(r, t);
  int rc = upload_plain_ntt(r, ln, d, small_to_words(hamming_mask(n, t, lanes, s->capacity), W), &s->d_full_mask,
                            s->mask_primes);
  cudaError_t e = cudaSuccess;
  if (!rc) e = cudaMalloc(&s->d_target, 8 * std::max<size_t>(1, target.w.size()));
  if (!rc && e == cudaSuccess)
    e = cudaMemcpy(s->d_target, target.w.data(), 8 * target.w.size(), cudaMemcpyHostToDevice);
  if (rc || e != cudaSuccess) {
    cuhe_bfv_server_release(s);
    return rc ? rc : fail(CUHE_CUDA_ERROR, "server setup");
  }
  *out = s;
  return CUHE_OK;
}

void cuhe_bfv_server_release(cuhe_bfv_server* server) {
  if (server && --server->refs == 0) delete server;
}

uint64_t cuhe_bfv_server_bytes(const cuhe_bfv_server* s) {
  if (!s) return 0;
  return s->ring->plan.residue_count * s->ring->plan.n * 8;
}

int cuhe_bfv_server_layout(const cuhe_bfv_server* s, uint64_t* capacity, uint64_t* padded,
                           uint64_t* input_packed_bytes, uint64_t* output_packed_bytes,
                           uint64_t* compact_packed_bytes) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null server");
  const auto& P = s->ring->plan;
  if (capacity) *capacity = s->capacity;
  if (padded) *padded = s->padded;
  if (input_packed_bytes) *input_packed_bytes = (P.n * P.q_bits + 7) / 8;
  if (output_packed_bytes) *output_packed_bytes = (P.n * P.q_bits + 7) / 8;
  if (compact_packed_bytes) *compact_packed_bytes = (P.n * s->target_bits + 7) / 8;
  return CUHE_OK;
}

int cuhe_bfv_last_profile(const cuhe_bfv_server* s, double* ms, int capacity) {
  if (!s || !ms) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lock(const_cast<cuhe_bfv_server*>(s)->mu);
  for (int i = 0; i < capacity && i < 6; ++i) ms[i] = s->profile_ms[i];
  return CUHE_OK;
}

int cuhe_bfv_set_lanes(cuhe_bfv_ring* ring, int lanes) {
  if (!ring) return fail(CUHE_INVALID_ARGUMENT, "null ring");
  if (lanes < 1 || lanes > kMaxLanes)
    return fail(CUHE_INVALID_ARGUMENT, "lane count must be 1.." + std::to_string(kMaxLanes));
  ring->active_lanes = lanes;
  return CUHE_OK;
}

int cuhe_bfv_get_lanes(const cuhe_bfv_ring* ring) { return ring ? ring->active_lanes.load() : 0; }

}  // extern "C"

struct cuhe_bfv_index {
  cuhe_bfv_server* server = nullptr;
  u64* d_words = nullptr;  // [tiles][2][N][W] composed coefficients
  uint64_t tiles = 0;
  ~cuhe_bfv_index() {
    if (d_words) {
      DeviceGuard g(server->ring->device);
      cudaFree(d_words);
    }
    cuhe_bfv_server_release(server);
  }
};

namespace {

// The Hamming search over tiles given either as packed host bytes (index) or
// as composed words already resident in HBM (resident).
// Workspace of one search chunk of ct tiles (whole response groups).
size_t search_chunk_bytes(const cuhe_bfv_server* s, size_t ct, unsigned out_bits) {
  const cuhe_bfv_ring* r = s->ring;
  const auto& P = r->plan;
  const size_t n = P.n, L = P.residue_count, W = size_t(r->host_dev.words);
  const size_t in_bytes = (n * P.q_bits + 7) / 8;
  const size_t out_words = (n * out_bits + 63) / 64;
  const size_t gc = (ct + s->padded - 1) / s->padded;
  const size_t small = (kSplitWays + 1) * small_switch_bytes(r);  // merge-wave scratch of every part
  if (!r->residue)
    return native_tile_bytes(r, ct, s->mask_primes) + slice(2 * in_bytes) + slice(ct * 2 * in_bytes) +
           slice(2 * n * W * 8) + slice(ct * 2 * n * W * 8) * 2 + slice(gc * 2 * n * W * 8) +
           slice(gc * 2 * out_words * 8) + slice(sizeof(int)) + slice(ct * n * W * 8) +
           slice(ct * sizeof(ComposeOp)) + slice(ct * sizeof(SwitchOp)) + small + 65536;
  return tile_arena_bytes(r, ct) + slice(2 * in_bytes) + slice(ct * 2 * in_bytes) + slice(2 * n * W * 8) +
         slice(ct * 2 * n * W * 8) + slice(ct * 2 * L * n * 8) + slice(gc * 2 * n * W * 8) +
         slice(gc * 2 * out_words * 8) + slice(sizeof(int)) + slice(ct * n * W * 8) + slice(ct * sizeof(ComposeOp)) +
         slice(ct * sizeof(SwitchOp)) + small + 65536;
}

// Tiles per search chunk: whole response groups, about 1024 tiles.
size_t search_chunk_tiles(const cuhe_bfv_server* s) {
  return std::max<size_t>(s->padded, 1024 / s->padded * s->padded);
}

// A free lane among the active ones (round robin from a rotating start), or
// else the start lane once it frees up.
Lane& acquire_lane(cuhe_bfv_ring* r, std::unique_lock<std::mutex>& lock) {
  const unsigned count = unsigned(std::max(1, std::min(kMaxLanes, r->active_lanes.load())));
  const unsigned start = r->next_lane++ % count;
  for (unsigned k = 0; k < count; ++k) {
    Lane& ln = *r->lanes[(start + k) % count];
    std::unique_lock<std::mutex> attempt(ln.mu, std::try_to_lock);
    if (attempt.owns_lock()) {
      lock = std::move(attempt);
      return ln;
    }
  }
  Lane& ln = *r->lanes[start];
  lock = std::unique_lock<std::mutex>(ln.mu);
  return ln;
}

int search_impl(cuhe_bfv_server* s, const uint8_t* query, const PolySource* index, const u64* resident,
                uint64_t tiles, uint64_t count, int compact, uint8_t* out, uint64_t out_capacity,
                uint64_t* responses) {
  if (!s || !query || (tiles && !index && !resident) || !responses) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (count > UINT64_MAX - s->capacity || (count + s->capacity - 1) / s->capacity != tiles)
    return fail(CUHE_INVALID_ARGUMENT, "vector_count does not match the packed ciphertext count");
  cuhe_bfv_ring* r = s->ring;
  const auto& P = r->plan;
  const size_t n = P.n, L = P.residue_count, W = size_t(r->host_dev.words);
  const size_t in_bytes = (n * P.q_bits + 7) / 8;
  const unsigned out_bits = compact ? s->target_bits : unsigned(P.q_bits);
  const size_t out_bytes = (n * out_bits + 7) / 8;
  const size_t groups = (size_t(tiles) + s->padded - 1) / s->padded;
  *responses = 0;
  if (groups * 2 * out_bytes > out_capacity) return fail(CUHE_INVALID_ARGUMENT, "output buffer too small");
  std::unique_lock<std::mutex> lock;
  Lane& ln = acquire_lane(r, lock);
  DeviceGuard guard(r->device);
  RingDev* d = s->d_ring;
  double prof[6] = {0, 0, 0, 0, 0, 0};
  // partial mask for the last tile
  const u64* partial = nullptr;
  if (count % s->capacity) {
    std::lock_guard<std::mutex> masks_lock(s->mu);
    auto it = s->partial_masks.find(size_t(count % s->capacity));
    if (it == s->partial_masks.end()) {
      u64* m = nullptr;
      if (int rc = upload_plain_ntt(r, ln, d,
                                    small_to_words(hamming_mask(n, s->t, s->lanes, size_t(count % s->capacity)), W),
                                    &m, s->mask_primes))
        return rc;
      it = s->partial_masks.emplace(size_t(count % s->capacity), m).first;
    }
    partial = it->second;
  }
  if (tiles == 0) return CUHE_OK;
  // chunks of whole groups, at most ~1024 tiles each
  const size_t max_tiles = search_chunk_tiles(s);
  const size_t out_words = (n * out_bits + 63) / 64;
  for (size_t g0 = 0; g0 < groups;) {
    const size_t first = g0 * s->padded;
    size_t ct = std::min<size_t>(size_t(tiles) - first, max_tiles);
    const size_t gc = (ct + s->padded - 1) / s->padded;
    ct = std::min<size_t>(size_t(tiles) - first, gc * s->padded);
    BFV_CUDA(ln.arena.reserve(search_chunk_bytes(s, ct, out_bits)), "workspace");
    ln.arena.reset();
    uint8_t* d_qb = ln.arena.take<uint8_t>(2 * in_bytes);
    uint8_t* d_ib = resident ? nullptr : ln.arena.take<uint8_t>(ct * 2 * in_bytes);
    u64* qw = ln.arena.take<u64>(2 * n * W);
    u64* tw = resident ? const_cast<u64*>(resident) + first * 2 * n * W : ln.arena.take<u64>(ct * 2 * n * W);
    u64* dist = ln.arena.take<u64>(r->residue ? ct * 2 * L * n : ct * 2 * n * W);
    u64* ow = ln.arena.take<u64>(gc * 2 * n * W);
    u64* packed = ln.arena.take<u64>(gc * 2 * out_words);
    int* d_status = ln.arena.take<int>(1);
    BFV_ARENA(ln.arena);
    BFV_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), ln.stream), "status");
    BFV_CUDA(cudaMemcpyAsync(d_qb, query, 2 * in_bytes, cudaMemcpyHostToDevice, ln.stream), "query upload");
    k_unpack<<<blocks_for((long long)(2 * n), 256), 256, 0, ln.stream>>>(d_qb, (long long)(in_bytes), int(P.q_bits), 2, qw, d,
                                                                         d_status);
    // Host-memory indexes of at least two pieces of kPipeTiles tiles are
    // uploaded piece by piece by a helper thread (pinned double buffer, the
    // lane's copy stream) while the lane runs the tile circuits of the
    // tiles already uploaded.
    const bool piped = !resident && ct >= 2 * kPipeTiles;
    if (!resident && !piped) {
      BFV_CUDA(stage_polys(ln, *index, first * 2, ct * 2, d_ib), "index upload");
      k_unpack<<<blocks_for((long long)(ct * 2 * n), 256), 256, 0, ln.stream>>>(
          d_ib, (long long)(in_bytes), int(P.q_bits), int(ct * 2), tw, d, d_status);
    }
    BFV_CUDA(cudaGetLastError(), "unpack");
    int status = 0;
    if (!piped) {
      BFV_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ln.stream), "status");
      BFV_CUDA(cudaStreamSynchronize(ln.stream), "unpack");
      if (status) return fail(CUHE_INVALID_ARGUMENT, "Noncanonical packed polynomial coefficient");
    }
    NativeScratch sc{};
    if (!r->residue)
      if (int rc = native_scratch(ln.arena, r, ct, s->mask_primes, &sc)) return rc;
    // Merge trees (bfv_server.h:15-45) of the chunk's response groups
    // [g_lo, g_hi), executed in waves of independent merges on `lane`;
    // native rings use `nsc` (scratch for the groups' tiles), residue rings
    // the lane's arena.  Writes each group's result slot.
    std::vector<size_t> result_slot(gc, 0);
    std::vector<char> merged(gc, 0);
    auto merge_groups = [&](Lane& lane, size_t g_lo, size_t g_hi, const NativeScratch& nsc, double* pr) -> int {
      if (g_lo >= g_hi) return CUHE_OK;
      cudaEvent_t m0, m1;
      cudaEventCreate(&m0);
      cudaEventCreate(&m1);
      cudaEventRecord(m0, lane.stream);
      struct Merge { size_t left, right; size_t level; size_t wave; };
      std::vector<Merge> merges;
      for (size_t gi = g_lo; gi < g_hi; ++gi) {
        struct Node { size_t slot, ready; };
        std::vector<std::pair<Node, size_t>> stack;
        const size_t gs = gi * s->padded, ge = std::min(gs + s->padded, ct);
        for (size_t at = gs; at < ge; ++at) {
          Node node{at, 0};
          size_t size = 1, level = 0;
          while (!stack.empty() && stack.back().second == size) {
            const Node left = stack.back().first;
            stack.pop_back();
            const size_t wave = std::max(left.ready, node.ready);
            merges.push_back({left.slot, node.slot, level, wave});
            node = Node{left.slot, wave + 1};
            size *= 2;
            ++level;
          }
          stack.emplace_back(node, size);
        }
        Node result = stack.back().first;
        stack.pop_back();
        while (!stack.empty()) {
          const size_t size = stack.back().second;
          size_t level = 0;
          while ((size_t(1) << level) < size) ++level;
          const Node left = stack.back().first;
          stack.pop_back();
          const size_t wave = std::max(left.ready, result.ready);
          merges.push_back({left.slot, result.slot, level, wave});
          result = Node{left.slot, wave + 1};
        }
        result_slot[gi] = result.slot;
      }
      size_t waves = 0;
      for (const auto& m : merges) waves = std::max(waves, m.wave + 1);
      if (!r->residue) {
        // native: rotate each right operand (grouped by level, one key each),
        // then add it into its left operand
        for (size_t w = 0; w < waves; ++w) {
          std::vector<NativeOp> adds;
          size_t used = 0;
          for (size_t level = 0; level < s->right.size(); ++level) {
            std::vector<NativeOp> rots;
            for (const auto& m : merges) {
              if (m.wave != w || m.level != level) continue;
              const size_t k = used + rots.size();
              rots.push_back(NativeOp{dist + m.right * 2 * n * W, nsc.perm + k * 2 * n * W, nsc.tmp + k * 2 * n * W,
                                      nullptr});
              adds.push_back(NativeOp{dist + m.left * 2 * n * W, nsc.tmp + k * 2 * n * W,
                                      dist + m.left * 2 * n * W, nullptr});
            }
            if (rots.empty()) continue;
            const u64 g = s->right.at(level);
            if (int rc = native_rotate(r, lane, d, rots, unsigned(g), s->keys.at(g), nsc.d_nops, nsc.ksres,
                                       nsc.ksw + used * 2 * n * W, nsc.d_sops, &lane.arena))
              return rc;
            used += rots.size();
          }
          if (int rc = native_add_ops(r, lane, d, adds, nsc.d_nops)) return rc;
        }
      } else {
        const size_t mark = lane.arena.used;
        const size_t most = merges.size();
        u64* mwords = lane.arena.take<u64>(std::max<size_t>(1, most) * n * W);
        ComposeOp* d_cops = lane.arena.take<ComposeOp>(std::max<size_t>(1, most));
        SwitchOp* d_sops = lane.arena.take<SwitchOp>(std::max<size_t>(1, most));
        BFV_ARENA(lane.arena);
        for (size_t w = 0; w < waves; ++w) {
          std::vector<ComposeOp> cops;
          std::vector<SwitchOp> sops;
          for (const auto& m : merges) {
            if (m.wave != w) continue;
            const u64 g = s->right.at(m.level);
            u64* words = mwords + cops.size() * n * W;
            cops.push_back(ComposeOp{dist + (m.right * 2 + 1) * L * n, words, unsigned(g), 0u});
            const cuhe_bfv_key* key = s->keys.at(g);
            sops.push_back(SwitchOp{dist + m.left * 2 * L * n, dist + m.right * 2 * L * n, words, key->d_key,
                                    key->d_key_q, dist + m.left * 2 * L * n, inverse_mod_2n(g, n), 0u});
          }
          // the arena past the op tables lends scratch to the small waves
          if (int rc = run_switch(r, lane, d, cops, sops, d_cops, d_sops, &lane.arena)) return rc;
        }
        lane.arena.used = mark;
      }
      cudaEventRecord(m1, lane.stream);
      BFV_CUDA(cudaEventSynchronize(m1), "merge");
      float x = 0;
      cudaEventElapsedTime(&x, m0, m1);
      pr[4] += x;
      cudaEventDestroy(m0);
      cudaEventDestroy(m1);
      for (size_t gi = g_lo; gi < g_hi; ++gi) merged[gi] = 1;
      return CUHE_OK;
    };
    // tile circuits of chunk tiles [t0, t0 + tc) into their dist slots, on
    // `lane` (its stream; residue rings take their workspace from its
    // arena, native rings use `nsc`, scratch for tc tiles)
    auto circuit = [&](Lane& lane, size_t t0, size_t tc, const NativeScratch& nsc, double* pr) -> int {
      if (r->residue) {
        TileArgs a;
        a.q_words = qw;
        a.t_words = tw + t0 * 2 * n * W;
        a.ct = tc;
        a.relin = s->relin;
        for (u64 g : s->left) {
          a.exps.push_back(g);
          a.keys.push_back(s->keys.at(g));
        }
        a.masks.assign(tc, s->d_full_mask);
        if (partial && first + t0 + tc == size_t(tiles)) a.masks[tc - 1] = partial;
        return tile_circuit(r, lane, d, a, dist + t0 * 2 * L * n, pr);
      }
      std::vector<u64> exps(s->left.begin(), s->left.end());
      std::vector<const cuhe_bfv_key*> rkeys;
      for (u64 g : s->left) rkeys.push_back(s->keys.at(g));
      std::vector<const u64*> masks(tc, s->d_full_mask);
      if (partial && first + t0 + tc == size_t(tiles)) masks[tc - 1] = partial;
      return native_tile_circuit(r, lane, d, qw, tw + t0 * 2 * n * W, tc, s->t, s->relin, exps, rkeys, masks,
                                 s->mask_primes, nsc, dist + t0 * 2 * n * W, pr);
    };
    auto run_tiles = [&](size_t t0, size_t tc) -> int {
      const size_t mark = ln.arena.used;  // the circuit's workspace is free again when it returns
      if (P.n > kMaxPlaneN || tc < kSplitTiles) {
        const int rc = circuit(ln, t0, tc, sc, prof);
        ln.arena.used = mark;
        return rc;
      }
      // kSplitWays parts on as many streams, each driven by its own host
      // thread: a launch's last partial wave of CTAs overlaps the other
      // parts' launches, and one part's host synchronisations leave the GPU
      // to the others.  Each part takes its own slice of the workspace
      // (residue rings) or of the chunk's scratch (native rings).  Part
      // boundaries fall on response-group boundaries where one lies near.
      constexpr int K = kSplitWays;
      size_t bound[K + 1];
      bound[0] = t0;
      bound[K] = t0 + tc;
      for (int k = 1; k < K; ++k) {
        const size_t mid = t0 + tc * k / K, pad = s->padded, slack = tc / (4 * K);  // parts stay non-empty
        const size_t lo = (mid / pad) * pad, hi = lo + pad;
        const size_t pick = mid - lo <= hi - mid ? lo : hi;
        bound[k] = pick + slack >= mid && pick <= mid + slack ? pick : mid;
      }
      Lane part[K];
      size_t offset = mark;
      for (int k = 0; k < K; ++k) {
        part[k].arena.owned = false;
        const size_t bytes = r->residue ? tile_arena_bytes(r, bound[k + 1] - bound[k]) : small_switch_bytes(r);
        part[k].arena.base = ln.arena.base + offset;
        part[k].arena.cap = bytes;
        offset += bytes;
      }
      if (offset > ln.arena.cap) return fail(CUHE_OUT_OF_MEMORY, "internal workspace exhausted");
      part[0].stream = ln.stream;
      for (int k = 1; k < K; ++k) {
        if (!ln.side[k - 1]) {
          int prio = 0;
          BFV_CUDA(cudaStreamGetPriority(ln.stream, &prio), "stream priority");
          BFV_CUDA(cudaStreamCreateWithPriority(&ln.side[k - 1], cudaStreamNonBlocking, prio), "side stream");
        }
        part[k].stream = ln.side[k - 1];
      }
      NativeScratch nsc[K];  // scratch of each part's tiles: every array offset by the part's first tile
      for (int k = 0; k < K; ++k) {
        const size_t off = bound[k] - t0;
        nsc[k] = sc;
        if (r->residue) continue;
        const size_t T = P.tensor_count, S = r->switch_prime_count, M = s->mask_primes;
        nsc[k].diff += off * 2 * n * W;
        nsc[k].dres += off * 2 * T * n;
        nsc[k].tens += off * 3 * T * n;
        nsc[k].words3 += off * 3 * n * W;
        nsc[k].ksres += off * 2 * S * n;
        nsc[k].ksw += off * 2 * n * W;
        nsc[k].perm += off * 2 * n * W;
        nsc[k].tmp += off * 2 * n * W;
        nsc[k].mres += off * 2 * M * n;
        nsc[k].d_sops += off;
        nsc[k].d_nops += off;
      }
      cudaEvent_t ready;
      BFV_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
      cudaError_t e = cudaEventRecord(ready, ln.stream);  // unpacked tiles and query
      for (int k = 1; k < K && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(part[k].stream, ready, 0);
      cudaEventDestroy(ready);
      BFV_CUDA(e, "side stream order");
      double part_prof[K][6] = {};
      int part_rc[K] = {};
      std::string part_err[K];
      const int device = r->device;
      // circuits of tiles [h0, h1), then, when this batch is the whole
      // chunk, the merges of the groups they hold whole (the batches of a
      // pipelined upload leave all merges to the end, where the waves of
      // every group together fill the GPU)
      auto run_part = [&](int k) {
        const size_t h0 = bound[k], h1 = bound[k + 1];
        int rc = circuit(part[k], h0, h1 - h0, nsc[k], part_prof[k]);
        if (!rc && tc == ct) {
          part[k].arena.used = 0;
          const size_t pad = s->padded;
          const size_t g_lo = (h0 + pad - 1) / pad;
          const size_t g_hi = h1 == ct ? gc : h1 / pad;
          rc = merge_groups(part[k], g_lo, std::max(g_lo, g_hi), nsc[k], part_prof[k]);
        }
        part_rc[k] = rc;
        if (rc) part_err[k] = t_error;
      };
      std::vector<std::thread> helpers;
      for (int k = 1; k < K; ++k)
        helpers.emplace_back([&, k] {
          cudaSetDevice(device);
          run_part(k);
        });
      run_part(0);
      for (auto& h : helpers) h.join();
      for (int k = 1; k < K; ++k) cudaStreamSynchronize(part[k].stream);  // idle whatever happened
      int rc = CUHE_OK;
      for (int k = 0; k < K && !rc; ++k)
        if (part_rc[k]) rc = fail(part_rc[k], part_err[k]);
      for (int k = 0; k < K; ++k)
        for (int j = 0; j < 6; ++j) prof[j] += part_prof[k][j] / K;  // the parts overlap
      ln.arena.used = mark;
      return rc;
    };
    if (!piped) {
      if (int rc = run_tiles(0, ct)) return rc;
    } else {
      const size_t subs = (ct + kPipeTiles - 1) / kPipeTiles;
      const size_t sub_bytes = kPipeTiles * 2 * in_bytes;
      if (!ln.copy) BFV_CUDA(cudaStreamCreateWithFlags(&ln.copy, cudaStreamNonBlocking), "copy stream");
      for (int h = 0; h < 2; ++h)
        if (ln.pin_cap[h] < sub_bytes) {
          if (ln.pin[h]) cudaFreeHost(ln.pin[h]);
          ln.pin[h] = nullptr;
          ln.pin_cap[h] = 0;
          BFV_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ln.pin[h]), sub_bytes, cudaHostAllocDefault), "pinned");
          ln.pin_cap[h] = sub_bytes;
        }
      std::vector<cudaEvent_t> up(subs, nullptr);
      for (auto& e : up) BFV_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
      std::mutex mu;
      std::condition_variable cv;
      size_t issued = 0;
      cudaError_t stage_error = cudaSuccess;
      std::atomic<bool> stop{false};
      const int device = r->device;
      std::thread stager([&] {
        cudaSetDevice(device);
        for (size_t k = 0; k < subs && !stop.load(); ++k) {
          const size_t t0 = k * kPipeTiles, tc = std::min(kPipeTiles, ct - t0);
          uint8_t* pin = ln.pin[k % 2];
          cudaError_t e = k >= 2 ? cudaEventSynchronize(up[k - 2]) : cudaSuccess;  // its half is free again
          if (e == cudaSuccess) {
            // the first piece is on the critical path: more threads for it
            copy_polys(*index, (first + t0) * 2, tc * 2, pin, k == 0 ? 8 : 4, k == 0 ? 21 : 22);
            e = cudaMemcpyAsync(d_ib + t0 * 2 * in_bytes, pin, tc * 2 * in_bytes, cudaMemcpyHostToDevice, ln.copy);
          }
          if (e == cudaSuccess) e = cudaEventRecord(up[k], ln.copy);
          {
            std::lock_guard<std::mutex> g(mu);
            if (e != cudaSuccess) stage_error = e;
            else issued = k + 1;
          }
          cv.notify_one();
          if (e != cudaSuccess) break;
        }
      });
      // compute in two batches: the first piece, then all the others (their
      // uploads hide under the first batch's circuits, and the large second
      // batch keeps the key-switch launches many waves long)
      int rc = CUHE_OK;
      for (size_t batch = 0; batch < 2 && rc == CUHE_OK; ++batch) {
        const size_t k = batch == 0 ? 0 : subs - 1;  // last piece of the batch
        const size_t t0 = batch == 0 ? 0 : kPipeTiles, tc = batch == 0 ? kPipeTiles : ct - kPipeTiles;
        {
          std::unique_lock<std::mutex> g(mu);
          cv.wait(g, [&] { return issued > k || stage_error != cudaSuccess; });
          if (stage_error != cudaSuccess) {
            rc = fail(CUHE_CUDA_ERROR, std::string("index upload: ") + cudaGetErrorString(stage_error));
            break;
          }
        }
        cudaError_t e = cudaStreamWaitEvent(ln.stream, up[k], 0);
        if (e == cudaSuccess) {
          k_unpack<<<blocks_for((long long)(tc * 2 * n), 256), 256, 0, ln.stream>>>(
              d_ib + t0 * 2 * in_bytes, (long long)(in_bytes), int(P.q_bits), int(tc * 2), tw + t0 * 2 * n * W, d,
              d_status);
          e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
          rc = fail(CUHE_CUDA_ERROR, std::string("unpack: ") + cudaGetErrorString(e));
          break;
        }
        rc = run_tiles(t0, tc);
      }
      stop.store(true);
      stager.join();
      cudaStreamSynchronize(ln.copy);  // no upload still writes the workspace
      for (auto& e : up) cudaEventDestroy(e);
      if (rc) return rc;
      BFV_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ln.stream), "status");
      BFV_CUDA(cudaStreamSynchronize(ln.stream), "unpack");
      if (status) return fail(CUHE_INVALID_ARGUMENT, "Noncanonical packed polynomial coefficient");
    }
    // groups not merged with their tiles' half batches
    for (size_t gi = 0; gi < gc;) {
      if (merged[gi]) {
        ++gi;
        continue;
      }
      size_t ge = gi;
      while (ge < gc && !merged[ge]) ++ge;
      const size_t mark = ln.arena.used;
      if (int rc = merge_groups(ln, gi, ge, sc, prof)) return rc;
      ln.arena.used = mark;
      gi = ge;
    }
    cudaEvent_t m1;
    cudaEventCreate(&m1);
    cudaEventRecord(m1, ln.stream);
    ComposeOp* d_cops = ln.arena.take<ComposeOp>(std::max<size_t>(1, 2 * gc));
    BFV_ARENA(ln.arena);
    // outputs: compose, optional compaction, packing
    if (r->residue) {
      std::vector<ComposeOp> cops;
      for (size_t gi = 0; gi < gc; ++gi)
        for (size_t comp = 0; comp < 2; ++comp)
          cops.push_back(ComposeOp{dist + (result_slot[gi] * 2 + comp) * L * n, ow + (gi * 2 + comp) * n * W, 1u, 0u});
      if (int rc = run_switch(r, ln, d, cops, {}, d_cops, nullptr)) return rc;
    } else {
      for (size_t gi = 0; gi < gc; ++gi)
        BFV_CUDA(cudaMemcpyAsync(ow + gi * 2 * n * W, dist + result_slot[gi] * 2 * n * W, 2 * n * W * 8,
                                 cudaMemcpyDeviceToDevice, ln.stream),
                 "result copy");
    }
    if (compact) {
      k_compact<<<blocks_for((long long)(gc * 2 * n), 128), 128, 0, ln.stream>>>(ow, (long long)(gc * 2 * n), s->d_target,
                                                                                 int(s->target_words.size()), d);
      BFV_CUDA(cudaGetLastError(), "compact");
    }
    k_pack<<<blocks_for((long long)(gc * 2 * out_words), 256), 256, 0, ln.stream>>>(ow, int(W), int(n), int(out_bits),
                                                                                   int(gc * 2), packed, (long long)(out_words));
    BFV_CUDA(cudaGetLastError(), "pack");
    std::vector<u64> host(gc * 2 * out_words);
    BFV_CUDA(cudaMemcpyAsync(host.data(), packed, host.size() * 8, cudaMemcpyDeviceToHost, ln.stream), "download");
    cudaEvent_t o1;
    cudaEventCreate(&o1);
    cudaEventRecord(o1, ln.stream);
    BFV_CUDA(cudaStreamSynchronize(ln.stream), "search");
    float x = 0;
    cudaEventElapsedTime(&x, m1, o1);
    prof[5] += x;
    cudaEventDestroy(m1);
    cudaEventDestroy(o1);
    for (size_t gi = 0; gi < gc * 2; ++gi)
      std::memcpy(out + (g0 * 2 + gi) * out_bytes, reinterpret_cast<const uint8_t*>(host.data() + gi * out_words),
                  out_bytes);
    g0 += gc;
  }
  *responses = groups;
  std::lock_guard<std::mutex> profile_lock(s->mu);
  std::copy(prof, prof + 6, s->profile_ms);
  return CUHE_OK;
}

}  // namespace

extern "C" {

int cuhe_bfv_packed_search(cuhe_bfv_server* s, const uint8_t* query, const uint8_t* index, uint64_t tiles,
                           uint64_t count, int compact, uint8_t* out, uint64_t out_capacity, uint64_t* responses) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  PolySource src;
  src.contiguous = index;
  src.poly_bytes = (s->ring->plan.n * s->ring->plan.q_bits + 7) / 8;
  return search_impl(s, query, index ? &src : nullptr, nullptr, tiles, count, compact, out, out_capacity, responses);
}

int cuhe_bfv_packed_search_parts(cuhe_bfv_server* s, const uint8_t* query, const uint8_t* const* polys,
                                 uint64_t tiles, uint64_t count, int compact, uint8_t* out, uint64_t out_capacity,
                                 uint64_t* responses) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  for (uint64_t k = 0; polys && k < 2 * tiles; ++k)
    if (!polys[k]) return fail(CUHE_INVALID_ARGUMENT, "null polynomial pointer");
  PolySource src;
  src.parts = polys;
  src.poly_bytes = (s->ring->plan.n * s->ring->plan.q_bits + 7) / 8;
  return search_impl(s, query, polys ? &src : nullptr, nullptr, tiles, count, compact, out, out_capacity, responses);
}

namespace {
int upload_index_impl(cuhe_bfv_server* s, const PolySource* index, uint64_t tiles, cuhe_bfv_index** out);
}

int cuhe_bfv_upload_index(cuhe_bfv_server* s, const uint8_t* index, uint64_t tiles, cuhe_bfv_index** out) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  PolySource src;
  src.contiguous = index;
  src.poly_bytes = (s->ring->plan.n * s->ring->plan.q_bits + 7) / 8;
  return upload_index_impl(s, index ? &src : nullptr, tiles, out);
}

int cuhe_bfv_upload_index_parts(cuhe_bfv_server* s, const uint8_t* const* polys, uint64_t tiles,
                                cuhe_bfv_index** out) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  for (uint64_t k = 0; polys && k < 2 * tiles; ++k)
    if (!polys[k]) return fail(CUHE_INVALID_ARGUMENT, "null polynomial pointer");
  PolySource src;
  src.parts = polys;
  src.poly_bytes = (s->ring->plan.n * s->ring->plan.q_bits + 7) / 8;
  return upload_index_impl(s, polys ? &src : nullptr, tiles, out);
}

}  // extern "C"

namespace {

int upload_index_impl(cuhe_bfv_server* s, const PolySource* index, uint64_t tiles, cuhe_bfv_index** out) {
  if (!s || !out || (tiles && !index)) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  cuhe_bfv_ring* r = s->ring;
  const auto& P = r->plan;
  const size_t n = P.n, W = size_t(r->host_dev.words);
  const size_t in_bytes = (n * P.q_bits + 7) / 8;
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  auto* idx = new (std::nothrow) cuhe_bfv_index();
  if (!idx) return fail(CUHE_OUT_OF_MEMORY, "index allocation");
  idx->server = s;
  ++s->refs;
  idx->tiles = tiles;
  if (tiles) {
    const size_t chunk = 256;
    if (cudaMalloc(&idx->d_words, size_t(tiles) * 2 * n * W * 8) != cudaSuccess) {
      cudaGetLastError();
      delete idx;
      return fail(CUHE_OUT_OF_MEMORY, "index does not fit in device memory");
    }
    const size_t need = slice(chunk * 2 * in_bytes) + slice(sizeof(int));
    if (ln.arena.reserve(need) != cudaSuccess) {
      delete idx;
      return fail(CUHE_OUT_OF_MEMORY, "workspace");
    }
    ln.arena.reset();
    uint8_t* d_ib = ln.arena.take<uint8_t>(chunk * 2 * in_bytes);
    int* d_status = ln.arena.take<int>(1);
    if (ln.arena.overflow) { delete idx; return fail(CUHE_OUT_OF_MEMORY, "internal workspace exhausted"); }
    cudaMemsetAsync(d_status, 0, sizeof(int), ln.stream);
    for (size_t t0 = 0; t0 < tiles; t0 += chunk) {
      const size_t ct = std::min<size_t>(chunk, size_t(tiles) - t0);
      if (stage_polys(ln, *index, t0 * 2, ct * 2, d_ib) != cudaSuccess) {
        cudaGetLastError();
        delete idx;
        return fail(CUHE_CUDA_ERROR, "index upload");
      }
      k_unpack<<<blocks_for((long long)(ct * 2 * n), 256), 256, 0, ln.stream>>>(
          d_ib, (long long)(in_bytes), int(P.q_bits), int(ct * 2), idx->d_words + t0 * 2 * n * W, s->d_ring, d_status);
      cudaStreamSynchronize(ln.stream);  // the staging slice is reused by the next chunk
    }
    int status = 0;
    cudaError_t e = cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { delete idx; return fail(CUHE_CUDA_ERROR, "index upload"); }
    if (status) { delete idx; return fail(CUHE_INVALID_ARGUMENT, "Noncanonical packed polynomial coefficient"); }
  }
  *out = idx;
  return CUHE_OK;
}

}  // namespace

extern "C" {

void cuhe_bfv_index_release(cuhe_bfv_index* index) { delete index; }

int cuhe_bfv_search_index(cuhe_bfv_server* s, cuhe_bfv_index* index, const uint8_t* query, uint64_t count,
                          int compact, uint8_t* out, uint64_t out_capacity, uint64_t* responses) {
  if (!index || index->server != s) return fail(CUHE_INVALID_ARGUMENT, "index belongs to another server");
  return search_impl(s, query, nullptr, index->d_words, index->tiles, count, compact, out, out_capacity, responses);
}

uint64_t cuhe_bfv_search_workspace(const cuhe_bfv_server* s, uint64_t tiles, int compact) {
  if (!s || !tiles) return 0;
  const size_t ct = std::min<size_t>(size_t(tiles), search_chunk_tiles(s));
  return search_chunk_bytes(s, ct, compact ? s->target_bits : unsigned(s->ring->plan.q_bits));
}

int cuhe_bfv_reserve_workspace(cuhe_bfv_server* s, uint64_t tiles, int compact) {
  if (!s) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (!tiles) return CUHE_OK;
  cuhe_bfv_ring* r = s->ring;
  const uint64_t bytes = cuhe_bfv_search_workspace(s, tiles, compact);
  const int lanes = std::max(1, std::min(kMaxLanes, r->active_lanes.load()));
  DeviceGuard guard(r->device);
  for (int k = 0; k < lanes; ++k) {
    Lane& ln = *r->lanes[size_t(k)];
    std::lock_guard<std::mutex> lock(ln.mu);
    BFV_CUDA(cudaStreamSynchronize(ln.stream), "lane drain");
    BFV_CUDA(ln.arena.reserve(size_t(bytes)), "workspace");
  }
  return CUHE_OK;
}

int cuhe_bfv_batch_encode(cuhe_bfv_ring* r, uint64_t t, const uint32_t* slots, uint64_t count, uint64_t* out) {
  if (!r || (count && (!slots || !out))) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (count == 0) return CUHE_OK;
  const size_t n = r->plan.n;
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  cuhe_bfv_ring::PlainRing pr;
  if (int rc = plain_ring(r, t, &pr)) return rc;
  const size_t chunk = std::min<size_t>(size_t(count), 1024);
  BFV_CUDA(ln.arena.reserve(slice(chunk * n * 4) + slice(chunk * n * 8) + slice(sizeof(int)) + 4096), "workspace");
  ln.arena.reset();
  uint32_t* d_slots = ln.arena.take<uint32_t>(chunk * n);
  u64* m = ln.arena.take<u64>(chunk * n);
  int* d_status = ln.arena.take<int>(1);
  BFV_ARENA(ln.arena);
  BFV_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), ln.stream), "status");
  for (size_t c0 = 0; c0 < size_t(count); c0 += chunk) {
    const size_t cc = std::min(chunk, size_t(count) - c0);
    BFV_CUDA(cudaMemcpyAsync(d_slots, slots + c0 * n, cc * n * 4, cudaMemcpyHostToDevice, ln.stream), "slots");
    k_scatter_slots<<<blocks_for((long long)(cc * n), 256), 256, 0, ln.stream>>>(d_slots, pr.d_perm, (long long)cc,
                                                                                 int(n), uint32_t(t), m, d_status);
    BFV_CUDA(cudaGetLastError(), "scatter");
    BFV_CUDA(ntt_planes(n, ln.stream, pr.d, m, (long long)cc, 0, 1, 1, 1), "batch encode");
    int status = 0;
    BFV_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ln.stream), "status");
    BFV_CUDA(cudaMemcpyAsync(out + c0 * n, m, cc * n * 8, cudaMemcpyDeviceToHost, ln.stream), "download");
    BFV_CUDA(cudaStreamSynchronize(ln.stream), "batch encode");
    if (status) return fail(CUHE_INVALID_ARGUMENT, "slot value not below the plaintext modulus");
  }
  return CUHE_OK;
}

}  // extern "C"

namespace {

// Public-key encryption with the noise either from the caller (u, e) or,
// with `keyed`, drawn on the device from a ChaCha20 keystream.
int encrypt_impl(cuhe_bfv_ring* r, const uint8_t* pk, uint64_t t, const uint32_t* slots, const int8_t* u,
                 const int8_t* e, const NoiseKey* keyed, uint64_t count, uint8_t* out) {
  if (!r || !pk || (count && (!slots || (!keyed && (!u || !e)) || !out)))
    return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (!r->residue) return fail(CUHE_INVALID_ARGUMENT, "client encryption needs a residue ring");
  if (count == 0) return CUHE_OK;
  const auto& P = r->plan;
  const size_t n = P.n, L = P.residue_count, W = size_t(r->host_dev.words);
  const size_t in_bytes = (n * P.q_bits + 7) / 8;
  if (!keyed)
    for (uint64_t k = 0; k < count * n; ++k)
      if (u[k] < -1 || u[k] > 1) return fail(CUHE_INVALID_ARGUMENT, "u must be ternary");
  std::vector<u64> pk_words;
  if (int rc = parse_polys(r, pk, 2, pk_words)) return rc;
  Lane& ln = *r->lanes[0];
  std::lock_guard<std::mutex> lock(ln.mu);
  DeviceGuard guard(r->device);
  RingDev* d = nullptr;
  if (int rc = device_ring(r, 0, &d)) return rc;
  cuhe_bfv_ring::PlainRing pr;
  if (int rc = plain_ring(r, t, &pr)) return rc;
  // delta = floor(Q / t) mod p_j = -(Q mod t) * t^-1 mod p_j (p_j divides Q)
  const u64 q_mod_t = H::mod_small(P.q, t);
  std::vector<u64> delta(L);
  for (size_t j = 0; j < L; ++j) {
    const u64 p = P.primes[j];
    const u64 t_inv = H::powmod(t % p, p - 2, p);
    delta[j] = u64(u128((p - q_mod_t % p) % p) * t_inv % p);
  }
  const size_t chunk = std::min<size_t>(size_t(count), 512);
  const size_t out_words = (n * P.q_bits + 63) / 64;
  const size_t need = slice(2 * n * W * 8) + slice(2 * L * n * 8) + slice(L * 8) + slice(sizeof(int)) +
                      slice(chunk * n * 4) + slice(chunk * n) + slice(chunk * 2 * n) + slice(chunk * n * 8) +
                      slice(chunk * L * n * 8) + slice(chunk * 2 * L * n * 8) + slice(chunk * 2 * n * W * 8) +
                      slice(chunk * 2 * out_words * 8) + slice(chunk * 2 * sizeof(ComposeOp)) + 65536;
  BFV_CUDA(ln.arena.reserve(need), "workspace");
  ln.arena.reset();
  u64* pk_w = ln.arena.take<u64>(2 * n * W);
  u64* pk_ntt = ln.arena.take<u64>(2 * L * n);
  u64* d_delta = ln.arena.take<u64>(L);
  int* d_status = ln.arena.take<int>(1);
  uint32_t* d_slots = ln.arena.take<uint32_t>(chunk * n);
  int8_t* d_u = ln.arena.take<int8_t>(chunk * n);
  int8_t* d_e = ln.arena.take<int8_t>(chunk * 2 * n);
  u64* m = ln.arena.take<u64>(chunk * n);
  u64* u_ntt = ln.arena.take<u64>(chunk * L * n);
  u64* ct = ln.arena.take<u64>(chunk * 2 * L * n);
  u64* words = ln.arena.take<u64>(chunk * 2 * n * W);
  u64* packed = ln.arena.take<u64>(chunk * 2 * out_words);
  ComposeOp* d_cops = ln.arena.take<ComposeOp>(chunk * 2);
  BFV_ARENA(ln.arena);
  // The client's secrets (message slots, u, e, the encoded message, NTT(u))
  // do not outlive the call in the lane's arena: cleared on every return.
  struct Wipe {
    cudaStream_t stream;
    std::pair<void*, size_t> spans[5];
    ~Wipe() {
      for (const auto& s : spans) cudaMemsetAsync(s.first, 0, s.second, stream);
      cudaStreamSynchronize(stream);
    }
  } wipe{ln.stream, {{d_slots, chunk * n * 4}, {d_u, chunk * n}, {d_e, chunk * 2 * n}, {m, chunk * n * 8},
                     {u_ntt, chunk * L * n * 8}}};
  BFV_CUDA(cudaMemcpyAsync(pk_w, pk_words.data(), pk_words.size() * 8, cudaMemcpyHostToDevice, ln.stream), "pk");
  BFV_CUDA(cudaMemcpyAsync(d_delta, delta.data(), L * 8, cudaMemcpyHostToDevice, ln.stream), "delta");
  BFV_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), ln.stream), "status");
  k_words_to_residues<<<blocks_for((long long)(2 * n), 256), 256, 0, ln.stream>>>(pk_w, 2, int(L), pk_ntt, d);
  BFV_CUDA(cudaGetLastError(), "pk residues");
  BFV_CUDA(launch_ntt(r, ln, d, pk_ntt, (long long)(2 * L), 0, int(L), 1, 0), "pk ntt");
  std::unique_ptr<u64[]> host(out_words * 8 == in_bytes ? nullptr : new u64[chunk * 2 * out_words]);
  for (size_t c0 = 0; c0 < size_t(count); c0 += chunk) {
    const size_t cc = std::min(chunk, size_t(count) - c0);
    BFV_CUDA(cudaMemcpyAsync(d_slots, slots + c0 * n, cc * n * 4, cudaMemcpyHostToDevice, ln.stream), "slots");
    if (keyed) {
      NoiseKey nk = *keyed;
      nk.first_ct += c0;
      k_keyed_noise<<<blocks_for((long long)(cc * nk.blocks_per_ct), 256), 256, 0, ln.stream>>>(
          nk, (long long)cc, int(n), d_u, d_e, d_status);
      BFV_CUDA(cudaGetLastError(), "keyed noise");
    } else {
      BFV_CUDA(cudaMemcpyAsync(d_u, u + c0 * n, cc * n, cudaMemcpyHostToDevice, ln.stream), "u");
      BFV_CUDA(cudaMemcpyAsync(d_e, e + c0 * 2 * n, cc * 2 * n, cudaMemcpyHostToDevice, ln.stream), "e");
    }
    // batch encoding: m = INTT_t(scattered slots)
    k_scatter_slots<<<blocks_for((long long)(cc * n), 256), 256, 0, ln.stream>>>(d_slots, pr.d_perm, (long long)cc,
                                                                                 int(n), uint32_t(t), m, d_status);
    BFV_CUDA(cudaGetLastError(), "scatter");
    BFV_CUDA(ntt_planes(n, ln.stream, pr.d, m, (long long)cc, 0, 1, 1, 1), "batch encode");
    // (b, a) * u + (e0 + delta m, e1)
    k_small_residues<<<blocks_for((long long)(cc * n), 256), 256, 0, ln.stream>>>(d_u, (long long)cc, int(L), u_ntt, d);
    BFV_CUDA(cudaGetLastError(), "u residues");
    BFV_CUDA(launch_ntt(r, ln, d, u_ntt, (long long)(cc * L), 0, int(L), 1, 0), "u ntt");
    k_mul_public<<<blocks_for((long long)(cc * 2 * L * n), 256), 256, 0, ln.stream>>>(u_ntt, pk_ntt, (long long)cc,
                                                                                     int(L), ct, d);
    BFV_CUDA(cudaGetLastError(), "products");
    BFV_CUDA(launch_ntt(r, ln, d, ct, (long long)(cc * 2 * L), 0, int(L), 1, 1), "intt");
    k_add_noise_message<<<blocks_for((long long)(cc * 2 * L * n), 256), 256, 0, ln.stream>>>(
        ct, d_e, m, d_delta, (long long)cc, int(L), d);
    BFV_CUDA(cudaGetLastError(), "noise");
    std::vector<ComposeOp> cops(cc * 2);
    for (size_t k = 0; k < cc * 2; ++k) cops[k] = ComposeOp{ct + k * L * n, words + k * n * W, 1u, 0u};
    if (int rc = run_switch(r, ln, d, cops, {}, d_cops, nullptr)) return rc;
    k_pack<<<blocks_for((long long)(cc * 2 * out_words), 256), 256, 0, ln.stream>>>(
        words, int(W), int(n), int(P.q_bits), int(cc * 2), packed, (long long)(out_words));
    BFV_CUDA(cudaGetLastError(), "pack");
    int status = 0;
    BFV_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, ln.stream), "status");
    // packed polys that fill whole words move through the lane's pinned
    // staging (full-speed DMA) and then to the caller's buffer on several
    // host threads
    const bool direct = out_words * 8 == in_bytes;
    const size_t down = cc * 2 * out_words * 8;
    if (direct && ln.host_cap < down) {
      if (ln.host_stage) cudaFreeHost(ln.host_stage);
      ln.host_stage = nullptr;
      ln.host_cap = 0;
      BFV_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ln.host_stage), down, cudaHostAllocDefault), "pinned");
      ln.host_cap = down;
    }
    BFV_CUDA(cudaMemcpyAsync(direct ? static_cast<void*>(ln.host_stage) : static_cast<void*>(host.get()), packed,
                             down, cudaMemcpyDeviceToHost, ln.stream),
             "download");
    BFV_CUDA(cudaStreamSynchronize(ln.stream), "encrypt");
    if (status & 1) return fail(CUHE_INVALID_ARGUMENT, "slot value not below the plaintext modulus");
    if (status & 2) return fail(CUHE_RANGE, "keystream draw rejected (eight bytes of 255): encrypt again with a new key");
    if (direct) {
      PolySource staged;
      staged.contiguous = ln.host_stage;
      staged.poly_bytes = in_bytes;
      copy_polys(staged, 0, cc * 2, out + c0 * 2 * in_bytes, 8, 21);
    } else {
      for (size_t k = 0; k < cc * 2; ++k)
        std::memcpy(out + (c0 * 2 + k) * in_bytes, reinterpret_cast<const uint8_t*>(host.get() + k * out_words),
                    in_bytes);
    }
  }
  return CUHE_OK;
}

}  // namespace

extern "C" {

int cuhe_bfv_encrypt(cuhe_bfv_ring* r, const uint8_t* pk, uint64_t t, const uint32_t* slots, const int8_t* u,
                     const int8_t* e, uint64_t count, uint8_t* out) {
  return encrypt_impl(r, pk, t, slots, u, e, nullptr, count, out);
}

int cuhe_bfv_encrypt_keyed(cuhe_bfv_ring* r, const uint8_t* pk, uint64_t t, const uint32_t* slots,
                           const uint8_t* key, const uint8_t* nonce, unsigned eta, uint64_t count, uint8_t* out) {
  if (!r || !key || !nonce) return fail(CUHE_INVALID_ARGUMENT, "null argument");
  if (eta < 1 || eta > 63) return fail(CUHE_INVALID_ARGUMENT, "eta must be 1..63");
  const uint64_t n = r->plan.n;
  if (n % 8) return fail(CUHE_INVALID_ARGUMENT, "ring degree must be a multiple of 8");
  NoiseKey nk{};
  for (int k = 0; k < 8; ++k)
    nk.key[k] = uint32_t(key[4 * k]) | uint32_t(key[4 * k + 1]) << 8 | uint32_t(key[4 * k + 2]) << 16 |
                uint32_t(key[4 * k + 3]) << 24;
  for (int k = 0; k < 3; ++k)
    nk.nonce[k] = uint32_t(nonce[4 * k]) | uint32_t(nonce[4 * k + 1]) << 8 | uint32_t(nonce[4 * k + 2]) << 16 |
                  uint32_t(nonce[4 * k + 3]) << 24;
  nk.eta = eta;
  nk.first_ct = 0;
  nk.e_blocks = uint32_t(eta <= 31 ? n / 4 : n / 2);
  nk.blocks_per_ct = nk.e_blocks + uint32_t(n / 8);
  if (count > (uint64_t(1) << 32) / nk.blocks_per_ct)
    return fail(CUHE_INVALID_ARGUMENT, "too many ciphertexts for one key: the 32-bit block counter would wrap");
  return encrypt_impl(r, pk, t, slots, nullptr, nullptr, &nk, count, out);
}

}  // extern "C"
