// C ABI of the Paillier / Paillier-Lookup path (see include/cuhe_paillier.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/cuhe_paillier.h"
#include "host_bigint.h"
#include "paillier_kernels.cuh"

using cuhe::host::Limbs;

// Scratch of cuhe_paillier_decode_hamming_static: one popcount per ciphertext
// chunk.  Host code must not pass this name to a kernel (on the host it is a
// stand-in, not a device address); the device address is looked up per device.
static __device__ __align__(256) uint32_t g_static_decode_counts[CUHE_STATIC_DECODE_MAX_CHUNKS];

namespace {

std::string g_create_error;

struct Variant {
  int K, TPI, W;
};

// (K, TPI, W) combinations compiled into the library.
#define CUHE_VARIANTS(X) \
  X(64, 8, 3)            \
  X(64, 8, 4)            \
  X(64, 16, 4)           \
  X(128, 8, 4)           \
  X(128, 16, 3)          \
  X(128, 16, 4)          \
  X(128, 16, 5)          \
  X(128, 32, 3)          \
  X(128, 32, 4)          \
  X(256, 16, 4)          \
  X(256, 32, 3)          \
  X(256, 32, 4)          \
  X(256, 32, 5)

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t reserve(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t grow = std::max(need, size_t(1) << 20);
    cudaError_t e = cudaMalloc(&ptr, grow);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

}  // namespace

struct cuhe_paillier {
  int device = 0;
  int K = 0;
  int n_words = 0;
  int tpi = 0, window = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t* d_consts = nullptr;
  int* d_status = nullptr;
  cuhe::KeyScalars ks{};
  Limbs n, n2;
  Limbs secret_exp;  // empty until set
  bool have_secret = false;
  int32_t* d_ops_n = nullptr;
  int nops_n = 0;
  int32_t* d_ops_sec = nullptr;
  int nops_sec = 0;
  int32_t* d_ops_sec52 = nullptr;  // the secret exponent's schedule for the FP64-pipe kernel's window
  int nops_sec52 = 0;
  uint32_t* d_crt = nullptr;  // CRT constant block, present once the factors are installed
  double* d_crt52 = nullptr;  // per side: M and R52 mod M as 52-bit limbs (FP64-pipe CRT kernel)
  double* d_n52 = nullptr;    // n^2 and R52 mod n^2 as 52-bit limbs, then R52 R and R52 mod n^2 in words
  unsigned long long ninv52 = 0;  // -(n^2)^-1 mod 2^52
  int32_t* d_ops_n52 = nullptr;   // the schedule of n for k_modexp52's window
  int nops_n52 = 0;
  cuhe::CrtScalars cs{};
  bool have_factors = false;
  bool fp64 = true;           // decrypt / decode exponentiations on the FP64 pipe (n^2 of 4096 bits or more)
  bool fp64_small = false;    // ... and for n^2 of 2048 bits (set_fp64(ctx, 2))
  uint32_t* d_gtab = nullptr;
  int message_chunks = 0;
  uint32_t* d_wide = nullptr;  // 16-bit-digit table W[j][D], built on demand (see cuhe_lookup_set_wide_table)
  double* d_wide52 = nullptr;  // ... as 52-bit limbs in the R52 domain (FP64-pipe encryption), with
  double* d_noise52 = nullptr; // the noise table likewise
  int wide_mode = 1;           // 0 never, 1 for large batches when it fits, 2 always
  uint32_t* d_noise = nullptr;
  int noise_entries = 0;
  DeviceBuffer work;
  DeviceBuffer tmp_ops;
  cudaStream_t copy = nullptr;  // host-buffer pipelines: transfers beside the compute
  cudaStream_t side = nullptr;  // and a second compute stream (created on first use)
  std::string error;
  std::mutex mu;
};

namespace {

int fail(cuhe_paillier* ctx, int code, const std::string& msg) {
  if (ctx) ctx->error = msg; else g_create_error = msg;
  return code;
}

int cuda_fail(cuhe_paillier* ctx, cudaError_t e, const char* where) {
  return fail(ctx, CUHE_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorName(e) + " (" +
                                         cudaGetErrorString(e) + ")");
}

#define CUHE_CUDA(ctx, call, where)                   \
  do {                                                \
    cudaError_t _e = (call);                          \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, where); \
  } while (0)

// ---- kernel launchers -----------------------------------------------------

template <int K, int TPI, int W>
size_t modexp_smem() {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  return size_t(5 * K + IPB * cuhe::inst_stride_words<K>((1 << (W - 1)) + 1)) * 4;
}

template <int K, int TPI, int W>
cudaError_t launch_modexp(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* aux, uint32_t* out,
                          long long count, const int32_t* ops, int nops, int mode, int pop_words) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = modexp_smem<K, TPI, W>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp<K, TPI, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_modexp<K, TPI, W><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      base, aux, K, out, count, ctx->d_consts, ctx->ks, ops, nops, mode, pop_words, ctx->d_status);
  return cudaGetLastError();
}

template <int KH, int TPI, int W>
size_t modexp_crt_smem() {
  constexpr int IPB = cuhe::kBlockThreads / (2 * TPI);
  return size_t(7 * 2 * KH + IPB * 2 * (((1 << (W - 1)) + 1) * KH + 4)) * 4;
}

// CRT decrypt / decode: KH = K/2 words per side, TPI lanes per side.
template <int KH, int TPI, int W>
cudaError_t launch_modexp_crt(cuhe_paillier* ctx, const uint32_t* base, uint32_t* out, long long count,
                              int mode, int pop_words) {
  constexpr int IPB = cuhe::kBlockThreads / (2 * TPI);
  const size_t smem = modexp_crt_smem<KH, TPI, W>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp_crt<KH, TPI, W>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_modexp_crt<KH, TPI, W><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      base, out, count, ctx->d_consts, ctx->ks, ctx->d_crt, ctx->cs, ctx->d_ops_sec, ctx->nops_sec, mode,
      pop_words, ctx->d_status);
  return cudaGetLastError();
}

// The same with both exponentiations on the FP64 pipe (KH / 16 lanes per
// side, ten 52-bit limbs per lane; a 3-bit window, with the secret
// exponent's own schedule).  Independent of the integer kernels' (threads
// per instance, window) tuning.
constexpr int kCrt52Window = 3;
template <int KH, int W>
size_t modexp_crt52_smem() {
  constexpr int TPI = KH / 16, K52 = 5 * KH / 8;
  constexpr int IPB = cuhe::kBlockThreads / (2 * TPI);
  return size_t(7 * 2 * KH) * 4 + size_t(K52 + IPB * 2 * (((1 << (W - 1)) + 1) * K52 + 2)) * 8;
}

template <int KH, int W>
cudaError_t launch_modexp_crt52(cuhe_paillier* ctx, const uint32_t* base, uint32_t* out, long long count,
                                int mode, int pop_words) {
  constexpr int IPB = cuhe::kBlockThreads / (2 * (KH / 16));
  const size_t smem = modexp_crt52_smem<KH, W>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp_crt52<KH, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_modexp_crt52<KH, W><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      base, out, count, ctx->d_consts, ctx->ks, ctx->d_crt, ctx->cs, ctx->d_crt52, ctx->d_ops_sec52,
      ctx->nops_sec52, mode, pop_words, ctx->d_status);
  return cudaGetLastError();
}

// The exponentiation mod n^2 on the FP64 pipe (no factors needed).
template <int K, int W>
size_t modexp52_smem() {
  constexpr int TPI = K / 16, K52 = 5 * K / 8;
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  return size_t(6 * K) * 4 + size_t(K52 + IPB * (((1 << (W - 1)) + 1) * K52 + 2)) * 8;
}

template <int K, int W>
cudaError_t launch_modexp52(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* aux, uint32_t* out,
                            long long count, const int32_t* ops, int nops, int mode, int pop_words) {
  constexpr int IPB = cuhe::kBlockThreads / (K / 16);
  const size_t smem = modexp52_smem<K, W>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp52<K, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_modexp52<K, W><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      base, aux, K, out, count, ctx->d_consts, ctx->ks, ctx->d_n52, ctx->ninv52, ops, nops, mode, pop_words,
      ctx->d_status);
  return cudaGetLastError();
}

// k_modexp52 for this context's width when the FP64 pipe is selected for it
// (n^2 of 4096 or 8192 bits; 2048 bits only with set_fp64(ctx, 2)), else null.
using Modexp52 = cudaError_t (*)(cuhe_paillier*, const uint32_t*, const uint32_t*, uint32_t*, long long,
                                 const int32_t*, int, int, int);
Modexp52 direct52(const cuhe_paillier* ctx) {
  if (!ctx->fp64 || !ctx->d_n52) return nullptr;
  if (ctx->K == 64 && ctx->fp64_small) return &launch_modexp52<64, kCrt52Window>;
  if (ctx->K == 128) return &launch_modexp52<128, kCrt52Window>;
  if (ctx->K == 256) return &launch_modexp52<256, kCrt52Window>;
  return nullptr;
}

// encode_hamming_server on the FP64 pipe: queries to R52 Montgomery limbs,
// then one product per output.
template <int K>
cudaError_t launch_outer52(cuhe_paillier* ctx, const uint32_t* query, long long nq, double* q52,
                           const uint32_t* index, long long nx, uint32_t* out) {
  constexpr int TPI = K / 16, K52 = 5 * K / 8, IPB = cuhe::kBlockThreads / TPI;
  const size_t csmem = size_t(K + IPB * K) * 4;
  cuhe::k_to_mont52<K><<<dim3(unsigned((nq + IPB - 1) / IPB)), cuhe::kBlockThreads, csmem, ctx->stream>>>(
      query, nq, q52, ctx->d_consts, ctx->ks, reinterpret_cast<const uint32_t*>(ctx->d_n52 + 2 * K52),
      ctx->d_status);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smem = size_t(K52 + IPB * K52) * 8;
  const long long bx = (nx + IPB - 1) / IPB;
  for (long long q0 = 0; q0 < nq; q0 += 65535) {
    const long long qn = std::min<long long>(65535, nq - q0);
    cuhe::k_mulmod_outer52<K><<<dim3(unsigned(bx), unsigned(qn)), cuhe::kBlockThreads, smem, ctx->stream>>>(
        q52 + q0 * K52, index, nx, out + q0 * nx * K, ctx->d_consts, ctx->d_n52, ctx->ninv52, ctx->d_status);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

using Outer52 = cudaError_t (*)(cuhe_paillier*, const uint32_t*, long long, double*, const uint32_t*, long long,
                                uint32_t*);
Outer52 outer52(const cuhe_paillier* ctx) {
  if (!direct52(ctx)) return nullptr;
  if (ctx->K == 64) return &launch_outer52<64>;
  if (ctx->K == 128) return &launch_outer52<128>;
  if (ctx->K == 256) return &launch_outer52<256>;
  return nullptr;
}

// The 16-bit-digit table and the noise table as 52-bit limbs in the R52
// domain (k_wide_table52 row by row, k_to_mont52 from the 32-bit Montgomery
// form), and encryption from them.
template <int K>
cudaError_t build_wide52(cuhe_paillier* ctx, double* wide52, double* noise52) {
  constexpr int TPI = K / 16, K52 = 5 * K / 8, IPB = cuhe::kBlockThreads / TPI;
  const uint32_t* r52w = reinterpret_cast<const uint32_t*>(ctx->d_n52 + 2 * K52) + K;
  const size_t smem = size_t(K + IPB * K) * 4;
  for (int j = 0; j < (ctx->message_chunks + 1) / 2; ++j) {
    cuhe::k_wide_table52<K><<<dim3(65536 / IPB), cuhe::kBlockThreads, smem, ctx->stream>>>(
        ctx->d_gtab, ctx->message_chunks, j, wide52, ctx->d_consts, ctx->ks, r52w);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  // no noise table: encryption reports every noise index as out of range
  if (ctx->noise_entries == 0) return cudaSuccess;
  cuhe::k_to_mont52<K><<<dim3(unsigned((ctx->noise_entries + IPB - 1) / IPB)), cuhe::kBlockThreads, smem,
                         ctx->stream>>>(ctx->d_noise, ctx->noise_entries, noise52, ctx->d_consts, ctx->ks, r52w,
                                        ctx->d_status);
  return cudaGetLastError();
}

template <int K>
cudaError_t launch_lookup52(cuhe_paillier* ctx, const uint8_t* bits, int embed_len, int chunk_len, int chunk_num,
                            const uint32_t* plain, long long count, const uint8_t* idx, uint32_t* out) {
  constexpr int TPI = K / 16, K52 = 5 * K / 8, IPB = cuhe::kBlockThreads / TPI;
  const size_t rows_bytes = size_t(IPB) * cuhe::lookup_rows_stride(ctx->message_chunks) * 2;
  const size_t smem = size_t(K52 + IPB * (K52 + 2)) * 8 + ((rows_bytes + 15) & ~size_t(15));
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_lookup_encrypt52<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  cuhe::k_lookup_encrypt52<K><<<dim3(unsigned((count + IPB - 1) / IPB)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      bits, embed_len, chunk_len, chunk_num, plain, K, count, ctx->message_chunks, ctx->d_wide52, ctx->d_noise52,
      ctx->noise_entries, idx, out, ctx->d_n52, ctx->ninv52, ctx->d_status);
  return cudaGetLastError();
}

struct Lookup52 {
  cudaError_t (*build)(cuhe_paillier*, double*, double*);
  cudaError_t (*launch)(cuhe_paillier*, const uint8_t*, int, int, int, const uint32_t*, long long, const uint8_t*,
                        uint32_t*);
};
bool lookup52(const cuhe_paillier* ctx, Lookup52* l) {
  if (!direct52(ctx)) return false;
  if (ctx->K == 64) *l = {&build_wide52<64>, &launch_lookup52<64>};
  else if (ctx->K == 128) *l = {&build_wide52<128>, &launch_lookup52<128>};
  else if (ctx->K == 256) *l = {&build_wide52<256>, &launch_lookup52<256>};
  else return false;
  return true;
}

template <int K>
cudaError_t prepare_tasks52(int device, int* grid) {
  const size_t smem = modexp52_smem<K, kCrt52Window>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp52_tasks<K, kCrt52Window>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cuhe::k_modexp52_tasks<K, kCrt52Window>,
                                                    cuhe::kBlockThreads, smem);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  *grid = std::max(1, per_sm) * sms;
  return cudaSuccess;
}

template <int K>
cudaError_t launch_tasks52(const cuhe::ModexpTask* tasks, int ntasks, long long units, unsigned long long* counter,
                           int* status, int grid, cudaStream_t stream) {
  cuhe::k_modexp52_tasks<K, kCrt52Window><<<grid, cuhe::kBlockThreads, modexp52_smem<K, kCrt52Window>(), stream>>>(
      tasks, ntasks, units, counter, status);
  return cudaGetLastError();
}

template <int K, int TPI>
cudaError_t launch_modexp_var(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* exps, int exp_words,
                              int windows, uint32_t* out, long long count) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(2 * K + IPB * cuhe::inst_stride_words<K>(17)) * 4;
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp_var<K, TPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_modexp_var<K, TPI><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      base, exps, exp_words, windows, out, count, ctx->d_consts, ctx->ks, ctx->d_status);
  return cudaGetLastError();
}

template <int K, int TPI>
cudaError_t launch_mulmod(cuhe_paillier* ctx, const uint32_t* a, const uint32_t* b, uint32_t* out,
                          long long count) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(K + IPB * cuhe::inst_stride_words<K>(1)) * 4;
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_mulmod<K, TPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_mulmod<K, TPI><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      a, b, out, count, ctx->d_consts, ctx->ks, ctx->d_status);
  return cudaGetLastError();
}

template <int K, int TPI>
cudaError_t launch_convert(cuhe_paillier* ctx, const uint32_t* in, uint32_t* out, long long count, int to_mont) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(K) * 4;
  const long long blocks = (count + IPB - 1) / IPB;
  cuhe::k_convert<K, TPI><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      in, out, count, ctx->d_consts, ctx->ks, to_mont, ctx->d_status);
  return cudaGetLastError();
}

template <int K, int TPI>
cudaError_t launch_outer(cuhe_paillier* ctx, const uint32_t* qmont, long long nq, const uint32_t* index,
                         long long nx, uint32_t* out) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(K) * 4;
  const long long bx = (nx + IPB - 1) / IPB;
  for (long long q0 = 0; q0 < nq; q0 += 65535) {
    const long long qn = std::min<long long>(65535, nq - q0);
    cuhe::k_mulmod_outer<K, TPI><<<dim3(unsigned(bx), unsigned(qn)), cuhe::kBlockThreads, smem, ctx->stream>>>(
        qmont + q0 * K, qn, index, nx, out + q0 * nx * K, ctx->d_consts, ctx->ks, ctx->d_status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int K, int TPI>
cudaError_t launch_lookup(cuhe_paillier* ctx, const uint8_t* bits, int embed_len, int chunk_len, int chunk_num,
                          const uint32_t* plain, long long count, const uint8_t* idx, uint32_t* out) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t rows_bytes = size_t(IPB) * cuhe::lookup_rows_stride(ctx->message_chunks) * 2;
  const size_t smem = size_t(K + IPB * cuhe::inst_stride_words<K>(1)) * 4 + ((rows_bytes + 15) & ~size_t(15));
  const bool wide = ctx->d_wide != nullptr;
  auto kernel = wide ? cuhe::k_lookup_encrypt<K, TPI, true> : cuhe::k_lookup_encrypt<K, TPI, false>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const long long blocks = (count + IPB - 1) / IPB;
  kernel<<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      bits, embed_len, chunk_len, chunk_num, plain, K, count, ctx->message_chunks, wide ? ctx->d_wide : ctx->d_gtab,
      ctx->d_noise, ctx->noise_entries, idx, out, ctx->d_consts, ctx->ks, ctx->d_status);
  return cudaGetLastError();
}

// W[j][D] = G[2j][D mod 256] * G[2j+1][D / 256] for every 16-bit D.
template <int K, int TPI>
cudaError_t launch_wide_table(cuhe_paillier* ctx, uint32_t* wide) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(IPB * cuhe::inst_stride_words<K>(1)) * 4;
  const long long entries = (long long)((ctx->message_chunks + 1) / 2) * 65536;
  cuhe::k_wide_table<K, TPI><<<dim3(unsigned((entries + IPB - 1) / IPB)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      ctx->d_gtab, ctx->message_chunks, wide, ctx->d_consts, ctx->ks);
  return cudaGetLastError();
}

template <int K, int TPI>
cudaError_t launch_table_rows(cuhe_paillier* ctx, const uint32_t* bases, int rows, uint32_t* gtab) {
  constexpr int IPB = cuhe::kBlockThreads / TPI;
  const size_t smem = size_t(IPB * cuhe::inst_stride_words<K>(2)) * 4;
  const long long blocks = ((long long)rows * 16 + IPB - 1) / IPB;
  cuhe::k_table_rows<K, TPI><<<dim3(unsigned(blocks)), cuhe::kBlockThreads, smem, ctx->stream>>>(
      bases, rows, gtab, ctx->d_consts, ctx->ks);
  return cudaGetLastError();
}

// Persistent mixed launch: shared memory attribute and a grid of one wave of
// resident CTAs (SMs x CTAs per SM).
template <int K, int TPI, int W>
cudaError_t prepare_tasks(int device, int* grid) {
  const size_t smem = modexp_smem<K, TPI, W>();
  cudaError_t e = cudaFuncSetAttribute(cuhe::k_modexp_tasks<K, TPI, W>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cuhe::k_modexp_tasks<K, TPI, W>, cuhe::kBlockThreads,
                                                    smem);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  *grid = std::max(1, per_sm) * sms;
  return cudaSuccess;
}

template <int K, int TPI, int W>
cudaError_t launch_tasks(const cuhe::ModexpTask* tasks, int ntasks, long long units, unsigned long long* counter,
                         int* status, int grid, cudaStream_t stream) {
  cuhe::k_modexp_tasks<K, TPI, W><<<grid, cuhe::kBlockThreads, modexp_smem<K, TPI, W>(), stream>>>(
      tasks, ntasks, units, counter, status);
  return cudaGetLastError();
}

// Runtime dispatch over the compiled variants.
struct Dispatch {
  cudaError_t (*modexp)(cuhe_paillier*, const uint32_t*, const uint32_t*, uint32_t*, long long, const int32_t*,
                        int, int, int) = nullptr;
  cudaError_t (*modexp_var)(cuhe_paillier*, const uint32_t*, const uint32_t*, int, int, uint32_t*, long long) = nullptr;
  cudaError_t (*modexp_crt)(cuhe_paillier*, const uint32_t*, uint32_t*, long long, int, int) = nullptr;
  cudaError_t (*mulmod)(cuhe_paillier*, const uint32_t*, const uint32_t*, uint32_t*, long long) = nullptr;
  cudaError_t (*convert)(cuhe_paillier*, const uint32_t*, uint32_t*, long long, int) = nullptr;
  cudaError_t (*outer)(cuhe_paillier*, const uint32_t*, long long, const uint32_t*, long long, uint32_t*) = nullptr;
  cudaError_t (*lookup)(cuhe_paillier*, const uint8_t*, int, int, int, const uint32_t*, long long, const uint8_t*,
                        uint32_t*) = nullptr;
  cudaError_t (*table_rows)(cuhe_paillier*, const uint32_t*, int, uint32_t*) = nullptr;
  cudaError_t (*wide_table)(cuhe_paillier*, uint32_t*) = nullptr;
  cudaError_t (*prepare_tasks)(int, int*) = nullptr;
  cudaError_t (*launch_tasks)(const cuhe::ModexpTask*, int, long long, unsigned long long*, int*, int,
                              cudaStream_t) = nullptr;
};

bool find_dispatch(int K, int TPI, int W, Dispatch* d) {
#define CUHE_MATCH(k, t, w)                                        \
  if (K == k && TPI == t && W == w) {                              \
    d->modexp = &launch_modexp<k, t, w>;                           \
    d->modexp_var = &launch_modexp_var<k, t>;                      \
    d->modexp_crt = &launch_modexp_crt<k / 2, t / 2, w>;           \
    d->mulmod = &launch_mulmod<k, t>;                              \
    d->convert = &launch_convert<k, t>;                            \
    d->outer = &launch_outer<k, t>;                                \
    d->lookup = &launch_lookup<k, t>;                              \
    d->table_rows = &launch_table_rows<k, t>;                      \
    d->wide_table = &launch_wide_table<k, t>;                      \
    d->prepare_tasks = &prepare_tasks<k, t, w>;                    \
    d->launch_tasks = &launch_tasks<k, t, w>;                      \
    return true;                                                   \
  }
  CUHE_VARIANTS(CUHE_MATCH)
#undef CUHE_MATCH
  return false;
}

// Exponentiation by the secret exponent (decrypt / decode): the CRT kernel
// when the factorisation is installed, else the direct kernel mod n^2.
cudaError_t secret_modexp(cuhe_paillier* ctx, const Dispatch& d, const uint32_t* base, uint32_t* out,
                          long long count, int mode, int pop_words) {
  if (ctx->have_factors && ctx->fp64) {
    // n^2 of 2048 bits (1024-bit sides) stays on the integer pipe: measured faster there
    if (ctx->K == 64 && ctx->fp64_small) return launch_modexp_crt52<32, kCrt52Window>(ctx, base, out, count, mode, pop_words);
    if (ctx->K == 128) return launch_modexp_crt52<64, kCrt52Window>(ctx, base, out, count, mode, pop_words);
    if (ctx->K == 256) return launch_modexp_crt52<128, kCrt52Window>(ctx, base, out, count, mode, pop_words);
  }
  if (ctx->have_factors) return d.modexp_crt(ctx, base, out, count, mode, pop_words);
  if (Modexp52 f = direct52(ctx)) return f(ctx, base, nullptr, out, count, ctx->d_ops_sec52, ctx->nops_sec52, mode,
                                           pop_words);
  return d.modexp(ctx, base, nullptr, out, count, ctx->d_ops_sec, ctx->nops_sec, mode, pop_words);
}

void default_tuning(int K, int* tpi, int* w) {
  *w = 4;
  *tpi = K / 8;  // eight limbs per lane
}

// ---- staging of host buffers ----------------------------------------------

struct Staged {
  const void* src;
  void* dev;
  size_t bytes;
  bool in;    // copy host->device before
  bool out;   // copy device->host after
  void* host_out;
};

class Stager {
 public:
  explicit Stager(cuhe_paillier* ctx) : ctx_(ctx) {}
  // Reserve space for all buffers first, then bind.
  void add(const void* host_or_dev, size_t bytes, bool in, bool out) {
    items_.push_back({host_or_dev, nullptr, bytes, in, out, const_cast<void*>(host_or_dev)});
  }
  // Device scratch that lives in the workspace for the duration of the call.
  void add_scratch(size_t bytes) { items_.push_back({nullptr, nullptr, bytes, false, false, nullptr}); }
  int bind() {
    size_t total = 0;
    for (auto& it : items_) {
      if ((!it.src || !is_device_pointer(it.src)) && it.bytes) total += (it.bytes + 255) & ~size_t(255);
    }
    if (total) {
      cudaError_t e = ctx_->work.reserve(total);
      if (e != cudaSuccess) return cuda_fail(ctx_, e, "workspace allocation");
    }
    size_t off = 0;
    for (auto& it : items_) {
      if (!it.bytes) { it.dev = nullptr; continue; }
      if (!it.src) {
        it.dev = static_cast<char*>(ctx_->work.ptr) + off;
        off += (it.bytes + 255) & ~size_t(255);
        continue;
      }
      if (is_device_pointer(it.src)) {
        it.dev = const_cast<void*>(it.src);
        it.in = it.out = false;
      } else {
        it.dev = static_cast<char*>(ctx_->work.ptr) + off;
        off += (it.bytes + 255) & ~size_t(255);
        staged_ = true;
        if (it.in) {
          cudaError_t e = cudaMemcpyAsync(it.dev, it.src, it.bytes, cudaMemcpyHostToDevice, ctx_->stream);
          if (e != cudaSuccess) return cuda_fail(ctx_, e, "host to device copy");
        }
      }
    }
    return CUHE_OK;
  }
  void* dev(size_t i) const { return items_[i].dev; }
  int finish() {
    for (auto& it : items_) {
      if (it.out) {
        cudaError_t e = cudaMemcpyAsync(it.host_out, it.dev, it.bytes, cudaMemcpyDeviceToHost, ctx_->stream);
        if (e != cudaSuccess) return cuda_fail(ctx_, e, "device to host copy");
      }
    }
    if (staged_) {
      cudaError_t e = cudaStreamSynchronize(ctx_->stream);
      if (e != cudaSuccess) return cuda_fail(ctx_, e, "stream synchronize");
    }
    return CUHE_OK;
  }
  bool staged() const { return staged_; }
  // item i lives in the workspace (its caller buffer is host memory)
  bool is_staged(size_t i) const { return items_[i].src && items_[i].dev != items_[i].src; }

 private:
  cuhe_paillier* ctx_;
  std::vector<Staged> items_;
  bool staged_ = false;
};

// Host buffers of at least this many bytes move piece by piece beside the
// compute instead of before or after it.
constexpr size_t kPipeBytes = size_t(64) << 20;

// The context's copy and side streams, created on first use; both start
// after the work already queued on the context's stream (which may still
// use the workspace the pipeline is about to fill).
int pipeline_streams(cuhe_paillier* ctx) {
  for (cudaStream_t* st : {&ctx->copy, &ctx->side})
    if (!*st) CUHE_CUDA(ctx, cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "pipeline stream");
  cudaEvent_t ready;
  CUHE_CUDA(ctx, cudaEventCreateWithFlags(&ready, cudaEventDisableTiming), "event");
  cudaError_t e = cudaEventRecord(ready, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy, ready, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->side, ready, 0);
  cudaEventDestroy(ready);
  CUHE_CUDA(ctx, e, "pipeline order");
  return CUHE_OK;
}

// `waiter` waits for the work queued so far on `from`.
cudaError_t stream_after(cudaStream_t waiter, cudaStream_t from) {
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(ev, from);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(waiter, ev, 0);
  cudaEventDestroy(ev);
  return e;
}

// The 16-bit-digit encryption table (W[j][D] = G[2j][D mod 256] *
// G[2j+1][D / 256], 65,536 rows per pair of 8-bit digits): half the table
// products per ciphertext, for (message_chunks + 1) / 2 * 65,536 * 4K bytes
// (4 GiB at key_len 1024) and one product per entry to build, which about
// 150,000 encryptions repay.  Mode 1 builds it for a call of at least
// kWideMinItems ciphertexts when it takes at most kWideMaxBytes and a quarter
// of the free device memory (else the 8-bit table serves); mode 2 builds it
// for any call and fails without memory; mode 0 never.
constexpr long long kWideMinItems = 1 << 16;
constexpr size_t kWideMaxBytes = size_t(8) << 30;

int ensure_wide_table(cuhe_paillier* ctx, const Dispatch& d, long long items);

int check_status(cuhe_paillier* ctx, bool synchronous) {
  // Range errors are reported by the kernels through d_status; reading it
  // needs a synchronisation, done only for calls that already synchronise.
  if (!synchronous) return CUHE_OK;
  int status = 0;
  cudaError_t e = cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "status read");
  if (status) {
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    return fail(ctx, CUHE_RANGE, "input outside its valid range (ciphertext >= n^2, plaintext >= n, or noise index)");
  }
  return CUHE_OK;
}

int upload_schedule(cuhe_paillier* ctx, const Limbs& e, int32_t** dptr, int* nops, int window = 0) {
  std::vector<int32_t> ops = cuhe::host::window_schedule(e, window ? window : ctx->window);
  if (*dptr) cudaFree(*dptr);
  *dptr = nullptr;
  *nops = int(ops.size());
  if (ops.empty()) return CUHE_OK;
  CUHE_CUDA(ctx, cudaMalloc(dptr, ops.size() * sizeof(int32_t)), "schedule allocation");
  CUHE_CUDA(ctx, cudaMemcpy(*dptr, ops.data(), ops.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
            "schedule upload");
  return CUHE_OK;
}

// k_modexp52's constants: n^2 and R52 mod n^2 as K52 = 5K/8 limbs of 52 bits
// (doubles), then R52 R mod n^2 as K words; R52 = 2^(52 K52), R = 2^(32K).
int setup_direct52(cuhe_paillier* ctx) {
  const size_t k = size_t(ctx->K), k52 = 5 * k / 8;
  Limbs one(k, 0u);
  one[0] = 1u;
  std::vector<double> block(2 * k52 + k, 0.0);
  auto put52 = [&](size_t row, const Limbs& v) {
    for (size_t i = 0; i < k52; ++i) {
      uint64_t limb = 0;
      for (int b = 0; b < 52; ++b) {
        const size_t bit = 52 * i + size_t(b);
        if (bit / 32 < v.size() && ((v[bit / 32] >> (bit % 32)) & 1u)) limb |= 1ull << b;
      }
      block[row * k52 + i] = double(limb);
    }
  };
  put52(0, ctx->n2);
  put52(1, cuhe::host::shift_mod(one, 52 * k52, ctx->n2));
  const Limbs r52r = cuhe::host::shift_mod(one, 52 * k52 + 32 * k, ctx->n2);
  std::memcpy(block.data() + 2 * k52, r52r.data(), 4 * k);
  const Limbs r52 = cuhe::host::shift_mod(one, 52 * k52, ctx->n2);
  std::memcpy(block.data() + 2 * k52 + k / 2, r52.data(), 4 * k);
  const uint64_t m0 = (uint64_t(ctx->n2[1]) << 32) | ctx->n2[0];
  uint64_t inv = m0;
  for (int it = 0; it < 6; ++it) inv *= 2 - m0 * inv;
  ctx->ninv52 = (0 - inv) & ((1ull << 52) - 1);
  CUHE_CUDA(ctx, cudaMalloc(&ctx->d_n52, block.size() * 8), "constants allocation");
  CUHE_CUDA(ctx, cudaMemcpy(ctx->d_n52, block.data(), block.size() * 8, cudaMemcpyHostToDevice), "constants upload");
  return CUHE_OK;
}

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

}  // namespace

extern "C" {

const char* cuhe_version(void) { return "cuhe_b200 paillier 1"; }

int cuhe_window_schedule(const uint32_t* exponent, int exponent_words, int window, int32_t* ops, int capacity) {
  if (!exponent || exponent_words <= 0 || window < 1 || window > 8 || capacity < 0) return CUHE_INVALID_ARGUMENT;
  Limbs e(exponent, exponent + exponent_words);
  std::vector<int32_t> sched = cuhe::host::window_schedule(e, window);
  for (int i = 0; i < capacity && i < int(sched.size()); ++i) ops[i] = sched[size_t(i)];
  return int(sched.size());
}

const char* cuhe_last_error(const cuhe_paillier* ctx) {
  return ctx ? ctx->error.c_str() : g_create_error.c_str();
}

int cuhe_paillier_words(const cuhe_paillier* ctx) { return ctx ? ctx->K : 0; }

int cuhe_paillier_create(const uint32_t* n_in, int n_words, int device, cuhe_paillier** out) {
  if (!out || !n_in || n_words <= 0) return fail(nullptr, CUHE_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  Limbs n(n_in, n_in + n_words);
  while (!n.empty() && n.back() == 0) n.pop_back();
  if (n.empty() || (n[0] & 1u) == 0) return fail(nullptr, CUHE_INVALID_ARGUMENT, "n must be odd and nonzero");
  const size_t nbits = cuhe::host::bit_length(n);
  int K = 0;
  for (int cand : {64, 128, 256}) {
    if (nbits <= size_t(cand) * 16) { K = cand; break; }
  }
  if (!K) return fail(nullptr, CUHE_INVALID_ARGUMENT, "n wider than 4096 bits is not supported");
  int count = 0;
  cudaError_t ce = cudaGetDeviceCount(&count);
  if (ce != cudaSuccess || count == 0) return fail(nullptr, CUHE_CUDA_ERROR, "no CUDA device available");
  if (device < 0 || device >= count) return fail(nullptr, CUHE_INVALID_ARGUMENT, "invalid device ordinal");
  DeviceGuard guard(device);

  auto* ctx = new (std::nothrow) cuhe_paillier();
  if (!ctx) return fail(nullptr, CUHE_OUT_OF_MEMORY, "context allocation");
  ctx->device = device;
  ctx->K = K;
  ctx->n_words = K / 2;
  default_tuning(K, &ctx->tpi, &ctx->window);

  const size_t k = size_t(K);
  Limbs nk = cuhe::host::resized(n.data(), n.size(), k);
  Limbs n2 = cuhe::host::mul(nk, nk, k);
  ctx->n = nk;
  ctx->n2 = n2;
  // R mod N = 2^(32K) mod N via doubling from 1; likewise R^2 = R * 2^(32K)
  Limbs one(k, 0u);
  one[0] = 1u;
  Limbs rm = cuhe::host::shift_mod(one, 32 * k, n2);
  Limbs r2 = cuhe::host::shift_mod(rm, 32 * k, n2);
  Limbs rmn = cuhe::host::shift_mod(one, 32 * k, nk);
  Limbs r2n = cuhe::host::shift_mod(rmn, 32 * k, nk);
  Limbs nneg(k, 0u);
  cuhe::host::sub_in_place(nneg, nk);  // 2^(32K) - n (mod 2^(32K))
  Limbs nr = cuhe::host::shift_mod(nk, 32 * k, n2);  // n < n^2
  Limbs multr(k, 0u);

  std::vector<uint32_t> block(size_t(cuhe::C_ROWS) * k, 0u);
  auto put = [&](int row, const Limbs& v) { std::memcpy(block.data() + size_t(row) * k, v.data(), 4 * k); };
  put(cuhe::C_N2, n2);
  put(cuhe::C_R2, r2);
  put(cuhe::C_ONE, one);
  put(cuhe::C_RM, rm);
  put(cuhe::C_N, nk);
  put(cuhe::C_R2N, r2n);
  put(cuhe::C_NNEG, nneg);
  put(cuhe::C_NR, nr);
  put(cuhe::C_MULTR, multr);
  ctx->ks.ninv2 = 0u - cuhe::host::inv32(n2[0]);
  ctx->ks.ninv1 = 0u - cuhe::host::inv32(nk[0]);
  ctx->ks.ndiv = cuhe::host::inv32(nk[0]);
  ctx->ks.mult_is_zero = 1u;

  cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_consts, block.size() * 4);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->d_consts, block.data(), block.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_status, 0, sizeof(int));
  if (e != cudaSuccess) {
    int rc = cuda_fail(nullptr, e, "context setup");
    cuhe_paillier_destroy(ctx);
    return rc;
  }
  ctx->stream = ctx->own_stream;
  if (upload_schedule(ctx, nk, &ctx->d_ops_n, &ctx->nops_n) != CUHE_OK ||
      upload_schedule(ctx, nk, &ctx->d_ops_n52, &ctx->nops_n52, kCrt52Window) != CUHE_OK ||
      setup_direct52(ctx) != CUHE_OK) {
    g_create_error = ctx->error;
    cuhe_paillier_destroy(ctx);
    return CUHE_CUDA_ERROR;
  }
  *out = ctx;
  return CUHE_OK;
}

void cuhe_paillier_destroy(cuhe_paillier* ctx) {
  if (!ctx) return;
  DeviceGuard guard(ctx->device);
  if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
  if (ctx->stream && ctx->stream != ctx->own_stream) cudaStreamSynchronize(ctx->stream);
  cudaFree(ctx->d_consts);
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_ops_n);
  cudaFree(ctx->d_ops_sec);
  cudaFree(ctx->d_ops_sec52);
  cudaFree(ctx->d_crt);
  cudaFree(ctx->d_crt52);
  cudaFree(ctx->d_n52);
  cudaFree(ctx->d_ops_n52);
  cudaFree(ctx->d_gtab);
  cudaFree(ctx->d_wide);
  cudaFree(ctx->d_wide52);
  cudaFree(ctx->d_noise52);
  cudaFree(ctx->d_noise);
  for (cudaStream_t st : {ctx->copy, ctx->side})
    if (st) cudaStreamSynchronize(st);
  ctx->work.release();
  ctx->tmp_ops.release();
  for (cudaStream_t st : {ctx->copy, ctx->side})
    if (st) cudaStreamDestroy(st);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

int cuhe_paillier_set_stream(cuhe_paillier* ctx, void* stream) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return CUHE_OK;
}

int cuhe_synchronize(cuhe_paillier* ctx) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
  return check_status(ctx, true);
}

int cuhe_paillier_set_tuning(cuhe_paillier* ctx, int tpi, int window) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  int dt, dw;
  default_tuning(ctx->K, &dt, &dw);
  if (!tpi) tpi = dt;
  if (!window) window = dw;
  Dispatch d;
  if (!find_dispatch(ctx->K, tpi, window, &d))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "tuning (threads per instance, window) not compiled for this width");
  const bool changed = window != ctx->window;
  ctx->tpi = tpi;
  ctx->window = window;
  if (changed) {
    int rc = upload_schedule(ctx, ctx->n, &ctx->d_ops_n, &ctx->nops_n);
    if (rc) return rc;
    if (ctx->have_secret) {
      rc = upload_schedule(ctx, ctx->secret_exp, &ctx->d_ops_sec, &ctx->nops_sec);
      if (rc) return rc;
    }
  }
  return CUHE_OK;
}

int cuhe_paillier_get_tuning(const cuhe_paillier* ctx, int* tpi, int* window) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  if (tpi) *tpi = ctx->tpi;
  if (window) *window = ctx->window;
  return CUHE_OK;
}

int cuhe_paillier_set_secret(cuhe_paillier* ctx, const uint32_t* exponent, int exponent_words,
                             const uint32_t* multiplier, int multiplier_words) {
  if (!ctx || !exponent || !multiplier || exponent_words <= 0 || multiplier_words <= 0)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "null secret");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  const size_t k = size_t(ctx->K);
  if (!cuhe::host::fits(exponent, size_t(exponent_words), k))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "secret exponent wider than n^2");
  if (!cuhe::host::fits(multiplier, size_t(multiplier_words), k))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "secret multiplier too wide");
  Limbs e = cuhe::host::resized(exponent, size_t(exponent_words), k);
  Limbs mult = cuhe::host::resized(multiplier, size_t(multiplier_words), k);
  if (cuhe::host::cmp(mult, ctx->n) >= 0) {
    // the reference reduces (x * mult) mod n; reduce the multiplier first
    while (cuhe::host::cmp(mult, ctx->n) >= 0) cuhe::host::sub_in_place(mult, ctx->n);
  }
  Limbs multr = cuhe::host::shift_mod(mult, 32 * k, ctx->n);
  // kernels already queued may still read the previous secret
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "synchronize before secret upload");
  CUHE_CUDA(ctx, cudaMemcpy(ctx->d_consts + size_t(cuhe::C_MULTR) * k, multr.data(), 4 * k, cudaMemcpyHostToDevice),
            "secret upload");
  ctx->ks.mult_is_zero = cuhe::host::is_zero(mult) ? 1u : 0u;
  ctx->secret_exp = e;
  ctx->have_secret = true;
  if (int rc = upload_schedule(ctx, e, &ctx->d_ops_sec52, &ctx->nops_sec52, kCrt52Window)) return rc;
  return upload_schedule(ctx, e, &ctx->d_ops_sec, &ctx->nops_sec);
}

int cuhe_paillier_set_factors(cuhe_paillier* ctx, const uint32_t* p_in, int p_words, const uint32_t* q_in,
                              int q_words) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  if (!p_in && !q_in) {
    ctx->have_factors = false;
    return CUHE_OK;
  }
  if (!p_in || !q_in || p_words <= 0 || q_words <= 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "null factor");
  const size_t k = size_t(ctx->K), kh = k / 2;
  if (!cuhe::host::fits(p_in, size_t(p_words), k) || !cuhe::host::fits(q_in, size_t(q_words), k))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "factor wider than n");
  Limbs p = cuhe::host::resized(p_in, size_t(p_words), k), q = cuhe::host::resized(q_in, size_t(q_words), k);
  Limbs n2k = cuhe::host::resized(ctx->n.data(), ctx->n.size(), 2 * k);
  if (cuhe::host::cmp(cuhe::host::mul(p, q, 2 * k), n2k) != 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "p * q != n");
  if (!(p[0] & 1u) || !(q[0] & 1u) || cuhe::host::bit_length(p) < 2 || cuhe::host::bit_length(q) < 2)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "factors must be odd and greater than 1");
  if (cuhe::host::bit_length(p) > 16 * kh || cuhe::host::bit_length(q) > 16 * kh)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "unbalanced factors: p^2 or q^2 wider than half of n^2");
  Limbs one(kh, 0u);
  one[0] = 1u;
  Limbs side[2] = {cuhe::host::mul(p, p, kh), cuhe::host::mul(q, q, kh)};  // p^2, q^2
  Limbs qinv;
  if (!cuhe::host::mod_inverse_odd(cuhe::host::mod_reduce(side[1], side[0]), side[0], &qinv))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "factors are not coprime");
  std::vector<uint32_t> block(size_t(cuhe::CR_ROWS) * k, 0u);
  auto put_half = [&](int row, int s, const Limbs& v) {
    std::memcpy(block.data() + size_t(row) * k + size_t(s) * kh, v.data(), 4 * kh);
  };
  // FP64-pipe kernel: K52 = 5 KH / 8 limbs of 52 bits per side, R52 = 2^(52 K52)
  const size_t k52 = 5 * kh / 8;
  std::vector<double> block52(2 * 2 * k52, 0.0);
  auto put52 = [&](int s, int row, const Limbs& v) {
    for (size_t i = 0; i < k52; ++i) {
      uint64_t limb = 0;
      for (int b = 0; b < 52; ++b) {
        const size_t bit = 52 * i + size_t(b);
        if (bit / 32 < v.size() && ((v[bit / 32] >> (bit % 32)) & 1u)) limb |= 1ull << b;
      }
      block52[(size_t(s) * 2 + size_t(row)) * k52 + i] = double(limb);
    }
  };
  for (int s = 0; s < 2; ++s) {
    Limbs rm = cuhe::host::shift_mod(one, 32 * kh, side[s]);
    put_half(cuhe::CR_M, s, side[s]);
    put_half(cuhe::CR_RM, s, rm);
    put_half(cuhe::CR_R3, s, cuhe::host::shift_mod(rm, 64 * kh, side[s]));
    put_half(cuhe::CR_R52, s, cuhe::host::shift_mod(one, 52 * k52 + 64 * kh, side[s]));
    ctx->cs.ninv[s] = 0u - cuhe::host::inv32(side[s][0]);
    // -(M^-1) mod 2^52 by Newton's iteration on the low 64 bits of M
    const uint64_t m0 = (uint64_t(side[s][1]) << 32) | side[s][0];
    uint64_t inv = m0;
    for (int it = 0; it < 6; ++it) inv *= 2 - m0 * inv;
    ctx->cs.ninv52[s] = (0 - inv) & ((1ull << 52) - 1);
    put52(s, 0, side[s]);
    put52(s, 1, cuhe::host::shift_mod(one, 52 * k52, side[s]));
  }
  put_half(cuhe::CR_H, 0, cuhe::host::shift_mod(qinv, 32 * kh, side[0]));
  Limbs cq = cuhe::host::shift_mod(cuhe::host::resized(side[1].data(), kh, k), 32 * k, ctx->n2);
  std::memcpy(block.data() + size_t(cuhe::CR_CQ) * k, cq.data(), 4 * k);
  // kernels already queued may still read the previous constants
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "synchronize before CRT constants upload");
  if (!ctx->d_crt) CUHE_CUDA(ctx, cudaMalloc(&ctx->d_crt, block.size() * 4), "CRT constants allocation");
  CUHE_CUDA(ctx, cudaMemcpy(ctx->d_crt, block.data(), block.size() * 4, cudaMemcpyHostToDevice), "CRT constants upload");
  if (!ctx->d_crt52) CUHE_CUDA(ctx, cudaMalloc(&ctx->d_crt52, block52.size() * 8), "CRT constants allocation");
  CUHE_CUDA(ctx, cudaMemcpy(ctx->d_crt52, block52.data(), block52.size() * 8, cudaMemcpyHostToDevice),
            "CRT constants upload");
  ctx->have_factors = true;
  return CUHE_OK;
}

int cuhe_paillier_has_factors(const cuhe_paillier* ctx) { return ctx && ctx->have_factors ? 1 : 0; }

int cuhe_paillier_set_fp64(cuhe_paillier* ctx, int enable) {
  if (!ctx) return CUHE_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->fp64 = enable != 0;
  ctx->fp64_small = enable == 2;
  return CUHE_OK;
}

int cuhe_paillier_get_fp64(const cuhe_paillier* ctx) { return !ctx || !ctx->fp64 ? 0 : ctx->fp64_small ? 2 : 1; }

int cuhe_paillier_encrypt(cuhe_paillier* ctx, const uint32_t* m, const uint32_t* r, uint32_t* c, int64_t count) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!m || !r || !c) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(m, bytes, true, false);
  st.add(r, bytes, true, false);
  st.add(c, bytes, false, true);
  if (int rc = st.bind()) return rc;
  if (Modexp52 f = direct52(ctx)) {
    CUHE_CUDA(ctx, f(ctx, (const uint32_t*)st.dev(1), (const uint32_t*)st.dev(0), (uint32_t*)st.dev(2), count,
                     ctx->d_ops_n52, ctx->nops_n52, cuhe::EXP_ENCRYPT, 0),
              "encrypt launch");
  } else {
    CUHE_CUDA(ctx, d.modexp(ctx, (const uint32_t*)st.dev(1), (const uint32_t*)st.dev(0), (uint32_t*)st.dev(2), count,
                            ctx->d_ops_n, ctx->nops_n, cuhe::EXP_ENCRYPT, 0),
              "encrypt launch");
  }
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

int cuhe_paillier_decrypt(cuhe_paillier* ctx, const uint32_t* c, uint32_t* m, int64_t count) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (!ctx->have_secret) return fail(ctx, CUHE_NOT_READY, "decrypt: secret key not installed");
  if (count == 0) return CUHE_OK;
  if (!c || !m) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(c, bytes, true, false);
  st.add(m, bytes, false, true);
  if (int rc = st.bind()) return rc;
  CUHE_CUDA(ctx, secret_modexp(ctx, d, (const uint32_t*)st.dev(0), (uint32_t*)st.dev(1), count, cuhe::EXP_DECRYPT, 0),
            "decrypt launch");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

int cuhe_paillier_decode_hamming(cuhe_paillier* ctx, const uint32_t* c, int64_t vectors, int chunk_num,
                                 int chunk_len, int64_t* distance) {
  if (!ctx || vectors < 0 || chunk_num <= 0 || chunk_len <= 0 || chunk_len % 32)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid decode layout");
  if (!ctx->have_secret) return fail(ctx, CUHE_NOT_READY, "decode: secret key not installed");
  if (vectors == 0) return CUHE_OK;
  if (!c || !distance) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  if (chunk_len / 32 > ctx->K) return fail(ctx, CUHE_INVALID_ARGUMENT, "chunk_len wider than n^2");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const int64_t total = vectors * chunk_num;
  const size_t cbytes = size_t(total) * ctx->K * 4;
  // A large host input moves in two pieces on the copy stream: the first
  // sixteenth, decoded on the context's stream as soon as it has arrived,
  // and the rest, decoded on the side stream (so the first launch's last
  // wave overlaps the second) while only the first piece's copy is exposed.
  const bool pipe = cbytes >= kPipeBytes && vectors >= 32 && !is_device_pointer(c);
  Stager st(ctx);
  st.add(c, cbytes, !pipe, false);
  st.add_scratch(size_t(total) * 4);  // per-chunk popcounts
  st.add(distance, size_t(vectors) * 8, false, true);
  if (int rc = st.bind()) return rc;
  uint32_t* d_counts = static_cast<uint32_t*>(st.dev(1));
  const uint32_t* d_c = static_cast<const uint32_t*>(st.dev(0));
  if (pipe && st.is_staged(0)) {
    if (int rc = pipeline_streams(ctx)) return rc;
    const int64_t first = std::max<int64_t>(1, vectors / 16) * chunk_num;
    const size_t fbytes = size_t(first) * ctx->K * 4;
    cudaEvent_t arrived[2];
    for (auto& ev : arrived) CUHE_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
    cudaError_t e = cudaMemcpyAsync(const_cast<uint32_t*>(d_c), c, fbytes, cudaMemcpyHostToDevice, ctx->copy);
    if (e == cudaSuccess) e = cudaEventRecord(arrived[0], ctx->copy);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(const_cast<uint32_t*>(d_c) + size_t(first) * ctx->K, c + size_t(first) * ctx->K,
                          cbytes - fbytes, cudaMemcpyHostToDevice, ctx->copy);
    if (e == cudaSuccess) e = cudaEventRecord(arrived[1], ctx->copy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, arrived[0], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->side, arrived[1], 0);
    for (auto& ev : arrived) cudaEventDestroy(ev);
    CUHE_CUDA(ctx, e, "piecewise upload");
    CUHE_CUDA(ctx, secret_modexp(ctx, d, d_c, d_counts, first, cuhe::EXP_DECODE, chunk_len / 32), "decode launch");
    cudaStream_t own = ctx->stream;
    ctx->stream = ctx->side;  // the launchers queue on ctx->stream
    e = secret_modexp(ctx, d, d_c + size_t(first) * ctx->K, d_counts + first, total - first, cuhe::EXP_DECODE,
                      chunk_len / 32);
    ctx->stream = own;
    CUHE_CUDA(ctx, e, "decode launch");
    CUHE_CUDA(ctx, stream_after(ctx->stream, ctx->side), "decode join");
  } else {
    CUHE_CUDA(ctx, secret_modexp(ctx, d, d_c, d_counts, total, cuhe::EXP_DECODE, chunk_len / 32), "decode launch");
  }
  cuhe::k_sum_chunks<<<unsigned((vectors + 255) / 256), 256, 0, ctx->stream>>>(
      d_counts, vectors, chunk_num, reinterpret_cast<long long*>(st.dev(2)));
  CUHE_CUDA(ctx, cudaGetLastError(), "decode reduction");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

}  // extern "C"

namespace {

constexpr int kMaxStaticDevices = 64;
std::mutex g_static_mu;
uint32_t* g_static_counts[kMaxStaticDevices] = {};

// Device address of g_static_decode_counts on `device` (which is current).
int static_counts(cuhe_paillier* ctx, int device, uint32_t** out) {
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (device < 0 || device >= kMaxStaticDevices) return fail(ctx, CUHE_INVALID_ARGUMENT, "device ordinal out of range");
  if (!g_static_counts[device]) {
    void* address = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&address, g_static_decode_counts);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "static scratch address");
    g_static_counts[device] = static_cast<uint32_t*>(address);
  }
  *out = g_static_counts[device];
  return CUHE_OK;
}

}  // namespace

extern "C" {

int cuhe_paillier_decode_hamming_static(cuhe_paillier* ctx, const uint32_t* c, int64_t vectors, int chunk_num,
                                        int chunk_len, int64_t* distance) {
  if (!ctx || vectors < 0 || chunk_num <= 0 || chunk_len <= 0 || chunk_len % 32)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid decode layout");
  if (!ctx->have_secret) return fail(ctx, CUHE_NOT_READY, "decode: secret key not installed");
  if (vectors == 0) return CUHE_OK;
  if (!c || !distance) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  if (chunk_len / 32 > ctx->K) return fail(ctx, CUHE_INVALID_ARGUMENT, "chunk_len wider than n^2");
  if (vectors > CUHE_STATIC_DECODE_MAX_CHUNKS / chunk_num)
    return fail(ctx, CUHE_INVALID_ARGUMENT,
                "decode_hamming_static: vectors*chunk_num exceeds the static scratch of " +
                    std::to_string(CUHE_STATIC_DECODE_MAX_CHUNKS) + " ciphertext chunks");
  DeviceGuard guard(ctx->device);
  if (!is_device_pointer(c) || !is_device_pointer(distance))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "decode_hamming_static needs device buffers for c and distance");
  std::lock_guard<std::mutex> lock(ctx->mu);
  uint32_t* counts = nullptr;
  if (int rc = static_counts(ctx, ctx->device, &counts)) return rc;
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const int64_t total = vectors * chunk_num;
  CUHE_CUDA(ctx, secret_modexp(ctx, d, c, counts, total, cuhe::EXP_DECODE, chunk_len / 32), "static decode launch");
  cuhe::k_sum_chunks<<<unsigned((vectors + 255) / 256), 256, 0, ctx->stream>>>(
      counts, vectors, chunk_num, reinterpret_cast<long long*>(distance));
  CUHE_CUDA(ctx, cudaGetLastError(), "static decode reduction");
  return CUHE_OK;
}

int cuhe_fp64_peak(int device, double* fp64_per_second) {
  if (!fp64_per_second) return fail(nullptr, CUHE_INVALID_ARGUMENT, "null output");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    return fail(nullptr, CUHE_CUDA_ERROR, "no such CUDA device");
  DeviceGuard guard(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* sink = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaMalloc(&sink, 8);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  const int iters = 8192, blocks = sms * 8, threads = 256;
  float ms = 0.f;
  if (e == cudaSuccess) {
    cuhe::k_fp64_probe<<<blocks, threads>>>(sink, iters, 1.0);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) cuhe::k_fp64_probe<<<blocks, threads>>>(sink, iters, 2.0 + r);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "fp64 probe");
  *fp64_per_second = 5.0 * blocks * threads * double(iters) * 8.0 / (double(ms) * 1e-3);
  return CUHE_OK;
}

int cuhe_imad_peak(int device, double* word_products_per_second) {
  if (!word_products_per_second) return fail(nullptr, CUHE_INVALID_ARGUMENT, "null output");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    return fail(nullptr, CUHE_CUDA_ERROR, "no such CUDA device");
  DeviceGuard guard(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint32_t* sink = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaMalloc(&sink, 4);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  const int iters = 4096, blocks = sms * 8, threads = 256;
  float ms_pairs = 0.f, ms_chain = 0.f;
  if (e == cudaSuccess) {
    cuhe::k_imad_probe<<<blocks, threads>>>(sink, iters, 1u);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) cuhe::k_imad_probe<<<blocks, threads>>>(sink, iters, 2u + r);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_pairs, a, b);
  }
  if (e == cudaSuccess) {
    cuhe::k_imad_chain_probe<<<blocks, threads>>>(sink, iters, 1u);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) cuhe::k_imad_chain_probe<<<blocks, threads>>>(sink, iters, 2u + r);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_chain, a, b);
  }
  float ms_wide = 0.f;
  if (e == cudaSuccess) {
    cuhe::k_imad_wide_probe<<<blocks, threads>>>(sink, iters, 1u);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) cuhe::k_imad_wide_probe<<<blocks, threads>>>(sink, iters, 2u + r);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms_wide, a, b);
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "imad probe");
  // word products per thread per iteration: 32 in the chain probe (4 rows of
  // 8 limbs), 8 in the lo/hi and wide probes
  const double products = 5.0 * blocks * threads * double(iters) * 32.0;
  const double pairs_rate = products / 4.0 / (double(ms_pairs) * 1e-3);
  const double chain_rate = products / (double(ms_chain) * 1e-3);
  const double wide_rate = products / 4.0 / (double(ms_wide) * 1e-3);
  *word_products_per_second = std::max(pairs_rate, std::max(chain_rate, wide_rate));
  return CUHE_OK;
}

int cuhe_paillier_modexp(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* exponent, int exponent_words,
                         uint32_t* out, int64_t count) {
  if (!ctx || count < 0 || !exponent || exponent_words <= 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!base || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  // exponent of any width: build its schedule
  Limbs e(exponent, exponent + exponent_words);
  while (e.size() > 1 && e.back() == 0) e.pop_back();
  const Modexp52 f52 = direct52(ctx);
  std::vector<int32_t> ops = cuhe::host::window_schedule(e, f52 ? kCrt52Window : ctx->window);
  if (!ops.empty()) {
    if (cudaError_t ce = ctx->tmp_ops.reserve(ops.size() * 4)) return cuda_fail(ctx, ce, "schedule allocation");
    CUHE_CUDA(ctx, cudaMemcpyAsync(ctx->tmp_ops.ptr, ops.data(), ops.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
              "schedule upload");
  }
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(base, bytes, true, false);
  st.add(out, bytes, false, true);
  if (int rc = st.bind()) return rc;
  if (f52) {
    CUHE_CUDA(ctx, f52(ctx, (const uint32_t*)st.dev(0), nullptr, (uint32_t*)st.dev(1), count,
                       (const int32_t*)ctx->tmp_ops.ptr, int(ops.size()), cuhe::EXP_POW, 0),
              "modexp launch");
  } else {
    CUHE_CUDA(ctx, d.modexp(ctx, (const uint32_t*)st.dev(0), nullptr, (uint32_t*)st.dev(1), count,
                            (const int32_t*)ctx->tmp_ops.ptr, int(ops.size()), cuhe::EXP_POW, 0),
              "modexp launch");
  }
  if (int rc = st.finish()) return rc;
  // the schedule buffer is reused by the next call: keep host order
  if (!st.staged()) CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "modexp synchronize");
  return check_status(ctx, true);
}

int cuhe_paillier_modexp_each(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* exponents,
                              int exponent_words, uint32_t* out, int64_t count) {
  if (!ctx || count < 0 || exponent_words <= 0 || exponent_words > ctx->K)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!base || !exponents || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(base, bytes, true, false);
  st.add(exponents, size_t(count) * exponent_words * 4, true, false);
  st.add(out, bytes, false, true);
  if (int rc = st.bind()) return rc;
  CUHE_CUDA(ctx, d.modexp_var(ctx, (const uint32_t*)st.dev(0), (const uint32_t*)st.dev(1), exponent_words,
                              exponent_words * 8, (uint32_t*)st.dev(2), count),
            "modexp_each launch");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

int cuhe_paillier_mulmod(cuhe_paillier* ctx, const uint32_t* a, const uint32_t* b, uint32_t* out, int64_t count) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!a || !b || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(a, bytes, true, false);
  st.add(b, bytes, true, false);
  st.add(out, bytes, false, true);
  if (int rc = st.bind()) return rc;
  CUHE_CUDA(ctx, d.mulmod(ctx, (const uint32_t*)st.dev(0), (const uint32_t*)st.dev(1), (uint32_t*)st.dev(2), count),
            "mulmod launch");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

int cuhe_paillier_from_hex(cuhe_paillier* ctx, const char* text, const int64_t* offsets, int64_t count, int reduce,
                           uint32_t* out) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!text || !offsets || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  if (offsets[0] != 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "offsets must start at 0");
  for (int64_t i = 0; i < count; ++i)
    if (offsets[i + 1] < offsets[i]) return fail(ctx, CUHE_INVALID_ARGUMENT, "offsets must not decrease");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t text_bytes = size_t(offsets[count]);
  const size_t bytes = size_t(count) * ctx->K * 4;
  Stager st(ctx);
  st.add(text, text_bytes ? text_bytes : 1, true, false);
  st.add(offsets, size_t(count + 1) * 8, true, false);
  st.add(out, bytes, false, true);
  if (int rc = st.bind()) return rc;
  const long long threads = count * ctx->K;
  cuhe::k_hex_to_limbs<<<unsigned((threads + 255) / 256), 256, 0, ctx->stream>>>(
      (const char*)st.dev(0), (const long long*)st.dev(1), count, ctx->K, (uint32_t*)st.dev(2), ctx->d_status);
  CUHE_CUDA(ctx, cudaGetLastError(), "hex parse launch");
  if (reduce) {
    // x mod n^2 for any x < 2^(32K): (x R mod n^2) R^-1
    CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(2), (uint32_t*)st.dev(2), count, 2), "reduce launch");
    CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(2), (uint32_t*)st.dev(2), count, 0), "reduce launch");
  }
  if (int rc = st.finish()) return rc;
  int status = 0;
  CUHE_CUDA(ctx, cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status");
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "hex parse");
  if (status) {
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    if (status & cuhe::ST_HEX) return fail(ctx, CUHE_INVALID_ARGUMENT, "Invalid hex digit");
    return fail(ctx, CUHE_RANGE, "input outside its valid range");
  }
  return CUHE_OK;
}

int cuhe_paillier_to_hex(cuhe_paillier* ctx, const uint32_t* limbs, int64_t count, char* out) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (count == 0) return CUHE_OK;
  if (!limbs || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  const size_t words = size_t(ctx->K);
  Stager st(ctx);
  st.add(limbs, size_t(count) * words * 4, true, false);
  st.add(out, size_t(count) * words * 8, false, true);
  if (int rc = st.bind()) return rc;
  const long long threads = count * ctx->K;
  cuhe::k_limbs_to_hex<<<unsigned((threads + 255) / 256), 256, 0, ctx->stream>>>(
      (const uint32_t*)st.dev(0), count, ctx->K, (char*)st.dev(1));
  CUHE_CUDA(ctx, cudaGetLastError(), "hex format launch");
  if (int rc = st.finish()) return rc;
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "hex format");
  return CUHE_OK;
}

int cuhe_paillier_mulmod_outer(cuhe_paillier* ctx, const uint32_t* query, int64_t nq, const uint32_t* index,
                               int64_t nx, uint32_t* out) {
  if (!ctx || nq < 0 || nx < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (nq == 0 || nx == 0) return CUHE_OK;
  if (!query || !index || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t kb = size_t(ctx->K) * 4;
  const size_t obytes = size_t(nq) * size_t(nx) * kb;
  // A large host output moves in query-row blocks on the copy stream, each
  // block's download beside the next block's products.
  const bool pipe = obytes >= kPipeBytes && nq >= 2 && !is_device_pointer(out);
  const Outer52 f52 = outer52(ctx);
  Stager st(ctx);
  st.add(query, size_t(nq) * kb, true, false);
  st.add(index, size_t(nx) * kb, true, false);
  st.add(out, obytes, false, !pipe);
  st.add_scratch(size_t(nq) * (f52 ? size_t(ctx->K) * 5 : kb));  // queries in Montgomery form (words or 52-bit limbs)
  if (int rc = st.bind()) return rc;
  uint32_t* qm = static_cast<uint32_t*>(st.dev(3));
  uint32_t* d_out = static_cast<uint32_t*>(st.dev(2));
  // the FP64 form converts each query block inside its launch
  auto outer = [&](int64_t q0, int64_t qn, uint32_t* o) -> cudaError_t {
    if (f52)
      return f52(ctx, (const uint32_t*)st.dev(0) + size_t(q0) * ctx->K, qn,
                 reinterpret_cast<double*>(qm) + size_t(q0) * (5 * size_t(ctx->K) / 8), (const uint32_t*)st.dev(1),
                 nx, o);
    return d.outer(ctx, qm + size_t(q0) * ctx->K, qn, (const uint32_t*)st.dev(1), nx, o);
  };
  if (!f52) CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(0), qm, nq, 1), "query conversion");
  if (pipe && st.is_staged(2)) {
    if (int rc = pipeline_streams(ctx)) return rc;
    const int64_t rows = std::max<int64_t>(1, nq / 8);
    const size_t row_words = size_t(nx) * ctx->K;
    for (int64_t q0 = 0; q0 < nq; q0 += rows) {
      const int64_t qn = std::min(rows, nq - q0);
      CUHE_CUDA(ctx, outer(q0, qn, d_out + size_t(q0) * row_words), "mulmod_outer launch");
      CUHE_CUDA(ctx, stream_after(ctx->copy, ctx->stream), "download order");
      CUHE_CUDA(ctx, cudaMemcpyAsync(out + size_t(q0) * row_words, d_out + size_t(q0) * row_words,
                                     size_t(qn) * row_words * 4, cudaMemcpyDeviceToHost, ctx->copy),
                "piecewise download");
    }
    CUHE_CUDA(ctx, stream_after(ctx->stream, ctx->copy), "download join");
  } else {
    CUHE_CUDA(ctx, outer(0, nq, d_out), "mulmod_outer launch");
  }
  if (int rc = st.finish()) return rc;
  // the scratch slice is reused by the next call: keep host order
  if (!st.staged()) CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "mulmod_outer synchronize");
  return check_status(ctx, true);
}

int cuhe_lookup_set_tables(cuhe_paillier* ctx, const uint32_t* g_table, int message_chunks, const uint32_t* noise,
                           int noise_entries) {
  if (!ctx || !g_table || !noise || message_chunks <= 0 || noise_entries <= 0 || noise_entries > 256)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid tables");
  if (message_chunks * 256 > 65536) return fail(ctx, CUHE_INVALID_ARGUMENT, "too many message chunks");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t kb = size_t(ctx->K) * 4;
  const size_t gbytes = size_t(message_chunks) * 256 * kb;
  cudaFree(ctx->d_gtab);
  cudaFree(ctx->d_noise);
  cudaFree(ctx->d_wide);
  cudaFree(ctx->d_wide52);
  cudaFree(ctx->d_noise52);
  ctx->d_gtab = nullptr;
  ctx->d_noise = nullptr;
  ctx->d_wide = nullptr;
  ctx->d_wide52 = nullptr;
  ctx->d_noise52 = nullptr;
  ctx->message_chunks = 0;
  ctx->noise_entries = 0;
  CUHE_CUDA(ctx, cudaMalloc(&ctx->d_gtab, gbytes), "table allocation");
  CUHE_CUDA(ctx, cudaMalloc(&ctx->d_noise, size_t(noise_entries) * kb), "table allocation");
  Stager st(ctx);
  st.add(g_table, gbytes, true, false);
  st.add(noise, size_t(noise_entries) * kb, true, false);
  if (int rc = st.bind()) return rc;
  CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(0), ctx->d_gtab, (long long)message_chunks * 256, 1),
            "table conversion");
  CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(1), ctx->d_noise, noise_entries, 1), "table conversion");
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "table synchronize");
  if (int rc = check_status(ctx, true)) return rc;
  ctx->message_chunks = message_chunks;
  ctx->noise_entries = noise_entries;
  return CUHE_OK;
}

int cuhe_lookup_build_tables(cuhe_paillier* ctx, const uint32_t* g, int message_chunks, const uint32_t* noise,
                             int noise_entries) {
  if (!ctx || !g || message_chunks <= 0 || message_chunks * 256 > 65536)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid table request");
  if (noise && (noise_entries <= 0 || noise_entries > 256)) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid noise");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const size_t k = size_t(ctx->K), kb = k * 4;
  // base_i = g^(2^(8i)) for all rows: one batched modexp per row exponent is
  // wasteful; square on the device 8 times per row in one group instead.
  std::vector<uint32_t> gk(k, 0u);
  std::memcpy(gk.data(), g, kb);  // caller passes K words
  DeviceBuffer bases, gdev, pows;
  CUHE_CUDA(ctx, bases.reserve(size_t(message_chunks) * kb), "table scratch");
  CUHE_CUDA(ctx, gdev.reserve(kb), "table scratch");
  CUHE_CUDA(ctx, cudaMemcpyAsync(gdev.ptr, gk.data(), kb, cudaMemcpyHostToDevice, ctx->stream), "upload g");
  // bases: row i = g^(2^(8i)); computed as a batched modexp over rows with
  // per-row exponent 2^(8i) is not fixed-exponent, so use successive
  // fixed-exponent launches of 2^8 on the previous row (message_chunks launches).
  std::vector<int32_t> ops256 = cuhe::host::window_schedule(Limbs{256u}, ctx->window);
  CUHE_CUDA(ctx, pows.reserve(ops256.size() * 4), "table scratch");
  CUHE_CUDA(ctx, cudaMemcpyAsync(pows.ptr, ops256.data(), ops256.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
            "upload schedule");
  uint32_t* b = static_cast<uint32_t*>(bases.ptr);
  CUHE_CUDA(ctx, cudaMemcpyAsync(b, gdev.ptr, kb, cudaMemcpyDeviceToDevice, ctx->stream), "row 0");
  for (int i = 1; i < message_chunks; ++i) {
    CUHE_CUDA(ctx, d.modexp(ctx, b + (i - 1) * k, nullptr, b + i * k, 1, (const int32_t*)pows.ptr, int(ops256.size()),
                            cuhe::EXP_POW, 0),
              "row base");
  }
  // to Montgomery form, then fill rows
  DeviceBuffer bm;
  CUHE_CUDA(ctx, bm.reserve(size_t(message_chunks) * kb), "table scratch");
  CUHE_CUDA(ctx, d.convert(ctx, b, (uint32_t*)bm.ptr, message_chunks, 1), "row conversion");
  cudaFree(ctx->d_gtab);
  cudaFree(ctx->d_wide);
  cudaFree(ctx->d_wide52);
  cudaFree(ctx->d_noise52);
  ctx->d_gtab = nullptr;
  ctx->d_wide = nullptr;
  ctx->d_wide52 = nullptr;
  ctx->d_noise52 = nullptr;
  ctx->message_chunks = 0;
  CUHE_CUDA(ctx, cudaMalloc(&ctx->d_gtab, size_t(message_chunks) * 256 * kb), "table allocation");
  CUHE_CUDA(ctx, d.table_rows(ctx, (const uint32_t*)bm.ptr, message_chunks, ctx->d_gtab), "table rows");
  if (noise) {
    cudaFree(ctx->d_noise);
    ctx->d_noise = nullptr;
    ctx->noise_entries = 0;
    CUHE_CUDA(ctx, cudaMalloc(&ctx->d_noise, size_t(noise_entries) * kb), "noise allocation");
    Stager st(ctx);
    st.add(noise, size_t(noise_entries) * kb, true, false);
    if (int rc = st.bind()) return rc;
    CUHE_CUDA(ctx, d.convert(ctx, (const uint32_t*)st.dev(0), ctx->d_noise, noise_entries, 1), "noise conversion");
  }
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "table synchronize");
  bases.release();
  gdev.release();
  pows.release();
  bm.release();
  if (int rc = check_status(ctx, true)) return rc;
  ctx->message_chunks = message_chunks;
  if (noise) ctx->noise_entries = noise_entries;
  return CUHE_OK;
}

int cuhe_lookup_get_g_table(cuhe_paillier* ctx, uint32_t* out) {
  if (!ctx || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  if (!ctx->d_gtab) return fail(ctx, CUHE_NOT_READY, "tables not installed");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const long long entries = (long long)ctx->message_chunks * 256;
  Stager st(ctx);
  st.add(out, size_t(entries) * ctx->K * 4, false, true);
  if (int rc = st.bind()) return rc;
  CUHE_CUDA(ctx, d.convert(ctx, ctx->d_gtab, (uint32_t*)st.dev(0), entries, 0), "table export");
  if (int rc = st.finish()) return rc;
  CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "table export");
  return check_status(ctx, true);
}

}  // extern "C"

namespace {

int ensure_wide_table(cuhe_paillier* ctx, const Dispatch& d, long long items) {
  if (ctx->d_wide || ctx->d_wide52 || ctx->wide_mode == 0 || !ctx->d_gtab) return CUHE_OK;
  if (ctx->wide_mode == 1 && items < kWideMinItems) return CUHE_OK;
  // the table as the selected pipe takes it: 52-bit limbs (doubles, K52 =
  // 5K/8 a row) for the FP64 pipe, else 32-bit words
  Lookup52 l52{};
  const bool fp52 = lookup52(ctx, &l52);
  const size_t entry = fp52 ? size_t(5 * ctx->K / 8) * 8 : size_t(ctx->K) * 4;
  const size_t bytes = size_t((ctx->message_chunks + 1) / 2) * 65536 * entry;
  if (ctx->wide_mode == 1) {
    size_t free_bytes = 0, total_bytes = 0;
    CUHE_CUDA(ctx, cudaMemGetInfo(&free_bytes, &total_bytes), "free memory");
    if (bytes > kWideMaxBytes || bytes > free_bytes / 4) return CUHE_OK;
  }
  void* wide = nullptr;
  void* noise52 = nullptr;
  cudaError_t e = cudaMalloc(&wide, bytes);
  if (e == cudaSuccess && fp52 && ctx->noise_entries > 0)
    e = cudaMalloc(&noise52, size_t(ctx->noise_entries) * entry);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(wide);
    if (ctx->wide_mode == 2) return fail(ctx, CUHE_OUT_OF_MEMORY, "wide table allocation");
    return CUHE_OK;
  }
  e = fp52 ? l52.build(ctx, static_cast<double*>(wide), static_cast<double*>(noise52))
           : d.wide_table(ctx, static_cast<uint32_t*>(wide));
  if (e != cudaSuccess) {
    cudaFree(wide);
    cudaFree(noise52);
    return cuda_fail(ctx, e, "wide table build");
  }
  if (fp52) {
    ctx->d_wide52 = static_cast<double*>(wide);
    ctx->d_noise52 = static_cast<double*>(noise52);
  } else {
    ctx->d_wide = static_cast<uint32_t*>(wide);
  }
  return CUHE_OK;
}

}  // namespace

extern "C" {

int cuhe_lookup_set_wide_table(cuhe_paillier* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 2) return fail(ctx, CUHE_INVALID_ARGUMENT, "wide table mode must be 0, 1 or 2");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->wide_mode = mode;
  if (mode == 0 && (ctx->d_wide || ctx->d_wide52)) {
    CUHE_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "wide table release");
    cudaFree(ctx->d_wide);
    cudaFree(ctx->d_wide52);
    cudaFree(ctx->d_noise52);
    ctx->d_wide = nullptr;
    ctx->d_wide52 = nullptr;
    ctx->d_noise52 = nullptr;
  }
  return CUHE_OK;
}

int cuhe_lookup_wide_table_ready(const cuhe_paillier* ctx) { return ctx && (ctx->d_wide || ctx->d_wide52) ? 1 : 0; }

int cuhe_lookup_encrypt_bits(cuhe_paillier* ctx, const uint8_t* bits, int64_t vectors, int embed_len, int chunk_len,
                             int chunk_num, const uint8_t* noise_index, uint32_t* out) {
  if (!ctx || vectors < 0 || embed_len <= 0 || chunk_len <= 0 || chunk_num <= 0)
    return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid layout");
  if (!ctx->d_gtab || !ctx->d_noise) return fail(ctx, CUHE_NOT_READY, "lookup tables not installed");
  if (int64_t(chunk_num) * chunk_len < 2 * int64_t(embed_len))
    return fail(ctx, CUHE_INVALID_ARGUMENT, "chunks do not cover the padded embedding");
  if (vectors == 0) return CUHE_OK;
  if (!bits || !noise_index || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  const int64_t total = vectors * chunk_num;
  if (int rc = ensure_wide_table(ctx, d, total)) return rc;
  Stager st(ctx);
  st.add(bits, size_t(vectors) * embed_len, true, false);
  st.add(noise_index, size_t(total) * cuhe::kNoiseMultiples, true, false);
  st.add(out, size_t(total) * ctx->K * 4, false, true);
  if (int rc = st.bind()) return rc;
  Lookup52 l52{};
  const bool fp52 = ctx->d_wide52 && lookup52(ctx, &l52);
  CUHE_CUDA(ctx, (fp52 ? l52.launch : d.lookup)(ctx, (const uint8_t*)st.dev(0), embed_len, chunk_len, chunk_num, nullptr,
                                               total, (const uint8_t*)st.dev(1), (uint32_t*)st.dev(2)),
            "lookup encrypt launch");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

int cuhe_lookup_encrypt_ints(cuhe_paillier* ctx, const uint32_t* m, int64_t count, const uint8_t* noise_index,
                             uint32_t* out) {
  if (!ctx || count < 0) return fail(ctx, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (!ctx->d_gtab || !ctx->d_noise) return fail(ctx, CUHE_NOT_READY, "lookup tables not installed");
  if (count == 0) return CUHE_OK;
  if (!m || !noise_index || !out) return fail(ctx, CUHE_INVALID_ARGUMENT, "null buffer");
  DeviceGuard guard(ctx->device);
  std::lock_guard<std::mutex> lock(ctx->mu);
  Dispatch d;
  find_dispatch(ctx->K, ctx->tpi, ctx->window, &d);
  if (int rc = ensure_wide_table(ctx, d, count)) return rc;
  Stager st(ctx);
  st.add(m, size_t(count) * ctx->K * 4, true, false);
  st.add(noise_index, size_t(count) * cuhe::kNoiseMultiples, true, false);
  st.add(out, size_t(count) * ctx->K * 4, false, true);
  if (int rc = st.bind()) return rc;
  Lookup52 l52{};
  const bool fp52 = ctx->d_wide52 && lookup52(ctx, &l52);
  CUHE_CUDA(ctx, (fp52 ? l52.launch : d.lookup)(ctx, nullptr, 0, 0, 1, (const uint32_t*)st.dev(0), count,
                                               (const uint8_t*)st.dev(1), (uint32_t*)st.dev(2)),
            "lookup encrypt launch");
  if (int rc = st.finish()) return rc;
  return check_status(ctx, st.staged());
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Mixed batches: many (key, exponent, bases) exponentiations of uneven sizes
// and widths in one persistent launch per width.
// ---------------------------------------------------------------------------
struct cuhe_mix {
  struct Entry {
    cuhe_paillier* ctx;
    const uint32_t* base;
    uint32_t* out;
    long long count;
    Limbs exponent;
  };
  struct Width {
    int K = 0, tpi = 0, window = 0, grid = 0, ntasks = 0;
    long long units = 0;
    cuhe::ModexpTask* d_tasks = nullptr;
    std::vector<int32_t*> d_ops;
    Dispatch d;
    bool fp52 = false;  // k_modexp52_tasks: every context of the width selects the FP64 pipe
    cudaError_t (*prepare)(int, int*) = nullptr;
    cudaError_t (*launch)(const cuhe::ModexpTask*, int, long long, unsigned long long*, int*, int,
                          cudaStream_t) = nullptr;
  };
  int device = 0;
  std::vector<Entry> entries;
  std::map<int, std::pair<int, int>> tuning;  // K -> (tpi, window)
  std::vector<Width> widths;
  unsigned long long* d_counters = nullptr;
  int* d_status = nullptr;
  bool planned = false;
  std::string error;
  // widths after the first run on their own streams, forked from and joined
  // back to the launch stream, so that one width's last wave overlaps the
  // next width's kernel (created by the plan: a launch allocates nothing)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr;

  void release_plan() {
    for (auto& w : widths) {
      cudaFree(w.d_tasks);
      for (int32_t* p : w.d_ops) cudaFree(p);
    }
    widths.clear();
    cudaFree(d_counters);
    d_counters = nullptr;
    for (cudaStream_t st : side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : done) cudaEventDestroy(ev);
    side.clear();
    done.clear();
    if (fork) cudaEventDestroy(fork);
    fork = nullptr;
    planned = false;
  }
};

namespace {
int mix_fail(cuhe_mix* mix, int code, const std::string& msg) {
  if (mix) mix->error = msg; else g_create_error = msg;
  return code;
}
}  // namespace

extern "C" {

const char* cuhe_mix_last_error(const cuhe_mix* mix) { return mix ? mix->error.c_str() : g_create_error.c_str(); }

int cuhe_mix_create(int device, cuhe_mix** out) {
  if (!out) return mix_fail(nullptr, CUHE_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return mix_fail(nullptr, CUHE_INVALID_ARGUMENT, "invalid device ordinal");
  }
  auto* mix = new (std::nothrow) cuhe_mix();
  if (!mix) return mix_fail(nullptr, CUHE_OUT_OF_MEMORY, "mix allocation");
  mix->device = device;
  DeviceGuard guard(device);
  if (cudaMalloc(&mix->d_status, sizeof(int)) != cudaSuccess || cudaMemset(mix->d_status, 0, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    delete mix;
    return mix_fail(nullptr, CUHE_OUT_OF_MEMORY, "mix status allocation");
  }
  *out = mix;
  return CUHE_OK;
}

void cuhe_mix_destroy(cuhe_mix* mix) {
  if (!mix) return;
  DeviceGuard guard(mix->device);
  cudaDeviceSynchronize();
  mix->release_plan();
  cudaFree(mix->d_status);
  delete mix;
}

int cuhe_mix_add_modexp(cuhe_mix* mix, cuhe_paillier* ctx, const uint32_t* base, uint32_t* out, int64_t count,
                        const uint32_t* exponent, int exponent_words) {
  if (!mix || !ctx || !exponent || exponent_words <= 0 || count < 0)
    return mix_fail(mix, CUHE_INVALID_ARGUMENT, "invalid argument");
  if (ctx->device != mix->device) return mix_fail(mix, CUHE_INVALID_ARGUMENT, "context on another device");
  if (count == 0) return CUHE_OK;
  DeviceGuard guard(mix->device);
  if (!is_device_pointer(base) || !is_device_pointer(out))
    return mix_fail(mix, CUHE_INVALID_ARGUMENT, "mixed batches take device buffers");
  if (!cuhe::host::fits(exponent, size_t(exponent_words), size_t(ctx->K)))
    return mix_fail(mix, CUHE_INVALID_ARGUMENT, "exponent wider than n^2");
  mix->entries.push_back({ctx, base, out, count, cuhe::host::resized(exponent, size_t(exponent_words), size_t(ctx->K))});
  mix->planned = false;
  return CUHE_OK;
}

int cuhe_mix_set_tuning(cuhe_mix* mix, int words, int tpi, int window) {
  if (!mix) return CUHE_INVALID_ARGUMENT;
  Dispatch d;
  if (!find_dispatch(words, tpi, window, &d))
    return mix_fail(mix, CUHE_INVALID_ARGUMENT, "tuning (threads per instance, window) not compiled for this width");
  mix->tuning[words] = {tpi, window};
  mix->planned = false;
  return CUHE_OK;
}

int cuhe_mix_plan(cuhe_mix* mix) {
  if (!mix) return CUHE_INVALID_ARGUMENT;
  DeviceGuard guard(mix->device);
  cudaDeviceSynchronize();
  mix->release_plan();
  std::map<int, std::vector<size_t>> by_width;
  for (size_t i = 0; i < mix->entries.size(); ++i) by_width[mix->entries[i].ctx->K].push_back(i);
  for (auto& kv : by_width) {
    cuhe_mix::Width w;
    w.K = kv.first;
    auto it = mix->tuning.find(w.K);
    if (it != mix->tuning.end()) {
      w.tpi = it->second.first;
      w.window = it->second.second;
    } else {
      default_tuning(w.K, &w.tpi, &w.window);
    }
    if (!find_dispatch(w.K, w.tpi, w.window, &w.d)) return mix_fail(mix, CUHE_INVALID_ARGUMENT, "no compiled variant");
    // the pipe follows the contexts, as their one-launch-per-batch calls do
    w.fp52 = true;
    for (size_t i : kv.second) w.fp52 = w.fp52 && direct52(mix->entries[i].ctx) != nullptr;
    w.prepare = w.d.prepare_tasks;
    w.launch = w.d.launch_tasks;
    if (w.fp52) {
      w.window = kCrt52Window;
      w.tpi = w.K / 16;
      if (w.K == 64) { w.prepare = &prepare_tasks52<64>; w.launch = &launch_tasks52<64>; }
      if (w.K == 128) { w.prepare = &prepare_tasks52<128>; w.launch = &launch_tasks52<128>; }
      if (w.K == 256) { w.prepare = &prepare_tasks52<256>; w.launch = &launch_tasks52<256>; }
    }
    const long long ipb = cuhe::kBlockThreads / w.tpi;
    std::vector<cuhe::ModexpTask> tasks;
    for (size_t i : kv.second) {
      const auto& e = mix->entries[i];
      std::vector<int32_t> ops = cuhe::host::window_schedule(e.exponent, w.window);
      int32_t* d_ops = nullptr;
      if (!ops.empty()) {
        if (cudaMalloc(&d_ops, ops.size() * 4) != cudaSuccess ||
            cudaMemcpy(d_ops, ops.data(), ops.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
          cudaGetLastError();
          cudaFree(d_ops);
          return mix_fail(mix, CUHE_OUT_OF_MEMORY, "schedule upload");
        }
        w.d_ops.push_back(d_ops);
      }
      cuhe::ModexpTask t{};
      t.base = e.base;
      t.out = e.out;
      t.count = e.count;
      t.consts = e.ctx->d_consts;
      t.ops = d_ops;
      t.first_unit = w.units;
      t.ks = e.ctx->ks;
      t.nops = int(ops.size());
      t.mode = cuhe::EXP_POW;
      t.n52 = e.ctx->d_n52;
      t.ninv52 = e.ctx->ninv52;
      tasks.push_back(t);
      w.units += (e.count + ipb - 1) / ipb;
    }
    w.ntasks = int(tasks.size());
    if (cudaMalloc(&w.d_tasks, tasks.size() * sizeof(cuhe::ModexpTask)) != cudaSuccess ||
        cudaMemcpy(w.d_tasks, tasks.data(), tasks.size() * sizeof(cuhe::ModexpTask), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
      cudaGetLastError();
      return mix_fail(mix, CUHE_OUT_OF_MEMORY, "task table upload");
    }
    cudaError_t e = w.prepare(mix->device, &w.grid);
    if (e != cudaSuccess) return mix_fail(mix, CUHE_CUDA_ERROR, std::string("mixed launch setup: ") + cudaGetErrorString(e));
    mix->widths.push_back(std::move(w));
  }
  if (!mix->widths.empty() &&
      cudaMalloc(&mix->d_counters, mix->widths.size() * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    return mix_fail(mix, CUHE_OUT_OF_MEMORY, "counter allocation");
  }
  if (mix->widths.size() > 1) {
    if (cudaEventCreateWithFlags(&mix->fork, cudaEventDisableTiming) != cudaSuccess)
      return mix_fail(mix, CUHE_CUDA_ERROR, "mixed launch events");
    for (size_t i = 1; i < mix->widths.size(); ++i) {
      cudaStream_t st = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return mix_fail(mix, CUHE_CUDA_ERROR, "mixed launch streams");
      mix->side.push_back(st);
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        return mix_fail(mix, CUHE_CUDA_ERROR, "mixed launch events");
      mix->done.push_back(ev);
    }
  }
  mix->planned = true;
  return CUHE_OK;
}

int cuhe_mix_launch(cuhe_mix* mix, void* stream) {
  if (!mix) return CUHE_INVALID_ARGUMENT;
  if (!mix->planned) return mix_fail(mix, CUHE_NOT_READY, "mixed batch not planned");
  if (mix->widths.empty()) return CUHE_OK;
  DeviceGuard guard(mix->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(mix->d_counters, 0, mix->widths.size() * sizeof(unsigned long long), s);
  if (e == cudaSuccess && mix->fork) e = cudaEventRecord(mix->fork, s);
  for (size_t i = 0; i < mix->widths.size() && e == cudaSuccess; ++i) {
    const auto& w = mix->widths[i];
    cudaStream_t ws = i == 0 ? s : mix->side[i - 1];
    if (i > 0) e = cudaStreamWaitEvent(ws, mix->fork, 0);
    if (e == cudaSuccess)
      e = w.launch(w.d_tasks, w.ntasks, w.units, mix->d_counters + i, mix->d_status, w.grid, ws);
    if (e == cudaSuccess && i > 0) e = cudaEventRecord(mix->done[i - 1], ws);
    if (e == cudaSuccess && i > 0) e = cudaStreamWaitEvent(s, mix->done[i - 1], 0);
  }
  if (e != cudaSuccess) return mix_fail(mix, CUHE_CUDA_ERROR, std::string("mixed launch: ") + cudaGetErrorString(e));
  return CUHE_OK;
}

int cuhe_mix_check(cuhe_mix* mix) {
  if (!mix) return CUHE_INVALID_ARGUMENT;
  DeviceGuard guard(mix->device);
  int status = 0;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&status, mix->d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return mix_fail(mix, CUHE_CUDA_ERROR, std::string("mixed batch: ") + cudaGetErrorString(e));
  if (status) {
    cudaMemset(mix->d_status, 0, sizeof(int));
    return mix_fail(mix, CUHE_RANGE, "input outside its valid range (base >= n^2)");
  }
  return CUHE_OK;
}

int cuhe_mix_info(const cuhe_mix* mix, int index, int* words, int* tpi, int* window, int* grid, int64_t* units,
                  int* tasks) {
  if (!mix || index < 0 || size_t(index) >= mix->widths.size()) return CUHE_INVALID_ARGUMENT;
  const auto& w = mix->widths[size_t(index)];
  if (words) *words = w.K;
  if (tpi) *tpi = w.tpi;
  if (window) *window = w.window;
  if (grid) *grid = w.grid;
  if (units) *units = w.units;
  if (tasks) *tasks = w.ntasks;
  return CUHE_OK;
}

int cuhe_mix_widths(const cuhe_mix* mix) { return mix ? int(mix->widths.size()) : 0; }

}  // extern "C"
