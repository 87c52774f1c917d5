/* C ABI of the B200 Paillier / Paillier-Lookup kernels (libcuhe_b200.so).
 *
 * Conventions
 *  - Big integers are arrays of little-endian 32-bit words.  A key of
 *    key_len-bit primes has an n of 2*key_len bits and an n^2 of 4*key_len
 *    bits; the library works with K = key_len/8 words per value mod n^2
 *    (64, 128 or 256 words for key_len 512, 1024, 2048).  Every batched
 *    array below uses a stride of K words per item, plaintexts included
 *    (plaintexts < n occupy the low K/2 words, the rest are zero).
 *  - Pointers may be host or device memory.  Host buffers are staged through
 *    a context-owned device workspace and the call returns when the result is
 *    back on the host.  Device buffers are processed on the context stream
 *    and the call returns after queueing; cuhe_synchronize() waits.
 *  - Every function returns 0 on success or a negative cuhe_status; the
 *    message of the last failure is available from cuhe_last_error().
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the cuhepy project).
 */
#ifndef CUHE_PAILLIER_H
#define CUHE_PAILLIER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cuhe_status {
  CUHE_OK = 0,
  CUHE_INVALID_ARGUMENT = -1, /* reference raises ValueError / RuntimeError */
  CUHE_OUT_OF_MEMORY = -2,
  CUHE_CUDA_ERROR = -3,
  CUHE_NOT_READY = -4,        /* keys or tables not loaded */
  CUHE_RANGE = -5             /* an input is outside [0, n^2) or [0, n) */
} cuhe_status;

typedef struct cuhe_paillier cuhe_paillier;

/* Library version string and the last error of a context (or of the last
 * failed cuhe_paillier_create when ctx is NULL). */
const char* cuhe_version(void);
const char* cuhe_last_error(const cuhe_paillier* ctx);

/* Create a context for the public modulus n (n_words words).  Replaces the
 * key material held inside PaillierGPUClient / PaillierGPULookupClient
 * (src/cuhepy/paillier/_gpu_ext/paillier_GPU_client.cu:747-760;
 *  _lookup_gpu_ext/paillier_GPU_lookup_client.cu:1570-1612) and the pk dict
 * of Paillier.encrypt (src/cuhepy/paillier/scheme.py:63-83). */
int cuhe_paillier_create(const uint32_t* n, int n_words, int device, cuhe_paillier** out);
void cuhe_paillier_destroy(cuhe_paillier* ctx);
/* Words per value mod n^2 (K) used by this context. */
int cuhe_paillier_words(const cuhe_paillier* ctx);
/* Use a caller stream (cudaStream_t passed as void*); NULL restores the
 * context's own stream. */
int cuhe_paillier_set_stream(cuhe_paillier* ctx, void* stream);
int cuhe_synchronize(cuhe_paillier* ctx);

/* Install the secret decryption exponent and multiplier:
 *   textbook Paillier: exponent = phi, multiplier = phi^-1 mod n
 *     (src/cuhepy/paillier/scheme.py:86-104)
 *   Paillier-Lookup:   exponent = a,   multiplier = g_a_inv
 *     (src/cuhepy/paillier/lookup.py:257-278) */
int cuhe_paillier_set_secret(cuhe_paillier* ctx, const uint32_t* exponent, int exponent_words,
                             const uint32_t* multiplier, int multiplier_words);

/* Install the prime factors of n (n = p * q, little-endian words) so that
 * decrypt and decode exponentiations run by the Chinese remainder theorem:
 * c^e mod p^2 and c^e mod q^2 on half-width lane groups, recombined to
 * c^e mod n^2 by Garner's formula before the same L() / multiplier / popcount
 * epilogue.  Results are identical to the direct path for every c < n^2.
 * p = q = NULL removes the factors.  Rejects p * q != n, even or unit
 * factors, and factors whose squares are wider than half of n^2.  No
 * reference counterpart: the reference exponentiates mod n^2 directly
 * (decrypt_only_kernel, src/cuhepy/paillier/_lookup_gpu_ext/
 * paillier_GPU_lookup_client.cu:1013-1050); both of its key formats carry
 * phi, from which the host recovers p and q. */
int cuhe_paillier_set_factors(cuhe_paillier* ctx, const uint32_t* p, int p_words, const uint32_t* q, int q_words);
/* 1 when factors are installed (decrypt / decode use the CRT kernel). */
int cuhe_paillier_has_factors(const cuhe_paillier* ctx);

/* Pipe of the exponentiations.  With enable = 1 (the default), keys with n^2
 * of 4096 or 8192 bits run them as Montgomery products of 52-bit limbs on the
 * FP64 pipe (three exact FP64 instructions per 52x52-bit product, sums in
 * 64-bit integers, ten limbs per lane, a 3-bit window): decrypt / decode by
 * the CRT when the factors are installed (both half-width exponentiations),
 * and otherwise mod n^2 itself, as do encryption (r^n), cuhe_paillier_modexp
 * and mixed batches (cuhe_mix_plan, per width whose contexts all select it).
 * Entry and exit go through 32-bit Montgomery products and the same
 * recombination and epilogues, so results are identical to the integer-pipe
 * kernels.  n^2 of 2048 bits stays on the integer pipe (measured faster
 * there) unless enable = 2; enable = 0 keeps every product on the integer
 * pipe.  get returns the setting.  No reference counterpart (the reference's
 * CGBN kernels multiply 32-bit words on the integer pipe). */
int cuhe_paillier_set_fp64(cuhe_paillier* ctx, int enable);
int cuhe_paillier_get_fp64(const cuhe_paillier* ctx);

/* c[i] = (1 + m[i]*n) * r[i]^n mod n^2, i.e. g^m r^n with g = n + 1.
 * Replaces Paillier.encrypt (src/cuhepy/paillier/scheme.py:63-83) with the
 * randomness r supplied by the caller, and the device half of
 * PaillierGPUClient.encrypt (paillier_GPU_client.cu:873-974, 458-546). */
int cuhe_paillier_encrypt(cuhe_paillier* ctx, const uint32_t* m, const uint32_t* r, uint32_t* c,
                          int64_t count);

/* m[i] = floor((c[i]^e mod n^2 - 1) / n) * multiplier mod n (the installed
 * secret).  Replaces Paillier.decrypt (scheme.py:86-104),
 * PaillierLookup.decrypt (lookup.py:257-278) and decrypt_only_kernel
 * (paillier_GPU_lookup_client.cu:1014-1050, 2440-2499). */
int cuhe_paillier_decrypt(cuhe_paillier* ctx, const uint32_t* c, uint32_t* m, int64_t count);

/* Hamming decode: distance[v] = sum over the chunk_num chunks of vector v of
 * popcount(even bits of decrypt(c)).  Replaces decode_hamming_client
 * (paillier_GPU_lookup_client.cu:2338-2437: decrypt_only_kernel +
 * odd_popcount_kernel + host sum; hamming/paillier_lookup.py:221-242). */
int cuhe_paillier_decode_hamming(cuhe_paillier* ctx, const uint32_t* c, int64_t vectors, int chunk_num,
                                 int chunk_len, int64_t* distance);

/* Allocation-free variant of cuhe_paillier_decode_hamming.  It has no
 * counterpart in the reference.  It is for callers that must not allocate GPU
 * memory while they run: serving processes whose device memory is owned by a
 * caching allocator or a fixed reservation, and runtimes that give the
 * library only buffers they already own.  cuhe_paillier_decode_hamming takes its per-chunk scratch from
 * the context workspace, which cudaMalloc's on growth; this entry point instead
 * keeps that scratch in a file-scope device array of
 * CUHE_STATIC_DECODE_MAX_CHUNKS uint32 counts (256 KiB), which every GPU that
 * loads the library holds until the process exits.
 *  - c (vectors*chunk_num ciphertexts, K words each) and distance (vectors
 *    int64) must be device memory; host pointers are rejected, because staging
 *    them would allocate.
 *  - vectors*chunk_num above CUHE_STATIC_DECODE_MAX_CHUNKS is rejected with
 *    CUHE_INVALID_ARGUMENT before anything is launched.
 *  - The first call on a device, with that device current, looks up the
 *    array's device address once (cudaGetSymbolAddress) and keeps it for the
 *    life of the process; make that first call before any stream capture.  A
 *    device reset (cudaDeviceReset) after that first call is not supported.
 *  - Work is queued on the context stream and the call returns without waiting;
 *    range errors surface at the next cuhe_synchronize.
 *  - All calls in the process share the one array per device, so two calls
 *    whose work overlaps on the GPU race on it: serialise them (one stream, or
 *    wait between calls).  Each call writes every count it later reads, so
 *    nothing has to be cleared between calls.
 * Calls no cudaMalloc, cudaFree or other allocating routine. */
#define CUHE_STATIC_DECODE_MAX_CHUNKS 65536
int cuhe_paillier_decode_hamming_static(cuhe_paillier* ctx, const uint32_t* c, int64_t vectors, int chunk_num,
                                        int chunk_len, int64_t* distance);

/* out[i] = base[i]^exponent mod n^2 (generic fixed-exponent batch). */
int cuhe_paillier_modexp(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* exponent,
                         int exponent_words, uint32_t* out, int64_t count);

/* out[i] = base[i]^exponents[i] mod n^2 with a per-item exponent of
 * exponent_words words (fixed 4-bit windows).  Replaces the per-entry
 * gmpy2.powmod of precompute_noise_table (src/cuhepy/paillier/lookup.py:113-117;
 * paillier_GPU_lookup_client.cu:593-626). */
int cuhe_paillier_modexp_each(cuhe_paillier* ctx, const uint32_t* base, const uint32_t* exponents,
                              int exponent_words, uint32_t* out, int64_t count);

/* out[i] = a[i] * b[i] mod n^2.  Replaces Paillier.add / PaillierLookup.add
 * (scheme.py:107-119; lookup.py:282-294) and modmul_pointwise_kernel behind
 * encode_hamming_server (paillier_GPU_lookup_client.cu:811-835, 2312-2335). */
/* Hexadecimal wire format on the device.  from_hex parses `count` strings
 * given as one host text buffer and count + 1 host offsets (string i is
 * text[offsets[i], offsets[i+1]), offsets[0] = 0): an optional 0x / 0X
 * prefix, upper- or lower-case digits, leading zeros allowed; out (host or
 * device, count x K words) receives the little-endian limbs, the digits
 * beyond K words dropped as the reference's hex_to_le_words does
 * (src/cuhepy/paillier/_gpu_ext/paillier_GPU_client.cu:218-262); any other
 * character returns CUHE_INVALID_ARGUMENT with "Invalid hex digit" (its
 * hex_nibble).  reduce != 0 then reduces every value mod n^2 on the device
 * (the reference's CGBN products reduce inputs of any width).  to_hex writes
 * count x 8K lowercase digits, most significant first, leading zeros kept
 * (the reference's le_words_to_hex strips them; the caller does).  Replace
 * the per-string host conversions of paillier_GPU_client.cu:235-279. */
int cuhe_paillier_from_hex(cuhe_paillier* ctx, const char* text, const int64_t* offsets, int64_t count, int reduce,
                           uint32_t* out);
int cuhe_paillier_to_hex(cuhe_paillier* ctx, const uint32_t* limbs, int64_t count, char* out);

int cuhe_paillier_mulmod(cuhe_paillier* ctx, const uint32_t* a, const uint32_t* b, uint32_t* out,
                         int64_t count);

/* out[q*nx + j] = query[q] * index[j] mod n^2: encode_hamming_server for a
 * batch of queries against a resident index (one Montgomery product each). */
int cuhe_paillier_mulmod_outer(cuhe_paillier* ctx, const uint32_t* query, int64_t nq,
                               const uint32_t* index, int64_t nx, uint32_t* out);

/* Install the fixed-base tables of Paillier-Lookup in normal (non-Montgomery)
 * form: g_table[(i*256 + j)*K ...] = g_table[i][j] and noise[k*K ...].
 * Replaces load_config(tables) / ensure_device_tables_
 * (paillier_GPU_lookup_client.cu:1771-1836, 2625-2652). */
int cuhe_lookup_set_tables(cuhe_paillier* ctx, const uint32_t* g_table, int message_chunks,
                           const uint32_t* noise, int noise_entries);
/* Build g_table[i][j] = (g^(2^(8i)))^j on the device (lookup.py:104-110;
 * precompute_g_table, paillier_GPU_lookup_client.cu:550-588) and install the
 * given noise table.  noise may be NULL to keep the current one. */
int cuhe_lookup_build_tables(cuhe_paillier* ctx, const uint32_t* g, int message_chunks,
                             const uint32_t* noise, int noise_entries);
/* Copy the installed g_table back in normal form (dump_tables,
 * paillier_GPU_lookup_client.cu:1838-1862).  out holds message_chunks*256*K words. */
int cuhe_lookup_get_g_table(cuhe_paillier* ctx, uint32_t* out);

/* Encrypt binary embeddings bits[vectors][embed_len] (0/1 bytes) into
 * vectors*chunk_num ciphertexts (chunk_len = 2*key_len bits of Hamming-padded
 * plaintext per chunk) using 14 caller-supplied noise indices per ciphertext.
 * Replaces PaillierGPULookupClient.encrypt / encrypt_kernel
 * (paillier_GPU_lookup_client.cu:1873-2002, 839-948) and
 * PaillierLookupCPU.encrypt (hamming/paillier_lookup.py:199-219). */
int cuhe_lookup_encrypt_bits(cuhe_paillier* ctx, const uint8_t* bits, int64_t vectors, int embed_len,
                             int chunk_len, int chunk_num, const uint8_t* noise_index, uint32_t* out);

/* The 16-bit-digit encryption table.  Pairs of the table's 8-bit digits are
 * looked up as one entry W[j][D] = G[2j][D mod 256] * G[2j+1][D / 256] (mod
 * n^2, Montgomery form), so each ciphertext takes half the table products and
 * the ciphertexts are the same.  The table holds (message_chunks + 1) / 2 *
 * 65,536 entries, K words each (4 GiB at key_len 1024), or 5K/8 doubles each
 * when the FP64 pipe is selected (cuhe_paillier_set_fp64; 5 GiB at key_len
 * 1024, with the noise table converted likewise, and the products then run
 * on that pipe), and costs one or two products per entry to build, which
 * about 150,000 encryptions repay.  mode 1 (the
 * default) builds it during an encryption call of at least 65,536
 * ciphertexts, when it takes at most 8 GiB and a quarter of the free device
 * memory; mode 2 builds it at the next encryption call of any size
 * (CUHE_OUT_OF_MEMORY without the memory); mode 0 frees it and keeps the
 * 8-bit table.  Installing new tables drops it.  The table is built for the
 * pipe selected at that time.  If cuhe_paillier_set_fp64 later selects the
 * other pipe, the table is kept; FP64-form limbs are then left unused and the
 * 8-bit table serves, while a word table still serves the FP64 selection on
 * the integer pipe.  Call mode 0, then mode 2, to rebuild it for the new
 * pipe.  ready returns 1 once it is built.  No reference counterpart (the
 * reference multiplies one entry per 8-bit digit, lookup.py:213-252). */
int cuhe_lookup_set_wide_table(cuhe_paillier* ctx, int mode);
int cuhe_lookup_wide_table_ready(const cuhe_paillier* ctx);

/* Encrypt plaintexts m[i] < n (K-word stride) by table product.  Replaces
 * PaillierLookup.encrypt (lookup.py:213-252) and encrypt_cts
 * (paillier_GPU_lookup_client.cu:2006-2131, 951-1011). */
int cuhe_lookup_encrypt_ints(cuhe_paillier* ctx, const uint32_t* m, int64_t count,
                             const uint8_t* noise_index, uint32_t* out);

/* Measure the integer multiply roofline of a device: 32x32->64-bit word
 * products per second over all SMs, the largest of three probe kernels: one
 * issuing mad.lo.u32 + mad.hi.u32 pairs on independent accumulators, one
 * issuing mad.wide.u32 on independent 64-bit accumulators, one running the
 * modexp kernel's own carry-chained multiply-accumulate row
 * (mad.lo.cc / madc.hi.cc) on four independent accumulator sets.  No
 * counterpart in the reference; it provides the denominator of the modexp
 * roofline. */
int cuhe_imad_peak(int device, double* word_products_per_second);
/* Measured FP64-pipe rate of `device` (fused multiply-adds per second, eight
 * independent chains per thread, the rounding of the limb products), the
 * ceiling of the FP64-pipe decode.  No reference counterpart. */
int cuhe_fp64_peak(int device, double* fp64_per_second);

/* Host-only helper (no device needed): the left-to-right sliding-window
 * schedule used for a fixed exponent.  Writes at most capacity ops, each
 * (squarings << 16) | (odd-power index + 1), and returns the op count.  It
 * has no counterpart in the reference; it exists so the schedule can be
 * checked on a machine without a GPU. */
int cuhe_window_schedule(const uint32_t* exponent, int exponent_words, int window, int32_t* ops, int capacity);

/* Select (threads per instance, window) for this context's width; 0 picks the
 * built-in default.  Used by the autotuner. */
int cuhe_paillier_set_tuning(cuhe_paillier* ctx, int threads_per_instance, int window);
int cuhe_paillier_get_tuning(const cuhe_paillier* ctx, int* threads_per_instance, int* window);

/* Mixed batches.  A cuhe_mix collects fixed-exponent exponentiations
 * out[i] = base[i]^e mod n^2 of uneven sizes over several keys and widths
 * (each added with its context and device buffers), and runs them as one
 * persistent launch per width: CTAs take units of a few instances from a
 * global counter until every batch is done, so small batches do not leave
 * the GPU idle between launches.  cuhe_mix_launch only enqueues work on the
 * given stream (no allocation, no synchronisation), so it can be captured
 * in a CUDA graph; the kernels of the second and later widths run on the
 * mix's own streams, forked from and joined back to the given stream, so a
 * width's last wave overlaps the next width's kernel.  cuhe_mix_plan (after
 * the last add or tuning change) builds the schedules, task tables and
 * those streams and must run outside capture.
 * cuhe_mix_check waits for the device and reports range errors (a base not
 * below n^2).  Contexts and buffers must outlive the mix.  No counterpart in
 * the reference, which launches one kernel per call
 * (paillier_GPU_client.cu:873-974). */
typedef struct cuhe_mix cuhe_mix;
int cuhe_mix_create(int device, cuhe_mix** out);
void cuhe_mix_destroy(cuhe_mix* mix);
const char* cuhe_mix_last_error(const cuhe_mix* mix);
int cuhe_mix_add_modexp(cuhe_mix* mix, cuhe_paillier* ctx, const uint32_t* base, uint32_t* out, int64_t count,
                        const uint32_t* exponent, int exponent_words);
/* (threads per instance, window) of the persistent launch for one width. */
int cuhe_mix_set_tuning(cuhe_mix* mix, int words, int threads_per_instance, int window);
int cuhe_mix_plan(cuhe_mix* mix);
int cuhe_mix_launch(cuhe_mix* mix, void* stream);
int cuhe_mix_check(cuhe_mix* mix);
/* Planned widths (ascending words) and, per width, its tuning, grid, CTA
 * units and batch count. */
int cuhe_mix_widths(const cuhe_mix* mix);
int cuhe_mix_info(const cuhe_mix* mix, int index, int* words, int* threads_per_instance, int* window, int* grid,
                  int64_t* units, int* tasks);

#ifdef __cplusplus
}
#endif

#endif /* CUHE_PAILLIER_H */
