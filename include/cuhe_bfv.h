/* C ABI of the B200 BFV evaluator (libcuhe_bfv_b200.so).
 *
 * Replaces the CPython module _bfv_rns (ABI_VERSION 4) of the reference,
 * src/cuhepy/bfv/_cpu_ext/bindings.cpp:405-433: rings whose ciphertext
 * modulus Q is a product of the first 60-bit NTT primes (the reference's
 * "residue" backend) and rings with any odd modulus q up to 512 bits (its
 * "native" backend).  Handles are reference counted: a key keeps its ring
 * alive and a server keeps its keys alive (bindings.cpp:25-38).
 *
 * Buffers: a "poly" is N coefficients of coefficient_bytes little-endian
 * bytes each (bindings.cpp:43-82); a "packed poly" is N coefficients of
 * bits(modulus) bits each, bit-packed little-endian (packed_wire.h:21-60).
 * All pointers are host memory.  Return codes follow cuhe_status of
 * cuhe_paillier.h; cuhe_bfv_last_error() gives the message of the last
 * failure on the calling thread.
 */
#ifndef CUHE_BFV_H
#define CUHE_BFV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cuhe_bfv_ring cuhe_bfv_ring;
typedef struct cuhe_bfv_key cuhe_bfv_key;
typedef struct cuhe_bfv_server cuhe_bfv_server;

const char* cuhe_bfv_last_error(void);

/* create_ring(n, q_hex, digit_bits, fast, residue, kernel_level)
 * (bindings.cpp:120-136).  residue != 0: q must be a product of the first
 * 60-bit NTT primes (the reference's residue backend); residue == 0: any odd
 * q of at most 512 bits (the native backend; exact products over auxiliary
 * primes), kernel_level 0. */
int cuhe_bfv_create_ring(uint64_t n, const char* q_hex, uint64_t digit_bits, int fast, int residue,
                         uint64_t kernel_level, int device, cuhe_bfv_ring** out);
void cuhe_bfv_ring_release(cuhe_bfv_ring* ring);
/* ring_info (bindings.cpp:254-270): primes (capacity entries), counts and
 * the bytes of the NTT tables. */
int cuhe_bfv_ring_info(const cuhe_bfv_ring* ring, uint64_t* primes, int capacity, int* prime_count,
                       int* switch_prime_count, int* residue_prime_count, uint64_t* table_bytes,
                       uint64_t* coefficient_bytes, int* kernel_level, int* fast);

/* compile_key(ring, ((b, a),) * digits) (bindings.cpp:194-208): the key as
 * digits*2 consecutive polys b_0, a_0, b_1, a_1, ... */
int cuhe_bfv_compile_key(cuhe_bfv_ring* ring, const uint8_t* key_polys, uint64_t digits, cuhe_bfv_key** out);
void cuhe_bfv_key_release(cuhe_bfv_key* key);
uint64_t cuhe_bfv_key_bytes(const cuhe_bfv_key* key);

/* apply_key(key, poly) -> (b, a) (bindings.cpp:210-220). out: 2 polys. */
int cuhe_bfv_apply_key(cuhe_bfv_key* key, const uint8_t* poly, uint8_t* out);
/* ring_product(ring, lhs, rhs) mod q (bindings.cpp:222-236). */
int cuhe_bfv_ring_product(cuhe_bfv_ring* ring, const uint8_t* lhs, const uint8_t* rhs, uint8_t* out);
/* multiply(ring, lhs2, rhs2 or NULL, t) -> 3 polys (bindings.cpp:238-252). */
int cuhe_bfv_multiply(cuhe_bfv_ring* ring, const uint8_t* lhs, const uint8_t* rhs, uint64_t t, uint8_t* out);
/* rotate_rows(key, ct2, exponent) -> 2 polys (bindings.cpp:154-165). */
int cuhe_bfv_rotate_rows(cuhe_bfv_key* key, const uint8_t* ct, uint64_t exponent, uint8_t* out);
/* hamming_tile(relin, query2, tile2, ((g, key),...), mask, t) -> 2 polys
 * (bindings.cpp:167-192). */
int cuhe_bfv_hamming_tile(cuhe_bfv_key* relin, const uint8_t* query, const uint8_t* tile,
                          const uint64_t* exponents, cuhe_bfv_key* const* keys, uint64_t rotations,
                          const uint8_t* mask, uint64_t t, uint8_t* out);

/* create_server(relin, ((g, key),...), padded, t, target_hex)
 * (bindings.cpp:278-313). */
int cuhe_bfv_create_server(cuhe_bfv_key* relin, const uint64_t* exponents, cuhe_bfv_key* const* keys,
                           uint64_t count, uint64_t padded, uint64_t t, const char* target_hex,
                           cuhe_bfv_server** out);
void cuhe_bfv_server_release(cuhe_bfv_server* server);
uint64_t cuhe_bfv_server_bytes(const cuhe_bfv_server* server);
/* Geometry of a server: vectors per tile (capacity), bytes of one packed
 * input poly, and of one packed output poly with and without compaction. */
int cuhe_bfv_server_layout(const cuhe_bfv_server* server, uint64_t* capacity, uint64_t* padded,
                           uint64_t* input_packed_bytes, uint64_t* output_packed_bytes,
                           uint64_t* compact_packed_bytes);

/* packed_search(server, (b, a), ((b, a),...), count, compact)
 * (bindings.cpp:329-367): query = 2 packed polys, index = tiles*2 packed
 * polys, tiles == ceil(count / capacity).  Writes responses*2 packed polys
 * (responses = ceil(tiles / padded)) into out, whose size must be
 * out_capacity bytes or more; *responses receives the count. */
int cuhe_bfv_packed_search(cuhe_bfv_server* server, const uint8_t* query, const uint8_t* index,
                           uint64_t tiles, uint64_t count, int compact, uint8_t* out, uint64_t out_capacity,
                           uint64_t* responses);

/* Serving form of packed_search: upload an encrypted index once (validated,
 * unpacked and kept resident in HBM), then search it with any number of
 * queries.  Results are identical to packed_search on the same bytes.  No
 * counterpart in the reference, whose packed_search re-imports the index on
 * every call (bindings.cpp:340-351). */
typedef struct cuhe_bfv_index cuhe_bfv_index;
int cuhe_bfv_upload_index(cuhe_bfv_server* server, const uint8_t* index, uint64_t tiles, cuhe_bfv_index** out);

/* packed_search and upload_index with the index given as 2 * tiles
 * pointers, one per packed polynomial (b_0, a_0, b_1, a_1, ...), so that a
 * caller holding the polynomials in separate buffers (the reference API's
 * tuple of bytes pairs) need not join them first.  The library gathers them
 * into pinned staging memory with several host threads and copies each
 * chunk to the device in one transfer.  Same results as the contiguous
 * forms. */
int cuhe_bfv_packed_search_parts(cuhe_bfv_server* server, const uint8_t* query, const uint8_t* const* polys,
                                 uint64_t tiles, uint64_t count, int compact, uint8_t* out, uint64_t out_capacity,
                                 uint64_t* responses);
int cuhe_bfv_upload_index_parts(cuhe_bfv_server* server, const uint8_t* const* polys, uint64_t tiles,
                                cuhe_bfv_index** out);
void cuhe_bfv_index_release(cuhe_bfv_index* index);
int cuhe_bfv_search_index(cuhe_bfv_server* server, cuhe_bfv_index* index, const uint8_t* query, uint64_t count,
                          int compact, uint8_t* out, uint64_t out_capacity, uint64_t* responses);

/* Per-phase device times (milliseconds) of the last packed_search on this
 * server, in the phase order tensor, relinearize, rotate, mask, merge,
 * output.  No counterpart in the reference; it feeds the profile_* calls. */
int cuhe_bfv_last_profile(const cuhe_bfv_server* server, double* ms, int capacity);

/* Batched negacyclic NTT of device-resident residue planes ([planes][N]
 * u64, plane b reduced mod the ring's prime b % primes, canonical in and
 * out): forward (bit-reversed output) or inverse (bit-reversed input,
 * 1/N folded in), in place.  Enqueued on `stream` (a cudaStream_t) with no
 * allocation or synchronisation, so it can be captured in a CUDA graph.
 * threads: CTA size (0: N/8, at most 1024; radix 16 has a smaller,
 * register-bound limit that a larger request exceeds with an error);
 * radix_log: register pass width, 1..4 stages (0: 3).  These two are the
 * knobs of the autotuner (at N = 32768 they are checked but the fixed split
 * transform runs: the two halves of a plane in shared memory, the stage that
 * pairs them on global memory).  The transform the reference runs per prime
 * (rns_ntt.h:178-255), batched. */
int cuhe_bfv_ntt(cuhe_bfv_ring* ring, uint64_t* planes, uint64_t count, int primes, int inverse, int threads,
                 int radix_log, void* stream);

/* Batch encoding mod t of `count` slot vectors ([count][N], < t, in the
 * reference's slot order; bfv/scheme.py:371-394): out receives the
 * [count][N] plaintext coefficients.  t prime with t = 1 mod 2N. */
int cuhe_bfv_batch_encode(cuhe_bfv_ring* ring, uint64_t t, const uint32_t* slots, uint64_t count, uint64_t* out);

/* Client-side public-key encryption of `count` batched plaintexts
 * (bfv/scheme.py:426-444 with the batch encoding of 371-394): for each c,
 *   m  = batch_encode(slots[c])                    (mod t)
 *   c0 = b u + e0 + floor(Q/t) m,  c1 = a u + e1   (mod Q)
 * with pk = (b, a) as two fixed-width polys, slots [count][N] (< t, in the
 * reference's slot order), u [count][N] ternary and e [count][2][N] signed
 * small noise drawn by the caller.  out receives count * 2 packed polys
 * (bits(Q) bits per coefficient, the packed_search wire), c0 then c1.
 * Residue rings only; t prime with t = 1 mod 2N.  The device copies of the
 * slots, u, e, the encoded message and NTT(u) are zeroed before the call
 * returns (on success and on error). */
int cuhe_bfv_encrypt(cuhe_bfv_ring* ring, const uint8_t* pk, uint64_t t, const uint32_t* slots, const int8_t* u,
                     const int8_t* e, uint64_t count, uint8_t* out);

/* The same encryption with the noise drawn on the device from a ChaCha20
 * keystream (RFC 8439 block function) under `key` (32 bytes) and `nonce`
 * (12 bytes), which the caller takes from a cryptographic generator and never
 * reuses.  The distributions are the reference's (bfv/scheme.py:236-246):
 * u uniform on {-1, 0, 1}, each e the difference of the popcounts of two
 * independent eta-bit words (eta 1..63).  Ciphertext c of the call uses the
 * keystream blocks with counters c * B .. c * B + B - 1, B = E + N/8:
 *   blocks [0, E), E = N/4 (eta <= 31) or N/2: the e words, little-endian,
 *     4 bytes each (eta <= 31) or 8, in pairs; pair v gives
 *     e[c][v / N][v % N] = popcount(w0 & mask) - popcount(w1 & mask);
 *   blocks [E, B): 8 bytes per coefficient i, u[c][i] = (first byte below
 *     255) % 3 - 1.
 * Eight bytes of 255 (probability 2^-64 per coefficient) return CUHE_RANGE:
 * encrypt again with a new key.  count * B must not exceed 2^32.  Replaces
 * the host-side draws of bfv/scheme.py:236-246 feeding BFV.encrypt
 * (scheme.py:426-444). */
int cuhe_bfv_encrypt_keyed(cuhe_bfv_ring* ring, const uint8_t* pk, uint64_t t, const uint32_t* slots,
                           const uint8_t* key, const uint8_t* nonce, unsigned eta, uint64_t count, uint8_t* out);

/* Execution lanes of a ring (1..8; 1 after create_ring).  Each lane is a
 * CUDA stream with its own device workspace.  packed_search / search_index
 * calls issued concurrently from several host threads take free lanes and
 * overlap on the GPU; every other call runs on lane 0.  Lane streams have
 * the device's highest stream priority, so a search's short dependent
 * kernels are scheduled ahead of queued blocks of bulk work on
 * default-priority streams.  Each lane keeps the workspace of the largest
 * search it ran until the ring is released.  No
 * counterpart in the reference, whose calls release the GIL but run on the
 * host (src/cuhepy/bfv/_cpu_ext/bindings.cpp:20-23). */
int cuhe_bfv_set_lanes(cuhe_bfv_ring* ring, int lanes);
int cuhe_bfv_get_lanes(const cuhe_bfv_ring* ring);
/* Device workspace (bytes) one lane holds for a search over `tiles` tiles:
 * searches run in chunks of about 1024 tiles, so this is the size of the
 * largest chunk (about 4.4 GB at N = 8192, L = 3, K = 7 for 1024 tiles).
 * Serving code admits a search when this fits in free device memory. */
uint64_t cuhe_bfv_search_workspace(const cuhe_bfv_server* server, uint64_t tiles, int compact);

/* Allocate that workspace now on every active lane of the server's ring
 * (each lane's device arena grows to it), so that later searches of up to
 * `tiles` tiles allocate nothing: a device allocation inside a search can
 * wait for unrelated work running on the GPU.  No counterpart in the
 * reference (serving addition). */
int cuhe_bfv_reserve_workspace(cuhe_bfv_server* server, uint64_t tiles, int compact);

#ifdef __cplusplus
}
#endif

#endif /* CUHE_BFV_H */
