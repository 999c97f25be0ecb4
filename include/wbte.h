/*
 * wbte.h -- C ABI of libwbte, the sm_100a (B200) implementation of the
 * batched threshold-decryption path of the btx / weighted_btx / pfe /
 * weighted_pfe crates over BLS12-381.
 *
 * The reference crates reach all of their heavy arithmetic through blst's C
 * ABI (blst 0.3.17 via blstrs 0.7.1).  Each entry point below replaces one of
 * those call sites, or one hot loop of the crate that is built from them, and
 * keeps blst's memory layout so that Rust wrappers can pass the same buffers:
 *
 *   Fp     48 bytes: 6 little-endian 64-bit limbs, Montgomery form, R = 2^384
 *   G1     96 bytes: affine (x, y)                    (blst_p1_affine)
 *   G2    192 bytes: affine (x.c0, x.c1, y.c0, y.c1)  (blst_p2_affine)
 *   GT    576 bytes: Fp12, c0.c0.c0 first             (blst_fp12)
 *   Fr     32 bytes: canonical little-endian integer  (Scalar::to_bytes_le,
 *                    the scalar format of blst_p{1,2}s_mult_pippenger)
 *   The point at infinity is all zero bytes (blst's affine convention).
 *
 * Buffers.  Every data pointer may be host memory or device memory of the
 * context's GPU; the library detects which.  Host inputs are copied in, host
 * outputs are copied out before the call returns (the call is then
 * synchronous).  When every data pointer is device memory the call only
 * enqueues work on the context's stream and returns; synchronise with
 * wbte_ctx_synchronize().  Arrays of indices and offsets marked "host" must
 * be host memory.  Callers own all buffers; nothing is retained after the
 * call except the context's own caches (twiddle tables, generator tables).
 *
 * Errors.  Every function returns 0 (WBTE_OK) or a negative status; the
 * message of the last failure is available from wbte_ctx_last_error().
 * Results never depend on launch configuration.
 */
#ifndef WBTE_H
#define WBTE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WBTE_OK 0
#define WBTE_ERR_INVALID_ARG (-1)
#define WBTE_ERR_SIZE (-2)
#define WBTE_ERR_OOM (-3)
#define WBTE_ERR_TIMEOUT (-4)
#define WBTE_ERR_CUDA (-5)
#define WBTE_ERR_NOT_ON_CURVE (-6)
#define WBTE_ERR_INTERPOLATION (-7)
#define WBTE_ERR_INTERNAL (-8)

#define WBTE_FE_FULL 0
#define WBTE_FE_EASY 1
#define WBTE_FE_HARD 2

typedef struct wbte_ctx wbte_ctx;

/* ------------------------------------------------------------ context */
int32_t wbte_version(void);
/* One context per GPU and caller thread.  hbm_budget_bytes = 0: no limit. */
int32_t wbte_ctx_create(int32_t device, uint64_t hbm_budget_bytes, wbte_ctx **out);
int32_t wbte_ctx_destroy(wbte_ctx *ctx);
/* Use a caller-owned cudaStream_t (NULL: the context's own non-blocking
 * stream; cudaStreamLegacy to order with the legacy default stream). */
int32_t wbte_ctx_set_stream(wbte_ctx *ctx, void *cuda_stream);
int32_t wbte_ctx_synchronize(wbte_ctx *ctx);
/* Knobs of the launchers' cost models for every later call on this context
 * (the per-size-class autotuner sets them; results never depend on them):
 *   WBTE_TUNE_GT_LANES     lanes per GT exponentiation in the radix-4 stages
 *                          of the GT transforms: 1, 2 or 4 (0: cost model)
 *   WBTE_TUNE_MSM_WINDOW   Pippenger window width c, 4..13 (0: cost model)
 *   WBTE_TUNE_MSM_SEGMENTS sorted-term segments per (MSM, window), 1..1024
 *                          (0: cost model)
 *   WBTE_TUNE_NTT_JOINT    G1/G2 transform stages: 1 one thread per
 *                          butterfly, 0 the lane split (-1: cost model)
 *   WBTE_TUNE_MILLER_CHUNK pairs per thread of the share checks' unprepared
 *                          multi-Miller loops, 1..8 (0: cost model)
 * WBTE_ERR_INVALID_ARG for an unknown knob or a value out of range. */
#define WBTE_TUNE_GT_LANES 1
#define WBTE_TUNE_MSM_WINDOW 2
#define WBTE_TUNE_MSM_SEGMENTS 3
#define WBTE_TUNE_NTT_JOINT 4
#define WBTE_TUNE_MILLER_CHUNK 5
int32_t wbte_ctx_set_tuning(wbte_ctx *ctx, int32_t knob, int64_t value);
const char *wbte_ctx_last_error(const wbte_ctx *ctx);
/* Number of kernels the library has launched so far (all contexts). */
uint64_t wbte_ctx_launch_count(const wbte_ctx *ctx);
/* Kernels the library has launched from the calling thread so far. */
uint64_t wbte_thread_launch_count(void);
/* Per-kernel timing.  While enabled, every kernel launch is bracketed by CUDA
 * events on its stream; enabling (or disabling) clears the records.
 * wbte_profile_read synchronises the device and returns, per kernel name,
 * the summed milliseconds and the number of launches (names are written as
 * NUL-terminated strings name_stride bytes apart). */
int32_t wbte_profile_enable(int32_t on);
/* Measures the sustained rate of 32-bit integer multiply-add instructions
 * (mad.lo/mad.hi) on the context's GPU with a calibration kernel; the
 * denominator of the integer-pipe roofline.  Synchronous. */
int32_t wbte_measure_imad_rate(wbte_ctx *ctx, double *imad_per_s);
int32_t wbte_profile_read(char *names, int32_t name_stride, double *ms, int64_t *counts,
                          int32_t max_entries, int32_t *n_out);

/* --------------------------------------------------------------- MSM */
/* Replaces blst_p1s_mult_pippenger with nbits = 255, one contiguous block
 * (weighted_btx/src/blst_utils.rs:43-67 g1_multi_exp_affine_bytes).
 * out: one G1.  n = 0 gives the identity. */
int32_t wbte_g1_msm(wbte_ctx *ctx, void *out, const void *points, const void *scalars, uint64_t n);
/* Replaces blst_p2s_mult_pippenger (weighted_btx/src/blst_utils.rs:88-99). */
int32_t wbte_g2_msm(wbte_ctx *ctx, void *out, const void *points, const void *scalars, uint64_t n);
/* The G1 MSM of wbte_g1_msm for callers that must not allocate device
 * memory while they serve a request -- for example a service that reserved
 * HBM up front for its resident keys and buffers, where a new allocation
 * could fail under memory pressure mid-request, stall on device-wide
 * synchronisation, or fragment the partition.  It has no counterpart in the
 * reference (blst takes caller scratch; this entry point needs none).
 * Working memory is one fixed 8 MiB array in the library's device image,
 * held by every GPU that loads the library until the process exits; the
 * call allocates nothing and needs no context.
 *   - out, points, scalars: device memory of the current device (host,
 *     managed and other GPUs' pointers are rejected with
 *     WBTE_ERR_INVALID_ARG); stream: a cudaStream_t (NULL: legacy default
 *     stream).  Asynchronous.
 *   - n <= 16384 points (every such n runs; larger n returns WBTE_ERR_SIZE).
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make that first call before any stream capture.
 *   - Every call shares the array and it keeps the last call's contents:
 *     calls whose work overlaps on the GPU (other streams, other threads)
 *     race and give wrong results; serialise them on one stream. */
int32_t wbte_g1_msm_static(void *out, const void *points, const void *scalars, uint64_t n, void *stream);
/* k MSMs of common length n in one launch sequence:
 *   out[j] = sum_t scalars[v_j * n + t] * points[point_base[j] + idx[t]]
 * with idx = point_index (NULL: t) and v_j = scalar_vector[j] (NULL: 0).
 * scalars holds num_vectors vectors of n scalars; points holds n_points.
 * Replaces the per-block and per-index calls of
 * weighted_btx/src/blst_utils.rs:106-152 (g2_multi_exp_affine_indexed,
 * g2_multi_exp_affine_raw) as issued by weighted_btx/src/decryption.rs:463-521.
 * point_base (k entries), point_index (n) and scalar_vector (k) are host. */
int32_t wbte_g1_msm_family(wbte_ctx *ctx, void *out, const void *points, uint64_t n_points,
                           const int64_t *point_base, const int32_t *point_index,
                           const void *scalars, const int32_t *scalar_vector, int32_t num_vectors,
                           uint64_t k, uint64_t n);
int32_t wbte_g2_msm_family(wbte_ctx *ctx, void *out, const void *points, uint64_t n_points,
                           const int64_t *point_base, const int32_t *point_index,
                           const void *scalars, const int32_t *scalar_vector, int32_t num_vectors,
                           uint64_t k, uint64_t n);

/* ------------------------------------------------- point arithmetic */
/* out[i] = scalars[i] * points[fixed_base ? 0 : i], affine out
 * (blstrs G1Projective * Scalar followed by blst_p1s_to_affine,
 * weighted_btx/src/blst_utils.rs:11-36). */
int32_t wbte_g1_mul(wbte_ctx *ctx, void *out, const void *points, int32_t fixed_base, const void *scalars, uint64_t n);
int32_t wbte_g2_mul(wbte_ctx *ctx, void *out, const void *points, int32_t fixed_base, const void *scalars, uint64_t n);
/* out[i] = scalars[i] * generator (G1Projective::generator() * s,
 * weighted_btx/src/encryption.rs:34 and setup.rs:476-484 append_g2_block). */
int32_t wbte_g1_mul_generator(wbte_ctx *ctx, void *out, const void *scalars, uint64_t n);
int32_t wbte_g2_mul_generator(wbte_ctx *ctx, void *out, const void *scalars, uint64_t n);
/* out[j] = sum of in[offsets[j] .. offsets[j+1]) (offsets host, k+1 entries). */
int32_t wbte_g1_sum(wbte_ctx *ctx, void *out, const void *in, const int64_t *offsets, uint64_t k);
int32_t wbte_g2_sum(wbte_ctx *ctx, void *out, const void *in, const int64_t *offsets, uint64_t k);
/* Projective to affine for n points (blst_p1s_to_affine / blst_p2s_to_affine
 * as called by batch_normalize_g1/g2, weighted_btx/src/blst_utils.rs:11-36):
 * in holds blst_p1 / blst_p2 records (Jacobian X, Y, Z; x = X/Z^2, y = Y/Z^3;
 * 144 / 288 bytes), out affine points; Z = 0 gives the identity.  Chunks of
 * consecutive points share one field inversion (Montgomery's trick).  out
 * and in must not overlap. */
int32_t wbte_g1_batch_normalize(wbte_ctx *ctx, void *out, const void *in, uint64_t n);
int32_t wbte_g2_batch_normalize(wbte_ctx *ctx, void *out, const void *in, uint64_t n);
/* ZCash compressed encodings, 48 / 96 bytes per point (to_compressed). */
int32_t wbte_g1_compress(wbte_ctx *ctx, void *out, const void *in, uint64_t n);
int32_t wbte_g2_compress(wbte_ctx *ctx, void *out, const void *in, uint64_t n);
/* Decoding of compressed points, as blstrs' checked G1Affine / G2Affine
 * ::from_compressed used when the crates deserialize keys and ciphertexts
 * (serde of the key material, weighted_btx/src/setup.rs:21-61; the wire sizes
 * of weighted_pfe/README.md:159-214): ZCash flags (0x80 compressed, 0x40
 * infinity, 0x20 larger y), canonical x, y from the curve equation, and when
 * check_group is nonzero [r]P = O.  n points of 48 (G1) or 96 (G2) bytes in,
 * affine points out; status (n bytes, may be NULL) per point: 0 ok, 1 bad
 * encoding, 2 not on the curve, 3 not in the subgroup, the point then written
 * as the identity.  Returns WBTE_ERR_NOT_ON_CURVE if any point was rejected. */
int32_t wbte_g1_decompress(wbte_ctx *ctx, void *out, uint8_t *status, const void *in, uint64_t n,
                           int32_t check_group);
int32_t wbte_g2_decompress(wbte_ctx *ctx, void *out, uint8_t *status, const void *in, uint64_t n,
                           int32_t check_group);

/* ------------------------------------------------------- transforms */
/* In-place radix-2 transform of n affine points over the size-n subgroup of
 * Fr: inverse = 0 is Radix2Domain::fft, inverse = 1 is ifft_unscaled
 * (btx/src/fft.rs:197-234, 357-411). */
int32_t wbte_g1_ntt(wbte_ctx *ctx, void *io, uint64_t n, int32_t inverse);
int32_t wbte_g2_ntt(wbte_ctx *ctx, void *io, uint64_t n, int32_t inverse);
/* In-place unscaled transform of n GT elements (ifft_gt_unscaled,
 * btx/src/fft.rs:242-274, and the forward fft for inverse = 0). */
int32_t wbte_gt_ntt(wbte_ctx *ctx, void *io, uint64_t n, int32_t inverse);
/* Truncated unscaled inverse transform over easy-final-exponentiated values;
 * the first out_count outputs are valid afterwards
 * (ifft_cyclotomic_prefix_unscaled, btx/src/fft.rs:284-350). */
int32_t wbte_gt_cyclotomic_prefix_ifft(wbte_ctx *ctx, void *io, uint64_t n, uint64_t out_count);
/* The two transforms above over count independent arrays of n values laid
 * back to back (array q at io + q * n * 576 bytes), one launch per stage for
 * all of them: the batched form of the reference's per-batch transforms. */
int32_t wbte_gt_ntt_many(wbte_ctx *ctx, void *io, uint64_t n, uint64_t count, int32_t inverse);
int32_t wbte_gt_cyclotomic_prefix_ifft_many(wbte_ctx *ctx, void *io, uint64_t n, uint64_t out_count,
                                            uint64_t count);

/* ----------------------------------------------------------- pairing */
/* Line tables of n G2 points: 68 lines x 288 bytes each, laid out
 * line-major (line s of point i at offset (s * n + i) * 288).
 * Replaces blst_precompute_lines (btx/src/final_exponentiation.rs:185-195). */
int32_t wbte_g2_prepare_lines(wbte_ctx *ctx, void *lines, const void *q, uint64_t n);
/* out[i] = Miller loop of (p[i], lines of point i); replaces
 * blst_miller_loop_lines (btx/src/final_exponentiation.rs:206-219). */
int32_t wbte_miller_loop_lines(wbte_ctx *ctx, void *out, const void *lines, const void *p, uint64_t n);
/* out[i] = Miller loop of (p[i], q[i]). */
int32_t wbte_miller_loop(wbte_ctx *ctx, void *out, const void *p, const void *q, uint64_t n);
/* out[j] = product over pairs [offsets[j], offsets[j+1]) of Miller loops,
 * identities contributing 1; replaces blst_miller_loop_n as used by
 * unprepared_multi_miller_loop (weighted_btx/src/final_exponentiation.rs:229-274).
 * offsets host, k+1 entries. */
int32_t wbte_multi_miller_loop(wbte_ctx *ctx, void *out, const void *p, const void *q,
                               const int64_t *offsets, uint64_t k);
/* mode WBTE_FE_FULL replaces blst_final_exp; WBTE_FE_EASY / WBTE_FE_HARD are
 * easy_final_exponentiation and hard_final_exponentiation
 * (btx/src/final_exponentiation.rs:276-336). */
int32_t wbte_final_exp(wbte_ctx *ctx, void *out, const void *in, uint64_t n, int32_t mode);
/* out[i] = base[fixed_base ? 0 : i] ^ scalars[i] on GT (Gt * Scalar; the
 * decomposed action of btx/src/fft.rs:73-154). */
int32_t wbte_gt_pow(wbte_ctx *ctx, void *out, const void *base, int32_t fixed_base, const void *scalars, uint64_t n);
/* out[i] = a[i] * b[i] in Fp12 (blst_fp12_mul). */
int32_t wbte_fp12_mul(wbte_ctx *ctx, void *out, const void *a, const void *b, uint64_t n);
/* Tagged torus encoding of GT, 289 bytes per element: 0 then zeros for the
 * identity, else 1 then (c0 + 1) / c1 (append_gt, weighted_btx/src/encoding.rs:11-19). */
int32_t wbte_gt_compress(wbte_ctx *ctx, void *out, const void *in, uint64_t n);

/* ----------------------------------------------------------- scalars */
/* Lagrange coefficients at zero of n distinct points
 * (lagrange_at_zero, weighted_btx/src/interpolation.rs:31-52). */
int32_t wbte_lagrange_at_zero(wbte_ctx *ctx, void *out, const void *points, uint64_t n);
/* valid[i] = 1 iff [s_i] G1 == R_i + [c_i] X_i (SchnorrProof::verify,
 * weighted_btx/src/proof.rs:56-70); c_i is the Fiat-Shamir challenge. */
int32_t wbte_schnorr_verify(wbte_ctx *ctx, uint8_t *valid, const void *X, const void *R,
                            const void *s, const void *c, uint64_t n);

/* One field of a Fiat-Shamir transcript.  Record i contributes the len bytes
 * at data + i * stride (stride 0: the same bytes for every record; data may
 * be host or device memory).  kind 0: plain bytes; kind 1: a 289-byte
 * wbte_gt_compress record, which contributes only its tag byte when the tag
 * is 0 (append_gt of the identity, weighted_btx/src/encoding.rs:11-19). */
typedef struct {
    const void *data;
    uint64_t stride;
    uint32_t len;
    uint32_t kind;
} wbte_transcript_field;
/* out[i] (32-byte canonical Fr) = the challenge of record i: the first
 * SHA-256(field_0 || ... || field_{count-1} || counter u32 LE), counter =
 * 0, 1, ..., whose little-endian value is below r -- challenge_scalar of
 * btx/src/proof.rs:49-77, pfe/src/proof.rs:148-176,
 * weighted_btx/src/proof.rs:72-100 and weighted_pfe/src/proof.rs:124-152
 * (Sha256 + Scalar::from_bytes_le).  count <= 8.  WBTE_ERR_INTERNAL if a
 * record exhausts 256 counters. */
int32_t wbte_transcript_challenges(wbte_ctx *ctx, void *out, const wbte_transcript_field *fields, uint32_t count,
                                   uint64_t n);

/* ---------------------------------------------------- weighted_btx */
typedef struct {
    const void *domain_points;     /* total_weight Fr: the virtual points       */
    const void *verification_keys; /* max_batch_size * party_count G2            */
    const void *negative_material; /* max_batch_size * total_weight G2            */
    const void *positive_material; /* (max_batch_size - 1) * total_weight G2      */
    const int64_t *party_offsets;  /* host, party_count + 1 prefix offsets        */
    uint64_t party_count;
    uint64_t total_weight;
    uint64_t max_batch_size;
} wbte_wbtx_key;

/* sigma[j] = sum_i q_j^(i+1) first[i] for the T secrets q (partial_decrypt,
 * weighted_btx/src/decryption.rs:205-233). first: batch_size G1 with the
 * identity at invalid slots. */
int32_t wbte_wbtx_partial_decrypt(wbte_ctx *ctx, void *sigma, const void *first, uint64_t batch_size,
                                  const void *q, uint64_t T);
/* *ok = 1 iff the random-linear aggregate share check passes
 * (verify_decryption_shares_batched, weighted_btx/src/decryption.rs:358-422);
 * with one share and challenge 1 this is verify_decryption_share (:236-272).
 * party_indices host (T entries). */
int32_t wbte_wbtx_verify_shares(wbte_ctx *ctx, int32_t *ok, const wbte_wbtx_key *key,
                                const void *first, const uint8_t *valid, uint64_t batch_size,
                                const void *sigma, const int64_t *party_indices,
                                const void *challenges, uint64_t T);
/* Committee preparation (prepare_decryption, weighted_btx/src/decryption.rs:427-551)
 * for the accepted parties party_indices (host, ascending):
 *   kernel_lines  m * 68 * 288 bytes, m = next_pow2(2 batch_size)
 *   opening_keys  batch_size * T G2, slot-major
 *   kernel        m G2 (the scaled transformed kernel), may be NULL. */
int32_t wbte_wbtx_prepare(wbte_ctx *ctx, const wbte_wbtx_key *key, const int64_t *party_indices, uint64_t T,
                          uint64_t batch_size, void *kernel_lines, void *opening_keys, void *kernel);
/* beta[i] (precompute_batch, weighted_btx/src/decryption.rs:555-603); first
 * carries the identity at invalid slots, beta is the identity there. */
int32_t wbte_wbtx_precompute(wbte_ctx *ctx, void *beta, const void *kernel_lines, const void *first,
                             const uint8_t *valid, uint64_t batch_size);
/* messages[i] = second[i] - alpha_i + beta[i] for valid slots (open_batch,
 * weighted_btx/src/decryption.rs:607-695); invalid slots get the identity. */
int32_t wbte_wbtx_open(wbte_ctx *ctx, void *messages, const void *opening_keys, const void *sigma, uint64_t T,
                       const void *second, const void *beta, const uint8_t *valid, uint64_t batch_size);
/* The batched form: K batches of one size B and one accepted committee per
 * call, batch-major arrays (batch b first).  Each is the K-fold version of the
 * call above it, with every kernel launched once over all K batches:
 *   partial_decrypt_many  sigma K*T G1, first K*B G1, q T Fr
 *   verify_shares_many    ok K int32 (one aggregate check per batch), first
 *                         K*B G1 with the identity at invalid slots, sigma K*T,
 *                         challenges K*T Fr, party_indices T (host)
 *   precompute_many       beta K*B GT over the committee's kernel lines
 *   open_many             messages K*B GT, opening_keys B*T G2 (shared),
 *                         opening_lines: their line tables (wbte_g2_prepare_lines
 *                         of the B*T keys) or NULL; with them each slot's T
 *                         pairings share one multi-Miller loop (in chunks of
 *                         8 pairs),
 *                         sigma K*T G1, second/beta K*B GT, valid K*B. */
int32_t wbte_wbtx_partial_decrypt_many(wbte_ctx *ctx, void *sigma, const void *first, uint64_t batch_size,
                                       const void *q, uint64_t T, uint64_t K);
int32_t wbte_wbtx_verify_shares_many(wbte_ctx *ctx, int32_t *ok, const wbte_wbtx_key *key, const void *first,
                                     uint64_t batch_size, const void *sigma, const int64_t *party_indices,
                                     const void *challenges, uint64_t T, uint64_t K, const void *vk_tables);
/* Fixed-base tables of the verification keys of T parties at slots
 * 1..batch_size (the points the share check aggregates with the challenges,
 * weighted_btx/src/decryption.rs:358-422): T * batch_size tables of
 * 11 * 32 affine G2 points ([m 64^w] vk, 67,584 bytes each), party-major.
 * Given to verify_shares_many as vk_tables (NULL: Pippenger over the keys),
 * each aggregate takes one mixed addition per nonzero signed radix-64 digit
 * of the challenges' base-|x| digits and no doublings.  The tables must have
 * been built for the same party_indices, in the same order, and the same
 * batch_size as the verify_shares_many call: the call reads T * batch_size
 * tables and cannot check the buffer it is given. */
int32_t wbte_wbtx_vk_tables(wbte_ctx *ctx, void *tables, const wbte_wbtx_key *key, const int64_t *party_indices,
                            uint64_t T, uint64_t batch_size);
int32_t wbte_wbtx_precompute_many(wbte_ctx *ctx, void *beta, const void *kernel_lines, const void *first,
                                  const uint8_t *valid, uint64_t batch_size, uint64_t K);
int32_t wbte_wbtx_open_many(wbte_ctx *ctx, void *messages, const void *opening_keys, const void *opening_lines,
                            const void *sigma, uint64_t T, const void *second, const void *beta,
                            const uint8_t *valid, uint64_t batch_size, uint64_t K);
/* Precompute and open in one call for K batches of one committee (the
 * batched form of decrypt(), weighted_btx/src/decryption.rs:555-695):
 * messages K*B GT, at valid slots second * beta / alpha, one elsewhere.  The
 * cross terms and the opening pairings meet before the hard part of the
 * final exponentiation, which is a fixed power (a homomorphism of the
 * cyclotomic subgroup), so each slot takes one hard part instead of two;
 * the messages equal precompute_many followed by open_many.  Arguments as
 * there: kernel_lines m tables, opening_keys B*T G2 and opening_lines (or
 * NULL), first K*B G1, second K*B GT, valid K*B, sigma K*T G1. */
int32_t wbte_wbtx_decrypt_many(wbte_ctx *ctx, void *messages, const void *kernel_lines, const void *opening_keys,
                               const void *opening_lines, const void *first, const void *second,
                               const uint8_t *valid, const void *sigma, uint64_t T, uint64_t batch_size,
                               uint64_t K);
/* Public key material of keygen_with_rng (weighted_btx/src/setup.rs:98-233):
 *   verification_keys[i * N + j] = [q_pos[i * N + j]] G2            (i < L)
 *   negative[i * W + w]          = [z[w] q_neg[i * N + owner[w]]] G2 (i < L)
 *   positive[i * W + w]          = [z[w] q_pos[i * N + owner[w]]] G2 (i < L - 1)
 * owner host (W entries). */
int32_t wbte_wbtx_keygen_material(wbte_ctx *ctx, const void *z, const int32_t *owner, const void *q_pos,
                                  const void *q_neg, uint64_t W, uint64_t N, uint64_t L,
                                  void *verification_keys, void *negative, void *positive);

/* ------------------------------------------------------------- btx */
/* MiddleProductKernel::new (btx/src/decryption.rs:131-190) for one batch size
 * B <= L from the key powers low = [tau^1 .. tau^L] G2 and
 * high = [tau^(L+2) .. tau^(2L)] G2:
 *   kernel_lines   m * 68 * 288 bytes, m = next_pow2(2 B): lines of the
 *                  transformed centered kernel scaled by 1/m
 *   opening_lines  B * 68 * 288 bytes: lines of h_{-(slot+1)} = tau^(L-slot)
 *   kernel         m G2 (the scaled transformed kernel), may be NULL. */
int32_t wbte_btx_kernel(wbte_ctx *ctx, const void *low_powers, const void *high_powers, uint64_t L,
                        uint64_t batch_size, void *kernel_lines, void *opening_lines, void *kernel);
/* beta (precompute_batch, btx/src/decryption.rs:201-246): the middle product
 * of wbte_wbtx_precompute over the btx kernel lines. */
int32_t wbte_btx_precompute(wbte_ctx *ctx, void *beta, const void *kernel_lines, const void *first,
                            const uint8_t *valid, uint64_t batch_size);
/* sigma = sum_i shares[i] first[i] (partial_decrypt, btx/src/decryption.rs:248-264);
 * first carries the identity at invalid slots. */
int32_t wbte_btx_partial_decrypt(wbte_ctx *ctx, void *sigma, const void *first, const void *shares,
                                 uint64_t batch_size);
/* sigma = sum_j lambda_j sigmas[j] with the Lagrange coefficients at zero of
 * the shares' domain points, in the given order (combine_shares,
 * btx/src/decryption.rs:266-306). */
int32_t wbte_btx_combine(wbte_ctx *ctx, void *sigma, const void *sigmas, const void *points, uint64_t T);
/* *ok = 1 iff prod_{valid i} e(first_i, slot_points[i]) * e(-sigma, G2) == 1.
 * slot_points = low powers: verify_combined_share (btx/src/decryption.rs:372-400);
 * slot_points = one server's share commitments: verify_decryption_share (:340-370). */
int32_t wbte_btx_verify(wbte_ctx *ctx, int32_t *ok, const void *first, const uint8_t *valid,
                        uint64_t batch_size, const void *slot_points, uint64_t n_slot_points,
                        const void *sigma);
/* messages[i] = second[i] - e(sigma, h_{-(i+1)}) + beta[i] for valid slots
 * (open_batch, btx/src/decryption.rs:402-458); invalid slots get the identity. */
int32_t wbte_btx_open(wbte_ctx *ctx, void *messages, const void *opening_lines, const void *sigma,
                      const void *second, const void *beta, const uint8_t *valid, uint64_t batch_size);

/* The batched form of btx: K batches of one size B against one key
 * (batch-major arrays), each kernel launched once over all K batches; per
 * batch the results equal the single-batch calls':
 *   precompute_many  beta K*B GT over the m kernel line tables (as wbte_btx_precompute)
 *   open_many        messages K*B GT; opening_lines B tables; sigma K G1 (one
 *                    combined share per batch); second, beta K*B GT; valid K*B
 *   decrypt_many     precompute_many then open_many in one call, the cross
 *                    terms and the opening pairing meeting before one hard part
 *                    per slot (btx/src/decryption.rs:201-246, :402-458). */
int32_t wbte_btx_precompute_many(wbte_ctx *ctx, void *beta, const void *kernel_lines, const void *first,
                                 const uint8_t *valid, uint64_t batch_size, uint64_t K);
int32_t wbte_btx_open_many(wbte_ctx *ctx, void *messages, const void *opening_lines, const void *sigma,
                           const void *second, const void *beta, const uint8_t *valid, uint64_t batch_size,
                           uint64_t K);
int32_t wbte_btx_decrypt_many(wbte_ctx *ctx, void *messages, const void *kernel_lines, const void *opening_lines,
                              const void *first, const void *second, const uint8_t *valid, const void *sigma,
                              uint64_t batch_size, uint64_t K);

/* ---------------------------------------------------- weighted_pfe */
typedef struct {
    const void *domain_points;     /* total_weight Fr: the virtual points             */
    const void *verification_keys; /* batch_size * party_count G2, slot-major: i N + j */
    const void *d1;                /* batch_size * total_weight G2, slot-major         */
    const void *d2;                /* batch_size * total_weight G2, slot-major         */
    const void *global_key;        /* 1 G2: [z (beta_{-1} + beta_0)] G2                 */
    const int64_t *party_offsets;  /* host, party_count + 1 prefix offsets              */
    uint64_t party_count;
    uint64_t total_weight;
    uint64_t batch_size;           /* a power of two                                    */
} wbte_wpfe_key;

/* Party fractions g = 1 / (rho_j + alpha_i) and, when u is not NULL, the mask
 * values u = g^2 + beta_{-1} / (alpha_i + 1) + beta_0 / alpha_i with
 * masks = (beta_{-1}, beta_0) (weighted_pfe/src/setup.rs:223-247, :620-631);
 * stored slot-major (i N + j) or party-major (j B + i). */
int32_t wbte_wpfe_fractions(wbte_ctx *ctx, void *g, void *u, const void *rho, const void *alpha,
                            const void *masks, uint64_t N, uint64_t B, int32_t party_major);
/* Public key material (weighted_pfe/src/setup.rs:249-281) from slot-major g, u:
 *   vk[i N + j] = [g_{j,i}] G2, d1[i W + w] = [z[w] g_{owner(w),i}] G2,
 *   d2[i W + w] = [z[w] u_{owner(w),i}] G2.  owner host (W entries). */
int32_t wbte_wpfe_keygen_material(wbte_ctx *ctx, const void *z, const int32_t *owner, const void *g,
                                  const void *u, uint64_t W, uint64_t N, uint64_t B, void *vk, void *d1,
                                  void *d2);
/* sigma[j] = sum_i g_{j,i} first[i] for the T party secrets rho
 * (partial_decrypt, weighted_pfe/src/decryption.rs:231-252). */
int32_t wbte_wpfe_partial_decrypt(wbte_ctx *ctx, void *sigma, const void *first, const void *rho,
                                  const void *alpha, uint64_t T, uint64_t B);
/* *ok = 1 iff the random-linear aggregate share check passes
 * (verify_decryption_shares_batched, weighted_pfe/src/decryption.rs:367-419);
 * one share with challenge 1 is verify_decryption_share (:254-275). */
int32_t wbte_wpfe_verify_shares(wbte_ctx *ctx, int32_t *ok, const wbte_wpfe_key *key, const void *first,
                                const void *sigma, const int64_t *party_indices, const void *challenges,
                                uint64_t T);
/* Committee preparation (prepare_decryption, weighted_pfe/src/decryption.rs:421-538)
 * for the accepted parties (host, ascending); mask_scalars = alpha_i (alpha_i + 1)
 * for every slot, then -alpha_i for every slot (2 B Fr):
 *   by_party     B * T G2: sum_{w in party k} lambda_w / 2B d1[i W + w]
 *   total_lines  B line tables of sum_k by_party[i T + k]
 *   mask_lines   B line tables of alpha(alpha+1) sum_w lambda_w d2[i W + w] - alpha V
 *   total, mask  B G2 each, may be NULL. */
int32_t wbte_wpfe_prepare(wbte_ctx *ctx, const wbte_wpfe_key *key, const int64_t *party_indices, uint64_t T,
                          const void *mask_scalars, void *by_party, void *total_lines, void *mask_lines,
                          void *total, void *mask);
/* Cauchy sums (precompute_batch, weighted_pfe/src/decryption.rs:540-574, :683-734):
 *   first_cauchy[i]   = 2B sum_{k != i} first[k] / (alpha_k - alpha_i)
 *   pairing_cauchy[i] = the same sums over e(first[k], total_k) on easy-final-
 *                       exponentiated values (canonical after the hard part). */
int32_t wbte_wpfe_precompute(wbte_ctx *ctx, void *first_cauchy, void *pairing_cauchy, const void *first,
                             const void *total_lines, uint64_t B);
/* messages[i] = second[i] - hard(e(first_i, mask_i) / (prod_k e(2B sigma_k -
 * first_cauchy[i], by_party[i T + k]) pairing_cauchy[i])^(alpha_i (alpha_i + 1)))
 * (open_batch, weighted_pfe/src/decryption.rs:576-644); alpha_products B Fr. */
int32_t wbte_wpfe_open(wbte_ctx *ctx, void *messages, const void *sigmas, uint64_t T, const void *by_party,
                       const void *first, const void *mask_lines, const void *first_cauchy,
                       const void *pairing_cauchy, const void *second, const void *alpha_products,
                       uint64_t B);

/* The batched form: K batches of one (power-of-two) size B against one
 * accepted committee per call, batch-major arrays (batch b first).  Each call
 * is the K-fold version of the call above it with every kernel launched once
 * over all K batches; per batch the results equal the single-batch call's.
 *   partial_decrypt_many  sigma K*T G1 (sigma[b T + j] of party j in batch b),
 *                         first K*B G1, rho T Fr, alpha B Fr
 *   verify_shares_many    ok K int32 (one aggregate check per batch,
 *                         weighted_pfe/src/decryption.rs:367-419), first K*B,
 *                         sigma K*T, challenges K*T Fr, party_indices T (host),
 *                         vk_tables from wbte_wpfe_vk_tables or NULL
 *   precompute_many       first_cauchy K*B G1, pairing_cauchy K*B GT over the
 *                         committee's B total line tables
 *   open_many             messages K*B GT; sigmas K*T G1; by_party B*T G2
 *                         (shared) and by_party_lines, their line tables
 *                         (wbte_g2_prepare_lines of the B*T points) or NULL --
 *                         with them each slot's T pairings share one
 *                         multi-Miller loop (in chunks of 8 pairs); first, first_cauchy K*B
 *                         G1; pairing_cauchy, second K*B GT; alpha_products B Fr
 *   decrypt_many          precompute_many followed by open_many in one call
 *                         (weighted_pfe/src/decryption.rs:540-644, the
 *                         decrypt() of :646-669 after acceptance), without the
 *                         intermediate outputs. */
int32_t wbte_wpfe_partial_decrypt_many(wbte_ctx *ctx, void *sigma, const void *first, const void *rho,
                                       const void *alpha, uint64_t T, uint64_t B, uint64_t K);
/* Fixed-base tables of the verification keys of T parties at every slot
 * (T * B tables, party-major, 67,584 bytes each), as wbte_wbtx_vk_tables. */
int32_t wbte_wpfe_vk_tables(wbte_ctx *ctx, void *tables, const wbte_wpfe_key *key, const int64_t *party_indices,
                            uint64_t T);
int32_t wbte_wpfe_verify_shares_many(wbte_ctx *ctx, int32_t *ok, const wbte_wpfe_key *key, const void *first,
                                     const void *sigma, const int64_t *party_indices, const void *challenges,
                                     uint64_t T, uint64_t K, const void *vk_tables);
int32_t wbte_wpfe_precompute_many(wbte_ctx *ctx, void *first_cauchy, void *pairing_cauchy, const void *first,
                                  const void *total_lines, uint64_t B, uint64_t K);
int32_t wbte_wpfe_open_many(wbte_ctx *ctx, void *messages, const void *sigmas, uint64_t T, const void *by_party,
                            const void *by_party_lines, const void *first, const void *mask_lines,
                            const void *first_cauchy, const void *pairing_cauchy, const void *second,
                            const void *alpha_products, uint64_t B, uint64_t K);
int32_t wbte_wpfe_decrypt_many(wbte_ctx *ctx, void *messages, const void *sigmas, uint64_t T, const void *by_party,
                               const void *by_party_lines, const void *total_lines, const void *mask_lines,
                               const void *first, const void *second, const void *alpha_products, uint64_t B,
                               uint64_t K);

/* The batched form of pfe: K batches of one size B against one kernel
 * (batch-major arrays), per batch equal to the single-batch calls:
 *   precompute_many  weighted_first K*B G1, weighted_pairings K*B GT from
 *                    first K*B G1, the B key line tables and the 2 B scalars
 *                    of wbte_pfe_precompute (shared by the batches)
 *   open_many        messages K*B GT from first, second K*B G1, third K*B GT,
 *                    weighted_first/pairings K*B, pre_decryption_key K G1 (one
 *                    combined key per batch), neg_scaled_s1 B Fr and the B
 *                    line tables of each kind (pfe/src/decryption.rs:417-469). */
int32_t wbte_pfe_precompute_many(wbte_ctx *ctx, void *weighted_first, void *weighted_pairings, const void *first,
                                 const void *key_lines, const void *scalars, uint64_t B, uint64_t K);
int32_t wbte_pfe_open_many(wbte_ctx *ctx, void *messages, const void *first, const void *second, const void *third,
                           const void *weighted_first, const void *weighted_pairings, const void *pre_decryption_key,
                           const void *neg_scaled_s1, const void *key_lines, const void *generator_lines,
                           const void *mix_lines, uint64_t B, uint64_t K);

/* ---------------------------------------- resident keys and served form */
/* A request loop in the library for callers without their own scheduler:
 * validate ciphertexts and accept shares with the calls above (the crates'
 * host logic), then submit each accepted batch's decryption -- precompute
 * and open, the heavy part of decrypt() (weighted_btx/src/decryption.rs:555-709,
 * weighted_pfe/src/decryption.rs:540-669) -- and poll for its messages.
 *
 * wbte_crs_upload_* copies one setup's public key material (host or device
 * sources) into HBM owned by the handle; weighted_pfe also takes its 2 B
 * mask scalars alpha_i (alpha_i + 1), then -alpha_i (as wbte_wpfe_prepare).
 * A handle must outlive every server request that names it. */
#define WBTE_SCHEME_WBTX 1
#define WBTE_SCHEME_WPFE 2
typedef struct wbte_crs wbte_crs;
int32_t wbte_crs_upload_wbtx(wbte_ctx *ctx, const wbte_wbtx_key *key, wbte_crs **out);
int32_t wbte_crs_upload_wpfe(wbte_ctx *ctx, const wbte_wpfe_key *key, const void *mask_scalars, wbte_crs **out);
int32_t wbte_crs_destroy(wbte_crs *crs);

typedef struct {
    const wbte_crs *crs;          /* the setup (for weighted_pfe: the size class) */
    uint64_t batch_size;          /* weighted_btx: <= the setup's maximum; weighted_pfe: the class size */
    const void *first;            /* B G1 after validation (weighted_btx: identity at invalid slots) */
    const void *second;           /* B GT */
    const uint8_t *valid;         /* weighted_btx: B flags (NULL: all valid); weighted_pfe: ignored */
    const void *sigma;            /* T G1: the accepted shares in party order */
    const int64_t *party_indices; /* T accepted parties, ascending */
    uint64_t party_count;         /* T */
    void *messages;               /* out: B GT, host memory, written before the request completes */
} wbte_request;

typedef struct wbte_server wbte_server;
/* `slots` worker threads on `device`, each with its own context and CUDA
 * stream.  Waiting requests of one setup, batch size and committee are
 * decrypted together, up to max_group batches per launch sequence (the
 * _many calls); prepared committees stay cached in HBM for the server's
 * lifetime; a request is admitted while the estimated device memory of the
 * running groups stays within hbm_budget_bytes (0: half the free memory).
 * Requests run in arrival order otherwise. */
int32_t wbte_server_create(int32_t device, uint32_t slots, uint32_t max_group, uint64_t hbm_budget_bytes,
                           wbte_server **out);
/* Copies the request's inputs (the caller may reuse them on return) and
 * queues it; *ticket names it for wbte_poll.  WBTE_ERR_OOM if the request
 * alone exceeds the budget, WBTE_ERR_SIZE for a batch size its setup does
 * not take. */
int32_t wbte_submit(wbte_server *srv, const wbte_request *req, uint64_t *ticket);
/* Waits at most timeout_ns for the request.  WBTE_ERR_TIMEOUT if it is still
 * queued or running (the ticket stays valid); otherwise WBTE_OK, *status is
 * the request's own status (its messages are written when it is WBTE_OK)
 * and the ticket is released.  WBTE_ERR_INVALID_ARG for an unknown ticket. */
int32_t wbte_poll(wbte_server *srv, uint64_t ticket, uint64_t timeout_ns, int32_t *status);
/* Finishes every queued request, then stops the workers and frees the
 * cached committees. */
int32_t wbte_server_destroy(wbte_server *srv);

/* ------------------------------------------------------------- pfe */
/* PartialFractionKernel::new (pfe/src/decryption.rs:151-257) from the slot
 * fraction keys DK_i = [1/(x + w^i)] G2 (B, a power of two) and their sum.
 * scalars: 6 B Fr, in blocks of B: 1/(2B) | B-1-2k mod r | c (gamma = 1/c) |
 * s2_i = w^i c | -s2_i | -(2B s1_i) o_i with s1_i = w^i (s2_i - 1) and o_i the
 * opening coefficient w^-i (B+1)/2 + 1/(w^i - gamma).  Outputs line tables of
 * DK_i/(2B), [s2_i] G2 and the fused third operand; the affine points
 * (scaled_keys, generators, mixes, B G2 each) may be NULL. */
int32_t wbte_pfe_kernel(wbte_ctx *ctx, const void *fraction_keys, const void *key_sum, uint64_t B,
                        const void *scalars, void *key_lines, void *generator_lines, void *mix_lines,
                        void *scaled_keys, void *generators, void *mixes);
/* precompute_batch (pfe/src/decryption.rs:259-298): the gamma-weighted cyclic
 * convolutions of first and of e(first_i, DK_i/(2B)); scalars: 2 B Fr
 * (B-1-2k mod r | c). */
int32_t wbte_pfe_precompute(wbte_ctx *ctx, void *weighted_first, void *weighted_pairings, const void *first,
                            const void *key_lines, const void *scalars, uint64_t B);
/* open_batch (pfe/src/decryption.rs:417-469): messages[i] = third[i] -
 * (e(second_i, [s2_i]) e(weighted_first_i - 2B s1_i (second_i - pdk), DK_i/(2B))
 *  e(first_i, mix_i) - weighted_pairings[i]); neg_scaled_s1 = -(2B s1_i), B Fr. */
int32_t wbte_pfe_open(wbte_ctx *ctx, void *messages, const void *first, const void *second, const void *third,
                      const void *weighted_first, const void *weighted_pairings, const void *pre_decryption_key,
                      const void *neg_scaled_s1, const void *key_lines, const void *generator_lines,
                      const void *mix_lines, uint64_t B);

#ifdef __cplusplus
}
#endif
#endif /* WBTE_H */
