// Host-side launchers for the sm_100a kernels (internal to libwbte).
// Every pointer here is a device pointer; every launch goes to `s`.
// Group elements use blst's memory layout (Montgomery Fp limbs):
//   G1 affine 96 B, G2 affine 192 B, Fp12 576 B, Fr scalars as canonical
//   32-byte little-endian integers, the point at infinity as zero bytes.
#pragma once
#include <cstddef>
#include <cstdint>
#include <atomic>
#include <cuda_runtime.h>

namespace wbte {

// kernels launched by this library since load
extern std::atomic<uint64_t> g_launches;
extern thread_local uint64_t t_launches;
inline void note_launch(uint64_t k = 1) {
    g_launches.fetch_add(k, std::memory_order_relaxed);
    t_launches += k;
}

// Optional per-kernel timing: while profiling is enabled, a ProfScope records
// CUDA events around the launches in its scope, tagged with a kernel name.
extern thread_local bool g_prof_suppress;  // set while no events may be created
void prof_begin(const char* tag, cudaStream_t s, void** token);
void prof_end(void* token, cudaStream_t s);
struct ProfScope {
    void* token = nullptr;
    cudaStream_t s;
    ProfScope(const char* tag, cudaStream_t st) : s(st) { prof_begin(tag, st, &token); }
    ~ProfScope() { prof_end(token, s); }
};

// Knobs of the launchers' cost models for the library call running on this
// thread (0 / -1: the cost model decides).  Each ABI call copies its
// context's knobs (wbte_ctx_set_tuning) here for its duration; the
// per-size-class autotuner measures candidate values through them.
struct Tuning {
    int gt_lanes = 0;      // lanes per GT exponentiation in the radix-4 transform stages: 1, 2 or 4
    int msm_window = 0;    // Pippenger window width c, 4..13
    int msm_segments = 0;  // sorted-term segments per (MSM, window), 1..1024
    int ntt_joint = -1;    // G1/G2 transform stages: 1 one thread per butterfly, 0 the lane split
    int miller_chunk = 0;  // pairs per thread of the chunked unprepared Miller loops, 1..8
};
extern thread_local Tuning g_tune;

constexpr size_t G1_AFF = 96, G2_AFF = 192, G1_XYZZ = 192, G2_XYZZ = 384, GT_SZ = 576, FR_SZ = 32;
constexpr size_t LINE_SZ = 288;  // three Fp2 coefficients
constexpr int LINES_PER_POINT = 68;

enum Group : int { GROUP_G1 = 1, GROUP_G2 = 2 };

// ---------------------------------------------------------------- scalars
// out[i] = base^(i + first_exponent), canonical in/out
void launch_fr_powers(uint8_t* out, const uint8_t* base, int64_t n, int64_t first_exponent, cudaStream_t s);
// out[i] = a[i] * b[bidx[i]] (bidx null: b[i]); canonical
void launch_fr_mul_gather(uint8_t* out, const uint8_t* a, const uint8_t* b, const int32_t* bidx, int64_t n, cudaStream_t s);
// out[i] = a[i] * c for a fixed canonical c
void launch_fr_scale(uint8_t* out, const uint8_t* a, const uint8_t* c, int64_t n, cudaStream_t s);
// out[i] = a[i] * (1 / 2^log_m)
void launch_fr_scale_size_inv(uint8_t* out, const uint8_t* a, int log_m, int64_t n, cudaStream_t s);
// out[r * W + w] = z[w] * qp[r * N + owner[w]] for r < rows
void launch_material_scalars(uint8_t* out, const uint8_t* z, const int32_t* owner, const uint8_t* qp, int64_t W,
                             int64_t N, int64_t rows, cudaStream_t s);
// out[i] = in[idx[i]] for fixed-size records
void launch_gather(uint8_t* out, const uint8_t* in, const int32_t* idx, int64_t n, int64_t record, cudaStream_t s);
// weighted_pfe party fractions g = 1/(rho_j + alpha_i) and mask values u
// (u may be null); slot-major (i * N + j) or party-major (j * B + i).
void launch_wpfe_fractions(uint8_t* g, uint8_t* u, const uint8_t* rho, const uint8_t* alpha, const uint8_t* masks,
                           int64_t N, int64_t B, bool party_major, cudaStream_t s);
// Lagrange coefficients at zero of the points x[0..n) (direct formula); status[0] = 1 on a repeated point
void launch_lagrange_at_zero(uint8_t* out, const uint8_t* x, int64_t n, int32_t* status, cudaStream_t s);
// tw[j] = w^j, j < count, w = generator (or its inverse) of the size-n domain; canonical
void launch_domain_twiddles(uint8_t* tw, int64_t n, int64_t count, bool inverse, cudaStream_t s);

// ---------------------------------------------------------------- points
// out[i] = scalars[i] * points[i * point_stride] (affine out); stride 0 = one base
void launch_mul_batch(Group g, uint8_t* out, const uint8_t* points, int64_t point_stride, const uint8_t* scalars, int64_t n, cudaStream_t s);
// out[i] = scalars[i] * generator, fixed-base table
void launch_mul_generator(Group g, uint8_t* out, const uint8_t* scalars, int64_t n, cudaStream_t s);
// out[i] = 2^k * in[i]  (affine in/out)
void launch_mul_pow2(Group g, uint8_t* out, const uint8_t* in, int64_t n, int k, cudaStream_t s);
// out[j] = sum over t in [offsets[j], offsets[j+1]) of in[t] (affine in/out)
void launch_segment_sum(Group g, uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k, cudaStream_t s);
void launch_negate(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s);
// XYZZ points (work) to affine (out), one inversion per chunk (Montgomery's trick)
void launch_xyzz_to_affine(Group g, uint8_t* out, const uint8_t* work, int64_t n, cudaStream_t s);
// out[i] = [c_i] in[i] for small signed integers c_i (affine in and out)
void launch_mul_small(Group g, uint8_t* out, const uint8_t* in, const int32_t* coeffs, int64_t n, cudaStream_t s);
// blst projective (Jacobian X, Y, Z) points to affine, one inversion per chunk
void launch_batch_normalize(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s);
// radix-2 DIT transform of n affine points in place (forward or unscaled inverse)
void launch_group_ntt(Group g, uint8_t* io_affine, uint8_t* work_xyzz, const uint8_t* twiddles, int64_t n, cudaStream_t s,
                      int64_t count = 1);
// compressed (ZCash) encodings
void launch_compress(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s);
// fixed-base tables of np G2 points (points[point_index[p]]): FIXED_TABLE_BYTES each
constexpr size_t FIXED_TABLE_BYTES = G2_AFF * 11 * 32;
void launch_fixed_tables_g2(uint8_t* tables, const uint8_t* points, const int64_t* point_index, int64_t np,
                            cudaStream_t s);
// out[o] = sum_t scalars[vsel[o] n + t] * (point of table tbase[o] + tidx[t]), k outputs
void launch_fixed_msm_g2(uint8_t* out, const uint8_t* tables, const int64_t* tbase, const int32_t* tidx,
                         const uint8_t* scalars, const int32_t* vsel, int64_t k, int64_t n, cudaStream_t s);
// ZCash-format decoding with canonical-x, curve and (check_group) subgroup
// checks; status[i] = 0 ok, 1 bad encoding, 2 not on the curve, 3 not in the
// prime-order subgroup (the point is written as the identity then)
void launch_decompress(Group g, uint8_t* out, uint8_t* status, const uint8_t* in, int64_t n, bool check_group,
                       cudaStream_t s);
// valid[i] = ([s_i] G == R_i + [c_i] X_i), G the G1 generator
void launch_schnorr_verify(uint8_t* valid, const uint8_t* X, const uint8_t* R, const uint8_t* s_resp, const uint8_t* c, int64_t n, cudaStream_t st);

// ------------------------------------------------------------------- MSM
// Family of k multi-scalar multiplications, all of length n:
//   out[j] = sum_t scalars[vsel[j]][t] * points[pbase[j] + (idx ? idx[t] : t)]
// vsel null: vector 0 for every j.  scalars holds V vectors of n canonical
// 32-byte scalars.  Scratch is allocated from the stream-ordered pool.
struct MsmPlan {
    int c = 0, windows = 0, buckets = 0;
    int64_t segment = 0, segments = 0;
};
MsmPlan msm_plan(Group g, int64_t n, int64_t k);
// MSMs of at most SMALL_MSM_MAX terms by a Straus loop over the base-|x|
// digits of every term, the digit pairs spread over 1..16 lanes per output
// (launch_msm_family dispatches here).
constexpr int64_t SMALL_MSM_MAX = 4;
void launch_small_msm(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                      const uint8_t* scalars, const int32_t* vsel, int64_t k, int64_t n, cudaStream_t s);
void launch_msm_family(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                       const uint8_t* scalars, const int32_t* vsel, int32_t V, int64_t k, int64_t n,
                       cudaStream_t s, const MsmPlan* forced = nullptr);
// Scratch-size query and launch with caller-supplied scratch (no allocation).
size_t msm_family_scratch_bytes(Group g, int32_t V, int64_t k, int64_t n, const MsmPlan& plan);
void launch_msm_family_scratch(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                               const uint8_t* scalars, const int32_t* vsel, int32_t V, int64_t k, int64_t n,
                               const MsmPlan& plan, void* scratch, cudaStream_t s);

// --------------------------------------------------------------- pairing
// lines[step * n + i] for step < 68: prepared line coefficients of q[i]
void launch_prepare_lines(uint8_t* lines, const uint8_t* q, int64_t n, cudaStream_t s);
// out[i] = Miller(p[i], lines of pair i), lines laid out as above with n pairs
// out[o] = prod_{t<T} Miller(p[(o / p_per) T + t], line table (o % per) T + t) for o < n
// (tables line-major, stride per * T; p_per <= 0 means per); any T >= 1, the
// pairs sharing their squarings in chunks of 8; returns false for T < 1.
bool launch_miller_lines_multi(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, int64_t per, int T,
                               cudaStream_t s, int64_t p_per = 0);
void launch_miller_lines(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, cudaStream_t s,
                         int64_t lines_n = 0);
// out[i] = Miller(p[p_mod ? i % p_mod : i], q[i])
// pair i: P[p_mod ? i % p_mod : i], Q[q_mod ? i % q_mod : i]
// K segments of `per` consecutive (P, Q) pairs: out[s * chunks + ch] is the
// product of the Miller loops of run ch (at most C pairs) of segment s;
// returns chunks = ceil(per / C).  miller_chunk picks C for `pairs` in all.
int miller_chunk(int64_t pairs);
int64_t launch_miller_chunks(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t per, int64_t K, int C,
                             cudaStream_t s);
void launch_miller(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t n, cudaStream_t s, int64_t p_mod = 0,
                   int64_t q_mod = 0);
// io[i] = 1 where valid[i] == 0
void launch_fp12_mask(uint8_t* io, const uint8_t* valid, int64_t n, cudaStream_t s);
// out[j] = product of in[offsets[j] .. offsets[j+1])
void launch_fp12_segment_product(uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k, cudaStream_t s);
enum FinalExpMode : int { FE_FULL = 0, FE_EASY = 1, FE_HARD = 2 };
void launch_final_exp(uint8_t* out, const uint8_t* in, int64_t n, FinalExpMode mode, cudaStream_t s);
// unscaled inverse transform over cyclotomic values keeping out_count outputs
void launch_cyclotomic_prefix_ifft(uint8_t* io, const uint8_t* twiddles_inv, int64_t n, int64_t out_count, cudaStream_t s,
                                   int64_t count = 1);
// full unscaled transform over GT values (forward if twiddles are powers of w, inverse with w^-1)
// twiddles from the inverse domain when inverse is set (selects the omega_4 action)
void launch_gt_ntt(uint8_t* io, const uint8_t* twiddles, int64_t n, cudaStream_t s, int64_t count = 1, bool inverse = false);
// out[i] = base[i * stride]^scalars[i] on GT
void launch_gt_pow(uint8_t* out, const uint8_t* base, int64_t base_stride, const uint8_t* scalars, int64_t n, cudaStream_t s);
// out[q B + i] = base[q B + i]^scalars[i] for K arrays sharing B exponents, with
// warp-uniform plans; returns false (launching nothing) when K is not 24..31
// or a multiple of 32
bool launch_gt_pow_shared(uint8_t* out, const uint8_t* base, const uint8_t* scalars, int64_t B, int64_t K,
                          cudaStream_t s);
// out[i] = base[i * stride]^coeffs[i] on cyclotomic values, small signed exponents
void launch_gt_pow_small(uint8_t* out, const uint8_t* base, int64_t stride, const int32_t* coeffs, int64_t n,
                         cudaStream_t s);
// out[i] = a[i * sa] * b[i * sb] (conj_b: b conjugated)
void launch_fp12_mul(uint8_t* out, const uint8_t* a, int64_t sa, const uint8_t* b, int64_t sb, bool conj_b, int64_t n, cudaStream_t s);
// out[i] = conjugate of in[i] (the inverse in the cyclotomic subgroup)
void launch_fp12_conj(uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s);
// messages[i] = valid[i] ? second[i] * conj(alpha[i]) * beta[i] : one
void launch_unmask(uint8_t* out, const uint8_t* second, const uint8_t* alpha, const uint8_t* beta, const uint8_t* valid, int64_t n, cudaStream_t s);
// torus-compressed GT encodings (tag byte + 288 bytes)
void launch_gt_compress(uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s);
// flags[i] = (in[i] == 1)
void launch_fp12_is_one(uint8_t* flags, const uint8_t* in, int64_t n, cudaStream_t s);
// ------------------------------------------------------------ transcripts
// One field of a Fiat-Shamir transcript: record i contributes the len bytes
// at data + i * stride (stride 0: the same bytes for every record).  A
// TRANSCRIPT_GT_VARIABLE field is a 289-byte compressed GT record that
// contributes only its tag byte when the tag is 0 (the identity).
enum TranscriptKind : uint32_t { TRANSCRIPT_BYTES = 0, TRANSCRIPT_GT_VARIABLE = 1 };
constexpr int TRANSCRIPT_MAX_FIELDS = 8;
constexpr uint32_t TRANSCRIPT_MAX_TRIES = 256;
struct TranscriptField {
    const uint8_t* data;
    uint64_t stride;
    uint32_t len;
    uint32_t kind;
};
struct TranscriptSpec {
    TranscriptField f[TRANSCRIPT_MAX_FIELDS];
    int32_t count;
};
// out[i] (32-byte canonical scalar) = SHA-256 rejection-sampled challenge of
// record i's fields followed by a u32 LE counter; *status = 1 if a record
// ran out of counters
void launch_transcript_challenges(uint8_t* out, const TranscriptSpec& spec, int64_t n, int32_t* status,
                                  cudaStream_t s);
// sustained 32-bit IMAD instructions per second (calibration kernel, synchronising)
double measure_imad_rate(cudaStream_t s);

}  // namespace wbte
