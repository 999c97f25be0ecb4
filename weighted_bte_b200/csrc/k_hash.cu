// Fiat-Shamir transcripts on the device: SHA-256 (FIPS 180-4) of
// prefix || per-record fields || counter (u32 LE), with the rejection
// sampling every crate uses to turn a digest into a canonical Fr scalar
// (btx/src/proof.rs:49-77, pfe/src/proof.rs:148-176,
// weighted_btx/src/proof.rs:72-100, weighted_pfe/src/proof.rs:124-152).
#include "launch.h"
#include "fields.cuh"

namespace wbte {

namespace {
constexpr int TPB = 128;
inline unsigned blocks_for(int64_t n) { return (unsigned)((n + TPB - 1) / TPB); }

// FIPS 180-4 section 4.2.2: first 32 bits of the fractional parts of the
// cube roots of the first 64 primes.
__device__ __constant__ const uint32_t C_SHA_K[64] = {
    0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
    0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
    0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
    0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
    0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
    0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
    0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
    0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};

WBTE_INL uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

// One compression of the 16-word (big-endian) block w into h.
__device__ __noinline__ void sha256_compress(uint32_t h[8], const uint32_t w_in[16]) {
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; i++) w[i] = w_in[i];
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
#pragma unroll
    for (int t = 0; t < 64; t++) {
        uint32_t wt;
        if (t < 16) {
            wt = w[t];
        } else {
            const uint32_t w15 = w[(t - 15) & 15], w2 = w[(t - 2) & 15];
            const uint32_t s0 = rotr(w15, 7) ^ rotr(w15, 18) ^ (w15 >> 3);
            const uint32_t s1 = rotr(w2, 17) ^ rotr(w2, 19) ^ (w2 >> 10);
            wt = w[t & 15] = w[t & 15] + s0 + w[(t - 7) & 15] + s1;
        }
        const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
        const uint32_t ch = (e & f) ^ (~e & g);
        const uint32_t t1 = hh + S1 + ch + C_SHA_K[t] + wt;
        const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        const uint32_t t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

// Streaming SHA-256 state of one thread: the block under construction is
// kept as 16 big-endian words.
struct Sha256 {
    uint32_t h[8];
    uint32_t w[16];
    uint32_t fill;    // bytes in the current block
    uint64_t total;   // bytes absorbed

    WBTE_INL void init() {
        // FIPS 180-4 section 5.3.3: fractional parts of the square roots of
        // the first 8 primes
        h[0] = 0x6a09e667u; h[1] = 0xbb67ae85u; h[2] = 0x3c6ef372u; h[3] = 0xa54ff53au;
        h[4] = 0x510e527fu; h[5] = 0x9b05688cu; h[6] = 0x1f83d9abu; h[7] = 0x5be0cd19u;
#pragma unroll
        for (int i = 0; i < 16; i++) w[i] = 0;
        fill = 0;
        total = 0;
    }
    WBTE_INL void byte(uint32_t v) {
        w[fill >> 2] |= (v & 0xffu) << (24 - 8 * (fill & 3));
        total++;
        if (++fill == 64) {
            sha256_compress(h, w);
#pragma unroll
            for (int i = 0; i < 16; i++) w[i] = 0;
            fill = 0;
        }
    }
    WBTE_INL void bytes(const uint8_t* p, uint32_t n) {
        uint32_t i = 0;
        // whole words while both the block and the source are word-aligned
        if ((fill & 3) == 0 && (reinterpret_cast<uintptr_t>(p) & 3) == 0) {
            for (; i + 4 <= n; i += 4) {
                const uint32_t v = *reinterpret_cast<const uint32_t*>(p + i);
                w[fill >> 2] = __byte_perm(v, 0, 0x0123);
                total += 4;
                fill += 4;
                if (fill == 64) {
                    sha256_compress(h, w);
#pragma unroll
                    for (int k = 0; k < 16; k++) w[k] = 0;
                    fill = 0;
                }
            }
        }
        for (; i < n; i++) byte(p[i]);
    }
    // Padding and length (FIPS 180-4 section 5.1.1); digest bytes are the
    // big-endian words h[0..7].
    WBTE_INL void finish() {
        const uint64_t bits = total * 8;
        byte(0x80);
        while (fill != 56) byte(0);
        for (int i = 7; i >= 0; i--) byte((uint32_t)(bits >> (8 * i)));
    }
};
}  // namespace

// out[i] = the first canonical scalar SHA-256(fields of record i || counter)
// for counter = 0, 1, ... (little-endian digest, accepted when below r).
// A record that exhausts TRANSCRIPT_MAX_TRIES counters (probability about
// 2^-220 each) gets a zero scalar and sets *status.
__global__ void k_transcript_challenges(uint8_t* out, TranscriptSpec spec, int64_t n, int32_t* status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t* o = out + 32 * i;
    for (uint32_t counter = 0; counter < TRANSCRIPT_MAX_TRIES; counter++) {
        Sha256 s;
        s.init();
        for (int k = 0; k < spec.count; k++) {
            const TranscriptField& f = spec.f[k];
            const uint8_t* p = f.data + f.stride * (uint64_t)i;
            uint32_t len = f.len;
            // a compressed GT record whose tag is 0 (the identity) is encoded as that one byte
            if (f.kind == TRANSCRIPT_GT_VARIABLE && p[0] == 0) len = 1;
            s.bytes(p, len);
        }
        s.byte(counter);
        s.byte(counter >> 8);
        s.byte(counter >> 16);
        s.byte(counter >> 24);
        s.finish();
        uint32_t limb[8];
#pragma unroll
        for (int k = 0; k < 8; k++) limb[k] = __byte_perm(s.h[k], 0, 0x0123);
        bool below = false;
#pragma unroll
        for (int k = 7; k >= 0; k--) {
            if (limb[k] != C_R[k]) {
                below = limb[k] < C_R[k];
                break;
            }
        }
        if (below) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                o[4 * k] = (uint8_t)limb[k];
                o[4 * k + 1] = (uint8_t)(limb[k] >> 8);
                o[4 * k + 2] = (uint8_t)(limb[k] >> 16);
                o[4 * k + 3] = (uint8_t)(limb[k] >> 24);
            }
            return;
        }
    }
    for (int k = 0; k < 32; k++) o[k] = 0;
    atomicExch(status, 1);
}

void launch_transcript_challenges(uint8_t* out, const TranscriptSpec& spec, int64_t n, int32_t* status,
                                  cudaStream_t s) {
    ProfScope prof_("transcript_challenges", s);
    if (n <= 0) return;
    note_launch();
    k_transcript_challenges<<<blocks_for(n), TPB, 0, s>>>(out, spec, n, status);
}

}  // namespace wbte
