// The opening's multi-Miller loops over prepared line tables: one loop per
// slot shares the Fp12 squarings across the slot's T pairings (in chunks of
// up to 8 pairs for larger committees).  Built with
// the library's default layout (out-of-line Fp2 products, inline Fp sums),
// which runs this kernel faster than the inline-Fp2 layout of k_pairing.cu.
#include "launch.h"
#include "pairing.cuh"

namespace wbte {

namespace {
constexpr int TPB = 64;
inline unsigned blocks_for(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

WBTE_INL Fp12* as_gt(uint8_t* p) { return reinterpret_cast<Fp12*>(p); }

// out[o] = prod_{t < T} Miller(P[(o / p_per) * T + t], lines of table (o % per) * T + t):
// the opening of K batches against one committee's prepared opening keys
// (tables line-major with stride per * T), each batch with its own T shares
// (p_per = per: weighted_btx) or each slot with its own T points (p_per = 1:
// weighted_pfe).
__global__ void k_miller_lines_multi(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, int64_t per,
                                     int64_t p_per, int T) {
    int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= n) return;
    const int64_t b = o / p_per, i = o % per;
    const Line* L = reinterpret_cast<const Line*>(lines) + i * T;
    const G1A* P = reinterpret_cast<const G1A*>(p) + b * T;
    // chunks of at most MULTI_MILLER_MAX pairs, each sharing its squarings;
    // the product of the chunks' loops is the multi-Miller value exactly
    Fp12 f;
    multi_miller_loop_lines(f, L, (size_t)(per * T), 1, P, T < MULTI_MILLER_MAX ? T : MULTI_MILLER_MAX);
    for (int t0 = MULTI_MILLER_MAX; t0 < T; t0 += MULTI_MILLER_MAX) {
        Fp12 g;
        const int c = T - t0 < MULTI_MILLER_MAX ? T - t0 : MULTI_MILLER_MAX;
        multi_miller_loop_lines(g, L + t0, (size_t)(per * T), 1, P + t0, c);
        fp12_mul(f, f, g);
    }
    store_vec(as_gt(out) + o, f);
}

}  // namespace

bool launch_miller_lines_multi(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, int64_t per, int T,
                               cudaStream_t s, int64_t p_per) {
    ProfScope prof_("miller_lines_multi", s);
    if (T < 1 || per < 1) return false;
    if (n <= 0) return true;
    note_launch();
    k_miller_lines_multi<<<blocks_for(n), TPB, 0, s>>>(out, lines, p, n, per, p_per > 0 ? p_per : per, T);
    return true;
}

}  // namespace wbte
