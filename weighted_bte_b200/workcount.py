"""Fp-product counts of the library's kernels: the numerators of the
integer-pipe roofline.

The unit is one 12-limb Montgomery product in Fp (588 multiply-add
instructions in the CIOS sequence of csrc/field_asm.cuh); Fp additions are
not counted.  Counts follow the kernels' own formulas (Karatsuba Fp2 / Fp6 /
Fp12 tower, XYZZ curve formulas, the hard-part chain, warp-uniform NAF plans),
so `achieved / peak` measures how well the kernel runs the work it does, not
how much work it avoids.  Counts are exact where the schedule is static
(Miller loops, final exponentiation, GT transforms whose plans depend only on
public twiddles); the MSM counts are the expected values of the Pippenger
plan (nonzero digits of uniform scalars), stated as such.
"""
from __future__ import annotations

R_FR = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
P_FP = int("1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab", 16)
X_ABS = 0xD201000000010000

FP2_MUL, FP2_SQR = 3, 2
FP6_MUL = 6 * FP2_MUL
FP12_MUL = 3 * FP6_MUL  # 54
FP12_SQR = 2 * FP6_MUL  # 36
CYC_SQR = 3 * 3 * FP2_SQR  # 18: three Fp4 squarings of three Fp2 squarings
FROB = 5 * FP2_MUL  # 15
LINE_MUL = 13 * FP2_MUL + 4  # 43: sparse Fp12 product plus the two Fp2 x Fp scalings
LINE_DOUBLE = 5 * FP2_SQR + 4 * FP2_MUL  # 22
LINE_ADD = 11 * FP2_MUL + 2 * FP2_SQR  # 37
MILLER_SQUARINGS, MILLER_LINES = 62, 68
MILLER_WITH_LINES = MILLER_SQUARINGS * FP12_SQR + MILLER_LINES * LINE_MUL  # 5156
MILLER_UNPREPARED = MILLER_WITH_LINES + 63 * LINE_DOUBLE + 5 * LINE_ADD  # 6727


MILLER_SQUARING_RUN = MILLER_SQUARINGS * FP12_SQR  # 2232


def multi_miller_unprepared(pairs: int, run: int) -> int:
    """Share-check Miller loops of `pairs` pairs in runs of `run` pairs per
    thread, each run one multi-Miller loop sharing the 62 squarings."""
    runs = -(-pairs // run)
    return runs * MILLER_SQUARING_RUN + pairs * (MILLER_UNPREPARED - MILLER_SQUARING_RUN)


def multi_miller_with_lines(T: int) -> int:
    """One slot's multi-Miller loop over T prepared line tables."""
    return MILLER_SQUARINGS * FP12_SQR + T * MILLER_LINES * LINE_MUL


def _fp_inv() -> int:
    e = P_FP - 2
    nib = [(e >> (4 * w)) & 15 for w in range(96)]
    top = max(w for w in range(96) if nib[w])
    return 14 + 4 * top + sum(1 for w in range(top) if nib[w])


FP_INV = _fp_inv()
FP2_INV = 2 + FP_INV + 2
FP6_INV = 3 * (FP2_SQR + FP2_MUL) + 3 * FP2_MUL + FP2_INV + 3 * FP2_MUL
FP12_INV = 2 * FP6_MUL + FP6_INV + 2 * FP6_MUL
FINAL_EXP_EASY = FP12_INV + FP12_MUL + FROB + FP12_MUL
RAISE_Z_HALF = (1 + 2 + 3 + 9 + 32 + 15) * CYC_SQR + 5 * FP12_MUL  # 1386
RAISE_Z = RAISE_Z_HALF + CYC_SQR
FINAL_EXP_HARD = (CYC_SQR + RAISE_Z + RAISE_Z_HALF + 2 * FP12_MUL + 2 * RAISE_Z + FP12_MUL + 2 * FROB + FP12_MUL
                  + RAISE_Z + 3 * FP12_MUL + FROB + FP12_MUL)  # 7497
FINAL_EXP = FINAL_EXP_EASY + FINAL_EXP_HARD

# XYZZ formulas (curves.cuh): products per operation in G1 (Fp) and G2 (Fp2)
G1_MADD, G1_ADD, G1_DBL = 10, 14, 9
G2_MADD = 8 * FP2_MUL + 2 * FP2_SQR  # 28
G2_ADD = 12 * FP2_MUL + 2 * FP2_SQR  # 40
G2_DBL = 5 * FP2_MUL + 4 * FP2_SQR  # 23


def decompose_base_x(s: int):
    d = []
    for _ in range(4):
        d.append(s % X_ABS)
        s //= X_ABS
    return d


def _naf_len_nonzero(v: int, w: int):
    length, nonzero = 0, 0
    half, full = 1 << (w - 1), 1 << w
    while v:
        if v & 1:
            d = v & (full - 1)
            if d >= half:
                d -= full
            v -= d
            nonzero += 1
        v >>= 1
        length += 1
    return length, nonzero


def gt_plan_power(s: int) -> int:
    """k_gt_radix4_pows_plan: the four base-|x| digits of s in width-4 NAF
    over one shared run of squarings, with a table of odd powers (1 squaring,
    3 products, 12 Frobenius maps)."""
    longest, nonzero = 0, 0
    for v in decompose_base_x(s):
        ln, nz = _naf_len_nonzero(v, 4)
        longest, nonzero = max(longest, ln), nonzero + nz
    return CYC_SQR + 3 * FP12_MUL + 12 * FROB + CYC_SQR * max(0, longest - 1) + FP12_MUL * max(0, nonzero - 1)


def domain_inverse_generator(m: int) -> int:
    w = pow(pow(7, (R_FR - 1) >> 32, R_FR), 1 << (32 - (m.bit_length() - 1)), R_FR)
    return pow(w, R_FR - 2, R_FR)


def gt_prefix_ifft(m: int, out_count: int, count: int) -> int:
    """The batched truncated GT inverse transform as the library runs it for
    count >= 32 transforms of an even number of radix-4 stages: per stage
    the warp-uniform-plan twiddle powers and the butterfly outputs (four
    outputs of 3 products, two of them with a Frobenius map; two outputs in
    the last, truncated stage)."""
    assert out_count == m // 2 and (m.bit_length() - 1) % 2 == 0
    w_inv = domain_inverse_generator(m)
    total, h = 0, 1
    while h < m:
        blocks = m // (4 * h)
        for j in range(h):
            for e in range(3):
                idx = (2 * j, j, 3 * j)[e] * blocks
                if idx >= m // 2:
                    idx -= m // 2
                if idx:
                    total += blocks * gt_plan_power(pow(w_inv, idx, R_FR))
        last = 4 * h == m
        total += (m // 4) * ((2 * 3 * FP12_MUL + FROB) if last else (4 * 3 * FP12_MUL + 2 * FROB))
        h *= 4
    return total * count


def _g1_joint_naf(s: int) -> int:
    """g1_mul_joint_naf: tables of 8 odd multiples of v and phi(v) + v, the two
    GLV digit groups in width-5 NAF over one run of doublings."""
    d = decompose_base_x(s)
    w0, w1 = d[0] + d[1] * X_ABS, d[2] + d[3] * X_ABS
    l0, n0 = _naf_len_nonzero(w0, 5)
    l1, n1 = _naf_len_nonzero(w1, 5)
    tables = 1 + G1_ADD + 2 * (G1_DBL + 7 * G1_ADD)  # phi, phi(v) + v, two tables
    return tables + G1_DBL * max(0, max(l0, l1) - 1) + G1_ADD * max(0, n0 + n1 - 1)


def g1_ntt_batched(m: int, count: int, inverse: bool = False) -> int:
    """The batched G1 transform (k_ntt_stage_joint with warp-uniform NAF
    twiddles, count a multiple of 32): per butterfly the twiddle
    multiplication (none for twiddle 1) and two XYZZ additions."""
    w = pow(pow(7, (R_FR - 1) >> 32, R_FR), 1 << (32 - (m.bit_length() - 1)), R_FR)
    if inverse:
        w = pow(w, R_FR - 2, R_FR)
    total, half = 0, 1
    while half < m:
        stride = m // (2 * half)
        for j in range(half):
            tw = _g1_joint_naf(pow(w, j * stride, R_FR)) if j else 0
            total += (m // (2 * half)) * (tw + 2 * G1_ADD)
        half *= 2
    return total * count


def msm_plan_window(n: int) -> int:
    lg = max(0, n.bit_length() - 1)
    c = lg - 1 if n < (1 << 14) else lg - 2
    return max(4, min(13, c))


def msm_expected(n: int, k: int, g2: bool, c: int = 0) -> int:
    """Expected products of k Pippenger MSMs of n uniform scalars with window
    c (default: the cost model's): one mixed addition per nonzero signed
    digit, one addition per occupied bucket, the window combination."""
    c = c or msm_plan_window(n)
    windows = -(-256 // c)
    buckets = 1 << (c - 1)
    nnz = n * (1.0 - 1.0 / (1 << c))
    occupied = buckets * (1.0 - (1.0 - 1.0 / buckets) ** nnz)
    madd, add, dbl = (G2_MADD, G2_ADD, G2_DBL) if g2 else (G1_MADD, G1_ADD, G1_DBL)
    per = windows * (nnz * madd + occupied * add) + windows * (c * dbl + add)
    return int(per * k)



# ----------------------------------------- single transforms, exact schedules
G2_PSI = 2 * FP2_MUL  # psi: two Fp2 products by constants


def r16_digits(v: int, top: int):
    """Signed radix-16 digits (in [-7, 8]) of v < 16^top, least significant
    first, top + 1 of them: the recoding of pairing.cuh r16_digit."""
    out, carry = [], 0
    for k in range(top + 1):
        nib = (v >> (4 * k)) & 15 if k < top else 0
        d = nib + carry
        carry = 1 if d > 8 else 0
        out.append(d - 16 if d > 8 else d)
    return out


def _xyzz_mul_r16(w: int, top: int, g2: bool) -> int:
    """xyzz_mul_r16: a table [1..8]P (one doubling, six additions), then
    top + 1 windows of four doublings and one addition per nonzero digit,
    free while the accumulator is the point at infinity."""
    dbl, add = (G2_DBL, G2_ADD) if g2 else (G1_DBL, G1_ADD)
    total = dbl + 6 * add
    started = False
    for d in reversed(r16_digits(w, top)):
        if started:
            total += 4 * dbl
        if d:
            total += add if started else 0
            started = True
    return total


def _glv_words(s: int):
    d = decompose_base_x(s)
    return [d[0] + d[1] * X_ABS, d[2] + d[3] * X_ABS]


def _twiddles(n: int, inverse: bool):
    w = pow(pow(7, (R_FR - 1) >> 32, R_FR), 1 << (32 - (n.bit_length() - 1)), R_FR)
    return pow(w, R_FR - 2, R_FR) if inverse else w


def group_ntt_lanes(n: int, g2: bool, inverse: bool = False) -> int:
    """k_ntt_stage (one transform, the lane split): per butterfly with
    twiddle t != 1 each lane runs xyzz_mul_r16 on its base-|x| digit group
    (G1: [a]v and [b](phi(v) + v), 128-bit; G2: [d_c] psi^c(v), 64-bit),
    the lanes' parts are added in a tree, and two additions give the outputs."""
    w = _twiddles(n, inverse)
    add = G2_ADD if g2 else G1_ADD
    L = 4 if g2 else 2
    total, half = 0, 1
    memo = {}
    while half < n:
        stride = n // (2 * half)
        for j in range(half):
            per = 2 * add
            if j and j * stride in memo:
                per += memo[j * stride]
            elif j:
                s = pow(w, j * stride, R_FR)
                base = per
                if g2:
                    for c, d in enumerate(decompose_base_x(s)):
                        per += c * G2_PSI + _xyzz_mul_r16(d, 16, True)
                else:
                    a, b = _glv_words(s)
                    per += _xyzz_mul_r16(a, 32, False) + 1 + G1_ADD + _xyzz_mul_r16(b, 32, False)
                per += (L - 1) * add
                memo[j * stride] = per - base
            total += (n // (2 * half)) * per
        half *= 2
    return total


def group_ntt_joint(n: int, g2: bool, inverse: bool = False) -> int:
    """k_ntt_stage_joint for one transform (mul_joint: every digit group of
    the twiddle on one thread over one run of doublings, signed radix-16
    Straus), plus two additions per butterfly."""
    w = _twiddles(n, inverse)
    dbl, add = (G2_DBL, G2_ADD) if g2 else (G1_DBL, G1_ADD)
    tables = (dbl + 6 * add) if g2 else 2 * (G1_DBL + 6 * G1_ADD) + 1 + G1_ADD
    total, half = 0, 1
    memo = {}
    while half < n:
        stride = n // (2 * half)
        for j in range(half):
            per = 2 * add
            if j and j * stride in memo:
                per += memo[j * stride]
            elif j:
                s = pow(w, j * stride, R_FR)
                base = per
                groups = [(d, 16) for d in decompose_base_x(s)] if g2 else [(v, 32) for v in _glv_words(s)]
                top = groups[0][1]
                digs = [r16_digits(v, top) for v, _ in groups]
                per += tables
                started = False
                for k in range(top, -1, -1):
                    if started:
                        per += 4 * dbl
                    for c, dg in enumerate(digs):
                        if dg[k]:
                            if started:
                                per += add
                            started = True
                            if g2:
                                per += c * G2_PSI  # the digit-c entry is psi^c of the table entry
                memo[j * stride] = per - base
            total += (n // (2 * half)) * per
        half *= 2
    return total


def _gt_lane(d: int, c: int) -> int:
    """gt_pow_lane: table (Frobenius^c for c > 0, one squaring, six
    products), 64 cyclotomic squarings, one product per nonzero digit of the
    17 signed radix-16 digits (the accumulator starts at one)."""
    nz = sum(1 for x in r16_digits(d, 16) if x)
    return (FROB if c else 0) + CYC_SQR + 6 * FP12_MUL + 64 * CYC_SQR + nz * FP12_MUL


def _gt_one_lane(s: int) -> int:
    """gt_pow_digits with all four digits on one lane: one table, the shared
    squarings, per nonzero digit one product (and a Frobenius map for c > 0)."""
    total = CYC_SQR + 6 * FP12_MUL + 64 * CYC_SQR
    for c, d in enumerate(decompose_base_x(s)):
        nz = sum(1 for x in r16_digits(d, 16) if x)
        total += nz * (FP12_MUL + (FROB if c else 0))
    return total


def gt_ntt_single(n: int, lanes: int, inverse: bool = False) -> int:
    """One GT transform (gt_transform with count 1): a radix-2 first stage
    for an odd number of stages (k_gt_stage, four lanes per power, three
    combine products, two outputs), then radix-4 stages with three powers
    per butterfly on `lanes` = 4 (k_gt_radix4: four lanes and three combine
    products per power) or 1 (k_gt_radix4_pows<1>), and four outputs of
    three products, two of them with a Frobenius map (omega_4)."""
    assert lanes in (1, 4) and n >= 4
    w = _twiddles(n, inverse)
    bits = n.bit_length() - 1
    total, half = 0, 1
    memo = {}

    def power(idx):
        if idx not in memo:
            memo[idx] = _power(pow(w, idx, R_FR))
        return memo[idx]

    def _power(s):
        if lanes == 4:
            return sum(_gt_lane(d, c) for c, d in enumerate(decompose_base_x(s))) + 3 * FP12_MUL
        return _gt_one_lane(s)

    if bits & 1:
        total += (n // 2) * 5 * FP12_MUL  # half = 1: twiddle 1, the combine and the two outputs
        half = 2
    while half < n:
        blocks = n // (4 * half)
        for j in range(half):
            for e in range(3):
                idx = (2 * j, j, 3 * j)[e] * blocks
                if idx >= n // 2:
                    idx -= n // 2
                if idx:
                    total += blocks * power(idx)
                elif lanes == 4:
                    total += blocks * 3 * FP12_MUL  # the combine still runs
        total += (n // 4) * (4 * 3 * FP12_MUL + 2 * FROB)
        half *= 4
    return total
