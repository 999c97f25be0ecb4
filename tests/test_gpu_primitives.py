"""Parity of the libwbte primitives with the CPU oracle on seeded inputs.

Every comparison is bit-exact on blst's memory layout (Montgomery Fp limbs),
which is canonical for affine points and for Fp12 values.
"""
import random

import pytest

from weighted_bte_b200 import ops

pytestmark = pytest.mark.gpu


def rs(rng, n, R):
    return [rng.randrange(R) for _ in range(n)]


@pytest.fixture(scope="module")
def pts(orc):
    rng = random.Random(11)
    g1 = orc.g1_mul_many(orc.g1_generator(), rs(rng, 64, orc.R))
    g2 = orc.g2_mul_many(orc.g2_generator(), rs(rng, 64, orc.R))
    return g1, g2


def test_fixed_base_mul_matches_oracle(orc):
    rng = random.Random(1)
    sc = rs(rng, 37, orc.R) + [0, 1, orc.R - 1]
    assert ops.split(ops.g1_mul_generator(sc), 96) == orc.g1_mul_many(orc.g1_generator(), sc)
    assert ops.split(ops.g2_mul_generator(sc), 192) == orc.g2_mul_many(orc.g2_generator(), sc)


def test_variable_base_mul_matches_oracle(orc, pts):
    rng = random.Random(2)
    g1, g2 = pts
    sc = rs(rng, len(g1), orc.R)
    assert ops.split(ops.g1_mul(b"".join(g1), sc), 96) == orc.g1_mul_many(g1, sc)
    assert ops.split(ops.g2_mul(b"".join(g2), sc), 192) == orc.g2_mul_many(g2, sc)


@pytest.mark.parametrize("n", [0, 1, 2, 7, 64, 513, 3000])
def test_g1_msm_matches_oracle(orc, n):
    rng = random.Random(100 + n)
    points = orc.g1_mul_many(orc.g1_generator(), rs(rng, n, orc.R)) if n else []
    sc = rs(rng, n, orc.R)
    if n > 3:
        points[1] = orc.G1_IDENTITY
        points[2] = points[3]
        sc[2] = sc[3]
    expect = orc.g1_msm(points, sc) if n else orc.G1_IDENTITY
    assert ops.g1_msm(b"".join(points) or b"\0" * 96, sc) == expect


@pytest.mark.parametrize("n", [1, 5, 300])
def test_g2_msm_matches_oracle(orc, n):
    rng = random.Random(200 + n)
    points = orc.g2_mul_many(orc.g2_generator(), rs(rng, n, orc.R))
    sc = rs(rng, n, orc.R)
    assert ops.g2_msm(b"".join(points), sc) == orc.g2_msm(points, sc)


@pytest.mark.parametrize("segments", [9, 31, 33, 64, 1000])
def test_msm_segment_trees_match_oracle(orc, segments):
    """Forced segment counts per window: the segment sums reduce by
    warp-shuffle trees of 32 (full and ragged last trees) and by a final
    per-thread sum, and the MSMs still equal the oracle's."""
    from weighted_bte_b200 import _lib

    rng = random.Random(300 + segments)
    p1 = orc.g1_mul_many(orc.g1_generator(), rs(rng, 513, orc.R))
    s1 = rs(rng, 513, orc.R)
    p2 = orc.g2_mul_many(orc.g2_generator(), rs(rng, 150, orc.R))
    s2 = rs(rng, 150, orc.R)
    ctx = _lib.default_context(0)
    ctx.set_tuning(_lib.TUNE_MSM_SEGMENTS, segments)
    try:
        assert ops.g1_msm(b"".join(p1), s1) == orc.g1_msm(p1, s1)
        assert ops.g2_msm(b"".join(p2), s2) == orc.g2_msm(p2, s2)
    finally:
        ctx.set_tuning(_lib.TUNE_MSM_SEGMENTS, 0)


def test_msm_family_indexed_and_vectors(orc, pts):
    g1, g2 = pts
    rng = random.Random(3)
    n, k, V = 9, 5, 2
    idx = rng.sample(range(20), n)
    base = [0, 7, 20, 44, 3]
    vsel = [0, 1, 1, 0, 1]
    scal = rs(rng, V * n, orc.R)
    for group, bank, size, msm in ((1, g1, 96, orc.g1_msm), (2, g2, 192, orc.g2_msm)):
        got = ops.split(ops.msm_family(group, b"".join(bank), len(bank), base, idx, scal, vsel, V, n), size)
        for j in range(k):
            pj = [bank[base[j] + t] for t in idx]
            sj = scal[vsel[j] * n : (vsel[j] + 1) * n]
            assert got[j] == msm(pj, sj), (group, j)


@pytest.mark.parametrize("lanes", ["auto", "1", "2", "4", "8", "16"])
def test_small_msm_lanes_match_oracle(orc, pts, lanes, monkeypatch):
    """The few-term MSM path (n <= 4) with every lane split: edge scalars
    (0, 1, r - 1), identity points, an output count off the warp size."""
    if lanes != "auto":
        monkeypatch.setenv("WBTE_SMALL_MSM_LANES", lanes)
    g1, g2 = pts
    rng = random.Random(31)
    for n in (1, 2, 3, 4):
        k, V = 37, 3
        idx = rng.sample(range(16), n)
        base = [rng.randrange(0, 40) for _ in range(k)]
        vsel = [rng.randrange(V) for _ in range(k)]
        scal = rs(rng, V * n, orc.R)
        scal[0], scal[-1] = 0, orc.R - 1
        if n > 1:
            scal[1] = 1
        for group, bank, size, msm, ident in ((1, g1, 96, orc.g1_msm, orc.G1_IDENTITY),
                                              (2, g2, 192, orc.g2_msm, bytes(192))):
            bank = list(bank)
            bank[base[2] + idx[0]] = ident
            got = ops.split(ops.msm_family(group, b"".join(bank), len(bank), base, idx, scal, vsel, V, n), size)
            for j in range(k):
                pj = [bank[base[j] + t] for t in idx]
                sj = scal[vsel[j] * n : (vsel[j] + 1) * n]
                assert got[j] == msm(pj, sj), (group, n, j)


def test_compressed_encodings_match_oracle(orc, pts):
    g1, g2 = pts
    g1 = g1[:8] + [orc.G1_IDENTITY]
    g2 = g2[:8] + [orc.G2_IDENTITY]
    assert ops.split(ops.g1_compress(b"".join(g1)), 48) == [orc.g1_compress(p) for p in g1]
    assert ops.split(ops.g2_compress(b"".join(g2)), 96) == [orc.g2_compress(p) for p in g2]


def test_pairing_matches_oracle(orc, pts):
    g1, g2 = pts
    P = g1[:6] + [orc.G1_IDENTITY, g1[0]]
    Q = g2[:6] + [g2[1], orc.G2_IDENTITY]
    got = ops.split(ops.final_exp(ops.miller_loop(b"".join(P), b"".join(Q))), 576)
    for a, b, v in zip(P, Q, got):
        assert v == orc.pairing(a, b)


def test_prepared_lines_match_direct_loop(orc, pts):
    g1, g2 = pts
    P, Q = g1[:5] + [g1[5]], g2[:5] + [orc.G2_IDENTITY]
    lines = ops.prepare_lines(b"".join(Q))
    a = ops.miller_loop_lines(lines, b"".join(P))
    b = ops.miller_loop(b"".join(P), b"".join(Q))
    assert a == b
    assert ops.split(ops.final_exp(a), 576) == [orc.pairing(x, y) for x, y in zip(P, Q)]


def test_final_exponentiation_parts_match_oracle(orc, pts):
    g1, g2 = pts
    fs = [orc.miller_loop(g1[i], g2[i]) for i in range(4)]
    easy = ops.split(ops.final_exp(b"".join(fs), mode=1), 576)
    assert easy == [orc.easy_final_exp(f) for f in fs]
    hard = ops.split(ops.final_exp(b"".join(easy), mode=2), 576)
    assert hard == [orc.hard_final_exp(e) for e in easy]
    full = ops.split(ops.final_exp(b"".join(fs)), 576)
    assert full == [orc.final_exp(f) for f in fs]


def test_multi_miller_matches_oracle(orc, pts):
    g1, g2 = pts
    groups = [(g1[0:3], g2[0:3]), ([], []), ([g1[4], orc.G1_IDENTITY], [g2[4], g2[5]])]
    P = b"".join(b"".join(a) for a, _ in groups)
    Q = b"".join(b"".join(b) for _, b in groups)
    offs = [0, 3, 3, 5]
    got = ops.split(ops.final_exp(ops.multi_miller_loop(P, Q, offs)), 576)
    expect = orc.final_exp_many(orc.multi_miller_many(groups))
    assert got == expect


def test_gt_pow_matches_oracle(orc):
    rng = random.Random(5)
    e = orc.pairing(orc.g1_generator(), orc.g2_generator())
    sc = rs(rng, 12, orc.R) + [0, 1, orc.R - 1, 0xD201000000010000]
    got = ops.split(ops.gt_pow(e, sc, fixed_base=True), 576)
    assert got == [orc.fp12_pow(e, s) for s in sc]


@pytest.mark.parametrize("n", [2, 8, 32])
@pytest.mark.parametrize("joint", ["auto", "0", "1"])
def test_group_ntt_matches_oracle(orc, n, joint, monkeypatch):
    """The lane-split and the one-thread (joint digit) butterflies."""
    if joint != "auto":
        monkeypatch.setenv("WBTE_NTT_JOINT", joint)
    rng = random.Random(300 + n)
    g1 = orc.g1_mul_many(orc.g1_generator(), rs(rng, n, orc.R))
    g2 = orc.g2_mul_many(orc.g2_generator(), rs(rng, n, orc.R))
    g1[0] = orc.G1_IDENTITY
    for inv in (False, True):
        assert ops.split(ops.g1_ntt(b"".join(g1), inverse=inv), 96) == orc.g1_ntt(g1, inverse=inv)
        assert ops.split(ops.g2_ntt(b"".join(g2), inverse=inv), 192) == orc.g2_ntt(g2, inverse=inv)


@pytest.mark.parametrize("lanes", ["auto", "1", "2"])
@pytest.mark.parametrize("n", [2, 4, 8, 16, 32])
def test_gt_transforms_match_oracle(orc, n, lanes, monkeypatch):
    """Radix-2 and radix-4 stages; the radix-4 twiddle powers on one, two or
    four lanes per exponentiation (auto picks four at these sizes)."""
    if lanes != "auto":
        monkeypatch.setenv("WBTE_GT_LANES", lanes)
    rng = random.Random(400 + n)
    e = orc.pairing(orc.g1_generator(), orc.g2_generator())
    vals = orc.gt_pow_many(e, rs(rng, n, orc.R))
    for inv in (False, True):
        assert ops.split(ops.gt_ntt(b"".join(vals), inverse=inv), 576) == orc.gt_ntt(vals, inverse=inv)
    # truncated cyclotomic transform agrees after the hard part
    g1 = orc.g1_mul_many(orc.g1_generator(), rs(rng, n, orc.R))
    g2 = orc.g2_mul_many(orc.g2_generator(), rs(rng, n, orc.R))
    easy = [orc.easy_final_exp(orc.miller_loop(a, b)) for a, b in zip(g1, g2)]
    k = n // 2
    got = ops.split(ops.final_exp(ops.cyclotomic_prefix_ifft(b"".join(easy), k), mode=2), 576)
    expect = orc.hard_final_exp_many(orc.cyclotomic_prefix_ifft(easy, k))
    assert got == expect


@pytest.mark.parametrize("count,lanes", [(32, "auto"), (32, "1"), (32, "2"), (33, "1"), (32, "4"), (27, "1"),
                                         (27, "auto"), (20, "1")])
def test_gt_transforms_many_match_oracle(orc, count, lanes, monkeypatch):
    """Batches of transforms in one launch per stage: 32 arrays give every
    warp one twiddle power (the warp-uniform NAF plan), 33 arrays run as 32
    plus one, 27 arrays run the plan padded to 32 slots, 20 arrays mix
    twiddles within warps (the fixed schedule)."""
    if lanes != "auto":
        monkeypatch.setenv("WBTE_GT_LANES", lanes)
    rng = random.Random(700 + count)
    e = orc.pairing(orc.g1_generator(), orc.g2_generator())
    n = 16
    vals = orc.gt_pow_many(e, rs(rng, n * count, orc.R))
    for inv in (False, True):
        got = ops.split(ops.gt_ntt_many(b"".join(vals), n, inverse=inv), 576)
        for q in range(count):
            assert got[n * q : n * (q + 1)] == orc.gt_ntt(vals[n * q : n * (q + 1)], inverse=inv), (inv, q)
    # truncated cyclotomic transforms agree after the hard part
    m = 8
    g1 = orc.g1_mul_many(orc.g1_generator(), rs(rng, m * count, orc.R))
    g2 = orc.g2_mul_many(orc.g2_generator(), rs(rng, m, orc.R))
    easy = [orc.easy_final_exp(orc.miller_loop(a, g2[i % m])) for i, a in enumerate(g1)]
    got = ops.cyclotomic_prefix_ifft_many(b"".join(easy), m, m // 2)
    for q in range(count):
        hard = ops.split(ops.final_exp(got[q], mode=2), 576)
        assert hard == orc.hard_final_exp_many(orc.cyclotomic_prefix_ifft(easy[m * q : m * (q + 1)], m // 2)), q


def test_lagrange_matches_oracle(orc):
    rng = random.Random(6)
    xs = rs(rng, 70, orc.R)
    assert ops.lagrange_at_zero(xs) == orc.lagrange_at_zero(xs)


def test_schnorr_verify(orc):
    rng = random.Random(7)
    n = 6
    r = rs(rng, n, orc.R)
    k = rs(rng, n, orc.R)
    c = rs(rng, n, orc.R)
    s = [(ki + ci * ri) % orc.R for ki, ci, ri in zip(k, c, r)]
    X = orc.g1_mul_many(orc.g1_generator(), r)
    Rc = orc.g1_mul_many(orc.g1_generator(), k)
    s[2] = (s[2] + 1) % orc.R
    ok = ops.schnorr_verify(b"".join(X), b"".join(Rc), s, c)
    assert list(ok) == [True, True, False, True, True, True]


def _host_challenge(parts, R):
    """Checker: SHA-256 rejection sampling over the concatenated parts."""
    import hashlib
    import struct

    msg = b"".join(parts)
    counter = 0
    while True:
        v = int.from_bytes(hashlib.sha256(msg + struct.pack("<I", counter)).digest(), "little")
        if v < R:
            return v
        counter += 1


@pytest.mark.parametrize("n", [1, 7, 300])
def test_transcript_challenges_match_sha256(orc, n):
    """Constant, fixed-stride and variable GT fields, record lengths crossing
    the 64-byte block and padding boundaries, identity GT records."""
    from weighted_bte_b200 import _lib

    rng = random.Random(100 + n)
    prefix = bytes(rng.randrange(256) for _ in range(rng.randrange(0, 130)))
    a_len = rng.randrange(1, 70)
    a = bytes(rng.randrange(256) for _ in range(a_len * n))
    te = bytearray(rng.randrange(256) for _ in range(289 * n))
    for i in range(n):
        te[289 * i] = 0 if i % 3 == 1 else 1  # every third record is the identity
    tail = bytes(rng.randrange(256) for _ in range(5))
    fields = [(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES), (a, a_len, a_len, _lib.TRANSCRIPT_BYTES),
              (bytes(te), 289, 289, _lib.TRANSCRIPT_GT_VARIABLE), (tail, 0, 5, _lib.TRANSCRIPT_BYTES)]
    got = ops.transcript_challenges(fields, n)
    for i in range(n):
        rec = bytes(te[289 * i : 289 * (i + 1)])
        gt = rec[:1] if rec[0] == 0 else rec
        assert got[i] == _host_challenge([prefix, a[a_len * i : a_len * (i + 1)], gt, tail], orc.R), i


def test_transcript_challenges_exact_block_lengths(orc):
    """Messages whose length before the counter is 55, 56, 60 and 64 bytes:
    the padding edge cases of SHA-256."""
    from weighted_bte_b200 import _lib

    for total in (51, 52, 56, 60, 119, 120):
        data = bytes((7 * i + total) & 0xFF for i in range(total * 3))
        got = ops.transcript_challenges([(data, total, total, _lib.TRANSCRIPT_BYTES)], 3)
        for i in range(3):
            assert got[i] == _host_challenge([data[total * i : total * (i + 1)]], orc.R)
