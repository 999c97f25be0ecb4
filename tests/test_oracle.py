"""CPU checks of the oracle: pinned against the constants the reference's own
tests hold, against algebraic identities of the pairing, and against the
reference's differential tests (FFT middle product vs the literal formula)."""
import json
import os
import random

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB


@pytest.fixture(scope="module")
def consts():
    with open(os.path.join(HERE, "golden", "reference_constants.json")) as f:
        return json.load(f)


def test_reference_constants_pin_the_curve(orc, consts):
    x = -consts["bls12_381_x_abs"]
    assert x ** 4 - x ** 2 + 1 == orc.R
    h = sum(l << (64 * i) for i, l in enumerate(consts["hard_exponent_limbs_le"]))
    assert h * orc.R == P ** 4 - P ** 2 + 1
    assert consts["miller_line_count"] == 63 + bin(consts["bls12_381_x_abs"]).count("1") - 1


def test_hard_part_is_the_reference_chain(orc, consts):
    """The addition chain of btx/src/final_exponentiation.rs:255-283 raises to 3h."""
    h = sum(l << (64 * i) for i, l in enumerate(consts["hard_exponent_limbs_le"]))
    f = orc.easy_final_exp(orc.miller_loop(orc.g1_mul(orc.g1_generator(), 5), orc.g2_mul(orc.g2_generator(), 9)))
    assert orc.hard_final_exp(f) == orc.fp12_pow(f, 3 * h)


def test_generators_and_encodings(orc):
    g1, g2 = orc.g1_generator(), orc.g2_generator()
    assert orc.g1_on_curve(g1) and orc.g2_on_curve(g2)
    assert orc.g1_mul(g1, orc.R) == orc.G1_IDENTITY and orc.g2_mul(g2, orc.R) == orc.G2_IDENTITY
    # ZCash serialisation of the standard generators (public BLS12-381 parameters)
    assert orc.g1_compress(g1).hex().startswith("97f1d3a73197d7942695638c4fa9ac0f")
    assert orc.g2_compress(g2).hex().startswith("93e02b6052719f607dacd3a088274f65")
    assert orc.g1_compress(orc.G1_IDENTITY)[0] == 0xC0


def test_pairing_is_bilinear_and_non_degenerate(orc):
    rng = random.Random(9)
    g1, g2 = orc.g1_generator(), orc.g2_generator()
    e = orc.pairing(g1, g2)
    a, b = rng.randrange(orc.R), rng.randrange(orc.R)
    assert orc.pairing(orc.g1_mul(g1, a), orc.g2_mul(g2, b)) == orc.fp12_pow(e, a * b % orc.R)
    assert orc.fp12_is_one(orc.fp12_pow(e, orc.R))
    assert not orc.fp12_is_one(e)
    assert orc.fp12_is_one(orc.pairing(orc.G1_IDENTITY, g2))


def test_split_final_exponentiation_agrees(orc):
    """btx/src/final_exponentiation.rs:430-482: split == full, batched easy == individual."""
    rng = random.Random(10)
    fs = [orc.miller_loop(orc.g1_mul(orc.g1_generator(), rng.randrange(orc.R)),
                          orc.g2_mul(orc.g2_generator(), rng.randrange(orc.R))) for _ in range(3)]
    easy = orc.batch_easy_final_exp(fs)
    assert easy == [orc.easy_final_exp(f) for f in fs]
    assert [orc.hard_final_exp(e) for e in easy] == [orc.final_exp(f) for f in fs]


def test_base_x_decomposition_recomposes(orc, consts):
    """btx/src/fft.rs:749-782."""
    xa = consts["bls12_381_x_abs"]
    rng = random.Random(11)
    for s in [0, 1, 2, xa - 1, xa, xa + 1, xa * xa % orc.R, orc.R - 1] + [rng.randrange(orc.R) for _ in range(16)]:
        comps = orc.base_x_decompose(s)
        assert all(c < xa for c in comps)
        assert sum(c * xa ** i for i, c in enumerate(comps)) % orc.R == s


def test_decomposed_gt_power_matches_ordinary(orc):
    """btx/src/fft.rs:811-846 and the raw-cyclotomic projection test :848-864."""
    rng = random.Random(12)
    e = orc.pairing(orc.g1_generator(), orc.g2_generator())
    for s in [0, 1, 2, orc.R - 1, rng.randrange(orc.R)]:
        assert orc.gt_pow_decomposed(e, s) == orc.fp12_pow(e, s)
    f = orc.easy_final_exp(orc.miller_loop(orc.g1_mul(orc.g1_generator(), 3), orc.g2_generator()))
    s = rng.randrange(orc.R)
    assert orc.hard_final_exp(orc.gt_pow_decomposed(f, s)) == orc.hard_final_exp(orc.fp12_pow(f, s))


def test_cyclotomic_prefix_ifft_matches_full_gt_ifft(orc):
    """btx/src/fft.rs:866-933."""
    rng = random.Random(13)
    n = 8
    g1, g2 = orc.g1_generator(), orc.g2_generator()
    pairs = [(orc.G1_IDENTITY, orc.G2_IDENTITY), (orc.G1_IDENTITY, g2), (g1, orc.G2_IDENTITY), (g1, g2)]
    pairs += [(orc.g1_mul(g1, rng.randrange(orc.R)), orc.g2_mul(g2, rng.randrange(orc.R))) for _ in range(n - 4)]
    miller = [orc.miller_loop(a, b) for a, b in pairs]
    easy = [orc.easy_final_exp(f) for f in miller]
    full = [orc.final_exp(f) for f in miller]
    expect = orc.gt_ntt(full, inverse=True)
    for k in (0, 1, 3, n // 2):
        got = [orc.hard_final_exp(v) for v in orc.cyclotomic_prefix_ifft(easy, k)]
        assert got == expect[:k]


def test_group_transforms_round_trip(orc):
    """btx/src/fft.rs:713-747."""
    n = 8
    inv = pow(n, orc.R - 2, orc.R)
    vals = orc.g1_mul_many(orc.g1_generator(), list(range(1, n + 1)))
    back = orc.g1_ntt(orc.g1_ntt(vals), inverse=True)
    assert orc.g1_mul_many(back, [inv] * n) == vals
    s = list(range(1, 17))
    assert [v * pow(16, orc.R - 2, orc.R) % orc.R for v in orc.fr_ntt(orc.fr_ntt(s), inverse=True)] == s


def test_lagrange_reconstructs_random_polynomials(orc):
    """weighted_btx/src/interpolation.rs tests: L_i(0) reconstruct P(0)."""
    rng = random.Random(14)
    for n in (1, 5, 40):
        xs = rng.sample(range(1, 10 ** 6), n)
        coeffs = [rng.randrange(orc.R) for _ in range(n)]
        ys = [sum(c * pow(x, i, orc.R) for i, c in enumerate(coeffs)) % orc.R for x in xs]
        lam = orc.lagrange_at_zero(xs)
        assert sum(l * y for l, y in zip(lam, ys)) % orc.R == coeffs[0]
    with pytest.raises(ValueError):
        orc.lagrange_at_zero([3, 3])


WEIGHTS, THRESHOLD = [1, 3, 2, 4, 1], 5


@pytest.fixture(scope="module")
def small_setup(orc):
    from oracle import wbtx_oracle as W
    from weighted_bte_b200.rng import ChaCha20Rng

    rng = ChaCha20Rng.seed_from_u64(5)
    key = W.keygen(8, WEIGHTS, THRESHOLD, rng)
    return W, key, rng


def test_oracle_keygen_shapes_and_reconstruction(orc, small_setup):
    """weighted_btx/src/setup.rs:531-671."""
    W, key, _ = small_setup
    assert len(key["vk"]) == 8 * 5 and len(key["neg_blob"]) == 192 * 8 * 11 and len(key["pos_blob"]) == 192 * 7 * 11
    assert key["domain"][0] == 1 and len(set(key["domain"])) == 11
    sel = [0, 2, 5, 7, 10, 3]
    pts = [key["domain"][i] for i in sel]
    lam = orc.lagrange_at_zero(pts)
    owner = [j for j, w in enumerate(WEIGHTS) for _ in range(w)]
    neg = W.points(key["neg_blob"])
    bases = [orc.g2_mul(neg[i], key["qs"][owner[i]]) for i in sel]
    rec = orc.g2_msm(bases, lam)
    assert orc.pairing(orc.g1_generator(), rec) == key["ek"]


def test_oracle_pipeline_round_trip_and_middle_product(orc, small_setup):
    """weighted_btx/src/decryption.rs:844-862: end to end, and the FFT middle
    product equals the literal quadratic formula."""
    W, key, rng = small_setup
    gt = W.gt_generator()
    for B, parties in ((7, [1, 3]), (3, [1, 2, 3]), (1, [1, 3])):
        msgs = [orc.fp12_pow(gt, 17 + i) for i in range(B)]
        cts = W.encrypt_many(key, msgs, rng)
        batch = W.validate(key["setup_id"], cts)
        assert all(batch["valid"])
        sig = [W.partial_decrypt(key["qs"][j], batch) for j in parties]
        assert W.verify_shares(key, batch, parties, sig, [3 + j for j in range(len(parties))])
        pre = W.prepare(key, parties, B)
        beta = W.precompute(pre, batch)
        assert beta == W.naive_beta(key, batch, parties)
        assert W.open_batch(pre, sig, batch, cts, beta) == msgs


def test_oracle_invalid_slot_opens_as_bottom(orc, small_setup):
    W, key, rng = small_setup
    gt = W.gt_generator()
    msgs = [orc.fp12_pow(gt, 30 + i) for i in range(4)]
    cts = W.encrypt_many(key, msgs, rng)
    cts[2] = dict(cts[2], response=(cts[2]["response"] + 1) % orc.R)
    batch = W.validate(key["setup_id"], cts)
    assert batch["valid"] == [True, True, False, True]
    sig = [W.partial_decrypt(key["qs"][j], batch) for j in (1, 3)]
    bad = orc.g1_add(sig[0], orc.g1_generator())
    assert not W.verify_shares(key, batch, [1, 3], [bad, sig[1]], [5, 7])
    pre = W.prepare(key, [1, 3], 4)
    out = W.open_batch(pre, sig, batch, cts, W.precompute(pre, batch))
    assert out == [msgs[0], msgs[1], None, msgs[3]]


def test_chacha20_block_matches_rfc8439():
    import struct

    from weighted_bte_b200.rng import chacha20_block

    key = list(struct.unpack("<8I", bytes(range(32))))
    out = chacha20_block(key, 1 | (0x09000000 << 32), 0x4A000000)
    assert out[0] == 0xE4E7F110 and out[1] == 0x15593BD1 and out[15] == 0x4E3C50A2


def test_work_counts_reproduce(orc):
    """The counting build of the oracle reproduces the recorded work table
    (oracle/count_work.py) for the hard final exponentiation, and counts
    nothing in the regular build."""
    import ctypes
    import json
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    count = ctypes.CDLL(os.path.join(root, "oracle", "_build", "liboracle_count.so"))
    count.orc_init()
    count.orc_fp_product_count.restype = ctypes.c_ulonglong
    with open(os.path.join(root, "weighted_bte_b200", "algorithmic_work.json")) as f:
        table = json.load(f)
    f12 = orc.easy_final_exp(orc.miller_loop(orc.g1_generator(), orc.g2_generator()))
    out = ctypes.create_string_buffer(576)
    count.orc_fp_product_count_reset()
    count.orc_hard_final_exp(out, f12)
    assert count.orc_fp_product_count() == table["hard_final_exp"]["fp_products"]
    assert out.raw == orc.hard_final_exp(f12)
    plain = orc.lib()
    plain.orc_fp_product_count.restype = ctypes.c_ulonglong
    assert plain.orc_fp_product_count() == 0


def test_vectorised_chacha20_blocks_equal_the_block_function():
    import random

    from weighted_bte_b200.rng import ChaCha20Rng, chacha20_block, chacha20_blocks

    rng = random.Random(5)
    key = [rng.getrandbits(32) for _ in range(8)]
    for counter in (0, 1, (1 << 32) - 3, (1 << 40) + 7):
        flat = chacha20_blocks(key, counter, 5)
        for b in range(5):
            assert flat[16 * b : 16 * (b + 1)] == chacha20_block(key, counter + b)
    # the generator's stream does not depend on how many blocks a refill makes
    a, b = ChaCha20Rng.seed_from_u64(9), ChaCha20Rng.seed_from_u64(9)
    b.REFILL_BLOCKS = 1
    assert [a.next_u64() for _ in range(300)] == [b.next_u64() for _ in range(300)]
