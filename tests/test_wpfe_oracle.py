"""The weighted_pfe CPU restatement against the reference crate's own tests
(weighted_pfe/src/decryption.rs:926-1124, setup.rs:755-980): round trips at
small batch sizes, the optimized Cauchy transforms against the literal
quadratic sums, the fused opening against Construction 5's displayed
formula, and a non-greedy authorized committee."""
import pytest

from weighted_bte_b200.rng import ChaCha20Rng


@pytest.fixture(scope="module")
def wp(orc):
    from oracle import wpfe_oracle

    return wpfe_oracle


def fixture(wp, orc, B, seed=1, weights=(1, 3, 2, 4), t=4):
    rng = ChaCha20Rng.seed_from_u64(seed)
    key = wp.keygen(B, list(weights), t, rng)
    gen = wp.gt_generator()
    msgs = [orc.fp12_pow(gen, s + 11) for s in range(B)]
    cts = wp.encrypt_many(key, msgs, rng)
    batch = wp.validate(key, cts)
    return key, msgs, cts, batch


def decrypt(wp, key, cts, batch, parties):
    sig = [wp.partial_decrypt(key, j, batch) for j in parties]
    pre = wp.prepare(key, parties)
    bp = wp.precompute(key, pre, batch)
    return wp.open_batch(key, pre, sig, batch, cts, bp), pre, sig


def test_key_material_dimensions(wp, orc):
    key = wp.keygen(4, [1, 3, 2, 4], 4, ChaCha20Rng.seed_from_u64(2))
    assert len(key["vk"]) == 192 * 4 * 4 and len(key["d1"]) == 192 * 4 * 10 and len(key["d2"]) == 192 * 4 * 10
    assert key["alpha"] == [(r + key["shift"]) % orc.R for r in wp.root_domain_prefix(4, 4)]
    # the party shifts and verification keys match the derived fractions
    j, i = 2, 3
    assert wp._pt(key["vk"], i * 4 + j) == orc.g2_mul(orc.g2_generator(), wp.inv(key["rhos"][j] + key["alpha"][i]))


@pytest.mark.parametrize("B", [1, 2, 4, 8])
def test_heterogeneous_weighted_round_trip(wp, orc, B):
    key, msgs, cts, batch = fixture(wp, orc, B, seed=10 + B)
    parties = wp.select_committee(key, range(4))
    assert parties == [1, 3]
    out, _, _ = decrypt(wp, key, cts, batch, parties)
    assert out == msgs


def test_non_greedy_committee(wp, orc):
    key, msgs, cts, batch = fixture(wp, orc, 4, seed=5)
    out, _, _ = decrypt(wp, key, cts, batch, [0, 3])
    assert out == msgs


@pytest.mark.parametrize("B", [1, 2, 4, 8])
def test_cauchy_transforms_match_literal_sums(wp, orc, B):
    key = wp.keygen(B, [1, 2], 1, ChaCha20Rng.seed_from_u64(20 + B))
    g1 = [orc.g1_mul(orc.g1_generator(), i + 3) for i in range(B)]
    raw = [orc.miller_loop(orc.g1_mul(orc.g1_generator(), i + 5), orc.g2_mul(orc.g2_generator(), 2 * i + 7))
           for i in range(B)]
    easy = orc.batch_easy_final_exp(raw)
    gt = [orc.final_exp(f) for f in raw]
    exp_g1, exp_gt = wp.literal_cauchy(key, g1, gt)
    assert wp.cauchy_group(g1) == exp_g1
    assert orc.hard_final_exp_many(wp.cauchy_cyclotomic(easy)) == exp_gt


def test_fused_opening_matches_displayed_formula(wp, orc):
    key, msgs, cts, batch = fixture(wp, orc, 4, seed=7)
    out, pre, sig = decrypt(wp, key, cts, batch, [1, 3])
    assert out == wp.literal_open(key, pre, sig, batch, cts) == msgs


def test_malformed_share_fails_and_invalid_proof_rejects_batch(wp, orc):
    key, _, cts, batch = fixture(wp, orc, 2, seed=9)
    s = wp.partial_decrypt(key, 3, batch)
    assert wp.verify_share(key, batch, 3, s)
    assert not wp.verify_share(key, batch, 3, orc.g1_add(s, orc.g1_generator()))
    bad = [dict(cts[0], response=(cts[0]["response"] + 1) % orc.R)] + cts[1:]
    with pytest.raises(ValueError):
        wp.validate(key, bad)
