"""The btx CPU restatement against the reference crate's own tests
(btx/src/decryption.rs:540-712, setup.rs:281-309): the FFT middle product
equals the quadratic cross-term formula, threshold decryption round-trips,
invalid slots keep their position, and share checks reject corruption."""
import pytest

from weighted_bte_b200.rng import ChaCha20Rng


@pytest.fixture(scope="module")
def btx(orc):
    from oracle import btx_oracle

    return btx_oracle


def fixture(btx, orc, L, B, seed):
    rng = ChaCha20Rng.seed_from_u64(seed)
    key = btx.keygen(L, 5, 2, rng)
    gen = btx.gt_generator()
    msgs = [orc.fp12_pow(gen, i + 17) for i in range(B)]
    cts = btx.encrypt_many(key, msgs, rng)
    return key, msgs, cts


def test_keygen_shapes(btx, orc):
    key = btx.keygen(8, 5, 2, ChaCha20Rng.seed_from_u64(1))
    assert len(key["low"]) == 192 * 8 and len(key["high"]) == 192 * 7
    assert len(key["shares"]) == 5 and all(len(s) == 8 for s in key["shares"])
    # power i is tau^i and the shares interpolate back to it at zero
    tau = key["tau"]
    assert btx.power(key, 3) == orc.g2_mul(orc.g2_generator(), pow(tau, 3, orc.R))
    lam = orc.lagrange_at_zero([1, 2, 3])
    assert sum(l * s for l, s in zip(lam, [key["shares"][j][4] for j in range(3)])) % orc.R == pow(tau, 5, orc.R)
    with pytest.raises(ValueError):
        btx.power(key, 9)


@pytest.mark.parametrize("B", [1, 2, 3, 5, 8])
def test_fft_middle_product_matches_quadratic_formula(btx, orc, B):
    key, _, cts = fixture(btx, orc, 8, B, 10 + B)
    batch = btx.validate(cts)
    assert btx.precompute(btx.kernel(key, B), batch) == btx.naive_beta(key, batch)


def test_threshold_end_to_end(btx, orc):
    key, msgs, cts = fixture(btx, orc, 8, 6, 3)
    batch = btx.validate(cts)
    kern = btx.kernel(key, 6)
    beta = btx.precompute(kern, batch)
    shares = [(j, btx.partial_decrypt(key, j, batch)) for j in range(3)]
    for j, s in shares:
        assert btx.verify_share(key, batch, j, s)
    sigma = btx.combine(key, shares)
    assert btx.verify_combined(key, batch, sigma)
    assert btx.open_batch(kern, batch, cts, beta, sigma) == msgs
    # a shuffled subset reconstructs the same aggregate
    sub = [(j, btx.partial_decrypt(key, j, batch)) for j in (4, 1, 3)]
    assert btx.combine(key, sub) == sigma


def test_invalid_proof_keeps_slot(btx, orc):
    key, msgs, cts = fixture(btx, orc, 8, 5, 4)
    cts[3] = dict(cts[3], response=(cts[3]["response"] + 1) % orc.R)
    batch = btx.validate(cts)
    assert batch["valid"] == [True, True, True, False, True]
    kern = btx.kernel(key, 5)
    beta = btx.precompute(kern, batch)
    sigma = btx.combine(key, [(j, btx.partial_decrypt(key, j, batch)) for j in range(3)])
    out = btx.open_batch(kern, batch, cts, beta, sigma)
    assert out == [m if i != 3 else None for i, m in enumerate(msgs)]


def test_corrupted_share_fails(btx, orc):
    key, _, cts = fixture(btx, orc, 8, 4, 5)
    batch = btx.validate(cts)
    s = btx.partial_decrypt(key, 0, batch)
    bad = orc.g1_add(s, orc.g1_generator())
    assert btx.verify_share(key, batch, 0, s)
    assert not btx.verify_share(key, batch, 0, bad)
