"""The pfe CPU restatement against the reference crate's own tests
(pfe/src/decryption.rs:676-905): the gamma-weighted convolution against its
literal denominators, threshold round trips at small power-of-two sizes,
subset reconstruction and share checks."""
import pytest

from weighted_bte_b200.rng import ChaCha20Rng


@pytest.fixture(scope="module")
def pf(orc):
    from oracle import pfe_oracle

    return pfe_oracle


def fixture(pf, orc, B, N=5, t=2, seed=1):
    rng = ChaCha20Rng.seed_from_u64(seed)
    key = pf.keygen(B, N, t, rng)
    gen = pf.gt_generator()
    msgs = [orc.fp12_pow(gen, i + 17) for i in range(B)]
    cts = pf.encrypt_many(key, msgs, rng)
    return key, msgs, cts, pf.validate(key, cts)


@pytest.mark.parametrize("B", [1, 2, 4, 8])
def test_convolution_matches_literal_denominators(pf, orc, B):
    gamma, c = pf.extra_index_data(B)
    pts = pf.index_points(B)
    ginv = orc.domain_generator(B, inverse=True) if B > 1 else 1
    values = [orc.g1_mul(orc.g1_generator(), i + 3) for i in range(B)]
    got = pf.conv_g1(values, c)
    for o in range(B):
        raw = orc.G1_IDENTITY
        for i, v in enumerate(values):
            if i == o:
                continue
            d = pf.inv(1 - pow(ginv, (o + B - i) % B, orc.R))
            raw = orc.g1_add(raw, orc.g1_mul(v, d))
        q = (pts[o] * c - 1) % orc.R
        assert got[o] == orc.g1_mul(raw, 2 * B * q % orc.R)
        assert q == (pts[o] - gamma) * c % orc.R


@pytest.mark.parametrize("B", [1, 2, 4, 8])
def test_threshold_round_trip(pf, orc, B):
    key, msgs, cts, batch = fixture(pf, orc, B, seed=10 + B)
    kern = pf.kernel(key)
    bp = pf.precompute(kern, batch)
    shares = [(j, pf.partial_decrypt(key, j, batch)) for j in range(3)]
    for j, s in shares:
        assert pf.verify_share(key, batch, j, s)
    pdk = pf.combine(key, shares)
    assert pf.verify_combined(key, batch, pdk)
    assert pf.open_batch(kern, batch, cts, bp, pdk) == msgs
    assert pf.combine(key, [(j, pf.partial_decrypt(key, j, batch)) for j in (4, 1, 3)]) == pdk


def test_identity_messages_and_bad_share(pf, orc):
    rng = ChaCha20Rng.seed_from_u64(3)
    key = pf.keygen(4, 5, 2, rng)
    msgs = [orc.fp12_one()] * 2 + [orc.fp12_pow(pf.gt_generator(), 5)] * 2
    cts = pf.encrypt_many(key, msgs, rng)
    batch = pf.validate(key, cts)
    kern = pf.kernel(key)
    pdk = pf.combine(key, [(j, pf.partial_decrypt(key, j, batch)) for j in range(3)])
    assert pf.open_batch(kern, batch, cts, pf.precompute(kern, batch), pdk) == msgs
    s = pf.partial_decrypt(key, 0, batch)
    assert not pf.verify_share(key, batch, 0, orc.g1_add(s, orc.g1_generator()))
    bad = [dict(cts[0], response=(cts[0]["response"] + 1) % orc.R)] + cts[1:]
    with pytest.raises(ValueError):
        pf.validate(key, bad)
