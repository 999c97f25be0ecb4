"""pfe on the GPU: bit-exact parity with the CPU restatement on the same
seeded inputs and the reference crate's protocol tests
(pfe/src/decryption.rs:724-905) through the public API."""
import pytest

from weighted_bte_b200 import pfe
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu


def gt_msgs(n, base=17):
    from weighted_bte_b200 import ops

    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def as_oracle_cts(cts):
    return [dict(first=c.first, second=c.second, third=c.third, response=c.proof.response,
                 c1=c.proof.first_commitment, c2=c.proof.second_commitment) for c in cts]


@pytest.mark.parametrize("B,N,t,seed", [(1, 3, 1, 2), (8, 5, 2, 3), (32, 16, 8, 0)])
def test_pipeline_matches_oracle_stage_by_stage(orc, B, N, t, seed):
    from oracle import pfe_oracle as X

    mat = pfe.keygen_with_rng(pfe.KeygenConfig(B, N, t), ChaCha20Rng.seed_from_u64(seed))
    key = X.keygen(B, N, t, ChaCha20Rng.seed_from_u64(seed))
    dk, ek = mat.decryption_key, mat.encryption_key
    assert ek.relation_base == key["relation_base"] and ek.masking_base == key["masking_base"]
    assert wb.to_host(dk.fraction_keys) == key["keys"] and wb.to_host(dk.fraction_key_sum) == key["key_sum"]
    assert [s.fraction_shares for s in mat.server_keys] == key["shares"]
    assert wb.to_host(dk.share_commitments) == b"".join(key["commitments"])

    msgs = gt_msgs(B)
    cts = pfe.encrypt_many(ek, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    octs = X.encrypt_many(key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    assert as_oracle_cts(cts) == octs
    batch = pfe.validate_batch(ek, cts)
    obatch = X.validate(key, octs)
    assert batch.digest() == obatch["digest"]

    kern = pfe.PartialFractionKernel.new(dk)
    okern = X.kernel(key)
    assert wb.to_host(kern.scaled_keys) == b"".join(okern["scaled_keys"])
    assert wb.to_host(kern.generators) == b"".join(okern["gens"])
    assert wb.to_host(kern.mixes) == b"".join(okern["mixes"])
    bp = pfe.precompute_batch(kern, batch)
    obp = X.precompute(okern, obatch)
    assert wb.to_host(bp.weighted_first) == b"".join(obp["weighted_first"])
    assert wb.to_host(bp.weighted_pairings) == b"".join(obp["weighted_pairings"])

    servers = list(range(t + 1))
    shares = [pfe.partial_decrypt(mat.server_keys[j], batch) for j in servers]
    assert [s.pre_decryption_key for s in shares] == [X.partial_decrypt(key, j, obatch) for j in servers]
    pdk = pfe.combine_shares(dk, batch, shares)
    assert pdk == X.combine(key, [(j, s.pre_decryption_key) for j, s in zip(servers, shares)])
    assert pfe.verify_combined_share(dk, batch, pdk)
    assert pfe.verify_decryption_share(dk, batch, shares[0])
    out = pfe.open_batch(kern, batch, cts, bp, pdk)
    assert out == X.open_batch(okern, obatch, octs, obp, pdk) == msgs


def fixture(B, N=5, t=2, seed=4):
    mat = pfe.keygen_with_rng(pfe.KeygenConfig(B, N, t), ChaCha20Rng.seed_from_u64(seed))
    msgs = gt_msgs(B)
    cts = pfe.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    batch = pfe.ValidatedBatch.verify(mat.encryption_key, cts)
    return mat, msgs, cts, batch, pfe.PartialFractionKernel.new(mat.decryption_key)


@pytest.mark.parametrize("B", [1, 2, 4, 8, 16])
def test_round_trips_small_power_of_two_sizes_and_identity_messages(B):
    mat, msgs, cts, batch, kern = fixture(B, seed=20 + B)
    assert pfe.decrypt(mat.encryption_key, mat.decryption_key, cts, mat.server_keys[:3], kern) == msgs
    ident = [wb.gt_identity()] * B
    cts2 = pfe.encrypt_many(mat.encryption_key, ident, ChaCha20Rng.seed_from_u64(7))
    assert pfe.decrypt(mat.encryption_key, mat.decryption_key, cts2, mat.server_keys[:3], kern) == ident


def test_arbitrary_eight_of_sixteen_subset_reconstructs():
    mat, msgs, cts, batch, kern = fixture(8, N=16, t=7)
    pre = pfe.precompute_batch(kern, batch)
    shares = [pfe.partial_decrypt(mat.server_keys[i], batch) for i in (15, 2, 9, 4, 11, 0, 7, 13)]
    pdk = pfe.combine_shares(mat.decryption_key, batch, shares)
    assert pfe.open_batch(kern, batch, cts, pre, pdk) == msgs


def test_checked_combine_discards_a_bad_share():
    from weighted_bte_b200 import ops

    mat, msgs, cts, batch, kern = fixture(4)
    pre = pfe.precompute_batch(kern, batch)
    shares = [pfe.partial_decrypt(k, batch) for k in mat.server_keys[:4]]
    shares[1].pre_decryption_key = ops.g1_sum(shares[1].pre_decryption_key + wb.g1_generator(), [0, 2])
    assert not pfe.verify_decryption_share(mat.decryption_key, batch, shares[1])
    pdk = pfe.combine_shares_checked(mat.decryption_key, batch, shares)
    assert pfe.open_batch(kern, batch, cts, pre, pdk) == msgs


def test_rejects_invalid_proof_and_share_sets():
    mat, _, cts, batch, _ = fixture(4)
    bad = list(cts)
    p = bad[2].proof
    bad[2] = pfe.Ciphertext(bad[2].first, bad[2].second, bad[2].third,
                            pfe.DleqProof((p.response + 1) % pfe.R, p.first_commitment, p.second_commitment))
    assert not bad[2].verify(mat.encryption_key) and cts[2].verify(mat.encryption_key)
    with pytest.raises(pfe.InvalidProof):
        pfe.validate_batch(mat.encryption_key, bad)
    share = pfe.partial_decrypt(mat.server_keys[0], batch)
    with pytest.raises(pfe.InsufficientShares):
        pfe.combine_shares(mat.decryption_key, batch, [share])
    with pytest.raises(pfe.DuplicateServerIndex):
        pfe.combine_shares(mat.decryption_key, batch, [share, share, share])
    with pytest.raises(pfe.InvalidBatchSize):
        pfe.keygen(3, 5, 2)
    with pytest.raises(pfe.InvalidCommittee):
        pfe.keygen(4, 3, 3)
