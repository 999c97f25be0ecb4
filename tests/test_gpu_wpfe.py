"""weighted_pfe on the GPU: bit-exact parity with the CPU restatement on the
same seeded inputs, and the reference crate's protocol tests
(weighted_pfe/src/decryption.rs:926-1229, setup.rs:755-980) through the public
API.  Cyclotomic intermediates are compared after the hard part only."""
import pytest

from weighted_bte_b200 import errors as E
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200 import weighted_pfe as wp
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu

WEIGHTS, T = [1, 3, 2, 4], 4


def gt_msgs(n, base=11):
    from weighted_bte_b200 import ops

    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def as_oracle_cts(cts):
    return [dict(first=c.first, second=c.second, commitment=c.proof.commitment, response=c.proof.response)
            for c in cts]


@pytest.mark.parametrize("B,seed", [(1, 3), (4, 4), (16, 5)])
def test_pipeline_matches_oracle_stage_by_stage(orc, B, seed):
    from oracle import wpfe_oracle as X

    mat = wp.keygen_with_rng(wp.KeygenConfig(B, WEIGHTS, T), ChaCha20Rng.seed_from_u64(seed))
    key = X.keygen(B, WEIGHTS, T, ChaCha20Rng.seed_from_u64(seed))
    dk = mat.decryption_key
    assert dk.alpha_points() == key["alpha"] and dk.domain_points() == key["eval_domain"]
    assert [p.rho for p in mat.party_keys] == key["rhos"]
    assert wb.to_host(dk.verification_keys) == key["vk"]
    assert wb.to_host(dk.d1) == key["d1"] and wb.to_host(dk.d2) == key["d2"]
    assert dk.global_key() == key["V"] and mat.encryption_key.element() == key["ek"]
    assert dk.setup_id() == key["setup_id"]
    assert mat.party_keys[2].fractions() == key["g"][2]

    msgs = gt_msgs(B)
    cts = wp.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 100))
    octs = X.encrypt_many(key, msgs, ChaCha20Rng.seed_from_u64(seed + 100))
    assert as_oracle_cts(cts) == octs
    batch = wp.validate_batch(mat.encryption_key, cts)
    obatch = X.validate(key, octs)
    assert batch.digest() == obatch["digest"]

    shares = wp.partial_decrypt_many(mat.party_keys, batch)
    assert [s.sigma for s in shares] == [X.partial_decrypt(key, j, obatch) for j in range(4)]
    accepted = wp.accept_decryption_shares(dk, batch, shares, ChaCha20Rng.seed_from_u64(1))
    assert accepted.party_indices() == X.select_committee(key, range(4)) == [1, 3]
    assert accepted.accepted_weight() == 7
    pre = wp.prepare_decryption(dk, accepted)
    opre = X.prepare(key, [1, 3])
    assert wb.to_host(pre.scaled_d1_by_party) == b"".join(opre["by_party"])
    assert wb.to_host(pre.scaled_d1_total) == b"".join(opre["total"])
    assert wb.to_host(pre.mask_keys) == b"".join(opre["mask"])
    assert pre.context_id == opre["context_id"]

    kern = wp.CauchyKernel.new(dk)
    bp = wp.precompute_batch(kern, pre, batch)
    obp = X.precompute(key, opre, obatch)
    assert wb.to_host(bp.scaled_first_cauchy, 96 * B) == b"".join(obp["first_cauchy"])
    from weighted_bte_b200 import ops

    got_pc = ops.split(ops.final_exp(wb.to_host(bp.pairing_cauchy, 576 * B), mode=2), 576)
    assert got_pc == orc.hard_final_exp_many(obp["pairing_cauchy"])

    out = wp.open_batch(dk, kern, pre, accepted, batch, cts, bp)
    assert out == X.open_batch(key, opre, [shares[1].sigma, shares[3].sigma], obatch, octs, obp) == msgs


def fixture(B, seed=8):
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, WEIGHTS, T), ChaCha20Rng.seed_from_u64(seed))
    msgs = gt_msgs(B)
    cts = wp.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    batch = wp.validate_batch(mat.encryption_key, cts)
    return mat, msgs, cts, batch


@pytest.mark.parametrize("B", [1, 2, 4, 8, 16])
def test_heterogeneous_weighted_protocol_round_trips(B):
    mat, msgs, cts, batch = fixture(B, seed=30 + B)
    shares = wp.partial_decrypt_many(mat.party_keys, batch)
    accepted = wp.accept_decryption_shares(mat.decryption_key, batch, shares)
    assert accepted.party_count() == 2 and accepted.accepted_weight() == 7
    assert wp.decrypt(mat.encryption_key, mat.decryption_key, cts, shares) == msgs


def test_non_greedy_authorized_committee():
    mat, msgs, cts, batch = fixture(4)
    shares = wp.partial_decrypt_many([mat.party_keys[0], mat.party_keys[3]], batch)
    accepted = wp.accept_decryption_shares(mat.decryption_key, batch, shares)
    assert accepted.party_indices() == [0, 3] and accepted.accepted_weight() == 5
    kern = wp.CauchyKernel.new(mat.decryption_key)
    pre = wp.prepare_decryption(mat.decryption_key, accepted)
    bp = wp.precompute_batch(kern, pre, batch)
    assert wp.open_batch(mat.decryption_key, kern, pre, accepted, batch, cts, bp) == msgs


def test_malformed_shares_are_blamed_and_authorization_is_weight_based():
    from weighted_bte_b200 import ops

    mat, msgs, cts, batch = fixture(4)
    dk = mat.decryption_key
    shares = wp.partial_decrypt_many(mat.party_keys, batch)
    shares[3].sigma = ops.g1_sum(shares[3].sigma + wb.g1_generator(), [0, 2])
    assert not wp.verify_decryption_share(dk, batch, shares[3])
    assert wp.verify_decryption_share(dk, batch, shares[1])
    accepted = wp.accept_decryption_shares(dk, batch, shares)
    assert accepted.rejected_parties() == [3]
    assert accepted.party_indices() == [1, 2] and accepted.accepted_weight() == 5
    assert wp.decrypt(mat.encryption_key, dk, cts, [s for s in shares if s.party_index != 3]) == msgs
    with pytest.raises(E.InsufficientWeight):
        wp.accept_decryption_shares(dk, batch, [shares[0], shares[2]])


def test_batch_validation_binds_proofs_and_size():
    mat, _, cts, _ = fixture(4)
    bad = list(cts)
    bad[1] = wp.Ciphertext(bad[1].first, bad[1].second, wp.SchnorrProof(bad[1].proof.commitment,
                                                                        (bad[1].proof.response + 1) % wp.R))
    assert not bad[1].verify(mat.encryption_key) and cts[1].verify(mat.encryption_key)
    with pytest.raises(E.InvalidProof):
        wp.validate_batch(mat.encryption_key, bad)
    with pytest.raises(E.MismatchedBatchSize):
        wp.validate_batch(mat.encryption_key, cts[:3])


def test_rejects_invalid_dimensions_and_weights():
    for args, exc in (((3, [1, 2], 1), E.InvalidBatchSize), ((4, [], 0), E.EmptyCommittee),
                      ((4, [1, 0], 0), E.InvalidPartyWeight), ((4, [1, 2], 3), E.InvalidCommittee)):
        with pytest.raises(exc):
            wp.keygen(*args)


def test_key_material_dimensions():
    mat = wp.keygen(8, WEIGHTS, T)
    dk = mat.decryption_key
    assert dk.verification_key_count() == 32 and dk.d1_point_count() == 80 and dk.d2_point_count() == 80
    assert dk.g2_point_count() == 32 + 161 and mat.party_keys[0].scalar_count() == 1
