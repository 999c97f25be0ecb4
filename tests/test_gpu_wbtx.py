"""weighted_btx on the GPU: bit-exact parity with the CPU oracle on the same
seeded inputs, and the reference crate's protocol tests
(weighted_btx/src/decryption.rs:844-1087, setup.rs:531-718) run through the
public API."""
import pytest

from weighted_bte_b200 import errors as E
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu

WEIGHTS, THRESHOLD = [1, 3, 2, 4, 1], 5


def gt_msgs(n, base=17):
    gen = wb.gt_generator()
    from weighted_bte_b200 import ops

    return ops.split(ops.gt_pow(gen, [base + i for i in range(n)], fixed_base=True), 576)


@pytest.fixture(scope="module")
def setup_pair(orc):
    from oracle import wbtx_oracle as W

    mat = wb.keygen_with_rng(wb.KeygenConfig(8, WEIGHTS, THRESHOLD), ChaCha20Rng.seed_from_u64(21))
    key = W.keygen(8, WEIGHTS, THRESHOLD, ChaCha20Rng.seed_from_u64(21))
    return W, mat, key


def test_keygen_matches_oracle(setup_pair):
    W, mat, key = setup_pair
    dk = mat.decryption_key
    assert mat.encryption_key.element() == key["ek"]
    assert dk.domain_points() == key["domain"]
    assert [pk.secret_scalar() for pk in mat.party_keys] == key["qs"]
    assert wb.to_host(dk.verification_keys) == b"".join(key["vk"])
    assert wb.to_host(dk.negative_material) == key["neg_blob"]
    assert wb.to_host(dk.positive_material, 192 * 7 * 11) == key["pos_blob"]
    assert dk.setup_id() == key["setup_id"]


def test_keygen_shapes_and_accessors(setup_pair):
    """weighted_btx/src/setup.rs:531-568, 673-718."""
    _, mat, _ = setup_pair
    dk = mat.decryption_key
    assert dk.party_count() == 5 and dk.total_weight() == 11 and dk.domain_size() == 16
    assert dk.required_weight() == 6
    assert list(dk.party_range(3)) == [6, 7, 8, 9]
    with pytest.raises(E.InvalidPartyIndex):
        dk.party_range(5)
    with pytest.raises(E.InvalidPower):
        dk.verification_key(0, 0)
    with pytest.raises(E.InvalidPower):
        dk.positive_power(8)
    for bad, exc in (((0, [1], 0), E.BatchIsEmpty), ((1, [], 0), E.EmptyCommittee),
                     ((1, [1, 0], 0), E.InvalidPartyWeight), ((1, [2, 1], 3), E.InvalidCommittee)):
        with pytest.raises(exc):
            wb.keygen(*bad)


def test_pipeline_matches_oracle_stage_by_stage(setup_pair):
    W, mat, key = setup_pair
    B, parties = 7, [1, 3]
    msgs = gt_msgs(B)
    cts = wb.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(3))
    octs = W.encrypt_many(key, msgs, ChaCha20Rng.seed_from_u64(3))
    assert [c.first for c in cts] == [c["first"] for c in octs]
    assert [c.second for c in cts] == [c["second"] for c in octs]
    assert [c.proof.response for c in cts] == [c["response"] for c in octs]
    batch = wb.validate_batch(mat.decryption_key, cts)
    obatch = W.validate(key["setup_id"], octs)
    assert batch.valid_mask() == obatch["valid"] and batch.digest() == obatch["digest"]
    shares = wb.partial_decrypt_many([mat.party_keys[j] for j in parties], batch)
    assert [s.sigma for s in shares] == [W.partial_decrypt(key["qs"][j], obatch) for j in parties]
    accepted = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    pre = wb.prepare_decryption(mat.decryption_key, accepted)
    opre = W.prepare(key, parties, B)
    assert wb.to_host(pre.transformed_kernel, 192 * pre.transform_size()) == b"".join(opre["kernel"])
    assert wb.to_host(pre.opening_keys, 192 * B * 2) == b"".join(opre["opening"])
    assert pre.context_id == opre["context_id"]
    cross = wb.precompute_batch(pre, batch)
    obeta = W.precompute(opre, obatch)
    assert wb.to_host(cross.beta, 576 * B) == b"".join(obeta)
    opened = wb.open_batch(pre, accepted, batch, cts, cross)
    assert opened == W.open_batch(opre, [s.sigma for s in shares], obatch, octs, obeta) == msgs


def test_weighted_threshold_end_to_end_with_shuffled_real_parties(setup_pair):
    _, mat, _ = setup_pair
    msgs = gt_msgs(7)
    cts = wb.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(4))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (3, 1)]
    accepted = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    assert accepted.accepted_weight() == 7 and accepted.party_indices() == [1, 3]
    pre = wb.prepare_decryption(mat.decryption_key, accepted)
    cross = wb.precompute_batch(pre, batch)
    assert wb.open_batch(pre, accepted, batch, cts, cross) == msgs


@pytest.mark.parametrize("B", [1, 2, 3, 7, 8])
def test_fft_middle_product_matches_literal_weighted_formula(setup_pair, B):
    W, mat, key = setup_pair
    parties = [1, 2, 3]
    cts = wb.encrypt_many(mat.encryption_key, gt_msgs(B), ChaCha20Rng.seed_from_u64(40 + B))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = wb.partial_decrypt_many([mat.party_keys[j] for j in parties], batch)
    pre = wb.prepare_decryption(mat.decryption_key, wb.accept_decryption_shares(mat.decryption_key, batch, shares))
    fast = wb.to_host(wb.precompute_batch(pre, batch).beta, 576 * B)
    obatch = dict(valid=[True] * B, first=[c.first for c in cts], B=B)
    assert fast == b"".join(W.naive_beta(key, obatch, parties))


def test_fewer_heavy_parties_can_outweigh_more_light_parties(setup_pair):
    _, mat, _ = setup_pair
    ct = wb.encrypt_many(mat.encryption_key, gt_msgs(1), ChaCha20Rng.seed_from_u64(5))
    batch = wb.validate_batch(mat.decryption_key, ct)
    heavy = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 3)]
    wb.accept_decryption_shares(mat.decryption_key, batch, heavy)
    light = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (0, 2, 4)]
    with pytest.raises(E.InsufficientWeight):
        wb.accept_decryption_shares(mat.decryption_key, batch, light)


def test_malformed_share_is_blamed_and_honest_remainder_opens(setup_pair):
    _, mat, _ = setup_pair
    msgs = gt_msgs(4)
    cts = wb.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(6))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 2, 3)]
    from weighted_bte_b200 import ops

    shares[1].sigma = ops.g1_msm(shares[1].sigma + wb.g1_generator(), [1, 1])
    accepted = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    assert accepted.rejected_parties() == [2] and accepted.accepted_weight() == 7
    pre = wb.prepare_decryption(mat.decryption_key, accepted)
    assert wb.open_batch(pre, accepted, batch, cts, wb.precompute_batch(pre, batch)) == msgs


def test_malformed_share_can_drop_set_below_weight_threshold(setup_pair):
    _, mat, _ = setup_pair
    cts = wb.encrypt_many(mat.encryption_key, gt_msgs(1), ChaCha20Rng.seed_from_u64(7))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 2, 4)]
    from weighted_bte_b200 import ops

    shares[0].sigma = ops.g1_msm(shares[0].sigma + wb.g1_generator(), [1, 1])
    with pytest.raises(E.InsufficientWeight) as info:
        wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    assert info.value.rejected_parties == [1]


def test_invalid_client_proof_preserves_slot_and_returns_bottom(setup_pair):
    _, mat, _ = setup_pair
    msgs = gt_msgs(4)
    cts = wb.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(8))
    cts[2].proof.response = (cts[2].proof.response + 1) % wb.R
    batch = wb.validate_batch(mat.decryption_key, cts)
    assert batch.valid_mask() == [True, True, False, True]
    shares = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 3)]
    acc = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    pre = wb.prepare_decryption(mat.decryption_key, acc)
    out = wb.open_batch(pre, acc, batch, cts, wb.precompute_batch(pre, batch))
    assert out == [msgs[0], msgs[1], None, msgs[3]]


def test_entirely_invalid_batch_returns_only_bottom():
    mat = wb.keygen_with_rng(wb.KeygenConfig(4, WEIGHTS, THRESHOLD), ChaCha20Rng.seed_from_u64(9))
    cts = wb.encrypt_many(mat.encryption_key, gt_msgs(3), ChaCha20Rng.seed_from_u64(10))
    for c in cts:
        c.proof.response = (c.proof.response + 1) % wb.R
    batch = wb.validate_batch(mat.decryption_key, cts)
    assert batch.valid_count() == 0
    shares = [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 3)]
    assert all(s.sigma == wb.G1_IDENTITY for s in shares)
    acc = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    pre = wb.prepare_decryption(mat.decryption_key, acc)
    assert wb.open_batch(pre, acc, batch, cts, wb.precompute_batch(pre, batch)) == [None] * 3


def test_one_party_one_weight_one_ciphertext_boundary_opens():
    mat = wb.keygen_with_rng(wb.KeygenConfig(1, [1], 0), ChaCha20Rng.seed_from_u64(11))
    msg = gt_msgs(1, base=99)
    cts = wb.encrypt_many(mat.encryption_key, msg, ChaCha20Rng.seed_from_u64(12))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = [wb.partial_decrypt(mat.party_keys[0], batch)]
    assert wb.verify_decryption_share(mat.decryption_key, batch, shares[0])
    acc = wb.accept_decryption_shares(mat.decryption_key, batch, shares)
    pre = wb.prepare_decryption(mat.decryption_key, acc)
    assert pre.transform_size() == 2
    assert wb.open_batch(pre, acc, batch, cts, wb.precompute_batch(pre, batch)) == msg


def test_phased_objects_are_bound_to_batch_setup_and_committee(setup_pair):
    _, mat, _ = setup_pair
    cts = wb.encrypt_many(mat.encryption_key, gt_msgs(3), ChaCha20Rng.seed_from_u64(13))
    batch = wb.validate_batch(mat.decryption_key, cts)
    acc_a = wb.accept_decryption_shares(mat.decryption_key, batch,
                                        [wb.partial_decrypt(mat.party_keys[j], batch) for j in (1, 3)])
    pre_a = wb.prepare_decryption(mat.decryption_key, acc_a)
    cross_a = wb.precompute_batch(pre_a, batch)
    acc_b = wb.accept_decryption_shares(mat.decryption_key, batch,
                                        [wb.partial_decrypt(mat.party_keys[j], batch) for j in (0, 2, 3)])
    pre_b = wb.prepare_decryption(mat.decryption_key, acc_b)
    with pytest.raises(E.MismatchedCommittee):
        wb.open_batch(pre_b, acc_b, batch, cts, cross_a)
    changed = list(cts)
    changed[0] = wb.Ciphertext(cts[0].first, cts[1].second, cts[0].proof)
    with pytest.raises(E.MismatchedBatchDigest):
        wb.open_batch(pre_a, acc_a, batch, changed, cross_a)
    other = wb.keygen_with_rng(wb.KeygenConfig(8, WEIGHTS, THRESHOLD), ChaCha20Rng.seed_from_u64(99))
    assert other.decryption_key.setup_id() != mat.decryption_key.setup_id()
    with pytest.raises(E.MismatchedSetup):
        wb.prepare_decryption(other.decryption_key, acc_a)
    with pytest.raises(E.MismatchedSetup):
        wb.partial_decrypt(other.party_keys[1], batch)
    batch_other = wb.validate_batch(other.decryption_key, cts)
    assert batch_other.valid_count() == 0


def test_oversized_and_duplicate_inputs_are_rejected():
    mat = wb.keygen_with_rng(wb.KeygenConfig(1, WEIGHTS, THRESHOLD), ChaCha20Rng.seed_from_u64(14))
    cts = wb.encrypt_many(mat.encryption_key, gt_msgs(2), ChaCha20Rng.seed_from_u64(15))
    with pytest.raises(E.BatchTooLarge):
        wb.validate_batch(mat.decryption_key, cts)
    batch = wb.validate_batch(mat.decryption_key, cts[:1])
    share = wb.partial_decrypt(mat.party_keys[1], batch)
    with pytest.raises(E.TooManyShares):
        wb.accept_decryption_shares(mat.decryption_key, batch, [share] * 6)
    with pytest.raises(E.DuplicatePartyIndex):
        wb.accept_decryption_shares(mat.decryption_key, batch, [share, share])


def test_decrypt_wrapper_round_trip(setup_pair):
    _, mat, _ = setup_pair
    msgs = gt_msgs(5, base=1000)
    cts = wb.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(16))
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = wb.partial_decrypt_many([mat.party_keys[j] for j in (0, 1, 3)], batch)
    assert wb.decrypt(mat.decryption_key, cts, shares) == msgs
