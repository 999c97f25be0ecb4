"""btx on the GPU: bit-exact parity with the CPU restatement on the same
seeded inputs (config: B=32, N=16, t=8, seed 0, and small cases), and the
reference crate's protocol tests (btx/src/decryption.rs:540-712,
setup.rs:281-309, encryption.rs:58-66) through the public API."""
import pytest

from weighted_bte_b200 import btx
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu


def gt_msgs(n, base=17):
    from weighted_bte_b200 import ops

    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def as_oracle_cts(cts):
    return [dict(first=c.first, second=c.second, commitment=c.proof.commitment, response=c.proof.response)
            for c in cts]


@pytest.mark.parametrize("L,N,t,B,seed", [(8, 5, 2, 5, 7), (32, 16, 8, 32, 0)])
def test_pipeline_matches_oracle_stage_by_stage(orc, L, N, t, B, seed):
    from oracle import btx_oracle as X

    mat = btx.keygen_with_rng(btx.KeygenConfig(L, N, t), ChaCha20Rng.seed_from_u64(seed))
    key = X.keygen(L, N, t, ChaCha20Rng.seed_from_u64(seed))
    dk = mat.decryption_key
    assert wb.to_host(dk.low_powers, 192 * L) == key["low"]
    assert wb.to_host(dk.high_powers, 192 * (L - 1)) == key["high"]
    assert [k.shares for k in mat.server_keys] == key["shares"]
    assert wb.to_host(dk.share_commitments) == b"".join(key["commitments"])
    assert mat.encryption_key.element == key["ek"]

    rng = ChaCha20Rng.seed_from_u64(seed + 1000)
    msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
    cts = btx.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    octs = X.encrypt_many(key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    assert as_oracle_cts(cts) == octs
    if B > 2:  # one broken proof
        cts[2] = btx.Ciphertext(cts[2].first, cts[2].second,
                                btx.SchnorrProof(cts[2].proof.commitment, (cts[2].proof.response + 1) % btx.R))
        octs[2] = dict(octs[2], response=(octs[2]["response"] + 1) % btx.R)
    batch = btx.validate_batch(cts)
    obatch = X.validate(octs)
    assert batch.valid_mask() == obatch["valid"] and batch.digest() == obatch["digest"]

    kern = btx.MiddleProductKernel.new(dk, B)
    okern = X.kernel(key, B)
    assert wb.to_host(kern.transformed_kernel, 192 * kern.transform_size()) == b"".join(okern["kernel"])
    pre = btx.precompute_batch(kern, batch)
    beta = X.precompute(okern, obatch)
    assert wb.to_host(pre.beta, 576 * B) == b"".join(beta)

    servers = list(range(t + 1))
    shares = [btx.partial_decrypt(mat.server_keys[j], batch) for j in servers]
    assert [s.sigma for s in shares] == [X.partial_decrypt(key, j, obatch) for j in servers]
    sigma = btx.combine_shares(dk, batch, shares)
    assert sigma == X.combine(key, [(j, s.sigma) for j, s in zip(servers, shares)])
    assert btx.verify_combined_share(dk, batch, sigma)
    assert all(btx.verify_decryption_share(dk, batch, s) for s in shares[:2])
    out = btx.open_batch(kern, batch, cts, pre, sigma)
    assert out == X.open_batch(okern, obatch, octs, beta, sigma)
    assert out == [m if v else None for m, v in zip(msgs, batch.valid_mask())]


def fixture(L, B, seed=3):
    mat = btx.keygen_with_rng(btx.KeygenConfig(L, 5, 2), ChaCha20Rng.seed_from_u64(seed))
    msgs = gt_msgs(B)
    cts = btx.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 1))
    batch = btx.ValidatedBatch.verify(cts)
    kern = btx.MiddleProductKernel.new(mat.decryption_key, B)
    return mat, msgs, cts, batch, kern


@pytest.mark.parametrize("B", [1, 2, 3, 7, 8, 15])
def test_fft_middle_product_matches_quadratic_formula(orc, B):
    from oracle import btx_oracle as X

    mat, _, cts, batch, kern = fixture(16, B, seed=50 + B)
    fast = btx.precompute_batch(kern, batch)
    dk = mat.decryption_key
    key = dict(L=16, low=wb.to_host(dk.low_powers, 192 * 16), high=wb.to_host(dk.high_powers, 192 * 15))
    slow = X.naive_beta(key, X.validate(as_oracle_cts(cts)))
    assert wb.to_host(fast.beta, 576 * B) == b"".join(slow)


def test_threshold_end_to_end():
    mat, msgs, cts, batch, kern = fixture(16, 8)
    pre = btx.precompute_batch(kern, batch)
    shares = [btx.partial_decrypt(k, batch) for k in mat.server_keys[:3]]
    for s in shares:
        assert btx.verify_decryption_share(mat.decryption_key, batch, s)
    sigma = btx.combine_shares(mat.decryption_key, batch, shares)
    assert btx.verify_combined_share(mat.decryption_key, batch, sigma)
    assert btx.open_batch(kern, batch, cts, pre, sigma) == msgs
    assert btx.decrypt(mat.decryption_key, cts, mat.server_keys[:3], kern) == msgs


def test_invalid_proof_preserves_slot_and_returns_bottom():
    mat, msgs, cts, _, kern = fixture(16, 8)
    cts[3] = btx.Ciphertext(cts[3].first, cts[3].second,
                            btx.SchnorrProof(cts[3].proof.commitment, (cts[3].proof.response + 1) % btx.R))
    batch = btx.ValidatedBatch.verify(cts)
    assert not batch.valid_mask()[3]
    pre = btx.precompute_batch(kern, batch)
    shares = [btx.partial_decrypt(k, batch) for k in mat.server_keys[:3]]
    sigma = btx.combine_shares(mat.decryption_key, batch, shares)
    out = btx.open_batch(kern, batch, cts, pre, sigma)
    assert out == [None if i == 3 else m for i, m in enumerate(msgs)]


def test_entirely_invalid_batch_returns_only_bottom():
    mat, _, cts, _, kern = fixture(8, 4)
    cts = [btx.Ciphertext(c.first, c.second, btx.SchnorrProof(c.proof.commitment, (c.proof.response + 1) % btx.R))
           for c in cts]
    batch = btx.ValidatedBatch.verify(cts)
    assert batch.valid_count() == 0
    pre = btx.precompute_batch(kern, batch)
    shares = [btx.partial_decrypt(k, batch) for k in mat.server_keys[:3]]
    sigma = btx.combine_shares(mat.decryption_key, batch, shares)
    assert sigma == btx.G1_IDENTITY
    assert btx.verify_combined_share(mat.decryption_key, batch, sigma)
    assert btx.open_batch(kern, batch, cts, pre, sigma) == [None] * 4


def test_shuffled_server_subset_reconstructs():
    mat, msgs, cts, batch, kern = fixture(8, 4)
    pre = btx.precompute_batch(kern, batch)
    shares = [btx.partial_decrypt(mat.server_keys[i], batch) for i in (4, 1, 3)]
    sigma = btx.combine_shares(mat.decryption_key, batch, shares)
    assert btx.open_batch(kern, batch, cts, pre, sigma) == msgs


def test_corrupted_share_fails_verification():
    from weighted_bte_b200 import ops

    mat, _, _, batch, _ = fixture(8, 4)
    share = btx.partial_decrypt(mat.server_keys[0], batch)
    share.sigma = ops.g1_sum(share.sigma + wb.g1_generator(), [0, 2])
    assert not btx.verify_decryption_share(mat.decryption_key, batch, share)


def test_checked_combine_excludes_a_corrupted_share():
    from weighted_bte_b200 import ops

    mat, msgs, cts, batch, kern = fixture(8, 4)
    pre = btx.precompute_batch(kern, batch)
    shares = [btx.partial_decrypt(k, batch) for k in mat.server_keys[:4]]
    shares[0].sigma = ops.g1_sum(shares[0].sigma + wb.g1_generator(), [0, 2])
    assert not btx.verify_combined_share(mat.decryption_key, batch, btx.combine_shares(mat.decryption_key, batch, shares))
    sigma = btx.combine_shares_checked(mat.decryption_key, batch, shares)
    assert btx.open_batch(kern, batch, cts, pre, sigma) == msgs


def test_rejects_duplicate_and_insufficient_shares():
    mat, _, _, batch, _ = fixture(8, 4)
    share = btx.partial_decrypt(mat.server_keys[0], batch)
    with pytest.raises(btx.InsufficientShares):
        btx.combine_shares(mat.decryption_key, batch, [share])
    with pytest.raises(btx.DuplicateServerIndex) as e:
        btx.combine_shares(mat.decryption_key, batch, [share, share, share])
    assert e.value.index == 0


def test_key_material_shapes_and_invalid_committee():
    mat = btx.keygen(16, 5, 2)
    dk = mat.decryption_key
    assert mat.encryption_key.max_batch_size == 16 and dk.low_powers.numel() == 192 * 16
    assert dk.high_powers.numel() == 192 * 15 and len(mat.server_keys) == 5
    assert len(mat.server_keys[0].shares) == 16 and dk.has_share_commitments()
    with pytest.raises(btx.InvalidBatchSize):
        dk.power(17)
    with pytest.raises(btx.InvalidCommittee):
        btx.keygen(8, 3, 3)


def test_encryption_proof_verifies():
    mat = btx.keygen(8, 3, 1)
    ct = btx.encrypt(mat.encryption_key, gt_msgs(1, 42)[0])
    assert ct.verify()
