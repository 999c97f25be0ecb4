"""weighted_btx at the benchmark's own shape (B = 512, n = 128 Zipf(1)
weights, W = 4096, t = W/3, heaviest-first committee): every stage of the
decryption compared byte for byte with the CPU oracle on the same inputs.

The oracle's keygen and committee preparation at this size take minutes on
the host, so the key material and the prepared committee come from the GPU
library (both are held byte-identical to the oracle's at small sizes by
test_gpu_wbtx.py); here the committee's opening keys are spot-checked
against the oracle's G2 MSMs, and validation, the partial decryptions, the
aggregate share check, the cross terms (the transform of m = 1024 points,
1,024 pairings, the truncated cyclotomic inverse transform and the hard
parts) and the opening are recomputed by the oracle in full."""
import random

import pytest

from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng
from weighted_bte_b200.workloads import WBTX_B512, minimal_authorized_parties

pytestmark = pytest.mark.gpu


def test_weighted_btx_benchmark_shape_matches_oracle_stage_by_stage(orc):
    from oracle import wbtx_oracle as W

    cfg = WBTX_B512
    B = cfg.batch_size
    rng = ChaCha20Rng.seed_from_u64(77)
    mat = wb.keygen_with_rng(wb.KeygenConfig(B, cfg.weights, cfg.threshold), rng)
    dk = mat.decryption_key
    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    parties = sorted(committee)
    N, T = dk.party_count(), len(parties)
    threads = orc.num_threads()
    vk = wb.to_host(dk.verification_keys, 192 * B * N)
    key = dict(N=N, vk=[vk[192 * i : 192 * (i + 1)] for i in range(B * N)], setup_id=dk.setup_id())

    msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
    cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
    bad = cts[100]  # one slot with a broken proof opens to nothing
    cts[100] = wb.Ciphertext(bad.first, bad.second, wb.SchnorrProof(bad.proof.commitment,
                                                                     (bad.proof.response + 1) % wb.R))
    octs = [dict(first=c.first, second=c.second, commitment=c.proof.commitment, response=c.proof.response)
            for c in cts]

    batch = wb.validate_batch(dk, cts)
    obatch = W.validate(key["setup_id"], octs, threads)
    assert batch.valid_mask() == obatch["valid"] and batch.digest() == obatch["digest"]
    assert obatch["valid"].count(False) == 1

    keys = [mat.party_keys[j] for j in parties]
    shares = wb.partial_decrypt_many(keys, batch)
    sig = [s.sigma for s in shares]
    assert sig == [W.partial_decrypt(k.secret_scalar(), obatch) for k in keys]

    challenges = [W.sample_nonzero(rng) for _ in parties]
    assert wb._verify_shares(dk, batch, shares, challenges)
    assert W.verify_shares(key, obatch, parties, sig, challenges, threads)

    accepted = wb.accept_decryption_shares(dk, batch, shares, rng)
    pre = wb.prepare_decryption(dk, accepted)
    m = wb.transform_size_for(B)
    kern = wb.to_host(pre.transformed_kernel, 192 * m)
    opening = wb.to_host(pre.opening_keys, 192 * B * T)
    opre = dict(kernel=[kern[192 * i : 192 * (i + 1)] for i in range(m)],
                opening=[opening[192 * i : 192 * (i + 1)] for i in range(B * T)], m=m, B=B)

    # opening keys of four slots against the oracle's MSMs of the committee's
    # negative material with the Lagrange coefficients at zero of its
    # virtual parties (weighted_btx/src/decryption.rs:463-481)
    selected = [w for j in parties for w in dk.party_range(j)]
    domain = dk.domain_points()
    lam = orc.lagrange_at_zero([domain[w] for w in selected])
    coef = dict(zip(selected, lam))
    for slot in random.Random(5).sample(range(B), 4):
        neg = dk.negative_power(slot + 1)
        expect_keys = [orc.g2_msm([neg[w] for w in dk.party_range(j)], [coef[w] for w in dk.party_range(j)])
                       for j in parties]
        assert opre["opening"][slot * T : (slot + 1) * T] == expect_keys

    cross = wb.precompute_batch(pre, batch)
    obeta = W.precompute(opre, obatch)
    assert wb.to_host(cross.beta, 576 * B) == b"".join(obeta)

    opened = wb.open_batch(pre, accepted, batch, cts, cross)
    expect = [mm if v else None for mm, v in zip(msgs, obatch["valid"])]
    assert opened == W.open_batch(opre, sig, obatch, octs, obeta) == expect


def test_weighted_pfe_b512_matches_oracle_stage_by_stage(orc):
    """weighted_pfe at B = 512 (the config-4 class of 512 slots), every stage
    against the oracle: key material, encryption, validation, partial
    decryptions, committee preparation, the Cauchy cross terms (compared
    after the hard part, where they are canonical) and the opened messages."""
    from oracle import wpfe_oracle as X
    from weighted_bte_b200 import ops
    from weighted_bte_b200 import weighted_pfe as wp

    B, weights, t, seed = 512, [1, 3, 2, 4], 4, 6
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, weights, t), ChaCha20Rng.seed_from_u64(seed))
    key = X.keygen(B, weights, t, ChaCha20Rng.seed_from_u64(seed))
    dk = mat.decryption_key
    assert dk.alpha_points() == key["alpha"] and dk.domain_points() == key["eval_domain"]
    assert wb.to_host(dk.verification_keys) == key["vk"]
    assert wb.to_host(dk.d1) == key["d1"] and wb.to_host(dk.d2) == key["d2"]
    assert dk.setup_id() == key["setup_id"]

    msgs = ops.split(ops.gt_pow(wb.gt_generator(), [11 + i for i in range(B)], fixed_base=True), 576)
    cts = wp.encrypt_many(mat.encryption_key, msgs, ChaCha20Rng.seed_from_u64(seed + 100))
    octs = X.encrypt_many(key, msgs, ChaCha20Rng.seed_from_u64(seed + 100))
    assert [dict(first=c.first, second=c.second, commitment=c.proof.commitment, response=c.proof.response)
            for c in cts] == octs
    batch = wp.validate_batch(mat.encryption_key, cts)
    obatch = X.validate(key, octs)
    assert batch.digest() == obatch["digest"]

    shares = wp.partial_decrypt_many(mat.party_keys, batch)
    assert [s.sigma for s in shares] == [X.partial_decrypt(key, j, obatch) for j in range(len(weights))]
    accepted = wp.accept_decryption_shares(dk, batch, shares, ChaCha20Rng.seed_from_u64(1))
    parties = accepted.party_indices()
    assert parties == X.select_committee(key, range(len(weights)))
    pre = wp.prepare_decryption(dk, accepted)
    opre = X.prepare(key, parties)
    assert wb.to_host(pre.scaled_d1_by_party) == b"".join(opre["by_party"])
    assert wb.to_host(pre.scaled_d1_total) == b"".join(opre["total"])
    assert wb.to_host(pre.mask_keys) == b"".join(opre["mask"])

    kern = wp.CauchyKernel.new(dk)
    bp = wp.precompute_batch(kern, pre, batch)
    obp = X.precompute(key, opre, obatch)
    assert wb.to_host(bp.scaled_first_cauchy, 96 * B) == b"".join(obp["first_cauchy"])
    got_pc = ops.split(ops.final_exp(wb.to_host(bp.pairing_cauchy, 576 * B), mode=2), 576)
    assert got_pc == orc.hard_final_exp_many(obp["pairing_cauchy"])

    out = wp.open_batch(dk, kern, pre, accepted, batch, cts, bp)
    assert out == X.open_batch(key, opre, [shares[j].sigma for j in parties], obatch, octs, obp) == msgs
