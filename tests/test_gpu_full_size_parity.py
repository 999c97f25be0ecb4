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
