"""The batched weighted_pfe form on the GPU: K batches per launch sequence
(wbte_wpfe_*_many) and uneven batch sizes padded to power-of-two classes.

Every batch decrypted in a group must equal the same batch decrypted alone
by the single-batch path (weighted_pfe/src/decryption.rs:646-669) and open
to its plaintexts."""
import pytest

from weighted_bte_b200 import errors as E
from weighted_bte_b200 import ops
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200 import weighted_pfe as wp
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu

WEIGHTS, T = [1, 3, 2, 4], 4
COMMITTEE = [3, 1]  # heaviest first, weight 7 > 4


def gt_msgs(n, base):
    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def test_many_entry_points_match_the_single_batch_calls():
    B, K = 8, 3
    rng = ChaCha20Rng.seed_from_u64(71)
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, WEIGHTS, T), rng)
    ek, dk = mat.encryption_key, mat.decryption_key
    msgs = [gt_msgs(B, 100 * (k + 1)) for k in range(K)]
    batches = [wp.encrypt_many(ek, m, rng) for m in msgs]
    validated = wp.validate_batches(ek, batches, ChaCha20Rng.seed_from_u64(5))
    alone = [wp.validate_batch(ek, cts) for cts in batches]
    assert [v.digest() for v in validated] == [a.digest() for a in alone]
    keys = [mat.party_keys[j] for j in sorted(COMMITTEE)]
    many = wp.partial_decrypt_batches(keys, validated)
    for b in range(K):
        assert [s.sigma for s in many[b]] == [s.sigma for s in wp.partial_decrypt_many(keys, alone[b])]
    acc = [wp.accept_decryption_shares(dk, alone[b], many[b], ChaCha20Rng.seed_from_u64(b)) for b in range(K)]
    pre = wp.prepare_decryption(dk, acc[0])
    kernel = wp.CauchyKernel(dk)
    singles = [wp.precompute_batch(kernel, pre, alone[b]) for b in range(K)]
    torch = wb._t()
    first = torch.cat([v.first_dev[: 96 * B] for v in validated])
    fc, pc = wb.empty_device(96 * B * K), wb.empty_device(576 * B * K)
    wb._ctx().call("wbte_wpfe_precompute_many", fc, pc, first, pre.total_lines, B, K)
    for b in range(K):
        assert wb.to_host(fc)[96 * B * b : 96 * B * (b + 1)] == wb.to_host(singles[b].scaled_first_cauchy, 96 * B)
        hard_many = ops.final_exp(wb.to_host(pc)[576 * B * b : 576 * B * (b + 1)], mode=2)
        hard_one = ops.final_exp(wb.to_host(singles[b].pairing_cauchy, 576 * B), mode=2)
        assert hard_many == hard_one
    # open_many without and with the per-party line tables, and the fused call
    alpha = dk.alpha_points()
    ap = ops.scalars_bytes([a * (a + 1) % ops.R for a in alpha])
    second = b"".join(c.second for cts in batches for c in cts)
    sig = b"".join(s.sigma for a in acc for s in a.shares())
    Ta = acc[0].party_count()
    lines = wb.empty_device(288 * 68 * B * Ta)
    wb._ctx().call("wbte_g2_prepare_lines", lines, pre.scaled_d1_by_party, B * Ta)
    outs = []
    for by_lines in (None, lines):
        out = bytearray(576 * B * K)
        wb._ctx().call("wbte_wpfe_open_many", out, sig, Ta, pre.scaled_d1_by_party, by_lines, first, pre.mask_lines,
                       fc, pc, second, ap, B, K)
        outs.append(bytes(out))
    fused = bytearray(576 * B * K)
    wb._ctx().call("wbte_wpfe_decrypt_many", fused, sig, Ta, pre.scaled_d1_by_party, lines, pre.total_lines,
                   pre.mask_lines, first, second, ap, B, K)
    expect = b"".join(b"".join(m) for m in msgs)
    assert outs[0] == outs[1] == bytes(fused) == expect
    for b in range(K):
        single = wp.open_batch(dk, kernel, pre, acc[b], alone[b], batches[b], singles[b])
        assert b"".join(single) == b"".join(msgs[b])


def test_group_equals_each_batch_alone_and_isolates_a_bad_batch():
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.serving import CommitteeCache

    B, K = 8, 4
    rng = ChaCha20Rng.seed_from_u64(72)
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, WEIGHTS, T), rng)
    ek, dk = mat.encryption_key, mat.decryption_key
    msgs = [gt_msgs(B, 1000 * (k + 1)) for k in range(K)]
    batches = [wp.encrypt_many(ek, m, rng) for m in msgs]
    # batch 2 carries a ciphertext with a wrong proof response: weighted_pfe
    # rejects that whole batch, and only that batch
    bad = batches[2][3]
    batches[2][3] = wp.Ciphertext(bad.first, bad.second, wb.SchnorrProof(bad.proof.commitment,
                                                                         (bad.proof.response + 1) % ops.R))
    keys = [mat.party_keys[j] for j in range(len(WEIGHTS))]
    cache = CommitteeCache(1 << 30)
    for _ in range(2):  # the second round takes the cached committee
        out = wpb.decrypt_group(ek, dk, batches, keys, ChaCha20Rng.seed_from_u64(9), cache)
        for b in range(K):
            if b == 2:
                assert isinstance(out[b], E.InvalidProof)
                with pytest.raises(E.InvalidProof):
                    wp.validate_batch(ek, batches[b])
                continue
            shares = wp.partial_decrypt_many(keys, wp.validate_batch(ek, batches[b]))
            alone = wp.decrypt(ek, dk, batches[b], shares, ChaCha20Rng.seed_from_u64(b))
            assert out[b] == alone == msgs[b]
    assert cache.hits >= 1


def test_group_blames_a_dishonest_party_and_decrypts_every_batch():
    from weighted_bte_b200 import wpfe_batched as wpb

    B, K = 4, 3
    rng = ChaCha20Rng.seed_from_u64(73)
    weights = [4, 3, 3, 2]
    t = 5
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, weights, t), rng)
    ek, dk = mat.encryption_key, mat.decryption_key
    msgs = [gt_msgs(B, 50 * (k + 1)) for k in range(K)]
    batches = [wp.encrypt_many(ek, m, rng) for m in msgs]

    class Liar:
        """Party 0's key with a wrong secret: its shares fail the check."""

        def __init__(self, pk):
            self.__dict__.update(pk.__dict__)
            self.rho = (pk.rho + 1) % ops.R

        def setup_id(self):
            return self._setup_id

        def batch_size(self):
            return self._batch_size

    keys = [Liar(mat.party_keys[0])] + mat.party_keys[1:]
    out = wpb.decrypt_group(ek, dk, batches, keys, ChaCha20Rng.seed_from_u64(3))
    for b in range(K):
        assert out[b] == msgs[b]


def test_uneven_batches_alone_and_in_the_mix_with_the_autotuner(tmp_path):
    from weighted_bte_b200 import autotune
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.workloads import minimal_authorized_parties, zipf_weights

    weights = zipf_weights(8, 24)
    t = 8
    committee, _ = minimal_authorized_parties(weights, t)
    sizes = [3, 5, 8, 2, 16, 9, 1, 12, 7, 4, 16, 6]
    classes = wpb.class_keys([wpb.size_class(s) for s in sizes], weights, t, committee, seed=11)
    rng = ChaCha20Rng.seed_from_u64(12)
    msgs, batches = [], []
    for k, s in enumerate(sizes):
        m = gt_msgs(s, 7 * k + 3)
        msgs.append(m)
        batches.append(wp.encrypt_many(classes[wpb.size_class(s)].material.encryption_key, m, rng))
    tuner = autotune.Autotuner(str(tmp_path / "tune.json"), trial_batches=2)
    dec = wpb.UnevenBatchDecryptor(classes, streams=3, tuner=tuner)
    mix = dec.decrypt(batches, seed=5)
    for b, s in enumerate(sizes):
        sc = classes[wpb.size_class(s)]
        padded = sc.pad(batches[b])
        mat = sc.material
        shares = wp.partial_decrypt_many(sc.party_keys, wp.validate_batch(mat.encryption_key, padded))
        alone = wp.decrypt(mat.encryption_key, mat.decryption_key, padded, shares)
        assert mix[b] == alone[:s] == msgs[b]
    # the tuned knobs were cached, and a fresh tuner reads them back
    again = autotune.Autotuner(str(tmp_path / "tune.json"))
    for B in classes:
        assert again.lookup("wpfe", B, len(committee)) is not None


def test_batched_configuration_256_uneven_batches_alone_and_in_the_mix(tmp_path):
    """256 batches with sizes log-uniform in [8, 2048] (seed 3) padded to
    powers of two, n = 64 parties with Zipf(1) weights W = 2048, t = W/3:
    every batch decrypted in the mix equals its plaintexts and the same batch
    decrypted alone (a group of one against the same cached committee)."""
    from weighted_bte_b200 import autotune
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.workloads import WPFE_BATCHED as cfg
    from weighted_bte_b200.workloads import minimal_authorized_parties

    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    sizes = cfg.sizes()
    classes = wpb.class_keys([wpb.size_class(s) for s in sizes], cfg.weights, cfg.threshold, committee, cfg.seed)
    rng = ChaCha20Rng.seed_from_u64(cfg.seed)
    msgs, batches = [], []
    for s in sizes:
        m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(s)])
        msgs.append(m)
        batches.append(wp.encrypt_many(classes[wpb.size_class(s)].material.encryption_key, m, rng))
    dec = wpb.UnevenBatchDecryptor(classes, streams=4, tuner=autotune.Autotuner(str(tmp_path / "t.json")))
    mix = dec.decrypt(batches, seed=1)
    for b, s in enumerate(sizes):
        assert mix[b] == msgs[b], f"batch {b} (size {s})"
    # alone: each batch as a group of one on the same cached committees
    for b, s in enumerate(sizes):
        sc = classes[wpb.size_class(s)]
        one = wpb.decrypt_group(sc.material.encryption_key, sc.material.decryption_key, [sc.pad(batches[b])],
                                sc.party_keys, ChaCha20Rng.seed_from_u64(b), dec.cache)[0]
        assert one[:s] == mix[b], f"batch {b} alone"
