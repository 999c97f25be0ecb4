"""The served weighted_pfe form on the GPU: requests of mixed sizes through
serving.DecryptionServer with wpfe_batched.WpfeBackend (power-of-two classes,
dummy padding, continuous batching of same-class requests).  Every result
must equal the same request decrypted alone and its plaintexts
(weighted_pfe/src/decryption.rs:646-669)."""
import concurrent.futures as cf

import pytest

from weighted_bte_b200 import errors as E
from weighted_bte_b200 import ops
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200 import weighted_pfe as wp
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu


def gt_msgs(n, base):
    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def test_served_requests_equal_alone_and_in_the_mix():
    from weighted_bte_b200 import serving
    from weighted_bte_b200 import wpfe_batched as wpb
    from weighted_bte_b200.workloads import minimal_authorized_parties, pareto_weights

    weights = pareto_weights(12, 48, seed=9)
    t = 48 // 3
    committee, _ = minimal_authorized_parties(weights, t)
    sizes = [3, 17, 9, 32, 5, 12, 30, 1, 16, 7, 25, 4, 11, 2, 19, 8]
    classes = wpb.class_keys([wpb.size_class(s) for s in sizes], weights, t, committee, seed=21)
    rng = ChaCha20Rng.seed_from_u64(22)
    msgs, reqs = [], []
    for k, s in enumerate(sizes):
        m = gt_msgs(s, 31 * k + 5)
        msgs.append(m)
        reqs.append(wp.encrypt_many(classes[wpb.size_class(s)].material.encryption_key, m, rng))
    # one request with a broken proof: rejected alone, the others unaffected
    bad_i = 5
    c = reqs[bad_i][2]
    reqs[bad_i][2] = wp.Ciphertext(c.first, c.second, wb.SchnorrProof(c.proof.commitment,
                                                                      (c.proof.response + 3) % ops.R))
    backend = wpb.WpfeBackend(classes)
    with serving.DecryptionServer(backend=backend, slots=3, max_group=4) as srv:
        futs = [srv.submit(r, classes[wpb.size_class(len(r))].party_keys, seed=k) for k, r in enumerate(reqs)]
        mix = []
        for f in futs:
            try:
                mix.append(f.result())
            except E.Error as exc:
                mix.append(exc)
        st = srv.stats()
    assert st["requests"] == len(sizes)
    for k, s in enumerate(sizes):
        sc = classes[wpb.size_class(s)]
        alone = wpb.decrypt_group(sc.material.encryption_key, sc.material.decryption_key, [sc.pad(reqs[k])],
                                  sc.party_keys, ChaCha20Rng.seed_from_u64(k))[0]
        if k == bad_i:
            assert isinstance(mix[k], E.InvalidProof) and isinstance(alone, E.InvalidProof)
            continue
        assert mix[k] == alone[:s] == msgs[k], f"request {k}"


def test_committee_of_more_than_eight_parties_matches_unprepared_pairings():
    """Ten unit-weight parties (t = 9) open with chunked multi-Miller loops
    over their line tables; the result equals T unprepared loops per slot."""
    B, K = 4, 2
    weights = [1] * 12
    t = 9
    rng = ChaCha20Rng.seed_from_u64(31)
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, weights, t), rng)
    ek, dk = mat.encryption_key, mat.decryption_key
    msgs = [gt_msgs(B, 70 * (k + 1)) for k in range(K)]
    batches = [wp.encrypt_many(ek, m, rng) for m in msgs]
    vb = [wp.validate_batch(ek, cts) for cts in batches]
    keys = mat.party_keys[:10]
    shares = wp.partial_decrypt_batches(keys, vb)
    acc = [wp.accept_decryption_shares(dk, vb[b], shares[b], ChaCha20Rng.seed_from_u64(b)) for b in range(K)]
    assert acc[0].party_count() == 10
    pre = wp.prepare_decryption(dk, acc[0])
    T = 10
    lines = wb.empty_device(288 * 68 * B * T)
    wb._ctx().call("wbte_g2_prepare_lines", lines, pre.scaled_d1_by_party, B * T)
    torch = wb._t()
    first = torch.cat([v.first_dev[: 96 * B] for v in vb])
    second = b"".join(c.second for cts in batches for c in cts)
    sig = b"".join(s.sigma for a in acc for s in a.shares())
    ap = ops.scalars_bytes([a * (a + 1) % ops.R for a in dk.alpha_points()])
    outs = []
    for by_lines in (None, lines):
        out = bytearray(576 * B * K)
        wb._ctx().call("wbte_wpfe_decrypt_many", out, sig, T, pre.scaled_d1_by_party, by_lines, pre.total_lines,
                       pre.mask_lines, first, second, ap, B, K)
        outs.append(bytes(out))
    assert outs[0] == outs[1] == b"".join(b"".join(m) for m in msgs)


def test_weighted_btx_opening_with_more_than_eight_parties():
    """weighted_btx's batched opening over the line tables of 10 parties'
    opening keys equals the unprepared opening."""
    from weighted_bte_b200 import serving

    B = 4
    weights = [1] * 12
    t = 9
    rng = ChaCha20Rng.seed_from_u64(41)
    mat = wb.keygen_with_rng(wb.KeygenConfig(B, weights, t), rng)
    dk = mat.decryption_key
    keys = mat.party_keys[:10]
    groups = []
    msgs = []
    for k in range(3):
        m = gt_msgs(B, 90 * (k + 1))
        msgs.append(m)
        groups.append(wb.encrypt_many(mat.encryption_key, m, rng))
    out = serving.decrypt_group(dk, groups, keys, ChaCha20Rng.seed_from_u64(1))
    one = [serving.decrypt_request(dk, cts, keys, ChaCha20Rng.seed_from_u64(2)) for cts in groups]
    assert out == one == msgs
