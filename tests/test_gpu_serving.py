"""Served and batched decryption: every request's result is byte-identical
whether it runs alone (the plain `decrypt` path) or in a mix of concurrent
requests of different batch sizes and committees, with and without the
committee cache, and admission respects the HBM budget."""
import numpy as np
import pytest

from weighted_bte_b200 import serving
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu

WEIGHTS, THRESHOLD, MAX_BATCH = [1, 3, 2, 4, 1], 5, 8


@pytest.fixture(scope="module")
def mix():
    mat = wb.keygen_with_rng(wb.KeygenConfig(MAX_BATCH, WEIGHTS, THRESHOLD), ChaCha20Rng.seed_from_u64(41))
    rng = ChaCha20Rng.seed_from_u64(42)
    # (batch size, committee): uneven sizes, two committees, repeated contexts
    shapes = [(8, [1, 3]), (3, [1, 3]), (5, [0, 2, 3]), (8, [1, 3]), (1, [3, 4, 0]), (6, [0, 2, 3]), (8, [1, 3])]
    reqs = []
    for B, parties in shapes:
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
        cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
        keys = [mat.party_keys[j] for j in sorted(parties)]
        reqs.append((cts, keys, msgs))
    # one ciphertext with a broken proof: its slot decrypts to None
    cts, keys, msgs = reqs[2]
    bad = cts[1]
    cts[1] = wb.Ciphertext(bad.first, bad.second, wb.SchnorrProof(bad.proof.commitment, (bad.proof.response + 1) % wb.R))
    return mat, reqs


def alone(mat, cts, keys):
    batch = wb.validate_batch(mat.decryption_key, cts)
    shares = wb.partial_decrypt_many(keys, batch)
    return wb.decrypt(mat.decryption_key, cts, shares, ChaCha20Rng.seed_from_u64(5))


def test_results_identical_alone_and_in_the_mix(mix):
    mat, reqs = mix
    solo = [alone(mat, cts, keys) for cts, keys, _ in reqs]
    for (cts, _, msgs), out in zip(reqs, solo):
        assert [o for o in out if o is not None] == [m for m, o in zip(msgs, out) if o is not None]
    assert solo[2][1] is None and sum(o is None for r in solo for o in r) == 1
    for cache in (True, False):
        with serving.DecryptionServer(mat.decryption_key, slots=3, cache_committees=cache) as srv:
            futs = [srv.submit(cts, keys, seed=i) for i, (cts, keys, _) in enumerate(reqs)]
            mixed = [f.result() for f in futs]
            st = srv.stats()
        assert mixed == solo
        assert st["requests"] == len(reqs) and st["p50_ms"] is not None and st["p99_ms"] >= st["p50_ms"]
        if cache:
            # three distinct (batch size, committee) contexts repeat: 8/[1,3] three times
            assert st["cache_misses"] == 5 and st["cache_hits"] == 2


def test_budget_admits_one_request_at_a_time(mix):
    mat, reqs = mix
    sizes = [serving.request_bytes(len(c), len(k)) + serving.preparation_bytes(
        len(c), len(k), sum(mat.decryption_key.party_weight(x.party_index) for x in k)) for c, k, _ in reqs]
    budget = max(sizes)  # the largest request never shares the GPU with another
    with serving.DecryptionServer(mat.decryption_key, slots=4, hbm_budget_bytes=budget) as srv:
        futs = [srv.submit(cts, keys) for cts, keys, _ in reqs]
        out = [f.result() for f in futs]
        st = srv.stats()
    assert out == [alone(mat, cts, keys) for cts, keys, _ in reqs]
    assert st["peak_bytes"] <= budget and st["peak_in_flight"] < len(reqs)
    with serving.DecryptionServer(mat.decryption_key, slots=2, hbm_budget_bytes=min(sizes) - 1) as srv:
        with pytest.raises(MemoryError):
            srv.submit(reqs[0][0], reqs[0][1])


def test_concurrent_streams_match_sequential(mix):
    mat, reqs = mix
    cache = serving.CommitteeCache(1 << 30)

    def fn(r):
        cts, keys, _ = r
        return serving.decrypt_request(mat.decryption_key, cts, keys, ChaCha20Rng.seed_from_u64(1), cache)

    outs, ms = serving.run_concurrent(fn, reqs, 4)
    assert ms > 0
    assert outs == [alone(mat, cts, keys) for cts, keys, _ in reqs]


def test_grouped_batches_match_one_by_one(mix):
    """The batched form (every phase launched once for K batches) gives each
    batch exactly what decrypting it alone gives, invalid slots included."""
    mat, reqs = mix
    group = [r for r in reqs if len(r[0]) == 8 and [k.party_index for k in r[1]] == [1, 3]]
    rng = ChaCha20Rng.seed_from_u64(42)
    extra = []
    for i in range(3):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(8)])
        cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
        if i == 1:
            bad = cts[5]
            cts[5] = wb.Ciphertext(bad.first, bad.second, wb.SchnorrProof(bad.proof.commitment,
                                                                          (bad.proof.response + 1) % wb.R))
        extra.append((cts, group[0][1], msgs))
    group = group + extra
    keys = group[0][1]
    cache = serving.CommitteeCache(1 << 30)
    out = serving.decrypt_group(mat.decryption_key, [g[0] for g in group], keys, ChaCha20Rng.seed_from_u64(3), cache)
    assert out == [alone(mat, cts, keys) for cts, _, _ in group]
    assert out[len(group) - 2][5] is None and sum(o is None for r in out for o in r) == 1
    dev = serving.decrypt_group(mat.decryption_key, [wb.CiphertextBatch.upload(g[0]) for g in group], keys,
                                ChaCha20Rng.seed_from_u64(4), cache, device_output=True)
    for o, r in zip(dev, out):
        assert [wb.to_host(o)[576 * i : 576 * (i + 1)] if x is not None else None for i, x in enumerate(r)] == r


def test_validate_batches_equals_validate_batch(mix):
    mat, reqs = mix
    batches = [r[0] for r in reqs] + [wb.CiphertextBatch.upload(reqs[2][0])]
    many = wb.validate_batches(mat.decryption_key, batches)
    for cts, v in zip(batches, many):
        one = wb.validate_batch(mat.decryption_key, cts)
        assert v.batch_size() == one.batch_size() and v.digest() == one.digest()
        assert v.valid_mask() == one.valid_mask()
        assert wb.to_host(v.first_dev) == wb.to_host(one.first_dev)
        assert wb.to_host(v.valid_dev) == wb.to_host(one.valid_dev)


def test_fixed_base_share_check_matches_pippenger():
    """The share check over fixed-base tables of the parties' verification
    keys accepts exactly what the Pippenger path accepts: honest shares of
    every batch, not a batch with a tampered share."""
    from weighted_bte_b200 import _lib
    from weighted_bte_b200.rng import ChaCha20Rng, sample_nonzero

    rng = ChaCha20Rng.seed_from_u64(21)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2], mat.party_keys[3]]
    K, B, T = 3, 8, len(keys)
    batches = []
    for _ in range(K):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
        batches.append(wb.validate_batch(dk, wb.encrypt_many(mat.encryption_key, msgs, rng)))
    import torch

    first = torch.cat([v.first_dev[: 96 * B] for v in batches])
    sig = b"".join(s.sigma for v in batches for s in wb.partial_decrypt_many(keys, v))
    parties = [k.party_index for k in keys]
    ch = b"".join(wb.fr_bytes(sample_nonzero(rng)) for _ in range(K * T))
    tables = wb.empty_device(_lib.FIXED_TABLE_BYTES * T * B)
    ctx = wb._ctx()
    ctx.call("wbte_wbtx_vk_tables", tables, dk.abi_key(), _lib.i64_array(parties), T, B)
    bad = bytearray(sig)
    bad[96 * (1 * T + 2) + 7] ^= 0x04  # batch 1, third share
    for s, expect in ((sig, [1, 1, 1]), (bytes(bad), [1, 0, 1])):
        got = {}
        for name, tab in (("tables", tables), ("pippenger", None)):
            ok = np.zeros(K, dtype=np.int32)
            ctx.call("wbte_wbtx_verify_shares_many", ok, dk.abi_key(), first, B, s, _lib.i64_array(parties), ch, T,
                     K, tab)
            got[name] = list(ok)
        assert got["tables"] == got["pippenger"] == expect


@pytest.mark.parametrize("chunk", [1, 2, 3, 8])
def test_share_checks_with_chunked_miller_loops(chunk):
    """The share checks' multi-Miller loops over runs of `chunk` pairs (9
    pairs per batch: ragged last runs for 2 and 8, one run-length of 3, one
    pair per thread for 1) accept honest shares and reject a tampered one,
    in the batched and the single-batch check."""
    from weighted_bte_b200 import _lib
    from weighted_bte_b200.rng import sample_nonzero

    rng = ChaCha20Rng.seed_from_u64(23)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2], mat.party_keys[3]]
    K, B, T = 3, 8, len(keys)
    batches = []
    for _ in range(K):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
        batches.append(wb.validate_batch(dk, wb.encrypt_many(mat.encryption_key, msgs, rng)))
    import torch

    first = torch.cat([v.first_dev[: 96 * B] for v in batches])
    shares = [wb.partial_decrypt_many(keys, v) for v in batches]
    sig = b"".join(s.sigma for sh in shares for s in sh)
    parties = [k.party_index for k in keys]
    chal = [sample_nonzero(rng) for _ in range(K * T)]
    ch = b"".join(wb.fr_bytes(x) for x in chal)
    bad = bytearray(sig)
    bad[96 * (2 * T + 1) + 7] ^= 0x04  # batch 2, second share
    ctx = wb._ctx()
    ctx.set_tuning(_lib.TUNE_MILLER_CHUNK, chunk)
    try:
        for s, expect in ((sig, [1, 1, 1]), (bytes(bad), [1, 1, 0])):
            ok = np.zeros(K, dtype=np.int32)
            ctx.call("wbte_wbtx_verify_shares_many", ok, dk.abi_key(), first, B, s, _lib.i64_array(parties), ch, T,
                     K, None)
            assert list(ok) == expect
        for b in range(K):
            assert wb._verify_shares(dk, batches[b], shares[b], chal[b * T : (b + 1) * T])
        tampered = list(shares[2])
        tampered[1] = wb.DecryptionShare(tampered[1].party_index, bytes(bad[96 * (2 * T + 1) : 96 * (2 * T + 2)]),
                                         tampered[1].batch_digest, tampered[1].setup_id)
        assert not wb._verify_shares(dk, batches[2], tampered, chal[2 * T : 3 * T])
    finally:
        ctx.set_tuning(_lib.TUNE_MILLER_CHUNK, 0)


def test_fused_decryption_matches_precompute_then_open():
    """wbte_wbtx_decrypt_many (one hard final exponentiation per slot), with
    and without the opening keys' line tables, equals precompute_many
    followed by open_many, invalid slots included."""
    from weighted_bte_b200 import _lib

    rng = ChaCha20Rng.seed_from_u64(23)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2]]
    K, B, T = 2, 8, len(keys)
    vals, cts_all = [], []
    for b in range(K):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
        cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
        if b == 1:  # an invalid proof at slot 3
            cts[3] = wb.Ciphertext(cts[3].first, cts[3].second,
                                   wb.SchnorrProof(cts[3].proof.commitment, (cts[3].proof.response + 1) % wb.R))
        cts_all.append(cts)
        vals.append(wb.validate_batch(dk, cts))
    import torch

    first = torch.cat([v.first_dev[: 96 * B] for v in vals])
    valid = torch.cat([v.valid_dev[:B] for v in vals])
    second = wb.to_device(b"".join(c.second for cts in cts_all for c in cts))
    accepted = wb.accept_decryption_shares(dk, vals[0], wb.partial_decrypt_many(keys, vals[0]))
    pre = wb.prepare_decryption(dk, accepted)
    sig = b"".join(s.sigma for v in vals for s in wb.partial_decrypt_many(keys, v))
    ctx = wb._ctx()
    beta = wb.empty_device(576 * B * K)
    ref = wb.empty_device(576 * B * K)
    ctx.call("wbte_wbtx_precompute_many", beta, pre.kernel_lines, first, valid, B, K)
    ctx.call("wbte_wbtx_open_many", ref, pre.opening_keys, pre.opening_lines, sig, T, second, beta, valid, B, K)
    for lines in (pre.opening_lines, None):
        out = wb.empty_device(576 * B * K)
        ctx.call("wbte_wbtx_decrypt_many", out, pre.kernel_lines, pre.opening_keys, lines, first, second, valid,
                 sig, T, B, K)
        assert torch.equal(out[: 576 * B * K], ref[: 576 * B * K]), lines is None
    host = wb.to_host(ref, 576 * B * K)
    plain = [wb.decrypt(dk, cts, wb.partial_decrypt_many(keys, wb.validate_batch(dk, cts))) for cts in cts_all]
    for b in range(K):
        for i in range(B):
            got = host[576 * (b * B + i) : 576 * (b * B + i + 1)]
            assert (plain[b][i] is None) == (not vals[b].valid[i])
            if plain[b][i] is not None:
                assert got == plain[b][i]


def test_group_of_32_batches_matches_one_by_one():
    """32 batches in one group: every batched transform runs its warp-uniform
    kernels (the G1 transform's NAF twiddles, the GT stages' NAF plans)."""
    rng = ChaCha20Rng.seed_from_u64(29)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2]]
    msgs, batches = [], []
    for _ in range(32):
        m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(8)])
        msgs.append(m)
        batches.append(wb.encrypt_many(mat.encryption_key, m, rng))
    out = serving.decrypt_group(dk, [wb.CiphertextBatch.upload(c) for c in batches], keys,
                                ChaCha20Rng.seed_from_u64(3), serving.CommitteeCache(1 << 30))
    assert out == msgs


def test_group_with_a_dishonest_party_matches_one_by_one():
    """A party whose shares are well-formed points but wrong fails every
    batch's aggregate share check: the group decryption blames that share in
    each batch and decrypts with the honest remainder, exactly as each batch
    alone does."""
    import dataclasses

    rng = ChaCha20Rng.seed_from_u64(31)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    bad = dataclasses.replace(mat.party_keys[1], _q=(mat.party_keys[1].secret_scalar() + 1) % wb.R)
    keys = [mat.party_keys[0], bad, mat.party_keys[2]]  # 0 and 2 alone carry weight 7 > 4
    batches = []
    for _ in range(3):
        msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(8)])
        batches.append(wb.encrypt_many(mat.encryption_key, msgs, rng))
    cache = serving.CommitteeCache(1 << 30)
    grouped = serving.decrypt_group(dk, batches, keys, ChaCha20Rng.seed_from_u64(5), cache)
    alone = [serving.decrypt_request(dk, cts, keys, ChaCha20Rng.seed_from_u64(5), cache) for cts in batches]
    assert grouped == alone
    assert all(r is not None for res in grouped for r in res)


def test_graph_replayed_groups_match_the_direct_groups():
    """The batched decryption captured once as a CUDA graph and replayed for
    later groups of the same shape (new inputs copied into its buffers) gives
    the direct call's messages, group after group; a committee or group size
    it has not seen is captured on first use."""
    rng = ChaCha20Rng.seed_from_u64(33)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2]]
    cache = serving.CommitteeCache(1 << 30)
    graphs = serving.DecryptGraphs()
    for k, K in enumerate((4, 4, 4, 2)):
        msgs, batches = [], []
        for _ in range(K):
            m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(8)])
            msgs.append(m)
            batches.append(wb.encrypt_many(mat.encryption_key, m, rng))
        direct = serving.decrypt_group(dk, batches, keys, ChaCha20Rng.seed_from_u64(k), cache)
        replayed = serving.decrypt_group(dk, batches, keys, ChaCha20Rng.seed_from_u64(k), cache, graphs=graphs)
        assert replayed == direct == msgs
    assert graphs.captures == 2 and graphs.replays == 4
    assert all(v > 10 for v in graphs.kernels.values())


def test_graph_captures_beside_concurrent_groups():
    """Three threads on their own streams run grouped decryptions with graph
    replay at once, so captures overlap other threads' uploads, validations
    and launches (the batched form's layout); every group gives the direct
    call's messages."""
    import threading

    import torch

    rng = ChaCha20Rng.seed_from_u64(34)
    mat = wb.keygen_with_rng(wb.KeygenConfig(8, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2]]
    cache = serving.CommitteeCache(1 << 30)
    graphs = serving.DecryptGraphs()
    work = []
    for _ in range(3):
        groups = []
        for _ in range(3):
            msgs = [wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(8)]) for _ in range(4)]
            groups.append((msgs, [wb.encrypt_many(mat.encryption_key, m, rng) for m in msgs]))
        work.append(groups)
    direct = [[serving.decrypt_group(dk, b, keys, ChaCha20Rng.seed_from_u64(7), cache) for _, b in groups]
              for groups in work]
    got, errors = [None] * 3, []
    device = torch.cuda.current_device()

    def worker(w):
        try:
            torch.cuda.set_device(device)
            with torch.cuda.stream(torch.cuda.Stream()):
                got[w] = [serving.decrypt_group(dk, b, keys, ChaCha20Rng.seed_from_u64(7), cache, graphs=graphs)
                          for _, b in work[w]]
                torch.cuda.current_stream().synchronize()
        except BaseException as exc:  # noqa: BLE001
            errors.append(exc)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for w in range(3):
        assert got[w] == direct[w] == [m for m, _ in work[w]]
    assert graphs.captures == 3 and graphs.replays == 9


@pytest.mark.parametrize("K", [27, 37])
def test_group_sizes_off_a_multiple_of_32_match_one_by_one(K):
    """27 batches run the batched transforms padded to 32 slots, 37 batches as
    32 plus a remainder of 5; both equal the batches decrypted one by one."""
    rng = ChaCha20Rng.seed_from_u64(35 + K)
    mat = wb.keygen_with_rng(wb.KeygenConfig(4, [3, 2, 4, 1], 4), rng)
    dk = mat.decryption_key
    keys = [mat.party_keys[0], mat.party_keys[2]]
    msgs, batches = [], []
    for _ in range(K):
        m = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(4)])
        msgs.append(m)
        batches.append(wb.encrypt_many(mat.encryption_key, m, rng))
    cache = serving.CommitteeCache(1 << 30)
    out = serving.decrypt_group(dk, batches, keys, ChaCha20Rng.seed_from_u64(3), cache)
    assert out == msgs
