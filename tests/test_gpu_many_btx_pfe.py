"""The batched forms of btx and pfe (wbte_btx_*_many, wbte_pfe_*_many): K
batches per launch sequence give, batch for batch, the single-batch calls'
results (btx/src/decryption.rs:201-246, :402-458; pfe/src/decryption.rs:259-298,
:417-469) and the plaintexts."""
import pytest

from weighted_bte_b200 import btx, pfe
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu


def gt_msgs(n, base):
    from weighted_bte_b200 import ops

    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


def test_btx_many_matches_single_batches():
    L, B, K, t = 8, 6, 3, 2
    mat = btx.keygen_with_rng(btx.KeygenConfig(L, 5, t), ChaCha20Rng.seed_from_u64(81))
    dk = mat.decryption_key
    kern = btx.MiddleProductKernel.new(dk, B)
    msgs, cts_all, batches, sigmas = [], [], [], []
    for k in range(K):
        m = gt_msgs(B, 20 * (k + 1))
        cts = btx.encrypt_many(mat.encryption_key, m, ChaCha20Rng.seed_from_u64(90 + k))
        if k == 1:  # a broken proof: that slot opens to nothing
            c = cts[3]
            cts[3] = btx.Ciphertext(c.first, c.second, btx.SchnorrProof(c.proof.commitment,
                                                                        (c.proof.response + 1) % btx.R))
        batch = btx.validate_batch(cts)
        shares = [btx.partial_decrypt(mat.server_keys[j], batch) for j in range(t + 1)]
        msgs.append(m)
        cts_all.append(cts)
        batches.append(batch)
        sigmas.append(btx.combine_shares(dk, batch, shares))
    singles = []
    for k in range(K):
        pre = btx.precompute_batch(kern, batches[k])
        singles.append((pre, btx.open_batch(kern, batches[k], cts_all[k], pre, sigmas[k], device_output=True)))
    torch = wb._t()
    first = torch.cat([b.first_dev[: 96 * B] for b in batches])
    valid = torch.cat([b.valid_dev[:B] for b in batches])
    second = b"".join(c.second for cts in cts_all for c in cts)
    beta = wb.empty_device(576 * B * K)
    wb._ctx().call("wbte_btx_precompute_many", beta, kern.kernel_lines, first, wb.to_device(b"\x01" * (B * K)), B, K)
    for k in range(K):
        assert wb.to_host(beta)[576 * B * k : 576 * B * (k + 1)] == wb.to_host(singles[k][0].beta, 576 * B)
    out = bytearray(576 * B * K)
    wb._ctx().call("wbte_btx_open_many", out, kern.opening_lines, b"".join(sigmas), second, beta, valid, B, K)
    fused = bytearray(576 * B * K)
    wb._ctx().call("wbte_btx_decrypt_many", fused, kern.kernel_lines, kern.opening_lines, first, second, valid,
                   b"".join(sigmas), B, K)
    expect = b"".join(wb.to_host(o, 576 * B) for _, o in singles)
    assert bytes(out) == bytes(fused) == expect
    for k in range(K):
        got = btx.open_batch(kern, batches[k], cts_all[k], singles[k][0], sigmas[k])
        assert got == [m if v else None for m, v in zip(msgs[k], batches[k].valid_mask())]


def test_pfe_many_matches_single_batches():
    B, K, t = 8, 3, 2
    mat = pfe.keygen_with_rng(pfe.KeygenConfig(B, 5, t), ChaCha20Rng.seed_from_u64(82))
    dk, ek = mat.decryption_key, mat.encryption_key
    kern = pfe.PartialFractionKernel.new(dk)
    msgs, cts_all, batches, pdks, singles = [], [], [], [], []
    for k in range(K):
        m = gt_msgs(B, 30 * (k + 1))
        cts = pfe.encrypt_many(ek, m, ChaCha20Rng.seed_from_u64(95 + k))
        batch = pfe.validate_batch(ek, cts)
        shares = [pfe.partial_decrypt(mat.server_keys[j], batch) for j in range(t + 1)]
        pdk = pfe.combine_shares(dk, batch, shares)
        pre = pfe.precompute_batch(kern, batch)
        msgs.append(m)
        cts_all.append(cts)
        batches.append(batch)
        pdks.append(pdk)
        singles.append((pre, pfe.open_batch(kern, batch, cts, pre, pdk)))
    torch = wb._t()
    first = torch.cat([b.first_dev[: 96 * B] for b in batches])
    second = torch.cat([b.second_dev[: 96 * B] for b in batches])
    wf, wpr = wb.empty_device(96 * B * K), wb.empty_device(576 * B * K)
    wb._ctx().call("wbte_pfe_precompute_many", wf, wpr, first, kern.key_lines, kern.conv_scalars, B, K)
    for k in range(K):
        assert wb.to_host(wf)[96 * B * k : 96 * B * (k + 1)] == wb.to_host(singles[k][0].weighted_first, 96 * B)
        assert wb.to_host(wpr)[576 * B * k : 576 * B * (k + 1)] == wb.to_host(singles[k][0].weighted_pairings,
                                                                             576 * B)
    out = bytearray(576 * B * K)
    wb._ctx().call("wbte_pfe_open_many", out, first, second, b"".join(c.third for cts in cts_all for c in cts), wf,
                   wpr, b"".join(pdks), kern.neg_scaled_s1, kern.key_lines, kern.generator_lines, kern.mix_lines, B, K)
    assert bytes(out) == b"".join(b"".join(o) for _, o in singles) == b"".join(b"".join(m) for m in msgs)
