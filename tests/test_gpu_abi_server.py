"""The served form through the C ABI alone: resident key handles
(wbte_crs_upload_*) and the library's request loop (wbte_server_create,
wbte_submit, wbte_poll), driven through ctypes the way a Rust `wbte-sys`
caller would, without the Python serving layer.  Every request's messages
must equal the plaintexts (weighted_btx/src/decryption.rs:698-709,
weighted_pfe/src/decryption.rs:646-669)."""
import ctypes

import numpy as np
import pytest

from weighted_bte_b200 import _lib, ops
from weighted_bte_b200 import weighted_btx as wb
from weighted_bte_b200 import weighted_pfe as wp
from weighted_bte_b200.rng import ChaCha20Rng

pytestmark = pytest.mark.gpu

WBTE_OK, WBTE_ERR_INVALID_ARG, WBTE_ERR_SIZE, WBTE_ERR_TIMEOUT = 0, -1, -2, -4


def gt_msgs(n, base):
    return ops.split(ops.gt_pow(wb.gt_generator(), [base + i for i in range(n)], fixed_base=True), 576)


class Keep:
    """Host buffers of one request, alive until it is polled."""

    def __init__(self, **arrays):
        self.arrays = {k: np.frombuffer(bytes(v), dtype=np.uint8).copy() if not isinstance(v, np.ndarray) else v
                       for k, v in arrays.items()}

    def ptr(self, k):
        return self.arrays[k].ctypes.data


def _submit(lib, srv, crs, B, first, second, valid, sigma, parties):
    keep = Keep(first=first, second=second, sigma=sigma, messages=bytes(576 * B))
    if valid is not None:
        keep.arrays["valid"] = np.frombuffer(bytes(valid), dtype=np.uint8).copy()
    keep.arrays["parties"] = np.asarray(parties, dtype=np.int64)
    req = _lib.Request(crs.value, B, keep.ptr("first"), keep.ptr("second"),
                       keep.ptr("valid") if valid is not None else None, keep.ptr("sigma"), keep.ptr("parties"),
                       len(parties), keep.ptr("messages"))
    ticket = ctypes.c_uint64()
    st = lib.wbte_submit(srv, ctypes.byref(req), ctypes.byref(ticket))
    return st, ticket.value, keep


def test_weighted_btx_requests_through_the_abi_server():
    import torch

    torch.cuda.set_device(0)
    lib = _lib.load()
    ctx = _lib.default_context(0)
    weights, t, L = [1, 3, 2, 4, 1], 5, 8
    rng = ChaCha20Rng.seed_from_u64(51)
    mat = wb.keygen_with_rng(wb.KeygenConfig(L, weights, t), rng)
    dk = mat.decryption_key
    key = dk.abi_key()
    crs = ctypes.c_void_p()
    assert lib.wbte_crs_upload_wbtx(ctx.handle, ctypes.byref(key), ctypes.byref(crs)) == WBTE_OK
    srv = ctypes.c_void_p()
    assert lib.wbte_server_create(0, 2, 4, 0, ctypes.byref(srv)) == WBTE_OK
    parties = [1, 3]
    keys = [mat.party_keys[j] for j in parties]
    pending = []
    for k, B in enumerate([8, 8, 4, 8, 4, 8]):
        msgs = gt_msgs(B, 40 * (k + 1))
        cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
        if k == 3:  # one ciphertext with a broken proof: that slot opens to the identity
            c = cts[2]
            cts[2] = wb.Ciphertext(c.first, c.second, wb.SchnorrProof(c.proof.commitment,
                                                                      (c.proof.response + 1) % ops.R))
            msgs = msgs[:2] + [ops.gt_pow(wb.gt_generator(), [0], fixed_base=True)] + msgs[3:]
        batch = wb.validate_batch(dk, cts)
        acc = wb.accept_decryption_shares(dk, batch, wb.partial_decrypt_many(keys, batch), rng)
        assert acc.party_indices() == parties
        valid = bytes(int(v) for v in batch.valid)
        st, ticket, keep = _submit(lib, srv, crs, B, wb.to_host(batch.first_dev, 96 * B),
                                   b"".join(c.second for c in cts), valid, b"".join(s.sigma for s in acc.shares()),
                                   parties)
        assert st == WBTE_OK
        pending.append((ticket, keep, msgs))
    # a bounded wait that ends before the work does reports a timeout and keeps the ticket
    status = ctypes.c_int32()
    first_poll = lib.wbte_poll(srv, pending[-1][0], 0, ctypes.byref(status))
    assert first_poll in (WBTE_OK, WBTE_ERR_TIMEOUT)
    for i, (ticket, keep, msgs) in enumerate(pending):
        if i == len(pending) - 1 and first_poll == WBTE_OK:
            continue
        assert lib.wbte_poll(srv, ticket, 120 * 10**9, ctypes.byref(status)) == WBTE_OK
        assert status.value == WBTE_OK
        assert keep.arrays["messages"].tobytes() == b"".join(msgs), f"request {i}"
    # released and unknown tickets, and a batch larger than the setup's maximum
    assert lib.wbte_poll(srv, pending[0][0], 0, ctypes.byref(status)) == WBTE_ERR_INVALID_ARG
    st, _, _ = _submit(lib, srv, crs, 16, bytes(96 * 16), bytes(576 * 16), None, bytes(96 * 2), parties)
    assert st == WBTE_ERR_SIZE
    assert lib.wbte_server_destroy(srv) == WBTE_OK
    assert lib.wbte_crs_destroy(crs) == WBTE_OK


def test_weighted_pfe_classes_through_the_abi_server():
    import torch

    from weighted_bte_b200 import wpfe_batched as wpb

    torch.cuda.set_device(0)
    lib = _lib.load()
    ctx = _lib.default_context(0)
    weights, t = [2, 3, 1, 4, 2], 5
    committee = [1, 3]  # heaviest first: 4 + 3 > 5
    classes = wpb.class_keys([4, 8], weights, t, committee, seed=61)
    handles = {}
    for B, sc in classes.items():
        dk = sc.material.decryption_key
        alpha = dk.alpha_points()
        mask = ops.scalars_bytes([a * (a + 1) % ops.R for a in alpha] + [(-a) % ops.R for a in alpha])
        h = ctypes.c_void_p()
        key = dk.abi_key()
        assert lib.wbte_crs_upload_wpfe(ctx.handle, ctypes.byref(key), mask, ctypes.byref(h)) == WBTE_OK
        handles[B] = h
    srv = ctypes.c_void_p()
    assert lib.wbte_server_create(0, 3, 8, 0, ctypes.byref(srv)) == WBTE_OK
    rng = ChaCha20Rng.seed_from_u64(62)
    pending = []
    for k, s in enumerate([3, 8, 4, 6, 3, 7]):
        B = wpb.size_class(s)
        sc = classes[B]
        msgs = gt_msgs(s, 11 * (k + 3))
        cts = sc.pad(wp.encrypt_many(sc.material.encryption_key, msgs, rng))
        batch = wp.validate_batch(sc.material.encryption_key, cts)
        acc = wp.accept_decryption_shares(sc.material.decryption_key, batch,
                                          wp.partial_decrypt_many(sc.party_keys, batch), rng)
        st, ticket, keep = _submit(lib, srv, handles[B], B, wb.to_host(batch.first_dev, 96 * B),
                                   b"".join(c.second for c in cts), None, b"".join(x.sigma for x in acc.shares()),
                                   acc.party_indices())
        assert st == WBTE_OK
        pending.append((ticket, keep, msgs, s))
    status = ctypes.c_int32()
    for ticket, keep, msgs, s in pending:
        assert lib.wbte_poll(srv, ticket, 120 * 10**9, ctypes.byref(status)) == WBTE_OK
        assert status.value == WBTE_OK
        assert keep.arrays["messages"].tobytes()[: 576 * s] == b"".join(msgs)
    assert lib.wbte_server_destroy(srv) == WBTE_OK
    for h in handles.values():
        assert lib.wbte_crs_destroy(h) == WBTE_OK
