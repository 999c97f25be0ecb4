"""Batched weighted_pfe decryption: many batches of uneven sizes on one GPU.

weighted_pfe is an exact-size scheme: its key material depends on the
batch size B (a power of two), and a batch of s < B ciphertexts is filled
with valid dummy encryptions before it is decrypted (weighted_pfe/README.md:60-66,
weighted_pfe/src/setup.rs:536).  A deployment therefore keeps one key per
power-of-two size class resident and routes every batch to the class of
next_pow2(s).

* `decrypt_group` decrypts K batches of one class against one committee with
  every GPU phase launched once over all of them: batched validation (one
  family of K Schnorr-aggregate MSMs), the committee's partial decryptions
  (one MSM family), the aggregate share check (one multi-Miller launch plus
  one final exponentiation per batch, over fixed-base tables of the
  committee's verification keys), the committee preparation (cached), and
  precompute + open fused in `wbte_wpfe_decrypt_many`.  Per batch the result
  equals `weighted_pfe.decrypt` of that batch alone.
* `UnevenBatchDecryptor` takes batches of any sizes, pads each to its class
  with dummies, groups them by class and runs the classes concurrently on
  CUDA streams, largest work first; each class's library calls use the knobs
  the autotuner picked for that class (`autotune.Autotuner`).
"""
from __future__ import annotations

import threading
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib, ops
from . import errors as E
from . import weighted_btx as wb
from . import weighted_pfe as wp
from .rng import ChaCha20Rng, sample_nonzero
from .serving import CommitteeCache

G1B, G2B, GTB = wb.G1B, wb.G2B, wb.GTB


def size_class(s: int) -> int:
    """The power-of-two class of a batch of s ciphertexts."""
    if s <= 0:
        raise E.BatchIsEmpty()
    return 1 << (s - 1).bit_length()


@dataclass
class PreparedCommittee:
    """A committee's preparation for one class, resident in HBM: the
    reference's DecryptionPrecomputation plus the line tables of its B*T
    per-party keys, over which each slot's opening pairings run as one
    multi-Miller loop."""

    pre: wp.DecryptionPrecomputation
    by_party_lines: object  # device, B * T line tables


def prepare_committee(dk: wp.PublicDecryptionKey, accepted: wp.AcceptedDecryptionShares) -> PreparedCommittee:
    pre = wp.prepare_decryption(dk, accepted)
    B, T = dk.batch_size(), accepted.party_count()
    lines = wb.empty_device(_lib.LINE_BYTES * _lib.MILLER_LINES * B * T)
    wb._ctx().call("wbte_g2_prepare_lines", lines, pre.scaled_d1_by_party, B * T)
    return PreparedCommittee(pre, lines)


def _committee(cache: Optional[CommitteeCache], dk, accepted) -> PreparedCommittee:
    if cache is None:
        return prepare_committee(dk, accepted)
    key = b"wpfe" + wp.committee_context_id(dk.setup_id(), accepted.party_indices())

    def build():
        pc = prepare_committee(dk, accepted)
        p = pc.pre
        return pc, [p.scaled_d1_by_party, p.total_lines, p.mask_lines, p.scaled_d1_total, p.mask_keys,
                    pc.by_party_lines]

    return cache.obtain(key, build)


VK_TABLE_LIMIT = 1 << 30  # bytes of fixed-base verification-key tables per class and committee


def _vk_tables(cache: Optional[CommitteeCache], dk, parties: Sequence[int]):
    """Fixed-base tables of the parties' verification keys at every slot
    (wbte_wpfe_vk_tables), cached per setup and party set; None (the share
    check's Pippenger path) without a cache or beyond VK_TABLE_LIMIT."""
    if cache is None or _lib.FIXED_TABLE_BYTES * len(parties) * dk.batch_size() > VK_TABLE_LIMIT:
        return None
    key = b"wpfe-vk" + dk.setup_id() + b"".join(int(j).to_bytes(8, "little") for j in parties)

    def build():
        T = len(parties)
        tables = wb.empty_device(_lib.FIXED_TABLE_BYTES * T * dk.batch_size())
        wb._ctx().call("wbte_wpfe_vk_tables", tables, dk.abi_key(), _lib.i64_array(parties), T)
        return tables, [tables]

    return cache.obtain(key, build, count=False)


def decrypt_group(encryption_key: wp.EncryptionKey, decryption_key: wp.PublicDecryptionKey, batches: Sequence,
                  party_keys: Sequence[wp.PartySecretKey], rng, cache: Optional[CommitteeCache] = None,
                  device_output: bool = False) -> list:
    """Decrypts K batches of the key's batch size, each submitted to the
    parties of `party_keys` (the reference's `decrypt` after every party's
    partial_decrypt, weighted_pfe/src/decryption.rs:231-252, :646-669).

    Entry b is batch b's plaintexts (a list of B GT elements, or a device
    tensor with device_output), or the error `decrypt` raises for that batch
    alone (an invalid proof rejects its whole batch; too little accepted
    weight rejects it at acceptance)."""
    torch = wb._t()
    ek, dk = encryption_key, decryption_key
    if ek.setup_id() != dk.setup_id():
        raise E.MismatchedSetup()
    K = len(batches)
    results: list = [None] * K
    if K == 0:
        return results
    B = dk.batch_size()
    arrays = [wp._device_arrays(cts) if len(cts) == B else None for cts in batches]
    validated = wp.validate_batches(ek, batches, rng, arrays)
    live = [b for b in range(K) if isinstance(validated[b], wp.ValidatedBatch)]
    for b in range(K):
        if b not in live:
            results[b] = validated[b]
    if not live:
        return results
    vb = [validated[b] for b in live]
    shares = wp.partial_decrypt_batches(party_keys, vb)
    T = len(party_keys)
    screened = [wp.screen_shares(dk, v, sh) for v, sh in zip(vb, shares)]
    accepted: list = [None] * len(live)
    if T > 0 and all(len(c) == T and not r for c, r in screened):
        # one aggregate share check per batch, all in one launch sequence
        # (verify_decryption_shares_batched, weighted_pfe/src/decryption.rs:367-419)
        parties = [pk.party_index for pk in party_keys]
        challenges = [[sample_nonzero(rng) for _ in range(T)] for _ in live]
        ok = np.zeros(len(live), dtype=np.int32)
        first = torch.cat([v.first_dev[: G1B * B] for v in vb])
        sig = b"".join(s.sigma for row in shares for s in row)
        wb._ctx().call("wbte_wpfe_verify_shares_many", ok, dk.abi_key(), first, sig, _lib.i64_array(parties),
                       b"".join(wb.fr_bytes(c) for row in challenges for c in row), T, len(live),
                       _vk_tables(cache, dk, parties))
        for q in range(len(live)):
            try:
                accepted[q] = wp.finish_acceptance(dk, vb[q], *screened[q], bool(ok[q]))
            except E.Error as exc:  # noqa: PERF203 -- per-batch outcome
                accepted[q] = exc
    else:
        for q in range(len(live)):
            try:
                accepted[q] = wp.accept_decryption_shares(dk, vb[q], shares[q], rng)
            except E.Error as exc:
                accepted[q] = exc
    # batches whose share check blamed a party keep their own accepted
    # committee; each committee's batches are decrypted as one group
    parts: Dict[tuple, List[int]] = {}
    for q, a in enumerate(accepted):
        if isinstance(a, BaseException):
            results[live[q]] = a
        else:
            parts.setdefault(tuple(a.party_indices()), []).append(q)
    alpha = dk.alpha_points()
    ap = ops.scalars_bytes([a * (a + 1) % R for a in alpha])
    for qs in parts.values():
        acc = accepted[qs[0]]
        pc = _committee(cache, dk, acc)
        Ta, Kp = acc.party_count(), len(qs)
        first = torch.cat([vb[q].first_dev[: G1B * B] for q in qs])
        second = torch.cat([arrays[live[q]][2] for q in qs])
        sig = b"".join(s.sigma for q in qs for s in accepted[q].shares())
        out = wb.empty_device(GTB * B * Kp)
        wb._ctx().call("wbte_wpfe_decrypt_many", out, sig, Ta, pc.pre.scaled_d1_by_party, pc.by_party_lines,
                       pc.pre.total_lines, pc.pre.mask_lines, first, second, ap, B, Kp)
        if device_output:
            for i, q in enumerate(qs):
                results[live[q]] = out[GTB * B * i : GTB * B * (i + 1)]
        else:
            host = wb.to_host(out, GTB * B * Kp)
            for i, q in enumerate(qs):
                results[live[q]] = [host[GTB * (i * B + j) : GTB * (i * B + j + 1)] for j in range(B)]
    return results


R = ops.R


# ------------------------------------------------------------- uneven sizes
class SizeClass:
    """One power-of-two class: its key material (resident in HBM), the
    submitting committee's secret keys and a pool of valid dummy ciphertexts
    (encryptions of the identity under the class key) that fill short batches."""

    def __init__(self, material: wp.KeyMaterial, committee: Sequence[int], rng):
        self.material = material
        self.B = material.encryption_key.batch_size()
        self.party_keys = [material.party_keys[j] for j in committee]
        one = ops.gt_pow(wb.gt_generator(), [0], fixed_base=True)
        n_dummy = max(1, self.B // 2)
        self.dummies = wp.encrypt_many(material.encryption_key, [one] * n_dummy, rng)

    def pad(self, cts: Sequence[wp.Ciphertext]) -> List[wp.Ciphertext]:
        """cts followed by valid dummies up to the class size."""
        if len(cts) > self.B:
            raise E.MismatchedBatchSize(self.B, len(cts))
        missing = self.B - len(cts)
        if missing > len(self.dummies):
            raise E.MismatchedBatchSize(self.B, len(cts))
        return list(cts) + self.dummies[:missing]


def class_keys(B_values: Sequence[int], weights: Sequence[int], threshold: int, committee: Sequence[int],
               seed: int) -> Dict[int, SizeClass]:
    """Key material for every class in B_values (generated on the GPU, one
    ChaCha20 stream per class derived from `seed`)."""
    out = {}
    for B in sorted(set(B_values)):
        rng = ChaCha20Rng.seed_from_u64(seed * 1000003 + B)
        mat = wp.keygen_with_rng(wp.KeygenConfig(B, list(weights), threshold), rng)
        out[B] = SizeClass(mat, committee, rng)
    return out


class UnevenBatchDecryptor:
    """Decrypts batches of uneven sizes: each batch goes to the class of
    next_pow2(size), is padded there with dummies, and every class decrypts
    its batches as groups of at most the tuned group size (`decrypt_group`).
    The classes run concurrently, one worker thread and CUDA stream each,
    largest work first; the results are cut back to the original sizes.

    `tuner` (autotune.Autotuner) picks each class's knobs and group size on
    first use and caches them; without it the library's cost models decide."""

    def __init__(self, classes: Dict[int, SizeClass], streams: int = 4, cache: Optional[CommitteeCache] = None,
                 tuner=None, max_group: int = 256):
        self.classes = classes
        self.streams = max(1, int(streams))
        self.cache = cache if cache is not None else CommitteeCache(16 << 30)
        self.tuner = tuner
        self.max_group = max_group
        self.class_ms: Dict[int, float] = {}

    def _run_class(self, B: int, batches: List[List[wp.Ciphertext]], seed: int, device_output: bool):
        sc = self.classes[B]
        knobs = self.tuner.knobs_for(B, sc, self) if self.tuner is not None else {}
        group = int(knobs.get("group", self.max_group)) or self.max_group
        ctx = wb._ctx()
        _apply_knobs(ctx, knobs)
        try:
            rng = ChaCha20Rng.seed_from_u64(seed)
            out = []
            for g0 in range(0, len(batches), group):
                chunk = [sc.pad(b) for b in batches[g0 : g0 + group]]
                out += decrypt_group(sc.material.encryption_key, sc.material.decryption_key, chunk, sc.party_keys,
                                     rng, self.cache, device_output=device_output)
            return out
        finally:
            _apply_knobs(ctx, {})

    def decrypt(self, batches: Sequence[Sequence[wp.Ciphertext]], seed: int = 0, device_output: bool = False):
        """Entry b: batch b's plaintexts (len(batches[b]) GT elements), or the
        error that `decrypt` raises for it.  With device_output, entry b is a
        device tensor of the padded batch's B GT values (the first
        len(batches[b]) are batch b's)."""
        torch = wb._t()
        by_class: Dict[int, List[int]] = {}
        for b, cts in enumerate(batches):
            by_class.setdefault(size_class(len(cts)), []).append(b)
        for B in by_class:
            if B not in self.classes:
                raise E.InvalidBatchSize(B)
        order = sorted(by_class, key=lambda B: -B * len(by_class[B]))
        results: list = [None] * len(batches)
        errors: List[BaseException] = []
        lock = threading.Lock()
        todo = list(order)
        device = torch.cuda.current_device()

        def worker():
            try:
                torch.cuda.set_device(device)
                stream = torch.cuda.Stream(device=device)
                while True:
                    with lock:
                        if not todo or errors:
                            return
                        B = todo.pop(0)
                    idx = by_class[B]
                    start = torch.cuda.Event(enable_timing=True)
                    end = torch.cuda.Event(enable_timing=True)
                    with torch.cuda.stream(stream):
                        start.record(stream)
                        outs = self._run_class(B, [list(batches[b]) for b in idx], seed + B, device_output)
                        end.record(stream)
                    stream.synchronize()
                    self.class_ms[B] = start.elapsed_time(end)
                    for b, o in zip(idx, outs):
                        if isinstance(o, list):
                            o = o[: len(batches[b])]
                        results[b] = o
            except BaseException as exc:  # noqa: BLE001 -- re-raised below
                with lock:
                    errors.append(exc)

        threads = [threading.Thread(target=worker) for _ in range(min(self.streams, len(order)))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return results


def _apply_knobs(ctx, knobs: dict):
    ctx.set_tuning(_lib.TUNE_GT_LANES, int(knobs.get("gt_lanes", 0)))
    ctx.set_tuning(_lib.TUNE_MSM_WINDOW, int(knobs.get("msm_window", 0)))
    ctx.set_tuning(_lib.TUNE_MSM_SEGMENTS, int(knobs.get("msm_segments", 0)))
    ctx.set_tuning(_lib.TUNE_NTT_JOINT, int(knobs.get("ntt_joint", -1)))


# ------------------------------------------------------------- served form
def request_bytes(B: int, T: int) -> int:
    """Device memory one weighted_pfe request of class B (committee of T)
    holds while it runs: the batch and its encodings, the validation MSM, the
    Cauchy transforms (G1 work, two GT arrays), the opening's per-(slot,
    party) G1 points and GT values, and the output."""
    return B * (6400 + 480 * T) + (1 << 20)


def preparation_bytes(B: int, T: int) -> int:
    """Device memory of one prepared committee of class B (kept in the cache)
    plus the working memory of preparing it: per-party keys and their line
    tables, the total and mask line tables, the verification-key tables
    (when within VK_TABLE_LIMIT), the preparation's MSM scratch."""
    tables = _lib.FIXED_TABLE_BYTES * T * B
    tables = tables if tables <= VK_TABLE_LIMIT else 0
    lines = _lib.LINE_BYTES * _lib.MILLER_LINES
    return B * T * (G2B + lines + 32 * 2 * G2B) + 2 * B * lines + tables


class WpfeBackend:
    """Runs weighted_pfe requests in serving.DecryptionServer: a request is a
    batch of any size s, routed to the class next_pow2(s), padded there with
    the class's dummies and decrypted by the class's committee; requests of
    one class and committee that wait together form one group
    (`decrypt_group`).  A request's result is its s plaintexts; a batch the
    scheme rejects raises that error through its future."""

    def __init__(self, classes: Dict[int, SizeClass]):
        self.classes = classes

    def _class(self, ciphertexts) -> SizeClass:
        B = size_class(len(ciphertexts))
        if B not in self.classes:
            raise E.InvalidBatchSize(B)
        return self.classes[B]

    def need(self, ciphertexts, party_keys) -> int:
        sc = self._class(ciphertexts)
        return request_bytes(sc.B, len(party_keys)) + preparation_bytes(sc.B, len(party_keys))

    def group_key(self, ciphertexts, party_keys):
        return size_class(len(ciphertexts)), tuple(k.party_index for k in party_keys)

    def run(self, group, rng, cache) -> list:
        sc = self._class(group[0].ciphertexts)
        mat = sc.material
        padded = [sc.pad(r.ciphertexts) for r in group]
        outs = decrypt_group(mat.encryption_key, mat.decryption_key, padded, group[0].party_keys, rng, cache)
        return [o[: len(r.ciphertexts)] if isinstance(o, list) else o for o, r in zip(outs, group)]
