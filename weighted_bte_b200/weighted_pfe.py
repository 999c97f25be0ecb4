"""Weighted partial-fraction batch threshold encryption (Construction 5) on B200.

Mirrors the public API of the reference crate `weighted_pfe`
(weighted_pfe/src/lib.rs:18-28): `keygen[_with_rng]`, `encrypt[_with_rng]`,
`validate_batch`, `partial_decrypt`, `verify_decryption_share`,
`accept_decryption_shares`, `CauchyKernel`, `prepare_decryption`,
`precompute_batch`, `open_batch`, `decrypt`, with the reference's checks and
its `Error` variants (weighted_bte_b200.errors).

Group work runs in libwbte (the wbte_wpfe_* phase calls of include/wbte.h and
the shared primitives); this module holds the protocol logic, SHA-256
transcripts and data layout.  The public decryption key (verification keys,
D and U material, global key) is resident in HBM.  Group elements are `bytes`
in blst's memory layout; scalars are Python ints.
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import _lib, ops
from . import errors as E
from . import weighted_btx as wb
from .rng import OsRng, random_scalar, sample_nonzero

R = ops.R
G1B, G2B, GTB = wb.G1B, wb.G2B, wb.GTB
SETUP_ID_DOMAIN = b"WEIGHTED-PFE-SETUP-BLS12381-v2"
TRANSCRIPT_DOMAIN = b"WEIGHTED-PFE-CIPHERTEXT-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"WEIGHTED-PFE-ORDERED-BATCH-v1"
COMMITTEE_CONTEXT_DOMAIN = b"WEIGHTED-PFE-COMMITTEE-v1"
G1_IDENTITY = bytes(G1B)


def _inv(x: int) -> int:
    return pow(x % R, R - 2, R)


def _append_gt_fixed_many(values, n: int) -> List[bytes]:
    """Tag byte and a fixed 288-byte body, all zero for the identity
    (weighted_pfe/src/encoding.rs:13-28): the library's 289-byte records."""
    enc = ops.gt_compress(values, n)
    return [enc[289 * i : 289 * (i + 1)] for i in range(n)]


def _is_pow2(n: int) -> bool:
    return n > 0 and n & (n - 1) == 0


def root_domain_prefix(size: int, length: int) -> List[int]:
    """weighted_pfe/src/setup.rs:592-603."""
    if size == 1:
        return [1][:length]
    g = wb.radix2_generator(size)
    out, x = [], 1
    for _ in range(length):
        out.append(x)
        x = x * g % R
    return out


def shifted_alpha_points(batch_size: int):
    """alpha_i = omega^i + c for the smallest c >= 2 keeping alpha_i and
    alpha_i + 1 nonzero (weighted_pfe/src/setup.rs:605-618)."""
    roots = root_domain_prefix(batch_size, batch_size)
    c = 2
    while True:
        pts = [(r + c) % R for r in roots]
        if all(a != 0 and (a + 1) % R != 0 for a in pts):
            return pts, c
        c += 1


# ------------------------------------------------------------------- keys
@dataclass
class KeygenConfig:
    batch_size: int
    party_weights: List[int]
    threshold_weight: int


class EncryptionKey:
    def __init__(self, batch_size: int, element: bytes, setup_id: bytes):
        self._B, self._element, self._setup_id = batch_size, element, setup_id

    def batch_size(self) -> int:
        return self._B

    def element(self) -> bytes:
        return self._element

    def setup_id(self) -> bytes:
        return self._setup_id


class PublicDecryptionKey:
    """weighted_pfe/src/setup.rs:35-55 with the G2 material in HBM."""

    def __init__(self, setup_id, batch_size, threshold_weight, total_weight, domain_size, party_weights, offsets,
                 evaluation_domain, alpha_points, alpha_shift, vk, d1, d2, global_key):
        self._setup_id, self._B, self._t, self._W = setup_id, batch_size, threshold_weight, total_weight
        self._domain_size, self._weights = domain_size, list(party_weights)
        self.party_offsets = np.asarray(offsets, dtype=np.int64)
        self._domain, self._alpha, self._shift = list(evaluation_domain), list(alpha_points), alpha_shift
        self.verification_keys, self.d1, self.d2 = vk, d1, d2
        self.global_key_dev = global_key
        self.domain_dev = wb.to_device(ops.scalars_bytes(self._domain))
        self.alpha_dev = wb.to_device(ops.scalars_bytes(self._alpha))

    def setup_id(self) -> bytes:
        return self._setup_id

    def batch_size(self) -> int:
        return self._B

    def party_count(self) -> int:
        return len(self._weights)

    def total_weight(self) -> int:
        return self._W

    def threshold_weight(self) -> int:
        return self._t

    def required_weight(self) -> int:
        return self._t + 1

    def party_weights(self) -> List[int]:
        return list(self._weights)

    def party_weight(self, party_index: int) -> int:
        if party_index >= len(self._weights):
            raise E.InvalidPartyIndex(party_index)
        return self._weights[party_index]

    def domain_points(self) -> List[int]:
        return list(self._domain)

    def domain_size(self) -> int:
        return self._domain_size

    def alpha_points(self) -> List[int]:
        return list(self._alpha)

    def alpha_shift_small(self) -> int:
        return self._shift

    def verification_key_count(self) -> int:
        return self._B * self.party_count()

    def d1_point_count(self) -> int:
        return self._B * self._W

    def d2_point_count(self) -> int:
        return self._B * self._W

    def core_g2_point_count(self) -> int:
        return 2 * self._B * self._W + 1

    def g2_point_count(self) -> int:
        return self.verification_key_count() + self.core_g2_point_count()

    def serialized_size_bytes(self) -> int:
        return 96 * self.g2_point_count()

    def party_range(self, party_index: int) -> range:
        if party_index >= self.party_count():
            raise E.InvalidPartyIndex(party_index)
        return range(int(self.party_offsets[party_index]), int(self.party_offsets[party_index + 1]))

    def global_key(self) -> bytes:
        return wb.to_host(self.global_key_dev, G2B)

    def abi_key(self) -> _lib.WpfeKey:
        k = _lib.WpfeKey()
        k.domain_points = self.domain_dev.data_ptr()
        k.verification_keys = self.verification_keys.data_ptr()
        k.d1 = self.d1.data_ptr()
        k.d2 = self.d2.data_ptr()
        k.global_key = self.global_key_dev.data_ptr()
        self._offsets_keep = np.ascontiguousarray(self.party_offsets, dtype=np.int64)
        k.party_offsets = self._offsets_keep.ctypes.data
        k.party_count = self.party_count()
        k.total_weight = self._W
        k.batch_size = self._B
        return k


@dataclass
class PartySecretKey:
    party_index: int
    _setup_id: bytes
    _batch_size: int
    alpha_shift_small: int
    rho: int

    def setup_id(self) -> bytes:
        return self._setup_id

    def batch_size(self) -> int:
        return self._batch_size

    def scalar_count(self) -> int:
        return 1

    def fractions(self) -> List[int]:
        """g_{j,i} = 1 / (rho_j + alpha_i) (weighted_pfe/src/setup.rs:620-631)."""
        alpha = [(r + self.alpha_shift_small) % R for r in root_domain_prefix(self._batch_size, self._batch_size)]
        vals = [(self.rho + a) % R for a in alpha]
        if any(v == 0 for v in vals):
            raise E.InvalidSecretKey()
        return [_inv(v) for v in vals]


@dataclass
class KeyMaterial:
    encryption_key: EncryptionKey
    decryption_key: PublicDecryptionKey
    party_keys: List[PartySecretKey]


def _validate_config(config: KeygenConfig):
    if not _is_pow2(config.batch_size):
        raise E.InvalidBatchSize(config.batch_size)
    if not config.party_weights:
        raise E.EmptyCommittee()
    for j, w in enumerate(config.party_weights):
        if w == 0:
            raise E.InvalidPartyWeight(j, w)
    W = sum(config.party_weights)
    if config.threshold_weight >= W:
        raise E.InvalidCommittee(len(config.party_weights), W, config.threshold_weight)
    domain = 1 << (W - 1).bit_length() if W > 1 else 1
    if domain > (1 << 32):
        raise E.InvalidEvaluationDomain(W)
    return W, domain


def keygen_with_rng(config: KeygenConfig, rng) -> KeyMaterial:
    """Trusted setup (weighted_pfe/src/setup.rs:149-354).  Scalar draws follow
    the reference: the nonzero master secret, t polynomial coefficients, the
    global masks (rejection-sampled), then one rho per party (rejection-sampled
    so that every rho_j + alpha_i is nonzero and distinct).  The fractions and
    the B (N + 2W) fixed-base G2 products run on the GPU."""
    W, domain = _validate_config(config)
    B, N, t = config.batch_size, len(config.party_weights), config.threshold_weight
    z = sample_nonzero(rng)
    coeffs = [z] + [random_scalar(rng) for _ in range(t)]
    shares = wb.scalar_fft(coeffs, domain)[:W] if domain > 1 else [z]
    evaluation_domain = root_domain_prefix(domain, W)
    offsets = np.zeros(N + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(config.party_weights)
    owner = np.repeat(np.arange(N, dtype=np.int32), config.party_weights)
    alpha, shift = shifted_alpha_points(B)
    while True:
        bm1, b0 = random_scalar(rng), random_scalar(rng)
        if b0 != 0 and (bm1 + b0) % R != 0:
            break
    occupied, rhos = set(), []
    for _ in range(N):
        while True:
            rho = random_scalar(rng)
            labels = [(rho + a) % R for a in alpha]
            if any(x == 0 for x in labels) or any(x in occupied for x in labels):
                continue
            occupied.update(labels)
            rhos.append(rho)
            break
    ctx = wb._ctx()
    g = wb.empty_device(32 * B * N)
    u = wb.empty_device(32 * B * N)
    alpha_b = ops.scalars_bytes(alpha)
    ctx.call("wbte_wpfe_fractions", g, u, ops.scalars_bytes(rhos), alpha_b, ops.scalars_bytes([bm1, b0]), N, B, 0)
    vk = wb.empty_device(G2B * B * N)
    d1 = wb.empty_device(G2B * B * W)
    d2 = wb.empty_device(G2B * B * W)
    ctx.call("wbte_wpfe_keygen_material", ops.scalars_bytes(shares), _lib.i32_array(owner), g, u, W, N, B, vk, d1, d2)
    V = wb.to_device(ops.g2_mul_generator([z * (bm1 + b0) % R]))
    element = ops.gt_pow(wb.gt_generator(), [z * b0 % R], fixed_base=True)
    h = hashlib.sha256()
    h.update(SETUP_ID_DOMAIN)
    for v in (B, t, domain, shift, N):
        h.update(struct.pack("<Q", v))
    for w in config.party_weights:
        h.update(struct.pack("<Q", w))
    h.update(ops.scalars_bytes(evaluation_domain))
    h.update(ops.scalars_bytes(alpha))
    target = _append_gt_fixed_many(element, 1)[0]
    h.update(struct.pack("<Q", len(target)))
    h.update(target)
    for arr, count in ((vk, B * N), (d1, B * W), (d2, B * W), (V, 1)):
        _hash_compressed_g2(h, arr, count)
    setup_id = h.digest()
    dk = PublicDecryptionKey(setup_id, B, t, W, domain, config.party_weights, offsets, evaluation_domain, alpha, shift,
                             vk, d1, d2, V)
    parties = [PartySecretKey(j, setup_id, B, shift, rho) for j, rho in enumerate(rhos)]
    return KeyMaterial(EncryptionKey(B, element, setup_id), dk, parties)


def _hash_compressed_g2(h, points_dev, count: int, chunk: int = 1 << 20):
    """h.update of the compressed encodings of `count` device G2 points, in
    chunks (the key material of large classes runs to tens of GB)."""
    for i in range(0, count, chunk):
        n = min(chunk, count - i)
        h.update(ops.g2_compress(points_dev[G2B * i : G2B * (i + n)], n))


def keygen(batch_size: int, party_weights: Sequence[int], threshold_weight: int) -> KeyMaterial:
    return keygen_with_rng(KeygenConfig(batch_size, list(party_weights), threshold_weight), OsRng())


# ------------------------------------------------------------- encryption
SchnorrProof = wb.SchnorrProof


@dataclass
class Ciphertext:
    first: bytes  # G1 affine
    second: bytes  # GT
    proof: SchnorrProof

    def verify(self, encryption_key: EncryptionKey) -> bool:
        ch = _challenges(encryption_key.setup_id(), *_encodings([self])[2:])
        out = np.zeros(1, dtype=np.uint8)
        ops.ctx().call("wbte_schnorr_verify", out, self.first, self.proof.commitment,
                       ops.scalars_bytes([self.proof.response]), ops.scalars_bytes(ch), 1)
        return bool(out[0])


def _encodings(cts):
    n = len(cts)
    first = b"".join(c.first for c in cts)
    comm = b"".join(c.proof.commitment for c in cts)
    second = b"".join(c.second for c in cts)
    return (first, comm, ops.split(ops.g1_compress(first, n), 48), ops.split(ops.g1_compress(comm, n), 48),
            _append_gt_fixed_many(second, n))


def _challenges(setup_id: bytes, first_c, comm_c, targets) -> List[int]:
    """Fiat-Shamir challenges with rejection sampling (weighted_pfe/src/proof.rs:124-152),
    hashed on the device: domain, setup id, compressed generator, then per
    ciphertext its compressed first component, the encoded target's length
    (u64 LE, always 289) and fixed-width encoding, and the compressed commitment."""
    n = len(first_c)
    if n == 0:
        return []
    prefix = TRANSCRIPT_DOMAIN + setup_id + ops.g1_compress(wb.g1_generator(), 1)
    tlen = struct.pack("<Q", 289)
    return ops.transcript_challenges([(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES),
                                      (b"".join(first_c), 48, 48, _lib.TRANSCRIPT_BYTES),
                                      (tlen, 0, 8, _lib.TRANSCRIPT_BYTES),
                                      (b"".join(targets), 289, 289, _lib.TRANSCRIPT_BYTES),
                                      (b"".join(comm_c), 48, 48, _lib.TRANSCRIPT_BYTES)], n)


def encrypt_many(encryption_key: EncryptionKey, messages: Sequence[bytes], rng) -> List[Ciphertext]:
    """Batched `encrypt_with_rng` (weighted_pfe/src/encryption.rs:22-36): per
    message a nonzero randomness, then the proof nonce, in order."""
    n = len(messages)
    if n == 0:
        return []
    rs, ks = [], []
    for _ in range(n):
        rs.append(sample_nonzero(rng))
        ks.append(random_scalar(rng))
    first = ops.g1_mul_generator(rs)
    comm = ops.g1_mul_generator(ks)
    second = ops.fp12_mul(b"".join(messages), ops.gt_pow(encryption_key.element(), rs, fixed_base=True))
    first_c = ops.split(ops.g1_compress(first, n), 48)
    comm_c = ops.split(ops.g1_compress(comm, n), 48)
    cs = _challenges(encryption_key.setup_id(), first_c, comm_c, _append_gt_fixed_many(second, n))
    return [Ciphertext(first[G1B * i : G1B * (i + 1)], second[GTB * i : GTB * (i + 1)],
                       SchnorrProof(comm[G1B * i : G1B * (i + 1)], (ks[i] + cs[i] * rs[i]) % R)) for i in range(n)]


def encrypt_with_rng(encryption_key: EncryptionKey, message: bytes, rng) -> Ciphertext:
    return encrypt_many(encryption_key, [message], rng)[0]


def encrypt(encryption_key: EncryptionKey, message: bytes) -> Ciphertext:
    return encrypt_with_rng(encryption_key, message, OsRng())


def batch_digest(cts, encodings=None) -> bytes:
    """weighted_pfe/src/decryption.rs:851-861."""
    _, _, first_c, comm_c, targets = encodings or _encodings(cts)
    body = [struct.pack("<Q", len(cts))]
    for i, ct in enumerate(cts):
        body.append(first_c[i] + targets[i] + comm_c[i] + wb.fr_bytes(ct.proof.response))
    return hashlib.sha256(BATCH_DIGEST_DOMAIN + b"".join(body)).digest()


# -------------------------------------------------------------- decryption
@dataclass
class ValidatedBatch:
    _setup_id: bytes
    _batch_size: int
    _digest: bytes
    first_dev: object  # device, B G1

    def setup_id(self) -> bytes:
        return self._setup_id

    def batch_size(self) -> int:
        return self._batch_size

    def digest(self) -> bytes:
        return self._digest

    @classmethod
    def verify(cls, encryption_key: EncryptionKey, ciphertexts: Sequence[Ciphertext]) -> "ValidatedBatch":
        return validate_batch(encryption_key, ciphertexts)


def validate_batch(encryption_key: EncryptionKey, ciphertexts: Sequence[Ciphertext], rng=None) -> ValidatedBatch:
    """weighted_pfe/src/decryption.rs:99-157: the exact-size batch is accepted
    only if the random-linear aggregate of all Schnorr equations holds
    (proof.rs:74-122)."""
    if len(ciphertexts) == 0:
        raise E.BatchIsEmpty()
    if len(ciphertexts) != encryption_key.batch_size():
        raise E.MismatchedBatchSize(encryption_key.batch_size(), len(ciphertexts))
    enc = _encodings(ciphertexts)
    first, comm, first_c, comm_c, targets = enc
    cs = _challenges(encryption_key.setup_id(), first_c, comm_c, targets)
    rng = rng or OsRng()
    coef = [sample_nonzero(rng) for _ in ciphertexts]
    gen_s = sum(a * ct.proof.response for a, ct in zip(coef, ciphertexts)) % R
    scal = [gen_s] + [(-a) % R for a in coef] + [(-a * c) % R for a, c in zip(coef, cs)]
    if ops.g1_msm(wb.g1_generator() + comm + first, scal) != G1_IDENTITY:
        raise E.InvalidProof()
    return ValidatedBatch(encryption_key.setup_id(), len(ciphertexts), batch_digest(ciphertexts, enc),
                          wb.to_device(first))


def _device_arrays(cts):
    """(first, commitment, second, responses) of one batch as device arrays
    (first three) and host ints; `cts` is a list of Ciphertext or a
    weighted_btx.CiphertextBatch (same fields, already in HBM)."""
    if isinstance(cts, wb.CiphertextBatch):
        n = len(cts)
        return cts.first[: G1B * n], cts.commitment[: G1B * n], cts.second[: GTB * n], list(cts.responses)
    return (wb.to_device(b"".join(c.first for c in cts)), wb.to_device(b"".join(c.proof.commitment for c in cts)),
            wb.to_device(b"".join(c.second for c in cts)), [c.proof.response for c in cts])


def validate_batches(encryption_key: EncryptionKey, batches: Sequence, rng=None, arrays=None) -> list:
    """`validate_batch` for K batches of the key's batch size in one pass on
    the device: every ciphertext's encodings and Fiat-Shamir challenge in one
    launch each, and the K random-linear Schnorr aggregates
    (weighted_pfe/src/proof.rs:74-122) as one family of K G1 MSMs of 2B + 1
    terms.  Entry b is the ValidatedBatch of batch b, or the error that
    validate_batch raises for it alone (a batch is rejected as a whole).
    `arrays`: the batches' _device_arrays when the caller has them already."""
    torch = wb._t()
    K = len(batches)
    if K == 0:
        return []
    B = encryption_key.batch_size()
    out: list = [None] * K
    live = []
    for b, cts in enumerate(batches):
        if len(cts) == 0:
            out[b] = E.BatchIsEmpty()
        elif len(cts) != B:
            out[b] = E.MismatchedBatchSize(B, len(cts))
        else:
            live.append(b)
    if not live:
        return out
    arrays = [arrays[b] if arrays is not None else _device_arrays(batches[b]) for b in live]
    n = B * len(live)
    first_all = torch.cat([a[0] for a in arrays])
    comm_all = torch.cat([a[1] for a in arrays])
    second_all = torch.cat([a[2] for a in arrays])
    responses = [r for a in arrays for r in a[3]]
    fc, te, cc = wb._encode_on_device(first_all, comm_all, second_all, n)
    prefix = TRANSCRIPT_DOMAIN + encryption_key.setup_id() + ops.g1_compress(wb.g1_generator(), 1)
    ch = ops.transcript_challenges([(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES),
                                    (fc, 48, 48, _lib.TRANSCRIPT_BYTES),
                                    (struct.pack("<Q", 289), 0, 8, _lib.TRANSCRIPT_BYTES),
                                    (te, 289, 289, _lib.TRANSCRIPT_BYTES),
                                    (cc, 48, 48, _lib.TRANSCRIPT_BYTES)], n)
    rng = rng or OsRng()
    scalars = []
    for q in range(len(live)):
        coef = [sample_nonzero(rng) for _ in range(B)]
        resp = responses[q * B : (q + 1) * B]
        chq = ch[q * B : (q + 1) * B]
        gen_s = sum(a * r for a, r in zip(coef, resp)) % R
        scalars += [gen_s] + [(-a) % R for a in coef] + [(-a * c) % R for a, c in zip(coef, chq)]
    g = wb.to_device(wb.g1_generator())
    pts = torch.cat([t for q in range(len(live))
                     for t in (g[:G1B], comm_all[G1B * B * q : G1B * B * (q + 1)],
                               first_all[G1B * B * q : G1B * B * (q + 1)])])
    n1 = 2 * B + 1
    agg = ops.msm_family(1, pts, n1 * len(live), [q * n1 for q in range(len(live))], None, scalars,
                         list(range(len(live))), len(live), n1)
    rec = wb._records_host(fc, te, cc, wb.to_device(ops.scalars_bytes(responses)), n)
    for q, b in enumerate(live):
        if agg[G1B * q : G1B * (q + 1)] != G1_IDENTITY:
            out[b] = E.InvalidProof()
            continue
        body = struct.pack("<Q", B) + rec[q * B : (q + 1) * B].tobytes()
        digest = hashlib.sha256(BATCH_DIGEST_DOMAIN + body).digest()
        out[b] = ValidatedBatch(encryption_key.setup_id(), B, digest, first_all[G1B * B * q : G1B * B * (q + 1)])
    return out


@dataclass
class DecryptionShare:
    party_index: int
    sigma: bytes  # G1 affine
    batch_digest: bytes
    setup_id: bytes


def partial_decrypt_many(party_keys: Sequence[PartySecretKey], batch: ValidatedBatch,
                         decryption_key: PublicDecryptionKey = None) -> List[DecryptionShare]:
    """`partial_decrypt` for several parties in one launch sequence
    (weighted_pfe/src/decryption.rs:231-252)."""
    for pk in party_keys:
        if pk.setup_id() != batch.setup_id():
            raise E.MismatchedSetup()
        if pk.batch_size() != batch.batch_size():
            raise E.MismatchedBatchSize(pk.batch_size(), batch.batch_size())
    T = len(party_keys)
    if T == 0:
        return []
    B = batch.batch_size()
    alpha = [(r + party_keys[0].alpha_shift_small) % R for r in root_domain_prefix(B, B)]
    for pk in party_keys:
        if any((pk.rho + a) % R == 0 for a in alpha):
            raise E.InvalidSecretKey()
    sig = bytearray(G1B * T)
    wb._ctx().call("wbte_wpfe_partial_decrypt", sig, batch.first_dev, ops.scalars_bytes([pk.rho for pk in party_keys]),
                   ops.scalars_bytes(alpha), T, B)
    return [DecryptionShare(pk.party_index, bytes(sig[G1B * j : G1B * (j + 1)]), batch.digest(), batch.setup_id())
            for j, pk in enumerate(party_keys)]


def partial_decrypt_batches(party_keys: Sequence[PartySecretKey], batches: Sequence[ValidatedBatch]):
    """`partial_decrypt` of every party for K validated batches of one size in
    one launch sequence (wbte_wpfe_partial_decrypt_many): shares[b][j] is party
    j's share of batch b, equal to partial_decrypt(party_keys[j], batches[b])."""
    torch = wb._t()
    K = len(batches)
    if K == 0 or not party_keys:
        return [[] for _ in range(K)]
    B = batches[0].batch_size()
    for bt in batches:
        if bt.batch_size() != B:
            raise E.MismatchedBatchSize(B, bt.batch_size())
        for pk in party_keys:
            if pk.setup_id() != bt.setup_id():
                raise E.MismatchedSetup()
    for pk in party_keys:
        if pk.batch_size() != B:
            raise E.MismatchedBatchSize(pk.batch_size(), B)
    T = len(party_keys)
    alpha = [(r + party_keys[0].alpha_shift_small) % R for r in root_domain_prefix(B, B)]
    for pk in party_keys:
        if any((pk.rho + a) % R == 0 for a in alpha):
            raise E.InvalidSecretKey()
    first = torch.cat([bt.first_dev[: G1B * B] for bt in batches])
    sig = bytearray(G1B * T * K)
    wb._ctx().call("wbte_wpfe_partial_decrypt_many", sig, first, ops.scalars_bytes([pk.rho for pk in party_keys]),
                   ops.scalars_bytes(alpha), T, B, K)
    return [[DecryptionShare(pk.party_index, bytes(sig[G1B * (b * T + j) : G1B * (b * T + j + 1)]),
                             batches[b].digest(), batches[b].setup_id()) for j, pk in enumerate(party_keys)]
            for b in range(K)]


def partial_decrypt(party_key: PartySecretKey, batch: ValidatedBatch) -> DecryptionShare:
    return partial_decrypt_many([party_key], batch)[0]


def _ensure_key_batch(dk: PublicDecryptionKey, batch: ValidatedBatch):
    if dk.setup_id() != batch.setup_id():
        raise E.MismatchedSetup()
    if dk.batch_size() != batch.batch_size():
        raise E.MismatchedBatchSize(dk.batch_size(), batch.batch_size())


def _verify_shares(dk, batch, shares, challenges) -> bool:
    ok = np.zeros(1, dtype=np.int32)
    wb._ctx().call("wbte_wpfe_verify_shares", ok, dk.abi_key(), batch.first_dev, b"".join(s.sigma for s in shares),
                   _lib.i64_array([s.party_index for s in shares]), ops.scalars_bytes(challenges), len(shares))
    return bool(ok[0])


def verify_decryption_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                            share: DecryptionShare) -> bool:
    """weighted_pfe/src/decryption.rs:254-275."""
    _ensure_key_batch(decryption_key, batch)
    if share.party_index >= decryption_key.party_count():
        raise E.InvalidPartyIndex(share.party_index)
    if share.setup_id != batch.setup_id() or share.batch_digest != batch.digest():
        return False
    return _verify_shares(decryption_key, batch, [share], [1])


@dataclass
class AcceptedDecryptionShares:
    setup_id: bytes
    batch_size: int
    digest: bytes
    _accepted_weight: int
    _shares: List[DecryptionShare]
    _rejected: List[int]

    def accepted_weight(self) -> int:
        return self._accepted_weight

    def party_count(self) -> int:
        return len(self._shares)

    def party_indices(self) -> List[int]:
        return [s.party_index for s in self._shares]

    def shares(self) -> List[DecryptionShare]:
        return list(self._shares)

    def rejected_parties(self) -> List[int]:
        return list(self._rejected)


def accept_decryption_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                             shares: Sequence[DecryptionShare], rng=None) -> AcceptedDecryptionShares:
    """weighted_pfe/src/decryption.rs:277-365: batched check, per-share blame
    on failure, weight check, then the minimum-cardinality heaviest-first
    authorized subset."""
    candidates, rejected = screen_shares(decryption_key, batch, shares)
    rng = rng or OsRng()
    ok = True
    if candidates:
        ok = _verify_shares(decryption_key, batch, candidates, [sample_nonzero(rng) for _ in candidates])
    return finish_acceptance(decryption_key, batch, candidates, rejected, ok)


def screen_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, shares: Sequence[DecryptionShare]):
    """The structural checks of accept_decryption_shares (weighted_pfe/src/decryption.rs:277-300):
    returns (candidates bound to this batch and setup, rejected party indices)."""
    _ensure_key_batch(decryption_key, batch)
    N = decryption_key.party_count()
    if len(shares) > N:
        raise E.TooManyShares(len(shares), N)
    seen = [False] * N
    candidates, rejected = [], []
    for s in shares:
        if s.party_index >= N:
            raise E.InvalidPartyIndex(s.party_index)
        if seen[s.party_index]:
            raise E.DuplicatePartyIndex(s.party_index)
        seen[s.party_index] = True
        if s.setup_id == batch.setup_id() and s.batch_digest == batch.digest():
            candidates.append(s)
        else:
            rejected.append(s.party_index)
    return candidates, rejected


def finish_acceptance(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, candidates, rejected,
                      aggregate_ok: bool) -> AcceptedDecryptionShares:
    """The rest of accept_decryption_shares (weighted_pfe/src/decryption.rs:300-365)
    once the aggregate check has run: per-share blame on failure, weight check,
    minimum heaviest-first authorized subset."""
    rejected = list(rejected)
    if aggregate_ok:
        valid = list(candidates)
    else:
        valid = []
        for s in candidates:
            if verify_decryption_share(decryption_key, batch, s):
                valid.append(s)
            else:
                rejected.append(s.party_index)
    weights = decryption_key.party_weights()
    weight = sum(weights[s.party_index] for s in valid)
    rejected.sort()
    if weight <= decryption_key.threshold_weight():
        raise E.InsufficientWeight(weight, decryption_key.required_weight(), rejected)
    valid.sort(key=lambda s: (-weights[s.party_index], s.party_index))
    selected, acc = [], 0
    for s in valid:
        if acc > decryption_key.threshold_weight():
            break
        acc += weights[s.party_index]
        selected.append(s)
    selected.sort(key=lambda s: s.party_index)
    return AcceptedDecryptionShares(batch.setup_id(), batch.batch_size(), batch.digest(), acc, selected, rejected)


class CauchyKernel:
    """Fixed Cauchy transform data of one setup (weighted_pfe/src/decryption.rs:194-213):
    the spectrum 2(B - 1 - 2k)/2 lives in the precompute call."""

    def __init__(self, decryption_key: PublicDecryptionKey):
        B = decryption_key.batch_size()
        if not _is_pow2(B):
            raise E.InvalidBatchSize(B)
        self.setup_id = decryption_key.setup_id()
        self._batch_size = B
        self.frequency_coefficients = [B - 1 - 2 * k for k in range(B)]
        self.two_batch_small = 2 * B

    @classmethod
    def new(cls, decryption_key: PublicDecryptionKey) -> "CauchyKernel":
        return cls(decryption_key)

    def batch_size(self) -> int:
        return self._batch_size


def committee_context_id(setup_id: bytes, party_indices: Sequence[int]) -> bytes:
    """weighted_pfe/src/decryption.rs:840-849."""
    h = hashlib.sha256()
    h.update(COMMITTEE_CONTEXT_DOMAIN)
    h.update(setup_id)
    h.update(struct.pack("<Q", len(party_indices)))
    for j in party_indices:
        h.update(struct.pack("<Q", j))
    return h.digest()


@dataclass
class DecryptionPrecomputation:
    setup_id: bytes
    context_id: bytes
    batch_size: int
    _accepted_weight: int
    party_indices: List[int]
    scaled_d1_by_party: object  # device, B * T G2
    total_lines: object  # device, B line tables
    mask_lines: object  # device, B line tables
    scaled_d1_total: object  # device, B G2
    mask_keys: object  # device, B G2

    def accepted_weight(self) -> int:
        return self._accepted_weight

    def party_count(self) -> int:
        return len(self.party_indices)


def prepare_decryption(decryption_key: PublicDecryptionKey,
                       accepted: AcceptedDecryptionShares) -> DecryptionPrecomputation:
    """weighted_pfe/src/decryption.rs:421-538 (committee-dependent G2 work, reusable)."""
    if decryption_key.setup_id() != accepted.setup_id or decryption_key.batch_size() != accepted.batch_size:
        raise E.MismatchedSetup()
    if accepted.accepted_weight() <= decryption_key.threshold_weight():
        raise E.InsufficientWeight(accepted.accepted_weight(), decryption_key.required_weight(), [])
    B = decryption_key.batch_size()
    parties = accepted.party_indices()
    T = len(parties)
    alpha = decryption_key.alpha_points()
    mask_scalars = [a * (a + 1) % R for a in alpha] + [(-a) % R for a in alpha]
    line_bytes = _lib.LINE_BYTES * _lib.MILLER_LINES * B
    by_party, total_lines, mask_lines = wb.empty_device(G2B * B * T), wb.empty_device(line_bytes), wb.empty_device(line_bytes)
    total, mask = wb.empty_device(G2B * B), wb.empty_device(G2B * B)
    try:
        wb._ctx().call("wbte_wpfe_prepare", decryption_key.abi_key(), _lib.i64_array(parties), T,
                       ops.scalars_bytes(mask_scalars), by_party, total_lines, mask_lines, total, mask)
    except _lib.WbteError as exc:
        if exc.status == -7:
            raise E.InvalidInterpolationSet() from exc
        raise
    return DecryptionPrecomputation(accepted.setup_id, committee_context_id(accepted.setup_id, parties), B,
                                    accepted.accepted_weight(), parties, by_party, total_lines, mask_lines, total, mask)


@dataclass
class BatchPrecomputation:
    setup_id: bytes
    context_id: bytes
    batch_size: int
    digest: bytes
    scaled_first_cauchy: object  # device, B G1
    pairing_cauchy: object  # device, B Fp12 (cyclotomic; canonical after the hard part)


def _ensure_precomputation_batch(kernel: CauchyKernel, decryption: DecryptionPrecomputation, batch: ValidatedBatch):
    if kernel.setup_id != batch.setup_id() or decryption.setup_id != batch.setup_id():
        raise E.MismatchedSetup()
    if kernel.batch_size() != batch.batch_size() or decryption.batch_size != batch.batch_size():
        raise E.MismatchedBatchSize(kernel.batch_size(), batch.batch_size())


def precompute_batch(kernel: CauchyKernel, decryption: DecryptionPrecomputation,
                     batch: ValidatedBatch) -> BatchPrecomputation:
    """weighted_pfe/src/decryption.rs:540-574."""
    _ensure_precomputation_batch(kernel, decryption, batch)
    B = batch.batch_size()
    fc, pc = wb.empty_device(G1B * B), wb.empty_device(GTB * B)
    wb._ctx().call("wbte_wpfe_precompute", fc, pc, batch.first_dev, decryption.total_lines, B)
    return BatchPrecomputation(batch.setup_id(), decryption.context_id, B, batch.digest(), fc, pc)


def open_batch(decryption_key: PublicDecryptionKey, kernel: CauchyKernel, decryption: DecryptionPrecomputation,
               accepted: AcceptedDecryptionShares, batch: ValidatedBatch, ciphertexts: Sequence[Ciphertext],
               precomputation: BatchPrecomputation, device_output: bool = False):
    """weighted_pfe/src/decryption.rs:576-644 with the bindings of :793-830."""
    _ensure_key_batch(decryption_key, batch)
    _ensure_precomputation_batch(kernel, decryption, batch)
    if accepted.setup_id != batch.setup_id() or precomputation.setup_id != batch.setup_id():
        raise E.MismatchedSetup()
    if (accepted.batch_size != batch.batch_size() or len(ciphertexts) != batch.batch_size()
            or precomputation.batch_size != batch.batch_size()):
        raise E.MismatchedBatchSize(batch.batch_size(), len(ciphertexts))
    if accepted.digest != batch.digest() or precomputation.digest != batch.digest() \
            or batch_digest(ciphertexts) != batch.digest():
        raise E.MismatchedBatchDigest()
    parties = accepted.party_indices()
    if (parties != decryption.party_indices
            or committee_context_id(accepted.setup_id, parties) != decryption.context_id
            or precomputation.context_id != decryption.context_id):
        raise E.MismatchedCommittee()
    B, T = batch.batch_size(), accepted.party_count()
    alpha = decryption_key.alpha_points()
    out = wb.empty_device(GTB * B) if device_output else bytearray(GTB * B)
    wb._ctx().call("wbte_wpfe_open", out, b"".join(s.sigma for s in accepted.shares()), T, decryption.scaled_d1_by_party,
                   batch.first_dev, decryption.mask_lines, precomputation.scaled_first_cauchy,
                   precomputation.pairing_cauchy, b"".join(c.second for c in ciphertexts),
                   ops.scalars_bytes([a * (a + 1) % R for a in alpha]), B)
    if device_output:
        return out
    return [bytes(out[GTB * i : GTB * (i + 1)]) for i in range(B)]


def decrypt(encryption_key: EncryptionKey, decryption_key: PublicDecryptionKey, ciphertexts: Sequence[Ciphertext],
            shares: Sequence[DecryptionShare], rng=None) -> List[bytes]:
    """weighted_pfe/src/decryption.rs:646-669."""
    if encryption_key.setup_id() != decryption_key.setup_id():
        raise E.MismatchedSetup()
    batch = validate_batch(encryption_key, ciphertexts, rng)
    accepted = accept_decryption_shares(decryption_key, batch, shares, rng)
    kernel = CauchyKernel(decryption_key)
    decryption = prepare_decryption(decryption_key, accepted)
    pre = precompute_batch(kernel, decryption, batch)
    return open_batch(decryption_key, kernel, decryption, accepted, batch, ciphertexts, pre)
