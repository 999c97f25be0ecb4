"""PFE: partial-fraction batch threshold encryption (Constructions 1-4) on B200.

Mirrors the public API of the reference crate `pfe` (pfe/src/lib.rs:16-26):
`keygen[_with_rng]`, `encrypt[_with_rng]`, `validate_batch`,
`PartialFractionKernel`, `precompute_batch`, `partial_decrypt`,
`combine_shares[_checked]`, `verify_decryption_share`,
`verify_combined_share`, `open_batch`.  The crate's `Error` variants are the
btx variants (pfe/src/error.rs:3-23), so this module raises the exception
classes of weighted_bte_b200.btx.

Group work runs in libwbte (the wbte_pfe_* calls of include/wbte.h and the
shared btx partial-decryption, combination and pairing-check calls); this
module holds the protocol logic, SHA-256 transcripts and the data layout.
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib, ops
from . import weighted_btx as wb
from .btx import (BatchIsEmpty, DuplicateServerIndex, Error, InsufficientShares, InvalidBatchSize,  # noqa: F401
                  InvalidCommittee, InvalidProof, InvalidServerIndex, InvalidShare, MismatchedBatchSize)
from .rng import OsRng, random_scalar, sample_nonzero

R = ops.R
G1B, G2B, GTB = wb.G1B, wb.G2B, wb.GTB
TRANSCRIPT_DOMAIN = b"PFE-CONSTRUCTION4-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"PFE-ORDERED-BATCH-BLS12381-v1"


def _inv(x: int) -> int:
    return pow(x % R, R - 2, R)


def _is_pow2(n: int) -> bool:
    return n > 0 and n & (n - 1) == 0


def index_points(batch_size: int) -> List[int]:
    """The B-th roots of unity in order (pfe/src/setup.rs:244-253)."""
    if not _is_pow2(batch_size):
        raise InvalidBatchSize(batch_size)
    g = wb.radix2_generator(batch_size) if batch_size > 1 else 1
    out, x = [], 1
    for _ in range(batch_size):
        out.append(x)
        x = x * g % R
    return out


def extra_index_data(batch_size: int):
    """(gamma, c): the smallest c >= 2 outside the slot subgroup, gamma = 1/c
    (pfe/src/setup.rs:255-273)."""
    if not _is_pow2(batch_size):
        raise InvalidBatchSize(batch_size)
    c = 2
    while pow(c, batch_size, R) == 1:
        c += 1
    return _inv(c), c


# ------------------------------------------------------------------- keys
@dataclass
class KeygenConfig:
    batch_size: int
    server_count: int
    threshold: int
    publish_share_commitments: bool = True


@dataclass
class EncryptionKey:
    batch_size: int
    relation_base: bytes  # G1: sum_a [1/(x + a)]
    masking_base: bytes  # GT: e(G1, G2)^(1/x)


class PublicDecryptionKey:
    """pfe/src/setup.rs:24-35 with the G2 material in HBM."""

    def __init__(self, batch_size, server_count, threshold, fraction_keys, fraction_key_sum, server_domain,
                 share_commitments):
        self._B, self._N, self._t = batch_size, server_count, threshold
        self.fraction_keys, self.fraction_key_sum = fraction_keys, fraction_key_sum
        self._domain = list(server_domain)
        self.share_commitments = share_commitments

    def batch_size(self) -> int:
        return self._B

    def server_count(self) -> int:
        return self._N

    def threshold(self) -> int:
        return self._t

    def required_shares(self) -> int:
        return self._t + 1

    def server_domain(self) -> List[int]:
        return list(self._domain)

    def has_share_commitments(self) -> bool:
        return self.share_commitments is not None

    def share_commitment_row(self, server_index: int):
        if server_index >= self._N:
            raise InvalidServerIndex(server_index)
        if self.share_commitments is None:
            raise InvalidShare()
        return self.share_commitments[G2B * self._B * server_index : G2B * self._B * (server_index + 1)]


@dataclass
class ServerSecretKey:
    server_index: int
    domain_point: int
    fraction_shares: List[int]

    def batch_size(self) -> int:
        return len(self.fraction_shares)


@dataclass
class KeyMaterial:
    encryption_key: EncryptionKey
    decryption_key: PublicDecryptionKey
    server_keys: List[ServerSecretKey]


def _poly_eval(coeffs: Sequence[int], x: int) -> int:
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % R
    return acc


def keygen_with_rng(config: KeygenConfig, rng) -> KeyMaterial:
    """Trusted-dealer setup (pfe/src/setup.rs:78-186): x resampled away from
    the poles 0, -gamma and -w^i, then per slot a degree-t sharing polynomial
    of 1/(x + w^i) with t random coefficients, drawn in that order."""
    if not _is_pow2(config.batch_size):
        raise InvalidBatchSize(config.batch_size)
    if config.server_count == 0 or config.threshold >= config.server_count:
        raise InvalidCommittee(config.server_count, config.threshold)
    B, N, t = config.batch_size, config.server_count, config.threshold
    pts = index_points(B)
    gamma, _ = extra_index_data(B)
    while True:
        x = random_scalar(rng)
        dens = [x, (x + gamma) % R] + [(x + p) % R for p in pts]
        if any(d == 0 for d in dens):
            continue
        invs = [_inv(d) for d in dens]
        break
    p_zero, fractions, rel = invs[0], invs[2:], sum(invs) % R
    relation_base = ops.g1_mul_generator([rel])
    masking_base = ops.gt_pow(wb.gt_generator(), [p_zero], fixed_base=True)
    keys = wb.empty_device(G2B * B)
    ops.g2_mul_generator(fractions, out=keys)
    key_sum = wb.to_device(ops.g2_sum(keys, [0, B]))
    domain = [j + 1 for j in range(N)]
    polys = [[f] + [random_scalar(rng) for _ in range(t)] for f in fractions]
    shares = [[_poly_eval(polys[i], domain[j]) for i in range(B)] for j in range(N)]
    commitments = None
    if config.publish_share_commitments:
        commitments = wb.empty_device(G2B * B * N)
        ops.g2_mul_generator([s for row in shares for s in row], out=commitments)
    dk = PublicDecryptionKey(B, N, t, keys, key_sum, domain, commitments)
    servers = [ServerSecretKey(j, domain[j], shares[j]) for j in range(N)]
    return KeyMaterial(EncryptionKey(B, relation_base, masking_base), dk, servers)


def keygen(batch_size: int, server_count: int, threshold: int) -> KeyMaterial:
    return keygen_with_rng(KeygenConfig(batch_size, server_count, threshold), OsRng())


# ------------------------------------------------------------- encryption
@dataclass
class DleqProof:
    response: int
    first_commitment: bytes  # G1 affine
    second_commitment: bytes  # G1 affine


@dataclass
class Ciphertext:
    first: bytes  # G1 affine: [r] G1
    second: bytes  # G1 affine: [r] relation_base
    third: bytes  # GT: message * masking_base^r
    proof: DleqProof

    def verify(self, encryption_key: EncryptionKey) -> bool:
        return _verify_proofs(encryption_key, [self], [1])


def _challenges(rb_c: bytes, first_c, second_c, c1_c, c2_c) -> List[int]:
    """Fiat-Shamir challenges with rejection sampling (pfe/src/proof.rs:148-176), hashed on
    the device: domain and compressed relation base, then per ciphertext four
    compressed G1 points."""
    n = len(first_c)
    if n == 0:
        return []
    prefix = TRANSCRIPT_DOMAIN + rb_c
    fields = [(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES)]
    fields += [(b"".join(x), 48, 48, _lib.TRANSCRIPT_BYTES) for x in (first_c, second_c, c1_c, c2_c)]
    return ops.transcript_challenges(fields, n)


def encrypt_many(encryption_key: EncryptionKey, messages: Sequence[bytes], rng) -> List[Ciphertext]:
    """Batched `encrypt_with_rng` (pfe/src/encryption.rs:23-41); draws
    (randomness, nonce) per message in order."""
    n = len(messages)
    if n == 0:
        return []
    rs, ks = [], []
    for _ in range(n):
        rs.append(random_scalar(rng))
        ks.append(random_scalar(rng))
    rb = encryption_key.relation_base
    first = ops.g1_mul_generator(rs)
    second = ops.g1_mul(rb, rs, fixed_base=True)
    third = ops.fp12_mul(b"".join(messages), ops.gt_pow(encryption_key.masking_base, rs, fixed_base=True))
    c1 = ops.g1_mul_generator(ks)
    c2 = ops.g1_mul(rb, ks, fixed_base=True)
    comp = lambda blob: ops.split(ops.g1_compress(blob, n), 48)  # noqa: E731
    cs = _challenges(ops.g1_compress(rb, 1), comp(first), comp(second), comp(c1), comp(c2))
    return [Ciphertext(first[G1B * i : G1B * (i + 1)], second[G1B * i : G1B * (i + 1)], third[GTB * i : GTB * (i + 1)],
                       DleqProof((ks[i] + cs[i] * rs[i]) % R, c1[G1B * i : G1B * (i + 1)], c2[G1B * i : G1B * (i + 1)]))
            for i in range(n)]


def encrypt_with_rng(encryption_key: EncryptionKey, message: bytes, rng) -> Ciphertext:
    return encrypt_many(encryption_key, [message], rng)[0]


def encrypt(encryption_key: EncryptionKey, message: bytes) -> Ciphertext:
    return encrypt_with_rng(encryption_key, message, OsRng())


def _verify_proofs(encryption_key: EncryptionKey, cts, weights) -> bool:
    """Both DLEQ equations, random-linearly aggregated (pfe/src/proof.rs:74-146)."""
    n = len(cts)
    rb = encryption_key.relation_base
    first = b"".join(c.first for c in cts)
    second = b"".join(c.second for c in cts)
    c1 = b"".join(c.proof.first_commitment for c in cts)
    c2 = b"".join(c.proof.second_commitment for c in cts)
    comp = lambda blob: ops.split(ops.g1_compress(blob, n), 48)  # noqa: E731
    cs = _challenges(ops.g1_compress(rb, 1), comp(first), comp(second), comp(c1), comp(c2))
    wc = [w * c % R for w, c in zip(weights, cs)]
    resp = sum(w * ct.proof.response for w, ct in zip(weights, cts)) % R
    scal = list(weights) + wc
    if ops.g1_msm(c1 + first, scal) != ops.g1_mul_generator([resp]):
        return False
    return ops.g1_msm(c2 + second, scal) == ops.g1_mul(rb, [resp], fixed_base=True)


def batch_digest(cts) -> bytes:
    """pfe/src/decryption.rs:633-645 over encryption.rs:48-55's canonical encoding."""
    n = len(cts)
    comp = lambda blob: ops.split(ops.g1_compress(blob, n), 48)  # noqa: E731
    f = comp(b"".join(c.first for c in cts))
    s = comp(b"".join(c.second for c in cts))
    c1 = comp(b"".join(c.proof.first_commitment for c in cts))
    c2 = comp(b"".join(c.proof.second_commitment for c in cts))
    third = wb.append_gt_many(b"".join(c.third for c in cts), n)
    body = [struct.pack("<Q", n)]
    for i, ct in enumerate(cts):
        body.append(f[i] + s[i] + third[i] + wb.fr_bytes(ct.proof.response) + c1[i] + c2[i])
    return hashlib.sha256(BATCH_DIGEST_DOMAIN + b"".join(body)).digest()


# -------------------------------------------------------------- decryption
@dataclass
class ValidatedBatch:
    _batch_size: int
    _digest: bytes
    first_dev: object  # device, B G1
    second_dev: object  # device, B G1
    valid_dev: object  # device, B ones

    def batch_size(self) -> int:
        return self._batch_size

    def digest(self) -> bytes:
        return self._digest

    @classmethod
    def verify(cls, encryption_key: EncryptionKey, ciphertexts) -> "ValidatedBatch":
        return _validated(encryption_key, ciphertexts, True)

    @classmethod
    def proofs_preverified(cls, encryption_key: EncryptionKey, ciphertexts) -> "ValidatedBatch":
        return _validated(encryption_key, ciphertexts, False)


def _validated(encryption_key, ciphertexts, verify_proofs: bool, rng=None) -> ValidatedBatch:
    """pfe/src/decryption.rs:85-138."""
    if len(ciphertexts) == 0:
        raise BatchIsEmpty()
    if len(ciphertexts) != encryption_key.batch_size:
        raise MismatchedBatchSize(encryption_key.batch_size, len(ciphertexts))
    if verify_proofs:
        rng = rng or OsRng()
        if not _verify_proofs(encryption_key, ciphertexts, [sample_nonzero(rng) for _ in ciphertexts]):
            raise InvalidProof()
    B = len(ciphertexts)
    return ValidatedBatch(B, batch_digest(ciphertexts), wb.to_device(b"".join(c.first for c in ciphertexts)),
                          wb.to_device(b"".join(c.second for c in ciphertexts)), wb.to_device(b"\x01" * B))


def validate_batch(encryption_key: EncryptionKey, ciphertexts, rng=None) -> ValidatedBatch:
    return _validated(encryption_key, ciphertexts, True, rng)


@dataclass
class DecryptionShare:
    server_index: int
    pre_decryption_key: bytes  # G1 affine
    batch_digest: bytes


@dataclass
class BatchPrecomputation:
    batch_size: int
    digest: bytes
    weighted_first: object  # device, B G1
    weighted_pairings: object  # device, B GT


class PartialFractionKernel:
    """All reusable domain and G2 preprocessing (pfe/src/decryption.rs:151-257),
    resident in HBM: line tables of DK_i/(2B), [s2_i] G2 and the fused third
    pairing operand."""

    def __init__(self, decryption_key: PublicDecryptionKey):
        B = decryption_key.batch_size()
        pts = index_points(B)
        gamma, c = extra_index_data(B)
        half_b1 = (B + 1) * _inv(2) % R
        inv2b = _inv(2 * B)
        s2 = [p * c % R for p in pts]
        s1_bar = [2 * B * (p * (s - 1)) % R for p, s in zip(pts, s2)]
        open_coef = [(_inv(p) * half_b1 + _inv(p - gamma)) % R for p in pts]
        coef = [(B - 1 - 2 * k) % R for k in range(B)]
        scalars = ([inv2b] * B + coef + [c] * B + s2 + [(-x) % R for x in s2]
                   + [(-sb * o) % R for sb, o in zip(s1_bar, open_coef)])
        lines = _lib.LINE_BYTES * _lib.MILLER_LINES * B
        self.key_lines, self.generator_lines, self.mix_lines = (wb.empty_device(lines) for _ in range(3))
        self.scaled_keys, self.generators, self.mixes = (wb.empty_device(G2B * B) for _ in range(3))
        wb._ctx().call("wbte_pfe_kernel", decryption_key.fraction_keys, decryption_key.fraction_key_sum, B,
                       ops.scalars_bytes(scalars), self.key_lines, self.generator_lines, self.mix_lines,
                       self.scaled_keys, self.generators, self.mixes)
        self._batch_size = B
        self.gamma_inverse_small = c
        self.frequency_coefficients = [B - 1 - 2 * k for k in range(B)]
        self.neg_scaled_s1 = ops.scalars_bytes([(-x) % R for x in s1_bar])
        self.conv_scalars = ops.scalars_bytes(coef + [c] * B)

    @classmethod
    def new(cls, decryption_key: PublicDecryptionKey) -> "PartialFractionKernel":
        return cls(decryption_key)

    def batch_size(self) -> int:
        return self._batch_size


def _ensure_kernel_batch(kernel: PartialFractionKernel, batch: ValidatedBatch):
    if kernel.batch_size() != batch.batch_size():
        raise MismatchedBatchSize(kernel.batch_size(), batch.batch_size())


def precompute_batch(kernel: PartialFractionKernel, batch: ValidatedBatch) -> BatchPrecomputation:
    """pfe/src/decryption.rs:259-298."""
    _ensure_kernel_batch(kernel, batch)
    B = batch.batch_size()
    wf, wp = wb.empty_device(G1B * B), wb.empty_device(GTB * B)
    wb._ctx().call("wbte_pfe_precompute", wf, wp, batch.first_dev, kernel.key_lines, kernel.conv_scalars, B)
    return BatchPrecomputation(B, batch.digest(), wf, wp)


def partial_decrypt(server_key: ServerSecretKey, batch: ValidatedBatch) -> DecryptionShare:
    """pfe/src/decryption.rs:300-319."""
    if server_key.batch_size() != batch.batch_size():
        raise MismatchedBatchSize(server_key.batch_size(), batch.batch_size())
    sigma = bytearray(G1B)
    wb._ctx().call("wbte_btx_partial_decrypt", sigma, batch.first_dev, ops.scalars_bytes(server_key.fraction_shares),
                   batch.batch_size())
    return DecryptionShare(server_key.server_index, bytes(sigma), batch.digest())


def _validate_share_set(dk: PublicDecryptionKey, batch: ValidatedBatch, shares):
    """pfe/src/decryption.rs:554-580."""
    if dk.batch_size() != batch.batch_size():
        raise MismatchedBatchSize(dk.batch_size(), batch.batch_size())
    if len(shares) < dk.required_shares():
        raise InsufficientShares(len(shares), dk.required_shares())
    seen = set()
    for s in shares:
        if s.batch_digest != batch.digest():
            raise InvalidShare()
        if s.server_index >= dk.server_count():
            raise InvalidServerIndex(s.server_index)
        if s.server_index in seen:
            raise DuplicateServerIndex(s.server_index)
        seen.add(s.server_index)


def combine_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                   shares: Sequence[DecryptionShare]) -> bytes:
    """pfe/src/decryption.rs:321-338."""
    _validate_share_set(decryption_key, batch, shares)
    domain = decryption_key.server_domain()
    out = bytearray(G1B)
    wb._ctx().call("wbte_btx_combine", out, b"".join(s.pre_decryption_key for s in shares),
                   ops.scalars_bytes([domain[s.server_index] for s in shares]), len(shares))
    return bytes(out)


def _pairing_check(batch: ValidatedBatch, slot_points, n_points: int, pdk: bytes) -> bool:
    ok = np.zeros(1, dtype=np.int32)
    wb._ctx().call("wbte_btx_verify", ok, batch.first_dev, batch.valid_dev, batch.batch_size(), slot_points, n_points,
                   pdk)
    return bool(ok[0])


def verify_decryption_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                            share: DecryptionShare) -> bool:
    """pfe/src/decryption.rs:372-397."""
    if share.batch_digest != batch.digest():
        return False
    if share.server_index >= decryption_key.server_count():
        raise InvalidServerIndex(share.server_index)
    if batch.batch_size() != decryption_key.batch_size():
        raise InvalidBatchSize(batch.batch_size())
    row = decryption_key.share_commitment_row(share.server_index)
    return _pairing_check(batch, row, decryption_key.batch_size(), share.pre_decryption_key)


def verify_combined_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, pdk: bytes) -> bool:
    """pfe/src/decryption.rs:399-415."""
    if decryption_key.batch_size() != batch.batch_size():
        raise MismatchedBatchSize(decryption_key.batch_size(), batch.batch_size())
    return _pairing_check(batch, decryption_key.fraction_keys, decryption_key.batch_size(), pdk)


def combine_shares_checked(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                           shares: Sequence[DecryptionShare]) -> bytes:
    """pfe/src/decryption.rs:340-370."""
    optimistic = combine_shares(decryption_key, batch, shares)
    if verify_combined_share(decryption_key, batch, optimistic):
        return optimistic
    if not decryption_key.has_share_commitments():
        raise InvalidShare()
    valid = [s for s in shares if verify_decryption_share(decryption_key, batch, s)]
    recovered = combine_shares(decryption_key, batch, valid)
    if verify_combined_share(decryption_key, batch, recovered):
        return recovered
    raise InvalidShare()


def open_batch(kernel: PartialFractionKernel, batch: ValidatedBatch, ciphertexts: Sequence[Ciphertext],
               precomputation: BatchPrecomputation, pre_decryption_key: bytes, device_output: bool = False):
    """pfe/src/decryption.rs:417-469: one GT message per slot."""
    _ensure_kernel_batch(kernel, batch)
    if len(ciphertexts) != batch.batch_size():
        raise MismatchedBatchSize(batch.batch_size(), len(ciphertexts))
    if precomputation.batch_size != batch.batch_size() or precomputation.digest != batch.digest():
        raise InvalidShare()
    B = batch.batch_size()
    out = wb.empty_device(GTB * B) if device_output else bytearray(GTB * B)
    wb._ctx().call("wbte_pfe_open", out, batch.first_dev, batch.second_dev, b"".join(c.third for c in ciphertexts),
                   precomputation.weighted_first, precomputation.weighted_pairings, pre_decryption_key,
                   kernel.neg_scaled_s1, kernel.key_lines, kernel.generator_lines, kernel.mix_lines, B)
    if device_output:
        return out
    return [bytes(out[GTB * i : GTB * (i + 1)]) for i in range(B)]


def decrypt(encryption_key: EncryptionKey, decryption_key: PublicDecryptionKey, ciphertexts,
            server_keys: Sequence[ServerSecretKey], kernel: Optional[PartialFractionKernel] = None) -> List[bytes]:
    """The reference's timed pipeline in one call: validate, precompute,
    partial decryption by the given servers, combine, open."""
    batch = validate_batch(encryption_key, ciphertexts)
    kernel = kernel or PartialFractionKernel(decryption_key)
    pre = precompute_batch(kernel, batch)
    shares = [partial_decrypt(k, batch) for k in server_keys]
    pdk = combine_shares(decryption_key, batch, shares)
    return open_batch(kernel, batch, ciphertexts, pre, pdk)
