"""BTX batched threshold encryption (unit-weight servers) on B200.

Mirrors the public API of the reference crate `btx` (btx/src/lib.rs:18-28):
`keygen[_with_rng]`, `encrypt[_with_rng]`, `validate_batch`,
`MiddleProductKernel`, `precompute_batch`, `partial_decrypt`,
`combine_shares[_checked]`, `verify_decryption_share`,
`verify_combined_share`, `open_batch`, with the reference's checks and its
`Error` variants (btx/src/error.rs:3-25, as exception classes below).

Group work runs in libwbte (include/wbte.h: the wbte_btx_* phase calls and
the shared primitives); this module holds the protocol logic, the SHA-256
transcripts and the data layout.  Key powers and share commitments are
resident in HBM.  Group elements are `bytes` in blst's memory layout; scalars
are Python ints.
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib, ops
from . import weighted_btx as wb
from .rng import OsRng, random_scalar, sample_nonzero

R = ops.R
G1B, G2B, GTB = wb.G1B, wb.G2B, wb.GTB
TRANSCRIPT_DOMAIN = b"BTX-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"BTX-ORDERED-BATCH-v1"
G1_IDENTITY = bytes(G1B)


# ----------------------------------------------------------------- errors
class Error(Exception):
    """The reference's `btx::Error` (btx/src/error.rs:3-25)."""


class BatchIsEmpty(Error):
    def __init__(self):
        super().__init__("the ciphertext batch is empty")


class BatchTooLarge(Error):
    def __init__(self, batch_size: int, max_batch_size: int):
        self.batch_size, self.max_batch_size = batch_size, max_batch_size
        super().__init__(f"batch size {batch_size} exceeds the configured maximum {max_batch_size}")


class InvalidBatchSize(Error):
    def __init__(self, size: int):
        self.size = size
        super().__init__(f"batch size {size} cannot be represented by the FFT domain")


class InvalidCommittee(Error):
    def __init__(self, server_count: int, threshold: int):
        self.server_count, self.threshold = server_count, threshold
        super().__init__(f"invalid committee: threshold {threshold} must be smaller than server count {server_count}")


class InvalidProof(Error):
    def __init__(self):
        super().__init__("ciphertext proof is invalid")


class InvalidServerIndex(Error):
    def __init__(self, index: int):
        self.index = index
        super().__init__(f"invalid server index {index}")


class InvalidShare(Error):
    def __init__(self):
        super().__init__("decryption share verification failed")


class InsufficientShares(Error):
    def __init__(self, supplied: int, required: int):
        self.supplied, self.required = supplied, required
        super().__init__(f"insufficient decryption shares: supplied {supplied}, require {required}")


class DuplicateServerIndex(Error):
    def __init__(self, index: int):
        self.index = index
        super().__init__(f"duplicate server index {index}")


class MismatchedBatchSize(Error):
    def __init__(self, expected: int, actual: int):
        self.expected, self.actual = expected, actual
        super().__init__(f"mismatched batch size: expected {expected}, got {actual}")


# ------------------------------------------------------------------- keys
@dataclass
class KeygenConfig:
    max_batch_size: int
    server_count: int
    threshold: int  # reconstruction takes threshold + 1 shares
    publish_share_commitments: bool = True


@dataclass
class EncryptionKey:
    max_batch_size: int
    element: bytes  # GT: e(G1, G2)^(tau^(L+1))


class PublicDecryptionKey:
    """btx/src/setup.rs:17-30: [tau^1..tau^L] G2, [tau^(L+2)..tau^(2L)] G2,
    the server domain 1..N and the optional share commitments
    [share_j(tau^i)] G2, all resident in HBM."""

    def __init__(self, max_batch_size, server_count, threshold, low_powers, high_powers, server_domain,
                 share_commitments):
        self._L, self._N, self._t = max_batch_size, server_count, threshold
        self.low_powers, self.high_powers = low_powers, high_powers
        self._domain = list(server_domain)
        self.share_commitments = share_commitments  # device N * L G2, or None

    def max_batch_size(self) -> int:
        return self._L

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

    def power(self, exponent: int) -> bytes:
        """[tau^exponent] G2 for exponent in 1..L or L+2..2L (setup.rs:214-222)."""
        L = self._L
        if 1 <= exponent <= L:
            return wb.to_host(self.low_powers[G2B * (exponent - 1) : G2B * exponent])
        if L + 2 <= exponent <= 2 * L:
            i = exponent - L - 2
            return wb.to_host(self.high_powers[G2B * i : G2B * (i + 1)])
        raise InvalidBatchSize(exponent)

    def centered_power(self, offset: int) -> bytes:
        exponent = self._L + 1 + offset
        if exponent <= 0:
            raise InvalidBatchSize(max(exponent, 0))
        return self.power(exponent)

    def share_commitment_row(self, server_index: int):
        if server_index >= self._N:
            raise InvalidServerIndex(server_index)
        if self.share_commitments is None:
            raise InvalidShare()
        return self.share_commitments[G2B * self._L * server_index : G2B * self._L * (server_index + 1)]


@dataclass
class ServerSecretKey:
    server_index: int
    domain_point: int
    shares: List[int]

    def max_batch_size(self) -> int:
        return len(self.shares)

    def shares_for_batch(self, batch_size: int) -> List[int]:
        if batch_size > len(self.shares):
            raise BatchTooLarge(batch_size, len(self.shares))
        return self.shares[:batch_size]


@dataclass
class KeyMaterial:
    encryption_key: EncryptionKey
    decryption_key: PublicDecryptionKey
    server_keys: List[ServerSecretKey]


def _validate_config(config: KeygenConfig):
    if config.max_batch_size == 0:
        raise BatchIsEmpty()
    if config.server_count == 0 or config.threshold >= config.server_count:
        raise InvalidCommittee(config.server_count, config.threshold)


def _poly_eval(coeffs: Sequence[int], x: int) -> int:
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % R
    return acc


def keygen_with_rng(config: KeygenConfig, rng) -> KeyMaterial:
    """Trusted-dealer setup (btx/src/setup.rs:92-178): nonzero tau, then per
    power i = 1..L a degree-t sharing polynomial with constant tau^i and t
    random coefficients, drawn in that order.  The fixed-base G2 products
    (2L - 1 powers and N L share commitments) run on the GPU."""
    _validate_config(config)
    L, N, t = config.max_batch_size, config.server_count, config.threshold
    tau = sample_nonzero(rng)
    powers = [1]
    for _ in range(2 * L):
        powers.append(powers[-1] * tau % R)
    element = ops.gt_pow(wb.gt_generator(), [powers[L + 1]], fixed_base=True)
    low = wb.empty_device(G2B * L)
    high = wb.empty_device(G2B * max(1, L - 1))
    ops.g2_mul_generator(powers[1 : L + 1], out=low)
    if L > 1:
        ops.g2_mul_generator(powers[L + 2 : 2 * L + 1], out=high)
    domain = [j + 1 for j in range(N)]
    polys = [[powers[i]] + [random_scalar(rng) for _ in range(t)] for i in range(1, L + 1)]
    shares = [[_poly_eval(polys[i], domain[j]) for i in range(L)] for j in range(N)]
    commitments = None
    if config.publish_share_commitments:
        commitments = wb.empty_device(G2B * L * N)
        ops.g2_mul_generator([s for row in shares for s in row], out=commitments)
    dk = PublicDecryptionKey(L, N, t, low, high, domain, commitments)
    servers = [ServerSecretKey(j, domain[j], shares[j]) for j in range(N)]
    return KeyMaterial(EncryptionKey(L, element), dk, servers)


def keygen(max_batch_size: int, server_count: int, threshold: int) -> KeyMaterial:
    return keygen_with_rng(KeygenConfig(max_batch_size, server_count, threshold), OsRng())


# ------------------------------------------------------------- encryption
SchnorrProof = wb.SchnorrProof


@dataclass
class Ciphertext:
    first: bytes  # G1 affine
    second: bytes  # GT
    proof: SchnorrProof

    def verify(self) -> bool:
        return bool(verify_ciphertexts([self])[0])


def _challenges(first_c: List[bytes], second_enc: List[bytes], comm_c: List[bytes]) -> List[int]:
    """Fiat-Shamir challenges with rejection sampling (btx/src/proof.rs:49-77), hashed on
    the device: domain, compressed generator, then per ciphertext its compressed
    first component, GT encoding and compressed commitment."""
    n = len(first_c)
    if n == 0:
        return []
    prefix = TRANSCRIPT_DOMAIN + ops.g1_compress(wb.g1_generator(), 1)
    te = b"".join(x if len(x) == 289 else x + bytes(289 - len(x)) for x in second_enc)
    return ops.transcript_challenges([(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES),
                                      (b"".join(first_c), 48, 48, _lib.TRANSCRIPT_BYTES),
                                      (te, 289, 289, _lib.TRANSCRIPT_GT_VARIABLE),
                                      (b"".join(comm_c), 48, 48, _lib.TRANSCRIPT_BYTES)], n)


def encrypt_many(encryption_key: EncryptionKey, messages: Sequence[bytes], rng) -> List[Ciphertext]:
    """Batched `encrypt_with_rng` (btx/src/encryption.rs:26-40); draws
    (randomness, nonce) per message in order, as sequential calls would."""
    n = len(messages)
    if n == 0:
        return []
    rs, ks = [], []
    for _ in range(n):
        rs.append(random_scalar(rng))
        ks.append(random_scalar(rng))
    first = ops.g1_mul_generator(rs)
    comm = ops.g1_mul_generator(ks)
    mask = ops.gt_pow(encryption_key.element, rs, fixed_base=True)
    second = ops.fp12_mul(b"".join(messages), mask)
    first_c = ops.split(ops.g1_compress(first, n), 48)
    comm_c = ops.split(ops.g1_compress(comm, n), 48)
    second_enc = wb.append_gt_many(second, n)
    cs = _challenges(first_c, second_enc, comm_c)
    return [Ciphertext(first[G1B * i : G1B * (i + 1)], second[GTB * i : GTB * (i + 1)],
                       SchnorrProof(comm[G1B * i : G1B * (i + 1)], (ks[i] + cs[i] * rs[i]) % R)) for i in range(n)]


def encrypt_with_rng(encryption_key: EncryptionKey, message: bytes, rng) -> Ciphertext:
    return encrypt_many(encryption_key, [message], rng)[0]


def encrypt(encryption_key: EncryptionKey, message: bytes) -> Ciphertext:
    return encrypt_with_rng(encryption_key, message, OsRng())


def _encodings(cts):
    n = len(cts)
    first = b"".join(c.first for c in cts)
    comm = b"".join(c.proof.commitment for c in cts)
    second = b"".join(c.second for c in cts)
    first_c = ops.split(ops.g1_compress(first, n), 48)
    comm_c = ops.split(ops.g1_compress(comm, n), 48)
    return first, comm, first_c, comm_c, wb.append_gt_many(second, n)


def verify_ciphertexts(cts: Sequence[Ciphertext], encodings=None) -> np.ndarray:
    """Batched `Ciphertext::verify` (btx/src/encryption.rs:43-45)."""
    if len(cts) == 0:
        return np.zeros(0, dtype=bool)
    first, comm, first_c, comm_c, second_enc = encodings or _encodings(cts)
    cs = _challenges(first_c, second_enc, comm_c)
    out = np.zeros(len(cts), dtype=np.uint8)
    ops.ctx().call("wbte_schnorr_verify", out, first, comm, ops.scalars_bytes([c.proof.response for c in cts]),
                   ops.scalars_bytes(cs), len(cts))
    return out.astype(bool)


def batch_digest(cts, encodings=None) -> bytes:
    """btx/src/decryption.rs:510-518."""
    _, _, first_c, comm_c, second_enc = encodings or _encodings(cts)
    h = hashlib.sha256()
    h.update(BATCH_DIGEST_DOMAIN)
    h.update(struct.pack("<Q", len(cts)))
    for i, ct in enumerate(cts):
        h.update(first_c[i] + second_enc[i] + comm_c[i] + wb.fr_bytes(ct.proof.response))
    return h.digest()


# -------------------------------------------------------------- decryption
@dataclass
class ValidatedBatch:
    _batch_size: int
    _digest: bytes
    valid: np.ndarray
    first_dev: object  # device, B G1 with the identity at invalid slots
    valid_dev: object  # device, B bytes

    def batch_size(self) -> int:
        return self._batch_size

    def digest(self) -> bytes:
        return self._digest

    def valid_mask(self) -> List[bool]:
        return [bool(v) for v in self.valid]

    def valid_count(self) -> int:
        return int(np.count_nonzero(self.valid))

    @classmethod
    def verify(cls, ciphertexts: Sequence[Ciphertext]) -> "ValidatedBatch":
        return _validated(ciphertexts, True)

    @classmethod
    def proofs_preverified(cls, ciphertexts: Sequence[Ciphertext]) -> "ValidatedBatch":
        return _validated(ciphertexts, False)


def _validated(ciphertexts, verify_proofs: bool) -> ValidatedBatch:
    """btx/src/decryption.rs:76-114: invalid slots stay in place as the identity."""
    if len(ciphertexts) == 0:
        raise BatchIsEmpty()
    enc = _encodings(ciphertexts)
    valid = verify_ciphertexts(ciphertexts, enc) if verify_proofs else np.ones(len(ciphertexts), dtype=bool)
    first = b"".join(ct.first if v else G1_IDENTITY for ct, v in zip(ciphertexts, valid))
    return ValidatedBatch(len(ciphertexts), batch_digest(ciphertexts, enc), valid, wb.to_device(first),
                          wb.to_device(valid.astype(np.uint8).tobytes()))


def validate_batch(ciphertexts: Sequence[Ciphertext]) -> ValidatedBatch:
    return _validated(ciphertexts, True)


@dataclass
class DecryptionShare:
    server_index: int
    sigma: bytes  # G1 affine
    batch_digest: bytes


@dataclass
class BatchPrecomputation:
    batch_size: int
    digest: bytes
    beta: object  # device, B GT


def transform_size_for(batch_size: int) -> int:
    return 1 << (2 * batch_size - 1).bit_length()


def _validate_batch_size(dk: PublicDecryptionKey, batch_size: int):
    if batch_size == 0:
        raise BatchIsEmpty()
    if batch_size > dk.max_batch_size():
        raise BatchTooLarge(batch_size, dk.max_batch_size())


class MiddleProductKernel:
    """Fixed, reusable G2 preprocessing for one batch size
    (btx/src/decryption.rs:131-190): line tables of the transformed centered
    kernel (scaled by 1/m) and of the opening powers, resident in HBM."""

    def __init__(self, decryption_key: PublicDecryptionKey, batch_size: int):
        _validate_batch_size(decryption_key, batch_size)
        B, L = batch_size, decryption_key.max_batch_size()
        m = transform_size_for(B)
        self._batch_size, self._transform_size = B, m
        self.kernel_lines = wb.empty_device(_lib.LINE_BYTES * _lib.MILLER_LINES * m)
        self.opening_lines = wb.empty_device(_lib.LINE_BYTES * _lib.MILLER_LINES * B)
        self.transformed_kernel = wb.empty_device(G2B * m)
        wb._ctx().call("wbte_btx_kernel", decryption_key.low_powers, decryption_key.high_powers, L, B,
                       self.kernel_lines, self.opening_lines, self.transformed_kernel)

    @classmethod
    def new(cls, decryption_key: PublicDecryptionKey, batch_size: int) -> "MiddleProductKernel":
        return cls(decryption_key, batch_size)

    def batch_size(self) -> int:
        return self._batch_size

    def transform_size(self) -> int:
        return self._transform_size


def _ensure_kernel_batch(kernel: MiddleProductKernel, batch: ValidatedBatch):
    if kernel.batch_size() != batch.batch_size():
        raise MismatchedBatchSize(kernel.batch_size(), batch.batch_size())


def precompute_batch(kernel: MiddleProductKernel, batch: ValidatedBatch) -> BatchPrecomputation:
    """btx/src/decryption.rs:201-246."""
    _ensure_kernel_batch(kernel, batch)
    B = batch.batch_size()
    beta = wb.empty_device(GTB * B)
    ones = wb.to_device(b"\x01" * B)  # the reference computes beta at every slot
    wb._ctx().call("wbte_btx_precompute", beta, kernel.kernel_lines, batch.first_dev, ones, B)
    return BatchPrecomputation(B, batch.digest(), beta)


def partial_decrypt(server_key: ServerSecretKey, batch: ValidatedBatch) -> DecryptionShare:
    """btx/src/decryption.rs:248-264."""
    scalars = server_key.shares_for_batch(batch.batch_size())
    sigma = bytearray(G1B)
    wb._ctx().call("wbte_btx_partial_decrypt", sigma, batch.first_dev, ops.scalars_bytes(scalars), batch.batch_size())
    return DecryptionShare(server_key.server_index, bytes(sigma), batch.digest())


def combine_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                   shares: Sequence[DecryptionShare]) -> bytes:
    """btx/src/decryption.rs:266-306: Lagrange at zero over the shares'
    server points, in the given order."""
    if len(shares) < decryption_key.required_shares():
        raise InsufficientShares(len(shares), decryption_key.required_shares())
    seen = set()
    for s in shares:
        if s.batch_digest != batch.digest():
            raise InvalidShare()
        if s.server_index >= decryption_key.server_count():
            raise InvalidServerIndex(s.server_index)
        if s.server_index in seen:
            raise DuplicateServerIndex(s.server_index)
        seen.add(s.server_index)
    domain = decryption_key.server_domain()
    out = bytearray(G1B)
    wb._ctx().call("wbte_btx_combine", out, b"".join(s.sigma for s in shares),
                   ops.scalars_bytes([domain[s.server_index] for s in shares]), len(shares))
    return bytes(out)


def _pairing_check(batch: ValidatedBatch, slot_points, n_points: int, sigma: bytes) -> bool:
    ok = np.zeros(1, dtype=np.int32)
    wb._ctx().call("wbte_btx_verify", ok, batch.first_dev, batch.valid_dev, batch.batch_size(), slot_points, n_points,
                   sigma)
    return bool(ok[0])


def verify_decryption_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                            share: DecryptionShare) -> bool:
    """btx/src/decryption.rs:340-370."""
    if share.batch_digest != batch.digest():
        return False
    if share.server_index >= decryption_key.server_count():
        raise InvalidServerIndex(share.server_index)
    if batch.batch_size() > decryption_key.max_batch_size():
        raise BatchTooLarge(batch.batch_size(), decryption_key.max_batch_size())
    row = decryption_key.share_commitment_row(share.server_index)
    return _pairing_check(batch, row, decryption_key.max_batch_size(), share.sigma)


def verify_combined_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, sigma: bytes) -> bool:
    """Optimistic aggregate check (btx/src/decryption.rs:372-400)."""
    _validate_batch_size(decryption_key, batch.batch_size())
    return _pairing_check(batch, decryption_key.low_powers, decryption_key.max_batch_size(), sigma)


def combine_shares_checked(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                           shares: Sequence[DecryptionShare]) -> bytes:
    """btx/src/decryption.rs:308-338: optimistic combine, then per-share
    checks against the share commitments and a second combine."""
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


def open_batch(kernel: MiddleProductKernel, batch: ValidatedBatch, ciphertexts: Sequence[Ciphertext],
               precomputation: BatchPrecomputation, sigma: bytes, device_output: bool = False):
    """btx/src/decryption.rs:402-458: one Optional[bytes] per slot (None at
    invalid slots), or with device_output=True a device array of B GT values
    (identity at invalid slots)."""
    _ensure_kernel_batch(kernel, batch)
    if len(ciphertexts) != batch.batch_size():
        raise MismatchedBatchSize(batch.batch_size(), len(ciphertexts))
    if precomputation.batch_size != batch.batch_size() or precomputation.digest != batch.digest():
        raise InvalidShare()
    B = batch.batch_size()
    second = b"".join(c.second for c in ciphertexts)
    out = wb.empty_device(GTB * B) if device_output else bytearray(GTB * B)
    wb._ctx().call("wbte_btx_open", out, kernel.opening_lines, sigma, second, precomputation.beta, batch.valid_dev, B)
    if device_output:
        return out
    return [bytes(out[GTB * i : GTB * (i + 1)]) if batch.valid[i] else None for i in range(B)]


def decrypt(decryption_key: PublicDecryptionKey, ciphertexts: Sequence[Ciphertext],
            server_keys: Sequence[ServerSecretKey], kernel: Optional[MiddleProductKernel] = None):
    """The reference's timed pipeline in one call: validate, precompute,
    partial decryption by the given servers, combine, open."""
    batch = validate_batch(ciphertexts)
    kernel = kernel or MiddleProductKernel(decryption_key, batch.batch_size())
    pre = precompute_batch(kernel, batch)
    shares = [partial_decrypt(k, batch) for k in server_keys]
    sigma = combine_shares(decryption_key, batch, shares)
    return open_batch(kernel, batch, ciphertexts, pre, sigma)
