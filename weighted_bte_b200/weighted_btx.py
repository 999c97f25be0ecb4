"""Weighted BTX batched threshold encryption (Construction 1) on B200.

Mirrors the public API of the reference crate `weighted_btx`
(weighted_btx/src/lib.rs:21-31): `keygen[_with_rng]`, `encrypt[_with_rng]`,
`validate_batch`, `partial_decrypt`, `verify_decryption_share`,
`accept_decryption_shares`, `prepare_decryption`, `precompute_batch`,
`open_batch`, `decrypt`, with the same argument meaning, the same checks and
the same error variants (weighted_bte_b200.errors).

Every group operation runs in libwbte (sm_100a kernels behind include/wbte.h);
this module holds the protocol logic: argument checks, SHA-256 transcripts
(host hashlib, as the reference uses sha2) and the data layout.  The public
decryption key is resident in HBM.  Group elements are `bytes` in blst's
memory layout (G1 96 B, G2 192 B, GT 576 B); scalars are Python ints.
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib, ops
from . import errors as E
from .rng import OsRng, random_scalar, sample_nonzero

R = ops.R
G1B, G2B, GTB = _lib.G1_BYTES, _lib.G2_BYTES, _lib.GT_BYTES
SETUP_ID_DOMAIN = b"WEIGHTED-BTX-SETUP-ID-v1"
TRANSCRIPT_DOMAIN = b"WEIGHTED-BTX-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"WEIGHTED-BTX-ORDERED-BATCH-v1"
DECRYPTION_CONTEXT_DOMAIN = b"WEIGHTED-BTX-DECRYPTION-CONTEXT-v1"
WIRE_MAGIC = b"WBTE-WBTX-PUBLIC-DECRYPTION-KEY-v1"
G1_IDENTITY = bytes(G1B)
ROOT_OF_UNITY = pow(7, (R - 1) >> 32, R)
TWO_ADICITY = 32

# ------------------------------------------------------------ device memory
_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch

        _torch = torch
    return _torch


def _device(device: Optional[int] = None):
    """The CUDA device `device`, by default the calling thread's current one
    (each rank of a multi-GPU run works on its own)."""
    torch = _t()
    return torch.device("cuda", torch.cuda.current_device() if device is None else device)


def to_device(data: bytes, device: Optional[int] = None):
    torch = _t()
    if len(data) == 0:
        return torch.empty(16, dtype=torch.uint8, device=_device(device))
    return torch.frombuffer(bytearray(data), dtype=torch.uint8).to(_device(device))


def empty_device(nbytes: int, device: Optional[int] = None):
    return _t().empty(max(16, nbytes), dtype=torch_uint8(), device=_device(device))


def torch_uint8():
    return _t().uint8


def to_host(tensor, nbytes: Optional[int] = None) -> bytes:
    data = tensor.detach().cpu().numpy().tobytes()
    return data if nbytes is None else data[:nbytes]


def _ctx():
    ctx = ops.ctx()
    torch = _t()
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    return ctx


# ----------------------------------------------------------- field helpers
def fr_bytes(s: int) -> bytes:
    return (s % R).to_bytes(32, "little")


def radix2_generator(size: int) -> int:
    """Generator of the size-`size` subgroup (btx/src/fft.rs:165-178)."""
    if size <= 0 or size & (size - 1):
        raise E.InvalidBatchSize(size)
    lg = size.bit_length() - 1
    if lg > TWO_ADICITY:
        raise E.InvalidBatchSize(size)
    g = ROOT_OF_UNITY
    for _ in range(lg, TWO_ADICITY):
        g = g * g % R
    return g


def scalar_fft(values: List[int], size: int) -> List[int]:
    """Radix-2 Fr transform (host; used for the Shamir evaluations of keygen)."""
    g = radix2_generator(size)
    a = list(values) + [0] * (size - len(values))
    bits = size.bit_length() - 1
    for i in range(size):
        j = int(format(i, f"0{bits}b")[::-1], 2) if bits else 0
        if i < j:
            a[i], a[j] = a[j], a[i]
    m = 2
    while m <= size:
        w_m = pow(g, size // m, R)
        for k in range(0, size, m):
            w = 1
            for j in range(m // 2):
                t = w * a[k + j + m // 2] % R
                u = a[k + j]
                a[k + j] = (u + t) % R
                a[k + j + m // 2] = (u - t) % R
                w = w * w_m % R
        m *= 2
    return a


_GT_GEN = None
_G1_GEN = None


def g1_generator() -> bytes:
    global _G1_GEN
    if _G1_GEN is None:
        _G1_GEN = ops.g1_mul_generator([1])
    return _G1_GEN


def gt_generator() -> bytes:
    """e(G1, G2) -- blstrs `Gt::generator()`."""
    global _GT_GEN
    if _GT_GEN is None:
        g2 = ops.g2_mul_generator([1])
        _GT_GEN = ops.pairing(g1_generator(), g2)
    return _GT_GEN


GT_IDENTITY = None


def gt_identity() -> bytes:
    one = bytearray(GTB)
    # Montgomery one = R mod p in the first coefficient
    p = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
    one[:48] = ((1 << 384) % p).to_bytes(48, "little")
    return bytes(one)


def message_from_bytes(data: bytes) -> bytes:
    """Map a byte string to GT: Gt::generator()^(LE(data) mod r)."""
    return ops.gt_pow(gt_generator(), [int.from_bytes(data, "little") % R], fixed_base=True)


def messages_from_bytes(datas: Sequence[bytes]) -> List[bytes]:
    if not datas:
        return []
    sc = [int.from_bytes(d, "little") % R for d in datas]
    return ops.split(ops.gt_pow(gt_generator(), sc, fixed_base=True), GTB)


def append_gt_many(values: bytes, n: int) -> List[bytes]:
    enc = ops.gt_compress(values, n)
    out = []
    for i in range(n):
        rec = enc[289 * i : 289 * (i + 1)]
        out.append(rec[:1] if rec[0] == 0 else rec)
    return out


# ------------------------------------------------------------------- keys
@dataclass
class KeygenConfig:
    max_batch_size: int
    party_weights: List[int]
    threshold_weight: int


@dataclass
class EncryptionKey:
    _max_batch_size: int
    _element: bytes
    _setup_id: bytes

    def max_batch_size(self) -> int:
        return self._max_batch_size

    def element(self) -> bytes:
        return self._element

    def setup_id(self) -> bytes:
        return self._setup_id


class PublicDecryptionKey:
    """Public weighted-BTX decryption material, resident in HBM.

    Layout as in weighted_btx/src/setup.rs:28-51: exponent-major blocks of
    verification keys [q_j^i]_2 (index (i-1) N + j), negative material
    [Z(w) q_owner(w)^-i]_2 and positive material [Z(w) q_owner(w)^i]_2
    (index (i-1) W + w).
    """

    def __init__(self, setup_id, max_batch_size, threshold_weight, total_weight, domain_size, party_weights,
                 party_offsets, evaluation_domain, verification_keys, negative_material, positive_material):
        self._setup_id = setup_id
        self._max_batch_size = max_batch_size
        self._threshold_weight = threshold_weight
        self._total_weight = total_weight
        self._domain_size = domain_size
        self._party_weights = list(party_weights)
        self.party_offsets = np.asarray(party_offsets, dtype=np.int64)
        self._evaluation_domain = list(evaluation_domain)
        self.domain_dev = to_device(b"".join(fr_bytes(x) for x in evaluation_domain))
        self.verification_keys = verification_keys
        self.negative_material = negative_material
        self.positive_material = positive_material

    def setup_id(self) -> bytes:
        return self._setup_id

    def max_batch_size(self) -> int:
        return self._max_batch_size

    def party_count(self) -> int:
        return len(self._party_weights)

    def total_weight(self) -> int:
        return self._total_weight

    def threshold_weight(self) -> int:
        return self._threshold_weight

    def required_weight(self) -> int:
        return self._threshold_weight + 1

    def party_weights(self) -> List[int]:
        return list(self._party_weights)

    def party_weight(self, party_index: int) -> int:
        if not 0 <= party_index < self.party_count():
            raise E.InvalidPartyIndex(party_index)
        return self._party_weights[party_index]

    def domain_points(self) -> List[int]:
        return list(self._evaluation_domain)

    def domain_size(self) -> int:
        return self._domain_size

    def party_range(self, party_index: int) -> range:
        if not 0 <= party_index < self.party_count():
            raise E.InvalidPartyIndex(party_index)
        return range(int(self.party_offsets[party_index]), int(self.party_offsets[party_index + 1]))

    def _validate_power(self, power: int, max_power: int):
        if power == 0 or power > max_power:
            raise E.InvalidPower(power, max_power)

    def verification_key(self, party_index: int, power: int) -> bytes:
        if not 0 <= party_index < self.party_count():
            raise E.InvalidPartyIndex(party_index)
        self._validate_power(power, self._max_batch_size)
        i = (power - 1) * self.party_count() + party_index
        return to_host(self.verification_keys[G2B * i : G2B * (i + 1)])

    def verification_power(self, power: int) -> List[bytes]:
        self._validate_power(power, self._max_batch_size)
        n = self.party_count()
        return ops.split(to_host(self.verification_keys[G2B * (power - 1) * n : G2B * power * n]), G2B)

    def negative_power(self, power: int) -> List[bytes]:
        self._validate_power(power, self._max_batch_size)
        W = self._total_weight
        return ops.split(to_host(self.negative_material[G2B * (power - 1) * W : G2B * power * W]), G2B)

    def positive_power(self, power: int) -> List[bytes]:
        self._validate_power(power, max(0, self._max_batch_size - 1))
        W = self._total_weight
        return ops.split(to_host(self.positive_material[G2B * (power - 1) * W : G2B * power * W]), G2B)

    # ------------------------------------------------------- wire format
    def to_wire(self) -> bytes:
        """The key as bytes: a header (WIRE_MAGIC, batch size, threshold, total
        weight, domain size, party count, setup id, party weights), the
        evaluation domain as 32-byte scalars, then the verification keys and
        the negative and positive material as compressed G2 points (96 bytes
        each, the crates' serialized size, weighted_pfe/README.md:159-214),
        compressed on the device."""
        B, N, W = self._max_batch_size, self.party_count(), self._total_weight
        head = WIRE_MAGIC + struct.pack("<5Q", B, self._threshold_weight, W, self._domain_size, N)
        head += self._setup_id + struct.pack(f"<{N}Q", *self._party_weights)
        domain = b"".join(fr_bytes(x) for x in self._evaluation_domain)
        streams = [ops.g2_compress(t, n) if n else b"" for t, n in
                   ((self.verification_keys, B * N), (self.negative_material, B * W),
                    (self.positive_material, (B - 1) * W))]
        return head + domain + b"".join(streams)

    @classmethod
    def from_wire(cls, blob: bytes, check_group: bool = True, device: Optional[int] = None) -> "PublicDecryptionKey":
        """Load a key written by to_wire: the compressed G2 streams are decoded
        on the device straight into the resident arrays, each point checked
        (canonical encoding, on the curve, and with check_group in the
        prime-order subgroup), as blstrs' checked deserialization does."""
        if not blob.startswith(WIRE_MAGIC):
            raise ValueError("not a weighted_btx public decryption key")
        o = len(WIRE_MAGIC)
        B, t, W, domain_size, N = struct.unpack_from("<5Q", blob, o)
        o += 40
        setup_id = blob[o : o + 32]
        o += 32
        weights = list(struct.unpack_from(f"<{N}Q", blob, o))
        o += 8 * N
        if sum(weights) != W or B == 0:
            raise ValueError("inconsistent key header")
        domain = [int.from_bytes(blob[o + 32 * i : o + 32 * (i + 1)], "little") for i in range(W)]
        o += 32 * W
        counts = (B * N, B * W, (B - 1) * W)
        if len(blob) != o + 96 * sum(counts):
            raise ValueError("key material has the wrong length")
        arrays = []
        for n in counts:
            out = empty_device(G2B * max(1, n), device)
            if n:
                try:
                    _ctx().call("wbte_g2_decompress", out, None, blob[o : o + 96 * n], n, int(check_group))
                except _lib.WbteError as err:
                    raise ValueError(f"invalid key material: {err}") from None
            arrays.append(out)
            o += 96 * n
        offsets = np.concatenate([[0], np.cumsum(weights)]).astype(np.int64)
        return cls(setup_id, B, t, W, domain_size, weights, offsets, domain, *arrays)

    def abi_key(self) -> _lib.WbtxKey:
        k = _lib.WbtxKey()
        k.domain_points = self.domain_dev.data_ptr()
        k.verification_keys = self.verification_keys.data_ptr()
        k.negative_material = self.negative_material.data_ptr()
        k.positive_material = self.positive_material.data_ptr()
        self._offsets_keep = np.ascontiguousarray(self.party_offsets, dtype=np.int64)
        k.party_offsets = self._offsets_keep.ctypes.data
        k.party_count = self.party_count()
        k.total_weight = self._total_weight
        k.max_batch_size = self._max_batch_size
        return k


@dataclass
class PartySecretKey:
    party_index: int
    _setup_id: bytes
    _max_batch_size: int
    _q: int

    def setup_id(self) -> bytes:
        return self._setup_id

    def max_batch_size(self) -> int:
        return self._max_batch_size

    def secret_scalar(self) -> int:
        return self._q


@dataclass
class KeyMaterial:
    encryption_key: EncryptionKey
    decryption_key: PublicDecryptionKey
    party_keys: List[PartySecretKey]


def _validate_config(config: KeygenConfig):
    if config.max_batch_size == 0:
        raise E.BatchIsEmpty()
    if not config.party_weights:
        raise E.EmptyCommittee()
    for j, w in enumerate(config.party_weights):
        if w == 0:
            raise E.InvalidPartyWeight(j, w)
    total = sum(config.party_weights)
    if total >= 1 << 64:
        raise E.TotalWeightOverflow()
    if config.threshold_weight >= total:
        raise E.InvalidCommittee(len(config.party_weights), total, config.threshold_weight)
    domain = 1 << (total - 1).bit_length() if total > 1 else 1
    if domain.bit_length() - 1 > TWO_ADICITY:
        raise E.InvalidEvaluationDomain(total)
    if config.max_batch_size * total * G2B >= 1 << 63:
        raise E.ParameterSizeOverflow()
    return total, domain


def setup_identifier(ek_element: bytes, max_batch_size: int, threshold: int, weights: Sequence[int],
                     first_vk_compressed: bytes, first_neg_compressed: bytes) -> bytes:
    """weighted_btx/src/setup.rs:486-513."""
    h = hashlib.sha256()
    h.update(SETUP_ID_DOMAIN)
    h.update(struct.pack("<Q", max_batch_size))
    h.update(struct.pack("<Q", threshold))
    h.update(struct.pack("<Q", len(weights)))
    for w in weights:
        h.update(struct.pack("<Q", w))
    h.update(append_gt_many(ek_element, 1)[0])
    h.update(first_vk_compressed)
    h.update(first_neg_compressed)
    return h.digest()


def keygen_with_rng(config: KeygenConfig, rng) -> KeyMaterial:
    """Trusted-dealer setup (weighted_btx/src/setup.rs:98-233).

    Scalar draws follow the reference: t+1 polynomial coefficients, then one
    nonzero secret per party.  The (2L - 1) W + N L fixed-base G2
    multiplications run on the GPU.
    """
    total, domain = _validate_config(config)
    N, L, W = len(config.party_weights), config.max_batch_size, total
    coeffs = [random_scalar(rng) for _ in range(config.threshold_weight + 1)]
    z = coeffs[0]
    z_evals = scalar_fft(coeffs, domain)[:W]
    g = radix2_generator(domain)
    evaluation_domain = [pow(g, i, R) for i in range(W)] if domain > 1 else [1]
    offsets = np.zeros(N + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(config.party_weights)
    owner = np.repeat(np.arange(N, dtype=np.int32), config.party_weights)
    qs = [sample_nonzero(rng) for _ in range(N)]
    qpos = bytearray(32 * L * N)
    qneg = bytearray(32 * L * N)
    for j, q in enumerate(qs):
        qi = pow(q, R - 2, R)
        p, n = q, qi
        for i in range(L):
            idx = 32 * (i * N + j)
            qpos[idx : idx + 32] = fr_bytes(p)
            qneg[idx : idx + 32] = fr_bytes(n)
            p = p * q % R
            n = n * qi % R
    vk = empty_device(G2B * L * N)
    neg = empty_device(G2B * L * W)
    pos = empty_device(G2B * max(1, (L - 1) * W))
    ctx = _ctx()
    ctx.call("wbte_wbtx_keygen_material", b"".join(fr_bytes(x) for x in z_evals), _lib.i32_array(owner),
             bytes(qpos), bytes(qneg), W, N, L, vk, neg, pos)
    element = ops.gt_pow(gt_generator(), [z], fixed_base=True)
    vk_c = ops.g2_compress(vk[: G2B * N], N)
    neg_c = ops.g2_compress(neg[: G2B * W], W)
    setup_id = setup_identifier(element, L, config.threshold_weight, config.party_weights, vk_c, neg_c)
    dk = PublicDecryptionKey(setup_id, L, config.threshold_weight, W, domain, config.party_weights, offsets,
                             evaluation_domain, vk, neg, pos)
    ek = EncryptionKey(L, element, setup_id)
    parties = [PartySecretKey(j, setup_id, L, q) for j, q in enumerate(qs)]
    return KeyMaterial(ek, dk, parties)


def keygen(max_batch_size: int, party_weights: Sequence[int], threshold_weight: int) -> KeyMaterial:
    return keygen_with_rng(KeygenConfig(max_batch_size, list(party_weights), threshold_weight), OsRng())


# ------------------------------------------------------------- encryption
@dataclass
class SchnorrProof:
    commitment: bytes  # G1 affine
    response: int


@dataclass
class Ciphertext:
    first: bytes  # G1 affine
    second: bytes  # GT
    proof: SchnorrProof

    def verify(self, encryption_key: EncryptionKey) -> bool:
        return bool(verify_ciphertexts([self], encryption_key.setup_id())[0])


def _transcript_prefix(setup_id: bytes) -> bytes:
    return TRANSCRIPT_DOMAIN + setup_id + ops.g1_compress(g1_generator(), 1)


def _challenge_fields(setup_id: bytes, first_c, second_enc, comm_c):
    """Transcript fields of challenge_scalar (weighted_btx/src/proof.rs:72-100):
    domain, setup id, compressed generator, then per ciphertext its compressed
    first component, GT encoding and compressed commitment."""
    prefix = _transcript_prefix(setup_id)
    return [(prefix, 0, len(prefix), _lib.TRANSCRIPT_BYTES), (first_c, 48, 48, _lib.TRANSCRIPT_BYTES),
            (second_enc, 289, 289, _lib.TRANSCRIPT_GT_VARIABLE), (comm_c, 48, 48, _lib.TRANSCRIPT_BYTES)]


def _challenges(setup_id: bytes, first_c: List[bytes], second_enc: List[bytes], comm_c: List[bytes]) -> List[int]:
    """Fiat-Shamir challenges with rejection sampling (weighted_btx/src/proof.rs:72-100),
    hashed on the device; identity GT encodings (one byte) travel as 289-byte records."""
    n = len(first_c)
    if n == 0:
        return []
    te = b"".join(b if len(b) == 289 else b + bytes(289 - len(b)) for b in second_enc)
    return ops.transcript_challenges(_challenge_fields(setup_id, b"".join(first_c), te, b"".join(comm_c)), n)


def encrypt_many(encryption_key: EncryptionKey, messages: Sequence[bytes], rng) -> List[Ciphertext]:
    """Batched `encrypt_with_rng` (weighted_btx/src/encryption.rs:28-49);
    draws (randomness, nonce) per message in order, as sequential calls would."""
    n = len(messages)
    if n == 0:
        return []
    rs, ks = [], []
    for _ in range(n):
        rs.append(random_scalar(rng))
        ks.append(random_scalar(rng))
    first = ops.g1_mul_generator(rs)
    comm = ops.g1_mul_generator(ks)
    mask = ops.gt_pow(encryption_key.element(), rs, fixed_base=True)
    second = ops.fp12_mul(b"".join(messages), mask)
    first_c = ops.split(ops.g1_compress(first, n), 48)
    comm_c = ops.split(ops.g1_compress(comm, n), 48)
    second_enc = append_gt_many(second, n)
    cs = _challenges(encryption_key.setup_id(), first_c, second_enc, comm_c)
    out = []
    for i in range(n):
        resp = (ks[i] + cs[i] * rs[i]) % R
        out.append(Ciphertext(first[G1B * i : G1B * (i + 1)], second[GTB * i : GTB * (i + 1)],
                              SchnorrProof(comm[G1B * i : G1B * (i + 1)], resp)))
    return out


def encrypt_with_rng(encryption_key: EncryptionKey, message: bytes, rng) -> Ciphertext:
    return encrypt_many(encryption_key, [message], rng)[0]


def encrypt(encryption_key: EncryptionKey, message: bytes) -> Ciphertext:
    return encrypt_with_rng(encryption_key, message, OsRng())


class CiphertextBatch:
    """An ordered ciphertext batch resident in HBM.

    The group elements live in device arrays (G1 first components, GT second
    components, G1 proof commitments); the proof responses stay on the host.
    The batch is immutable, so its canonical encodings and digest are
    computed once and cached.
    """

    def __init__(self, first, second, commitment, responses: Sequence[int]):
        self.first, self.second, self.commitment = first, second, commitment
        self.responses = [int(r) for r in responses]
        self._enc = None
        self._digest = None
        self._records = None
        self._resp_bytes = None

    @classmethod
    def upload(cls, cts: Sequence[Ciphertext]) -> "CiphertextBatch":
        return cls(to_device(b"".join(c.first for c in cts)), to_device(b"".join(c.second for c in cts)),
                   to_device(b"".join(c.proof.commitment for c in cts)), [c.proof.response for c in cts])

    def __len__(self) -> int:
        return len(self.responses)

    def to_ciphertexts(self) -> List[Ciphertext]:
        n = len(self)
        f, s, c = to_host(self.first, G1B * n), to_host(self.second, GTB * n), to_host(self.commitment, G1B * n)
        return [Ciphertext(f[G1B * i : G1B * (i + 1)], s[GTB * i : GTB * (i + 1)],
                           SchnorrProof(c[G1B * i : G1B * (i + 1)], self.responses[i])) for i in range(n)]

    def responses_bytes(self) -> bytes:
        if self._resp_bytes is None:
            self._resp_bytes = ops.scalars_bytes(self.responses)
        return self._resp_bytes

    def records(self) -> np.ndarray:
        """Canonical per-ciphertext records (n x 417 bytes: compressed first,
        GT encoding as a 289-byte record, compressed commitment, response),
        encoded on the device."""
        if self._records is None:
            n = len(self)
            fc, te, cc = _encode_on_device(self.first, self.commitment, self.second, n)
            self._records = _records_host(fc, te, cc, to_device(self.responses_bytes()), n)
        return self._records

    def encodings(self):
        if self._enc is None:
            self._enc = (self.first, self.commitment) + _encodings_of_records(self.records())
        return self._enc

    def digest(self) -> bytes:
        if self._digest is None:
            self._digest = _digest_of_records(self.records())
        return self._digest


# one ciphertext's canonical record: compressed first component, GT record,
# compressed commitment, response (weighted_btx/src/decryption.rs:740-748)
RECORD_BYTES = 48 + 289 + 48 + 32
_GT_AT, _COMM_AT, _RESP_AT = 48, 48 + 289, 48 + 289 + 48


def _encode_on_device(first_dev, comm_dev, second_dev, n: int):
    """Compressed first components, GT records and compressed commitments of
    n ciphertexts, as device buffers."""
    fc, cc, te = empty_device(48 * n), empty_device(48 * n), empty_device(289 * n)
    ctx = _ctx()
    ctx.call("wbte_g1_compress", fc, first_dev, n)
    ctx.call("wbte_g1_compress", cc, comm_dev, n)
    ctx.call("wbte_gt_compress", te, second_dev, n)
    return fc, te, cc


def _records_host(fc, te, cc, resp_dev, n: int) -> np.ndarray:
    torch = _t()
    rec = torch.cat([fc[: 48 * n].view(n, 48), te[: 289 * n].view(n, 289), cc[: 48 * n].view(n, 48),
                     resp_dev[: 32 * n].view(n, 32)], 1)
    return rec.cpu().numpy()


def _encodings_of_records(rec: np.ndarray):
    first_c = [bytes(r[:_GT_AT]) for r in rec]
    comm_c = [bytes(r[_COMM_AT:_RESP_AT]) for r in rec]
    second_enc = [bytes(r[_GT_AT:_COMM_AT]) if r[_GT_AT] else b"\x00" for r in rec]
    return first_c, comm_c, second_enc


def _digest_of_records(rec: np.ndarray) -> bytes:
    """batch_digest over canonical records (weighted_btx/src/decryption.rs:740-748):
    an identity GT contributes its tag byte only."""
    h = hashlib.sha256()
    h.update(BATCH_DIGEST_DOMAIN)
    h.update(struct.pack("<Q", len(rec)))
    ident = rec[:, _GT_AT] == 0
    if ident.any():
        keep = np.ones(rec.shape, dtype=bool)
        keep[ident, _GT_AT + 1 : _COMM_AT] = False
        h.update(rec[keep].tobytes())
    else:
        h.update(np.ascontiguousarray(rec).data)
    return h.digest()


def _encodings(cts):
    if isinstance(cts, CiphertextBatch):
        return cts.encodings()
    n = len(cts)
    first = b"".join(c.first for c in cts)
    comm = b"".join(c.proof.commitment for c in cts)
    second = b"".join(c.second for c in cts)
    first_c = ops.split(ops.g1_compress(first, n), 48)
    comm_c = ops.split(ops.g1_compress(comm, n), 48)
    second_enc = append_gt_many(second, n)
    return first, comm, first_c, comm_c, second_enc


def _responses(cts) -> List[int]:
    if isinstance(cts, CiphertextBatch):
        return cts.responses
    return [c.proof.response for c in cts]


def verify_ciphertexts(cts: Sequence[Ciphertext], setup_id: bytes, encodings=None) -> np.ndarray:
    """Batched `Ciphertext::verify_for_setup` (weighted_btx/src/encryption.rs:57-59)."""
    if len(cts) == 0:
        return np.zeros(0, dtype=bool)
    first, comm, first_c, comm_c, second_enc = encodings or _encodings(cts)
    cs = _challenges(setup_id, first_c, second_enc, comm_c)
    out = np.zeros(len(cts), dtype=np.uint8)
    ops.ctx().call("wbte_schnorr_verify", out, first, comm, ops.scalars_bytes(_responses(cts)),
                   ops.scalars_bytes(cs), len(cts))
    return out.astype(bool)


def _canonical(first_c: bytes, second_enc: bytes, comm_c: bytes, response: int) -> bytes:
    return first_c + second_enc + comm_c + fr_bytes(response)


def batch_digest(cts, encodings=None) -> bytes:
    """weighted_btx/src/decryption.rs:740-748."""
    if isinstance(cts, CiphertextBatch):
        return cts.digest()
    _, _, first_c, comm_c, second_enc = encodings or _encodings(cts)
    h = hashlib.sha256()
    h.update(BATCH_DIGEST_DOMAIN)
    h.update(struct.pack("<Q", len(cts)))
    for i, ct in enumerate(cts):
        h.update(_canonical(first_c[i], second_enc[i], comm_c[i], ct.proof.response))
    return h.digest()


def decryption_context_id(setup_id: bytes, batch_size: int, party_indices: Sequence[int]) -> bytes:
    """weighted_btx/src/decryption.rs:750-764."""
    h = hashlib.sha256()
    h.update(DECRYPTION_CONTEXT_DOMAIN)
    h.update(setup_id)
    h.update(struct.pack("<Q", batch_size))
    h.update(struct.pack("<Q", len(party_indices)))
    for j in party_indices:
        h.update(struct.pack("<Q", j))
    return h.digest()


# -------------------------------------------------------------- decryption
@dataclass
class ValidatedBatch:
    _setup_id: bytes
    _batch_size: int
    _digest: bytes
    valid: np.ndarray
    first_affine: bytes
    first_dev: object = None
    valid_dev: object = None

    def batch_size(self) -> int:
        return self._batch_size

    def setup_id(self) -> bytes:
        return self._setup_id

    def digest(self) -> bytes:
        return self._digest

    def valid_mask(self) -> List[bool]:
        return [bool(v) for v in self.valid]

    def valid_count(self) -> int:
        return int(self.valid.sum())


@dataclass
class DecryptionShare:
    party_index: int
    sigma: bytes  # G1 affine
    batch_digest: bytes
    setup_id: bytes


@dataclass
class AcceptedDecryptionShares:
    setup_id: bytes
    batch_size: int
    digest: bytes
    _accepted_weight: int
    _shares: List[DecryptionShare]
    _rejected_parties: List[int]

    def accepted_weight(self) -> int:
        return self._accepted_weight

    def party_count(self) -> int:
        return len(self._shares)

    def party_indices(self) -> List[int]:
        return [s.party_index for s in self._shares]

    def rejected_parties(self) -> List[int]:
        return list(self._rejected_parties)

    def shares(self) -> List[DecryptionShare]:
        return list(self._shares)


@dataclass
class DecryptionPrecomputation:
    setup_id: bytes
    context_id: bytes
    _batch_size: int
    _accepted_weight: int
    party_indices: List[int]
    _transform_size: int
    kernel_lines: object  # device, m * 68 * 288 bytes
    opening_keys: object  # device, B * T G2
    transformed_kernel: object  # device, m G2
    opening_lines: object = None  # device, line tables of the B * T opening keys

    def batch_size(self) -> int:
        return self._batch_size

    def accepted_weight(self) -> int:
        return self._accepted_weight

    def party_count(self) -> int:
        return len(self.party_indices)

    def transform_size(self) -> int:
        return self._transform_size


@dataclass
class BatchPrecomputation:
    context_id: bytes
    batch_size: int
    digest: bytes
    beta: object  # device, B GT


def _validate_batch_size(dk: PublicDecryptionKey, batch_size: int):
    if batch_size == 0:
        raise E.BatchIsEmpty()
    if batch_size > dk.max_batch_size():
        raise E.BatchTooLarge(batch_size, dk.max_batch_size())


def validate_batch(decryption_key: PublicDecryptionKey, ciphertexts: Sequence[Ciphertext]) -> ValidatedBatch:
    """weighted_btx/src/decryption.rs:85-140: verify every proof, keep slot positions."""
    return validate_batches(decryption_key, [ciphertexts])[0]


def validate_batches(decryption_key: PublicDecryptionKey, batches: Sequence) -> List[ValidatedBatch]:
    """`validate_batch` for several batches in one pass on the device: the
    ciphertexts are encoded (compressed G1, GT records), hashed into their
    Fiat-Shamir challenges and proof-checked with one launch each; each result
    equals `validate_batch` of that batch alone.  The host only hashes the
    canonical records into each batch digest."""
    if not batches:
        return []
    for cts in batches:
        _validate_batch_size(decryption_key, len(cts))
    sizes = [len(cts) for cts in batches]
    total = sum(sizes)
    torch = _t()

    def dev(cts, attr, rec):
        if isinstance(cts, CiphertextBatch):
            return getattr(cts, attr)[: rec * len(cts)]
        if attr == "first":
            return to_device(b"".join(c.first for c in cts))
        if attr == "commitment":
            return to_device(b"".join(c.proof.commitment for c in cts))
        return to_device(b"".join(c.second for c in cts))

    def resp(cts):
        return cts.responses_bytes() if isinstance(cts, CiphertextBatch) else ops.scalars_bytes(_responses(cts))

    first_all = torch.cat([dev(cts, "first", G1B) for cts in batches])
    comm_all = torch.cat([dev(cts, "commitment", G1B) for cts in batches])
    second_all = torch.cat([dev(cts, "second", GTB) for cts in batches])
    resp_all = to_device(b"".join(resp(cts) for cts in batches))
    fc, te, cc = _encode_on_device(first_all, comm_all, second_all, total)
    ch = empty_device(32 * total)
    ops.transcript_challenges(_challenge_fields(decryption_key.setup_id(), fc, te, cc), total, out=ch)
    ok = np.zeros(total, dtype=np.uint8)
    _ctx().call("wbte_schnorr_verify", ok, first_all, comm_all, resp_all, ch, total)
    records = _records_host(fc, te, cc, resp_all, total)
    valid_all = ok.astype(bool)
    valid_dev_all = to_device(ok.tobytes())
    first_masked = (first_all.view(total, G1B) * valid_dev_all[:total].view(total, 1)).reshape(-1)
    out, o = [], 0
    for cts, n in zip(batches, sizes):
        rec = records[o : o + n]
        if isinstance(cts, CiphertextBatch):
            if cts._records is None:
                cts._records = rec
            digest = cts.digest()
        else:
            digest = _digest_of_records(rec)
        out.append(ValidatedBatch(decryption_key.setup_id(), n, digest, valid_all[o : o + n], None,
                                  first_masked[G1B * o : G1B * (o + n)], valid_dev_all[o : o + n]))
        o += n
    return out


def partial_decrypt_many(party_keys: Sequence[PartySecretKey], batch: ValidatedBatch) -> List[DecryptionShare]:
    """`partial_decrypt` for several parties in one launch sequence
    (weighted_btx/src/decryption.rs:205-233)."""
    for pk in party_keys:
        if batch.setup_id() != pk.setup_id():
            raise E.MismatchedSetup()
        if batch.batch_size() > pk.max_batch_size():
            raise E.BatchTooLarge(batch.batch_size(), pk.max_batch_size())
    T = len(party_keys)
    if T == 0:
        return []
    sig = bytearray(G1B * T)
    _ctx().call("wbte_wbtx_partial_decrypt", sig, batch.first_dev, batch.batch_size(),
                b"".join(fr_bytes(pk.secret_scalar()) for pk in party_keys), T)
    return [DecryptionShare(pk.party_index, bytes(sig[G1B * j : G1B * (j + 1)]), batch.digest(), pk.setup_id())
            for j, pk in enumerate(party_keys)]


def partial_decrypt(party_key: PartySecretKey, batch: ValidatedBatch) -> DecryptionShare:
    return partial_decrypt_many([party_key], batch)[0]


def _verify_shares(dk: PublicDecryptionKey, batch: ValidatedBatch, shares: Sequence[DecryptionShare],
                   challenges: Sequence[int]) -> bool:
    ok = np.zeros(1, dtype=np.int32)
    T = len(shares)
    _ctx().call("wbte_wbtx_verify_shares", ok, dk.abi_key(), batch.first_dev, batch.valid_dev, batch.batch_size(),
                b"".join(s.sigma for s in shares), _lib.i64_array([s.party_index for s in shares]),
                b"".join(fr_bytes(c) for c in challenges), T)
    return bool(ok[0])


def verify_decryption_share(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                            share: DecryptionShare) -> bool:
    """weighted_btx/src/decryption.rs:236-272."""
    _validate_batch_size(decryption_key, batch.batch_size())
    if batch.setup_id() != decryption_key.setup_id():
        raise E.MismatchedSetup()
    if share.batch_digest != batch.digest() or share.setup_id != decryption_key.setup_id():
        return False
    if share.party_index >= decryption_key.party_count():
        raise E.InvalidPartyIndex(share.party_index)
    return _verify_shares(decryption_key, batch, [share], [1])


def screen_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, shares: Sequence[DecryptionShare]):
    """The structural checks of accept_decryption_shares (weighted_btx/src/decryption.rs:282-305):
    returns (candidates bound to this batch and setup, rejected party indices)."""
    _validate_batch_size(decryption_key, batch.batch_size())
    if batch.setup_id() != decryption_key.setup_id():
        raise E.MismatchedSetup()
    if len(shares) > decryption_key.party_count():
        raise E.TooManyShares(len(shares), decryption_key.party_count())
    seen = [False] * decryption_key.party_count()
    candidates, rejected = [], []
    for s in shares:
        if s.party_index >= decryption_key.party_count():
            raise E.InvalidPartyIndex(s.party_index)
        if seen[s.party_index]:
            raise E.DuplicatePartyIndex(s.party_index)
        seen[s.party_index] = True
        if s.batch_digest == batch.digest() and s.setup_id == decryption_key.setup_id():
            candidates.append(s)
        else:
            rejected.append(s.party_index)
    return candidates, rejected


def finish_acceptance(decryption_key: PublicDecryptionKey, batch: ValidatedBatch, candidates, rejected,
                      aggregate_ok: bool) -> AcceptedDecryptionShares:
    """The rest of accept_decryption_shares (decryption.rs:306-353) once the
    batched aggregate check has run: per-share blame on failure, weight check."""
    rejected = list(rejected)
    if aggregate_ok:
        accepted = list(candidates)
    else:
        accepted = []
        for s in candidates:
            if verify_decryption_share(decryption_key, batch, s):
                accepted.append(s)
            else:
                rejected.append(s.party_index)
    accepted.sort(key=lambda s: s.party_index)
    rejected.sort()
    weight = sum(decryption_key.party_weight(s.party_index) for s in accepted)
    if weight <= decryption_key.threshold_weight():
        raise E.InsufficientWeight(weight, decryption_key.required_weight(), rejected)
    return AcceptedDecryptionShares(decryption_key.setup_id(), batch.batch_size(), batch.digest(), weight, accepted,
                                    rejected)


def accept_decryption_shares(decryption_key: PublicDecryptionKey, batch: ValidatedBatch,
                             shares: Sequence[DecryptionShare], rng=None) -> AcceptedDecryptionShares:
    """weighted_btx/src/decryption.rs:276-353 (batched check, per-share fallback, weight check)."""
    candidates, rejected = screen_shares(decryption_key, batch, shares)
    rng = rng or OsRng()
    if candidates:
        challenges = [sample_nonzero(rng) for _ in candidates]
        aggregate_ok = _verify_shares(decryption_key, batch, candidates, challenges)
    else:
        aggregate_ok = True
    return finish_acceptance(decryption_key, batch, candidates, rejected, aggregate_ok)


def transform_size_for(batch_size: int) -> int:
    return 1 << (2 * batch_size - 1).bit_length()


def prepare_decryption(decryption_key: PublicDecryptionKey,
                       accepted: AcceptedDecryptionShares) -> DecryptionPrecomputation:
    """weighted_btx/src/decryption.rs:427-551 (committee-dependent G2 work, cacheable)."""
    _validate_batch_size(decryption_key, accepted.batch_size)
    if accepted.setup_id != decryption_key.setup_id():
        raise E.MismatchedSetup()
    if accepted.accepted_weight() <= decryption_key.threshold_weight():
        raise E.InsufficientWeight(accepted.accepted_weight(), decryption_key.required_weight(), [])
    parties = accepted.party_indices()
    B = accepted.batch_size
    m = transform_size_for(B)
    lines = empty_device(_lib.LINE_BYTES * _lib.MILLER_LINES * m)
    opening = empty_device(G2B * B * len(parties))
    kernel = empty_device(G2B * m)
    try:
        _ctx().call("wbte_wbtx_prepare", decryption_key.abi_key(), _lib.i64_array(parties), len(parties), B, lines,
                    opening, kernel)
    except _lib.WbteError as exc:
        if exc.status == -7:
            raise E.InvalidInterpolationSet() from exc
        raise
    ctx_id = decryption_context_id(decryption_key.setup_id(), B, parties)
    # line tables of the opening keys, for the batched opening's multi-Miller loops
    opening_lines = empty_device(_lib.LINE_BYTES * _lib.MILLER_LINES * B * len(parties))
    _ctx().call("wbte_g2_prepare_lines", opening_lines, opening, B * len(parties))
    return DecryptionPrecomputation(decryption_key.setup_id(), ctx_id, B, accepted.accepted_weight(), parties, m,
                                    lines, opening, kernel, opening_lines)


def _ensure_precomputation_batch(pre: DecryptionPrecomputation, batch: ValidatedBatch):
    if pre.batch_size() != batch.batch_size():
        raise E.MismatchedBatchSize(pre.batch_size(), batch.batch_size())
    if pre.setup_id != batch.setup_id():
        raise E.MismatchedSetup()


def precompute_batch(precomputation: DecryptionPrecomputation, batch: ValidatedBatch) -> BatchPrecomputation:
    """weighted_btx/src/decryption.rs:555-603 (middle product via G1 NTT, prepared
    Miller loops, easy part, truncated cyclotomic inverse transform, hard part)."""
    _ensure_precomputation_batch(precomputation, batch)
    B = batch.batch_size()
    beta = empty_device(GTB * B)
    _ctx().call("wbte_wbtx_precompute", beta, precomputation.kernel_lines, batch.first_dev, batch.valid_dev, B)
    return BatchPrecomputation(precomputation.context_id, B, batch.digest(), beta)


def open_batch(precomputation: DecryptionPrecomputation, accepted: AcceptedDecryptionShares, batch: ValidatedBatch,
               ciphertexts, cross_terms: BatchPrecomputation, device_output: bool = False):
    """weighted_btx/src/decryption.rs:607-695.

    Returns one `Optional[bytes]` per slot (None for invalid slots), or with
    device_output=True a device array of B GT values (identity at invalid
    slots) that stays in HBM."""
    _ensure_precomputation_batch(precomputation, batch)
    if accepted.batch_size != batch.batch_size():
        raise E.MismatchedBatchSize(batch.batch_size(), accepted.batch_size)
    if accepted.digest != batch.digest():
        raise E.MismatchedBatchDigest()
    if len(ciphertexts) != batch.batch_size():
        raise E.MismatchedBatchSize(batch.batch_size(), len(ciphertexts))
    if batch_digest(ciphertexts) != batch.digest():
        raise E.MismatchedBatchDigest()
    if cross_terms.batch_size != batch.batch_size() or cross_terms.digest != batch.digest():
        raise E.MismatchedBatchDigest()
    if cross_terms.context_id != precomputation.context_id:
        raise E.MismatchedCommittee()
    if accepted.setup_id != precomputation.setup_id:
        raise E.MismatchedSetup()
    if accepted.party_indices() != precomputation.party_indices:
        raise E.MismatchedCommittee()
    if isinstance(ciphertexts, CiphertextBatch):
        second = ciphertexts.second
    else:
        second = b"".join(c.second for c in ciphertexts)
    if device_output:
        out = empty_device(GTB * batch.batch_size())
        _open_into(out, precomputation, accepted, batch, second, cross_terms)
        return out
    msgs = bytearray(GTB * batch.batch_size())
    _open_into(msgs, precomputation, accepted, batch, second, cross_terms)
    return [bytes(msgs[GTB * i : GTB * (i + 1)]) if batch.valid[i] else None for i in range(batch.batch_size())]


def _open_into(out, pre, accepted, batch, second, cross_terms) -> None:
    _ctx().call("wbte_wbtx_open", out, pre.opening_keys, b"".join(s.sigma for s in accepted.shares()),
                accepted.party_count(), second, cross_terms.beta, batch.valid_dev, batch.batch_size())


def decrypt(decryption_key: PublicDecryptionKey, ciphertexts: Sequence[Ciphertext],
            shares: Sequence[DecryptionShare], rng=None) -> List[Optional[bytes]]:
    """Convenience wrapper around all public phases (weighted_btx/src/decryption.rs:698-709)."""
    _validate_batch_size(decryption_key, len(ciphertexts))
    batch = validate_batch(decryption_key, ciphertexts)
    accepted = accept_decryption_shares(decryption_key, batch, shares, rng)
    fixed = prepare_decryption(decryption_key, accepted)
    cross = precompute_batch(fixed, batch)
    return open_batch(fixed, accepted, batch, ciphertexts, cross)
