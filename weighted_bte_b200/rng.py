"""Seeded randomness for key generation and encryption.

`ChaCha20Rng` produces the ChaCha20 keystream (RFC 8439 quarter-round and
block function, 20 rounds, 64-bit block counter, zero stream id) as little-
endian 32-bit words; `seed_from_u64` expands a 64-bit seed into the 32-byte
key with the PCG32 sequence that rand_core 0.6's `SeedableRng::seed_from_u64`
publishes.  `random_scalar` draws eight 64-bit words and reduces the 512-bit
little-endian integer modulo r (the wide reduction used by `Scalar::random`
in the ff/bls12_381 family).  `OsRng` mirrors `rand_core::OsRng`.

The reference's tests draw from OsRng only, so these seeded streams are a
convention of this project for reproducible inputs.
"""
from __future__ import annotations

import os
import struct

R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
_M32 = 0xFFFFFFFF
_M64 = 0xFFFFFFFFFFFFFFFF


def _rotl(x: int, n: int) -> int:
    return ((x << n) | (x >> (32 - n))) & _M32


def _quarter(s, a, b, c, d):
    s[a] = (s[a] + s[b]) & _M32
    s[d] = _rotl(s[d] ^ s[a], 16)
    s[c] = (s[c] + s[d]) & _M32
    s[b] = _rotl(s[b] ^ s[c], 12)
    s[a] = (s[a] + s[b]) & _M32
    s[d] = _rotl(s[d] ^ s[a], 8)
    s[c] = (s[c] + s[d]) & _M32
    s[b] = _rotl(s[b] ^ s[c], 7)


def chacha20_block(key_words, counter: int, stream: int = 0):
    state = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key_words) + [
        counter & _M32,
        (counter >> 32) & _M32,
        stream & _M32,
        (stream >> 32) & _M32,
    ]
    w = list(state)
    for _ in range(10):
        _quarter(w, 0, 4, 8, 12)
        _quarter(w, 1, 5, 9, 13)
        _quarter(w, 2, 6, 10, 14)
        _quarter(w, 3, 7, 11, 15)
        _quarter(w, 0, 5, 10, 15)
        _quarter(w, 1, 6, 11, 12)
        _quarter(w, 2, 7, 8, 13)
        _quarter(w, 3, 4, 9, 14)
    return [(w[i] + state[i]) & _M32 for i in range(16)]


def chacha20_blocks(key_words, counter: int, n: int):
    """n consecutive keystream blocks (counters counter .. counter + n - 1,
    stream 0) as one flat list of 16 n words, computed for all blocks at once
    with numpy uint32 vectors (the same function as chacha20_block)."""
    import numpy as np

    st = np.empty((16, n), dtype=np.uint32)
    st[0:4] = np.array([0x61707865, 0x3320646E, 0x79622D32, 0x6B206574], dtype=np.uint32)[:, None]
    st[4:12] = np.array(list(key_words), dtype=np.uint32)[:, None]
    ctr = np.arange(counter, counter + n, dtype=np.uint64)
    st[12] = (ctr & np.uint64(_M32)).astype(np.uint32)
    st[13] = (ctr >> np.uint64(32)).astype(np.uint32)
    st[14] = 0
    st[15] = 0
    w = [st[i].copy() for i in range(16)]

    def rotl(x, k):
        return (x << np.uint32(k)) | (x >> np.uint32(32 - k))

    def quarter(a, b, c, d):
        w[a] += w[b]
        w[d] = rotl(w[d] ^ w[a], 16)
        w[c] += w[d]
        w[b] = rotl(w[b] ^ w[c], 12)
        w[a] += w[b]
        w[d] = rotl(w[d] ^ w[a], 8)
        w[c] += w[d]
        w[b] = rotl(w[b] ^ w[c], 7)

    for _ in range(10):
        quarter(0, 4, 8, 12)
        quarter(1, 5, 9, 13)
        quarter(2, 6, 10, 14)
        quarter(3, 7, 11, 15)
        quarter(0, 5, 10, 15)
        quarter(1, 6, 11, 12)
        quarter(2, 7, 8, 13)
        quarter(3, 4, 9, 14)
    out = np.stack(w) + st
    return out.T.reshape(-1).tolist()


def _pcg32(state: int):
    state = (state * 6364136223846793005 + 11634580027462260723) & _M64
    xorshifted = (((state >> 18) ^ state) >> 27) & _M32
    rot = state >> 59
    x = ((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & _M32
    return state, x


class ChaCha20Rng:
    def __init__(self, seed: bytes):
        if len(seed) != 32:
            raise ValueError("ChaCha20Rng takes a 32-byte seed")
        self.key = list(struct.unpack("<8I", seed))
        self.counter = 0
        self.buf = []

    @classmethod
    def seed_from_u64(cls, state: int) -> "ChaCha20Rng":
        words = []
        s = state & _M64
        for _ in range(8):
            s, x = _pcg32(s)
            words.append(x)
        return cls(struct.pack("<8I", *words))

    # keystream blocks generated per refill: the words come out in the same
    # order whatever the refill size (blocks depend only on key and counter)
    REFILL_BLOCKS = 64

    def next_u32(self) -> int:
        if not self.buf:
            self.buf = chacha20_blocks(self.key, self.counter, self.REFILL_BLOCKS)
            self.counter += self.REFILL_BLOCKS
            self.buf.reverse()
        return self.buf.pop()

    def next_u64(self) -> int:
        lo = self.next_u32()
        hi = self.next_u32()
        return lo | (hi << 32)

    def fill_bytes(self, n: int) -> bytes:
        out = bytearray()
        while len(out) < n:
            out += struct.pack("<I", self.next_u32())
        return bytes(out[:n])


class OsRng:
    def next_u64(self) -> int:
        return int.from_bytes(os.urandom(8), "little")

    def fill_bytes(self, n: int) -> bytes:
        return os.urandom(n)


def random_scalar(rng) -> int:
    acc = 0
    for i in range(8):
        acc |= rng.next_u64() << (64 * i)
    return acc % R


def sample_nonzero(rng) -> int:
    while True:
        s = random_scalar(rng)
        if s:
            return s
