"""ctypes front end for the CPU oracle (test infrastructure only).

Only tests/, the smoke check and the CPU-baseline leg of bench.py import
this module, and only as the checker.  The product package never imports it.

Values cross this interface in blst's memory layout (Montgomery-form Fp
limbs; 96-byte affine G1, 192-byte affine G2, 576-byte Fp12, all-zero
bytes for the point at infinity).  Scalars are Python ints, converted to
canonical 32-byte little-endian strings.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
X_ABS = 0xD201000000010000
G1_BYTES, G2_BYTES, GT_BYTES, FR_BYTES = 96, 192, 576, 32

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_init()
    return _lib


def _buf(n: int):
    return ctypes.create_string_buffer(n)


def _i64arr(values):
    arr = (ctypes.c_int64 * max(1, len(values)))(*values)
    return arr


def s2b(s: int) -> bytes:
    return (s % R).to_bytes(32, "little")


def scalars_bytes(scalars) -> bytes:
    return b"".join(s2b(s) for s in scalars)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ----------------------------------------------------------------- groups
def g1_generator() -> bytes:
    b = _buf(96)
    lib().orc_g1_generator(b)
    return b.raw


def g2_generator() -> bytes:
    b = _buf(192)
    lib().orc_g2_generator(b)
    return b.raw


G1_IDENTITY = bytes(96)
G2_IDENTITY = bytes(192)


def fr_root_of_unity() -> int:
    b = _buf(32)
    lib().orc_fr_root_of_unity(b)
    return int.from_bytes(b.raw, "little")


def g1_add(a: bytes, b: bytes) -> bytes:
    o = _buf(96)
    lib().orc_g1_add(o, a, b)
    return o.raw


def g2_add(a: bytes, b: bytes) -> bytes:
    o = _buf(192)
    lib().orc_g2_add(o, a, b)
    return o.raw


def g1_neg(a: bytes) -> bytes:
    o = _buf(96)
    lib().orc_g1_neg(o, a)
    return o.raw


def g2_neg(a: bytes) -> bytes:
    o = _buf(192)
    lib().orc_g2_neg(o, a)
    return o.raw


def g1_mul_many(points, scalars) -> list:
    """points: list of 96-byte points (or a single bytes object used for all)."""
    n = len(scalars)
    if isinstance(points, (bytes, bytearray)):
        pts, stride = bytes(points), 0
    else:
        pts, stride = b"".join(points), 96
    o = _buf(96 * n)
    lib().orc_g1_mul_batch(o, pts, ctypes.c_int64(stride), scalars_bytes(scalars), ctypes.c_int64(n))
    return [o.raw[96 * i : 96 * (i + 1)] for i in range(n)]


def g2_mul_many(points, scalars) -> list:
    n = len(scalars)
    if isinstance(points, (bytes, bytearray)):
        pts, stride = bytes(points), 0
    else:
        pts, stride = b"".join(points), 192
    o = _buf(192 * n)
    lib().orc_g2_mul_batch(o, pts, ctypes.c_int64(stride), scalars_bytes(scalars), ctypes.c_int64(n))
    return [o.raw[192 * i : 192 * (i + 1)] for i in range(n)]


def g1_mul(p: bytes, s: int) -> bytes:
    return g1_mul_many([p], [s])[0]


def g2_mul(p: bytes, s: int) -> bytes:
    return g2_mul_many([p], [s])[0]


def g1_on_curve(p: bytes) -> bool:
    return bool(lib().orc_g1_on_curve(p))


def g2_on_curve(p: bytes) -> bool:
    return bool(lib().orc_g2_on_curve(p))


def g1_compress(p: bytes) -> bytes:
    o = _buf(48)
    lib().orc_g1_compress(o, p)
    return o.raw


def g2_compress(p: bytes) -> bytes:
    o = _buf(96)
    lib().orc_g2_compress(o, p)
    return o.raw


def fp12_to_bytes(f: bytes) -> bytes:
    o = _buf(576)
    lib().orc_fp12_to_bytes(o, f)
    return o.raw


# ------------------------------------------------------------------- MSM
def g1_msm(points, scalars) -> bytes:
    o = _buf(96)
    lib().orc_g1_msm(o, b"".join(points), scalars_bytes(scalars), ctypes.c_int64(len(scalars)))
    return o.raw


def g2_msm(points, scalars) -> bytes:
    o = _buf(192)
    lib().orc_g2_msm(o, b"".join(points), scalars_bytes(scalars), ctypes.c_int64(len(scalars)))
    return o.raw


def _msm_gather(fn, size, bases: bytes, groups, scalar_blob: bytes):
    """groups: list of (point_indices, scalar_indices)."""
    pidx, sidx, offs = [], [], [0]
    for pi, si in groups:
        pidx.extend(pi)
        sidx.extend(si)
        offs.append(len(pidx))
    k = len(groups)
    o = _buf(size * max(1, k))
    fn(o, bases, _i64arr(pidx), scalar_blob, _i64arr(sidx), _i64arr(offs), ctypes.c_int64(k))
    return [o.raw[size * j : size * (j + 1)] for j in range(k)]


def g1_msm_gather(bases: bytes, groups, scalar_blob: bytes):
    return _msm_gather(lib().orc_g1_msm_gather, 96, bases, groups, scalar_blob)


def g2_msm_gather(bases: bytes, groups, scalar_blob: bytes):
    return _msm_gather(lib().orc_g2_msm_gather, 192, bases, groups, scalar_blob)


# ------------------------------------------------------------ transforms
def g1_ntt(points, inverse=False) -> list:
    n = len(points)
    b = ctypes.create_string_buffer(b"".join(points), 96 * n)
    lib().orc_g1_ntt(b, ctypes.c_int64(n), int(inverse))
    return [b.raw[96 * i : 96 * (i + 1)] for i in range(n)]


def g2_ntt(points, inverse=False) -> list:
    n = len(points)
    b = ctypes.create_string_buffer(b"".join(points), 192 * n)
    lib().orc_g2_ntt(b, ctypes.c_int64(n), int(inverse))
    return [b.raw[192 * i : 192 * (i + 1)] for i in range(n)]


def gt_ntt(values, inverse=False) -> list:
    n = len(values)
    b = ctypes.create_string_buffer(b"".join(values), 576 * n)
    lib().orc_gt_ntt(b, ctypes.c_int64(n), int(inverse))
    return [b.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def fr_ntt(values, inverse=False) -> list:
    n = len(values)
    b = ctypes.create_string_buffer(scalars_bytes(values), 32 * n)
    lib().orc_fr_ntt(b, ctypes.c_int64(n), int(inverse))
    return [int.from_bytes(b.raw[32 * i : 32 * (i + 1)], "little") for i in range(n)]


def cyclotomic_prefix_ifft(values, out_count: int) -> list:
    n = len(values)
    b = ctypes.create_string_buffer(b"".join(values), 576 * n)
    lib().orc_cyclotomic_prefix_ifft(b, ctypes.c_int64(n), ctypes.c_int64(out_count))
    return [b.raw[576 * i : 576 * (i + 1)] for i in range(out_count)]


# --------------------------------------------------------------- pairing
def miller_loop(g1: bytes, g2: bytes) -> bytes:
    o = _buf(576)
    lib().orc_miller_loop(o, g1, g2)
    return o.raw


def miller_loop_many(g1s, g2s) -> list:
    n = len(g1s)
    o = _buf(576 * max(1, n))
    lib().orc_miller_loop_batch(o, b"".join(g1s), b"".join(g2s), ctypes.c_int64(n))
    return [o.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def multi_miller_many(groups) -> list:
    """groups: list of (list_of_g1, list_of_g2)."""
    g1s, g2s, offs = [], [], [0]
    for a, b in groups:
        g1s.extend(a)
        g2s.extend(b)
        offs.append(len(g1s))
    k = len(groups)
    o = _buf(576 * max(1, k))
    lib().orc_multi_miller_batch(o, b"".join(g1s) or b"\0", b"".join(g2s) or b"\0", _i64arr(offs), ctypes.c_int64(k))
    return [o.raw[576 * j : 576 * (j + 1)] for j in range(k)]


def final_exp(f: bytes) -> bytes:
    o = _buf(576)
    lib().orc_final_exp(o, f)
    return o.raw


def final_exp_many(fs) -> list:
    n = len(fs)
    o = _buf(576 * max(1, n))
    lib().orc_final_exp_batch(o, b"".join(fs) or b"\0", ctypes.c_int64(n))
    return [o.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def easy_final_exp(f: bytes) -> bytes:
    o = _buf(576)
    lib().orc_easy_final_exp(o, f)
    return o.raw


def batch_easy_final_exp(fs) -> list:
    n = len(fs)
    o = _buf(576 * max(1, n))
    lib().orc_batch_easy_final_exp(o, b"".join(fs) or b"\0", ctypes.c_int64(n))
    return [o.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def hard_final_exp(f: bytes) -> bytes:
    o = _buf(576)
    lib().orc_hard_final_exp(o, f)
    return o.raw


def hard_final_exp_many(fs) -> list:
    n = len(fs)
    o = _buf(576 * max(1, n))
    lib().orc_hard_final_exp_batch(o, b"".join(fs) or b"\0", ctypes.c_int64(n))
    return [o.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def pairing(g1: bytes, g2: bytes) -> bytes:
    o = _buf(576)
    lib().orc_pairing(o, g1, g2)
    return o.raw


# ------------------------------------------------------------------ Fp12
def fp12_one() -> bytes:
    o = _buf(576)
    lib().orc_fp12_one(o)
    return o.raw


GT_IDENTITY = None  # filled lazily by gt_identity()


def gt_identity() -> bytes:
    return fp12_one()


def fp12_is_one(a: bytes) -> bool:
    return bool(lib().orc_fp12_is_one(a))


def fp12_mul(a: bytes, b: bytes) -> bytes:
    o = _buf(576)
    lib().orc_fp12_mul(o, a, b)
    return o.raw


def fp12_inv(a: bytes) -> bytes:
    o = _buf(576)
    lib().orc_fp12_inv(o, a)
    return o.raw


def fp12_conj(a: bytes) -> bytes:
    o = _buf(576)
    lib().orc_fp12_conj(o, a)
    return o.raw


def fp12_frobenius(a: bytes, k: int) -> bytes:
    o = _buf(576)
    lib().orc_fp12_frobenius(o, a, int(k))
    return o.raw


def fp12_pow(a: bytes, e: int) -> bytes:
    nbytes = max(1, (e.bit_length() + 7) // 8)
    o = _buf(576)
    lib().orc_fp12_pow(o, a, e.to_bytes(nbytes, "little"), nbytes)
    return o.raw


def gt_pow_many(bases, scalars) -> list:
    n = len(scalars)
    if isinstance(bases, (bytes, bytearray)):
        blob, stride = bytes(bases), 0
    else:
        blob, stride = b"".join(bases), 576
    o = _buf(576 * max(1, n))
    lib().orc_gt_pow_batch(o, blob, ctypes.c_int64(stride), scalars_bytes(scalars), ctypes.c_int64(n))
    return [o.raw[576 * i : 576 * (i + 1)] for i in range(n)]


def gt_pow_decomposed(a: bytes, s: int) -> bytes:
    o = _buf(576)
    lib().orc_gt_pow_decomposed(o, a, s2b(s))
    return o.raw


def base_x_decompose(s: int) -> list:
    out = (ctypes.c_uint64 * 4)()
    lib().orc_base_x_decompose(out, s2b(s))
    return list(out)


def wnaf4(v: int):
    out = (ctypes.c_int8 * 65)()
    n = lib().orc_wnaf4(out, ctypes.c_uint64(v))
    return list(out), int(n)


# ---------------------------------------------------------------- scalars
def lagrange_at_zero(points) -> list:
    n = len(points)
    o = _buf(32 * max(1, n))
    rc = lib().orc_lagrange_at_zero(o, scalars_bytes(points), ctypes.c_int64(n))
    if rc != 0:
        raise ValueError("interpolation points must be distinct")
    return [int.from_bytes(o.raw[32 * i : 32 * (i + 1)], "little") for i in range(n)]


def domain_generator(n: int, inverse: bool = False) -> int:
    """Generator of the size-n radix-2 subgroup (btx/src/fft.rs:165-178)."""
    lg = n.bit_length() - 1
    assert 1 << lg == n and lg <= 32
    g = fr_root_of_unity()
    for _ in range(lg, 32):
        g = g * g % R
    return pow(g, R - 2, R) if inverse else g


def gt_compress(a: bytes) -> bytes:
    o = _buf(289)
    lib().orc_gt_compress(o, a)
    return o.raw


def append_gt(a: bytes) -> bytes:
    """Tagged GT encoding: b'\\x00' for the identity, else b'\\x01' + 288 bytes."""
    c = gt_compress(a)
    return c[:1] if c[0] == 0 else c


def g1_mul_generator_many(scalars) -> list:
    n = len(scalars)
    o = _buf(96 * max(1, n))
    lib().orc_g1_mul_generator_batch(o, scalars_bytes(scalars), ctypes.c_int64(n))
    return [o.raw[96 * i : 96 * (i + 1)] for i in range(n)]


def g2_mul_generator_blob(scalar_blob: bytes, n: int) -> bytes:
    o = _buf(192 * max(1, n))
    lib().orc_g2_mul_generator_batch(o, scalar_blob, ctypes.c_int64(n))
    return o.raw[: 192 * n]
