"""Primitive operations of libwbte with bytes-in / bytes-out conveniences.

All values use blst's memory layout (see include/wbte.h).  Inputs may also
be CUDA tensors (resident in HBM); outputs are returned as `bytes` unless an
`out=` buffer is given.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import _lib
from ._lib import FR_BYTES, G1_BYTES, G2_BYTES, GT_BYTES, LINE_BYTES, MILLER_LINES

R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


def current_device() -> int:
    """The calling thread's current CUDA device as torch sees it (0 before
    torch is imported)."""
    import sys

    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available():
        return torch.cuda.current_device()
    return 0


def ctx(device: Optional[int] = None) -> _lib.Context:
    """The calling thread's library context on `device`, by default the
    thread's current CUDA device."""
    return _lib.default_context(current_device() if device is None else device)


def scalars_bytes(scalars) -> bytes:
    if isinstance(scalars, (bytes, bytearray)):
        return bytes(scalars)
    return b"".join((int(s) % R).to_bytes(32, "little") for s in scalars)


def _out(n: int, out=None):
    return out if out is not None else bytearray(n)


def _ret(buf, out):
    return bytes(buf) if out is None else out


def _nbytes(x) -> int:
    if hasattr(x, "nbytes"):
        return int(x.nbytes)
    return len(x)


# ------------------------------------------------------------------ MSM
def g1_msm(points, scalars, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G1_BYTES, out)
    ctx().call("wbte_g1_msm", buf, points, sc, n)
    return _ret(buf, out)


def g2_msm(points, scalars, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G2_BYTES, out)
    ctx().call("wbte_g2_msm", buf, points, sc, n)
    return _ret(buf, out)


def msm_family(group: int, points, n_points: int, point_base, point_index, scalars, scalar_vector, num_vectors: int,
               n: int, out=None):
    k = len(point_base)
    size = G1_BYTES if group == 1 else G2_BYTES
    buf = _out(size * k, out)
    name = "wbte_g1_msm_family" if group == 1 else "wbte_g2_msm_family"
    ctx().call(name, buf, points, n_points, _lib.i64_array(point_base),
               None if point_index is None else _lib.i32_array(point_index), scalars_bytes(scalars),
               None if scalar_vector is None else _lib.i32_array(scalar_vector), num_vectors, k, n)
    return _ret(buf, out)


# --------------------------------------------------------- point ops
def g1_mul(points, scalars, fixed_base=False, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G1_BYTES * n, out)
    ctx().call("wbte_g1_mul", buf, points, int(fixed_base), sc, n)
    return _ret(buf, out)


def g2_mul(points, scalars, fixed_base=False, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G2_BYTES * n, out)
    ctx().call("wbte_g2_mul", buf, points, int(fixed_base), sc, n)
    return _ret(buf, out)


def g1_mul_generator(scalars, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G1_BYTES * n, out)
    ctx().call("wbte_g1_mul_generator", buf, sc, n)
    return _ret(buf, out)


def g2_mul_generator(scalars, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(G2_BYTES * n, out)
    ctx().call("wbte_g2_mul_generator", buf, sc, n)
    return _ret(buf, out)


def g1_sum(points, offsets, out=None):
    k = len(offsets) - 1
    buf = _out(G1_BYTES * k, out)
    ctx().call("wbte_g1_sum", buf, points, _lib.i64_array(offsets), k)
    return _ret(buf, out)


def g2_sum(points, offsets, out=None):
    k = len(offsets) - 1
    buf = _out(G2_BYTES * k, out)
    ctx().call("wbte_g2_sum", buf, points, _lib.i64_array(offsets), k)
    return _ret(buf, out)


def g1_compress(points, n: int | None = None):
    n = _nbytes(points) // G1_BYTES if n is None else n
    buf = bytearray(48 * n)
    ctx().call("wbte_g1_compress", buf, points, n)
    return bytes(buf)


def g2_compress(points, n: int | None = None):
    n = _nbytes(points) // G2_BYTES if n is None else n
    buf = bytearray(96 * n)
    ctx().call("wbte_g2_compress", buf, points, n)
    return bytes(buf)


# -------------------------------------------------------- transforms
def _decompress(name: str, size: int, blob, check_group: bool):
    n = _nbytes(blob) // (size // 2)
    out = bytearray(size * n)
    status = np.zeros(max(1, n), dtype=np.uint8)
    try:
        ctx().call(name, out, status, blob, n, int(check_group))
    except _lib.WbteError as err:
        if err.status != -6:  # WBTE_ERR_NOT_ON_CURVE: the per-point status says which
            raise
    return bytes(out), [int(x) for x in status[:n]]


def g1_decompress(blob, check_group: bool = True):
    """Affine points and per-point status (0 ok, 1 bad encoding, 2 not on the
    curve, 3 not in the subgroup) of 48-byte compressed G1 points."""
    return _decompress("wbte_g1_decompress", G1_BYTES, blob, check_group)


def g2_decompress(blob, check_group: bool = True):
    """As g1_decompress for 96-byte compressed G2 points."""
    return _decompress("wbte_g2_decompress", G2_BYTES, blob, check_group)


def g1_ntt(points, inverse=False):
    buf = bytearray(points)
    ctx().call("wbte_g1_ntt", buf, len(buf) // G1_BYTES, int(inverse))
    return bytes(buf)


def g2_ntt(points, inverse=False):
    buf = bytearray(points)
    ctx().call("wbte_g2_ntt", buf, len(buf) // G2_BYTES, int(inverse))
    return bytes(buf)


def gt_ntt(values, inverse=False):
    buf = bytearray(values)
    ctx().call("wbte_gt_ntt", buf, len(buf) // GT_BYTES, int(inverse))
    return bytes(buf)


def gt_ntt_many(values, n: int, inverse=False):
    """`gt_ntt` of len(values) / (576 n) arrays of n values laid back to back."""
    buf = bytearray(values)
    ctx().call("wbte_gt_ntt_many", buf, n, len(buf) // (GT_BYTES * n), int(inverse))
    return bytes(buf)


def cyclotomic_prefix_ifft_many(values, n: int, out_count: int) -> list:
    """`cyclotomic_prefix_ifft` of arrays of n values laid back to back; the
    first out_count outputs of each."""
    buf = bytearray(values)
    count = len(buf) // (GT_BYTES * n)
    ctx().call("wbte_gt_cyclotomic_prefix_ifft_many", buf, n, out_count, count)
    return [bytes(buf[GT_BYTES * n * q : GT_BYTES * (n * q + out_count)]) for q in range(count)]


def cyclotomic_prefix_ifft(values, out_count: int):
    buf = bytearray(values)
    ctx().call("wbte_gt_cyclotomic_prefix_ifft", buf, len(buf) // GT_BYTES, out_count)
    return bytes(buf[: GT_BYTES * out_count])


# ------------------------------------------------------------ pairing
def prepare_lines(q):
    n = _nbytes(q) // G2_BYTES
    buf = bytearray(LINE_BYTES * MILLER_LINES * n)
    ctx().call("wbte_g2_prepare_lines", buf, q, n)
    return bytes(buf)


def miller_loop_lines(lines, p):
    n = _nbytes(p) // G1_BYTES
    buf = bytearray(GT_BYTES * n)
    ctx().call("wbte_miller_loop_lines", buf, lines, p, n)
    return bytes(buf)


def miller_loop(p, q):
    n = _nbytes(p) // G1_BYTES
    buf = bytearray(GT_BYTES * n)
    ctx().call("wbte_miller_loop", buf, p, q, n)
    return bytes(buf)


def multi_miller_loop(p, q, offsets):
    k = len(offsets) - 1
    buf = bytearray(GT_BYTES * k)
    ctx().call("wbte_multi_miller_loop", buf, p, q, _lib.i64_array(offsets), k)
    return bytes(buf)


def final_exp(values, mode=_lib.FE_FULL):
    n = _nbytes(values) // GT_BYTES
    buf = bytearray(GT_BYTES * n)
    ctx().call("wbte_final_exp", buf, values, n, mode)
    return bytes(buf)


def gt_pow(bases, scalars, fixed_base=False, out=None):
    sc = scalars_bytes(scalars)
    n = len(sc) // 32
    buf = _out(GT_BYTES * n, out)
    ctx().call("wbte_gt_pow", buf, bases, int(fixed_base), sc, n)
    return _ret(buf, out)


def fp12_mul(a, b, out=None):
    n = _nbytes(a) // GT_BYTES
    buf = _out(GT_BYTES * n, out)
    ctx().call("wbte_fp12_mul", buf, a, b, n)
    return _ret(buf, out)


def gt_compress(values, n: int | None = None):
    n = _nbytes(values) // GT_BYTES if n is None else n
    buf = bytearray(289 * n)
    ctx().call("wbte_gt_compress", buf, values, n)
    return bytes(buf)


def pairing(p, q):
    return final_exp(miller_loop(p, q))


# ------------------------------------------------------------ scalars
def lagrange_at_zero(points) -> list:
    sc = scalars_bytes(points)
    n = len(sc) // 32
    buf = bytearray(32 * n)
    ctx().call("wbte_lagrange_at_zero", buf, sc, n)
    return [int.from_bytes(buf[32 * i : 32 * i + 32], "little") for i in range(n)]


def schnorr_verify(X, Rc, s, c) -> np.ndarray:
    n = _nbytes(X) // G1_BYTES
    out = np.zeros(n, dtype=np.uint8)
    ctx().call("wbte_schnorr_verify", out, X, Rc, scalars_bytes(s), scalars_bytes(c), n)
    return out.astype(bool)


def transcript_challenges(fields, n: int, out=None):
    """Fiat-Shamir challenges of n records on the device (wbte_transcript_challenges).

    `fields` lists (data, stride, length, kind) in transcript order: record i
    contributes `length` bytes at data + i * stride (stride 0: constant bytes);
    kind TRANSCRIPT_GT_VARIABLE marks 289-byte compressed GT records encoded
    as one byte when they hold the identity.  Returns the scalars as ints, or
    writes 32-byte canonical scalars into `out` (host or device) and returns it.
    """
    keep = _lib._Keep()
    arr = (_lib.TranscriptField * max(1, len(fields)))()
    for k, (data, stride, length, kind) in enumerate(fields):
        arr[k].data = keep.ptr(data) if length else None
        arr[k].stride, arr[k].len, arr[k].kind = int(stride), int(length), int(kind)
    buf = out if out is not None else bytearray(32 * n)
    ctx().call("wbte_transcript_challenges", buf, arr, len(fields), n)
    if out is not None:
        return out
    return [int.from_bytes(buf[32 * i : 32 * i + 32], "little") for i in range(n)]


def split(blob: bytes, size: int) -> list:
    return [bytes(blob[i : i + size]) for i in range(0, len(blob), size)]
