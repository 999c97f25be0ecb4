"""Shared inversions (Montgomery's trick): the batched easy part of the final
exponentiation (batch_easy_final_exponentiation,
btx/src/final_exponentiation.rs:228-252) and batched projective-to-affine
normalization (blst_p{1,2}s_to_affine, weighted_btx/src/blst_utils.rs:11-36)
must equal the per-value results bit for bit, including the values the
shared product has to leave out (zero Fp12 values, points at infinity)."""
import random

import pytest

from weighted_bte_b200 import ops

pytestmark = pytest.mark.gpu

P = int("1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab", 16)
R_MONT = pow(2, 384, P)
R_INV = pow(R_MONT, P - 2, P)
N_CHUNKED = 80000  # enough values that the launchers give each thread a chunk of several


def fp_from(b: bytes) -> int:
    return int.from_bytes(b, "little") * R_INV % P


def fp_to(v: int) -> bytes:
    return (v % P * R_MONT % P).to_bytes(48, "little")


def fp2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def test_batched_easy_part_equals_the_per_value_easy_part():
    import torch

    torch.cuda.set_device(0)
    rng = random.Random(91)
    n = 2 * N_CHUNKED
    g1 = ops.g1_mul_generator([rng.randrange(ops.R) for _ in range(n)])
    g2 = ops.g2_mul_generator([rng.randrange(ops.R) for _ in range(n)])
    f = bytearray(ops.miller_loop(g1, g2))
    f[576 * 7 : 576 * 8] = bytes(576)  # a zero value: no inverse, must not spoil its chunk
    f = bytes(f)
    for mode in (1, 0):
        batched = ops.final_exp(f, mode=mode)
        # per value: launches small enough that every thread takes one value
        for lo in (0, n // 2, n - 1000):
            per = ops.final_exp(f[576 * lo : 576 * (lo + 1000)], mode=mode)
            assert batched[576 * lo : 576 * (lo + 1000)] == per, f"mode {mode} at {lo}"
        assert batched[576 * 7 : 576 * 8] == bytes(576)


@pytest.mark.parametrize("group", [1, 2])
def test_batch_normalize_equals_the_affine_points(group):
    import torch

    torch.cuda.set_device(0)
    rng = random.Random(92 + group)
    n = N_CHUNKED
    aff = (ops.g1_mul_generator if group == 1 else ops.g2_mul_generator)([rng.randrange(ops.R) for _ in range(n)])
    size = 96 if group == 1 else 192
    idents = {5, 6, n // 2, n - 1}
    jac = bytearray()
    for i in range(n):
        if i in idents:
            jac += bytes(3 * size // 2)
            continue
        a = aff[size * i : size * (i + 1)]
        if group == 1:
            x, y = fp_from(a[:48]), fp_from(a[48:])
            z = rng.randrange(1, P)
            z2 = z * z % P
            jac += fp_to(x * z2) + fp_to(y * z2 * z) + fp_to(z)
        else:
            x = (fp_from(a[0:48]), fp_from(a[48:96]))
            y = (fp_from(a[96:144]), fp_from(a[144:192]))
            z = (rng.randrange(P), rng.randrange(1, P))
            z2 = fp2_mul(z, z)
            X, Y = fp2_mul(x, z2), fp2_mul(y, fp2_mul(z2, z))
            jac += b"".join(fp_to(v) for v in (X[0], X[1], Y[0], Y[1], z[0], z[1]))
    out = bytearray(size * n)
    ops.ctx().call("wbte_g1_batch_normalize" if group == 1 else "wbte_g2_batch_normalize", out, bytes(jac), n)
    expect = bytearray(aff)
    for i in idents:
        expect[size * i : size * (i + 1)] = bytes(size)
    assert bytes(out) == bytes(expect)
