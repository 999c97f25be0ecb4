"""Decoding of compressed G1 / G2 points (the key material's wire format) on
the GPU: round trips against the encoder, the identity, and every rejection
the checked decoder makes (flags, non-canonical x, not on the curve, not in
the prime-order subgroup).  Off-subgroup and off-curve inputs are built here
with Python integers; the oracle supplies the points that round-trip."""
import random

import pytest

from weighted_bte_b200 import ops

pytestmark = pytest.mark.gpu
P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R_MONT_INV = pow(1 << 384, P - 2, P)


def _legendre(v):
    return pow(v % P, (P - 1) // 2, P)


def _fp_from_limbs(b: bytes) -> int:
    """Canonical value of a Montgomery Fp in the library's layout."""
    return int.from_bytes(b, "little") * R_MONT_INV % P


def _be48(x: int, flags: int = 0x80) -> bytes:
    out = bytearray(x.to_bytes(48, "big"))
    out[0] |= flags
    return bytes(out)


def test_round_trip_and_identity(orc):
    rng = random.Random(9)
    g1 = orc.g1_mul_many(orc.g1_generator(), [rng.randrange(1, orc.R) for _ in range(200)]) + [orc.G1_IDENTITY]
    g2 = orc.g2_mul_many(orc.g2_generator(), [rng.randrange(1, orc.R) for _ in range(100)]) + [bytes(192)]
    for pts, size, comp, dec in ((g1, 96, ops.g1_compress, ops.g1_decompress),
                                 (g2, 192, ops.g2_compress, ops.g2_decompress)):
        blob = comp(b"".join(pts), len(pts))
        out, status = dec(blob)
        assert status == [0] * len(pts)
        assert out == b"".join(pts)
        # the sort flag selects the other root: the negated point
        flipped = bytearray(blob[: size // 2])
        flipped[0] ^= 0x20
        neg, st = dec(bytes(flipped))
        assert st == [0] and neg != pts[0][:size] and comp(neg, 1) == bytes(flipped)


def test_g1_rejections():
    rng = random.Random(10)
    cases, expect = [], []
    cases.append(_be48(5, flags=0x00)); expect.append(1)                 # not compressed
    inf = bytearray(48); inf[0] = 0xC0; inf[47] = 1
    cases.append(bytes(inf)); expect.append(1)                           # identity with payload
    inf = bytearray(48); inf[0] = 0xE0
    cases.append(bytes(inf)); expect.append(1)                           # identity with sort flag
    cases.append(_be48(P)); expect.append(1)                              # x = p
    while True:                                                           # x^3 + 4 not a square
        x = rng.randrange(P)
        if _legendre(x * x * x + 4) == P - 1:
            break
    cases.append(_be48(x)); expect.append(2)
    while True:                                                           # on E(Fp), not in G1
        x = rng.randrange(P)
        if _legendre(x * x * x + 4) == 1:
            break
    cases.append(_be48(x)); expect.append(3)
    out, status = ops.g1_decompress(b"".join(cases))
    assert status == expect
    assert out[96 * 5 : 96 * 6] == bytes(96)
    # without the subgroup check the curve point decodes
    out, status = ops.g1_decompress(cases[-1], check_group=False)
    assert status == [0]
    xx, yy = _fp_from_limbs(out[:48]), _fp_from_limbs(out[48:96])
    assert xx == x and yy * yy % P == (x ** 3 + 4) % P


def _fp2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def _g2_rhs(x):
    x3 = _fp2_mul(_fp2_mul(x, x), x)
    return ((x3[0] + 4) % P, (x3[1] + 4) % P)


def _be96(x, flags=0x80):
    return _be48(x[1], flags) + x[0].to_bytes(48, "big")


def test_g2_rejections():
    rng = random.Random(11)
    cases, expect = [], []
    cases.append(_be96((3, 5), flags=0x00)); expect.append(1)
    cases.append(_be96((P, 1))); expect.append(1)                         # x.c0 = p
    cases.append(_be96((1, P))); expect.append(1)                         # x.c1 = p
    while True:                                                           # rhs not a square in Fp2
        x = (rng.randrange(P), rng.randrange(P))
        r = _g2_rhs(x)
        if _legendre(r[0] * r[0] + r[1] * r[1]) == P - 1:
            break
    cases.append(_be96(x)); expect.append(2)
    while True:                                                           # on E'(Fp2), not in G2
        x = (rng.randrange(P), rng.randrange(P))
        r = _g2_rhs(x)
        if _legendre(r[0] * r[0] + r[1] * r[1]) == 1:
            break
    cases.append(_be96(x)); expect.append(3)
    out, status = ops.g2_decompress(b"".join(cases))
    assert status == expect
    out, status = ops.g2_decompress(cases[-1], check_group=False)
    assert status == [0]
    y = (_fp_from_limbs(out[96:144]), _fp_from_limbs(out[144:192]))
    assert _fp_from_limbs(out[:48]) == x[0] and _fp_from_limbs(out[48:96]) == x[1]
    assert _fp2_mul(y, y) == r


def test_key_material_round_trips_through_the_wire_format():
    """A G2 stream of key material (CRS points) decodes to the same points."""
    from weighted_bte_b200 import weighted_btx as wb

    rng = random.Random(12)
    pts = ops.g2_mul_generator([rng.randrange(1, ops.R) for _ in range(4096)])
    blob = ops.g2_compress(pts, 4096)
    out, status = ops.g2_decompress(blob)
    assert status == [0] * 4096 and out == pts
    assert wb.to_host(wb.to_device(pts)) == pts


def test_public_decryption_key_wire_round_trip():
    """weighted_btx key material written as compressed G2 streams and loaded
    back through the checked device decoder decrypts the same batch; a
    corrupted point is refused."""
    from weighted_bte_b200 import weighted_btx as wb
    from weighted_bte_b200.rng import ChaCha20Rng

    rng = ChaCha20Rng.seed_from_u64(13)
    mat = wb.keygen_with_rng(wb.KeygenConfig(4, [3, 2, 4], 4), rng)
    dk = mat.decryption_key
    blob = dk.to_wire()
    assert len(blob) > 96 * (4 * 3 + 4 * 9 + 3 * 9)
    dk2 = wb.PublicDecryptionKey.from_wire(blob)
    assert dk2.setup_id() == dk.setup_id() and dk2.party_weights() == dk.party_weights()
    assert dk2.domain_points() == dk.domain_points() and dk2.threshold_weight() == dk.threshold_weight()
    for power in (1, 4):
        assert dk2.verification_power(power) == dk.verification_power(power)
        assert dk2.negative_power(power) == dk.negative_power(power)
    assert dk2.positive_power(3) == dk.positive_power(3)
    msgs = wb.messages_from_bytes([bytes([i]) * 32 for i in range(4)])
    cts = wb.encrypt_many(mat.encryption_key, msgs, rng)
    batch = wb.validate_batch(dk2, cts)
    shares = wb.partial_decrypt_many([mat.party_keys[0], mat.party_keys[2]], batch)
    assert wb.decrypt(dk2, cts, shares) == msgs
    bad = bytearray(blob)
    bad[-96 * 5 + 20] ^= 0x01  # a point of the positive material
    with pytest.raises(ValueError):
        wb.PublicDecryptionKey.from_wire(bytes(bad))
