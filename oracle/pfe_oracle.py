"""CPU restatement of the pfe (partial-fraction BTE, Constructions 1-4)
pipeline (test infrastructure only).

Follows the reference crate step by step with the C oracle's group
arithmetic: keygen with the auxiliary index gamma and per-slot Shamir sharing
(pfe/src/setup.rs:78-186, :244-273), encryption and the DLEQ proof
(encryption.rs:23-53, proof.rs:24-176), validation and the ordered-batch digest
(decryption.rs:64-147, :633-645), the partial-fraction kernel (:151-257),
precomputation (:259-298), partial decryption, combination and checks
(:300-415), opening (:417-469) and the gamma-weighted cyclic convolution
(:471-526).

Randomness is drawn from the caller's generator in the reference's order.
"""
from __future__ import annotations

import hashlib
import struct

from . import oracle as O
from .wbtx_oracle import gt_generator, random_scalar

R = O.R
TRANSCRIPT_DOMAIN = b"PFE-CONSTRUCTION4-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"PFE-ORDERED-BATCH-BLS12381-v1"


def inv(x: int) -> int:
    return pow(x % R, R - 2, R)


def index_points(B: int) -> list:
    if B == 1:
        return [1]
    g = O.domain_generator(B)
    out, x = [], 1
    for _ in range(B):
        out.append(x)
        x = x * g % R
    return out


def extra_index_data(B: int):
    """Smallest c >= 2 with c^B != 1; gamma = 1/c (setup.rs:255-273)."""
    c = 2
    while pow(c, B, R) == 1:
        c += 1
    return inv(c), c


def _poly_eval(coeffs, x: int) -> int:
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % R
    return acc


def keygen(B: int, N: int, t: int, rng, publish: bool = True) -> dict:
    pts = index_points(B)
    gamma, c = extra_index_data(B)
    while True:
        x = random_scalar(rng)
        dens = [x, (x + gamma) % R] + [(x + p) % R for p in pts]
        if any(d == 0 for d in dens):
            continue
        invs = [inv(d) for d in dens]
        p_zero, fractions, rel = invs[0], invs[2:], sum(invs) % R
        break
    relation_base = O.g1_mul(O.g1_generator(), rel)
    masking_base = O.fp12_pow(gt_generator(), p_zero)
    keys = O.g2_mul_generator_blob(b"".join(O.s2b(f) for f in fractions), B)
    key_sum = O.G2_IDENTITY
    for i in range(B):
        key_sum = O.g2_add(key_sum, keys[192 * i : 192 * (i + 1)])
    domain = [j + 1 for j in range(N)]
    polys = [[f] + [random_scalar(rng) for _ in range(t)] for f in fractions]
    shares = [[_poly_eval(polys[i], domain[j]) for i in range(B)] for j in range(N)]
    commitments = None
    if publish:
        commitments = [O.g2_mul_generator_blob(b"".join(O.s2b(s) for s in shares[j]), B) for j in range(N)]
    return dict(B=B, N=N, t=t, x=x, gamma=gamma, c=c, points=pts, relation_base=relation_base,
                masking_base=masking_base, keys=keys, key_sum=key_sum, domain=domain, shares=shares,
                commitments=commitments, fractions=fractions)


def _challenge(rb, first, second, c1, c2) -> int:
    prefix = TRANSCRIPT_DOMAIN + b"".join(O.g1_compress(p) for p in (rb, first, second, c1, c2))
    counter = 0
    while True:
        d = hashlib.sha256(prefix + struct.pack("<I", counter)).digest()
        v = int.from_bytes(d, "little")
        if v < R:
            return v
        counter += 1


def encrypt_many(key: dict, messages, rng) -> list:
    out = []
    g1, rb = O.g1_generator(), key["relation_base"]
    for m in messages:
        r = random_scalar(rng)
        first, second = O.g1_mul(g1, r), O.g1_mul(rb, r)
        third = O.fp12_mul(m, O.fp12_pow(key["masking_base"], r))
        k = random_scalar(rng)
        c1, c2 = O.g1_mul(g1, k), O.g1_mul(rb, k)
        ch = _challenge(rb, first, second, c1, c2)
        out.append(dict(first=first, second=second, third=third, response=(k + ch * r) % R, c1=c1, c2=c2))
    return out


def verify_ct(key: dict, ct) -> bool:
    rb = key["relation_base"]
    ch = _challenge(rb, ct["first"], ct["second"], ct["c1"], ct["c2"])
    ok1 = O.g1_add(ct["c1"], O.g1_mul(ct["first"], ch)) == O.g1_mul(O.g1_generator(), ct["response"])
    ok2 = O.g1_add(ct["c2"], O.g1_mul(ct["second"], ch)) == O.g1_mul(rb, ct["response"])
    return ok1 and ok2


def batch_digest(cts) -> bytes:
    body = struct.pack("<Q", len(cts))
    for ct in cts:
        body += (O.g1_compress(ct["first"]) + O.g1_compress(ct["second"]) + O.append_gt(ct["third"])
                 + ct["response"].to_bytes(32, "little") + O.g1_compress(ct["c1"]) + O.g1_compress(ct["c2"]))
    return hashlib.sha256(BATCH_DIGEST_DOMAIN + body).digest()


def validate(key: dict, cts) -> dict:
    if len(cts) != key["B"]:
        raise ValueError("mismatched batch size")
    if not all(verify_ct(key, ct) for ct in cts):
        raise ValueError("invalid proof")
    return dict(first=[ct["first"] for ct in cts], second=[ct["second"] for ct in cts], digest=batch_digest(cts),
                B=len(cts))


def _coeffs(B: int) -> list:
    return [B - 1 - 2 * k for k in range(B)]


def conv_group(values, c: int, mul, add, neg, ntt) -> list:
    """FFT, times B - 1 - 2k, remap to c spec[k+1] - spec[k], unscaled inverse
    FFT (decryption.rs:471-499)."""
    B = len(values)
    spec = ntt(list(values), False) if B > 1 else list(values)
    spec = [mul(v, e % R) for v, e in zip(spec, _coeffs(B))]
    rem = [add(mul(spec[(i + 1) % B], c), neg(spec[i])) for i in range(B)]
    return ntt(rem, True) if B > 1 else rem


def conv_g1(values, c):
    return conv_group(values, c, O.g1_mul, O.g1_add, O.g1_neg, lambda v, inv_: O.g1_ntt(v, inverse=inv_))


def conv_g2(values, c):
    return conv_group(values, c, O.g2_mul, O.g2_add, O.g2_neg, lambda v, inv_: O.g2_ntt(v, inverse=inv_))


def conv_gt(values, c):
    return conv_group(values, c, O.fp12_pow, O.fp12_mul, O.fp12_inv, lambda v, inv_: O.gt_ntt(v, inverse=inv_))


def kernel(key: dict) -> dict:
    B = key["B"]
    pts, gamma, c = key["points"], key["gamma"], key["c"]
    half_b1 = (B + 1) * inv(2) % R
    open_coef = [(inv(p) * half_b1 + inv(p - gamma)) % R for p in pts]
    inv2b = inv(2 * B)
    scaled_keys = [O.g2_mul(key["keys"][192 * i : 192 * (i + 1)], inv2b) for i in range(B)]
    weighted = conv_g2(scaled_keys, c)
    s1_bar, gens, mixes = [], [], []
    for i, p in enumerate(pts):
        s2 = p * c % R
        s1 = p * (s2 - 1) % R
        sb = 2 * B * s1 % R
        s1_bar.append(sb)
        gens.append(O.g2_mul(O.g2_generator(), s2))
        proof_term = O.g2_mul(scaled_keys[i], sb * open_coef[i] % R)
        mixes.append(O.g2_add(O.g2_add(weighted[i], O.g2_neg(O.g2_mul(key["key_sum"], s2))), O.g2_neg(proof_term)))
    return dict(B=B, c=c, s1_bar=s1_bar, scaled_keys=scaled_keys, gens=gens, mixes=mixes)


def precompute(kern: dict, batch: dict) -> dict:
    wf = conv_g1(batch["first"], kern["c"])
    pairings = [O.pairing(f, k) for f, k in zip(batch["first"], kern["scaled_keys"])]
    return dict(weighted_first=wf, weighted_pairings=conv_gt(pairings, kern["c"]))


def partial_decrypt(key: dict, j: int, batch: dict) -> bytes:
    return O.g1_msm(batch["first"], key["shares"][j])


def combine(key: dict, shares) -> bytes:
    lam = O.lagrange_at_zero([key["domain"][j] for j, _ in shares])
    return O.g1_msm([s for _, s in shares], lam)


def _pairing_product_is_one(left, right) -> bool:
    return O.fp12_is_one(O.final_exp(O.multi_miller_many([(left, right)])[0]))


def verify_combined(key: dict, batch: dict, pdk: bytes) -> bool:
    left = list(batch["first"]) + [O.g1_neg(pdk)]
    right = [key["keys"][192 * i : 192 * (i + 1)] for i in range(key["B"])] + [O.g2_generator()]
    return _pairing_product_is_one(left, right)


def verify_share(key: dict, batch: dict, j: int, sigma: bytes) -> bool:
    com = key["commitments"][j]
    left = list(batch["first"]) + [O.g1_neg(sigma)]
    right = [com[192 * i : 192 * (i + 1)] for i in range(key["B"])] + [O.g2_generator()]
    return _pairing_product_is_one(left, right)


def open_batch(kern: dict, batch: dict, cts, bp: dict, pdk: bytes) -> list:
    out = []
    for i, ct in enumerate(cts):
        b0 = batch["second"][i]
        b1 = O.g1_add(bp["weighted_first"][i], O.g1_neg(O.g1_mul(O.g1_add(b0, O.g1_neg(pdk)), kern["s1_bar"][i])))
        b2 = batch["first"][i]
        f = O.multi_miller_many([([b0, b1, b2], [kern["gens"][i], kern["scaled_keys"][i], kern["mixes"][i]])])[0]
        mask = O.fp12_mul(O.final_exp(f), O.fp12_inv(bp["weighted_pairings"][i]))
        out.append(O.fp12_mul(ct["third"], O.fp12_inv(mask)))
    return out
