"""CPU restatement of the btx decryption pipeline (test infrastructure only).

Follows the reference crate step by step with the C oracle's group
arithmetic: trusted-dealer keygen with per-power Shamir sharing
(btx/src/setup.rs:92-178), encryption and Schnorr proofs
(btx/src/encryption.rs:20-40, btx/src/proof.rs:28-77), validation and the
ordered-batch digest (btx/src/decryption.rs:57-128, 510-518), the middle
product kernel (decryption.rs:131-190), precomputation (:201-246),
partial decryption (:248-264), share combination and checks (:266-400),
opening (:402-458), and the quadratic cross-term formula of the reference's
differential test (:520-537).

Randomness is drawn from the caller's generator in the reference's order.
"""
from __future__ import annotations

import hashlib
import struct

from . import oracle as O
from .wbtx_oracle import gt_generator, random_scalar, sample_nonzero

R = O.R
TRANSCRIPT_DOMAIN = b"BTX-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"BTX-ORDERED-BATCH-v1"


def _poly_eval(coeffs, x: int) -> int:
    acc = 0
    for c in reversed(coeffs):
        acc = (acc * x + c) % R
    return acc


def keygen(L: int, N: int, t: int, rng, publish: bool = True) -> dict:
    tau = sample_nonzero(rng)
    powers = [1]
    for _ in range(2 * L):
        powers.append(powers[-1] * tau % R)
    ek = O.fp12_pow(gt_generator(), powers[L + 1])
    low = O.g2_mul_generator_blob(b"".join(O.s2b(p) for p in powers[1 : L + 1]), L)
    high = O.g2_mul_generator_blob(b"".join(O.s2b(p) for p in powers[L + 2 : 2 * L + 1]), L - 1) if L > 1 else b""
    domain = [j + 1 for j in range(N)]
    polys = []
    for power in range(1, L + 1):
        polys.append([powers[power]] + [random_scalar(rng) for _ in range(t)])
    shares = [[_poly_eval(polys[i], domain[j]) for i in range(L)] for j in range(N)]
    commitments = None
    if publish:
        commitments = [O.g2_mul_generator_blob(b"".join(O.s2b(s) for s in shares[j]), L) for j in range(N)]
    return dict(L=L, N=N, t=t, tau=tau, ek=ek, low=low, high=high, domain=domain, shares=shares,
                commitments=commitments)


def power(key: dict, e: int) -> bytes:
    L = key["L"]
    if 1 <= e <= L:
        return key["low"][192 * (e - 1) : 192 * e]
    if L + 2 <= e <= 2 * L:
        i = e - L - 2
        return key["high"][192 * i : 192 * (i + 1)]
    raise ValueError(f"no key power {e}")


def centered_power(key: dict, offset: int) -> bytes:
    return power(key, key["L"] + 1 + offset)


def _challenge(first, second, commitment) -> int:
    prefix = (TRANSCRIPT_DOMAIN + O.g1_compress(O.g1_generator()) + O.g1_compress(first) + O.append_gt(second)
              + O.g1_compress(commitment))
    counter = 0
    while True:
        d = hashlib.sha256(prefix + struct.pack("<I", counter)).digest()
        v = int.from_bytes(d, "little")
        if v < R:
            return v
        counter += 1


def encrypt_many(key: dict, messages, rng) -> list:
    out = []
    g1 = O.g1_generator()
    for m in messages:
        r = random_scalar(rng)
        k = random_scalar(rng)
        first = O.g1_mul(g1, r)
        second = O.fp12_mul(m, O.fp12_pow(key["ek"], r))
        comm = O.g1_mul(g1, k)
        c = _challenge(first, second, comm)
        out.append(dict(first=first, second=second, commitment=comm, response=(k + c * r) % R))
    return out


def verify_ct(ct) -> bool:
    c = _challenge(ct["first"], ct["second"], ct["commitment"])
    lhs = O.g1_mul(O.g1_generator(), ct["response"])
    rhs = O.g1_add(ct["commitment"], O.g1_mul(ct["first"], c))
    return lhs == rhs


def batch_digest(cts) -> bytes:
    h = hashlib.sha256()
    h.update(BATCH_DIGEST_DOMAIN)
    h.update(struct.pack("<Q", len(cts)))
    for ct in cts:
        h.update(O.g1_compress(ct["first"]) + O.append_gt(ct["second"]) + O.g1_compress(ct["commitment"])
                 + ct["response"].to_bytes(32, "little"))
    return h.digest()


def validate(cts, verify: bool = True) -> dict:
    valid = [verify_ct(ct) for ct in cts] if verify else [True] * len(cts)
    first = [ct["first"] if v else O.G1_IDENTITY for ct, v in zip(cts, valid)]
    return dict(valid=valid, first=first, digest=batch_digest(cts), B=len(cts))


def kernel(key: dict, B: int) -> dict:
    """MiddleProductKernel::new: centered cyclic kernel K[d] = h_{-d},
    K[m-d] = h_d, forward transform, 1/m scaling, and the opening powers
    h_{-(slot+1)}."""
    m = 1 << (2 * B - 1).bit_length()
    ker = [O.G2_IDENTITY] * m
    for d in range(1, B):
        ker[d] = centered_power(key, -d)
        ker[m - d] = centered_power(key, d)
    ker = O.g2_ntt(ker)
    ker = O.g2_mul_many(ker, [pow(m, R - 2, R)] * m)
    opening = [centered_power(key, -(slot + 1)) for slot in range(B)]
    return dict(m=m, B=B, kernel=ker, opening=opening)


def precompute(kern: dict, batch: dict) -> list:
    m, B = kern["m"], batch["B"]
    x = O.g1_ntt(batch["first"] + [O.G1_IDENTITY] * (m - B))
    f = O.miller_loop_many(x, kern["kernel"])
    easy = O.batch_easy_final_exp(f)
    conv = O.cyclotomic_prefix_ifft(easy, B)
    return O.hard_final_exp_many(conv)


def partial_decrypt(key: dict, server: int, batch: dict) -> bytes:
    return O.g1_msm(batch["first"], key["shares"][server][: batch["B"]])


def combine(key: dict, shares) -> bytes:
    """shares: [(server_index, sigma)] in the caller's order."""
    lam = O.lagrange_at_zero([key["domain"][j] for j, _ in shares])
    return O.g1_msm([s for _, s in shares], lam)


def _pairing_product_is_one(left, right) -> bool:
    f = O.multi_miller_many([(left, right)])[0]
    return O.fp12_is_one(O.final_exp(f))


def verify_combined(key: dict, batch: dict, sigma: bytes) -> bool:
    slots = [i for i, v in enumerate(batch["valid"]) if v]
    left = [batch["first"][i] for i in slots] + [O.g1_neg(sigma)]
    right = [power(key, i + 1) for i in slots] + [O.g2_generator()]
    return _pairing_product_is_one(left, right)


def verify_share(key: dict, batch: dict, server: int, sigma: bytes) -> bool:
    slots = [i for i, v in enumerate(batch["valid"]) if v]
    com = key["commitments"][server]
    left = [batch["first"][i] for i in slots] + [O.g1_neg(sigma)]
    right = [com[192 * i : 192 * (i + 1)] for i in slots] + [O.g2_generator()]
    return _pairing_product_is_one(left, right)


def open_batch(kern: dict, batch: dict, cts, beta, sigma: bytes) -> list:
    alpha = O.final_exp_many(O.miller_loop_many([sigma] * batch["B"], kern["opening"]))
    out = []
    for i, ct in enumerate(cts):
        if not batch["valid"][i]:
            out.append(None)
            continue
        out.append(O.fp12_mul(O.fp12_mul(ct["second"], O.fp12_inv(alpha[i])), beta[i]))
    return out


def naive_beta(key: dict, batch: dict) -> list:
    out = []
    B = batch["B"]
    for o in range(B):
        acc = O.fp12_one()
        for i in range(B):
            if i == o or not batch["valid"][i]:
                continue
            acc = O.fp12_mul(acc, O.pairing(batch["first"][i], centered_power(key, i - o)))
        out.append(acc)
    return out
