"""CPU restatement of the weighted_btx decryption pipeline (test infrastructure only).

Follows the reference crate step by step using the C oracle's group
arithmetic: keygen (weighted_btx/src/setup.rs:98-233), encryption and
Schnorr proofs (encryption.rs:28-66, proof.rs:38-100), validation,
partial decryption, batched share verification, preparation, precomputation
and opening (decryption.rs:85-709), and the literal quadratic cross-term
formula of the reference's differential test (decryption.rs:806-842).

Randomness is drawn from the caller's generator in the reference's order; the
seeded generator (weighted_bte_b200.rng) is only an input source here.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import struct

from . import oracle as O

R = O.R
SETUP_ID_DOMAIN = b"WEIGHTED-BTX-SETUP-ID-v1"
TRANSCRIPT_DOMAIN = b"WEIGHTED-BTX-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"WEIGHTED-BTX-ORDERED-BATCH-v1"
DECRYPTION_CONTEXT_DOMAIN = b"WEIGHTED-BTX-DECRYPTION-CONTEXT-v1"


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


def gt_generator() -> bytes:
    return O.pairing(O.g1_generator(), O.g2_generator())


def domain_generator(size: int) -> int:
    return O.domain_generator(size)


def setup_identifier(ek, L, t, weights, vk_first, neg_first) -> bytes:
    h = hashlib.sha256()
    h.update(SETUP_ID_DOMAIN)
    for v in (L, t, len(weights)):
        h.update(struct.pack("<Q", v))
    for w in weights:
        h.update(struct.pack("<Q", w))
    h.update(O.append_gt(ek))
    for p in vk_first:
        h.update(O.g2_compress(p))
    for p in neg_first:
        h.update(O.g2_compress(p))
    return h.digest()


def keygen(L: int, weights, t: int, rng) -> dict:
    N, W = len(weights), sum(weights)
    domain = 1 << (W - 1).bit_length() if W > 1 else 1
    coeffs = [random_scalar(rng) for _ in range(t + 1)]
    z = coeffs[0]
    z_evals = O.fr_ntt(coeffs + [0] * (domain - len(coeffs)))[:W] if domain > 1 else [coeffs[0]]
    evaluation_domain = O.fr_ntt([0, 1] + [0] * (domain - 2))[:W] if domain > 1 else [1]
    offsets = [0]
    for w in weights:
        offsets.append(offsets[-1] + w)
    owner = [j for j, w in enumerate(weights) for _ in range(w)]
    qs = [sample_nonzero(rng) for _ in range(N)]
    vk_sc, neg_sc, pos_sc = bytearray(), bytearray(), bytearray()
    qinv = [pow(q, R - 2, R) for q in qs]
    qp, qn = list(qs), list(qinv)
    for i in range(1, L + 1):
        vk_sc += b"".join(O.s2b(v) for v in qp)
        neg_sc += b"".join(O.s2b(z_evals[w] * qn[owner[w]]) for w in range(W))
        if i < L:
            pos_sc += b"".join(O.s2b(z_evals[w] * qp[owner[w]]) for w in range(W))
        qp = [a * b % R for a, b in zip(qp, qs)]
        qn = [a * b % R for a, b in zip(qn, qinv)]
    vk_blob = O.g2_mul_generator_blob(bytes(vk_sc), L * N)
    neg_blob = O.g2_mul_generator_blob(bytes(neg_sc), L * W)
    pos_blob = O.g2_mul_generator_blob(bytes(pos_sc), (L - 1) * W) if L > 1 else b""
    ek = O.fp12_pow(gt_generator(), z)
    vk = [vk_blob[192 * i : 192 * (i + 1)] for i in range(L * N)]
    setup_id = setup_identifier(ek, L, t, weights, vk[:N], [neg_blob[192 * i : 192 * (i + 1)] for i in range(W)])
    return dict(ek=ek, setup_id=setup_id, L=L, t=t, weights=list(weights), W=W, N=N, domain=evaluation_domain,
                offsets=offsets, vk=vk, neg_blob=neg_blob, pos_blob=pos_blob, qs=qs, z=z)


def points(blob: bytes, size: int = 192) -> list:
    return [blob[size * i : size * (i + 1)] for i in range(len(blob) // size)]


def _challenge(setup_id, first, second, commitment) -> int:
    prefix = (TRANSCRIPT_DOMAIN + setup_id + O.g1_compress(O.g1_generator()) + O.g1_compress(first)
              + O.append_gt(second) + O.g1_compress(commitment))
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
        c = _challenge(key["setup_id"], first, second, comm)
        out.append(dict(first=first, second=second, commitment=comm, response=(k + c * r) % R))
    return out


def verify_ct(setup_id, ct) -> bool:
    c = _challenge(setup_id, ct["first"], ct["second"], ct["commitment"])
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


def _map(fn, items, threads: int):
    """map on `threads` host threads (the C calls release the interpreter lock),
    mirroring the reference's per-item rayon parallelism."""
    if threads <= 1 or len(items) < 2:
        return [fn(x) for x in items]
    with cf.ThreadPoolExecutor(threads) as ex:
        return list(ex.map(fn, items, chunksize=max(1, len(items) // (4 * threads))))


def validate(setup_id, cts, threads: int = 1) -> dict:
    valid = _map(lambda ct: verify_ct(setup_id, ct), list(cts), threads)
    first = [ct["first"] if v else O.G1_IDENTITY for ct, v in zip(cts, valid)]
    return dict(valid=valid, first=first, digest=batch_digest(cts), B=len(cts))


def partial_decrypt(q: int, batch: dict) -> bytes:
    B = batch["B"]
    scalars = [pow(q, i + 1, R) for i in range(B)]
    return O.g1_msm(batch["first"], scalars)


def verify_shares(key, batch, parties, sigmas, challenges, threads: int = 1) -> bool:
    """weighted_btx/src/decryption.rs:358-422 with the given challenges."""
    agg = O.g1_msm(sigmas, challenges)
    N = key["N"]
    slots = [slot for slot, v in enumerate(batch["valid"]) if v]
    right = _map(lambda slot: O.g2_msm([key["vk"][slot * N + j] for j in parties], challenges), slots, threads)
    left = [batch["first"][slot] for slot in slots]
    left.append(O.g1_neg(agg))
    right.append(O.g2_generator())
    f = O.multi_miller_many([(left, right)])[0]
    return O.fp12_is_one(O.final_exp(f))


def lagrange(key, selected):
    return O.lagrange_at_zero([key["domain"][i] for i in selected])


def prepare(key: dict, parties, B: int) -> dict:
    """weighted_btx/src/decryption.rs:427-551."""
    W = key["W"]
    selected, coef_off = [], [0]
    for j in parties:
        selected.extend(range(key["offsets"][j], key["offsets"][j + 1]))
        coef_off.append(len(selected))
    lam = lagrange(key, selected)
    T = len(parties)
    lam_blob = O.scalars_bytes(lam)
    neg_blob = key["neg_blob"]
    groups = []
    for slot in range(B):
        for k, j in enumerate(parties):
            lo, hi = key["offsets"][j], key["offsets"][j + 1]
            groups.append(([slot * W + w for w in range(lo, hi)], list(range(coef_off[k], coef_off[k + 1]))))
    opening = O.g2_msm_gather(neg_blob, groups, lam_blob)
    m = 1 << (2 * B - 1).bit_length()
    kernel = [O.G2_IDENTITY] * m
    for d in range(1, B):
        acc = O.G2_IDENTITY
        for p in opening[(d - 1) * T : d * T]:
            acc = O.g2_add(acc, p)
        kernel[d] = acc
    if B > 1:
        pos_blob = key["pos_blob"]
        pgroups = [([(d - 1) * W + w for w in selected], list(range(len(selected)))) for d in range(1, B)]
        pos = O.g2_msm_gather(pos_blob, pgroups, lam_blob)
        for d, p in zip(range(1, B), pos):
            kernel[m - d] = p
    kernel = O.g2_ntt(kernel)
    kernel = O.g2_mul_many(kernel, [pow(m, R - 2, R)] * m)
    h = hashlib.sha256()
    h.update(DECRYPTION_CONTEXT_DOMAIN)
    h.update(key["setup_id"])
    h.update(struct.pack("<Q", B))
    h.update(struct.pack("<Q", T))
    for j in parties:
        h.update(struct.pack("<Q", j))
    return dict(kernel=kernel, opening=opening, m=m, B=B, parties=list(parties), context_id=h.digest(),
                lam=lam, selected=selected)


def precompute(pre: dict, batch: dict) -> list:
    """weighted_btx/src/decryption.rs:555-603."""
    m, B = pre["m"], batch["B"]
    x = batch["first"] + [O.G1_IDENTITY] * (m - B)
    x = O.g1_ntt(x)
    f = O.miller_loop_many(x, pre["kernel"])
    easy = O.batch_easy_final_exp(f)
    conv = O.cyclotomic_prefix_ifft(easy, B)
    hard = O.hard_final_exp_many(conv)
    return [h if v else O.fp12_one() for h, v in zip(hard, batch["valid"])]


def open_batch(pre: dict, sigmas, batch: dict, cts, beta) -> list:
    """weighted_btx/src/decryption.rs:607-695."""
    T = len(sigmas)
    groups = [(list(sigmas), pre["opening"][i * T : (i + 1) * T]) for i in range(batch["B"])]
    alpha = O.final_exp_many(O.multi_miller_many(groups))
    out = []
    for i, ct in enumerate(cts):
        if not batch["valid"][i]:
            out.append(None)
            continue
        out.append(O.fp12_mul(O.fp12_mul(ct["second"], O.fp12_inv(alpha[i])), beta[i]))
    return out


def naive_beta(key: dict, batch: dict, parties) -> list:
    """Literal quadratic cross terms (weighted_btx/src/decryption.rs:806-842)."""
    selected = []
    for j in parties:
        selected.extend(range(key["offsets"][j], key["offsets"][j + 1]))
    lam = lagrange(key, selected)
    W, B = key["W"], batch["B"]
    out = []
    for o in range(B):
        acc = O.fp12_one()
        for i in range(B):
            if i == o or not batch["valid"][i]:
                continue
            off = i - o
            bank = key["neg_blob"] if off < 0 else key["pos_blob"]
            power = abs(off)
            bases = [bank[192 * ((power - 1) * W + w) : 192 * ((power - 1) * W + w + 1)] for w in selected]
            agg = O.g2_msm(bases, lam)
            acc = O.fp12_mul(acc, O.pairing(batch["first"][i], agg))
        out.append(acc)
    return out
