"""CPU restatement of the weighted_pfe (Construction 5) pipeline (test
infrastructure only).

Follows the reference crate step by step with the C oracle's group
arithmetic: keygen with global masks and partial-fraction party keys
(weighted_pfe/src/setup.rs:142-354, helpers :592-749), encryption and Schnorr
transcripts (encryption.rs:22-55, proof.rs:27-152), the ordered-batch digest
(decryption.rs:851-861), partial decryption and share checks
(decryption.rs:231-419), committee preparation (:421-538), the Cauchy sums
through the closed-form spectrum B - 1 - 2k (:540-574, :683-760), the fused
opening (:576-644), and the literal formulas of the reference's differential
tests (:981-1124).

Randomness is drawn from the caller's generator in the reference's order.
Intermediate cyclotomic values are not canonical; only hard-final-exponentiated
values and group elements are compared.
"""
from __future__ import annotations

import hashlib
import struct

from . import oracle as O
from .wbtx_oracle import gt_generator, random_scalar, sample_nonzero

R = O.R
SETUP_ID_DOMAIN = b"WEIGHTED-PFE-SETUP-BLS12381-v2"
TRANSCRIPT_DOMAIN = b"WEIGHTED-PFE-CIPHERTEXT-SCHNORR-BLS12381-v1"
BATCH_DIGEST_DOMAIN = b"WEIGHTED-PFE-ORDERED-BATCH-v1"
COMMITTEE_CONTEXT_DOMAIN = b"WEIGHTED-PFE-COMMITTEE-v1"


def inv(x: int) -> int:
    return pow(x % R, R - 2, R)


def append_gt_fixed(value: bytes) -> bytes:
    """Tag and a fixed 288-byte body, zeros for the identity (encoding.rs:13-28)."""
    if O.fp12_is_one(value):
        return b"\x00" + bytes(288)
    return O.append_gt(value)


def root_domain_prefix(size: int, length: int) -> list:
    if size == 1:
        return [1][:length]
    return O.fr_ntt([0, 1] + [0] * (size - 2))[:length]


def shifted_alpha_points(B: int):
    roots = root_domain_prefix(B, B)
    c = 2
    while True:
        pts = [(r + c) % R for r in roots]
        if all(a != 0 and (a + 1) % R != 0 for a in pts):
            return pts, c
        c += 1


def keygen(B: int, weights, t: int, rng) -> dict:
    N, W = len(weights), sum(weights)
    domain_size = 1 << (W - 1).bit_length() if W > 1 else 1
    z = sample_nonzero(rng)
    poly = [z] + [random_scalar(rng) for _ in range(t)]
    poly += [0] * (domain_size - len(poly))
    shares = (O.fr_ntt(poly) if domain_size > 1 else poly)[:W]
    eval_domain = root_domain_prefix(domain_size, W)
    offsets = [0]
    for w in weights:
        offsets.append(offsets[-1] + w)
    owners = [j for j, w in enumerate(weights) for _ in range(w)]
    alpha, shift = shifted_alpha_points(B)
    while True:
        bm1, b0 = random_scalar(rng), random_scalar(rng)
        if b0 != 0 and (bm1 + b0) % R != 0:
            break
    occupied, rhos = set(), []
    for _ in range(N):
        while True:
            rho = random_scalar(rng)
            labels = [(rho + a) % R for a in alpha]
            if any(x == 0 for x in labels) or any(x in occupied for x in labels):
                continue
            occupied.update(labels)
            rhos.append(rho)
            break
    g = [[inv(rho + a) for a in alpha] for rho in rhos]  # g[j][i]
    u = [[(g[j][i] * g[j][i] + bm1 * inv(alpha[i] + 1) + b0 * inv(alpha[i])) % R for i in range(B)]
         for j in range(N)]
    vk = O.g2_mul_generator_blob(b"".join(O.s2b(g[j][i]) for i in range(B) for j in range(N)), B * N)
    d1 = O.g2_mul_generator_blob(b"".join(O.s2b(shares[w] * g[owners[w]][i]) for i in range(B) for w in range(W)),
                                 B * W)
    d2 = O.g2_mul_generator_blob(b"".join(O.s2b(shares[w] * u[owners[w]][i]) for i in range(B) for w in range(W)),
                                 B * W)
    V = O.g2_mul(O.g2_generator(), z * (bm1 + b0) % R)
    ek = O.fp12_pow(gt_generator(), z * b0 % R)
    h = hashlib.sha256()
    h.update(SETUP_ID_DOMAIN)
    for v in (B, t, domain_size, shift, N):
        h.update(struct.pack("<Q", v))
    for w in weights:
        h.update(struct.pack("<Q", w))
    for p in eval_domain + alpha:
        h.update(O.s2b(p))
    target = append_gt_fixed(ek)
    h.update(struct.pack("<Q", len(target)))
    h.update(target)
    for blob in (vk, d1, d2):
        for i in range(len(blob) // 192):
            h.update(O.g2_compress(blob[192 * i : 192 * (i + 1)]))
    h.update(O.g2_compress(V))
    return dict(B=B, t=t, N=N, W=W, weights=list(weights), domain_size=domain_size, offsets=offsets, owners=owners,
                shares=shares, eval_domain=eval_domain, alpha=alpha, shift=shift, bm1=bm1, b0=b0, z=z, rhos=rhos,
                g=g, u=u, vk=vk, d1=d1, d2=d2, V=V, ek=ek, setup_id=h.digest())


def _pt(blob: bytes, i: int) -> bytes:
    return blob[192 * i : 192 * (i + 1)]


def _challenge(setup_id, first, second, commitment) -> int:
    target = append_gt_fixed(second)
    prefix = (TRANSCRIPT_DOMAIN + setup_id + O.g1_compress(O.g1_generator()) + O.g1_compress(first)
              + struct.pack("<Q", len(target)) + target + O.g1_compress(commitment))
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
        r = sample_nonzero(rng)
        first = O.g1_mul(g1, r)
        second = O.fp12_mul(m, O.fp12_pow(key["ek"], r))
        k = random_scalar(rng)
        comm = O.g1_mul(g1, k)
        c = _challenge(key["setup_id"], first, second, comm)
        out.append(dict(first=first, second=second, commitment=comm, response=(k + c * r) % R))
    return out


def batch_digest(cts) -> bytes:
    body = struct.pack("<Q", len(cts))
    for ct in cts:
        body += (O.g1_compress(ct["first"]) + append_gt_fixed(ct["second"]) + O.g1_compress(ct["commitment"])
                 + ct["response"].to_bytes(32, "little"))
    return hashlib.sha256(BATCH_DIGEST_DOMAIN + body).digest()


def verify_batch(setup_id, cts, coefficients) -> bool:
    """Random-linear aggregate of the Schnorr equations (proof.rs:74-122)."""
    cs = [_challenge(setup_id, ct["first"], ct["second"], ct["commitment"]) for ct in cts]
    gen_s = sum(a * ct["response"] for a, ct in zip(coefficients, cts)) % R
    bases = [O.g1_generator()] + [ct["commitment"] for ct in cts] + [ct["first"] for ct in cts]
    scal = [gen_s] + [(-a) % R for a in coefficients] + [(-a * c) % R for a, c in zip(coefficients, cs)]
    return O.g1_msm(bases, scal) == O.G1_IDENTITY


def validate(key: dict, cts) -> dict:
    if len(cts) != key["B"]:
        raise ValueError("mismatched batch size")
    ok = verify_batch(key["setup_id"], cts, [i + 1 for i in range(len(cts))])
    if not ok:
        raise ValueError("invalid proof")
    return dict(first=[ct["first"] for ct in cts], digest=batch_digest(cts), B=len(cts))


def partial_decrypt(key: dict, j: int, batch: dict) -> bytes:
    return O.g1_msm(batch["first"], key["g"][j])


def verify_share(key: dict, batch: dict, j: int, sigma: bytes) -> bool:
    N = key["N"]
    left = list(batch["first"]) + [O.g1_neg(sigma)]
    right = [_pt(key["vk"], i * N + j) for i in range(key["B"])] + [O.g2_generator()]
    return O.fp12_is_one(O.final_exp(O.multi_miller_many([(left, right)])[0]))


def select_committee(key: dict, valid_parties) -> list:
    """Minimum-cardinality heaviest-first authorized subset (decryption.rs:339-356)."""
    w = key["weights"]
    order = sorted(valid_parties, key=lambda j: (-w[j], j))
    sel, acc = [], 0
    for j in order:
        if acc > key["t"]:
            break
        acc += w[j]
        sel.append(j)
    return sorted(sel)


def committee_context_id(setup_id: bytes, parties) -> bytes:
    h = hashlib.sha256()
    h.update(COMMITTEE_CONTEXT_DOMAIN)
    h.update(setup_id)
    h.update(struct.pack("<Q", len(parties)))
    for j in parties:
        h.update(struct.pack("<Q", j))
    return h.digest()


def prepare(key: dict, parties) -> dict:
    B, W = key["B"], key["W"]
    selected, coef_off = [], [0]
    for j in parties:
        selected.extend(range(key["offsets"][j], key["offsets"][j + 1]))
        coef_off.append(len(selected))
    lam = O.lagrange_at_zero([key["eval_domain"][w] for w in selected])
    lam_s = [x * inv(2 * B) % R for x in lam]
    T = len(parties)
    by_party = []
    for slot in range(B):
        for k, j in enumerate(parties):
            lo, hi = key["offsets"][j], key["offsets"][j + 1]
            by_party.append(O.g2_msm([_pt(key["d1"], slot * W + w) for w in range(lo, hi)],
                                     lam_s[coef_off[k] : coef_off[k + 1]]))
    total = []
    for slot in range(B):
        acc = O.G2_IDENTITY
        for p in by_party[slot * T : (slot + 1) * T]:
            acc = O.g2_add(acc, p)
        total.append(acc)
    mask = []
    for slot in range(B):
        d2 = O.g2_msm([_pt(key["d2"], slot * W + w) for w in selected], lam)
        a = key["alpha"][slot]
        mask.append(O.g2_add(O.g2_mul(d2, a * (a + 1) % R), O.g2_neg(O.g2_mul(key["V"], a))))
    return dict(parties=list(parties), selected=selected, lam=lam, by_party=by_party, total=total, mask=mask,
                context_id=committee_context_id(key["setup_id"], parties))


def _coeffs(B: int) -> list:
    return [B - 1 - 2 * k for k in range(B)]


def cauchy_group(values) -> list:
    """2B sum_{k != i} v_k / (alpha_k - alpha_i) through the spectrum (decryption.rs:683-708)."""
    B = len(values)
    spec = O.g1_ntt(list(values)) if B > 1 else list(values)
    spec = [O.g1_mul(v, c % R) for v, c in zip(spec, _coeffs(B))]
    rem = [O.g1_neg(spec[(i + B - 1) % B]) for i in range(B)]
    return O.g1_ntt(rem, inverse=True) if B > 1 else rem


def _small_pow(x: bytes, c: int) -> bytes:
    if c == 0:
        return O.fp12_one()
    r = O.fp12_pow(x, abs(c))
    return O.fp12_conj(r) if c < 0 else r


def cauchy_cyclotomic(values) -> list:
    """decryption.rs:710-734; agrees with the reference after the hard part."""
    B = len(values)
    spec = O.gt_ntt(list(values)) if B > 1 else list(values)
    spec = [_small_pow(v, c) for v, c in zip(spec, _coeffs(B))]
    rem = [O.fp12_conj(spec[(i + B - 1) % B]) for i in range(B)]
    return O.gt_ntt(rem, inverse=True) if B > 1 else rem


def precompute(key: dict, pre: dict, batch: dict) -> dict:
    first_c = cauchy_group(batch["first"])
    miller = O.miller_loop_many(batch["first"], pre["total"])
    pairing_c = cauchy_cyclotomic(O.batch_easy_final_exp(miller))
    return dict(first_cauchy=first_c, pairing_cauchy=pairing_c)


def open_batch(key: dict, pre: dict, sigmas, batch: dict, cts, bp: dict) -> list:
    B, T = key["B"], len(sigmas)
    scaled = [O.g1_mul(s, 2 * B) for s in sigmas]
    groups = []
    for slot in range(B):
        left = [O.g1_add(scaled[k], O.g1_neg(bp["first_cauchy"][slot])) for k in range(T)]
        groups.append((left, pre["by_party"][slot * T : (slot + 1) * T]))
    first_terms = O.batch_easy_final_exp(O.multi_miller_many(groups))
    mask_pairs = O.batch_easy_final_exp(O.miller_loop_many(batch["first"], pre["mask"]))
    out = []
    for slot in range(B):
        a = key["alpha"][slot]
        cf = O.fp12_mul(first_terms[slot], bp["pairing_cauchy"][slot])
        sub = O.fp12_pow(cf, a * (a + 1) % R)
        mask = O.hard_final_exp(O.fp12_mul(mask_pairs[slot], O.fp12_conj(sub)))
        out.append(O.fp12_mul(cts[slot]["second"], O.fp12_inv(mask)))
    return out


def literal_cauchy(key: dict, g1_values, gt_values):
    """The quadratic sums of decryption.rs:1018-1036, times 2B."""
    B = len(g1_values)
    al = key["alpha"]
    g1_out, gt_out = [], []
    for o in range(B):
        eg, et = O.G1_IDENTITY, O.fp12_one()
        for i in range(B):
            if i == o:
                continue
            c = inv(al[i] - al[o])
            eg = O.g1_add(eg, O.g1_mul(g1_values[i], c))
            et = O.fp12_mul(et, O.fp12_pow(gt_values[i], c))
        g1_out.append(O.g1_mul(eg, 2 * B))
        gt_out.append(O.fp12_pow(et, 2 * B))
    return g1_out, gt_out


def literal_open(key: dict, pre: dict, sigmas, batch: dict, cts) -> list:
    """Construction 5's displayed formula (decryption.rs:1042-1124)."""
    B, W = key["B"], key["W"]
    al = key["alpha"]
    coef = dict(zip(pre["selected"], pre["lam"]))
    out = []
    for o in range(B):
        a = al[o]
        excl = O.G1_IDENTITY
        for i in range(B):
            if i != o:
                excl = O.g1_add(excl, O.g1_mul(batch["first"][i], inv(al[i] - a)))
        l_sum = O.fp12_one()
        for j, sigma in zip(pre["parties"], sigmas):
            lo, hi = key["offsets"][j], key["offsets"][j + 1]

            def party_d1(slot):
                return O.g2_msm([_pt(key["d1"], slot * W + w) for w in range(lo, hi)],
                                [coef[w] for w in range(lo, hi)])

            l_sum = O.fp12_mul(l_sum, O.pairing(O.g1_add(sigma, O.g1_neg(excl)), party_d1(o)))
            for i in range(B):
                if i != o:
                    l_sum = O.fp12_mul(l_sum, O.fp12_pow(O.pairing(batch["first"][i], party_d1(i)), inv(al[i] - a)))
        d2 = O.g2_msm([_pt(key["d2"], o * W + w) for w in pre["selected"]], [coef[w] for w in pre["selected"]])
        d2_pair = O.pairing(batch["first"][o], d2)
        glob = O.pairing(batch["first"][o], key["V"])
        mask = O.fp12_mul(O.fp12_pow(O.fp12_mul(d2_pair, O.fp12_inv(l_sum)), a * (a + 1) % R),
                          O.fp12_inv(O.fp12_pow(glob, a)))
        out.append(O.fp12_mul(cts[o]["second"], O.fp12_inv(mask)))
    return out
