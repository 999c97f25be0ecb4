"""Parity at the benchmark configurations' full sizes, through identities that
do not need the CPU oracle to run at those sizes.

* MSMs and group transforms over points G * u_i: the result must be the
  generator times the same combination of the u_i in Fr, computed here with
  Python integers (the kernel sweep configuration: MSMs up to 2^20 points,
  transforms up to 2^16).
* GT transforms over true GT elements gt^u_i: there the decomposed
  exponentiation is the ordinary power (Frobenius acts as p = x mod r), so
  the outputs are gt^(transformed u) exactly; the batched form at the
  weighted_btx shape (64 transforms of 1024) runs the warp-uniform plan.
* Multi-pairings of k pairs (a_i G1, b_i G2): e(G1, G2)^(sum a_i b_i).
* Round trips of the protocols at the configurations' shapes: weighted_btx
  B = 512 with Zipf weights W = 4096; weighted_pfe with n = 64, W = 2048 at
  batch sizes up to 512; weighted_pfe with n = 1000 Pareto(1.2) weights,
  W = 16384.
"""
import random

import pytest

from weighted_bte_b200 import ops
from weighted_bte_b200 import weighted_btx as wb

pytestmark = pytest.mark.gpu
R = ops.R


def _scalars(rng, n):
    return [rng.randrange(R) for _ in range(n)]


def _host_ntt(vals, inverse=False):
    """Unscaled transform over the size-n subgroup of Fr (natural order),
    y_k = sum_i x_i w^(+-ik): the checker's plain recursive form."""
    n = len(vals)
    w = wb.radix2_generator(n)
    if inverse:
        w = pow(w, R - 2, R)

    def rec(xs, w):
        m = len(xs)
        if m == 1:
            return list(xs)
        ev, od = rec(xs[0::2], w * w % R), rec(xs[1::2], w * w % R)
        out, t = [0] * m, 1
        for k in range(m // 2):
            x = od[k] * t % R
            out[k], out[k + m // 2] = (ev[k] + x) % R, (ev[k] - x) % R
            t = t * w % R
        return out

    return rec(vals, w)


@pytest.mark.parametrize("group", [1, 2])
@pytest.mark.parametrize("logn", [10, 14, 17, 20])
def test_msm_equals_generator_times_combination(group, logn):
    rng = random.Random(2000 + 10 * logn + group)
    n = 1 << logn
    u, c = _scalars(rng, n), _scalars(rng, n)
    c[0], c[1] = 0, 1
    gen, msm = (ops.g1_mul_generator, ops.g1_msm) if group == 1 else (ops.g2_mul_generator, ops.g2_msm)
    points = gen(u)
    expect = gen([sum(a * b for a, b in zip(u, c)) % R])
    assert msm(points, c) == expect


@pytest.mark.parametrize("group", [1, 2])
@pytest.mark.parametrize("logn", [8, 12, 16])
def test_group_ntt_equals_generator_times_transform(group, logn):
    rng = random.Random(3000 + 10 * logn + group)
    n = 1 << logn
    u = _scalars(rng, n)
    gen, ntt = (ops.g1_mul_generator, ops.g1_ntt) if group == 1 else (ops.g2_mul_generator, ops.g2_ntt)
    points = gen(u)
    for inv in (False, True):
        assert ntt(points, inverse=inv) == gen(_host_ntt(u, inv)), inv


@pytest.mark.parametrize("logn", [8, 12])
def test_gt_ntt_on_gt_elements_is_exact(logn):
    rng = random.Random(4000 + logn)
    n = 1 << logn
    u = _scalars(rng, n)
    g = wb.gt_generator()
    vals = ops.gt_pow(g, u, fixed_base=True)
    for inv in (False, True):
        assert ops.gt_ntt(vals, inverse=inv) == ops.gt_pow(g, _host_ntt(u, inv), fixed_base=True), inv


def test_batched_gt_transforms_at_the_benchmark_shape():
    """64 transforms of m = 1024 in one launch per stage (the precomputation's
    shape for a group of 64 batches of 512), forward and truncated inverse."""
    rng = random.Random(4100)
    m, count = 1024, 64
    u = _scalars(rng, m * count)
    g = wb.gt_generator()
    vals = ops.gt_pow(g, u, fixed_base=True)
    fwd = ops.gt_ntt_many(vals, m)
    expect = [x for q in range(count) for x in _host_ntt(u[m * q : m * (q + 1)])]
    assert fwd == ops.gt_pow(g, expect, fixed_base=True)
    pre = ops.cyclotomic_prefix_ifft_many(vals, m, m // 2)
    inv = [x for q in range(count) for x in _host_ntt(u[m * q : m * (q + 1)], True)[: m // 2]]
    assert b"".join(pre) == ops.gt_pow(g, inv, fixed_base=True)


@pytest.mark.parametrize("k", [1, 16, 256, 4096])
def test_multi_pairing_equals_gt_power(k):
    rng = random.Random(5000 + k)
    a, b = _scalars(rng, k), _scalars(rng, k)
    P, Q = ops.g1_mul_generator(a), ops.g2_mul_generator(b)
    got = ops.final_exp(ops.multi_miller_loop(P, Q, [0, k]))
    assert got == ops.gt_pow(wb.gt_generator(), [sum(x * y for x, y in zip(a, b)) % R], fixed_base=True)


def test_weighted_btx_round_trip_at_the_benchmark_configuration():
    from weighted_bte_b200 import serving
    from weighted_bte_b200.rng import ChaCha20Rng
    from weighted_bte_b200.workloads import WBTX_B512, minimal_authorized_parties

    cfg = WBTX_B512
    rng = ChaCha20Rng.seed_from_u64(cfg.seed)
    mat = wb.keygen_with_rng(wb.KeygenConfig(cfg.batch_size, cfg.weights, cfg.threshold), rng)
    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    keys = [mat.party_keys[j] for j in committee]
    msgs = [wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(cfg.batch_size)]) for _ in range(2)]
    cts = [wb.encrypt_many(mat.encryption_key, mm, rng) for mm in msgs]
    batch = wb.validate_batch(mat.decryption_key, cts[0])
    shares = wb.partial_decrypt_many(keys, batch)
    assert wb.decrypt(mat.decryption_key, cts[0], shares) == msgs[0]
    grouped = serving.decrypt_group(mat.decryption_key, [wb.CiphertextBatch.upload(c) for c in cts], keys,
                                    ChaCha20Rng.seed_from_u64(7), serving.CommitteeCache(1 << 31))
    assert grouped == msgs


def _wpfe_round_trip(weights, B, seed):
    from weighted_bte_b200 import weighted_pfe as wp
    from weighted_bte_b200.rng import ChaCha20Rng
    from weighted_bte_b200.workloads import minimal_authorized_parties

    W = sum(weights)
    t = W // 3
    rng = ChaCha20Rng.seed_from_u64(seed)
    mat = wp.keygen_with_rng(wp.KeygenConfig(B, weights, t), rng)
    msgs = wb.messages_from_bytes([rng.fill_bytes(32) for _ in range(B)])
    cts = wp.encrypt_many(mat.encryption_key, msgs, rng)
    batch = wp.validate_batch(mat.encryption_key, cts)
    committee, _ = minimal_authorized_parties(weights, t)
    shares = wp.partial_decrypt_many([mat.party_keys[j] for j in committee], batch)
    assert wp.decrypt(mat.encryption_key, mat.decryption_key, cts, shares) == msgs


@pytest.mark.parametrize("B", [8, 64, 512])
def test_weighted_pfe_round_trips_at_the_batched_configuration(B):
    """n = 64 parties, Zipf(1) weights W = 2048, threshold W/3; batch sizes of
    the log-uniform range [8, 2048] padded to powers of two."""
    from weighted_bte_b200.workloads import zipf_weights

    _wpfe_round_trip(zipf_weights(64, 2048), B, seed=300 + B)


def test_weighted_pfe_round_trip_with_the_served_configuration_parties():
    """n = 1000 parties with Pareto(1.2) weights scaled to W = 16384."""
    from weighted_bte_b200.workloads import pareto_weights

    _wpfe_round_trip(pareto_weights(1000, 16384), 16, seed=4)
