"""Synthetic workloads for the decryption benchmarks.

No public dataset is involved: party weights, secrets and plaintexts are
seeded synthetic inputs with the shapes of the benchmark configurations.

* weighted_btx, B = 512: n = 128 parties with Zipf(s = 1) weights w_k ~ 1/k
  scaled to W = 4096 (largest-remainder rounding, every weight >= 1);
  a set is authorized when its weight exceeds t = floor(W / 3); the
  committee is the heaviest-first minimal authorized set
  (weighted_btx/examples/paper_reproduction.rs:581-607); ChaCha20 seed 1.
* weighted_pfe served form: n = 1000 parties with Pareto(1.2) weights
  scaled to W = 16384; batched form: n = 64 parties with Zipf(1) weights
  scaled to W = 2048; threshold floor(W / 3).
* Plaintexts are uniform 32-byte strings mapped to GT as
  Gt::generator()^(LE(bytes) mod r); the crates encrypt GT elements only.
"""
from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction
from typing import List, Tuple


def zipf_weights(n: int, total: int, s: float = 1.0) -> List[int]:
    """Integer weights proportional to 1/k^s summing to `total`, each >= 1."""
    if total < n:
        raise ValueError("total weight must be at least the party count")
    raw = [Fraction(1, 1) / Fraction(k) ** Fraction(s).limit_denominator(1000) if s != 1.0 else Fraction(1, k)
           for k in range(1, n + 1)]
    norm = sum(raw)
    quotas = [r * total / norm for r in raw]
    base = [max(1, int(q)) for q in quotas]
    rest = total - sum(base)
    order = sorted(range(n), key=lambda i: (-(quotas[i] - int(quotas[i])), i))
    i = 0
    while rest > 0:
        base[order[i % n]] += 1
        rest -= 1
        i += 1
    while rest < 0:
        j = max(range(n), key=lambda k: (base[k], -k))
        base[j] -= 1
        rest += 1
    return base


def scale_weights(raw: List[float], total: int) -> List[int]:
    """Largest-remainder integer weights proportional to `raw`, each >= 1,
    summing to `total`."""
    n = len(raw)
    if total < n:
        raise ValueError("total weight must be at least the party count")
    norm = sum(raw)
    quotas = [r * total / norm for r in raw]
    base = [max(1, int(q)) for q in quotas]
    rest = total - sum(base)
    order = sorted(range(n), key=lambda i: (-(quotas[i] - int(quotas[i])), i))
    i = 0
    while rest > 0:
        base[order[i % n]] += 1
        rest -= 1
        i += 1
    while rest < 0:
        j = max(range(n), key=lambda k: (base[k], -k))
        base[j] -= 1
        rest += 1
    return base


def pareto_weights(n: int, total: int, alpha: float = 1.2, seed: int = 4) -> List[int]:
    """Heavy-tailed integer weights: n seeded Pareto(alpha) draws
    (1 - U)^(-1/alpha), scaled to `total` (each >= 1)."""
    import random

    rng = random.Random(seed)
    return scale_weights([(1.0 - rng.random()) ** (-1.0 / alpha) for _ in range(n)], total)


def minimal_authorized_parties(weights: List[int], threshold: int) -> Tuple[List[int], int]:
    """Heaviest-first minimal committee with weight > threshold."""
    ranked = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    chosen, acc = [], 0
    for i in ranked:
        acc += weights[i]
        chosen.append(i)
        if acc > threshold:
            return chosen, acc
    raise ValueError("total weight does not exceed the threshold")


@dataclass
class WeightedBtxConfig:
    name: str
    batch_size: int
    parties: int
    total_weight: int
    seed: int

    @property
    def weights(self) -> List[int]:
        return zipf_weights(self.parties, self.total_weight)

    @property
    def threshold(self) -> int:
        return self.total_weight // 3


WBTX_B512 = WeightedBtxConfig("weighted_btx B=512 n=128 Zipf(1) W=4096 t=W/3", 512, 128, 4096, 1)


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> List[int]:
    """`count` batch sizes round(exp(U[ln lo, ln hi])) from a seeded stream."""
    import math
    import random

    rng = random.Random(seed)
    a, b = math.log(lo), math.log(hi)
    return [min(hi, max(lo, int(round(math.exp(rng.uniform(a, b)))))) for _ in range(count)]


@dataclass
class WeightedPfeBatchedConfig:
    """The batched form: `count` independent weighted_pfe batches with sizes
    log-uniform in [lo, hi], padded to powers of two with valid dummy
    encryptions; n parties with Zipf(1) weights scaled to W; threshold W/3."""

    name: str
    count: int
    lo: int
    hi: int
    parties: int
    total_weight: int
    seed: int

    @property
    def weights(self) -> List[int]:
        return zipf_weights(self.parties, self.total_weight)

    @property
    def threshold(self) -> int:
        return self.total_weight // 3

    def sizes(self) -> List[int]:
        return log_uniform_sizes(self.count, self.lo, self.hi, self.seed)


@dataclass
class WeightedPfeServedConfig:
    """The served form: requests of weighted_pfe batch decryption with sizes
    log-uniform in [lo, hi] (padded to powers of two), n parties with
    Pareto(alpha) weights scaled to W, threshold W/3, Poisson arrivals."""

    name: str
    lo: int
    hi: int
    parties: int
    total_weight: int
    alpha: float
    seed: int

    @property
    def weights(self) -> List[int]:
        return pareto_weights(self.parties, self.total_weight, self.alpha, self.seed)

    @property
    def threshold(self) -> int:
        return self.total_weight // 3


WPFE_BATCHED = WeightedPfeBatchedConfig(
    "weighted_pfe batched: 256 batches, sizes log-uniform [8, 2048] padded to pow2, n=64 Zipf(1) W=2048 t=W/3",
    256, 8, 2048, 64, 2048, 3)
WPFE_SERVED = WeightedPfeServedConfig(
    "weighted_pfe served: sizes log-uniform [16, 4096] padded to pow2, n=1000 Pareto(1.2) W=16384 t=W/3, "
    "Poisson arrivals", 16, 4096, 1000, 16384, 1.2, 4)
