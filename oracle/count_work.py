"""Counts the algorithmic work of the reference's algorithms with the oracle's
counting build (test infrastructure: its output is a table of constants).

Runs, single-threaded, the oracle's restatement of each operation at the
weighted_btx benchmark's sizes and records the number of Fp Montgomery
products (products and squares, each counted once) it performs:

* the G2 MSMs of the committee preparation (Pippenger, one MSM per party
  block size of the heaviest-first committee, and one of the committee
  weight), weighted_btx/src/decryption.rs:463-506;
* the truncated cyclotomic inverse transform of the cross-term
  precomputation (m = 1024 values, first 512 outputs), btx/src/fft.rs:284-350;
* one hard final exponentiation, btx/src/final_exponentiation.rs:255-283.

    python -m oracle.count_work      # writes weighted_bte_b200/algorithmic_work.json

Counts of one MSM depend on its random scalars only through zero digits and
empty buckets, so one MSM per size stands for all MSMs of that size.
"""
from __future__ import annotations

import ctypes
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
COUNT_LIB = os.path.join(HERE, "_build", "liboracle_count.so")
OUT = os.path.join(ROOT, "weighted_bte_b200", "algorithmic_work.json")


def main():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from weighted_bte_b200.workloads import WBTX_B512, minimal_authorized_parties

    O.build()
    count = ctypes.CDLL(COUNT_LIB)
    count.orc_init()
    count.orc_fp_product_count.restype = ctypes.c_ulonglong
    plain = O.lib()
    rng = random.Random(11)

    def measure(fn):
        O._lib = count
        try:
            count.orc_fp_product_count_reset()
            fn()
            return int(count.orc_fp_product_count())
        finally:
            O._lib = plain

    cfg = WBTX_B512
    committee, _ = minimal_authorized_parties(cfg.weights, cfg.threshold)
    sizes = sorted({cfg.weights[j] for j in committee} | {sum(cfg.weights[j] for j in committee)})
    gen2 = O.g2_generator()
    msm = {}
    for n in sizes:
        pts = O.g2_mul_many(gen2, [rng.randrange(1, O.R) for _ in range(n)])
        sc = [rng.randrange(O.R) for _ in range(n)]
        msm[str(n)] = measure(lambda: O.g2_msm(pts, sc))

    m, out = 1024, 512
    g1s = O.g1_mul_many(O.g1_generator(), [rng.randrange(1, O.R) for _ in range(m)])
    easy = O.batch_easy_final_exp(O.miller_loop_many(g1s, [gen2] * m))
    prefix = measure(lambda: O.cyclotomic_prefix_ifft(easy, out))
    hard = measure(lambda: O.hard_final_exp(easy[0]))

    table = {
        "unit": "Fp Montgomery products (product or square) in the oracle's restatement",
        "workload": cfg.name,
        "committee": committee,
        "g2_msm_by_size": msm,
        "cyclotomic_prefix_ifft": {"m": m, "outputs": out, "fp_products": prefix},
        "hard_final_exp": {"fp_products": hard},
    }
    with open(OUT, "w") as f:
        json.dump(table, f, indent=1)
        f.write("\n")
    print(json.dumps(table))


if __name__ == "__main__":
    main()
