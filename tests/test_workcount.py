"""The roofline numerators (weighted_bte_b200/workcount.py): the per-operation
Fp-product counts of the tower and curve formulas the kernels use, and the
composite counts built from them."""
from weighted_bte_b200 import workcount as wc


def test_tower_counts():
    assert (wc.FP2_MUL, wc.FP2_SQR) == (3, 2)
    assert wc.FP6_MUL == 18 and wc.FP12_MUL == 54 and wc.FP12_SQR == 36
    assert wc.CYC_SQR == 18 and wc.FROB == 15
    assert (wc.LINE_MUL, wc.LINE_DOUBLE, wc.LINE_ADD) == (43, 22, 37)


def test_miller_loop_counts():
    # 62 squarings and 68 lines (63 doublings, 5 additions: the set bits of |x|)
    assert bin(wc.X_ABS).count("1") == 6 and wc.X_ABS.bit_length() == 64
    assert wc.MILLER_WITH_LINES == 62 * 36 + 68 * 43 == 5156
    assert wc.MILLER_UNPREPARED == 5156 + 63 * 22 + 5 * 37 == 6727
    assert wc.multi_miller_with_lines(1) == wc.MILLER_WITH_LINES


def test_chunked_share_check_counts():
    per_pair = wc.MILLER_UNPREPARED - wc.MILLER_SQUARING_RUN
    assert wc.multi_miller_unprepared(513, 1) == 513 * wc.MILLER_UNPREPARED
    assert wc.multi_miller_unprepared(513, 3) == 171 * wc.MILLER_SQUARING_RUN + 513 * per_pair
    # a ragged last run still pays one run of squarings
    assert wc.multi_miller_unprepared(10, 4) == 3 * wc.MILLER_SQUARING_RUN + 10 * per_pair


def test_final_exponentiation_counts():
    assert wc.FINAL_EXP_HARD == 7497
    assert wc.FINAL_EXP == wc.FINAL_EXP_EASY + wc.FINAL_EXP_HARD
    assert wc.FP_INV > 381  # a Fermat chain over the 381-bit p - 2


def test_msm_counts_grow_with_size():
    g1 = [wc.msm_expected(1 << lg, 1, False) for lg in range(10, 21, 2)]
    g2 = [wc.msm_expected(1 << lg, 1, True) for lg in range(10, 21, 2)]
    assert g1 == sorted(g1) and g2 == sorted(g2)
    assert all(b > a for a, b in zip(g1, g2))  # G2 additions cost more products
    # a family of k equal MSMs counts k times one (up to the rounding of each)
    assert abs(wc.msm_expected(512, 384, False) - 384 * wc.msm_expected(512, 1, False)) < 384
