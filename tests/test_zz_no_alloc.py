"""The allocation-free G1 MSM, wbte_g1_msm_static.

It serves callers that must not allocate device memory while handling a
request (for example a service that reserved HBM up front for its resident
keys and buffers, where a new allocation could fail mid-request or stall on
device-wide synchronisation).  Its working memory is a fixed array in the
library's device image.  This file is collected last so that a run which
stops at the first failure has already run every other test; it passes alone
in a fresh process (where the first call does the one-time set-up) and after
the other tests.
"""
import random

import pytest

pytestmark = pytest.mark.gpu

WBTE_ERR_INVALID_ARG, WBTE_ERR_SIZE = -1, -2


def _dev(torch, data: bytes):
    return torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()


def test_static_msm_matches_the_allocating_entry_point_on_consecutive_calls():
    import torch

    from weighted_bte_b200 import _lib, ops

    torch.cuda.set_device(0)
    lib = _lib.load()
    rng = random.Random(4242)
    # calls in a row through the C ABI, each reusing the array that still
    # holds the previous call's intermediates: the documented maximum, sizes
    # that the allocating entry point sends to its small-MSM kernel (n <= 4),
    # and sizes in between
    for n in (16384, 3000, 517, 4, 1):
        points = ops.g1_mul_generator([rng.randrange(ops.R) for _ in range(n)])
        scalars = ops.scalars_bytes([rng.randrange(ops.R) for _ in range(n)])
        expect = ops.g1_msm(points, scalars)  # the existing, allocating entry point
        d_pts, d_sc = _dev(torch, points), _dev(torch, scalars)
        d_out = torch.zeros(96, dtype=torch.uint8, device="cuda")
        status = lib.wbte_g1_msm_static(d_out.data_ptr(), d_pts.data_ptr(), d_sc.data_ptr(), n, None)
        assert status == 0
        torch.cuda.synchronize()
        assert bytes(d_out.cpu().numpy()) == expect, f"n={n}"


def test_static_msm_rejects_oversize_and_host_buffers():
    import torch

    from weighted_bte_b200 import _lib

    torch.cuda.set_device(0)
    lib = _lib.load()
    d = torch.zeros(96 * 8, dtype=torch.uint8, device="cuda")
    assert lib.wbte_g1_msm_static(d.data_ptr(), d.data_ptr(), d.data_ptr(), 16385, None) == WBTE_ERR_SIZE
    host = bytearray(96)
    import ctypes

    hp = ctypes.addressof((ctypes.c_char * 96).from_buffer(host))
    assert lib.wbte_g1_msm_static(hp, d.data_ptr(), d.data_ptr(), 1, None) == WBTE_ERR_INVALID_ARG
