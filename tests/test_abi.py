"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every entry point include/wbte.h declares; the Python binding covers
them all; host-side workload logic."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wbte.h")
LIB = os.path.join(ROOT, "weighted_bte_b200", "libwbte.so")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|uint64_t|const char \*)\s*(wbte_\w+)\(", src, re.M)))


def test_header_declares_the_boundary():
    names = declared()
    for required in ("wbte_g1_msm", "wbte_g2_msm_family", "wbte_miller_loop_lines", "wbte_final_exp",
                     "wbte_wbtx_prepare", "wbte_wbtx_precompute", "wbte_wbtx_open", "wbte_wbtx_partial_decrypt"):
        assert required in names


@pytest.mark.skipif(not os.path.exists(LIB), reason="libwbte.so not built")
def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (wbte_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="libwbte.so not built")
def test_binding_loads_without_gpu_and_covers_the_header():
    from weighted_bte_b200 import _lib

    lib = _lib.load()
    assert lib.wbte_version() > 0
    assert sorted(_lib.EXPORTED) == declared()


def test_missing_library_fails_loudly(monkeypatch):
    from weighted_bte_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libwbte.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.LibraryMissing):
        _lib.load()


def test_zipf_weights_and_committee():
    from weighted_bte_b200.workloads import WBTX_B512, minimal_authorized_parties, zipf_weights

    w = WBTX_B512.weights
    assert len(w) == 128 and sum(w) == 4096 and min(w) >= 1
    assert w == sorted(w, reverse=True)
    committee, weight = minimal_authorized_parties(w, WBTX_B512.threshold)
    assert weight > 4096 // 3 and committee == [0, 1, 2]
    assert sum(zipf_weights(10, 100)) == 100


def test_seeded_scalars_are_reproducible():
    from weighted_bte_b200.rng import R, ChaCha20Rng, random_scalar

    a = [random_scalar(ChaCha20Rng.seed_from_u64(3)) for _ in range(2)]
    assert a[0] == a[1] and 0 <= a[0] < R


def test_error_variants_mirror_the_reference():
    from weighted_bte_b200 import errors as E

    e = E.InsufficientWeight(3, 6, [2])
    assert "accepted 3, require 6" in str(e) and "rejected parties [2]" in str(e)
    assert issubclass(E.MismatchedCommittee, E.Error)
