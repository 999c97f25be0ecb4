"""ctypes binding of libwbte (include/wbte.h).

The library is the product's only compute path: there is no CPU fallback.
If libwbte.so is missing, importing a compute entry point raises
`LibraryMissing` -- build it with `python -m weighted_bte_b200.build`.

Buffers: every data argument may be `bytes`/`bytearray`/`memoryview`, a
NumPy array, a torch tensor (host or CUDA), or a raw integer address.  The
library itself decides whether an address is device or host memory.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("WBTE_LIB") or os.path.join(PKG, "libwbte.so")

WBTE_OK = 0
STATUS_NAMES = {
    -1: "WBTE_ERR_INVALID_ARG",
    -2: "WBTE_ERR_SIZE",
    -3: "WBTE_ERR_OOM",
    -4: "WBTE_ERR_TIMEOUT",
    -5: "WBTE_ERR_CUDA",
    -6: "WBTE_ERR_NOT_ON_CURVE",
    -7: "WBTE_ERR_INTERPOLATION",
    -8: "WBTE_ERR_INTERNAL",
}
FE_FULL, FE_EASY, FE_HARD = 0, 1, 2
TUNE_GT_LANES, TUNE_MSM_WINDOW, TUNE_MSM_SEGMENTS, TUNE_NTT_JOINT, TUNE_MILLER_CHUNK = 1, 2, 3, 4, 5
CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy
G1_BYTES, G2_BYTES, GT_BYTES, FR_BYTES, LINE_BYTES, MILLER_LINES = 96, 192, 576, 32, 288, 68
FIXED_TABLE_BYTES = 192 * 11 * 32  # fixed-base table of one G2 point (wbte_wbtx_vk_tables)


class LibraryMissing(RuntimeError):
    pass


class WbteError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class WbtxKey(ctypes.Structure):
    _fields_ = [
        ("domain_points", ctypes.c_void_p),
        ("verification_keys", ctypes.c_void_p),
        ("negative_material", ctypes.c_void_p),
        ("positive_material", ctypes.c_void_p),
        ("party_offsets", ctypes.c_void_p),
        ("party_count", ctypes.c_uint64),
        ("total_weight", ctypes.c_uint64),
        ("max_batch_size", ctypes.c_uint64),
    ]


class TranscriptField(ctypes.Structure):
    """wbte_transcript_field: record i contributes `len` bytes at data + i * stride."""

    _fields_ = [
        ("data", ctypes.c_void_p),
        ("stride", ctypes.c_uint64),
        ("len", ctypes.c_uint32),
        ("kind", ctypes.c_uint32),
    ]


TRANSCRIPT_BYTES, TRANSCRIPT_GT_VARIABLE = 0, 1


class Request(ctypes.Structure):
    """wbte_request: one accepted batch submitted to a wbte_server."""

    _fields_ = [
        ("crs", ctypes.c_void_p),
        ("batch_size", ctypes.c_uint64),
        ("first", ctypes.c_void_p),
        ("second", ctypes.c_void_p),
        ("valid", ctypes.c_void_p),
        ("sigma", ctypes.c_void_p),
        ("party_indices", ctypes.c_void_p),
        ("party_count", ctypes.c_uint64),
        ("messages", ctypes.c_void_p),
    ]


SCHEME_WBTX, SCHEME_WPFE = 1, 2


class WpfeKey(ctypes.Structure):
    _fields_ = [
        ("domain_points", ctypes.c_void_p),
        ("verification_keys", ctypes.c_void_p),
        ("d1", ctypes.c_void_p),
        ("d2", ctypes.c_void_p),
        ("global_key", ctypes.c_void_p),
        ("party_offsets", ctypes.c_void_p),
        ("party_count", ctypes.c_uint64),
        ("total_weight", ctypes.c_uint64),
        ("batch_size", ctypes.c_uint64),
    ]


_VP, _U64, _I32, _I64 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_int64
# name -> argument types after the context pointer
_SIGNATURES = {
    "wbte_g1_msm": [_VP, _VP, _VP, _U64],
    "wbte_g2_msm": [_VP, _VP, _VP, _U64],
    "wbte_g1_msm_family": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _I32, _U64, _U64],
    "wbte_g2_msm_family": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _I32, _U64, _U64],
    "wbte_g1_mul": [_VP, _VP, _I32, _VP, _U64],
    "wbte_g2_mul": [_VP, _VP, _I32, _VP, _U64],
    "wbte_g1_mul_generator": [_VP, _VP, _U64],
    "wbte_g2_mul_generator": [_VP, _VP, _U64],
    "wbte_g1_sum": [_VP, _VP, _VP, _U64],
    "wbte_g2_sum": [_VP, _VP, _VP, _U64],
    "wbte_g1_batch_normalize": [_VP, _VP, _U64],
    "wbte_g2_batch_normalize": [_VP, _VP, _U64],
    "wbte_g1_compress": [_VP, _VP, _U64],
    "wbte_g2_compress": [_VP, _VP, _U64],
    "wbte_g1_ntt": [_VP, _U64, _I32],
    "wbte_g2_ntt": [_VP, _U64, _I32],
    "wbte_gt_ntt": [_VP, _U64, _I32],
    "wbte_gt_ntt_many": [_VP, _U64, _U64, _I32],
    "wbte_gt_cyclotomic_prefix_ifft_many": [_VP, _U64, _U64, _U64],
    "wbte_gt_cyclotomic_prefix_ifft": [_VP, _U64, _U64],
    "wbte_g2_prepare_lines": [_VP, _VP, _U64],
    "wbte_miller_loop_lines": [_VP, _VP, _VP, _U64],
    "wbte_miller_loop": [_VP, _VP, _VP, _U64],
    "wbte_multi_miller_loop": [_VP, _VP, _VP, _VP, _U64],
    "wbte_final_exp": [_VP, _VP, _U64, _I32],
    "wbte_gt_pow": [_VP, _VP, _I32, _VP, _U64],
    "wbte_fp12_mul": [_VP, _VP, _VP, _U64],
    "wbte_gt_compress": [_VP, _VP, _U64],
    "wbte_lagrange_at_zero": [_VP, _VP, _U64],
    "wbte_schnorr_verify": [_VP, _VP, _VP, _VP, _VP, _U64],
    "wbte_transcript_challenges": [_VP, _VP, ctypes.c_uint32, _U64],
    "wbte_g1_decompress": [_VP, _VP, _VP, _U64, _I32],
    "wbte_g2_decompress": [_VP, _VP, _VP, _U64, _I32],
    "wbte_wbtx_partial_decrypt": [_VP, _VP, _U64, _VP, _U64],
    "wbte_wbtx_verify_shares": [_VP, _VP, _VP, _VP, _U64, _VP, _VP, _VP, _U64],
    "wbte_wbtx_prepare": [_VP, _VP, _U64, _U64, _VP, _VP, _VP],
    "wbte_wbtx_precompute": [_VP, _VP, _VP, _VP, _U64],
    "wbte_wbtx_open": [_VP, _VP, _VP, _U64, _VP, _VP, _VP, _U64],
    "wbte_wbtx_keygen_material": [_VP, _VP, _VP, _VP, _U64, _U64, _U64, _VP, _VP, _VP],
    "wbte_measure_imad_rate": [_VP],
    "wbte_btx_kernel": [_VP, _VP, _U64, _U64, _VP, _VP, _VP],
    "wbte_btx_precompute": [_VP, _VP, _VP, _VP, _U64],
    "wbte_btx_partial_decrypt": [_VP, _VP, _VP, _U64],
    "wbte_btx_combine": [_VP, _VP, _VP, _U64],
    "wbte_btx_verify": [_VP, _VP, _VP, _U64, _VP, _U64, _VP],
    "wbte_btx_open": [_VP, _VP, _VP, _VP, _VP, _VP, _U64],
    "wbte_wpfe_fractions": [_VP, _VP, _VP, _VP, _VP, _U64, _U64, _I32],
    "wbte_wpfe_keygen_material": [_VP, _VP, _VP, _VP, _U64, _U64, _U64, _VP, _VP, _VP],
    "wbte_wpfe_partial_decrypt": [_VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_wpfe_verify_shares": [_VP, _VP, _VP, _VP, _VP, _VP, _U64],
    "wbte_wpfe_prepare": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _VP, _VP],
    "wbte_wpfe_precompute": [_VP, _VP, _VP, _VP, _U64],
    "wbte_wpfe_open": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64],
    "wbte_wbtx_partial_decrypt_many": [_VP, _VP, _U64, _VP, _U64, _U64],
    "wbte_wbtx_verify_shares_many": [_VP, _VP, _VP, _U64, _VP, _VP, _VP, _U64, _U64, _VP],
    "wbte_wbtx_vk_tables": [_VP, _VP, _VP, _U64, _U64],
    "wbte_wbtx_precompute_many": [_VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_wbtx_open_many": [_VP, _VP, _VP, _VP, _U64, _VP, _VP, _VP, _U64, _U64],
    "wbte_wbtx_decrypt_many": [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64, _U64],
    "wbte_wpfe_partial_decrypt_many": [_VP, _VP, _VP, _VP, _U64, _U64, _U64],
    "wbte_wpfe_vk_tables": [_VP, _VP, _VP, _U64],
    "wbte_wpfe_verify_shares_many": [_VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64, _VP],
    "wbte_wpfe_precompute_many": [_VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_wpfe_open_many": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_wpfe_decrypt_many": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_btx_precompute_many": [_VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_btx_open_many": [_VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_btx_decrypt_many": [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_pfe_precompute_many": [_VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_pfe_open_many": [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64, _U64],
    "wbte_pfe_kernel": [_VP, _VP, _U64, _VP, _VP, _VP, _VP, _VP, _VP, _VP],
    "wbte_pfe_precompute": [_VP, _VP, _VP, _VP, _VP, _U64],
    "wbte_pfe_open": [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _U64],
}
EXPORTED = sorted(
    list(_SIGNATURES)
    + ["wbte_version", "wbte_ctx_create", "wbte_ctx_destroy", "wbte_ctx_set_stream", "wbte_ctx_synchronize",
       "wbte_ctx_last_error", "wbte_ctx_launch_count", "wbte_thread_launch_count", "wbte_profile_enable",
       "wbte_profile_read",
       "wbte_g1_msm_static", "wbte_ctx_set_tuning", "wbte_crs_upload_wbtx", "wbte_crs_upload_wpfe",
       "wbte_crs_destroy", "wbte_server_create", "wbte_submit", "wbte_poll", "wbte_server_destroy"]
)


def profile_enable(on: bool = True) -> None:
    """Start (or stop) per-kernel CUDA-event timing; clears earlier records."""
    load().wbte_profile_enable(1 if on else 0)


def profile_read() -> dict:
    """{kernel name: (milliseconds summed over launches, launches)}."""
    lib = load()
    stride, cap = 64, 256
    names = ctypes.create_string_buffer(stride * cap)
    ms = (ctypes.c_double * cap)()
    cnt = (ctypes.c_int64 * cap)()
    n = _I32(0)
    st = lib.wbte_profile_read(names, stride, ms, cnt, cap, ctypes.byref(n))
    if st != WBTE_OK:
        raise WbteError(st, "profile read failed")
    out = {}
    for i in range(n.value):
        name = names.raw[i * stride : (i + 1) * stride].split(b"\0", 1)[0].decode()
        out[name] = (float(ms[i]), int(cnt[i]))
    return out

_lib = None
_lock = threading.Lock()


def load():
    """Load libwbte.so (raises LibraryMissing if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is missing: the CUDA library must be built "
                "(python -m weighted_bte_b200.build); there is no CPU fallback"
            )
        lib = ctypes.CDLL(LIB_PATH)
        lib.wbte_version.restype = _I32
        lib.wbte_ctx_create.argtypes = [_I32, _U64, ctypes.POINTER(_VP)]
        lib.wbte_ctx_create.restype = _I32
        lib.wbte_ctx_destroy.argtypes = [_VP]
        lib.wbte_ctx_destroy.restype = _I32
        lib.wbte_ctx_set_stream.argtypes = [_VP, _VP]
        lib.wbte_ctx_set_stream.restype = _I32
        lib.wbte_ctx_set_tuning.argtypes = [_VP, _I32, _I64]
        lib.wbte_ctx_set_tuning.restype = _I32
        lib.wbte_ctx_synchronize.argtypes = [_VP]
        lib.wbte_ctx_synchronize.restype = _I32
        lib.wbte_ctx_last_error.argtypes = [_VP]
        lib.wbte_ctx_last_error.restype = ctypes.c_char_p
        lib.wbte_ctx_launch_count.argtypes = [_VP]
        lib.wbte_ctx_launch_count.restype = _U64
        lib.wbte_thread_launch_count.argtypes = []
        lib.wbte_thread_launch_count.restype = _U64
        lib.wbte_profile_enable.argtypes = [_I32]
        lib.wbte_profile_enable.restype = _I32
        lib.wbte_profile_read.argtypes = [_VP, _I32, _VP, _VP, _I32, ctypes.POINTER(_I32)]
        lib.wbte_profile_read.restype = _I32
        for name, args in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = [_VP] + args
            fn.restype = _I32
        # resident keys and the served form
        lib.wbte_crs_upload_wbtx.argtypes = [_VP, _VP, ctypes.POINTER(_VP)]
        lib.wbte_crs_upload_wpfe.argtypes = [_VP, _VP, _VP, ctypes.POINTER(_VP)]
        lib.wbte_crs_destroy.argtypes = [_VP]
        lib.wbte_server_create.argtypes = [_I32, ctypes.c_uint32, ctypes.c_uint32, _U64, ctypes.POINTER(_VP)]
        lib.wbte_submit.argtypes = [_VP, _VP, ctypes.POINTER(_U64)]
        lib.wbte_poll.argtypes = [_VP, _U64, _U64, ctypes.POINTER(_I32)]
        lib.wbte_server_destroy.argtypes = [_VP]
        for name in ("wbte_crs_upload_wbtx", "wbte_crs_upload_wpfe", "wbte_crs_destroy", "wbte_server_create",
                     "wbte_submit", "wbte_poll", "wbte_server_destroy"):
            getattr(lib, name).restype = _I32
        # context-free, allocation-free G1 MSM: (out, points, scalars, n, stream)
        lib.wbte_g1_msm_static.argtypes = [_VP, _VP, _VP, _U64, _VP]
        lib.wbte_g1_msm_static.restype = _I32
        _lib = lib
        return lib


class _Keep:
    """Holds ctypes buffers alive for the duration of one call."""

    def __init__(self):
        self.items = []

    def ptr(self, x):
        if x is None:
            return None
        if isinstance(x, int):
            return x
        mod = type(x).__module__
        if mod.startswith("torch"):
            return x.data_ptr()
        if isinstance(x, np.ndarray):
            if not x.flags["C_CONTIGUOUS"]:
                raise ValueError("arrays must be C-contiguous")
            self.items.append(x)
            return x.ctypes.data
        if isinstance(x, bytes):
            buf = ctypes.create_string_buffer(x, len(x))
            self.items.append(buf)
            return ctypes.addressof(buf)
        if isinstance(x, (bytearray, memoryview)):
            mv = memoryview(x)
            if mv.readonly:
                buf = ctypes.create_string_buffer(mv.tobytes(), mv.nbytes)
                self.items.append(buf)
                return ctypes.addressof(buf)
            arr = (ctypes.c_char * mv.nbytes).from_buffer(mv)
            self.items.append(arr)
            return ctypes.addressof(arr)
        if isinstance(x, ctypes.Array):
            return ctypes.addressof(x)
        raise TypeError(f"unsupported buffer type {type(x)}")


def i64_array(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.int64))


def i32_array(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.int32))


class Context:
    """A libwbte context bound to one GPU."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = load()
        h = _VP()
        st = self.lib.wbte_ctx_create(int(device), int(hbm_budget_bytes), ctypes.byref(h))
        if st != WBTE_OK:
            raise WbteError(st, f"could not create a context on device {device}")
        self.handle = h.value
        self.device = device

    def close(self):
        if self.handle:
            self.lib.wbte_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        """Issue work on `stream_handle` (a cudaStream_t).  Handle 0 is the
        legacy default stream, passed on as cudaStreamLegacy; None selects the
        context's own stream."""
        if stream_handle is None:
            self.lib.wbte_ctx_set_stream(self.handle, None)
        else:
            self.lib.wbte_ctx_set_stream(self.handle, stream_handle if stream_handle else CUDA_STREAM_LEGACY)

    def synchronize(self):
        self._check(self.lib.wbte_ctx_synchronize(self.handle))

    def set_tuning(self, knob: int, value: int):
        """One knob of the launchers' cost models (TUNE_*) for later calls."""
        self._check(self.lib.wbte_ctx_set_tuning(self.handle, int(knob), int(value)))

    def launch_count(self) -> int:
        return int(self.lib.wbte_ctx_launch_count(self.handle))

    def _check(self, st: int):
        if st != WBTE_OK:
            msg = self.lib.wbte_ctx_last_error(self.handle)
            raise WbteError(st, msg.decode() if msg else "")

    def call(self, name: str, *args):
        keep = _Keep()
        conv = []
        for a in args:
            if isinstance(a, ctypes.Structure):
                conv.append(ctypes.addressof(a))
                keep.items.append(a)
            elif isinstance(a, (bool, np.integer)):
                conv.append(int(a))
            elif isinstance(a, int) and not isinstance(a, bool):
                conv.append(a)
            else:
                conv.append(keep.ptr(a))
        st = getattr(self.lib, name)(self.handle, *conv)
        self._check(st)
        return keep


_default = threading.local()


def default_context(device: int = 0) -> Context:
    """The calling thread's context on `device`.  Contexts are per thread so
    that threads working on separate streams never share a context's stream
    setting or error state."""
    table = getattr(_default, "table", None)
    if table is None:
        table = _default.table = {}
    ctx = table.get(device)
    if ctx is None:
        ctx = Context(device)
        table[device] = ctx
    return ctx
