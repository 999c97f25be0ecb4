"""B200-native batched threshold decryption over BLS12-381.

The compute path is libwbte.so (hand-written sm_100a kernels behind the C ABI
of include/wbte.h).  `weighted_btx` mirrors the public API of the reference
crate of the same name; `ops` exposes the primitives.
"""
__version__ = "0.1.0"
