"""CPU oracle for the decryption path -- test infrastructure only.

`oracle.oracle` is the ctypes front end of the C restatement in
bls12_381_oracle.c; `oracle.wbtx_oracle` restates the weighted_btx pipeline on
top of it.  Only tests/, the smoke check and the CPU-baseline leg of bench.py
use this package, and only as the checker.
"""
