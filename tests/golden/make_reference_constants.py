"""Extracts the constants that the reference's own tests pin for this path
and writes reference_constants.json beside this script.

    python tests/golden/make_reference_constants.py /path/to/reference

Sources (paths inside the reference project):
  btx/src/fft.rs:22       BLS12_381_X_ABS
  btx/src/fft.rs:656-681  HARD_EXPONENT, (p^4 - p^2 + 1) / r as u64 limbs
  btx/src/final_exponentiation.rs:33  MILLER_LINE_COUNT
"""
import json
import os
import re
import sys


def main(ref_root: str) -> None:
    fft = open(os.path.join(ref_root, "btx/src/fft.rs")).read()
    fe = open(os.path.join(ref_root, "btx/src/final_exponentiation.rs")).read()
    x_abs = re.search(r"const BLS12_381_X_ABS: u64 = (0x[0-9a-f_]+);", fft).group(1)
    block = re.search(r"const HARD_EXPONENT: \[u64; 20\] = \[(.*?)\];", fft, re.S).group(1)
    limbs = [int(v.replace("_", ""), 16) for v in re.findall(r"0x[0-9a-f_]+", block)]
    lines = int(re.search(r"MILLER_LINE_COUNT: usize = (\d+);", fe).group(1))
    out = {
        "source": "btx/src/fft.rs:22,656-681; btx/src/final_exponentiation.rs:33",
        "bls12_381_x_abs": int(x_abs.replace("_", ""), 16),
        "hard_exponent_limbs_le": limbs,
        "miller_line_count": lines,
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_constants.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_constants.py <path of the reference project>")
    main(sys.argv[1])
