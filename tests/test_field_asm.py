"""The generated inline-PTX field arithmetic (csrc/field_asm.cuh), executed by
a small interpreter of the PTX subset it uses and checked against Python
big-integer arithmetic.  Runs on the CPU: it proves the carry chains of the
generated instruction sequences, not the compiler or the GPU.
"""
import random
import re
from pathlib import Path

import pytest

ASM = Path(__file__).resolve().parents[1] / "weighted_bte_b200" / "csrc" / "field_asm.cuh"
P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
M32 = 0xFFFFFFFF


def _functions():
    text = ASM.read_text()
    out = {}
    for m in re.finditer(r"void (\w+)\((.*?)\) \{\n    asm\(\"\{\\n\\t\"\n(.*?)\n        \"\}\"\n"
                         r"        : (.*?)\n        : (.*?)\);\n\}", text, re.S):
        name, _, body, outs, ins = m.groups()
        instrs = [l.strip()[1:-len("\\n\\t\"")] for l in body.split("\n")]
        operands = re.findall(r"\"=?&?r\"\((\w+)\[(\d+)\]\)", outs + ", " + ins)
        out[name] = (instrs, [(v, int(i)) for v, i in operands], len(re.findall(r"\"=", outs)))
    return out


FUNCS = _functions()


class Machine:
    """Executes the PTX subset of field_asm.cuh with 32-bit registers, one
    carry flag (CC.CF) and predicates."""

    def __init__(self, operands):
        self.reg = dict(operands)
        self.cf = 0

    def val(self, tok):
        tok = tok.strip()
        if tok.startswith("0x"):
            return int(tok, 16)
        if re.fullmatch(r"\d+", tok):
            return int(tok)
        return self.reg[tok]

    def run(self, instrs):
        labels = {ins[:-1]: k for k, ins in enumerate(instrs) if ins.endswith(":")}
        pc, steps = 0, 0
        while pc < len(instrs):
            ins = instrs[pc]
            pc += 1
            steps += 1
            assert steps < 100000, "runaway loop"
            if ins.startswith(".reg") or ins.endswith(":"):
                continue
            if ins.startswith("@"):
                guard, ins = ins.split(None, 1)
                if not self.reg[guard[1:]]:
                    continue
            op, rest = ins.rstrip(";").split(None, 1)
            if op == "bra":
                pc = labels[rest.strip()]
                continue
            args = [a.strip() for a in rest.split(",")]
            parts = op.split(".")
            base = parts[0]
            cc = "cc" in parts
            if base == "mov":
                self.reg[args[0]] = self.val(args[1])
            elif base in ("mad", "madc"):
                a, b, c = (self.val(x) for x in args[1:])
                prod = a * b
                half = (prod >> 32) if "hi" in parts else prod & M32
                s = half + c + (self.cf if base == "madc" else 0)
                self.reg[args[0]] = s & M32
                if cc:
                    self.cf = s >> 32
            elif base == "mul":
                assert "lo" in parts
                self.reg[args[0]] = (self.val(args[1]) * self.val(args[2])) & M32
            elif base in ("add", "addc"):
                s = self.val(args[1]) + self.val(args[2]) + (self.cf if base == "addc" else 0)
                self.reg[args[0]] = s & M32
                if cc:
                    self.cf = s >> 32
            elif base in ("sub", "subc"):
                s = self.val(args[1]) - self.val(args[2]) - (self.cf if base == "subc" else 0)
                self.reg[args[0]] = s & M32
                if cc:
                    self.cf = 1 if s < 0 else 0
            elif base == "and":
                self.reg[args[0]] = self.val(args[1]) & self.val(args[2])
            elif base == "setp":
                x, y = self.val(args[1]), self.val(args[2])
                self.reg[args[0]] = {"eq": x == y, "lt": x < y, "ne": x != y}[parts[1]]
            elif base == "selp":
                self.reg[args[0]] = self.val(args[1]) if self.reg[args[3]] else self.val(args[2])
            else:
                raise AssertionError("unhandled instruction " + ins)


def call(name, **arrays):
    instrs, operands, n_out = FUNCS[name]
    regs = {}
    for k, (v, i) in enumerate(operands):
        if k >= n_out:
            regs["%%%d" % k] = arrays[v][i]
    mach = Machine(regs)
    mach.run(instrs)
    res = {}
    for k, (v, i) in enumerate(operands[:n_out]):
        res.setdefault(v, {})[i] = mach.reg["%%%d" % k]
    return {v: [d[i] for i in range(len(d))] for v, d in res.items()}


def limbs(v, n):
    return [(v >> (32 * i)) & M32 for i in range(n)]


def value(ls):
    return sum(x << (32 * i) for i, x in enumerate(ls))


def edge_values(m):
    return [0, 1, 2, m - 1, m - 2, (m - 1) // 2, 1 << 255 if m > 1 << 256 else 1 << 200, m >> 1]


@pytest.mark.parametrize("name,modulus,n", [("fp_mont_mul", P, 12), ("fp_mont_mul_r4", P, 12),
                                            ("fp_mont_mul_r6", P, 12), ("fr_mont_mul", R, 8)])
def test_montgomery_product(name, modulus, n):
    rng = random.Random(1)
    rinv = pow(1 << (32 * n), -1, modulus)
    vals = edge_values(modulus) + [rng.randrange(modulus) for _ in range(40)]
    for i, a in enumerate(vals):
        b = vals[(7 * i + 3) % len(vals)]
        r = value(call(name, a=limbs(a, n), b=limbs(b, n))["r"])
        assert r == a * b * rinv % modulus


@pytest.mark.parametrize("name,modulus,n", [("fp_add_raw", P, 12), ("fp_sub_raw", P, 12),
                                            ("fr_add_raw", R, 8), ("fr_sub_raw", R, 8)])
def test_modular_sum(name, modulus, n):
    rng = random.Random(2)
    vals = edge_values(modulus) + [rng.randrange(modulus) for _ in range(40)]
    for i, a in enumerate(vals):
        b = vals[(5 * i + 1) % len(vals)]
        r = value(call(name, a=limbs(a, n), b=limbs(b, n))["r"])
        want = (a + b) % modulus if "add" in name else (a - b) % modulus
        assert r == want


def test_fp2_lazy_product():
    """c0 + c1 u = (a0 + a1 u)(b0 + b1 u) / R mod p, u^2 = -1, for canonical
    inputs and for the unreduced (< 2p) inputs the Montgomery product also
    accepts."""
    rng = random.Random(3)
    rinv = pow(1 << 384, -1, P)
    vals = edge_values(P) + [2 * P - 1, P, P + 1] + [rng.randrange(P) for _ in range(30)] + \
        [rng.randrange(2 * P) for _ in range(10)]
    for i in range(len(vals)):
        a0, a1 = vals[i], vals[(3 * i + 1) % len(vals)]
        b0, b1 = vals[(5 * i + 2) % len(vals)], vals[(11 * i + 7) % len(vals)]
        out = call("fp2_mont_mul_lazy", a0=limbs(a0, 12), a1=limbs(a1, 12), b0=limbs(b0, 12), b1=limbs(b1, 12))
        assert value(out["r0"]) == (a0 * b0 - a1 * b1) * rinv % P
        assert value(out["r1"]) == (a0 * b1 + a1 * b0) * rinv % P
