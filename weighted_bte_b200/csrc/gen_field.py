"""Generates field_asm.cuh and constants.cuh for the sm_100a kernels.

field_asm.cuh holds the Montgomery multiplication and modular add/sub for
Fp (12 x 32-bit limbs, R = 2^384) and Fr (8 x 32-bit limbs, R = 2^256) as
single inline-PTX blocks, so that every carry chain (mad.lo.cc / madc.hi.cc)
lives inside one asm statement and the carry flag is never exposed to the
compiler between statements.

constants.cuh holds the curve constants in Montgomery form: generators,
Frobenius coefficients, the curve coefficients, the GLV cube root, and the
BLS parameter.  Every constant is derived here from p, r and x (the public
BLS12-381 parameters) and checked (on-curve, subgroup order) before emission.

Run:  python gen_field.py   (writes both headers next to this file)
"""
import os

P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
X = -0xD201000000010000
G1X = 0x17F1D3A73197D7942695638C4FA9AC0FC3688C4F9774B905A14E3A3F171BAC586C55E83FF97A1AEFFB3AF00ADB22C6BB
G1Y = 0x08B3F481E3AAA0F1A09E30ED741D8AE4FCF5E095D5D00AF600DB18CB2C04B3EDD03CC744A2888AE40CAA232946C5E7E1
G2X0 = 0x024AA2B2F08F0A91260805272DC51051C6E47AD4FA403B02B4510B647AE3D1770BAC0326A805BBEFD48056C8C121BDB8
G2X1 = 0x13E02B6052719F607DACD3A088274F65596BD0D09920B61AB5DA61BBDC7F5049334CF11213945D57E5AC7D055D042B7E
G2Y0 = 0x0CE5D527727D6E118CC9CDC6DA2E351AADFD9BAA8CBDD3A76D429A695160D12C923AC9CC3BACA289E193548608B82801
G2Y1 = 0x0606C4A02EA734CC32ACD2B02BC28B99CB3E287E85A763AF267492AB572E99AB3F370D275CEC1DA1AAA9075FF05F79BE

HERE = os.path.dirname(os.path.abspath(__file__))


def limbs32(v, n):
    return [(v >> (32 * i)) & 0xFFFFFFFF for i in range(n)]


# --------------------------------------------------------------- PTX code
def gen_mont_mul(name, modulus, n):
    """CIOS Montgomery product of a, b (< 2m when 4m < 2^(32n), else < m)."""
    pinv = (-pow(modulus, -1, 1 << 32)) % (1 << 32)
    ml = limbs32(modulus, n)
    lines = []
    w = lines.append
    w(".reg .u32 t<%d>, m, bw, d<%d>;" % (n + 2, n))
    w(".reg .pred nb;")
    t = ["t%d" % i for i in range(n + 2)]
    a = ["%%%d" % (n + i) for i in range(n)]
    b = ["%%%d" % (2 * n + i) for i in range(n)]
    out = ["%%%d" % i for i in range(n)]
    for i in range(n + 1):
        w("mov.u32 %s, 0;" % t[i])
    for i in range(n):
        bi = b[i]
        # t += a * b_i, low halves
        w("mad.lo.cc.u32 %s, %s, %s, %s;" % (t[0], a[0], bi, t[0]))
        for j in range(1, n):
            w("madc.lo.cc.u32 %s, %s, %s, %s;" % (t[j], a[j], bi, t[j]))
        w("addc.cc.u32 %s, %s, 0;" % (t[n], t[n]))
        w("addc.u32 %s, 0, 0;" % t[n + 1])
        # high halves
        w("mad.hi.cc.u32 %s, %s, %s, %s;" % (t[1], a[0], bi, t[1]))
        for j in range(1, n):
            w("madc.hi.cc.u32 %s, %s, %s, %s;" % (t[j + 1], a[j], bi, t[j + 1]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        # m = t0 * pinv ; t += m * modulus
        w("mul.lo.u32 m, %s, 0x%08x;" % (t[0], pinv))
        w("mad.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[0], ml[0], t[0]))
        for j in range(1, n):
            w("madc.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[j], ml[j], t[j]))
        w("addc.cc.u32 %s, %s, 0;" % (t[n], t[n]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        w("mad.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[1], ml[0], t[1]))
        for j in range(1, n):
            w("madc.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[j + 1], ml[j], t[j + 1]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        # shift right by one limb: rename registers
        t = t[1:] + [t[0]]
    # conditional subtraction: result in t[0..n-1] (t[n] is zero by the bound)
    w("sub.cc.u32 d0, %s, 0x%08x;" % (t[0], ml[0]))
    for j in range(1, n):
        w("subc.cc.u32 d%d, %s, 0x%08x;" % (j, t[j], ml[j]))
    w("subc.cc.u32 bw, %s, 0;" % t[n])
    w("subc.u32 bw, 0, 0;")
    w("setp.eq.u32 nb, bw, 0;")
    for j in range(n):
        w("selp.u32 %s, d%d, %s, nb;" % (out[j], j, t[j]))
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join('"=r"(r[%d])' % i for i in range(n))
    ins = ", ".join(['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r[%d], const uint32_t a[%d], const uint32_t b[%d]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, n, n, n, body, outs, ins)
    )


def gen_mont_mul_rolled(name, modulus, n, unroll):
    """The CIOS product of gen_mont_mul as a loop of n / unroll iterations of
    `unroll` rows each (about a third of the code of the straight-line
    sequence for unroll = 4, at the cost of the register rotation between
    iterations).  Emitted for the code-size experiments of fetch-bound
    kernels; one instance per translation unit (the loop label is fixed)."""
    assert n % unroll == 0
    pinv = (-pow(modulus, -1, 1 << 32)) % (1 << 32)
    ml = limbs32(modulus, n)
    lines = []
    w = lines.append
    w(".reg .u32 t<%d>, bb<%d>, m, bw, d<%d>, cnt, tmp;" % (n + 2, n, n))
    w(".reg .pred nb, more;")
    a = ["%%%d" % (n + i) for i in range(n)]
    b = ["%%%d" % (2 * n + i) for i in range(n)]
    out = ["%%%d" % i for i in range(n)]
    canon = ["t%d" % i for i in range(n + 2)]
    for i in range(n + 1):
        w("mov.u32 %s, 0;" % canon[i])
    for i in range(n):
        w("mov.u32 bb%d, %s;" % (i, b[i]))
    w("mov.u32 cnt, 0;")
    w("$Lcios_%s:" % name)
    t = list(canon)
    for r in range(unroll):
        bi = "bb%d" % r
        w("mad.lo.cc.u32 %s, %s, %s, %s;" % (t[0], a[0], bi, t[0]))
        for j in range(1, n):
            w("madc.lo.cc.u32 %s, %s, %s, %s;" % (t[j], a[j], bi, t[j]))
        w("addc.cc.u32 %s, %s, 0;" % (t[n], t[n]))
        w("addc.u32 %s, 0, 0;" % t[n + 1])
        w("mad.hi.cc.u32 %s, %s, %s, %s;" % (t[1], a[0], bi, t[1]))
        for j in range(1, n):
            w("madc.hi.cc.u32 %s, %s, %s, %s;" % (t[j + 1], a[j], bi, t[j + 1]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        w("mul.lo.u32 m, %s, 0x%08x;" % (t[0], pinv))
        w("mad.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[0], ml[0], t[0]))
        for j in range(1, n):
            w("madc.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[j], ml[j], t[j]))
        w("addc.cc.u32 %s, %s, 0;" % (t[n], t[n]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        w("mad.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[1], ml[0], t[1]))
        for j in range(1, n):
            w("madc.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[j + 1], ml[j], t[j + 1]))
        w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
        t = t[1:] + [t[0]]
    # back to the canonical names: canon[k] <- t[k] for all n + 2 registers,
    # k -> k + unroll (mod n + 2) being a permutation, moved cycle by cycle
    src = {canon[k]: t[k] for k in range(n + 2)}
    done = set()
    for start in canon:
        if start in done or src[start] == start:
            continue
        chain = [start]
        cur = src[start]
        while cur != start:
            chain.append(cur)
            cur = src[cur]
        w("mov.u32 tmp, %s;" % chain[0])
        for k in range(len(chain) - 1):
            w("mov.u32 %s, %s;" % (chain[k], chain[k + 1]))
        w("mov.u32 %s, tmp;" % chain[-1])
        done.update(chain)
    for k in range(n - unroll):
        w("mov.u32 bb%d, bb%d;" % (k, k + unroll))
    w("add.u32 cnt, cnt, %d;" % unroll)
    w("setp.lt.u32 more, cnt, %d;" % n)
    w("@more bra $Lcios_%s;" % name)
    t = list(canon)
    w("sub.cc.u32 d0, %s, 0x%08x;" % (t[0], ml[0]))
    for j in range(1, n):
        w("subc.cc.u32 d%d, %s, 0x%08x;" % (j, t[j], ml[j]))
    w("subc.cc.u32 bw, %s, 0;" % t[n])
    w("subc.u32 bw, 0, 0;")
    w("setp.eq.u32 nb, bw, 0;")
    for j in range(n):
        w("selp.u32 %s, d%d, %s, nb;" % (out[j], j, t[j]))
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join('"=r"(r[%d])' % i for i in range(n))
    ins = ", ".join(['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r[%d], const uint32_t a[%d], const uint32_t b[%d]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, n, n, n, body, outs, ins)
    )


def gen_add(name, modulus, n):
    """r = a + b mod m (inputs < m)."""
    ml = limbs32(modulus, n)
    lines = [".reg .u32 s<%d>, d<%d>, bw;" % (n + 1, n), ".reg .pred nb;"]
    w = lines.append
    a = ["%%%d" % (n + i) for i in range(n)]
    b = ["%%%d" % (2 * n + i) for i in range(n)]
    w("add.cc.u32 s0, %s, %s;" % (a[0], b[0]))
    for j in range(1, n):
        w("addc.cc.u32 s%d, %s, %s;" % (j, a[j], b[j]))
    w("addc.u32 s%d, 0, 0;" % n)
    w("sub.cc.u32 d0, s0, 0x%08x;" % ml[0])
    for j in range(1, n):
        w("subc.cc.u32 d%d, s%d, 0x%08x;" % (j, j, ml[j]))
    w("subc.cc.u32 bw, s%d, 0;" % n)
    w("subc.u32 bw, 0, 0;")
    w("setp.eq.u32 nb, bw, 0;")
    for j in range(n):
        w("selp.u32 %%%d, d%d, s%d, nb;" % (j, j, j))
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join('"=r"(r[%d])' % i for i in range(n))
    ins = ", ".join(['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r[%d], const uint32_t a[%d], const uint32_t b[%d]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, n, n, n, body, outs, ins)
    )


def gen_sub(name, modulus, n):
    """r = a - b mod m (inputs < m)."""
    ml = limbs32(modulus, n)
    lines = [".reg .u32 s<%d>, bw;" % n]
    w = lines.append
    a = ["%%%d" % (n + i) for i in range(n)]
    b = ["%%%d" % (2 * n + i) for i in range(n)]
    w("sub.cc.u32 s0, %s, %s;" % (a[0], b[0]))
    for j in range(1, n):
        w("subc.cc.u32 s%d, %s, %s;" % (j, a[j], b[j]))
    w("subc.u32 bw, 0, 0;")
    # add (m & bw)
    w("and.b32 %%0, bw, 0x%08x;" % ml[0])
    w("add.cc.u32 %0, s0, %0;")
    for j in range(1, n):
        w("and.b32 %%%d, bw, 0x%08x;" % (j, ml[j]))
        w("addc.cc.u32 %%%d, s%d, %%%d;" % (j, j, j))
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join('"=&r"(r[%d])' % i for i in range(n))
    ins = ", ".join(['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r[%d], const uint32_t a[%d], const uint32_t b[%d]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, n, n, n, body, outs, ins)
    )


def gen_add_nr(name, n):
    """r = a + b without reduction (caller guarantees no overflow)."""
    lines = []
    w = lines.append
    a = ["%%%d" % (n + i) for i in range(n)]
    b = ["%%%d" % (2 * n + i) for i in range(n)]
    w("add.cc.u32 %%0, %s, %s;" % (a[0], b[0]))
    for j in range(1, n - 1):
        w("addc.cc.u32 %%%d, %s, %s;" % (j, a[j], b[j]))
    w("addc.u32 %%%d, %s, %s;" % (n - 1, a[n - 1], b[n - 1]))
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join('"=r"(r[%d])' % i for i in range(n))
    ins = ", ".join(['"r"(a[%d])' % i for i in range(n)] + ['"r"(b[%d])' % i for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r[%d], const uint32_t a[%d], const uint32_t b[%d]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, n, n, n, body, outs, ins)
    )



def gen_fp2_mul_lazy(name):
    """Fp2 product (a0 + a1 u)(b0 + b1 u), u^2 = -1, with lazy reduction.

    Karatsuba over double-width products: x = a0 b0, y = a1 b1 and
    z = (a0 + a1)(b0 + b1) are formed as full 768-bit products, and only the
    two results are Montgomery-reduced:
        c0 = REDC(x - y  [+ 4 p^2 when negative]),   c1 = REDC(z - x - y).
    Three 12x12-limb products (288 multiply-adds each) and two reductions
    (300 each): 1,464 multiply-adds against 1,764 for three CIOS products.
    Inputs < 2p (so both REDC inputs stay below 8 p^2 < p R); outputs < p.
    """
    n = 12
    ml = limbs32(P, n)
    p2 = limbs32(4 * P * P, 2 * n)
    pinv = (-pow(P, -1, 1 << 32)) % (1 << 32)
    lines = []
    w = lines.append
    w(".reg .u32 x<24>, y<24>, z<24>, sa<12>, sb<12>, t<14>, d<12>, m, bw;")
    w(".reg .pred nb;")
    c0 = ["%%%d" % i for i in range(n)]
    c1 = ["%%%d" % (n + i) for i in range(n)]
    a0 = ["%%%d" % (2 * n + i) for i in range(n)]
    a1 = ["%%%d" % (3 * n + i) for i in range(n)]
    b0 = ["%%%d" % (4 * n + i) for i in range(n)]
    b1 = ["%%%d" % (5 * n + i) for i in range(n)]

    def add_nr(dst, u, v):
        w("add.cc.u32 %s, %s, %s;" % (dst[0], u[0], v[0]))
        for j in range(1, n - 1):
            w("addc.cc.u32 %s, %s, %s;" % (dst[j], u[j], v[j]))
        w("addc.u32 %s, %s, %s;" % (dst[n - 1], u[n - 1], v[n - 1]))

    def mul_wide(dst, u, v):
        # Operand scanning.  After row i the partial sum u * (v mod 2^(32(i+1)))
        # fits dst[0 .. i + 12], so the top word of each row's high chain
        # takes no carry out.
        for j in range(n):
            w("mul.lo.u32 %s, %s, %s;" % (dst[j], u[j], v[0]))
        w("mad.hi.cc.u32 %s, %s, %s, %s;" % (dst[1], u[0], v[0], dst[1]))
        for j in range(1, n - 1):
            w("madc.hi.cc.u32 %s, %s, %s, %s;" % (dst[j + 1], u[j], v[0], dst[j + 1]))
        w("madc.hi.u32 %s, %s, %s, 0;" % (dst[n], u[n - 1], v[0]))
        for i in range(1, n):
            w("mad.lo.cc.u32 %s, %s, %s, %s;" % (dst[i], u[0], v[i], dst[i]))
            for j in range(1, n):
                w("madc.lo.cc.u32 %s, %s, %s, %s;" % (dst[i + j], u[j], v[i], dst[i + j]))
            w("addc.u32 %s, 0, 0;" % dst[i + n])
            w("mad.hi.cc.u32 %s, %s, %s, %s;" % (dst[i + 1], u[0], v[i], dst[i + 1]))
            for j in range(1, n - 1):
                w("madc.hi.cc.u32 %s, %s, %s, %s;" % (dst[i + 1 + j], u[j], v[i], dst[i + 1 + j]))
            w("madc.hi.u32 %s, %s, %s, %s;" % (dst[i + n], u[n - 1], v[i], dst[i + n]))

    def redc(out, src):
        # Montgomery reduction of a 24-limb value < p R into out (< p).
        t = ["t%d" % k for k in range(n + 2)]
        for k in range(n):
            w("mov.u32 %s, %s;" % (t[k], src[k]))
        w("mov.u32 %s, 0;" % t[n])
        for i in range(n):
            w("add.cc.u32 %s, %s, %s;" % (t[n], t[n], src[n + i]))
            w("addc.u32 %s, 0, 0;" % t[n + 1])
            w("mul.lo.u32 m, %s, 0x%08x;" % (t[0], pinv))
            w("mad.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[0], ml[0], t[0]))
            for j in range(1, n):
                w("madc.lo.cc.u32 %s, m, 0x%08x, %s;" % (t[j], ml[j], t[j]))
            w("addc.cc.u32 %s, %s, 0;" % (t[n], t[n]))
            w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
            w("mad.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[1], ml[0], t[1]))
            for j in range(1, n):
                w("madc.hi.cc.u32 %s, m, 0x%08x, %s;" % (t[j + 1], ml[j], t[j + 1]))
            w("addc.u32 %s, %s, 0;" % (t[n + 1], t[n + 1]))
            t = t[1:] + [t[0]]
        w("sub.cc.u32 d0, %s, 0x%08x;" % (t[0], ml[0]))
        for j in range(1, n):
            w("subc.cc.u32 d%d, %s, 0x%08x;" % (j, t[j], ml[j]))
        w("subc.cc.u32 bw, %s, 0;" % t[n])
        w("subc.u32 bw, 0, 0;")
        w("setp.eq.u32 nb, bw, 0;")
        for j in range(n):
            w("selp.u32 %s, d%d, %s, nb;" % (out[j], j, t[j]))

    x = ["x%d" % k for k in range(2 * n)]
    y = ["y%d" % k for k in range(2 * n)]
    z = ["z%d" % k for k in range(2 * n)]
    sa = ["sa%d" % k for k in range(n)]
    sb = ["sb%d" % k for k in range(n)]
    add_nr(sa, a0, a1)
    add_nr(sb, b0, b1)
    mul_wide(x, a0, b0)
    mul_wide(y, a1, b1)
    # z <- x - y, plus 4 p^2 when it borrowed
    w("sub.cc.u32 z0, x0, y0;")
    for k in range(1, 2 * n):
        w("subc.cc.u32 z%d, x%d, y%d;" % (k, k, k))
    w("subc.u32 bw, 0, 0;")
    w("and.b32 m, bw, 0x%08x;" % p2[0])
    w("add.cc.u32 z0, z0, m;")
    for k in range(1, 2 * n):
        w("and.b32 m, bw, 0x%08x;" % p2[k])
        w("addc.cc.u32 z%d, z%d, m;" % (k, k))
    redc(c0, z)
    # x <- x + y (below 2^768: both are below 4 p^2)
    w("add.cc.u32 x0, x0, y0;")
    for k in range(1, 2 * n - 1):
        w("addc.cc.u32 x%d, x%d, y%d;" % (k, k, k))
    w("addc.u32 x%d, x%d, y%d;" % (2 * n - 1, 2 * n - 1, 2 * n - 1))
    mul_wide(z, sa, sb)
    w("sub.cc.u32 z0, z0, x0;")
    for k in range(1, 2 * n - 1):
        w("subc.cc.u32 z%d, z%d, x%d;" % (k, k, k))
    w("subc.u32 z%d, z%d, x%d;" % (2 * n - 1, 2 * n - 1, 2 * n - 1))
    redc(c1, z)
    body = "\n".join("        \"" + l + "\\n\\t\"" for l in lines)
    outs = ", ".join(['"=&r"(r0[%d])' % i for i in range(n)] + ['"=&r"(r1[%d])' % i for i in range(n)])
    ins = ", ".join(['"r"(%s[%d])' % (v, i) for v in ("a0", "a1", "b0", "b1") for i in range(n)])
    return (
        "__device__ __forceinline__ void %s(uint32_t r0[12], uint32_t r1[12], const uint32_t a0[12], "
        "const uint32_t a1[12],\n        const uint32_t b0[12], const uint32_t b1[12]) {\n"
        "    asm(\"{\\n\\t\"\n%s\n        \"}\"\n        : %s\n        : %s);\n}\n" % (name, body, outs, ins)
    )


# ------------------------------------------------------------- constants
def fp2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def fp2_pow(a, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = fp2_mul(r, a)
        a = fp2_mul(a, a)
        e >>= 1
    return r


def fp2_inv(a):
    n = pow(a[0] * a[0] + a[1] * a[1], P - 2, P)
    return (a[0] * n % P, (-a[1]) * n % P)


def ec_add(P1, Q1, mul, add, sub, inv, zero, three, two):
    if P1 is None:
        return Q1
    if Q1 is None:
        return P1
    if P1[0] == Q1[0]:
        if P1[1] == Q1[1] and P1[1] != zero:
            l = mul(mul(three, mul(P1[0], P1[0])), inv(mul(two, P1[1])))
        else:
            return None
    else:
        l = mul(sub(Q1[1], P1[1]), inv(sub(Q1[0], P1[0])))
    x3 = sub(sub(mul(l, l), P1[0]), Q1[0])
    return (x3, sub(mul(l, sub(P1[0], x3)), P1[1]))


def ec_mul(Pt, k, ops):
    acc, Q = None, Pt
    while k:
        if k & 1:
            acc = ec_add(acc, Q, *ops)
        Q = ec_add(Q, Q, *ops)
        k >>= 1
    return acc


FP_OPS = (lambda a, b: a * b % P, lambda a, b: (a + b) % P, lambda a, b: (a - b) % P,
          lambda a: pow(a, P - 2, P), 0, 3, 2)
FP2_OPS = (fp2_mul, lambda a, b: ((a[0] + b[0]) % P, (a[1] + b[1]) % P),
           lambda a, b: ((a[0] - b[0]) % P, (a[1] - b[1]) % P), fp2_inv, (0, 0), (3, 0), (2, 0))


def mont(v):
    return (v << 384) % P


def fp_lit(v):
    return "{" + ", ".join("0x%08xu" % l for l in limbs32(mont(v), 12)) + "}"


def fp2_lit(a):
    return "{" + fp_lit(a[0]) + ", " + fp_lit(a[1]) + "}"


def gen_constants():
    assert X ** 4 - X ** 2 + 1 == R
    g1 = (G1X, G1Y)
    g2 = ((G2X0, G2X1), (G2Y0, G2Y1))
    assert (G1Y * G1Y - G1X ** 3 - 4) % P == 0
    lhs = fp2_mul(g2[1], g2[1])
    rhs = fp2_mul(fp2_mul(g2[0], g2[0]), g2[0])
    assert lhs == ((rhs[0] + 4) % P, (rhs[1] + 4) % P)
    assert ec_mul(g1, R, FP_OPS) is None
    assert ec_mul(g2, R, FP2_OPS) is None
    # GLV: phi(x, y) = (beta x, y) acts as [lambda] with lambda = x^2 - 1
    lam = (X * X - 1) % R
    assert (lam * lam + lam + 1) % R == 0
    beta = None
    gg = 2
    while beta is None:
        c = pow(gg, (P - 1) // 3, P)
        if c != 1:
            for cand in (c, c * c % P):
                if (G1X * cand % P, G1Y) == ec_mul(g1, lam, FP_OPS):
                    beta = cand
        gg += 1
    # Frobenius coefficients FROB[k][i] = xi^{i (p^k - 1)/6}, xi = 1 + u
    xi = (1, 1)
    frob = []
    for k in range(1, 4):
        frob.append([fp2_pow(xi, i * (P ** k - 1) // 6) for i in range(6)])
    # psi (untwist-Frobenius-twist) on G2: psi(x, y) = (conj(x) * cx, conj(y) * cy)
    cx = fp2_inv(fp2_pow(xi, (P - 1) // 3))
    cy = fp2_inv(fp2_pow(xi, (P - 1) // 2))

    def psi(pt):
        (x0, x1), (y0, y1) = pt
        return (fp2_mul((x0, (-x1) % P), cx), fp2_mul((y0, (-y1) % P), cy))

    assert psi(g2) == ec_mul(g2, X % R, FP2_OPS), "psi must act as [x]"
    out = []
    w = out.append
    w("// Generated by gen_field.py from the BLS12-381 parameters p, r and x.")
    w("// All field constants are in Montgomery form (R = 2^384).")
    w("#pragma once")
    w("#include <cstdint>")
    w("namespace wbte {")
    w("__device__ __constant__ const uint32_t C_FP_ONE[12] = %s;" % fp_lit(1))
    w("__device__ __constant__ const uint32_t C_FP_B1[12] = %s;  // 4" % fp_lit(4))
    w("__device__ __constant__ const uint32_t C_FP_B2X3[2][12] = %s;  // 3 * 4(1+u)" % fp2_lit((12, 12)))
    w("__device__ __constant__ const uint32_t C_G1_GEN[2][12] = {%s, %s};" % (fp_lit(G1X), fp_lit(G1Y)))
    w("__device__ __constant__ const uint32_t C_G2_GEN[4][12] = {%s, %s, %s, %s};" % (
        fp_lit(G2X0), fp_lit(G2X1), fp_lit(G2Y0), fp_lit(G2Y1)))
    w("__device__ __constant__ const uint32_t C_GLV_BETA[12] = %s;" % fp_lit(beta))
    w("__device__ __constant__ const uint32_t C_PSI_CX[2][12] = %s;" % fp2_lit(cx))
    w("__device__ __constant__ const uint32_t C_PSI_CY[2][12] = %s;" % fp2_lit(cy))
    rows = []
    for k in range(3):
        rows.append("{" + ", ".join(fp2_lit(c) for c in frob[k]) + "}")
    w("// C_FROB[k-1][i] = xi^{i (p^k - 1) / 6}, coefficient of w^i")
    w("__device__ __constant__ const uint32_t C_FROB[3][6][2][12] = {%s};" % ", ".join(rows))
    w("__device__ __constant__ const uint32_t C_P[12] = {%s};" % ", ".join("0x%08xu" % l for l in limbs32(P, 12)))
    w("__device__ __constant__ const uint32_t C_R[8] = {%s};" % ", ".join("0x%08xu" % l for l in limbs32(R, 8)))
    w("__device__ __constant__ const uint32_t C_FR_ONE[8] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((1 << 256) % R, 8)))
    w("__device__ __constant__ const uint32_t C_FR_R2[8] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((1 << 512) % R, 8)))
    w("__device__ __constant__ const uint32_t C_FP_R2[12] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((1 << 768) % P, 12)))
    w("// (p - 1) / 2, canonical, for the compressed-point sign flag")
    w("__device__ __constant__ const uint32_t C_P_HALF[12] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((P - 1) // 2, 12)))
    w("__device__ __constant__ const uint32_t C_P_MINUS_2[12] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32(P - 2, 12)))
    w("// square-root exponents: (p + 1) / 4 in Fp, (p - 3) / 4 in Fp2 (p = 3 mod 4)")
    w("__device__ __constant__ const uint32_t C_P_PLUS1_DIV4[12] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((P + 1) // 4, 12)))
    w("__device__ __constant__ const uint32_t C_P_MINUS3_DIV4[12] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32((P - 3) // 4, 12)))
    w("__device__ __constant__ const uint32_t C_R_MINUS_2[8] = {%s};" % ", ".join(
        "0x%08xu" % l for l in limbs32(R - 2, 8)))
    # Radix-2 domain generators: the two-adic root 7^((r-1)/2^32), squared down.
    root = pow(7, (R - 1) >> 32, R)
    assert pow(root, 1 << 32, R) == 1 and pow(root, 1 << 31, R) != 1
    gens, gens_inv, size_inv = [], [], []
    for k in range(33):
        g = pow(root, 1 << (32 - k), R)
        gens.append(g)
        gens_inv.append(pow(g, R - 2, R))
        size_inv.append(pow(1 << k, R - 2, R))

    def fr_lit(v):
        return "{" + ", ".join("0x%08xu" % l for l in limbs32((v << 256) % R, 8)) + "}"

    w("// C_DOMAIN_GEN[k]: generator of the order-2^k subgroup of Fr^*, Montgomery form")
    w("__device__ __constant__ const uint32_t C_DOMAIN_GEN[33][8] = {%s};" % ", ".join(fr_lit(g) for g in gens))
    w("__device__ __constant__ const uint32_t C_DOMAIN_GEN_INV[33][8] = {%s};" % ", ".join(fr_lit(g) for g in gens_inv))
    w("__device__ __constant__ const uint32_t C_DOMAIN_SIZE_INV[33][8] = {%s};" % ", ".join(fr_lit(g) for g in size_inv))
    w("constexpr uint64_t X_ABS = 0x%016xull;" % (-X))
    w("constexpr uint64_t GLV_LAMBDA_LO = 0x%016xull;" % (lam & ((1 << 64) - 1)))
    w("constexpr uint64_t GLV_LAMBDA_HI = 0x%016xull;" % (lam >> 64))
    w("}  // namespace wbte")
    return "\n".join(out) + "\n"


def main():
    parts = [
        "// Generated by gen_field.py: Montgomery arithmetic as single inline-PTX blocks.",
        "#pragma once",
        "#include <cstdint>",
        "namespace wbte {",
        gen_mont_mul("fp_mont_mul", P, 12),
        gen_add("fp_add_raw", P, 12),
        gen_sub("fp_sub_raw", P, 12),
        gen_add_nr("fp_add_nored", 12),
        gen_fp2_mul_lazy("fp2_mont_mul_lazy"),
        gen_mont_mul_rolled("fp_mont_mul_r4", P, 12, 4),
        gen_mont_mul_rolled("fp_mont_mul_r6", P, 12, 6),
        gen_mont_mul("fr_mont_mul", R, 8),
        gen_add("fr_add_raw", R, 8),
        gen_sub("fr_sub_raw", R, 8),
        "}  // namespace wbte",
    ]
    with open(os.path.join(HERE, "field_asm.cuh"), "w") as f:
        f.write("\n".join(parts))
    with open(os.path.join(HERE, "constants.cuh"), "w") as f:
        f.write(gen_constants())


if __name__ == "__main__":
    main()
