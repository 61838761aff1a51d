"""Writes pge_crmath_tables.inc: the constants of pge_crmath.cuh as double pairs.

Each value is computed with 100-digit decimal arithmetic (series summed far
past the needed precision) and split into hi = the value rounded to double,
lo = the rest rounded to double.  Run: python gen_crmath_tables.py > pge_crmath_tables.inc.  The includer
defines PGE_CR_QUAL (the declarations' qualifiers: constant memory for the
device, plain static arrays for the host).
"""
from decimal import Decimal as D, getcontext

getcontext().prec = 100
EPS = D(10) ** -95


def atan(x: D) -> D:
    h = 0
    while abs(x) > D("0.01"):  # atan(x) = 2 atan(x / (1 + sqrt(1 + x^2)))
        x = x / (1 + (1 + x * x).sqrt())
        h += 1
    s, t, n = D(0), x, 0
    while abs(t) > EPS:
        s += t / (2 * n + 1) if n % 2 == 0 else -t / (2 * n + 1)
        t *= x * x
        n += 1
    return s * (2 ** h)


def sincos(x: D):
    s, c, t, n = D(0), D(0), D(1), 0
    while abs(t) > EPS or n < 4:
        sign = 1 if (n // 2) % 2 == 0 else -1
        if n % 2 == 0:
            c += sign * t
        else:
            s += sign * t
        n += 1
        t = t * x / n
    return s, c


def split(v: D, parts: int = 2):
    out = []
    for _ in range(parts):
        h = float(v)
        out.append(h)
        v -= D(h)
    return out


def row(vals):
    return "{" + ", ".join(repr(v) for v in vals) + "}"


def main():
    pi = 4 * atan(D(1))
    lines = ["// generated by gen_crmath_tables.py: exact values rounded to (hi, lo) double pairs"]
    lines.append("// pi/2 in three parts")
    lines.append("PGE_CR_QUAL double kPio2[3] = " + row(split(pi / 2, 3)) + ";")
    lines.append("// sin(j/32), cos(j/32) for j = 0..26 (j/32 reaches past pi/4)")
    lines.append("PGE_CR_QUAL double kSinJ[27][2] = {" + ", ".join(row(split(sincos(D(j) / 32)[0])) for j in range(27)) + "};")
    lines.append("PGE_CR_QUAL double kCosJ[27][2] = {" + ", ".join(row(split(sincos(D(j) / 32)[1])) for j in range(27)) + "};")
    lines.append("// atan(k/64) for k = 0..64")
    lines.append("PGE_CR_QUAL double kAtanK[65][2] = {" + ", ".join(row(split(atan(D(k) / 64))) for k in range(65)) + "};")
    lines.append("// series coefficients: 1/3!, 1/5!, 1/2!, 1/4!, 1/6! and 1/3, 1/5, 1/7 as pairs")
    fact = lambda n: D(1) if n <= 1 else n * fact(n - 1)
    for name, v in (("kInv3f", 1 / fact(3)), ("kInv5f", 1 / fact(5)), ("kInv2f", 1 / fact(2)), ("kInv4f", 1 / fact(4)),
                    ("kInv6f", 1 / fact(6)), ("kInv3", D(1) / 3), ("kInv5", D(1) / 5), ("kInv7", D(1) / 7)):
        lines.append(f"PGE_CR_QUAL double {name}[2] = " + row(split(v)) + ";")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
