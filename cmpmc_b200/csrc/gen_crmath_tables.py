"""Generates crmath_tables.h: double-double constants of the correctly rounded math
functions in crmath.cuh, computed with 80-digit decimal arithmetic.

  kLogC[n - 85] = log(n / 128) for n = 85 .. 171 (as hi + lo)
  kLn2          = log(2)
  kInvOdd[k]    = 1 / (2k + 1)                     (atanh series of log1p)
  kSinC[k]      = (-1)^k / (2k + 1)!, kCosC[k] = (-1)^k / (2k)!
  kPio2_1..4    = pi/2 split into 33 + 33 + 53 + 53 significant bits (Cody-Waite)

Usage: python cmpmc_b200/csrc/gen_crmath_tables.py > cmpmc_b200/csrc/crmath_tables.h
"""
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 80
PI = Decimal("3.1415926535897932384626433832795028841971693993751058209749445923078164062862089986280348253421170679")


def dd(x: Decimal):
    hi = float(x)
    lo = float(x - Decimal(hi))
    return hi, lo


def trunc_bits(x: Decimal, bits: int) -> float:
    """x rounded to `bits` significant bits (exactly representable in a double)."""
    f = Fraction(x)
    e = 0
    while f >= 1:
        f /= 2
        e += 1
    while f < Fraction(1, 2):
        f *= 2
        e -= 1
    m = round(f * (1 << bits))
    return float(Fraction(m, 1 << bits) * (Fraction(2) ** e))


def h(v: float) -> str:
    return float.hex(v)


def main() -> None:
    out = ["// Generated by gen_crmath_tables.py (80-digit decimal arithmetic). Do not edit.",
           "// Each table is a brace initializer; crmath.cuh instantiates a host and a device copy.",
           "#pragma once", ""]
    out.append("// log(n / 128), n = 85 .. 171")
    out.append("#define CMPMC_CR_LOGC { \\")
    for n in range(85, 172):
        hi, lo = dd((Decimal(n) / Decimal(128)).ln())
        out.append(f"    {{{h(hi)}, {h(lo)}}}, \\")
    out.append("  }")
    hi, lo = dd(Decimal(2).ln())
    out.append(f"#define CMPMC_CR_LN2_HI {h(hi)}\n#define CMPMC_CR_LN2_LO {h(lo)}")
    # log 2 split for the fast path: a 42-bit head (e * head exact for |e| < 2^11) and a tail
    l2 = Decimal(2).ln()
    h42 = trunc_bits(l2, 42)
    out.append(f"#define CMPMC_CR_LN2_H42 {h(h42)}\n#define CMPMC_CR_LN2_T42 {h(float(l2 - Decimal(h42)))}")
    # 1/6 and 1/24 as double-doubles (leading Taylor terms of the fast sin / cos paths)
    for name, v in (("INV6", Decimal(1) / 6), ("INV24", Decimal(1) / 24)):
        a, b = dd(v)
        out.append(f"#define CMPMC_CR_{name}_HI {h(a)}\n#define CMPMC_CR_{name}_LO {h(b)}")
    out.append("// 1 / (2k + 1)")
    out.append("#define CMPMC_CR_INVODD { \\")
    for k in range(12):
        hi, lo = dd(Decimal(1) / Decimal(2 * k + 1))
        out.append(f"    {{{h(hi)}, {h(lo)}}}, \\")
    out.append("  }")
    fact = [Decimal(1)]
    for i in range(1, 40):
        fact.append(fact[-1] * i)
    out.append("// (-1)^k / (2k + 1)!")
    out.append("#define CMPMC_CR_SINC { \\")
    for k in range(16):
        hi, lo = dd(Decimal((-1) ** k) / fact[2 * k + 1])
        out.append(f"    {{{h(hi)}, {h(lo)}}}, \\")
    out.append("  }")
    out.append("// (-1)^k / (2k)!")
    out.append("#define CMPMC_CR_COSC { \\")
    for k in range(17):
        hi, lo = dd(Decimal((-1) ** k) / fact[2 * k])
        out.append(f"    {{{h(hi)}, {h(lo)}}}, \\")
    out.append("  }")
    pio2 = PI / 2
    p1 = trunc_bits(pio2, 33)
    p2 = trunc_bits(pio2 - Decimal(p1), 33)
    rest = pio2 - Decimal(p1) - Decimal(p2)
    p3 = float(rest)
    p4 = float(rest - Decimal(p3))
    out.append("// pi/2 = kPio2[0] + kPio2[1] + kPio2[2] + kPio2[3]; the first two carry 33 bits")
    out.append(f"#define CMPMC_CR_PIO2_1 {h(p1)}\n#define CMPMC_CR_PIO2_2 {h(p2)}\n#define CMPMC_CR_PIO2_3 {h(p3)}\n#define CMPMC_CR_PIO2_4 {h(p4)}")
    out.append(f"#define CMPMC_CR_TWO_OVER_PI {h(float(2 / PI))}")
    out.append("")
    print("\n".join(out))


if __name__ == "__main__":
    main()
