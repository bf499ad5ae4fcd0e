"""Generate the constants of gf_math.h from high-precision decimal arithmetic.

Every constant in gf_math.h is derived here from first principles: ln 2 and
ln 10 from Python's arbitrary-precision ``decimal`` logarithm, pi from
Machin's formula, atan(i/8) from the Taylor series of atan after argument
halving, and the polynomial coefficients from the Taylor series of exp,
sin, cos and atan (1/n!, (-1)^k/(2k+1)).  The output is a C header fragment
with exact hexadecimal double literals; run

    python galfast_b200/csrc/gen_math_consts.py > galfast_b200/csrc/gf_math_consts.h

and commit the result.  Nothing here is copied from a vendor math library.
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 80


def dec_atan(x: Decimal) -> Decimal:
    # halve the argument until it is small: atan(x) = 2 atan(x / (1 + sqrt(1 + x^2)))
    k = 0
    while abs(x) > Decimal("0.01"):
        x = x / (1 + (1 + x * x).sqrt())
        k += 1
    s, term, n = Decimal(0), x, 0
    x2 = x * x
    while True:
        t = term / (2 * n + 1)
        if t == 0 or abs(t) < Decimal(10) ** (-getcontext().prec + 2):
            break
        s += t if n % 2 == 0 else -t
        term *= x2
        n += 1
    return s * (2 ** k)


PI = 16 * dec_atan(Decimal(1) / 5) - 4 * dec_atan(Decimal(1) / 239)
LN2 = Decimal(2).ln()
LN10 = Decimal(10).ln()


def hexd(v) -> str:
    return float(v).hex()


def hi_lo(v: Decimal):
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def chop(v: Decimal, bits: int) -> float:
    """Round v to a double whose significand has at most `bits` bits."""
    f = float(v)
    m, e = math.frexp(f)
    scale = 2 ** bits
    m = math.floor(m * scale) / scale
    return math.ldexp(m, e)


def main():
    out = []
    w = out.append
    w("/* Generated by gen_math_consts.py from high-precision decimal arithmetic. Do not edit. */")
    w("#pragma once")
    # ln2 split for Cody-Waite reduction of exp: hi has 32 significant bits
    l2hi = chop(LN2, 32)
    l2lo = float(LN2 - Decimal(l2hi))
    w(f"#define GFM_LN2_HI {hexd(l2hi)}")
    w(f"#define GFM_LN2_LO {hexd(l2lo)}")
    w(f"#define GFM_INV_LN2 {hexd(1 / LN2)}")
    ln10_hi, ln10_lo = hi_lo(LN10)
    w(f"#define GFM_LN10_HI {hexd(ln10_hi)}")
    w(f"#define GFM_LN10_LO {hexd(ln10_lo)}")
    w(f"#define GFM_INV_LN10 {hexd(1 / LN10)}")
    # pi/2 split in three 33-bit pieces for the sin/cos reduction
    pio2 = PI / 2
    p1 = chop(pio2, 33)
    r = pio2 - Decimal(p1)
    p2 = chop(r, 33)
    r = r - Decimal(p2)
    p3 = float(r)
    w(f"#define GFM_PIO2_1 {hexd(p1)}")
    w(f"#define GFM_PIO2_2 {hexd(p2)}")
    w(f"#define GFM_PIO2_3 {hexd(p3)}")
    w(f"#define GFM_TWO_OVER_PI {hexd(2 / PI)}")
    pio2_hi, pio2_lo = hi_lo(pio2)
    w(f"#define GFM_PIO2_HI {hexd(pio2_hi)}")
    w(f"#define GFM_PIO2_LO {hexd(pio2_lo)}")
    pi_hi, pi_lo = hi_lo(PI)
    w(f"#define GFM_PI_HI {hexd(pi_hi)}")
    w(f"#define GFM_PI_LO {hexd(pi_lo)}")
    def coef_macros(name, vals):
        w(f"#define GFM_{name}_NCOEF {len(vals)}")
        for i, v in enumerate(vals):
            w(f"#define GFM_{name}_C{i} {hexd(v)}")

    # Taylor coefficients of exp: 1/n!, n = 0..13
    coef_macros("EXP", [Fraction(1, math.factorial(n)) for n in range(14)])
    # log series: log(m) = s * sum 2 z^k/(2k+1), k = 0..11, z = s^2
    coef_macros("LOG", [Fraction(2, 2 * k + 1) for k in range(12)])
    # sin(r) = r * sum (-1)^k r^(2k)/(2k+1)!, cos(r) = sum (-1)^k r^(2k)/(2k)!, k = 0..9
    coef_macros("SIN", [Fraction((-1) ** k, math.factorial(2 * k + 1)) for k in range(10)])
    coef_macros("COS", [Fraction((-1) ** k, math.factorial(2 * k)) for k in range(10)])
    # atan(u) = u * sum (-1)^k u^(2k)/(2k+1), k = 0..7 for |u| <= 1/16
    coef_macros("ATAN", [Fraction((-1) ** k, 2 * k + 1) for k in range(8)])
    # atan(i/8), i = 0..8, as hi/lo pairs
    his, los = [], []
    for i in range(9):
        v = dec_atan(Decimal(i) / 8) if i else Decimal(0)
        hi, lo = hi_lo(v)
        his.append(hexd(hi))
        los.append(hexd(lo))
    w("#define GFM_ATAN_TAB_HI_LIST { " + ", ".join(his) + " }")
    w("#define GFM_ATAN_TAB_LO_LIST { " + ", ".join(los) + " }")
    print("\n".join(out))


if __name__ == "__main__":
    main()
