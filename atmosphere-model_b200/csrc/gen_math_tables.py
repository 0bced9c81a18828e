"""Generate atm_math_tables.h: the constant tables of the portable log/exp
(and, with --kappa, atm_kappa_tables.h: those of the mixed form's p**kappa).

The tables follow the table-driven method of P. T. P. Tang ("Table-driven
implementation of the exponential function in IEEE floating-point
arithmetic", ACM TOMS 15(2), 1989; "Table-driven implementation of the
logarithm function in IEEE floating-point arithmetic", ACM TOMS 16(4), 1990).
Every entry is computed here with Python's decimal module at 60 significant
digits and rounded to nearest double, so the header is reproducible:

    python gen_math_tables.py > atm_math_tables.h
    python gen_math_tables.py --kappa > atm_kappa_tables.h

p**kappa for the fixed kappa = R_dry / cp_dry of the dynamical core (the
double the C code computes, R_dry the single-precision literal
287.052874): with p = 2^e m, m in [1, 2), and F_j = 1 + (2j + 1)/256 the
midpoint of the j-th of 128 mantissa intervals, p**kappa = 2^(kappa e)
F_j**kappa (1 + r)**kappa with r = m / F_j - 1, |r| < 1/256; the first two
factors are tables (e in [-126, 127], j in [0, 128)), the third the
binomial series to r^7 (truncation below 1e-18).
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import struct

getcontext().prec = 60


def dec_to_double(d: Decimal) -> float:
    # correctly rounded conversion through an exact fraction
    f = Fraction(d)
    x = float(f)  # Fraction -> float is correctly rounded
    return x


def dd(d: Decimal):
    hi = dec_to_double(d)
    lo = dec_to_double(d - Decimal(hi))
    return hi, lo


def h(x: float) -> str:
    return float.hex(x)


def truncate_bits(x: float, keep: int) -> float:
    # zero all but the leading `keep` significant bits of x
    b = struct.unpack('<Q', struct.pack('<d', x))[0]
    drop = 52 - (keep - 1)
    b &= ~((1 << drop) - 1)
    return struct.unpack('<d', struct.pack('<Q', b))[0]


def main():
    ln2 = Decimal(2).ln()
    out = []
    out.append('// Generated by gen_math_tables.py; do not edit.')
    out.append('#pragma once')
    # log: reduction points F = i/128 for i in [90, 182], so that every
    # mantissa m in [sqrt(2)/2, sqrt(2)) has |m - F| <= 1/256.
    out.append('#define ATM_LOG_TAB_FIRST 90')
    out.append('#define ATM_LOG_TAB_SIZE 93')
    inv, lhi, llo = [], [], []
    for i in range(90, 183):
        invf = float(Fraction(128, i))  # nearest double to 1/F
        val = -Decimal(invf).ln()       # log(1/invf), exact reduction point
        a, b = dd(val)
        inv.append(invf); lhi.append(a); llo.append(b)
    def arr(name, vals):
        body = ', \\\n  '.join(h(v) for v in vals)
        return '#define %s \\\n  %s' % (name, body)
    out.append(arr('ATM_LOG_INVF_VALUES', inv))
    out.append(arr('ATM_LOG_TAB_HI_VALUES', lhi))
    out.append(arr('ATM_LOG_TAB_LO_VALUES', llo))
    # exp: T_j = 2^(j/32) as double-double
    thi, tlo = [], []
    for j in range(32):
        val = (Decimal(j) / 32 * ln2).exp()
        a, b = dd(val)
        thi.append(a); tlo.append(b)
    out.append(arr('ATM_EXP_TAB_HI_VALUES', thi))
    out.append(arr('ATM_EXP_TAB_LO_VALUES', tlo))
    # ln2 split so that e*LN2_HI is exact for |e| < 2^11
    ln2_hi = truncate_bits(dec_to_double(ln2), 42)
    ln2_lo = dec_to_double(ln2 - Decimal(ln2_hi))
    # ln2/32 split so that N*L1 is exact for |N| < 2^11
    l = ln2 / 32
    l1 = truncate_bits(dec_to_double(l), 42)
    l2 = dec_to_double(l - Decimal(l1))
    inv_l = dec_to_double(32 / ln2)
    out.append('#define ATM_LN2_HI %s' % h(ln2_hi))
    out.append('#define ATM_LN2_LO %s' % h(ln2_lo))
    out.append('#define ATM_EXP_L1 %s' % h(l1))
    out.append('#define ATM_EXP_L2 %s' % h(l2))
    out.append('#define ATM_EXP_INV_L %s' % h(inv_l))
    # Taylor coefficients 1/n! (exp) and (-1)^(n+1)/n (log1p)
    for n in range(2, 10):
        out.append('#define ATM_EXP_C%d %s' % (n, h(dec_to_double(Decimal(1) / Decimal(__import__('math').factorial(n))))))
    for n in range(2, 10):
        v = Decimal((-1) ** (n + 1)) / Decimal(n)
        out.append('#define ATM_LOG_C%d %s' % (n, h(dec_to_double(v))))
    print('\n'.join(out))


def kappa_main():
    r_dry = float(__import__('numpy').float32(287.052874))
    kappa = r_dry / 1005.0  # the double the C code forms
    k = Decimal(kappa)
    ln2 = Decimal(2).ln()
    out = ['// Generated by gen_math_tables.py --kappa; do not edit.', '#pragma once',
           '#define ATM_KAP_E_FIRST (-126)', '#define ATM_KAP_E_LAST 127', '#define ATM_KAP_KAPPA %s' % h(kappa)]

    def arr(name, vals):
        body = ', \\\n  '.join(h(v) for v in vals)
        return '#define %s \\\n  %s' % (name, body)
    out.append(arr('ATM_KAP_E_VALUES', [dec_to_double((k * e * ln2).exp()) for e in range(-126, 128)]))
    fs = [Fraction(256 + 2 * j + 1, 256) for j in range(128)]
    out.append(arr('ATM_KAP_F_VALUES', [dec_to_double((k * (Decimal(f.numerator) / Decimal(f.denominator)).ln()).exp())
                                        for f in fs]))
    out.append(arr('ATM_KAP_INVF_VALUES', [float(1 / f) for f in fs]))
    c = Decimal(1)
    for n in range(1, 8):
        c = c * (k - n + 1) / n  # binomial(kappa, n)
        out.append('#define ATM_KAP_C%d %s' % (n, h(dec_to_double(c))))
    print('\n'.join(out))


if __name__ == '__main__':
    import sys
    if '--kappa' in sys.argv:
        kappa_main()
    else:
        main()
