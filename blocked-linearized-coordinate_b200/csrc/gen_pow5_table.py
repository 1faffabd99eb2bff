"""Writes pow5_table.h: 128-bit approximations of 5^q for the decimal
parser in tns_parse.cu (run once; the output is committed).

For every q in [Q_MIN, Q_MAX] the table holds T_q, a 128-bit integer with
2^127 <= T_q < 2^128, and e_q such that 5^q ~= T_q * 2^e_q:
  * q >= 0: T_q = floor(5^q / 2^e_q) (exact while 5^q < 2^128);
  * q <  0: T_q = ceil(2^-e_q / 5^-q).
Either way |T_q * 2^e_q - 5^q| < 2^e_q, i.e. T_q is within one unit of its
last bit.  The parser multiplies a normalised 64-bit decimal significand by
T_q exactly (192 bits) and decides the rounding only when that one-unit
error cannot change it.

usage: python gen_pow5_table.py > pow5_table.h
"""
from fractions import Fraction

Q_MIN, Q_MAX = -342, 308


def entry(q):
    v = Fraction(5) ** q
    # e with 2^127 <= v / 2^e < 2^128
    e = v.numerator.bit_length() - v.denominator.bit_length() - 128
    while v / Fraction(2) ** e >= 2 ** 128:
        e += 1
    while v / Fraction(2) ** e < 2 ** 127:
        e -= 1
    x = v / Fraction(2) ** e
    t = x.numerator // x.denominator
    if q < 0 and t * x.denominator != x.numerator:
        t += 1
    assert 2 ** 127 <= t < 2 ** 128 or (q < 0 and t == 2 ** 128)
    if t == 2 ** 128:  # cannot happen for 5^q, kept as a guard
        raise AssertionError(q)
    return t, e


def main():
    print("// Generated by gen_pow5_table.py: T_q (hi, lo 64-bit words) and e_q with")
    print("// 5^q ~= T_q * 2^e_q, 2^127 <= T_q < 2^128, for q in [%d, %d]." % (Q_MIN, Q_MAX))
    print("#pragma once")
    print("#define POW5_QMIN (%d)" % Q_MIN)
    print("#define POW5_QMAX (%d)" % Q_MAX)
    print("#define POW5_COUNT %d" % (Q_MAX - Q_MIN + 1))
    rows, exps = [], []
    for q in range(Q_MIN, Q_MAX + 1):
        t, e = entry(q)
        rows.append("{0x%016xull, 0x%016xull}" % (t >> 64, t & (2 ** 64 - 1)))
        exps.append(str(e))
    print("#define POW5_T_INIT { \\")
    for i in range(0, len(rows), 2):
        print("    " + ", ".join(rows[i:i + 2]) + ", \\")
    print("}")
    print("#define POW5_E_INIT { \\")
    for i in range(0, len(exps), 16):
        print("    " + ", ".join(exps[i:i + 16]) + ", \\")
    print("}")


if __name__ == "__main__":
    main()
