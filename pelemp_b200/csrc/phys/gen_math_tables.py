"""Generate the tables of the project's table-driven exp and log (pmp_math.h).

exp (Tang, ACM TOMS 15(2), 1989): x = (128 m + j) ln2/128 + r, |r| <= ln2/256,
   exp(x) = 2^m * T[j] * exp(r), T[j] = 2^(j/128) rounded to double.
log (Tang, ACM TOMS 16(4), 1990): x = 2^e m, m in [sqrt(1/2), sqrt(2)),
   c_j = 1 + j/128 with j = trunc((m - 1) * 128) in [-38, 54],
   log(x) = e ln2 + L_j + log1p(m * INV[j] - 1), INV[j] = 1/c_j rounded,
   L_j = -log(INV[j]) stored as hi + lo.
Values come from 60-digit decimal arithmetic.

Run: python gen_math_tables.py  (rewrites pmp_math_tables.h beside this file).
"""
import os
import struct
from decimal import Decimal, getcontext

getcontext().prec = 60

LOG_JMIN = -38
LOG_JMAX = 54


def d2b(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def b2d(b):
    return struct.unpack("<d", struct.pack("<Q", b))[0]


def rn(dec):
    """Round a Decimal to the nearest double."""
    return float(dec)


def main():
    ln2 = Decimal(2).ln()
    exp2 = [rn(Decimal(2) ** (Decimal(j) / 128)) for j in range(128)]
    step = ln2 / 128
    hi = b2d(d2b(rn(step)) & ~((1 << 18) - 1))  # 35 significant bits
    lo = rn(step - Decimal(hi))
    inv, lhi, llo = [], [], []
    for j in range(LOG_JMIN, LOG_JMAX + 1):
        c = Decimal(1) + Decimal(j) / 128
        iv = rn(1 / c)
        L = -Decimal(iv).ln()
        h = rn(L)
        inv.append(iv)
        lhi.append(h)
        llo.append(rn(L - Decimal(h)))

    def arr(v):
        return ",\n  ".join(", ".join(repr(x) for x in v[i:i + 4]) for i in range(0, len(v), 4))

    text = f"""/* Generated by gen_math_tables.py; do not edit by hand.
 * Tables of the table-driven exp and log in pmp_math.h. */
#ifndef PMP_MATH_TABLES_H
#define PMP_MATH_TABLES_H
#define PMP_EXP_N 128
#define PMP_LN2_128_HI {hi!r}
#define PMP_LN2_128_LO {lo!r}
#define PMP_INV_LN2_128 {rn(128 / ln2)!r}
#define PMP_LOG_JMIN ({LOG_JMIN})
#define PMP_LOG_NTAB {LOG_JMAX - LOG_JMIN + 1}
#define PMP_EXP2_TABLE \\
  {{{arr(exp2)}}}
#define PMP_LOG_INV_TABLE \\
  {{{arr(inv)}}}
#define PMP_LOG_LHI_TABLE \\
  {{{arr(lhi)}}}
#define PMP_LOG_LLO_TABLE \\
  {{{arr(llo)}}}
#endif
"""
    text = text.replace(",\n  ", ", \\\n  ")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pmp_math_tables.h")
    with open(out, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main()
