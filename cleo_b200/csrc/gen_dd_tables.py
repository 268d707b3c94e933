"""Generate dd_tables.h: double-double tables for the accurate pow/exp of ddmath.h.

    python cleo_b200/csrc/gen_dd_tables.py > cleo_b200/csrc/dd_tables.h

Values are computed with Python's decimal module at 80 significant digits and split into
(hi, lo) doubles with hi = round(v), lo = round(v - hi).
"""
from decimal import Decimal, getcontext

getcontext().prec = 80


def split(v: Decimal):
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def main():
    ln2 = Decimal(2).ln()
    out = ["// Generated by gen_dd_tables.py: double-double constants (hi, lo) for ddmath.h.",
           "// Included once per target (host / device) inside a namespace, so no include guard.", ""]
    hi, lo = split(ln2)
    out.append(f"#define CLEO_DD_LN2_HI {hi.hex()}")
    out.append(f"#define CLEO_DD_LN2_LO {lo.hex()}")
    hi, lo = split(1 / ln2)
    out.append(f"#define CLEO_DD_INV_LN2 {hi.hex()}")
    out.append("")
    # 2^(j/64), j = -32..32
    out.append("// 2^(j/64) for j = -32..32")
    out.append("CLEO_DD_TABLE double cleo_dd_exp2_tab[65][2] = {")
    for j in range(-32, 33):
        v = Decimal(2) ** (Decimal(j) / 64)
        hi, lo = split(v)
        out.append(f"  {{{hi.hex()}, {lo.hex()}}},")
    out.append("};")
    # log(1 + k/64), k = -20..28 (mantissa reduced to [sqrt(1/2), sqrt(2)))
    out.append("// ln(1 + k/64) for k = -20..28")
    out.append("CLEO_DD_TABLE double cleo_dd_log_tab[49][2] = {")
    for k in range(-20, 29):
        v = (1 + Decimal(k) / 64).ln()
        hi, lo = split(v)
        out.append(f"  {{{hi.hex()}, {lo.hex()}}},")
    out.append("};")
    # fast first phase of log: centres c = i/512 of the reduced mantissa (i = 362..724), the
    # double rc = RN(1/c) and -ln(rc) exactly for that double, as (rc, hi, lo)
    out.append("// fast log: rc = RN(512/i) and -ln(rc) as double-double, i = 362..724")
    out.append("CLEO_DD_TABLE double cleo_fast_log_tab[363][3] = {")
    for i in range(362, 725):
        rc = float(Decimal(512) / Decimal(i))
        v = -Decimal(rc).ln()
        hi, lo = split(v)
        out.append(f"  {{{rc.hex()}, {hi.hex()}, {lo.hex()}}},")
    out.append("};")
    # fast first phase of exp: 2^(j/512), j = 0..511
    out.append("// fast exp: 2^(j/512) for j = 0..511")
    out.append("CLEO_DD_TABLE double cleo_fast_exp2_tab[512][2] = {")
    for j in range(512):
        v = Decimal(2) ** (Decimal(j) / 512)
        hi, lo = split(v)
        out.append(f"  {{{hi.hex()}, {lo.hex()}}},")
    out.append("};")
    # series coefficients needed in double-double
    for name, v in (("THIRD", Decimal(1) / 3), ("FIFTH", Decimal(1) / 5), ("SEVENTH", Decimal(1) / 7),
                    ("INV6", Decimal(1) / 6), ("INV24", Decimal(1) / 24), ("INV120", Decimal(1) / 120)):
        hi, lo = split(v)
        out.append(f"#define CLEO_DD_{name}_HI {hi.hex()}")
        out.append(f"#define CLEO_DD_{name}_LO {lo.hex()}")
    print("\n".join(out))


if __name__ == "__main__":
    main()
