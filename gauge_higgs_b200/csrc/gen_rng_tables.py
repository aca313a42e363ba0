"""Generate gh_rng_tables.cuh: double-double tables for the correctly rounded
log and cos of gh_rng.cuh (table-driven argument reduction, Tang 1989/1990).

    python gauge_higgs_b200/csrc/gen_rng_tables.py

Every entry is a mathematical constant (log(i/128), cos(j pi/32), sin(j pi/32),
reciprocal factorials, 1/(2k+1)) evaluated with mpmath at 400 bits and split
into hi + lo doubles (hi = nearest double, lo = nearest double to the rest).
"""
import os

from mpmath import mp, mpf, log, cos, sin, pi, factorial

mp.prec = 400
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gh_rng_tables.cuh")


def dd(x):
    hi = float(x)
    lo = float(x - mpf(hi))
    return hi, lo


def fmt(v):
    return repr(v) if v != 0 else "0.0"


def table(name, vals):
    lines = [f"#define {name} \\"]
    body = ", ".join(f"{fmt(h)}, {fmt(l)}" for h, l in vals)
    # wrap
    items = body.split(", ")
    row = []
    out = []
    for it in items:
        row.append(it)
        if len(row) == 4:
            out.append("  " + ", ".join(row) + ", \\")
            row = []
    if row:
        out.append("  " + ", ".join(row) + ", \\")
    out[-1] = out[-1].rstrip(", \\")
    return "\n".join(lines + out) + "\n"


def main():
    log_c = [dd(log(mpf(i) / 128)) for i in range(90, 182)]           # c_i = i/128, i = 90..181
    cs = [dd(cos(j * pi / 32)) for j in range(0, 65)]
    sn = [dd(sin(j * pi / 32)) for j in range(0, 65)]
    odd = [dd(mpf(1) / (2 * k + 1)) for k in range(0, 12)]            # 1/(2k+1)
    cfac = [dd((-1) ** j / factorial(2 * j)) for j in range(0, 12)]   # (-1)^j/(2j)!
    sfac = [dd((-1) ** j / factorial(2 * j + 1)) for j in range(0, 12)]
    pi32 = pi / 32
    p1 = float(pi32)
    p2 = float(pi32 - mpf(p1))
    p3 = float(pi32 - mpf(p1) - mpf(p2))
    ln2 = dd(log(2))
    s = ["// gh_rng_tables.cuh -- generated by gen_rng_tables.py; do not edit.",
         "// Double-double (hi, lo) tables for the correctly rounded log / cos of gh_rng.cuh.",
         "#pragma once",
         "// log(i/128), i = 90..181 (the reduced mantissa range [1/sqrt2, sqrt2))",
         table("GH_TAB_LOGC", log_c),
         "// cos(j pi/32), sin(j pi/32), j = 0..64",
         table("GH_TAB_COS", cs),
         table("GH_TAB_SIN", sn),
         "// 1/(2k+1), (-1)^j/(2j)!, (-1)^j/(2j+1)!, k, j = 0..11",
         table("GH_TAB_ODD", odd),
         table("GH_TAB_CFAC", cfac),
         table("GH_TAB_SFAC", sfac),
         f"#define GH_PI32_1 {fmt(p1)}",
         f"#define GH_PI32_2 {fmt(p2)}",
         f"#define GH_PI32_3 {fmt(p3)}",
         f"#define GH_32_OVER_PI {fmt(float(32 / pi))}",
         f"#define GH_LN2_HI {fmt(ln2[0])}",
         f"#define GH_LN2_LO {fmt(ln2[1])}",
         ""]
    with open(OUT, "w") as f:
        f.write("\n".join(s))
    print(OUT)


if __name__ == "__main__":
    main()
