"""Writes afc_roots.cuh: cos / sin of 2 pi e / R for the composite radices of
the nested butterflies (R = 6, 9, 10, 12, 14, 15), as correctly rounded double
literals (Taylor series in 60-digit decimal arithmetic, pi by Machin's formula)
in constexpr switch tables.  Run from this directory: python gen_roots.py"""
from decimal import Decimal, getcontext

RADICES = (6, 9, 10, 12, 14, 15)
getcontext().prec = 60


def _pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239), arctangent series at 60 digits
    def atan_inv(x):
        x = Decimal(x)
        total, term, k, x2 = Decimal(0), 1 / x, 0, x * x
        while True:
            t = term / (2 * k + 1)
            if t == 0 or abs(t) < Decimal(10) ** -70:
                break
            total += t if k % 2 == 0 else -t
            term /= x2
            k += 1
        return total
    return 16 * atan_inv(5) - 4 * atan_inv(239)


PI = _pi()


def _series(x, start):
    # cos (start 0) / sin (start 1) by the Taylor series at 60 digits, rounded once to double
    total, term, k = Decimal(0), Decimal(1), 0
    for i in range(1, start + 1):
        term *= x / i
    n = start
    while abs(term) > Decimal(10) ** -70:
        total += term if k % 2 == 0 else -term
        term *= x * x / ((n + 1) * (n + 2))
        n += 2
        k += 1
    return float(total)


def cos_turn(e, R):
    return _series(2 * PI * e / R, 0)


def sin_turn(e, R):
    return _series(2 * PI * e / R, 1)


def table(R, fn, name):
    lines = [f"  __host__ __device__ __forceinline__ static constexpr double {name}(int e) {{", "    switch (e) {"]
    for e in range(R):
        lines.append(f"      case {e}: return {fn(e, R)!r};")
    lines += ["      default: return 0.0;", "    }", "  }"]
    return lines


out = ["// afc_roots.cuh -- generated by gen_roots.py: cos / sin (2 pi e / R) for the",
       "// composite radices of the nested butterflies.",
       "#pragma once", "", "namespace afc {", "", "template <int R> struct CompRoots;"]
for R in RADICES:
    out.append(f"template <> struct CompRoots<{R}> {{")
    out += table(R, cos_turn, "c")
    out += table(R, sin_turn, "s")
    out.append("};")
out += ["", "}  // namespace afc", ""]
open("afc_roots.cuh", "w").write("\n".join(out))
