"""Generate crexp_tables.h: the constants of the correctly rounded exp in
crexp.cuh, computed with Python's decimal module at 80 significant digits.

    python bb_pd_b200/csrc/gen_crexp_tables.py > bb_pd_b200/csrc/crexp_tables.h

Tables (N = 256 points per octave):
  T[j] = 2^(j/256) as a double-double (hi, lo) and as a 128-bit fixed-point
         number with 126 fractional bits (for the accurate step);
  ln2/256 in three doubles (the first with 32 significant bits, so that m * it
         is exact for |m| < 2^21) and as a 192-bit fixed-point number with 145
         fractional bits;
  1/i! for the polynomials: doubles, double-doubles for 1/6 and 1/24, and
         128-bit fixed-point numbers with 125 fractional bits for i = 0..10.
"""
from decimal import Decimal, getcontext, ROUND_HALF_EVEN, ROUND_FLOOR
import math

getcontext().prec = 80
N = 256
LN2 = Decimal(2).ln()


def dbl(v: Decimal) -> float:
    """The double nearest to v (float() of a decimal string rounds correctly)."""
    return float(str(v))


def dd(v: Decimal):
    h = dbl(v)
    return h, dbl(v - Decimal(h))


def hexf(x: float) -> str:
    return "0.0" if x == 0.0 else float.hex(x)


def fixed(v: Decimal, frac_bits: int) -> int:
    return int((v * (Decimal(2) ** frac_bits)).to_integral_value(rounding=ROUND_HALF_EVEN))


def top_bits(v: Decimal, bits: int) -> float:
    """v truncated to `bits` significant bits (a double)."""
    e = math.floor(math.log2(abs(float(v))))
    scale = Decimal(2) ** (bits - 1 - e)
    t = (v * scale).to_integral_value(rounding=ROUND_FLOOR) / scale
    f = float(str(t))
    assert Decimal(f) == t
    return f


def main():
    out = []
    w = out.append
    w("// Generated by gen_crexp_tables.py (decimal arithmetic, 80 digits). Do not edit.")
    w("#pragma once")
    w("#include <cstdint>")
    w("namespace bbpd {")
    w("namespace crexp_tab {")
    w(f"constexpr double INV_LN2_N = {hexf(dbl(N / LN2))};   // 256 / ln 2")
    c = LN2 / N
    l1 = top_bits(c, 32)
    l2 = dbl(c - Decimal(l1))
    l3 = dbl(c - Decimal(l1) - Decimal(l2))
    w(f"constexpr double LN2_N_1 = {hexf(l1)};   // ln2/256, first 32 bits")
    w(f"constexpr double LN2_N_2 = {hexf(l2)};")
    w(f"constexpr double LN2_N_3 = {hexf(l3)};")
    c145 = fixed(c, 145)
    assert c145 < 2 ** 192
    m64 = 2 ** 64 - 1
    w("// ln2/256 * 2^145 in three 64-bit limbs, most significant first")
    w(f"constexpr uint64_t LN2_N_FX2 = 0x{c145 >> 128:016x}ull, LN2_N_FX1 = 0x{(c145 >> 64) & m64:016x}ull, "
      f"LN2_N_FX0 = 0x{c145 & m64:016x}ull;")
    for i in (5, 6, 7, 8):
        w(f"constexpr double C{i} = {hexf(dbl(Decimal(1) / math.factorial(i)))};   // 1/{i}!")
    for i in (3, 4):
        h, lo = dd(Decimal(1) / math.factorial(i))
        w(f"constexpr double C{i}H = {hexf(h)}, C{i}L = {hexf(lo)};   // 1/{i}! as a double-double")
    w("}  // namespace crexp_tab")
    w("}  // namespace bbpd")
    w("// Array initialisers (crexp.cuh instantiates them in device and host memory).")
    w("// 2^125 / i!, i = 0..10, as (high, low) 64-bit halves of a 128-bit number")
    w("#define BBPD_CREXP_FACT_FX { \\")
    for i in range(11):
        v = fixed(Decimal(1) / math.factorial(i), 125)
        assert v < 2 ** 127
        w(f"    {{0x{v >> 64:016x}ull, 0x{v & m64:016x}ull}}, \\")
    w("}")
    w("// 2^(j/256): double-double (hi, lo)")
    w("#define BBPD_CREXP_T_DD { \\")
    for j in range(N):
        h, lo = dd((LN2 * j / N).exp())
        w(f"    {{{hexf(h)}, {hexf(lo)}}}, \\")
    w("}")
    w("// 2^(j/256) * 2^126 as (high, low) 64-bit halves")
    w("#define BBPD_CREXP_T_FX { \\")
    for j in range(N):
        v = fixed((LN2 * j / N).exp(), 126)
        assert 2 ** 126 <= v < 2 ** 127
        w(f"    {{0x{v >> 64:016x}ull, 0x{v & m64:016x}ull}}, \\")
    w("}")
    print("\n".join(out))


if __name__ == "__main__":
    main()
