"""Writes exp_table.h: 2^(j/64), j = 0..63, as double hi parts and the
double nearest the remainder (lo), and ln2/64 split in two doubles, from
50-digit decimal arithmetic, for the table-driven exponential of the
batched solver (fast_math.cuh)."""
import decimal
import os
import sys

decimal.getcontext().prec = 50
D = decimal.Decimal
N = 64
LN2 = D(2).ln()


def nearest(d):
    """the double nearest the decimal d"""
    return float(d)   # Decimal -> float rounds correctly


def remainder(d, h):
    return float(d - D(h))


vals = [(LN2 * j / N).exp() for j in range(N)]
hi = [nearest(v) for v in vals]
lo = [remainder(v, h) for v, h in zip(vals, hi)]
q = LN2 / N
l1 = float(int(q * D(2) ** 32 + D("0.5")) / D(2) ** 32)          # low mantissa bits zero: n * l1 exact
l2 = float(q - D(l1))
inv = float(D(N) / LN2)
out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "exp_table.h")
with open(out, "w") as f:
    f.write("// exp_table.h -- generated by gen_exp_table.py (50-digit decimal arithmetic):\n")
    f.write("// 2^(j/64) for j = 0..63 as hi (the double nearest) + lo (the double nearest\n")
    f.write("// the remainder), and ln2/64 and 64/ln2 for the argument reduction.\n#pragma once\n\n")
    f.write("namespace cyc {\n\n")
    f.write("__device__ const double kExp2Hi[64] = {\n")
    for i in range(0, N, 4):
        f.write("    " + ", ".join(h.hex() for h in hi[i:i + 4]) + ",\n")
    f.write("};\n__device__ const double kExp2Lo[64] = {\n")
    for i in range(0, N, 4):
        f.write("    " + ", ".join(x.hex() for x in lo[i:i + 4]) + ",\n")
    f.write("};\n\n")
    f.write("// ln2/64 = kLn2By64Hi + kLn2By64Lo (the high part's low 32 mantissa bits are\n")
    f.write("// zero, so n * kLn2By64Hi is exact for |n| < 2^20), and 64/ln2\n")
    f.write(f"constexpr double kLn2By64Hi = {l1.hex()};\n")
    f.write(f"constexpr double kLn2By64Lo = {l2.hex()};\n")
    f.write(f"constexpr double kInvLn2By64 = {inv.hex()};\n\n")
    f.write("}  // namespace cyc\n")
print(out)
