"""Print the constants of sin_rn.cuh from exact rational arithmetic.

pi comes from Machin's formula (pi/4 = 4 atan(1/5) - atan(1/239)) summed as
exact fractions; the Taylor coefficients (-1)^k / n! are exact fractions.  Each
constant is split into doubles, every part the nearest double to what the
previous parts leave, and printed as a C hex-float literal.
"""
from fractions import Fraction
from math import factorial


def atan_inv(n, terms=120):
    # atan(1/n) = sum (-1)^k / ((2k+1) n^(2k+1))
    return sum(Fraction((-1) ** k, (2 * k + 1) * n ** (2 * k + 1)) for k in range(terms))


def split(v, parts):
    out = []
    for _ in range(parts):
        d = float(v)
        out.append(d)
        v -= Fraction(d)
    return out


def main():
    pi = 4 * (4 * atan_inv(5) - atan_inv(239))
    p1, p2, p3 = split(pi / 2, 3)
    print(f"PIO2 = {p1.hex()}, {p2.hex()}, {p3.hex()}")
    print(f"TWO_OVER_PI = {float(2 / pi).hex()}")
    # sin(r) = r + r^3 sum_k a_k r^(2k), a_k = (-1)^(k+1) / (2k+3)!
    for k in range(10):
        hi, lo = split(Fraction((-1) ** (k + 1), factorial(2 * k + 3)), 2)
        print(f"a{k} = {hi.hex()}, {lo.hex()}")
    # cos(r) = 1 + r^2 sum_k b_k r^(2k), b_k = (-1)^(k+1) / (2k+2)!
    for k in range(11):
        hi, lo = split(Fraction((-1) ** (k + 1), factorial(2 * k + 2)), 2)
        print(f"b{k} = {hi.hex()}, {lo.hex()}")


if __name__ == "__main__":
    main()
