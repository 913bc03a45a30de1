#!/usr/bin/env python3
"""Generate weno9_tables.cuh: the order-9 WENO tables of the GPU limiter.

The limiter is the reference's WenoLimiter<real,9> (WenoLimiter.h:349-437),
with tables derived here from exact rational arithmetic and rewritten into a
form that needs fewer operations per stencil:

* Everything is expressed in the eight stencil differences d_m = s_{m+1}-s_m.
  Window k (k = 0..4) covers stencil entries k..k+4 and therefore the four
  differences d_k..d_{k+3}.
* Smoothness indicator.  The reference forms the window polynomial's
  coefficients a_1..a_4 (TransformMatrices.h:19841-19880) and evaluates the
  quadratic form TV(a) (TransformMatrices.h:429-433, with the truncation of its
  generator, sage/poly_utils.sage:23-26).  TV is a positive definite quadratic
  form B_k in the window's four differences; with B_k = L D L^T (unit lower L,
  diagonal D > 0, both rational) it becomes
      TV_k = sum_r D_r * y_r^2,   y_r = d_{k+r} + sum_{c>r} L[c][r] d_{k+c}
  which costs 6 multiply-adds for the y's and 4 for the sum, and is a sum of
  non-negative terms (no cancellation in the final sum).
* Edge values.  Each window polynomial's value at the cell's left and right
  edge (WenoLimiter.h:382-426) is s_4 plus a linear form in the window's four
  differences.
* The nine-cell linear edge operator of the weno_all == false path
  (dynamics_rk.h:539-545) is s_4 plus a linear form in all eight differences.

Usage: python gen_weno9.py > weno9_tables.cuh
"""
from fractions import Fraction as Fr
import sys


def integrate_monomial(d, x1, x2):
    return (x2 ** (d + 1) - x1 ** (d + 1)) / (d + 1)


def solve(A, b):
    n = len(A)
    M = [row[:] + [b[i]] for i, row in enumerate(A)]
    for c in range(n):
        piv = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[piv] = M[piv], M[c]
        inv = 1 / M[c][c]
        M[c] = [v * inv for v in M[c]]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c]
                M[r] = [vr - f * vc for vr, vc in zip(M[r], M[c])]
    return [M[r][n] for r in range(n)]


def coef_matrix(offsets):
    """C[d][j]: coefficient a_d of the polynomial whose unit-cell averages at
    the given offsets (target cell = [-1/2,1/2]) are the stencil values."""
    n = len(offsets)
    A = [[integrate_monomial(d, Fr(2 * o - 1, 2), Fr(2 * o + 1, 2)) for d in range(n)] for o in offsets]
    cols = [solve(A, [Fr(int(i == j)) for i in range(n)]) for j in range(n)]
    return [[cols[j][d] for j in range(n)] for d in range(n)]


def poly_mul(p, q):
    r = [Fr(0)] * (len(p) + len(q) - 1)
    for i, a in enumerate(p):
        for j, b in enumerate(q):
            r[i + j] += a * b
    return r


def tv_matrix(n=5):
    """Symmetric Q over coefficients a_0..a_{n-1}: TV(a) = a^T Q a, keeping the
    first n Taylor coefficients of each squared derivative."""
    def tv(c):
        tot = Fr(0)
        p = c[:]
        for _ in range(1, n):
            p = [p[i] * i for i in range(1, len(p))]
            sq = poly_mul(p, p)[:n]
            tot += sum(coef * integrate_monomial(d, Fr(-1, 2), Fr(1, 2)) for d, coef in enumerate(sq))
        return tot
    Q = [[Fr(0)] * n for _ in range(n)]
    for i in range(n):
        for j in range(n):
            a = [Fr(int(m == i)) for m in range(n)]
            b = [Fr(int(m == j)) for m in range(n)]
            s = [x + y for x, y in zip(a, b)]
            Q[i][j] = (tv(s) - tv(a) - tv(b)) / 2
    return Q


def ldl(B):
    n = len(B)
    L = [[Fr(int(i == j)) for j in range(n)] for i in range(n)]
    D = [Fr(0)] * n
    for j in range(n):
        D[j] = B[j][j] - sum(L[j][k] ** 2 * D[k] for k in range(j))
        assert D[j] > 0
        for i in range(j + 1, n):
            L[i][j] = (B[i][j] - sum(L[i][k] * L[j][k] * D[k] for k in range(j))) / D[j]
    return L, D


def lit(v):
    return repr(float(v))


def main():
    w = sys.stdout.write
    Q = tv_matrix(5)
    # Cumulative-difference map: s_{j} - s_0 = sum_{m<j} d_m within a window.
    chol_L, chol_D, lin_l, lin_r = [], [], [], []
    for k in range(5):
        offs = [j - 4 for j in range(k, k + 5)]          # window entries k..k+4, centre entry 4
        C = coef_matrix(offs)
        # a_d (d>=1) as a linear form in the window's differences.
        Cd = [[sum(C[d][j] for j in range(m + 1, 5)) for m in range(4)] for d in range(1, 5)]
        Q4 = [[Q[i][j] for j in range(1, 5)] for i in range(1, 5)]
        B = [[sum(Cd[a][r] * Q4[a][b] * Cd[b][c] for a in range(4) for b in range(4)) for c in range(4)] for r in range(4)]
        L, D = ldl(B)
        chol_L.append(L)
        chol_D.append(D)
        # Edge value minus s_4 as a linear form in the differences.
        for x, store in ((Fr(-1, 2), lin_l), (Fr(1, 2), lin_r)):
            e = [sum(C[d][j] * x ** d for d in range(5)) for j in range(5)]   # weights on entries k..k+4
            assert sum(e) == 1
            centre = 4 - k
            # sum_j e_j (s_j - s_centre) with s_j - s_centre = +-sum of differences
            f = [Fr(0)] * 4
            for j in range(5):
                if j > centre:
                    for m in range(centre, j):
                        f[m] += e[j]
                elif j < centre:
                    for m in range(j, centre):
                        f[m] -= e[j]
            store.append(f)
    # Ideal weights (WenoLimiter.h:383-387, 406-410).
    ideal_l = [Fr(5, 126), Fr(40, 126), Fr(60, 126), Fr(20, 126), Fr(1, 126)]
    ideal_r = ideal_l[::-1]
    # Nine-cell linear operator in differences.
    C9 = coef_matrix(list(range(-4, 5)))
    s2e = []
    for x in (Fr(-1, 2), Fr(1, 2)):
        e = [sum(C9[d][j] * x ** d for d in range(9)) for j in range(9)]
        f = [Fr(0)] * 8
        for j in range(9):
            if j > 4:
                for m in range(4, j):
                    f[m] += e[j]
            elif j < 4:
                for m in range(j, 4):
                    f[m] -= e[j]
        s2e.append(f)
    # Verify the reformulation against the direct forms on random rationals.
    import random
    rnd = random.Random(1)
    for _ in range(20):
        s = [Fr(rnd.randint(-1000, 1000), rnd.randint(1, 50)) for _ in range(9)]
        d = [s[m + 1] - s[m] for m in range(8)]
        for k in range(5):
            C = coef_matrix([j - 4 for j in range(k, k + 5)])
            a = [sum(C[dd][j] * s[k + j] for j in range(5)) for dd in range(5)]
            tv_direct = sum(a[i] * Q[i][j] * a[j] for i in range(5) for j in range(5))
            y = [d[k + r] + sum(chol_L[k][c][r] * d[k + c] for c in range(r + 1, 4)) for r in range(4)]
            assert sum(chol_D[k][r] * y[r] ** 2 for r in range(4)) == tv_direct
            el = sum(a[dd] * Fr(-1, 2) ** dd for dd in range(5))
            assert el == s[4] + sum(lin_l[k][m] * d[k + m] for m in range(4))

    w("// Generated by gen_weno9.py from exact rational arithmetic. Do not edit.\n")
    w("// Order-9 WENO tables in stencil-difference form; see gen_weno9.py.\n")
    w("#pragma once\n\nnamespace pu_weno9 {\n\n")
    w("// TV_k = sum_r D[k][r] * y_r^2,  y_r = d_{k+r} + sum_{c>r} L[k][c][r] d_{k+c}\n")
    w("__device__ constexpr double TV_D[5][4] = {\n")
    for k in range(5):
        w("  {%s},\n" % ", ".join(lit(v) for v in chol_D[k]))
    w("};\n")
    w("__device__ constexpr double TV_L[5][4][4] = {\n")
    for k in range(5):
        w("  {%s},\n" % ", ".join("{%s}" % ", ".join(lit(chol_L[k][c][r]) for r in range(4)) for c in range(4)))
    w("};\n")
    w("// Left / right edge value of window k minus s_4, over d_k..d_{k+3}.\n")
    for nm, tab in (("LIN_L", lin_l), ("LIN_R", lin_r)):
        w("__device__ constexpr double %s[5][4] = {\n" % nm)
        for k in range(5):
            w("  {%s},\n" % ", ".join(lit(v) for v in tab[k]))
        w("};\n")
    w("__device__ constexpr double IDEAL_L[5] = {%s};\n" % ", ".join(lit(v) for v in ideal_l))
    w("__device__ constexpr double IDEAL_R[5] = {%s};\n" % ", ".join(lit(v) for v in ideal_r))
    w("// Nine-cell linear edges minus s_4, over d_0..d_7.\n")
    w("__device__ constexpr double S2E_L[8] = {%s};\n" % ", ".join(lit(v) for v in s2e[0]))
    w("__device__ constexpr double S2E_R[8] = {%s};\n" % ", ".join(lit(v) for v in s2e[1]))
    w("\n}  // namespace pu_weno9\n")


if __name__ == "__main__":
    main()
