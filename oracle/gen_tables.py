#!/usr/bin/env python3
"""Derive the order-9 WENO tables of the oracle from exact rational arithmetic.

This is test infrastructure: the tables feed only the CPU oracle
(``oracle/dycore_oracle.cpp``).  The product kernels derive their own tables
(``porturb_b200/csrc/gen_weno9.py``).

The mathematics follows the reference's coefficient generator
(model/modules/helpers/sage/transformation_matrices.sage):

* ``stencil_to_coefs`` (:19-27): a degree-4 polynomial p(x)=sum a_d x^d whose
  averages over five unit cells equal the five stencil values.  The target
  cell is x in [-1/2, 1/2]; window ``M`` (1..5) covers stencil entries
  M-1..M+3 of a 9-point stencil whose centre is entry 4
  (TransformMatrices.h:19841-19880, ``coefs5_shift1..5``).
* ``coefs_to_TV`` (:140-146): TV = sum_{d=1..4} int_{-1/2}^{1/2} (p^(d))^2 dx,
  where ``integrate_poly`` (poly_utils.sage:23-26) keeps only the first N=5
  Taylor coefficients of the squared derivative.  That truncation drops the
  x^6 term of (p')^2, which is why the a4^2 weight is 625.8 and not
  625.8357 (TransformMatrices.h:429-433).
* edge values p(-1/2) (left, ``gll_1``) and p(+1/2) (right, ``gll_2``)
  (WenoLimiter.h:382-426), and the ideal (linear) weights that make the
  weighted sub-stencil edge values equal the degree-8 nine-cell polynomial's
  edge value (WenoLimiter.h:383-387, 406-410).
* the nine-cell linear edge operator ``s2e`` used when ``weno_all`` is false
  (dynamics_rk.h:539-545).

Every linear form is emitted as a left-to-right sum of products in stencil
order with zero terms omitted, which is the evaluation order of the
reference's generated code; the REF variant of the oracle relies on this to
be bit-identical to the reference when both are built by the same compiler.

Usage: python oracle/gen_tables.py > oracle/weno9_tables.h
"""
from fractions import Fraction as Fr
import sys


def poly_mul(p, q):
    r = [Fr(0)] * (len(p) + len(q) - 1)
    for i, a in enumerate(p):
        for j, b in enumerate(q):
            r[i + j] += a * b
    return r


def poly_deriv(p):
    return [p[i] * i for i in range(1, len(p))] or [Fr(0)]


def integrate_monomial(d, x1, x2):
    return (x2 ** (d + 1) - x1 ** (d + 1)) / (d + 1)


def solve(A, b):
    """Exact Gauss-Jordan solve of the square system A x = b (lists of Fractions)."""
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


def inverse(A):
    n = len(A)
    cols = [solve(A, [Fr(int(i == j)) for i in range(n)]) for j in range(n)]
    return [[cols[j][i] for j in range(n)] for i in range(n)]


def stencil_to_coefs(offsets):
    """Matrix C with a = C s: polynomial coefficients from cell averages at the
    given integer cell offsets relative to the target cell [-1/2, 1/2]."""
    n = len(offsets)
    A = [[integrate_monomial(d, Fr(2 * o - 1, 2), Fr(2 * o + 1, 2)) for d in range(n)] for o in offsets]
    return inverse(A)  # rows: coefficient d, cols: stencil entry


def tv_quadratic_form(n=5):
    """TV as {(i,j): weight} over coefficient pairs, with the reference's
    truncation of each squared derivative to degree n-1."""
    form = {}
    for i in range(n):
        for j in range(i, n):
            a = [Fr(0)] * n
            b = [Fr(0)] * n
            a[i] = Fr(1)
            b[j] = Fr(1)
            # TV is bilinear: evaluate the cross term through polarisation.
            def tv(c):
                tot = Fr(0)
                p = c[:]
                for _ in range(1, n):
                    p = poly_deriv(p)
                    sq = poly_mul(p, p)[:n]  # integrate_poly keeps n coefficients
                    tot += sum(coef * integrate_monomial(d, Fr(-1, 2), Fr(1, 2)) for d, coef in enumerate(sq))
                return tot
            if i == j:
                w = tv(a)
            else:
                s = [x + y for x, y in zip(a, b)]
                w = tv(s) - tv(a) - tv(b)
            if w != 0:
                form[(i, j)] = w
    return form


def edge_rows(C, x):
    n = len(C)
    return [sum(C[d][k] * x ** d for d in range(n)) for k in range(len(C[0]))]


def lit(v):
    return repr(float(v))


def linear_expr(coefs, names):
    terms = []
    for c, nm in zip(coefs, names):
        if c == 0:
            continue
        terms.append("T(%s)*%s" % (lit(c), nm))
    return " + ".join(terms) if terms else "T(0)"


def main():
    out = sys.stdout
    w = out.write
    # Sub-stencil windows of the order-9 limiter.
    windows = []
    for M in range(1, 6):
        offs = [o - 4 for o in range(M - 1, M + 4)]
        windows.append((M, offs, stencil_to_coefs(offs)))
    form = tv_quadratic_form(5)
    # Full nine-cell polynomial for the ideal weights and the linear path.
    C9 = stencil_to_coefs(list(range(-4, 5)))
    P9L = edge_rows(C9, Fr(-1, 2))
    P9R = edge_rows(C9, Fr(1, 2))
    EL = [edge_rows(C, Fr(-1, 2)) for _, _, C in windows]
    ER = [edge_rows(C, Fr(1, 2)) for _, _, C in windows]

    def ideal(E, P):
        # sum_M d_M * E_M(s) = P(s) for all 9-point s; window M touches entries M-1..M+3.
        rows = []
        rhs = []
        for col in range(9):
            rows.append([E[M][col - M] if 0 <= col - M < 5 else Fr(0) for M in range(5)])
            rhs.append(P[col])
        d = solve(rows[:5], rhs[:5])
        for r, v in zip(rows, rhs):
            assert sum(a * b for a, b in zip(r, d)) == v
        return d

    DL = ideal(EL, P9L)
    DR = ideal(ER, P9R)
    assert DL == [Fr(5, 126), Fr(40, 126), Fr(60, 126), Fr(20, 126), Fr(1, 126)]
    assert DR == DL[::-1]

    w("// Generated by oracle/gen_tables.py from exact rational arithmetic. Do not edit.\n")
    w("// Oracle-only tables for the order-9 WENO limiter (test infrastructure).\n")
    w("#pragma once\n\nnamespace orc_tables {\n\n")
    # Window coefficient functions a1..a4 (a0 is never used by the limiter).
    for M, offs, C in windows:
        w("template <class T> inline void coefs_win%d(T s0, T s1, T s2, T s3, T s4, T *a) {\n" % M)
        for d in range(1, 5):
            w("  a[%d] = %s;\n" % (d, linear_expr(C[d], ["s0", "s1", "s2", "s3", "s4"])))
        w("}\n\n")
    # TV with the reference's term order: (1,1),(2,2),(1,3),(3,3),(2,4),(4,4).
    order = [(1, 1), (2, 2), (1, 3), (3, 3), (2, 4), (4, 4)]
    assert set(order) == set(form.keys()), form
    w("// TV quadratic form weights, term order (1,1),(2,2),(1,3),(3,3),(2,4),(4,4).\n")
    w("static const double TVW[6] = {%s};\n\n" % ", ".join(lit(form[o]) for o in order))
    names = ["s%d" % i for i in range(9)]
    for tag, E, D in (("left", EL, DL), ("right", ER, DR)):
        w("// Ideal weights for the %s edge.\n" % tag)
        w("static const double IDEAL_%s[5] = {%s};\n" % (tag.upper(), ", ".join(lit(v) for v in D)))
        for M in range(5):
            w("template <class T> inline T edge_%s_win%d(const T *s) {\n" % (tag, M + 1))
            w("  return %s;\n}\n" % linear_expr(E[M], ["s[%d]" % (M + c) for c in range(5)]))
        w("\n")
    w("// Nine-cell linear edge operator (weno_all == false path).\n")
    w("static const double S2E_LEFT[9] = {%s};\n" % ", ".join(lit(v) for v in P9L))
    w("static const double S2E_RIGHT[9] = {%s};\n" % ", ".join(lit(v) for v in P9R))
    w("// sten_to_coefs for the nine-cell stencil, indexed (stencil entry, coefficient)\n")
    w("// like TransformMatrices::sten_to_coefs(SArray<FP,2,9,9>).\n")
    w("static const double STEN_TO_COEFS9[9][9] = {\n")
    for j in range(9):
        w("  {%s},\n" % ", ".join(lit(C9[dd][j]) for dd in range(9)))
    w("};\n")
    w("\n}  // namespace orc_tables\n")


if __name__ == "__main__":
    main()
