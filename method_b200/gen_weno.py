"""Generates the FP64 WENO point reconstructions of orders 7, 9 and 11.

The Jiang-Shu scheme of order 2r-1 (r = 4, 5, 6) is derived here in exact
rational arithmetic: for each r-cell stencil k of the 2r-1 cells v0..v(2r-2)
the degree r-1 polynomial with those cell averages gives the candidate value
at the right face of the centre cell (v(r-1)) and the smoothness indicator
beta_k = sum_l int_cell (d^l p / dx^l)^2 dx (l = 1..r-1, unit cells) as a
quadratic form in the values; the linear weights d_k are those for which the
weighted candidates equal the (2r-1)-cell reconstruction.  The emitted code
evaluates, like the reconstructions of orders 3 and 5 (weno.cuh), each
indicator term by term from zero in the fixed order (a descending from the
stencil's last cell, b from the last cell down to a: coefficient * v_a * v_b),
alpha_k = d_k / (1e-16 + beta_k^2), weights by division by the alpha sum, and
candidates term by term from the stencil's last cell down; the coefficients
are the doubles nearest the exact rationals, written with 17 significant
digits.

    python -m method_b200.gen_weno          # rewrites csrc/weno_hi.cuh
"""
from __future__ import annotations

import os
from fractions import Fraction as Fr

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "weno_hi.cuh")


def _solve(M, b):
    """Exact Gauss-Jordan solve of M x = b (lists of Fractions); b may be a
    list of vectors (columns), returning the matching solution columns."""
    n = len(M)
    A = [row[:] + [bb[i] for bb in b] for i, row in enumerate(M)]
    m = len(b)
    for c in range(n):
        p = next(r for r in range(c, n) if A[r][c] != 0)
        A[c], A[p] = A[p], A[c]
        inv = 1 / A[c][c]
        A[c] = [x * inv for x in A[c]]
        for r in range(n):
            if r != c and A[r][c] != 0:
                f = A[r][c]
                A[r] = [x - f * y for x, y in zip(A[r], A[c])]
    return [[A[i][n + j] for i in range(n)] for j in range(m)]


def _poly_coeffs(cells):
    """Polynomial coefficients a_n (n < len(cells)) of the reconstruction on
    `cells` (cell j spans [j - 1/2, j + 1/2]) as linear forms in the cell
    values: out[n][q] is the weight of cells[q] in a_n."""
    r = len(cells)
    M = [[((Fr(j) + Fr(1, 2)) ** (n + 1) - (Fr(j) - Fr(1, 2)) ** (n + 1)) / (n + 1)
          for n in range(r)] for j in cells]
    unit = [[Fr(int(i == q)) for i in range(r)] for q in range(r)]
    sols = _solve(M, unit)  # sols[q] = coefficients a_n when v = e_q
    return [[sols[q][n] for q in range(r)] for n in range(r)]


def _value_at(cells, x):
    a = _poly_coeffs(cells)
    return [sum(a[n][q] * Fr(x) ** n for n in range(len(cells))) for q in range(len(cells))]


def _indicator(cells, c):
    """beta as a symmetric matrix over `cells` on the cell c."""
    r = len(cells)
    a = _poly_coeffs(cells)
    Q = [[Fr(0)] * r for _ in range(r)]
    lo, hi = Fr(c) - Fr(1, 2), Fr(c) + Fr(1, 2)
    for l in range(1, r):
        # d^l p / dx^l = sum_n a_n n!/(n-l)! x^(n-l); square, integrate over the cell
        terms = []
        for n in range(l, r):
            f = Fr(1)
            for t in range(n - l + 1, n + 1):
                f *= t
            terms.append((n - l, [f * a[n][q] for q in range(r)]))
        for (e1, w1) in terms:
            for (e2, w2) in terms:
                e = e1 + e2
                integ = (hi ** (e + 1) - lo ** (e + 1)) / (e + 1)
                for q1 in range(r):
                    for q2 in range(r):
                        Q[q1][q2] += integ * w1[q1] * w2[q2]
    return Q


def scheme(r):
    """(indicator terms, candidate terms, linear weights) of order 2r - 1."""
    c = r - 1
    face = Fr(c) + Fr(1, 2)
    betas, cands = [], []
    for k in range(r):
        cells = list(range(k, k + r))
        Q = _indicator(cells, c)
        terms = []
        for ia in range(r - 1, -1, -1):
            for ib in range(r - 1, ia - 1, -1):
                coef = Q[ia][ib] * (1 if ia == ib else 2)
                terms.append((coef, cells[ia], cells[ib]))
        betas.append(terms)
        w = _value_at(cells, face)
        cands.append([(w[q], cells[q]) for q in range(r - 1, -1, -1)])
    big = _value_at(list(range(2 * r - 1)), face)
    # d_k: sum_k d_k w_k(cell) = big(cell) for every cell; least cells determine it
    M = [[Fr(0)] * r for _ in range(2 * r - 1)]
    for k in range(r):
        w = _value_at(list(range(k, k + r)), face)
        for q in range(r):
            M[k + q][k] = w[q]
    d = _solve([M[j] for j in range(r)], [[big[j] for j in range(r)]])[0]
    assert all(sum(M[j][k] * d[k] for k in range(r)) == big[j] for j in range(2 * r - 1))
    return betas, cands, d


def lit(x: Fr) -> str:
    v = float(x)
    s = repr(v)
    return s if ("e" in s or "." in s) else s + ".0"


def emit_function(r, qual="__device__ __forceinline__ double", name=None):
    betas, cands, d = scheme(r)
    n = 2 * r - 1
    name = name or f"weno{n}_exact"
    args = ", ".join(f"double v{q}" for q in range(n))
    L = [f"{qual} {name}({args}) {{", "  const double eps = 1e-16;"]
    for k in range(r):
        L.append(f"  double b{k} = 0, s{k} = 0;")
    for k in range(r):
        for coef, a, b in betas[k]:
            L.append(f"  b{k} += {lit(coef)} * v{a} * v{b};")
        L.append(f"  const double a{k} = {lit(d[k])} / (eps + b{k} * b{k});")
    L.append("  const double asum = " + " + ".join(f"a{k}" for k in range(r)) + ";")
    for k in range(r):
        L.append(f"  const double w{k} = a{k} / asum;")
    for k in range(r):
        for coef, q in cands[k]:
            L.append(f"  s{k} += {lit(coef)} * v{q};")
    L.append("  return (" + " + ".join(f"w{k} * s{k}" for k in range(r)) + ");")
    L.append("}")
    return "\n".join(L)


def indicator_ldl(r, k):
    """beta_k as sum_i D_i z_i^2 with z = L^T dv over the stencil's first
    differences dv_j = v(k+j+1) - v(k+j) (P = L D L^T, L unit lower
    triangular, exact): the form evaluated in FP32 without the cancellation
    of the expanded quadratic form."""
    c = r - 1
    Q = _indicator(list(range(k, k + r)), c)
    m = r - 1
    # v = v_k 1 + T dv, T[q][j] = 1 for j < q; Q annihilates constants
    T = [[Fr(int(j < q)) for j in range(m)] for q in range(r)]
    P = [[sum(T[a][i] * Q[a][b] * T[b][j] for a in range(r) for b in range(r))
          for j in range(m)] for i in range(m)]
    Lm = [[Fr(int(i == j)) for j in range(m)] for i in range(m)]
    Dg = [Fr(0)] * m
    for j in range(m):
        Dg[j] = P[j][j] - sum(Lm[j][t] ** 2 * Dg[t] for t in range(j))
        for i in range(j + 1, m):
            Lm[i][j] = (P[i][j] - sum(Lm[i][t] * Lm[j][t] * Dg[t] for t in range(j))) / Dg[j]
    return Lm, Dg


def emit_fast(r):
    """FP32 form for the mixed-precision flux path: the same weights, FMA
    allowed, indicators from first differences in L D L^T form, one
    approximate reciprocal per indicator and for the sum."""
    betas, cands, d = scheme(r)
    n = 2 * r - 1
    m = r - 1
    args = ", ".join(f"float v{q}" for q in range(n))
    L = [f"__device__ __forceinline__ float weno{n}_fast({args}) {{"]
    for q in range(n - 1):
        L.append(f"  const float d{q} = v{q + 1} - v{q};")
    for k in range(r):
        Lm, Dg = indicator_ldl(r, k)
        zs = []
        for i in range(m):
            terms = [f"d{k + i}"] + [f"{lit(Lm[j][i])}f * d{k + j}" for j in range(i + 1, m)
                                     if Lm[j][i] != 0]
            L.append(f"  const float z{k}_{i} = {' + '.join(terms)};")
            zs.append(f"{lit(Dg[i])}f * z{k}_{i} * z{k}_{i}")
        L.append(f"  const float b{k} = {' + '.join(zs)};")
        L.append(f"  const float a{k} = {lit(d[k])}f * __fdividef(1.0f, 1e-16f + b{k} * b{k});")
    # candidates anchored at the centre cell (in every stencil; the weights
    # sum to one): v_c + sum_q c_q (v_q - v_c), small corrections to v_c
    cc = r - 1
    for q in range(n):
        if q != cc:
            L.append(f"  const float e{q} = v{q} - v{cc};")
    for k in range(r):
        expr = " + ".join(f"{lit(coef)}f * e{q}" for coef, q in cands[k] if q != cc)
        L.append(f"  const float s{k} = v{cc} + ({expr});")
    num = " + ".join(f"a{k} * s{k}" for k in range(r))
    den = " + ".join(f"a{k}" for k in range(r))
    L.append(f"  return ({num}) * __fdividef(1.0f, {den});")
    L.append("}")
    return "\n".join(L)


def header():
    body = "\n\n".join(emit_function(r) for r in (4, 5, 6))
    fast = "\n\n".join(emit_fast(r) for r in (4, 5, 6))
    return ("// Generated by method_b200/gen_weno.py: WENO7, WENO9 and WENO11 upwind point\n"
            "// reconstructions (Jiang-Shu weights derived in exact arithmetic; see that\n"
            "// script).  The FP64 forms are evaluated term by term in a fixed order and,\n"
            "// compiled without FMA contraction, round like the plain C evaluation; the\n"
            "// FP32 forms serve the mixed-precision flux path.\n"
            "#pragma once\n\nnamespace mth {\n\n" + body + "\n\n" + fast +
            "\n\n}  // namespace mth\n")


def oracle_header():
    body = "\n\n".join(emit_function(r, qual="static double", name=f"orc_weno{2 * r - 1}")
                        for r in (4, 5, 6))
    return ("/* Generated by method_b200/gen_weno.py: WENO7, WENO9 and WENO11 upwind point\n"
            " * reconstructions for the C oracle (test infrastructure). */\n" + body + "\n")


ORACLE_OUT = os.path.join(os.path.dirname(HERE), "oracle", "weno_hi.h")

if __name__ == "__main__":
    with open(OUT, "w") as f:
        f.write(header())
    with open(ORACLE_OUT, "w") as f:
        f.write(oracle_header())
    print(f"wrote {OUT} and {ORACLE_OUT}")
