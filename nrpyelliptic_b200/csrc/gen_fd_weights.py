"""Generate fd_weights.h: exact first-derivative finite-difference weights.

The radiation boundary condition of NRPyElliptic differentiates with an
11-point (10th-order) first-derivative stencil whose centre is shifted by an
"upwind offset" k in [-5, 5] so that it never leaves the grid (reference:
NRPyElliptic_Ccodes/apply_bcs_outerradiation_and_inner.c:6-286).  For offset
k the stencil covers the nodes j = k-5 .. k+5 relative to the evaluation
point.  The weights are unique; they are computed here with Fornberg's
recursion (B. Fornberg, Math. Comp. 51 (1988) 699) in exact rational
arithmetic and written out as p/q literals, so the compiled constants are the
correctly rounded doubles of the exact weights.

Run:  python gen_fd_weights.py > fd_weights.h
"""
from fractions import Fraction


def fornberg(nodes, x0, max_order):
    """Return c[m][j]: weight of nodes[j] for the m-th derivative at x0."""
    n = len(nodes)
    c = [[Fraction(0)] * n for _ in range(max_order + 1)]
    c[0][0] = Fraction(1)
    c1 = Fraction(1)
    c4 = nodes[0] - x0
    for i in range(1, n):
        mn = min(i, max_order)
        c2 = Fraction(1)
        c5 = c4
        c4 = nodes[i] - x0
        for j in range(i):
            c3 = nodes[i] - nodes[j]
            c2 *= c3
            if j == i - 1:
                for m in range(mn, 0, -1):
                    c[m][i] = c1 * (m * c[m - 1][i - 1] - c5 * c[m][i - 1]) / c2
                c[0][i] = -c1 * c5 * c[0][i - 1] / c2
            for m in range(mn, 0, -1):
                c[m][j] = (c4 * c[m][j] - m * c[m - 1][j]) / c3
            c[0][j] = c4 * c[0][j] / c3
        c1 = c2
    return c


def main():
    out = []
    out.append("/* Generated by gen_fd_weights.py -- exact 11-point first-derivative weights.")
    out.append(" * NRPYELL_FD1_UPWIND[k+5][j] is the weight of node (k-5+j) for upwind offset k. */")
    out.append("#ifndef NRPYELL_FD_WEIGHTS_H")
    out.append("#define NRPYELL_FD_WEIGHTS_H")
    out.append("#define NRPYELL_FD1_UPWIND_INIT { \\")
    for k in range(-5, 6):
        nodes = [Fraction(j) for j in range(k - 5, k + 6)]
        w = fornberg(nodes, Fraction(0), 1)[1]
        terms = []
        for f in w:
            terms.append("(%d.0/%d.0)" % (f.numerator, f.denominator))
        out.append("  { " + ", ".join(terms) + " }%s \\" % ("," if k < 5 else ""))
    out.append("}")
    out.append("#endif")
    print("\n".join(out))


if __name__ == "__main__":
    main()
