"""Generate khat_classes.h: the value classes of the unit-cube Hexa8 stiffness.

For a cube element with isotropic D = lambda m m^T + mu diag(2,2,2,1,1,1),
K = lambda * K_lambda + mu * K_mu where K_lambda and K_mu are fixed rational
24x24 matrices (exact integrals of the trilinear shape-function gradients,
which 2x2x2 Gauss quadrature reproduces). Entries with the same pair
(K_lambda_ij, K_mu_ij) up to a common sign are equal for every (E, nu, h), so
the whole matrix is determined by a handful of class values. This script
integrates K_lambda and K_mu in exact rational arithmetic, groups the 576
entries into classes, and writes, for every entry, its class index and sign.
The matrix-free lattice operator keeps the class values in registers and
applies each entry as a signed register operand.

Run: python msolve_b200/csrc/gen_khat_classes.py  (writes khat_classes.h beside it)
"""
from __future__ import annotations

import os
from fractions import Fraction as F

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def poly_mul(p, q):
    r = {}
    for a, x in p.items():
        for b, y in q.items():
            k = (a[0] + b[0], a[1] + b[1], a[2] + b[2])
            r[k] = r.get(k, F(0)) + x * y
    return r


def integral(p):
    """Integral over the reference cube [-1,1]^3."""
    s = F(0)
    for (i, j, k), v in p.items():
        if i % 2 == 0 and j % 2 == 0 and k % 2 == 0:
            s += v * F(2, i + 1) * F(2, j + 1) * F(2, k + 1)
    return s


def grad(corner):
    """d N_a / d x_i for the unit cube (x = (xi + 1)/2, so d/dx = 2 d/dxi)."""
    s = [1 if c else -1 for c in corner]
    out = []
    for i in range(3):
        p = {(0, 0, 0): F(2 * s[i], 8)}
        for a in range(3):
            if a != i:
                e = [0, 0, 0]
                e[a] = 1
                p = poly_mul(p, {(0, 0, 0): F(1), tuple(e): F(s[a])})
        out.append(p)
    return out


def main():
    g = [grad(c) for c in CORNERS]
    jac = F(1, 8)  # dV = (1/2)^3 dxi
    Kl = [[F(0)] * 24 for _ in range(24)]
    Km = [[F(0)] * 24 for _ in range(24)]
    for a in range(8):
        for b in range(8):
            for i in range(3):
                for j in range(3):
                    # lambda part: (div u)(div v) -> dNa/dxi * dNb/dxj
                    Kl[3 * a + i][3 * b + j] = integral(poly_mul(g[a][i], g[b][j])) * jac
                    # mu part: 2 eps:eps -> delta_ij grad Na . grad Nb + dNa/dxj dNb/dxi
                    v = integral(poly_mul(g[a][j], g[b][i]))
                    if i == j:
                        for k in range(3):
                            v += integral(poly_mul(g[a][k], g[b][k]))
                    Km[3 * a + i][3 * b + j] = v * jac
    classes = {}
    table = []
    for r in range(24):
        for c in range(24):
            key = (Kl[r][c], Km[r][c])
            if key == (0, 0):
                raise SystemExit("zero entry: not expected for the cube")
            neg = (-key[0], -key[1])
            if key in classes:
                table.append(classes[key] + 1)
            elif neg in classes:
                table.append(-(classes[neg] + 1))
            else:
                classes[key] = len(classes)
                table.append(classes[key] + 1)
    reps = [None] * len(classes)
    for idx, code in enumerate(table):
        if code > 0 and reps[code - 1] is None:
            reps[code - 1] = idx
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "khat_classes.h"), "w") as f:
        f.write("// Generated by gen_khat_classes.py: value classes of the unit-cube Hexa8\n")
        f.write("// stiffness K = lambda K_lambda + mu K_mu (exact rational integration).\n")
        f.write("// kKhatClass[24*row + col] = +(class+1) or -(class+1); kKhatRep[class] is an\n")
        f.write("// entry of that class with positive sign.\n#pragma once\n\n")
        f.write(f"constexpr int kKhatClasses = {len(classes)};\n\n")
        f.write("constexpr signed char kKhatClass[576] = {\n")
        for r in range(24):
            f.write("    " + ", ".join(f"{v:3d}" for v in table[24 * r:24 * r + 24]) + ",\n")
        f.write("};\n\n")
        f.write("constexpr short kKhatRep[kKhatClasses] = {" + ", ".join(str(v) for v in reps) + "};\n")
    print(f"{len(classes)} classes -> khat_classes.h")


if __name__ == "__main__":
    main()
