"""Generate tests/golden/hexa8_exact.json: closed-form Hexa8 stiffness matrices.

For an affine hexahedron (parallelepiped) the strain-displacement matrix B is a
polynomial of degree <= 1 in each natural coordinate, so K = int B^T D B dV is
a polynomial integral that 2x2x2 Gauss-Legendre quadrature evaluates exactly.
This script integrates it in exact rational arithmetic (fractions.Fraction),
independently of both the oracle and the CUDA code, for
  - the unit cube (E = 1, nu = 3/10) and
  - a sheared, stretched parallelepiped (E = 2, nu = 1/4),
and writes the packed row-wise upper 300 entries (node order and DOF order of
the Hexa8 element: corners (-,-,-),(+,-,-),(+,+,-),(-,+,-),(-,-,+),(+,-,+),
(+,+,+),(-,+,+); DOFs node-major x, y, z). The reference's Gauss point literal
is 0.5773502691896 (13 digits), so its K differs from these exact values by a
relative ~1e-13; tests compare at 1e-12.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
from fractions import Fraction as F

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def padd(p, q, s=F(1)):
    r = dict(p)
    for k, v in q.items():
        r[k] = r.get(k, F(0)) + s * v
    return {k: v for k, v in r.items() if v != 0}


def pmul(p, q):
    r = {}
    for k1, v1 in p.items():
        for k2, v2 in q.items():
            k = (k1[0] + k2[0], k1[1] + k2[1], k1[2] + k2[2])
            r[k] = r.get(k, F(0)) + v1 * v2
    return r


def pscale(p, s):
    return {k: v * s for k, v in p.items() if v * s != 0}


def integrate(p):
    """Exact integral over [-1,1]^3."""
    tot = F(0)
    for (a, b, c), v in p.items():
        if a % 2 or b % 2 or c % 2:
            continue
        tot += v * F(2, a + 1) * F(2, b + 1) * F(2, c + 1)
    return tot


def lin(axis, sign):
    """(1 + sign * xi_axis) as a polynomial."""
    e = [0, 0, 0]
    e[axis] = 1
    return {(0, 0, 0): F(1), tuple(e): F(sign)}


def dN_dxi(corner, axis):
    """d/dxi_axis of N = prod (1 + s_i xi_i) / 8."""
    s = [1 if c else -1 for c in corner]
    p = {(0, 0, 0): F(s[axis], 8)}
    for a in range(3):
        if a != axis:
            p = pmul(p, lin(a, s[a]))
    return p


def inv3(M):
    a, b, c = M[0]
    d, e, f = M[1]
    g, h, i = M[2]
    det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g)
    adj = [[e * i - f * h, c * h - b * i, b * f - c * e],
           [f * g - d * i, a * i - c * g, c * d - a * f],
           [d * h - e * g, b * g - a * h, a * e - b * d]]
    return [[adj[r][k] / det for k in range(3)] for r in range(3)], det


def stiffness(A, E, nu):
    """A: columns are the edge vectors of the parallelepiped (x = x0 + A c, c in [0,1]^3)."""
    J = [[F(A[i][a]) / 2 for i in range(3)] for a in range(3)]  # J[a][i] = dx_i/dxi_a
    Ji, detJ = inv3(J)
    e1 = E / (1 + nu)
    e2 = e1 * nu / (1 - 2 * nu)
    D = [[F(0)] * 6 for _ in range(6)]
    for i in range(3):
        for j in range(3):
            D[i][j] = e1 + e2 if i == j else e2
    for i in range(3, 6):
        D[i][i] = e1 / 2
    # dN_a/dx_i = sum_k Ji[i][k] dN_a/dxi_k
    dx = []
    for cn in CORNERS:
        row = []
        for i in range(3):
            p = {}
            for k in range(3):
                p = padd(p, pscale(dN_dxi(cn, k), Ji[i][k]))
            row.append(p)
        dx.append(row)
    B = [[{} for _ in range(24)] for _ in range(6)]
    for n in range(8):
        bx, by, bz = dx[n]
        B[0][3 * n] = bx
        B[1][3 * n + 1] = by
        B[2][3 * n + 2] = bz
        B[3][3 * n], B[3][3 * n + 1] = by, bx
        B[4][3 * n + 1], B[4][3 * n + 2] = bz, by
        B[5][3 * n], B[5][3 * n + 2] = bz, bx
    K = []
    for i in range(24):
        DB = []
        for k in range(6):
            p = {}
            for l in range(6):
                if D[k][l] != 0 and B[l][i]:
                    p = padd(p, pscale(B[l][i], D[k][l]))
            DB.append(p)
        for j in range(i, 24):
            p = {}
            for k in range(6):
                if B[k][j] and DB[k]:
                    p = padd(p, pmul(B[k][j], DB[k]))
            K.append(integrate(p) * detJ)
    xyz = []
    for cn in CORNERS:
        xyz.append([float(sum(A[i][a] * cn[a] for a in range(3))) for i in range(3)])
    return K, xyz


def main():
    out = {}
    K, xyz = stiffness([[F(1), 0, 0], [0, F(1), 0], [0, 0, F(1)]], F(1), F(3, 10))
    out["unit_cube"] = dict(E=1.0, nu=0.3, xyz=xyz, K300=[float(v) for v in K],
                            K300_exact=[f"{v.numerator}/{v.denominator}" for v in K])
    A = [[F(2), F(1, 2), F(0)], [F(0), F(1), F(1, 4)], [F(0), F(0), F(3, 2)]]
    K2, xyz2 = stiffness(A, F(2), F(1, 4))
    out["parallelepiped"] = dict(E=2.0, nu=0.25, xyz=xyz2, K300=[float(v) for v in K2],
                                 K300_exact=[f"{v.numerator}/{v.denominator}" for v in K2])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hexa8_exact.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
