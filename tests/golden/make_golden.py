"""Generate tests/golden/*.npz: overlap integrals and solid harmonics computed
independently of the oracle's recursions, to pin the oracle.

* Cartesian-Gaussian 2- and 3-center overlaps by Gauss-Hermite quadrature of
  the 1-D factors after the Gaussian product theorem (exact for the
  polynomial degrees involved), then placed into the reference's aliased
  block layout: component pair (c1, c2[, c3]) accumulates into the flat block
  index lin = c1 + (2la+1) c2 [+ (2la+1)(2lb+1) c3], read back with the
  shell's own nbf strides (src/integrals/kernels_2c.jl:99-124,
  src/integrals/kernels_3c.jl:134-161).  Component order: for x = l..0,
  for z = 0..l-x: (x, l-x-z, z).
* Real solid harmonics Z_lm (l <= 3, index l^2+l+m) from their explicit
  Cartesian polynomials (standard real-harmonic table, L2-normalised on the
  unit sphere, no Condon-Shortley phase): the convention of SpheriCart
  (Bigi et al., J. Chem. Phys. 159, 064802 (2023)), whose F_l^m and Q_m^m each
  carry a (-1)^m that cancel; tests/helpers.py restates that definition and
  tests/test_oracle.py checks this table against it.

Run from the repo root:  python tests/golden/make_golden.py
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
XG, WG = np.polynomial.hermite.hermgauss(24)


def comps(l):
    return [(x, l - x - z, z) for x in range(l, -1, -1) for z in range(0, l - x + 1)]


def ov1d_2(i, j, a, b, A, B):
    p = a + b
    P = (a * A + b * B) / p
    t = XG / math.sqrt(p)
    f = (t + P - A) ** i * (t + P - B) ** j
    return math.exp(-a * b / p * (A - B) ** 2) * float(np.dot(WG, f)) / math.sqrt(p)


def ov1d_3(i, j, k, a, b, c, A, B, C):
    q = a + b + c
    Q = (a * A + b * B + c * C) / q
    t = XG / math.sqrt(q)
    f = (t + Q - A) ** i * (t + Q - B) ** j * (t + Q - C) ** k
    ex = (a * b * (A - B) ** 2 + a * c * (A - C) ** 2 + b * c * (B - C) ** 2) / q
    return math.exp(-ex) * float(np.dot(WG, f)) / math.sqrt(q)


def block2(sa, sb, A, B):
    (la, ca, za), (lb, cb, zb) = sa, sb
    na, nb = len(comps(la)), len(comps(lb))
    blk = np.zeros(na * nb)
    N1 = 2 * la + 1
    for c1, (x1, y1, z1) in enumerate(comps(la)):
        for c2, (x2, y2, z2) in enumerate(comps(lb)):
            v = 0.0
            for cp, ap in zip(ca, za):
                for cq, aq in zip(cb, zb):
                    v += cp * cq * ov1d_2(x1, x2, ap, aq, A[0], B[0]) * ov1d_2(y1, y2, ap, aq, A[1], B[1]) * \
                        ov1d_2(z1, z2, ap, aq, A[2], B[2])
            blk[c1 + N1 * c2] += v
    return blk.reshape((na, nb), order="F")


def block3(sa, sb, sc, A, B, C):
    (la, ca, za), (lb, cb, zb), (lc, cc, zc) = sa, sb, sc
    na, nb, nc = len(comps(la)), len(comps(lb)), len(comps(lc))
    blk = np.zeros(na * nb * nc)
    N1, N2 = 2 * la + 1, 2 * lb + 1
    for c1, (x1, y1, z1) in enumerate(comps(la)):
        for c2, (x2, y2, z2) in enumerate(comps(lb)):
            for c3, (x3, y3, z3) in enumerate(comps(lc)):
                v = 0.0
                for cp, ap in zip(ca, za):
                    for cq, aq in zip(cb, zb):
                        for cr, ar in zip(cc, zc):
                            v += cp * cq * cr * ov1d_3(x1, x2, x3, ap, aq, ar, A[0], B[0], C[0]) * \
                                ov1d_3(y1, y2, y3, ap, aq, ar, A[1], B[1], C[1]) * \
                                ov1d_3(z1, z2, z3, ap, aq, ar, A[2], B[2], C[2])
                blk[c1 + N1 * c2 + N1 * N2 * c3] += v
    return blk.reshape((na, nb, nc), order="F")


def full2(shells, A, B):
    nbf = [len(comps(s[0])) for s in shells]
    off = np.concatenate([[0], np.cumsum(nbf)])
    N = off[-1]
    S = np.zeros((N, N))
    for a, sa in enumerate(shells):
        for b, sb in enumerate(shells):
            S[off[a]:off[a + 1], off[b]:off[b + 1]] = block2(sa, sb, A, B)
    return S


def full3(shells, A, B, C):
    nbf = [len(comps(s[0])) for s in shells]
    off = np.concatenate([[0], np.cumsum(nbf)])
    N = off[-1]
    V = np.zeros((N, N, N))
    for a, sa in enumerate(shells):
        for b, sb in enumerate(shells):
            for c, sc in enumerate(shells):
                V[off[a]:off[a + 1], off[b]:off[b + 1], off[c]:off[c + 1]] = block3(sa, sb, sc, A, B, C)
    return V


def solid_harmonics_table(x, y, z):
    """Z_lm for l <= 3 from the explicit real-harmonic polynomials."""
    r2 = x * x + y * y + z * z
    pi = math.pi
    Z = [0.5 * math.sqrt(1 / pi)]
    c1 = math.sqrt(3 / (4 * pi))
    Z += [c1 * y, c1 * z, c1 * x]
    Z += [0.5 * math.sqrt(15 / pi) * x * y, 0.5 * math.sqrt(15 / pi) * y * z,
          0.25 * math.sqrt(5 / pi) * (3 * z * z - r2), 0.5 * math.sqrt(15 / pi) * x * z,
          0.25 * math.sqrt(15 / pi) * (x * x - y * y)]
    Z += [0.25 * math.sqrt(35 / (2 * pi)) * y * (3 * x * x - y * y), 0.5 * math.sqrt(105 / pi) * x * y * z,
          0.25 * math.sqrt(21 / (2 * pi)) * y * (5 * z * z - r2), 0.25 * math.sqrt(7 / pi) * z * (5 * z * z - 3 * r2),
          0.25 * math.sqrt(21 / (2 * pi)) * x * (5 * z * z - r2), 0.25 * math.sqrt(105 / pi) * z * (x * x - y * y),
          0.25 * math.sqrt(35 / (2 * pi)) * x * (x * x - 3 * y * y)]
    return np.array(Z)


def main():
    rng = np.random.default_rng(20240601)
    # shells (l, coef, exp): s, s(3 prims), p(2), d(2), f(1)
    shells = [(0, [0.4, 0.7], [3.1, 0.45]), (0, [1.0], [0.21]), (1, [0.7, 0.3], [1.2, 0.4]),
              (2, [0.6, 0.5], [2.0, 0.35]), (3, [1.0], [0.8])]
    geoms = [(np.zeros(3), np.zeros(3)), (np.array([0.1, -0.2, 0.3]), np.array([1.3, 0.4, -0.5])),
             (rng.normal(size=3), rng.normal(size=3) + np.array([2.5, 0, 0]))]
    out2 = np.stack([full2(shells, A, B) for A, B in geoms], axis=-1)
    sh3 = [(0, [0.4, 0.7], [3.1, 0.45]), (1, [0.7, 0.3], [1.2, 0.4]), (2, [1.0], [0.9])]
    g3 = [(np.zeros(3), np.array([1.2, 0, 0]), np.array([0, 1.0, 0])),
          (rng.normal(size=3) * 0.4, rng.normal(size=3) * 0.4 + [1.2, 0, 0], rng.normal(size=3) * 0.4 + [0, 1, 0])]
    out3 = np.stack([full3(sh3, A, B, C) for A, B, C in g3], axis=-1)
    pts = rng.normal(size=(3, 7)) * 1.5
    Z = np.stack([solid_harmonics_table(*pts[:, j]) for j in range(pts.shape[1])], axis=0)

    def pack(sh):
        ls = np.array([s[0] for s in sh], dtype=np.int64)
        nprim = np.array([len(s[1]) for s in sh], dtype=np.int64)
        coef = np.concatenate([np.array(s[1], float) for s in sh])
        alpha = np.concatenate([np.array(s[2], float) for s in sh])
        return ls, nprim, coef, alpha

    ls, nprim, coef, alpha = pack(shells)
    ls3, nprim3, coef3, alpha3 = pack(sh3)
    np.savez(os.path.join(HERE, "overlap_golden.npz"),
             ls=ls, nprim=nprim, coef=coef, alpha=alpha,
             posA=np.stack([g[0] for g in geoms], 1), posB=np.stack([g[1] for g in geoms], 1), S=out2,
             ls3=ls3, nprim3=nprim3, coef3=coef3, alpha3=alpha3,
             posA3=np.stack([g[0] for g in g3], 1), posB3=np.stack([g[1] for g in g3], 1),
             posC3=np.stack([g[2] for g in g3], 1), V=out3,
             pts=pts, Z=Z)
    print("wrote overlap_golden.npz", out2.shape, out3.shape, Z.shape)
    make_f3(pack)


def make_f3(pack):
    """3C with an f shell (every class with l = 3 against s, p and f): overlap3c_f_golden.npz."""
    rng = np.random.default_rng(20241203)
    sh3 = [(0, [0.8], [1.3]), (3, [0.6, 0.5], [1.1, 0.45]), (1, [1.0], [0.7])]
    g3 = [(np.zeros(3), np.array([1.1, 0.2, 0]), np.array([0, 0.9, -0.3])),
          (rng.normal(size=3) * 0.4, rng.normal(size=3) * 0.4 + [1.2, 0, 0], rng.normal(size=3) * 0.4 + [0, 1, 0])]
    out3 = np.stack([full3(sh3, A, B, C) for A, B, C in g3], axis=-1)
    ls3, nprim3, coef3, alpha3 = pack(sh3)
    np.savez(os.path.join(HERE, "overlap3c_f_golden.npz"), ls3=ls3, nprim3=nprim3, coef3=coef3, alpha3=alpha3,
             posA3=np.stack([g[0] for g in g3], 1), posB3=np.stack([g[1] for g in g3], 1),
             posC3=np.stack([g[2] for g in g3], 1), V=out3)
    print("wrote overlap3c_f_golden.npz", out3.shape)


if __name__ == "__main__":
    main()
