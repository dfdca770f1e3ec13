"""Shared helpers for the parity tests (no product code here)."""
import math

import numpy as np
import torch


def rel_fro(x, ref):
    x = np.asarray(x.cpu() if torch.is_tensor(x) else x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((x - ref).ravel()) / (den if den > 0 else 1.0))


def max_abs(x, ref):
    x = np.asarray(x.cpu() if torch.is_tensor(x) else x, dtype=np.float64)
    return float(np.max(np.abs(x - np.asarray(ref, dtype=np.float64)))) if x.size else 0.0


def to_np(t):
    return np.asarray(t.detach().cpu().numpy() if torch.is_tensor(t) else t, dtype=np.float64)


def f32_round(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def sphericart_solid_harmonics(X, L):
    """Real solid harmonics Z (nX, (L+1)^2), index l^2+l+m, as SpheriCart defines them
    (F. Bigi, G. Fraux, N. J. Browning, M. Ceriotti, "Fast evaluation of spherical
    harmonics with sphericart", J. Chem. Phys. 159, 064802 (2023), Sec. II), restated
    factor by factor with both of its sign conventions:

        Z_l^m = F_l^|m| Q_l^|m|(z, r) * { s_|m|(x, y)  m < 0;  1/sqrt(2)  m = 0;  c_m(x, y)  m > 0 }
        F_l^m = (-1)^m sqrt((2l+1)/(2 pi) (l-m)!/(l+m)!)
        Q_m^m = (-1)^m (2m-1)!!,   Q_{m+1}^m = (2m+1) z Q_m^m,
        Q_l^m = ((2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m) / (l-m)
        c_0 = 1, s_0 = 0, c_{m+1} = x c_m - y s_m, s_{m+1} = x s_m + y c_m.

    Q carries the Condon-Shortley phase of the associated Legendre functions and F
    carries a second (-1)^m, so the two cancel: Z_1^{-1} : Z_1^0 : Z_1^1 = y : z : x with
    positive factors.  This is the convention the reference's SolidHarmonics (SpheriCart
    0.3) evaluates; written here independently of the kernels and the oracle."""
    X = np.asarray(X, dtype=np.float64)
    x, y, z = X[0], X[1], X[2]
    r2 = x * x + y * y + z * z
    nX = X.shape[1]
    Z = np.zeros((nX, (L + 1) ** 2))
    c = [np.ones(nX)]
    s = [np.zeros(nX)]
    for m in range(L):
        c.append(x * c[m] - y * s[m])
        s.append(x * s[m] + y * c[m])
    for m in range(L + 1):
        dfac = 1.0
        for k in range(2 * m - 1, 0, -2):
            dfac *= k
        Q = {m: (-1.0) ** m * dfac * np.ones(nX)}
        if m + 1 <= L:
            Q[m + 1] = (2 * m + 1) * z * Q[m]
        for l in range(m + 2, L + 1):
            Q[l] = ((2 * l - 1) * z * Q[l - 1] - (l + m - 1) * r2 * Q[l - 2]) / (l - m)
        for l in range(m, L + 1):
            F = (-1.0) ** m * math.sqrt((2 * l + 1) / (2 * math.pi) * math.factorial(l - m) / math.factorial(l + m))
            if m == 0:
                Z[:, l * l + l] = F * Q[l] / math.sqrt(2.0)
            else:
                Z[:, l * l + l + m] = F * Q[l] * c[m]
                Z[:, l * l + l - m] = F * Q[l] * s[m]
    return Z
