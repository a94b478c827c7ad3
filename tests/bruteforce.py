"""O(N) brute-force evaluators used by the reference's tests, restated in numpy.

Follows test/interpolation_test_common.jl:31-351 of the reference: support
radius K max(ha, hb) (symmetric) / K ha (gather) / K hb (scatter), inclusion
d2 <= radius^2, kernel weight and gradient averaged over ha and hb in the
symmetric strategy, Shepard-normalised quantities and the error-reduced
gradient / divergence / curl forms.  Test helper only.
"""
import math

import numpy as np

SIG = 1.0 / math.pi
K = 2.0
KERNEL = 0  # 0 M4, 1 M5, 2 M6, 3 C2, 4 C4, 5 C6 (kernel_function/kernels/*.jl)
_SUPPORT = [2.0, 2.5, 3.0, 2.0, 2.0, 2.0]
_NORM3 = [1 / math.pi, 0.05 / math.pi, 1 / (120 * math.pi), 21 / (16 * math.pi), 495 / (256 * math.pi),
          1365 / (512 * math.pi)]


def set_kernel(kid):
    """Kernel family of the evaluators below."""
    global SIG, K, KERNEL
    KERNEL, SIG, K = kid, _NORM3[kid], _SUPPORT[kid]


def f(q):
    q = np.asarray(q, dtype=float)
    if KERNEL == 1:
        a, b, c = 2.5 - q, 1.5 - q, 0.5 - q
        return np.where(q < 0.5, a ** 4 - 5 * b ** 4 + 10 * c ** 4,
                        np.where(q < 1.5, a ** 4 - 5 * b ** 4, np.where(q < 2.5, a ** 4, 0.0)))
    if KERNEL == 2:
        a, b, c = 3 - q, 2 - q, 1 - q
        return np.where(q < 1, a ** 5 - 6 * b ** 5 + 15 * c ** 5,
                        np.where(q < 2, a ** 5 - 6 * b ** 5, np.where(q < 3, a ** 5, 0.0)))
    if KERNEL >= 3:
        a = 1 - 0.5 * q
        poly = {3: 2 * q + 1, 4: 35 / 12 * q ** 2 + 3 * q + 1, 5: 4 * q ** 3 + 6.25 * q ** 2 + 4 * q + 1}[KERNEL]
        return np.where(q < 2, a ** {3: 4, 4: 6, 5: 8}[KERNEL] * poly, 0.0)
    a, b = 2 - q, 1 - q
    return np.where(q < 1, 0.25 * a ** 3 - b ** 3, np.where(q < 2, 0.25 * a ** 3, 0.0))


def df(q):
    q = np.asarray(q, dtype=float)
    if KERNEL == 1:
        a, b, c = 2.5 - q, 1.5 - q, 0.5 - q
        return np.where(q < 0.5, -4 * a ** 3 + 20 * b ** 3 - 40 * c ** 3,
                        np.where(q < 1.5, -4 * a ** 3 + 20 * b ** 3, np.where(q < 2.5, -4 * a ** 3, 0.0)))
    if KERNEL == 2:
        a, b, c = 3 - q, 2 - q, 1 - q
        return np.where(q < 1, -5 * a ** 4 + 30 * b ** 4 - 75 * c ** 4,
                        np.where(q < 2, -5 * a ** 4 + 30 * b ** 4, np.where(q < 3, -5 * a ** 4, 0.0)))
    if KERNEL == 3:
        a = 1 - 0.5 * q
        return np.where(q < 2, 2 * a ** 4 - a ** 3 * (4 * q + 2), 0.0)
    if KERNEL == 4:
        a = 1 - 0.5 * q
        return np.where(q < 2, a ** 6 * (35 / 6 * q + 3) - a ** 5 * (35 / 4 * q ** 2 + 9 * q + 3), 0.0)
    if KERNEL == 5:
        a = 1 - 0.5 * q
        return np.where(q < 2, a ** 8 * (12 * q ** 2 + 12.5 * q + 4) -
                        a ** 7 * (16 * q ** 3 + 25 * q ** 2 + 16 * q + 4), 0.0)
    a, b = 2 - q, 1 - q
    return np.where(q < 1, -0.75 * a ** 2 + 3 * b ** 2, np.where(q < 2, -0.75 * a ** 2, 0.0))


def W(r, h):
    return SIG * f(r / h) / h ** 3


def gradW(d, h):
    """d: (3, n) separations p - x; returns (3, n)."""
    r = np.sqrt(np.sum(d * d, axis=0))
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.where(r > 0, df(r / h) * SIG / (r * h ** 4), 0.0)
    return d * c


def _neighbours(P, p, ha, strategy):
    d = p[:, None] - np.stack([P["x"], P["y"], P["z"]])
    d2 = np.sum(d * d, axis=0)
    hb = P["h"]
    if strategy == "gather":
        rad = K * ha * np.ones_like(hb)
    elif strategy == "scatter":
        rad = K * hb
    else:
        rad = K * np.maximum(ha, hb)
    sel = d2 <= rad * rad
    return sel, d[:, sel], np.sqrt(d2[sel]), hb[sel]


def _weights(d, r, hb, ha, strategy):
    if strategy == "gather":
        return W(r, ha), gradW(d, ha)
    if strategy == "scatter":
        return W(r, hb), gradW(d, hb)
    return 0.5 * (W(r, ha) + W(r, hb)), 0.5 * (gradW(d, ha) + gradW(d, hb))


def nearest_h(P, p):
    d2 = (P["x"] - p[0]) ** 2 + (P["y"] - p[1]) ** 2 + (P["z"] - p[2]) ** 2
    return P["h"][int(np.argmin(d2))]


def general(P, cols, p, ha, strategy, scalars=(), shepard=(), grads=(), divs=(), curls=()):
    """All outputs of one sample in catalog order (0-based column indices)."""
    sel, d, r, hb = _neighbours(P, np.asarray(p, float), ha, strategy)
    L = len(scalars) + 3 * len(grads) + len(divs) + 3 * len(curls)
    if not sel.any():
        return [math.nan] * L
    Wv, G = _weights(d, r, hb, ha, strategy)
    m, rho = P["m"][sel], P["rho"][sel]
    w = m * Wv / rho
    g = (m / rho) * G
    S1 = w.sum()
    if S1 == 0:
        return [math.nan] * L
    out = []
    for c, sh in zip(scalars, shepard):
        A = cols[c][sel]
        v = np.sum(A * w)
        out.append(v / S1 if sh else v)
    for c in grads:
        if c < 0:  # gradient of the particle density (catalog grad slot 0)
            f_ = np.sum(m * G, axis=1)
            A = np.sum(m * Wv) / S1
        else:
            Acol = cols[c][sel]
            f_ = np.sum(Acol * g, axis=1)
            A = np.sum(Acol * w) / S1
        out.extend(list(f_ - A * g.sum(axis=1)))
    for cx, cy, cz in divs:
        Av = np.stack([cols[cx][sel], cols[cy][sel], cols[cz][sel]])
        f_ = np.sum(Av * g)
        At = np.sum(Av * w, axis=1) / S1
        out.append(f_ - np.dot(At, g.sum(axis=1)))
    for cx, cy, cz in curls:
        Av = np.stack([cols[cx][sel], cols[cy][sel], cols[cz][sel]])
        f_ = np.sum(np.cross(Av.T, g.T), axis=0)
        At = np.sum(Av * w, axis=1) / S1
        b = np.cross(At, g.sum(axis=1))
        out.extend(list(-(f_ - b)))
    return out


def line_quantities(P, cols, o, m_dir, ha, strategy, scalars, shepard, table):
    """Line-integrated scalars (line_integrated_scalar_interpolation.jl:76-214)."""
    Q, I = table
    X = np.stack([P["x"], P["y"], P["z"]])
    D = X - np.asarray(o, float)[:, None]
    Dm = np.sum(D * np.asarray(m_dir, float)[:, None], axis=0)
    d2 = np.sum(D * D, axis=0) - Dm * Dm
    hb = P["h"]
    rad = {"gather": K * ha * np.ones_like(hb), "scatter": K * hb, "symmetric": K * np.maximum(ha, hb)}[strategy]
    sel = d2 <= rad * rad
    if not sel.any():
        return [math.nan] * len(scalars)
    dr = np.sqrt(np.maximum(d2[sel], 0))

    def lk(r, h):
        q = r / h
        dq = Q[1] - Q[0]
        idxf = q / dq + 1
        i = np.clip(np.trunc(idxf).astype(int), 1, len(Q) - 1)
        t = idxf - i
        v = I[i - 1] * (1 - t) + I[i] * t
        return np.where(q >= K, 0.0, v) / h

    hbs = hb[sel]
    Wv = {"gather": lambda: lk(dr, ha), "scatter": lambda: lk(dr, hbs),
          "symmetric": lambda: 0.5 * (lk(dr, ha) + lk(dr, hbs))}[strategy]()
    w = P["m"][sel] * Wv / P["rho"][sel]
    S1 = w.sum()
    if S1 == 0:
        return [math.nan] * len(scalars)
    return [np.sum(cols[c][sel] * w) / S1 if sh else np.sum(cols[c][sel] * w) for c, sh in zip(scalars, shepard)]
