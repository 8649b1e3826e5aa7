"""CPU restatement of the learned subgrid closure -- test infrastructure only.

The closure has no counterpart in the reference (theparvezahmad/compChan3Dmpi
resolves every scale); this module restates, in numpy and float64, what the
library's closure kernels compute, so the tests can check them:

* ``sample``: the Favre box filter of width fw in x and spanwise, the 13
  features (velocity and temperature gradients at the sample strides, y+)
  and the 9 subgrid fluxes, from a primitive field var[7, nP3, nP2, nP1]
  (rho, u, v, w, E, T, p) as chan_download returns it;
* ``forward`` / ``grad``: the 13 -> 64 -> 64 -> 9 MLP (tanh-form GELU) with the BF16
  rounding the tensor-core path applies (inputs, hidden activations, output
  and hidden gradients rounded to BF16 before each product; products and
  sums exact here, F32 on the device);
* ``adam``: one Adam step;
* ``source``: the closure source -d tau_ab/dx_b, -gama d q_b/dx_b at the
  interior points from the MLP outputs.
"""
from __future__ import annotations

import math

import numpy as np

N_IN, N_HID, N_OUT = 13, 64, 9
OFF_W1, OFF_B1 = 0, 64 * 13
OFF_W2 = OFF_B1 + 64
OFF_B2 = OFF_W2 + 64 * 64
OFF_W3 = OFF_B2 + 64
OFF_B3 = OFF_W3 + 9 * 64
N_PARAM = OFF_B3 + 9


def bf16(x):
    """Round to BF16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(64, 13), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(64, 64),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(9, 64), p[OFF_B3:N_PARAM])


GELU_A, GELU_B = math.sqrt(2.0 / math.pi), 0.044715


def gelu(z):
    """GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(GELU_A * (z + GELU_B * z ** 3)))


def gelu_d(z):
    t = np.tanh(GELU_A * (z + GELU_B * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_A * (1.0 + 3.0 * GELU_B * z * z)


def _norm(norm):
    n = np.asarray(norm, dtype=np.float64)
    return n[:13], n[13:26], n[26:35], n[35:44]


def forward(params, norm, X):
    """Outputs in physical units, and the intermediates grad() needs."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    xmu, xsd, ymu, ysd = _norm(norm)
    xn = (np.asarray(X, np.float32) - xmu.astype(np.float32)) / xsd.astype(np.float32)
    x = bf16(xn)
    z1 = x @ bf16(W1).T + b1
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(W2).T + b2
    h2 = bf16(gelu(z2))
    yn = h2 @ bf16(W3).T + b3
    return yn * ysd + ymu, (x, z1, h1, z2, h2, yn)


def grad(params, norm, X, T):
    """(loss sum, gradient vector) of the mean squared error of the normalised
    outputs over the batch, as one training step of the device computes it."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    xmu, xsd, ymu, ysd = _norm(norm)
    _, (x, z1, h1, z2, h2, yn) = forward(params, norm, X)
    n = x.shape[0]
    tn = (np.asarray(T, np.float32) - ymu.astype(np.float32)) / ysd.astype(np.float32)
    e = yn - tn
    loss = float(np.sum(e * e))
    dy = e * (2.0 / (9.0 * n))
    dyb = bf16(dy)
    dh2 = dyb @ bf16(W3)
    dz2 = dh2 * gelu_d(z2)
    dz2b = bf16(dz2)
    dh1 = dz2b @ bf16(W2)
    dz1 = dh1 * gelu_d(z1)
    dz1b = bf16(dz1)
    g = np.zeros(N_PARAM)
    g[OFF_W1:OFF_B1] = (dz1b.T @ x)[:, :13].ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    g[OFF_W2:OFF_B2] = (dz2b.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    g[OFF_W3:OFF_B3] = (dyb.T @ h2).ravel()
    g[OFF_B3:N_PARAM] = dy.sum(axis=0)
    return loss, g


def adam(w, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v


# ------------------------------------------------------------------ sampling
def _wrap(i, n):
    return (i - 2) % (n - 2) + 2


def _favre(var, i, j, k, fw):
    """Favre-filtered (rho, u, v, w, T) and the filtered products at 1-based (i, j, k)."""
    n3, n2, n1 = var.shape[1:]
    h = fw // 2
    offs = [0] if fw == 0 else list(range(-h, h + 1))
    wts = [1.0] if fw == 0 else [0.5 if abs(a) == h else 1.0 for a in offs]
    s = np.zeros(5)
    sp = np.zeros(9)
    for b, wb in zip(offs, wts):
        for a, wa in zip(offs, wts):
            ii, jj = _wrap(i + a, n1), _wrap(j + b, n2)
            r, u, v, w, T = (var[m, k - 1, jj - 1, ii - 1] for m in (0, 1, 2, 3, 5))
            wg = wa * wb
            rw = wg * r
            s += [wg * r, rw * u, rw * v, rw * w, rw * T]
            sp += [rw * u * u, rw * v * v, rw * w * w, rw * u * v, rw * u * w, rw * v * w,
                   rw * u * T, rw * v * T, rw * w * T]
    nrm = 1.0 if fw == 0 else 1.0 / (fw * fw)
    f = np.array([s[0] * nrm, s[1] / s[0], s[2] / s[0], s[3] / s[0], s[4] / s[0]])
    return f, sp * nrm


def features_at(var, x3, dx, dy, Re, i, j, k, sx, sy, sz, fw, tau2, rho_w, mu_w):
    n3 = var.shape[1]
    fxp, _ = _favre(var, i + sx, j, k, fw)
    fxm, _ = _favre(var, i - sx, j, k, fw)
    fyp, _ = _favre(var, i, j + sy, k, fw)
    fym, _ = _favre(var, i, j - sy, k, fw)
    kp, km = min(k + sz, n3), max(k - sz, 1)
    fzp, _ = _favre(var, i, j, kp, fw)
    fzm, _ = _favre(var, i, j, km, fw)
    X = np.zeros(13)
    for m in range(4):
        X[3 * m + 0] = (fxp[m + 1] - fxm[m + 1]) / (2.0 * sx * dx)
        X[3 * m + 1] = (fyp[m + 1] - fym[m + 1]) / (2.0 * sy * dy)
        X[3 * m + 2] = (fzp[m + 1] - fzm[m + 1]) / (x3[kp - 1] - x3[km - 1])
    tw = 0.5 * (tau2[0] - tau2[1])
    ut = math.sqrt(max(tw, 0.0) / rho_w) if rho_w > 0 else 0.0
    d = min(x3[k - 1] - x3[0], x3[n3 - 1] - x3[k - 1])
    X[12] = rho_w * ut * d * Re / mu_w
    return X


def sample(var, x3, dx, dy, Re, sx, sy, sz, fw, tau2, stat1, Tw=(1.0, 1.0)):
    """(X [n][13], T [n][9]) at the library's sample points, in its order."""
    n3, n2, n1 = var.shape[1:]
    rho_w = 0.5 * (stat1[0][0] + stat1[0][n3 - 1])
    mu_w = 0.5 * (Tw[0] ** 0.7 + Tw[1] ** 0.7)
    ni, nj, nk = (n1 - 3) // sx + 1, (n2 - 3) // sy + 1, (n3 - 1) // sz - 1
    Xs, Ts = [], []
    for c in range(nk):
        for b in range(nj):
            for a in range(ni):
                i, j, k = 2 + sx * a, 2 + sy * b, 1 + sz + sz * c
                Xs.append(features_at(var, x3, dx, dy, Re, i, j, k, sx, sy, sz, fw, tau2, rho_w, mu_w))
                f, p = _favre(var, i, j, k, fw)
                r, u, v, w, T = f
                Ts.append([p[0] - r * u * u, p[1] - r * v * v, p[2] - r * w * w, p[3] - r * u * v,
                           p[4] - r * u * w, p[5] - r * v * w, p[6] - r * u * T, p[7] - r * v * T,
                           p[8] - r * w * T])
    return np.array(Xs), np.array(Ts)


def source(var, x3, czh, dx, dy, Re, gama, params, norm, tau2, stat1, Tw=(1.0, 1.0)):
    """Closure source S[4][n3-2][n2-2][n1-2] (rows rho*u, rho*v, rho*w, rho*E)
    of a coarse state, from the MLP's fluxes at every interior point."""
    n3, n2, n1 = var.shape[1:]
    rho_w = 0.5 * (stat1[0][0] + stat1[0][n3 - 1])
    mu_w = 0.5 * (Tw[0] ** 0.7 + Tw[1] ** 0.7)
    pts = [(i, j, k) for k in range(2, n3) for j in range(2, n2) for i in range(2, n1)]
    X = np.array([features_at(var, x3, dx, dy, Re, i, j, k, 1, 1, 1, 0, tau2, rho_w, mu_w) for i, j, k in pts])
    Y, _ = forward(params, norm, X.astype(np.float32))
    F = np.zeros((9, n3, n2 + 2, n1 + 2))   # fluxes on interior k with a periodic frame in i, j
    Yg = Y.reshape(n3 - 2, n2 - 2, n1 - 2, 9)
    for c in range(9):
        F[c, 1:n3 - 1, 2:n2, 2:n1] = Yg[..., c]
    # periodic duplicates / ghosts of the interior unique points
    for i in list(range(0, 2)) + [n1, n1 + 1]:
        F[:, :, 2:n2, i] = F[:, :, 2:n2, _wrap(i, n1)]
    for j in list(range(0, 2)) + [n2, n2 + 1]:
        F[:, :, j, :] = F[:, :, _wrap(j, n2), :]
    comp = [[0, 3, 4], [3, 1, 5], [4, 5, 2], [6, 7, 8]]
    S = np.zeros((4, n3 - 2, n2 - 2, n1 - 2))
    hdx, hdy = 0.5 / dx, 0.5 / dy
    for a in range(4):
        cx, cy, cz = comp[a]
        for k in range(2, n3):
            ddx = (F[cx, k - 1, 2:n2, 3:n1 + 1] - F[cx, k - 1, 2:n2, 1:n1 - 1]) * hdx
            ddy = (F[cy, k - 1, 3:n2 + 1, 2:n1] - F[cy, k - 1, 1:n2 - 1, 2:n1]) * hdy
            ddz = (F[cz, k, 2:n2, 2:n1] - F[cz, k - 2, 2:n2, 2:n1]) * czh[k]
            d = ddx + ddy + ddz
            S[a, k - 2] = -d if a < 3 else -gama * d
    return S
