"""Pure numpy / Python restatement of the hot path, for small cases.

TEST INFRASTRUCTURE ONLY.  A second, independent restatement used to check
the C oracle (oracle/gpv_oracle.c): it shares no code with it (numpy.fft in
place of the hand-written FFT, straight loops in place of the C kernels).
Paths cited are within the reference geopyv-dev crate.
"""
from __future__ import annotations

import numpy as np

# Q (src/image.rs:183-190)
Q = np.array([
    [1 / 120, 13 / 60, 11 / 20, 13 / 60, 1 / 120, 0],
    [-1 / 24, -5 / 12, 0, 5 / 12, 1 / 24, 0],
    [1 / 12, 1 / 6, -1 / 2, 1 / 6, 1 / 12, 0],
    [-1 / 12, 1 / 6, 0, -1 / 6, 1 / 12, 0],
    [1 / 24, -1 / 6, 1 / 4, -1 / 6, 1 / 24, 0],
    [-1 / 120, 1 / 24, -1 / 12, 1 / 12, -1 / 24, 1 / 120],
])


def get_c(img, border=20):
    """get_c (src/image.rs:252-327) with numpy.fft."""
    P = np.pad(np.asarray(img, float), border, mode="edge").astype(complex)
    k = [1 / 120, 13 / 60, 11 / 20, 13 / 60, 1 / 120, 0]

    def kern(n):  # build_kernel (src/image.rs:422-430)
        v = np.zeros(n, complex)
        v[0], v[1], v[2], v[n - 2], v[n - 1] = k[2], k[3], k[4], k[0], k[1]
        return np.fft.fft(v)

    P = np.fft.ifft(np.fft.fft(P, axis=1) / kern(P.shape[1]), axis=1)
    P = np.fft.ifft(np.fft.fft(P, axis=0) / kern(P.shape[0])[:, None], axis=0)
    return P.real


def qt_poly(t):
    return Q.T @ np.array([1, t, t * t, t ** 3, t ** 4, t ** 5])


def qt_dpoly(t):
    return Q.T @ np.array([0, 1, 2 * t, 3 * t * t, 4 * t ** 3, 5 * t ** 4])


def eval_grad(C, shape, border, x, y):
    """Image::eval_grad (src/image.rs:115-178)."""
    h, w = shape
    x = min(max(x, 0.0), w - 1e-9)
    y = min(max(y, 0.0), h - 1e-9)
    xf, yf = int(np.floor(x)), int(np.floor(y))
    a, da = qt_poly(y - yf), qt_dpoly(y - yf)
    b, db = qt_poly(x - xf), qt_dpoly(x - xf)
    blk = C[yf + border - 2:yf + border + 4, xf + border - 2:xf + border + 4]
    return a @ blk @ b, (a @ blk @ db, da @ blk @ b)


def circle(r):
    """LocalMask::circle (src/masks.rs:69-109)."""
    return np.array([[x, y] for y in range(-r, r + 1) for x in range(-r, r + 1)
                     if np.sqrt(x * x + y * y) <= r], float)


def p_len(order):
    return {0: 2, 1: 6, 2: 12}[order]


def warp(coord, p, xy):
    """apply_warp (src/subset.rs:262-300)."""
    dx, dy = xy[:, 0] - coord[0], xy[:, 1] - coord[1]
    if len(p) == 2:
        return xy + np.array(p)
    u = p[0] + p[2] * dx + p[4] * dy
    v = p[1] + p[3] * dx + p[5] * dy
    if len(p) == 12:
        u = u + 0.5 * p[6] * dx * dx + p[8] * dx * dy + 0.5 * p[10] * dy * dy
        v = v + 0.5 * p[7] * dx * dx + p[9] * dx * dy + 0.5 * p[11] * dy * dy
    return np.stack([xy[:, 0] + u, xy[:, 1] + v], 1)


def sdi(coord, xy, grad, order):
    """steepest_descent (src/subset.rs:311-343)."""
    dx, dy = xy[:, 0] - coord[0], xy[:, 1] - coord[1]
    gx, gy = grad[:, 0], grad[:, 1]
    cols = [gx, gy]
    if order >= 1:
        cols += [gx * dx, gy * dx, gx * dy, gy * dy]
    if order == 2:
        cols += [gx * 0.5 * dx * dx, gy * 0.5 * dx * dx, gx * dx * dy, gy * dx * dy, gx * 0.5 * dy * dy, gy * 0.5 * dy * dy]
    return np.stack(cols, 1)


def compose(p, dp):
    """compose_icgn (src/subset.rs:487-611)."""
    p, dp = np.asarray(p, float), np.asarray(dp, float)
    if p.size == 2:
        return p - dp
    if p.size == 6:
        def W(q):
            return np.array([[1 + q[2], q[4], q[0]], [q[3], 1 + q[5], q[1]], [0, 0, 1.0]])
        n = W(p) @ np.linalg.inv(W(dp))
        return np.array([n[0, 2], n[1, 2], n[0, 0] - 1, n[1, 0], n[0, 1], n[1, 1] - 1])

    def L(q):
        u, v, ux, vx, uy, vy, uxx, vxx, uxy, vxy, uyy, vyy = q
        s = [2 * ux + ux * ux + u * uxx, 2 * u * uxy + 2 * (1 + ux) * uy, uy * uy + u * uyy, 2 * u * (1 + ux),
             2 * u * uy, u * u, 0.5 * (v * uxx + 2 * (1 + ux) * vx + u * vxx),
             uy * vx + ux * vy + v * uxy + u * vxy + vy + ux, 0.5 * (v * uyy + 2 * uy * (1 + vy) + u * vyy),
             v + v * ux + u * vx, u + v * uy + u * vy, u * v, vx * vx + v * vxx, 2 * v * vxy + 2 * vx * (1 + vy),
             2 * vy + vy * vy + v * vyy, 2 * v * vx, 2 * v * (1 + vy), v * v]
        return np.array([
            [1 + s[0], s[1], s[2], s[3], s[4], s[5]],
            [s[6], 1 + s[7], s[8], s[9], s[10], s[11]],
            [s[12], s[13], 1 + s[14], s[15], s[16], s[17]],
            [0.5 * uxx, uxy, 0.5 * uyy, 1 + ux, uy, u],
            [0.5 * vxx, vxy, 0.5 * vyy, vx, 1 + vy, v],
            [0, 0, 0, 0, 0, 1.0]])
    n = L(p) @ np.linalg.inv(L(dp))
    return np.array([n[3, 5], n[4, 5], n[3, 3] - 1, n[4, 3], n[3, 4], n[4, 4] - 1,
                     2 * n[3, 0], 2 * n[4, 0], n[3, 1], n[4, 1], 2 * n[3, 2], 2 * n[4, 2]])


def norm(dp, size):
    """convergence_norm (src/subset.rs:622-649)."""
    dp = np.asarray(dp, float)
    s = dp[0] ** 2 + dp[1] ** 2
    if dp.size >= 6:
        s += np.sum((dp[2:6] * size) ** 2)
    if dp.size == 12:
        s += np.sum((0.5 * dp[6:12] * size * size) ** 2)
    return float(np.sqrt(s))


def solve_icgn(Cf, Cg, shape, border, coord, radius, order, p0=None, max_norm=1e-5, max_iterations=50,
               tolerance=0.75):
    """Subset::new + solve_icgn_result (src/subset.rs:836-919, 1117-1219), straight loops."""
    offs = circle(radius)
    fc = offs + np.asarray(coord, float)
    n = fc.shape[0]
    f = np.empty(n)
    grad = np.empty((n, 2))
    for i in range(n):
        f[i], (grad[i, 0], grad[i, 1]) = eval_grad(Cf, shape, border, fc[i, 0], fc[i, 1])
    f_m = f.sum() / n
    df = np.sqrt(np.sum((f - f_m) ** 2))
    m = p_len(order)
    p = np.zeros(m)
    if p0 is not None:
        p[:min(m, len(p0))] = np.asarray(p0, float)[:m]
    S = sdi(coord, fc, grad, order)
    Hi = np.linalg.inv(S.T @ S)
    size = np.sqrt(n)
    hist = []
    converged = False
    for it in range(1, max_iterations + 1):
        gc = warp(coord, p, fc)
        g = np.array([eval_grad(Cg, shape, border, gc[i, 0], gc[i, 1])[0] for i in range(n)])
        g_m = g.sum() / n
        dg = np.sqrt(np.sum((g - g_m) ** 2))
        a, b = f - f_m, g - g_m
        zn = np.sum((a / df - b / dg) ** 2)
        grad_z = S.T @ (a - (df / dg) * b)
        dp = -(Hi @ grad_z)
        p = compose(p, dp)
        nrm = norm(dp, size)
        hist.append((it, nrm, 1 - zn / 2, zn))
        if nrm < max_norm:
            converged = True
            break
    zncc = hist[-1][2] if hist else 0.0
    return dict(p=p, c_zncc=zncc, c_znssd=hist[-1][3] if hist else 4.0, iterations=len(hist), converged=converged,
                quality_ok=converged and zncc >= tolerance, history=hist, f_m=f_m, delta_f=df, n_px=n)
