"""Dense FP64 reference for the adjoint of a converged bundle adjustment (test infrastructure only).

The adjoint (vector-Jacobian product by implicit differentiation, ``tba_bundle_vjp``) has no
counterpart in the reference, so its parity is unpinned by the reference itself.  This module
checks it independently of the CUDA code's second-order formulas: it builds the dense Hessian of
the robust cost by central differences of the analytic gradient, and handles the gauge with the
KKT system of the baseline constraint instead of the CUDA path's oblique projection.

Model (the reference's projection and robust cost, src/geometry/camera.ts:15-61,
src/geometry/pose.ts:61-88, src/sfm/bundle/bundle-shared.ts:32-54): q = R X + t, pinhole with the
two-term radial factor, residual r = pi(q) - y, Huber cost rho(e) = e^2 (e <= h), 2 h e - h^2.
Local coordinates are the solver's update (src/geometry/pose.ts:40-57): R' = exp([w]x) R,
t' = exp([w]x) t + v, X' = X + dX, for every variable camera and point.  The gradient of the
pulled-back cost E(theta (+) delta) is exact at any delta (the SO(3) left Jacobian enters), so its
central differences give the Hessian in the chart at theta.
"""
from __future__ import annotations

import numpy as np


def skew(w):
    w = np.asarray(w)
    K = np.zeros(w.shape[:-1] + (3, 3))
    K[..., 0, 1], K[..., 0, 2] = -w[..., 2], w[..., 1]
    K[..., 1, 0], K[..., 1, 2] = w[..., 2], -w[..., 0]
    K[..., 2, 0], K[..., 2, 1] = -w[..., 1], w[..., 0]
    return K


def so3_exp(w):
    th = np.linalg.norm(w, axis=-1)[..., None, None]
    K = skew(w)
    small = th < 1e-8
    ths = np.where(small, 1.0, th)
    a = np.where(small, 1.0 - th**2 / 6, np.sin(ths) / ths)
    b = np.where(small, 0.5 - th**2 / 24, (1 - np.cos(ths)) / ths**2)
    return np.eye(3) + a * K + b * (K @ K)


def so3_left_jacobian(w):
    th = np.linalg.norm(w, axis=-1)[..., None, None]
    K = skew(w)
    small = th < 1e-6
    ths = np.where(small, 1.0, th)
    a = np.where(small, 0.5 - th**2 / 24, (1 - np.cos(ths)) / ths**2)
    b = np.where(small, 1.0 / 6 - th**2 / 120, (ths - np.sin(ths)) / ths**3)
    return np.eye(3) + a * K + b * (K @ K)


class Problem:
    """A packed problem (the reference's scene and index layouts) at an evaluation point."""

    def __init__(self, C, P, M, scene, index, anchor=0, scale_view=1, huber=2.0):
        self.C, self.P, self.M = C, P, M
        self.anchor, self.scale_view, self.huber = anchor, scale_view, huber
        self.poses = scene[:12 * C].reshape(C, 12).copy()
        self.points = scene[12 * C:12 * C + 3 * P].reshape(P, 3).copy()
        self.cams = scene[12 * C + 3 * P:18 * C + 3 * P].reshape(C, 6).copy()
        self.pixels = scene[18 * C + 3 * P:].reshape(M, 2).copy()
        self.obs_camera = index[:M].astype(np.int64)
        self.obs_point = index[M:2 * M].astype(np.int64)
        self.active = index[3 * M + P + C + 2:3 * M + P + 2 * C + 2].astype(bool)
        self.var = np.flatnonzero(self.active)
        self.slot = -np.ones(C, dtype=np.int64)
        self.slot[self.var] = np.arange(len(self.var))
        self.n = 6 * len(self.var) + 3 * P

    # ---- local coordinates --------------------------------------------------------------------
    def split(self, delta):
        nv = len(self.var)
        return delta[:6 * nv].reshape(nv, 6), delta[6 * nv:].reshape(self.P, 3)

    def retract(self, delta):
        dc, dp = self.split(delta)
        R = self.poses[:, :9].reshape(-1, 3, 3).copy()
        t = self.poses[:, 9:].copy()
        E = so3_exp(dc[:, :3])
        R[self.var] = E @ R[self.var]
        t[self.var] = np.einsum("cij,cj->ci", E, t[self.var]) + dc[:, 3:]
        return R, t, self.points + dp

    def flat(self, delta):
        R, t, X = self.retract(delta)
        return np.concatenate([np.concatenate([R.reshape(-1, 9), t], axis=1).ravel(), X.ravel()])

    # ---- the gradient of the pulled-back robust cost -------------------------------------------
    def gradient(self, delta, cams=None, pixels=None, per_obs=False):
        cams = self.cams if cams is None else cams
        pixels = self.pixels if pixels is None else pixels
        dc, dp = self.split(delta)
        R, t, X = self.retract(delta)
        c, p = self.obs_camera, self.obs_point
        a = np.einsum("nij,nj->ni", self.poses[c, :9].reshape(-1, 3, 3), X[p]) + self.poses[c, 9:]
        w_loc = np.zeros((self.M, 3))
        var_obs = self.active[c]
        w_loc[var_obs] = dc[self.slot[c[var_obs]], :3]
        Eo = so3_exp(w_loc)
        q = np.einsum("nij,nj->ni", Eo, a)
        v_loc = np.zeros((self.M, 3))
        v_loc[var_obs] = dc[self.slot[c[var_obs]], 3:]
        q = q + v_loc
        k = cams[c]
        z = q[:, 2]
        x, y = q[:, 0] / z, q[:, 1] / z
        r2 = x * x + y * y
        d = 1 + k[:, 4] * r2 + k[:, 5] * r2 * r2
        d1 = k[:, 4] + 2 * k[:, 5] * r2
        fx, fy = k[:, 0], k[:, 1]
        r = np.stack([fx * x * d + k[:, 2], fy * y * d + k[:, 3]], axis=1) - pixels
        Pux, Puy = fx * (d + 2 * x * x * d1), 2 * fx * x * y * d1
        Pvx, Pvy = 2 * fy * x * y * d1, fy * (d + 2 * y * y * d1)
        Dx = np.stack([1 / z, np.zeros_like(z), -x / z], axis=1)
        Dy = np.stack([np.zeros_like(z), 1 / z, -y / z], axis=1)
        du = Pux[:, None] * Dx + Puy[:, None] * Dy
        dv = Pvx[:, None] * Dx + Pvy[:, None] * Dy
        e = np.sqrt((r * r).sum(1))
        w = np.where(e > self.huber, self.huber / np.where(e > 0, e, 1), 1.0)
        gu = w * r[:, 0]
        gv = w * r[:, 1]
        hq = gu[:, None] * du + gv[:, None] * dv  # d rho/2 / dq
        gX = np.einsum("nij,ni->nj", R[c], hq)   # (dq/dX)^T h, dq/dX = R'
        gw = np.einsum("nij,ni->nj", -skew(q - v_loc) @ so3_left_jacobian(w_loc), hq)
        if per_obs:
            return gw, hq, gX
        out_c = np.zeros((len(self.var), 6))
        np.add.at(out_c[:, :3], self.slot[c[var_obs]], gw[var_obs])
        np.add.at(out_c[:, 3:], self.slot[c[var_obs]], hq[var_obs])
        out_p = np.zeros((self.P, 3))
        np.add.at(out_p, p, gX)
        return np.concatenate([out_c.ravel(), out_p.ravel()])

    def half_cost(self, delta):
        """Half the robust cost at theta (+) delta (the function whose gradient `gradient` is)."""
        R, t, X = self.retract(delta)
        c, p = self.obs_camera, self.obs_point
        q = np.einsum("nij,nj->ni", R[c], X[p]) + t[c]
        k = self.cams[c]
        x, y = q[:, 0] / q[:, 2], q[:, 1] / q[:, 2]
        r2 = x * x + y * y
        d = 1 + k[:, 4] * r2 + k[:, 5] * r2 * r2
        r = np.stack([k[:, 0] * x * d + k[:, 2], k[:, 1] * y * d + k[:, 3]], axis=1) - self.pixels
        e = np.sqrt((r * r).sum(1))
        h = self.huber
        return 0.5 * np.where(e <= h, e * e, 2 * h * e - h * h).sum()

    def hessian(self, h=1e-6):
        H = np.zeros((self.n, self.n))
        e = np.zeros(self.n)
        for j in range(self.n):
            e[j] = h
            H[:, j] = (self.gradient(e) - self.gradient(-e)) / (2 * h)
            e[j] = 0
        return 0.5 * (H + H.T)

    def baseline(self, delta):
        R, t, _ = self.retract(delta)
        centre = lambda k: -R[k].T @ t[k]
        return np.linalg.norm(centre(self.scale_view) - centre(self.anchor))

    def vjp(self, cotangent, h=1e-6):
        """(pixels_bar M x 2, [d/ds, d/dk1]) of <cotangent, solution> by the dense KKT system."""
        zero = np.zeros(self.n)
        H = self.hessian(h)
        e = np.zeros(self.n)
        gbar = np.zeros(self.n)
        gc = np.zeros(self.n)
        for j in range(self.n):
            e[j] = h
            gbar[j] = (cotangent @ (self.flat(e) - self.flat(-e))) / (2 * h)
            gc[j] = (self.baseline(e) - self.baseline(-e)) / (2 * h)
            e[j] = 0
        single_fixed = (~self.active).sum() == 1
        if single_fixed:
            K = np.zeros((self.n + 1, self.n + 1))
            K[:self.n, :self.n] = H
            K[:self.n, self.n] = gc
            K[self.n, :self.n] = gc
            lam = np.linalg.solve(K, np.concatenate([gbar, [0.0]]))[:self.n]
        else:
            lam = np.linalg.solve(H, gbar)
        dc, dp = self.split(lam)
        # dF/dy by central differences of each observation's own gradient share
        c, p = self.obs_camera, self.obs_point
        lam_w = np.zeros((self.M, 3))
        lam_v = np.zeros((self.M, 3))
        var_obs = self.active[c]
        lam_w[var_obs] = dc[self.slot[c[var_obs]], :3]
        lam_v[var_obs] = dc[self.slot[c[var_obs]], 3:]
        lam_x = dp[p]
        ybar = np.zeros((self.M, 2))
        for col in range(2):
            plus = self.pixels.copy()
            minus = self.pixels.copy()
            plus[:, col] += h
            minus[:, col] -= h
            gp = self.gradient(zero, pixels=plus, per_obs=True)
            gm = self.gradient(zero, pixels=minus, per_obs=True)
            dF = [(a - b) / (2 * h) for a, b in zip(gp, gm)]
            ybar[:, col] = -((dF[0] * lam_w).sum(1) + (dF[1] * lam_v).sum(1) + (dF[2] * lam_x).sum(1))
        # dF/ds (every fx, fy scaled by exp(s)) and dF/dk1 (k1 shifted), by central differences
        kbar = np.zeros(2)
        for which in range(2):
            cp = self.cams.copy()
            cm = self.cams.copy()
            if which == 0:
                cp[:, :2] *= np.exp(h)
                cm[:, :2] *= np.exp(-h)
            else:
                cp[:, 4] += h
                cm[:, 4] -= h
            dF = (self.gradient(zero, cams=cp) - self.gradient(zero, cams=cm)) / (2 * h)
            kbar[which] = -lam @ dF
        return ybar, kbar
