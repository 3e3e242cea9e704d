"""Seeded synthetic bundle-adjustment scenes (the benchmark configurations).

No public dataset is used: every scene is drawn from numpy's PCG64 generator with a fixed seed,
with Gaussians from the generator's normal sampler.  Poses follow the reference's convention
(world-to-camera, q = R X + t, src/contracts/camera.ts:17-21); cameras carry the reference's
camera record (fx, fy, cx, cy, k1, k2; src/contracts/camera-record.ts:12-38).

* ``ring_scene``    cameras evenly on a ring facing the origin, points uniform in a cube,
                    each point observed by every camera it projects into (config 0; the
                    arcs of config 3).
* ``helix_scene``   cameras on a multi-lap helix facing its axis, per-camera focal lengths,
                    each point kept in a uniform 3-12 of the cameras that see it (configs 1, 4).
* ``sphere_scene``  cameras on a jittered sphere facing its centre, points from a mixture of
                    Gaussians in a ball, geometric track lengths (config 2).
* ``arc_scene``     a local window: cameras on an arc of the ring facing the origin, tracks of
                    2-10 of the nearest cameras (``batch_scenes``: the 512 windows of config 3).
* ``inverse_depth_rows`` inverse-depth measurements packed as the 34-word rows of
                    ``tba_linearize_inverse_depth``: points anchored in a ring camera, each seen by
                    one of the next cameras of the ring.
* ``inverse_depth_corridor`` a reconstruction (views and landmarks as records) for the joint
                    inverse-depth bundle adjustment: translated views along a corridor, each run of
                    consecutive views seeing points of its own.

Every scene then gets Gaussian pixel noise, uniform in-image outliers and a perturbed
initialisation (rotation by an axis-angle of fixed size, translation by a fraction of its norm,
Gaussian point noise, a common focal factor); camera 0 is the gauge anchor and stays exact.
The result is packed in the reference's layout (``typecv_b200.bundle.pack_arrays``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .bundle import pack_arrays


@dataclass
class Scene:
    name: str
    poses: np.ndarray     # C x 12 (R row-major, t), perturbed initialisation
    points: np.ndarray    # P x 3, perturbed
    cameras: np.ndarray   # C x 6 (fx, fy, cx, cy, k1, k2), perturbed focal
    obs_camera: np.ndarray  # M, point-major
    obs_point: np.ndarray   # M, non-decreasing
    pixels: np.ndarray      # M x 2
    truth_poses: np.ndarray
    truth_points: np.ndarray
    truth_cameras: np.ndarray
    options: dict = field(default_factory=dict)
    anchor: int = 0
    scale_view: int = 1

    @property
    def C(self):
        return len(self.poses)

    @property
    def P(self):
        return len(self.points)

    @property
    def M(self):
        return len(self.obs_camera)

    def packed(self, active=None):
        if active is None:
            active = np.ones(self.C, dtype=np.uint32)
            active[self.anchor] = 0
        return pack_arrays(self.poses, self.points, self.cameras, self.obs_camera, self.obs_point, self.pixels,
                           active)

    def as_reconstruction(self):
        """The scene as the reference's SparseReconstruction object model (small scenes)."""
        views = [{"id": 10 * (c + 1), "camera": dict(zip(("fx", "fy", "cx", "cy", "k1", "k2"), map(float, self.cameras[c]))),
                  "pose": {"R": self.poses[c, :9].copy(), "t": self.poses[c, 9:].copy()}} for c in range(self.C)]
        starts = np.searchsorted(self.obs_point, np.arange(self.P + 1))
        landmarks = []
        for p in range(self.P):
            obs = [{"viewId": 10 * (int(self.obs_camera[i]) + 1), "featureId": p,
                    "pixel": [float(self.pixels[i, 0]), float(self.pixels[i, 1])]} for i in range(starts[p], starts[p + 1])]
            landmarks.append({"trackId": p, "xyz": self.points[p].copy(), "observations": obs})
        return {"views": views, "landmarks": landmarks}


def look_at(centers: np.ndarray, targets: np.ndarray) -> np.ndarray:
    """World-to-camera rotations (rows x, y, z) of cameras at `centers` looking at `targets`,
    image y pointing down (world z up)."""
    z = targets - centers
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    up = np.tile([0.0, 0.0, 1.0], (len(z), 1))
    polar = np.abs(z[:, 2]) > 0.99
    up[polar] = [0.0, 1.0, 0.0]
    x = np.cross(z, up)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def poses_from(R: np.ndarray, centers: np.ndarray) -> np.ndarray:
    t = -np.einsum("cij,cj->ci", R, centers)
    return np.concatenate([R.reshape(-1, 9), t], axis=1)


def project(poses, cameras, cam_idx, X):
    """Pinhole + two-term radial projection of points X (n x 3) in cameras cam_idx (n);
    returns pixels (n x 2) and depth (n)."""
    R = poses[cam_idx, :9].reshape(-1, 3, 3)
    q = np.einsum("nij,nj->ni", R, X) + poses[cam_idx, 9:]
    z = q[:, 2]
    zs = np.where(z > 1e-12, z, 1.0)
    x, y = q[:, 0] / zs, q[:, 1] / zs
    r2 = x * x + y * y
    k = cameras[cam_idx]
    d = 1 + k[:, 4] * r2 + k[:, 5] * r2 * r2
    return np.stack([k[:, 0] * x * d + k[:, 2], k[:, 1] * y * d + k[:, 3]], axis=1), z, r2


def visible(poses, cameras, cam_idx, X, width, height, margin=2.0):
    px, z, r2 = project(poses, cameras, cam_idx, X)
    k1 = cameras[cam_idx, 4]
    # stay well inside the radial model's injective branch (r^2 < -1/(3 k1) for k1 < 0)
    fold = np.where(k1 < 0, -1.0 / (3.0 * np.where(k1 < 0, k1, -1.0)), np.inf)
    return ((z > 0.1) & (px[:, 0] > margin) & (px[:, 0] < width - margin) & (px[:, 1] > margin)
            & (px[:, 1] < height - margin) & (r2 < 0.5 * fold))


def axis_angle_rotations(rng, n, angle):
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    w = axis * angle
    th = np.linalg.norm(w, axis=1)
    K = np.zeros((n, 3, 3))
    K[:, 0, 1], K[:, 0, 2], K[:, 1, 0] = -w[:, 2], w[:, 1], w[:, 2]
    K[:, 1, 2], K[:, 2, 0], K[:, 2, 1] = -w[:, 0], -w[:, 1], w[:, 0]
    a = (np.sin(th) / th)[:, None, None]
    b = ((1 - np.cos(th)) / th**2)[:, None, None]
    return np.eye(3)[None] + a * K + b * (K @ K)


def finish(name, rng, poses, cameras, points, obs_camera, obs_point, *, width, height, noise_px=0.5,
           outlier_rate=0.03, rot_rad=0.01, trans_frac=0.01, point_sigma=0.01, focal_factor=1.03,
           options=None) -> Scene:
    """Observations with noise and outliers, then the perturbed initialisation."""
    px, _, _ = project(poses, cameras, obs_camera, points[obs_point])
    px = px + rng.normal(scale=noise_px, size=px.shape)
    out = rng.random(len(px)) < outlier_rate
    px[out, 0] = rng.uniform(0, width, out.sum())
    px[out, 1] = rng.uniform(0, height, out.sum())
    C = len(poses)
    dR = axis_angle_rotations(rng, C, rot_rad)
    R0 = poses[:, :9].reshape(-1, 3, 3)
    t0 = poses[:, 9:]
    u = rng.normal(size=(C, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    R1 = dR @ R0
    t1 = t0 + trans_frac * np.linalg.norm(t0, axis=1, keepdims=True) * u
    R1[0], t1[0] = R0[0], t0[0]
    init_poses = np.concatenate([R1.reshape(-1, 9), t1], axis=1)
    init_points = points + rng.normal(scale=point_sigma, size=points.shape)
    init_cameras = cameras.copy()
    init_cameras[:, :2] *= focal_factor
    return Scene(name, init_poses, init_points, init_cameras, obs_camera.astype(np.uint32), obs_point.astype(np.uint32),
                 px, poses, points, cameras, dict(options or {}))


def intrinsics(C, f=800.0, width=1024, height=768, k1=-0.05, k2=0.0):
    cams = np.zeros((C, 6))
    cams[:, 0] = cams[:, 1] = f
    cams[:, 2], cams[:, 3] = width / 2, height / 2
    cams[:, 4], cams[:, 5] = k1, k2
    return cams


def ring_scene(seed=0, cameras=10, points=2000, radius=5.0, cube=2.0, arc=2 * np.pi, **kw) -> Scene:
    """Configuration 0: 10 cameras on a 5 m ring facing the origin, 2,000 points uniform in a
    2 m cube, every in-image observation kept."""
    rng = np.random.default_rng(seed)
    ang = arc * np.arange(cameras) / (cameras if arc >= 2 * np.pi - 1e-9 else max(1, cameras - 1))
    centers = np.stack([radius * np.cos(ang), radius * np.sin(ang), np.zeros(cameras)], axis=1)
    poses = poses_from(look_at(centers, np.zeros_like(centers)), centers)
    cams = intrinsics(cameras)
    X = rng.uniform(-cube / 2, cube / 2, size=(points, 3))
    pc = np.repeat(np.arange(points), cameras)
    cc = np.tile(np.arange(cameras), points)
    vis = visible(poses, cams, cc, X[pc], 1024, 768)
    keep = np.bincount(pc[vis], minlength=points) >= 2
    sel = vis & keep[pc]
    remap = np.cumsum(keep) - 1
    options = {"iterations": 20, "huberPx": 2.0, "cgRelativeTolerance": 1e-6, "refineSharedFocal": True}
    return finish(f"ring-{cameras}x{points}", rng, poses, cams, X[keep], cc[sel], remap[pc[sel]],
                  width=1024, height=768, options={**options, **kw.pop("options", {})}, **kw)


def helix_scene(seed=1, cameras=200, points=100_000, radius=8.0, laps=3, pitch=1.0, cube=4.0, track=(3, 12),
                **kw) -> Scene:
    """Configuration 1: 200 cameras on a 3-lap helix (radius 8 m, pitch 1 m) facing its axis,
    focal lengths 700-900 px, 100k points in a 4 m cube, each kept in 3-12 cameras."""
    rng = np.random.default_rng(seed)
    th = 2 * np.pi * laps * np.arange(cameras) / cameras
    h = pitch * th / (2 * np.pi) - pitch * laps / 2
    centers = np.stack([radius * np.cos(th), radius * np.sin(th), h], axis=1)
    targets = np.stack([np.zeros(cameras), np.zeros(cameras), h], axis=1)
    poses = poses_from(look_at(centers, targets), centers)
    cams = intrinsics(cameras)
    cams[:, 0] = cams[:, 1] = rng.uniform(700, 900, cameras)
    X = rng.uniform(-cube / 2, cube / 2, size=(points, 3))
    oc, op, keep = _tracks(rng, poses, cams, X, track, 1024, 768, geometric=False)
    X = X[keep]
    options = {"iterations": 30, "huberPx": 2.0, "cgRelativeTolerance": 1e-6, "refineSharedFocal": True}
    return finish(f"helix-{cameras}x{points}", rng, poses, cams, X, oc, op, width=1024, height=768,
                  options={**options, **kw.pop("options", {})}, **kw)


def sphere_scene(seed=2, cameras=1500, points=1_000_000, radius=20.0, clusters=64, sigma=0.5, ball=10.0,
                 track_mean=6.0, track=(2, 40), **kw) -> Scene:
    """Configuration 2: 1,500 cameras on a jittered 20 m sphere facing its centre, 1M points
    from 64 Gaussians (sigma 0.5 m) inside a 10 m ball, geometric tracks (mean 6, 2-40)."""
    rng = np.random.default_rng(seed)
    k = np.arange(cameras) + 0.5
    phi = np.arccos(1 - 2 * k / cameras)
    th = np.pi * (1 + 5**0.5) * k
    dirs = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    dirs += rng.normal(scale=0.02, size=dirs.shape)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    centers = radius * dirs
    poses = poses_from(look_at(centers, np.zeros_like(centers)), centers)
    cams = intrinsics(cameras)
    cams[:, 0] = cams[:, 1] = rng.uniform(700, 900, cameras)
    mu = rng.normal(size=(clusters, 3))
    mu *= (ball - 3 * sigma) * rng.random((clusters, 1)) ** (1 / 3) / np.linalg.norm(mu, axis=1, keepdims=True)
    X = mu[rng.integers(0, clusters, points)] + rng.normal(scale=sigma, size=(points, 3))
    r = np.linalg.norm(X, axis=1)
    X[r > ball] *= (ball / r[r > ball])[:, None]
    oc, op, keep = _tracks(rng, poses, cams, X, track, 1024, 768, geometric=True, mean=track_mean)
    X = X[keep]
    options = {"iterations": 10, "huberPx": 2.0, "cgRelativeTolerance": 1e-6, "refineSharedFocal": True}
    return finish(f"sphere-{cameras}x{points}", rng, poses, cams, X, oc, op, width=1024, height=768,
                  options={**options, **kw.pop("options", {})}, **kw)


def _tracks(rng, poses, cams, X, track, width, height, geometric, mean=6.0, candidates=48, chunk=200_000):
    """Each point's observing cameras: a random home camera that sees it and its nearest
    cameras (by centre distance) that see it, up to the point's track length."""
    C, P = len(poses), len(X)
    R = poses[:, :9].reshape(-1, 3, 3)
    centers = -np.einsum("cji,cj->ci", R, poses[:, 9:])
    d2 = ((centers[:, None, :] - centers[None, :, :]) ** 2).sum(-1)
    K = min(candidates, C)
    knn = np.argsort(d2, axis=1)[:, :K]
    lo, hi = track
    if geometric:
        want = np.clip(rng.geometric(1.0 / mean, size=P), lo, hi)
    else:
        want = rng.integers(lo, hi + 1, size=P)
    home = rng.integers(0, C, size=P)
    for _ in range(16):  # re-draw homes that do not see their point
        bad = ~visible(poses, cams, home, X, width, height)
        if not bad.any():
            break
        home[bad] = rng.integers(0, C, size=int(bad.sum()))
    cams_out, pts_out = [], []
    for s in range(0, P, chunk):
        e = min(P, s + chunk)
        cand = knn[home[s:e]]  # n x K, home first
        n = e - s
        vis = visible(poses, cams, cand.reshape(-1), np.repeat(X[s:e], K, axis=0), width, height).reshape(n, K)
        rank = np.cumsum(vis, axis=1)
        take = vis & (rank <= want[s:e, None])
        ok = take.sum(1) >= lo
        take &= ok[:, None]
        rows, cols = np.nonzero(take)
        cc = cand[rows, cols]
        order = np.lexsort((cc, rows))
        cams_out.append(cc[order])
        pts_out.append(rows[order] + s)
    oc = np.concatenate(cams_out)
    op = np.concatenate(pts_out)
    # drop points with too short a track and renumber
    counts = np.bincount(op, minlength=P)
    keep = counts >= lo
    remap = np.cumsum(keep) - 1
    sel = keep[op]
    return oc[sel], remap[op[sel]], keep


def arc_scene(seed=0, cameras=20, points=5000, radius=5.0, cube=2.0, spacing=np.pi / 24, track=(2, 10),
              **kw) -> Scene:
    """A local window of configuration 3: cameras evenly on an arc of the 5 m ring of
    configuration 0 (7.5 degrees apart) facing the origin, points uniform in a 2 m cube, each kept
    in a uniform 2-10 of the nearest cameras that see it."""
    rng = np.random.default_rng(seed)
    ang = spacing * (np.arange(cameras) - (cameras - 1) / 2)
    centers = np.stack([radius * np.cos(ang), radius * np.sin(ang), np.zeros(cameras)], axis=1)
    poses = poses_from(look_at(centers, np.zeros_like(centers)), centers)
    cams = intrinsics(cameras)
    X = rng.uniform(-cube / 2, cube / 2, size=(points, 3))
    oc, op, keep = _tracks(rng, poses, cams, X, track, 1024, 768, geometric=False)
    X = X[keep]
    options = {"iterations": 10, "huberPx": 2.0, "cgRelativeTolerance": 1e-6, "refineSharedFocal": False}
    return finish(f"arc-{cameras}x{points}", rng, poses, cams, X, oc, op, width=1024, height=768,
                  options={**options, **kw.pop("options", {})}, **kw)


def batch_scenes(seed=3, count=512, cameras=(5, 40), points=(500, 20_000), track=(2, 10)) -> list[Scene]:
    """Configuration 3: `count` independent arc windows, camera counts uniform in 5-40, point
    counts log-uniform in 500-20,000, each drawn from its own sub-seed."""
    rng = np.random.default_rng(seed)
    Cs = rng.integers(cameras[0], cameras[1] + 1, size=count)
    Ps = np.rint(np.exp(rng.uniform(np.log(points[0]), np.log(points[1]), size=count))).astype(int)
    subs = rng.integers(0, 2**31 - 1, size=count)
    return [arc_scene(int(s), int(c), int(p), track=track) for s, c, p in zip(subs, Cs, Ps)]


CONFIGS = {
    "cfg0": lambda: ring_scene(),
    "cfg1": lambda: helix_scene(),
    "cfg2": lambda: sphere_scene(),
}


def inverse_depth_rows(seed=5, measurements=4 << 20, cameras=512, radius=5.0, cube=2.0, reach=8) -> np.ndarray:
    """(measurements x 34) rows: a point uniform in a cube about the origin, anchored in a ring camera
    (a, b the normalised bearing, rho the inverse depth), observed by one of the `reach` cameras that
    follow its anchor on the ring; the cameras carry the intrinsics of ``intrinsics`` and their
    squared radial limit."""
    rng = np.random.default_rng(seed)
    angles = np.arange(cameras) * (2 * np.pi / cameras)
    centers = np.stack([radius * np.cos(angles), radius * np.sin(angles), 0.3 * np.sin(3 * angles)], axis=1)
    poses = poses_from(look_at(centers, np.zeros((cameras, 3))), centers)
    K = intrinsics(cameras)
    k1 = K[:, 4]
    limit = np.where(k1 < 0, -1 / (3 * np.where(k1 < 0, k1, -1)), 1e30)
    ref = rng.integers(0, cameras, measurements)
    obs = (ref + rng.integers(1, reach + 1, measurements)) % cameras
    X = rng.uniform(-cube / 2, cube / 2, (measurements, 3))
    R = poses[ref, :9].reshape(-1, 3, 3)
    q = np.einsum("nij,nj->ni", R, X) + poses[ref, 9:]
    rows = np.empty((measurements, 34))
    rows[:, 0] = q[:, 0] / q[:, 2]
    rows[:, 1] = q[:, 1] / q[:, 2]
    rows[:, 2] = 1 / q[:, 2]
    rows[:, 3:15] = poses[ref]
    rows[:, 15:27] = poses[obs]
    rows[:, 27:33] = K[obs, :6]
    rows[:, 33] = limit[obs]
    return rows



def inverse_depth_corridor(seed=11, views=120, window=4, points=12, noise_px=0.2, pose_noise=0.004,
                           point_noise=0.02) -> dict:
    """{"views", "landmarks"} records: `views` cameras with identity rotation whose centres follow
    a corridor (0.3 apart along x, small sinusoidal y and z), the camera of the inverse-depth
    fixtures (fx 800, fy 760, cx 320, cy 240, k1 -0.03); every run of `window` consecutive views
    sees `points` points of its own, 5-8 in front.  Pixels are exact projections plus Gaussian
    noise; the views after the first and the points start perturbed."""
    rng = np.random.default_rng(seed)
    camera = {"fx": 800.0, "fy": 760.0, "cx": 320.0, "cy": 240.0, "k1": -0.03}
    i = np.arange(views)
    centres = np.stack([0.3 * i, 0.04 * np.sin(i), 0.02 * np.sin(0.2 * i)], axis=1)
    out_views = []
    for k in range(views):
        t = -centres[k]
        if k:
            t = t + rng.normal(0, pose_noise, 3)
        out_views.append({"id": k, "camera": dict(camera), "pose": {"R": np.eye(3).ravel(), "t": t}})
    landmarks = []
    for start in range(views - window + 1):
        lo, hi = centres[start, 0], centres[start + window - 1, 0]
        X = np.stack([rng.uniform(lo - 1, hi + 1, points), rng.uniform(-1, 1, points), rng.uniform(5, 8, points)],
                     axis=1)
        for j in range(points):
            track = start * points + j
            q = X[j][None, :] - centres[start:start + window]
            x, y = q[:, 0] / q[:, 2], q[:, 1] / q[:, 2]
            d = 1 + camera["k1"] * (x * x + y * y)
            u = camera["fx"] * x * d + camera["cx"] + rng.normal(0, noise_px, window)
            v = camera["fy"] * y * d + camera["cy"] + rng.normal(0, noise_px, window)
            landmarks.append({"trackId": track, "xyz": X[j] + rng.normal(0, point_noise, 3),
                              "observations": [{"viewId": start + w, "featureId": track, "pixel": [float(u[w]), float(v[w])]}
                                               for w in range(window)]})
    return {"views": out_views, "landmarks": landmarks}
