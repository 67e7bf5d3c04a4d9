"""Seeded synthetic bundle-adjustment scenes and their Jacobians.

No public dataset backs the benchmark configurations, so scenes are generated
with the shapes and value distributions the configurations describe. The
camera model is the 9-parameter Snavely model of uncertaintyTE
(snavely_reprojection_error.h:309-370, unit weights):

    pC = X - C;  p = R(aa) pC;  xp = p0/p2, yp = p1/p2
    r2 = xp^2 + yp^2;  d = 1 + k1 r2 + k2 r2^2;  residual = f * (xp, yp) * d - obs

with camera parameters [aa(3), C(3), f, k1, k2] and point parameters X(3).
The Jacobian is the analytic 2x9 / 2x3 block per observation, evaluated at
ground truth, laid out as the reference expects: observations sorted by
point, two consecutive CRS rows of 12 entries (9 camera columns then 3 point
columns).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .jacob import Jacobian


@dataclasses.dataclass
class Scene:
    cams: np.ndarray  # (C, 9): aa, C, f, k1, k2
    points: np.ndarray  # (P, 3)
    obs_cam: np.ndarray  # (nobs,)
    obs_pt: np.ndarray  # (nobs,)


def _look_at_aa(centers: np.ndarray, target: np.ndarray) -> np.ndarray:
    """Angle-axis of world->camera rotations whose +z axis points at target."""
    z = target[None, :] - centers
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    up = np.tile(np.array([0.0, 0.0, 1.0]), (len(z), 1))
    par = np.abs((z * up).sum(1)) > 0.95
    up[par] = np.array([0.0, 1.0, 0.0])
    x = np.cross(up, z)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    R = np.stack([x, y, z], axis=1)  # rows: camera axes in world coordinates
    return _rot_to_aa(R)


def _rot_to_aa(R: np.ndarray) -> np.ndarray:
    tr = np.clip((np.trace(R, axis1=1, axis2=2) - 1) / 2, -1.0, 1.0)
    th = np.arccos(tr)
    w = np.stack([R[:, 2, 1] - R[:, 1, 2], R[:, 0, 2] - R[:, 2, 0], R[:, 1, 0] - R[:, 0, 1]], axis=1)
    s = np.sin(th)
    small = s < 1e-8
    scale = np.where(small, 0.5, th / (2 * np.where(small, 1.0, s)))
    aa = w * scale[:, None]
    # near pi: fall back to the symmetric part
    bad = th > np.pi - 1e-6
    if bad.any():
        for i in np.where(bad)[0]:
            B = (R[i] + np.eye(3)) / 2
            k = np.argmax(np.diag(B))
            v = B[:, k] / np.sqrt(B[k, k])
            aa[i] = v * th[i]
    return aa


def _aa_to_rot(aa: np.ndarray) -> np.ndarray:
    th = np.linalg.norm(aa, axis=1)
    k = aa / np.where(th > 0, th, 1.0)[:, None]
    K = np.zeros((len(aa), 3, 3))
    K[:, 0, 1], K[:, 0, 2] = -k[:, 2], k[:, 1]
    K[:, 1, 0], K[:, 1, 2] = k[:, 2], -k[:, 0]
    K[:, 2, 0], K[:, 2, 1] = -k[:, 1], k[:, 0]
    s, c = np.sin(th)[:, None, None], np.cos(th)[:, None, None]
    return np.eye(3)[None] + s * K + (1 - c) * (K @ K)


def _skew(v: np.ndarray) -> np.ndarray:
    S = np.zeros(v.shape[:-1] + (3, 3))
    S[..., 0, 1], S[..., 0, 2] = -v[..., 2], v[..., 1]
    S[..., 1, 0], S[..., 1, 2] = v[..., 2], -v[..., 0]
    S[..., 2, 0], S[..., 2, 1] = -v[..., 1], v[..., 0]
    return S


def _right_jacobian(aa: np.ndarray) -> np.ndarray:
    """J_r(w) with R(w + d) ~= R(w) Exp(J_r(w) d)."""
    th = np.linalg.norm(aa, axis=1)
    W = _skew(aa)
    W2 = W @ W
    small = th < 1e-6
    ths = np.where(small, 1.0, th)
    a = np.where(small, 0.5, (1 - np.cos(ths)) / ths ** 2)
    b = np.where(small, 1.0 / 6.0, (ths - np.sin(ths)) / ths ** 3)
    return np.eye(3)[None] - a[:, None, None] * W + b[:, None, None] * W2


def observation_blocks(cams: np.ndarray, points: np.ndarray, obs_cam: np.ndarray,
                       obs_pt: np.ndarray):
    """Analytic Jacobian blocks: returns (Jc (n,2,9), Jp (n,2,3)).

    The rotation and its right Jacobian are formed once per camera and
    gathered per observation (each matrix is computed on its own, so the
    values do not depend on how many are formed together)."""
    Cc = cams[obs_cam, 3:6]
    f = cams[obs_cam, 6]
    k1 = cams[obs_cam, 7]
    k2 = cams[obs_cam, 8]
    X = points[obs_pt]
    R = _aa_to_rot(cams[:, 0:3])[obs_cam]
    Jr = _right_jacobian(cams[:, 0:3])[obs_cam]
    pC = X - Cc
    p = np.einsum("nij,nj->ni", R, pC)
    xp, yp, z = p[:, 0] / p[:, 2], p[:, 1] / p[:, 2], p[:, 2]
    r2 = xp * xp + yp * yp
    d = 1 + k1 * r2 + k2 * r2 * r2
    g = k1 + 2 * k2 * r2
    M = np.empty((len(f), 2, 2))
    M[:, 0, 0] = f * (d + 2 * xp * xp * g)
    M[:, 0, 1] = f * 2 * xp * yp * g
    M[:, 1, 0] = f * 2 * xp * yp * g
    M[:, 1, 1] = f * (d + 2 * yp * yp * g)
    Q = np.zeros((len(f), 2, 3))
    Q[:, 0, 0] = 1 / z
    Q[:, 0, 2] = -p[:, 0] / (z * z)
    Q[:, 1, 1] = 1 / z
    Q[:, 1, 2] = -p[:, 1] / (z * z)
    dUdp = M @ Q  # (n,2,3)
    Jp = dUdp @ R  # d/dX
    Jc = np.empty((len(f), 2, 9))
    Jc[:, :, 0:3] = -dUdp @ R @ _skew(pC) @ Jr
    Jc[:, :, 3:6] = -Jp
    Jc[:, 0, 6], Jc[:, 1, 6] = xp * d, yp * d
    Jc[:, 0, 7], Jc[:, 1, 7] = f * xp * r2, f * yp * r2
    Jc[:, 0, 8], Jc[:, 1, 8] = f * xp * r2 * r2, f * yp * r2 * r2
    return Jc, Jp


def project(cams: np.ndarray, points: np.ndarray, obs_cam: np.ndarray, obs_pt: np.ndarray):
    """Residual-free projections (u, v) for finite-difference checks."""
    R = _aa_to_rot(cams[obs_cam, 0:3])
    p = np.einsum("nij,nj->ni", R, points[obs_pt] - cams[obs_cam, 3:6])
    xp, yp = p[:, 0] / p[:, 2], p[:, 1] / p[:, 2]
    r2 = xp * xp + yp * yp
    d = 1 + cams[obs_cam, 7] * r2 + cams[obs_cam, 8] * r2 * r2
    return np.stack([cams[obs_cam, 6] * xp * d, cams[obs_cam, 6] * yp * d], axis=1)


def farthest_triple(points: np.ndarray) -> np.ndarray:
    """Deterministic fixed points: a locally largest-perimeter triangle, sorted."""
    cen = points.mean(0)
    dist = lambda i: np.linalg.norm(points - points[i], axis=1)
    a = int(np.argmax(np.linalg.norm(points - cen, axis=1)))
    da = dist(a)
    b = int(np.argmax(da))
    db = dist(b)
    s = da + db
    s[[a, b]] = -1
    c = int(np.argmax(s))
    for _ in range(16):
        db, dc = dist(b), dist(c)
        s = db + dc
        s[[b, c]] = -1
        a2 = int(np.argmax(s))
        da, dc = dist(a2), dist(c)
        s = da + dc
        s[[a2, c]] = -1
        b2 = int(np.argmax(s))
        da, db = dist(a2), dist(b2)
        s = da + db
        s[[a2, b2]] = -1
        c2 = int(np.argmax(s))
        same = (a2, b2, c2) == (a, b, c)
        a, b, c = a2, b2, c2
        if same:
            break
    return np.sort(np.array([a, b, c], dtype=np.int32))


def _choose(rng, n_pts, counts, pool_size, pool_offset):
    """For each point pick counts[p] distinct cameras from its pool window."""
    kmax = int(counts.max())
    keys = rng.random((n_pts, pool_size), dtype=np.float32)
    order = np.argsort(keys, axis=1)[:, :kmax]
    sel = order + pool_offset[:, None]
    mask = np.arange(kmax)[None, :] < counts[:, None]
    return sel, mask


def make_scene(name: str, seed: int = 0) -> Scene:
    """Synthetic scenes of the benchmark configurations.

    small : 10 cams on a ring r=10, 500 pts in [-1,1]^3, 2+Poisson(4) views/pt
    medium: 200 cams on a sphere cap r=20, 50k pts in a 4x4x2 box, 2+Poisson(5)
    large : 2000 cams on a 3-loop trajectory, 500k pts, 2+Poisson(5), f ~ U(500,3000)
    tiny  : 6 cams, 40 pts (unit tests)
    """
    rng = np.random.default_rng(seed)
    if name in ("small", "tiny"):
        C, P, lam = (10, 500, 4) if name == "small" else (6, 40, 3)
        ang = 2 * np.pi * np.arange(C) / C
        centers = np.stack([10 * np.cos(ang), 10 * np.sin(ang), rng.uniform(-0.5, 0.5, C)], 1)
        f = rng.uniform(800, 1200, C)
        pts = rng.uniform(-1, 1, (P, 3))
        window = None
    elif name == "medium":
        C, P, lam = 200, 50_000, 5
        th = np.arccos(rng.uniform(np.cos(np.radians(60)), np.cos(np.radians(15)), C))
        ph = rng.uniform(0, 2 * np.pi, C)
        centers = 20 * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
        f = rng.uniform(800, 1200, C)
        pts = rng.uniform([-2, -2, -1], [2, 2, 1], (P, 3))
        window = None
    elif name == "large":
        C, P, lam = 2000, 500_000, 5
        loop = np.arange(C) % 3
        ang = 3 * 2 * np.pi * np.arange(C) / C + 0.01 * rng.standard_normal(C)
        rad = np.array([25.0, 30.0, 35.0])[loop] + rng.uniform(-1, 1, C)
        hgt = np.array([-4.0, 0.0, 4.0])[loop] + rng.uniform(-0.5, 0.5, C)
        centers = np.stack([rad * np.cos(ang), rad * np.sin(ang), hgt], 1)
        f = rng.uniform(500, 3000, C)
        pts = rng.uniform([-6, -6, -2], [6, 6, 2], (P, 3))
        window = 96
    else:
        raise ValueError(f"unknown scene {name!r}")
    aa = _look_at_aa(centers, np.zeros(3))
    k12 = rng.normal(0, 1e-2, (C, 2))
    cams = np.concatenate([aa, centers, f[:, None], k12], axis=1)
    counts = np.minimum(2 + rng.poisson(lam, P), C if window is None else window)
    if window is None:
        sel, mask = _choose(rng, P, counts, C, np.zeros(P, dtype=np.int64))
    else:
        # cameras along the trajectory whose azimuth is closest to the point's
        cam_az = np.mod(np.arctan2(centers[:, 1], centers[:, 0]), 2 * np.pi)
        order = np.argsort(cam_az)
        pt_az = np.mod(np.arctan2(pts[:, 1], pts[:, 0]), 2 * np.pi)
        idx = np.searchsorted(cam_az[order], pt_az)
        start = np.clip(idx - window // 2 + rng.integers(-8, 9, P), 0, C - window)
        sel, mask = _choose(rng, P, counts, window, start)
        sel = order[sel]
    obs_pt = np.repeat(np.arange(P), counts)
    obs_cam = sel[mask]
    # sort cameras ascending within each point (observations are point-major)
    key = obs_pt.astype(np.int64) * (C + 1) + obs_cam
    o = np.argsort(key, kind="stable")
    return Scene(cams, pts, obs_cam[o].astype(np.int32), obs_pt[o].astype(np.int32))


def make_sized_scene(num_cams: int, points_per_cam: int, lam: float, seed: int = 0, window: int = 48) -> Scene:
    """A scene of any size for the batched and serving workloads: num_cams
    cameras on a sphere cap (r = 20, 15-60 degrees from the pole) looking at
    the origin, f ~ U(800, 1200), k1, k2 ~ N(0, 1e-2); points_per_cam * num_cams
    points uniform in a 4 x 4 x 2 box; each point seen by 2 + Poisson(lam)
    distinct cameras drawn from the `window` cameras nearest to it in azimuth."""
    rng = np.random.default_rng(seed)
    C, P = int(num_cams), int(points_per_cam) * int(num_cams)
    th = np.arccos(rng.uniform(np.cos(np.radians(60)), np.cos(np.radians(15)), C))
    ph = rng.uniform(0, 2 * np.pi, C)
    centers = 20 * np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    f = rng.uniform(800, 1200, C)
    pts = rng.uniform([-2, -2, -1], [2, 2, 1], (P, 3))
    aa = _look_at_aa(centers, np.zeros(3))
    k12 = rng.normal(0, 1e-2, (C, 2))
    cams = np.concatenate([aa, centers, f[:, None], k12], axis=1)
    w = min(window, C)
    counts = np.minimum(2 + rng.poisson(lam, P), w)
    order = np.argsort(ph)
    pt_az = np.mod(np.arctan2(pts[:, 1], pts[:, 0]), 2 * np.pi)
    idx = np.searchsorted(ph[order], pt_az)
    start = np.clip(idx - w // 2, 0, C - w)
    sel, mask = _choose(rng, P, counts, w, start)
    sel = order[sel]
    obs_pt = np.repeat(np.arange(P), counts)
    obs_cam = sel[mask]
    key = obs_pt.astype(np.int64) * (C + 1) + obs_cam
    o = np.argsort(key, kind="stable")
    return Scene(cams, pts, obs_cam[o].astype(np.int32), obs_pt[o].astype(np.int32))


def sample_camera_counts(n: int, median: float, sigma: float, lo: int, hi: int, seed: int) -> np.ndarray:
    """Camera counts lognormal(median, sigma) clipped to [lo, hi] (batched / serving workloads)."""
    rng = np.random.default_rng(seed)
    return np.clip(np.round(median * np.exp(sigma * rng.standard_normal(n))), lo, hi).astype(int)


def scene_jacobian(scene: Scene, with_fixed: bool = True) -> Jacobian:
    """CRS Jacobian (reference layout) of a synthetic scene."""
    C, P = len(scene.cams), len(scene.points)
    n = len(scene.obs_cam)
    Jc, Jp = observation_blocks(scene.cams, scene.points, scene.obs_cam, scene.obs_pt)
    vals = np.empty((n, 2, 12))
    vals[:, :, 0:9] = Jc
    vals[:, :, 9:12] = Jp
    cols = np.empty((n, 2, 12), dtype=np.int32)
    cols[:, :, 0:9] = (9 * scene.obs_cam)[:, None, None] + np.arange(9)[None, None, :]
    cols[:, :, 9:12] = (9 * C + 3 * scene.obs_pt)[:, None, None] + np.arange(3)[None, None, :]
    rows = (12 * np.arange(2 * n + 1)).astype(np.int32)
    fix = farthest_triple(scene.points) if with_fixed else None
    return Jacobian(C, 9, P, n, 2 * n, 9 * C + 3 * P, rows, cols.reshape(-1),
                    vals.reshape(-1).copy(), -1.0, fix, algorithm=2, epsilon=1e-10, svd_remove_n=7)


def synthetic_jacobian(name: str, seed: int = 0) -> Jacobian:
    return scene_jacobian(make_scene(name, seed))
