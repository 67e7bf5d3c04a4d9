"""`.jacob` input and `.cov` output formats of uncertaintyTE.

`.jacob` (JacobianIO.cpp:32-63; documented in
test/input_jacobians/template_of_jacobian.txt): whitespace-separated text

    lambda numCams camParams numPoints numObs
    fix0 fix1 fix2                    (-1 -1 -1 = none)
    nrows ncols nnz
    rowptr[nrows+1]  cols[nnz]  values[nnz]

Loading a `.jacob` file forces TAYLOR_EXPANSION, epsilon 1e-10 and
svdRemoveN 7 (JacobianIO.cpp:25,40-43); `load_jacob` returns those defaults.

`.cov` (IO.cpp:15-60): '#' header lines with the statistics, then one line of
45 values per camera and one line of 6 values per point, written with the
default 6-significant-digit stream formatting.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np

ALGORITHMS = {"SVD_QR_ITERATION": 0, "SVD_DEVIDE_AND_CONQUER": 1, "TAYLOR_EXPANSION": 2}
ALGORITHM_NAMES = {v: k for k, v in ALGORITHMS.items()}


@dataclasses.dataclass
class Jacobian:
    """A Ceres-style CRS Jacobian plus the scene header of a `.jacob` file."""

    num_cams: int
    cam_params: int
    num_points: int
    num_obs: int
    num_rows: int
    num_cols: int
    rows: np.ndarray  # int32 rowptr, num_rows + 1
    cols: np.ndarray  # int32, nnz
    values: np.ndarray  # float64, nnz
    lam: float = -1.0
    pts2fix: Optional[np.ndarray] = None  # 3 ints or None
    algorithm: int = 2
    epsilon: float = 1e-10
    svd_remove_n: int = 7

    @property
    def nnz(self) -> int:
        return int(self.rows[-1])


def _tokens(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        data = f.read()
    if b"#" in data:  # strip comment lines (the documented template carries some)
        data = b"\n".join(l.split(b"#", 1)[0] for l in data.splitlines())
    return np.array(data.split(), dtype=np.float64)


def load_jacob(path: str) -> Jacobian:
    """Read a `.jacob` file (JacobianIO::loadJacobian, JacobianIO.cpp:32-63), text
    or binary, with the library's parallel parser."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"The input file doesn't exist: {path}")
    from . import native
    return native.read_jacob(path)


def load_jacob_numpy(path: str) -> Jacobian:
    """The same with numpy alone (one Python token per number: small files)."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"The input file doesn't exist: {path}")
    t = _tokens(path)
    lam, nc, cp, npts, nobs = t[0], int(t[1]), int(t[2]), int(t[3]), int(t[4])
    fix = t[5:8].astype(np.int64)
    nr, ncol, nnz = int(t[8]), int(t[9]), int(t[10])
    o = 11
    need = o + (nr + 1) + 2 * nnz
    if t.size < need:
        raise ValueError(f"truncated .jacob file {path}: {t.size} tokens, {need} needed")
    rows = t[o:o + nr + 1].astype(np.int32)
    o += nr + 1
    cols = t[o:o + nnz].astype(np.int32)
    o += nnz
    vals = np.ascontiguousarray(t[o:o + nnz])
    pts2fix = fix.astype(np.int32) if (fix >= 0).all() else None
    return Jacobian(nc, cp, npts, nobs, nr, ncol, rows, cols, vals, float(lam), pts2fix,
                    algorithm=2, epsilon=1e-10, svd_remove_n=7)


def save_jacob(path: str, j: Jacobian) -> None:
    """Write a `.jacob` file in the reference's layout (full double precision)."""
    fix = j.pts2fix if j.pts2fix is not None else np.array([-1, -1, -1])
    with open(path, "w") as f:
        lam = int(j.lam) if j.lam == -1 else repr(float(j.lam))
        f.write(f"{lam} {j.num_cams} {j.cam_params} {j.num_points} {j.num_obs}\n")
        f.write(f"{int(fix[0])} {int(fix[1])} {int(fix[2])}\n")
        f.write(f"{j.num_rows} {j.num_cols} {j.nnz}\n")
        f.write(" ".join(map(str, j.rows.tolist())) + "\n")
        f.write(" ".join(map(str, j.cols.tolist())) + "\n")
        f.write(" ".join(f"{v:.17g}" for v in j.values.tolist()) + "\n")


def _g6(x: float) -> str:
    """C++ ostream default formatting (%g with 6 significant digits)."""
    return f"{x:g}"


def save_cov(path: str, j: Jacobian, stats: dict, cam_unc: np.ndarray, pt_unc: np.ndarray,
             algorithm: int = 2) -> None:
    """Write a `.cov` file with the header keys of saveResults (IO.cpp:15-60).

    Times are written in true seconds (the reference's timer prints ms/100)."""
    per_cam = j.cam_params * (j.cam_params + 1) // 2
    L = ["# ---- Covariance v0.1 ----",
         f"# Number of cameras: {j.num_cams}",
         f"# Number of camera parameters: {j.cam_params}",
         f"# Number of points in 3D: {j.num_points}",
         f"# Number of observations: {j.num_obs}",
         f"# Used algorithm: {ALGORITHM_NAMES.get(algorithm, 'not defined')}"]
    if algorithm == 2:
        fp = stats.get("fixed_pts")
        if fp is not None:
            L.append(f"# Fixed points: {fp[0]}, {fp[1]}, {fp[2]}")
        L.append(f"# Used lambda: {_g6(stats.get('lambda', 0.0))}")
        for key, name in [("time_create_j", "Loading jacobian time"),
                          ("time_norm_j", "Normalization of jacobian time"),
                          ("time_multiply_jj", "Compose information matrix time"),
                          ("time_split_jj", "Split infromation matrix time"),
                          ("time_inv_v", "Inverse V time"),
                          ("time_compose_z", "Compose Z time"),
                          ("time_inv_z", "Inverse Z time"),
                          ("time_te", "Taylor expansion time"),
                          ("time_pts_unc", "Point uncertainty time")]:
            L.append(f"# {name}: {_g6(stats.get(key, 0.0))}s")
        cc = list(stats.get("cycle_change", []))
        L.append(f"# TE number of iterations: {len(cc)}")
        L.append("# TE cycle change: " + "".join(_g6(c) + " " for c in cc))
    L.append(f"# Time of the algorithm: {_g6(stats.get('time_all', 0.0))}s")
    L.append("# -----------------------")
    cam = np.asarray(cam_unc).reshape(j.num_cams, per_cam)
    for r in cam:
        L.append("".join(_g6(v) + " " for v in r))
    pt = np.asarray(pt_unc).reshape(j.num_points, 6)
    for r in pt:
        L.append("".join(_g6(v) + " " for v in r))
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def load_cov(path: str, num_cams: int, cam_params: int = 9):
    """Parse a `.cov` file: returns (header dict, cam (C, p(p+1)/2), pt (P, 6))."""
    hdr = {}
    cams, pts = [], []
    per_cam = cam_params * (cam_params + 1) // 2
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                if ":" in line:
                    k, v = line[1:].split(":", 1)
                    hdr[k.strip()] = v.strip()
                continue
            if len(line.strip()) == 0:
                continue
            vals = [float(x) for x in line.split()]
            (cams if len(cams) < num_cams else pts).append(vals)
    cam = np.array(cams, dtype=np.float64).reshape(-1, per_cam)
    pt = np.array(pts, dtype=np.float64).reshape(-1, 6)
    return hdr, cam, pt
