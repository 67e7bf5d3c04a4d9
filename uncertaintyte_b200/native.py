"""ctypes binding of libuncte.so (the C ABI in include/uncte.h).

The product path is the CUDA library; there is no CPU fallback. Importing
this module without the built library raises ImportError, and every call
returns the library's status as an UncError.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .jacob import Jacobian

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libuncte.so")

UNC_OK = 0
UNC_ERR_TIMEOUT = -9  # unc_server_wait: the request is still running
TAYLOR_EXPANSION = 2
SVD_QR_ITERATION = 0
SVD_SCHUR = 3  # extension: SVD pseudo-inverse of the camera Schur complement
SVD_DEVIDE_AND_CONQUER = 1
PRECISION = {"fp64": 0, "mixed": 1, "mixed4": 2, "mixed3": 3}


class UncError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class UncOptions(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int),
        ("epsilon", C.c_double),
        ("lam", C.c_double),
        ("num_cams", C.c_int),
        ("cam_params", C.c_int),
        ("num_points", C.c_int),
        ("num_obs", C.c_int),
        ("svd_remove_n", C.c_int),
        ("max_iter_te", C.c_int),
        ("pts2fix", C.c_int * 3),
        ("has_pts2fix", C.c_int),
        ("precision", C.c_int),
        ("taylor_eval", C.c_int),
    ]


class UncStatistic(C.Structure):
    _fields_ = [
        ("time_create_j", C.c_double),
        ("time_fix_j", C.c_double),
        ("time_norm_j", C.c_double),
        ("time_multiply_jj", C.c_double),
        ("time_split_jj", C.c_double),
        ("time_inv_v", C.c_double),
        ("time_compose_z", C.c_double),
        ("time_inv_z", C.c_double),
        ("time_te", C.c_double),
        ("time_pts_unc", C.c_double),
        ("time_all", C.c_double),
        ("lam", C.c_double),
        ("fixed_pts", C.c_int * 3),
        ("te_iterations", C.c_int),
        ("cycle_change", C.c_double * 20),
        ("device_bytes", C.c_longlong),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("fixed_pts", "cycle_change", "lam")}
        d["lambda"] = self.lam
        d["fixed_pts"] = list(self.fixed_pts)
        d["cycle_change"] = list(self.cycle_change[: self.te_iterations])
        return d


# every symbol declared in include/uncte.h
EXPORTS = ("unc_options_init", "unc_context_create", "unc_context_destroy", "unc_compute",
           "unc_context_set_profiling", "unc_context_profile", "unc_context_profile_int8",
           "unc_compute_device", "unc_workspace_bytes", "unc_dense_inverse_device",
           "unc_dense_inverse_noalloc", "unc_spd_task_list", "unc_spd_inverse_tasks_bounded", "unc_pinv_psd_device", "unc_jtj_crs",
           "unc_gemm_f64_device", "unc_gemm_mixed_device", "unc_gram_lower_mixed_device", "unc_status_string",
           "unc_last_error",
           "unc_kernel_launches", "unc_request_bytes", "unc_context_device_bytes", "unc_context_release",
           "unc_context_set_priority", "unc_jacobian_device", "unc_compute_scene",
           "unc_block_eigen_device", "unc_block_eigen", "unc_jacob_read_header", "unc_jacob_read",
           "unc_jacob_write_binary",
           "unc_server_create", "unc_server_submit", "unc_server_wait", "unc_server_destroy",
           "unc_batch_create", "unc_batch_destroy", "unc_batch_compute", "unc_batch_last_timing",
           "unc_batch_device_bytes", "unc_batch_release", "unc_batch_set_tile_width")

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C uncertaintyte_b200/csrc` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    L.unc_options_init.argtypes = [P(UncOptions), C.c_int, C.c_int, C.c_int, C.c_int]
    L.unc_options_init.restype = None
    L.unc_context_create.argtypes = [C.c_int, P(vp)]
    L.unc_context_destroy.argtypes = [vp]
    L.unc_compute.argtypes = [vp, P(UncOptions), C.c_int, C.c_int, vp, vp, vp, vp, vp, P(UncStatistic)]
    L.unc_compute_device.argtypes = [vp, P(UncOptions), C.c_int, C.c_int, vp, vp, vp, vp, vp,
                                     P(UncStatistic), vp]
    L.unc_context_set_profiling.argtypes = [vp, C.c_int]
    L.unc_context_profile.argtypes = [vp, P(C.c_longlong), P(C.c_double), P(C.c_double), C.c_int]
    L.unc_context_profile_int8.argtypes = [vp, P(C.c_double)]
    L.unc_workspace_bytes.argtypes = [P(UncOptions), C.c_int, C.c_int]
    L.unc_workspace_bytes.restype = C.c_longlong
    L.unc_dense_inverse_device.argtypes = [vp, C.c_int, C.c_int, vp]
    L.unc_dense_inverse_noalloc.argtypes = [vp, C.c_int, C.c_int, vp]
    L.unc_spd_task_list.argtypes = [C.c_int, vp, C.c_int]
    L.unc_spd_inverse_tasks_bounded.argtypes = [vp, C.c_int, C.c_int, C.c_longlong, C.c_int, vp]
    L.unc_pinv_psd_device.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, vp]
    L.unc_request_bytes.argtypes = [P(UncOptions), C.c_int, C.c_int, vp, vp]
    L.unc_request_bytes.restype = C.c_longlong
    L.unc_context_device_bytes.argtypes = [vp]
    L.unc_context_device_bytes.restype = C.c_longlong
    L.unc_context_release.argtypes = [vp]
    L.unc_context_set_priority.argtypes = [vp, C.c_int]
    L.unc_jacob_read_header.argtypes = [C.c_char_p, P(UncJacobHeader)]
    L.unc_jacob_read.argtypes = [C.c_char_p, P(UncJacobHeader), vp, vp, vp]
    L.unc_jacob_write_binary.argtypes = [C.c_char_p, P(UncJacobHeader), vp, vp, vp]
    L.unc_block_eigen_device.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]
    L.unc_block_eigen.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
    L.unc_jacobian_device.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    L.unc_compute_scene.argtypes = [vp, P(UncOptions), vp, vp, vp, vp, vp, vp, P(UncStatistic)]
    L.unc_batch_create.argtypes = [C.c_int, P(vp)]
    L.unc_batch_destroy.argtypes = [vp]
    L.unc_batch_compute.argtypes = [vp, C.c_int, P(UncOptions), P(C.c_int), P(C.c_int), P(vp), P(vp), P(vp),
                                    P(vp), P(vp), P(C.c_int), P(UncStatistic)]
    L.unc_batch_last_timing.argtypes = [vp, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int), P(C.c_int)]
    L.unc_batch_device_bytes.argtypes = [vp]
    L.unc_batch_device_bytes.restype = C.c_longlong
    L.unc_batch_release.argtypes = [vp]
    L.unc_batch_set_tile_width.argtypes = [vp, C.c_int]
    L.unc_server_create.argtypes = [C.c_int, C.c_longlong, C.c_int, P(vp)]
    L.unc_server_submit.argtypes = [vp, P(UncOptions), C.c_int, C.c_int, vp, vp, vp, vp, vp, P(C.c_longlong)]
    L.unc_server_wait.argtypes = [vp, C.c_longlong, C.c_double, P(C.c_int), P(UncStatistic), P(C.c_double),
                                  P(C.c_double)]
    L.unc_server_destroy.argtypes = [vp]
    L.unc_jtj_crs.argtypes = [C.c_int, C.c_int, vp, vp, vp, C.c_int, C.c_int, P(C.c_longlong), vp,
                              vp, vp]
    L.unc_gemm_f64_device.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp, C.c_int,
                                      C.c_double, vp, C.c_int, vp]
    L.unc_gemm_mixed_device.argtypes = [C.c_int, vp, vp, C.c_int, vp, C.c_int, vp]
    L.unc_gram_lower_mixed_device.argtypes = [C.c_int, vp, C.c_int, vp, vp]
    L.unc_status_string.argtypes = [C.c_int]
    L.unc_status_string.restype = C.c_char_p
    L.unc_last_error.restype = C.c_char_p
    L.unc_kernel_launches.restype = C.c_longlong
    _lib = L
    return L


def _check(rc: int):
    if rc != UNC_OK:
        L = lib()
        raise UncError(rc, f"{L.unc_status_string(rc).decode()}: {L.unc_last_error().decode()}")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


TAYLOR_EVAL = {"powers": 0, "sequential": 1}


def make_options(jac: Jacobian, algorithm: Optional[int] = None, precision: str = "fp64",
                 lam: Optional[float] = None, taylor: str = "powers") -> UncOptions:
    o = UncOptions()
    lib().unc_options_init(C.byref(o), jac.num_cams, jac.cam_params, jac.num_points, jac.num_obs)
    o.algorithm = jac.algorithm if algorithm is None else algorithm
    o.epsilon = jac.epsilon
    o.lam = jac.lam if lam is None else lam
    o.svd_remove_n = jac.svd_remove_n
    if jac.pts2fix is not None:
        o.pts2fix[:] = [int(x) for x in jac.pts2fix]
        o.has_pts2fix = 1
    o.precision = PRECISION[precision]
    o.taylor_eval = TAYLOR_EVAL[taylor]
    return o


class UncJacobHeader(C.Structure):
    _fields_ = [("lam", C.c_double), ("num_cams", C.c_int), ("cam_params", C.c_int), ("num_points", C.c_int),
                ("num_obs", C.c_int), ("pts2fix", C.c_int * 3), ("num_rows", C.c_int), ("num_cols", C.c_int),
                ("nnz", C.c_longlong), ("binary", C.c_int)]


def read_jacob(path: str) -> Jacobian:
    """A `.jacob` file (text, parsed by all host threads, or the binary form) as a Jacobian."""
    h = UncJacobHeader()
    bp = os.fsencode(path)
    _check(lib().unc_jacob_read_header(bp, C.byref(h)))
    rows = np.empty(h.num_rows + 1, dtype=np.int32)
    cols = np.empty(h.nnz, dtype=np.int32)
    vals = np.empty(h.nnz, dtype=np.float64)
    _check(lib().unc_jacob_read(bp, C.byref(h), _ptr(rows), _ptr(cols), _ptr(vals)))
    fix = np.array(list(h.pts2fix), dtype=np.int32)
    return Jacobian(h.num_cams, h.cam_params, h.num_points, h.num_obs, h.num_rows, h.num_cols, rows, cols, vals,
                    float(h.lam), fix if (fix >= 0).all() else None, algorithm=2, epsilon=1e-10, svd_remove_n=7)


def write_jacob_binary(path: str, jac: Jacobian) -> None:
    """The binary form of a `.jacob` file (64-byte header, then the three arrays)."""
    h = UncJacobHeader()
    h.lam = jac.lam
    h.num_cams, h.cam_params, h.num_points, h.num_obs = jac.num_cams, jac.cam_params, jac.num_points, jac.num_obs
    fix = jac.pts2fix if jac.pts2fix is not None else [-1, -1, -1]
    h.pts2fix[:] = [int(x) for x in fix]
    h.num_rows, h.num_cols, h.nnz, h.binary = jac.num_rows, jac.num_cols, int(jac.rows[-1]), 1
    rows = np.ascontiguousarray(jac.rows, dtype=np.int32)
    cols = np.ascontiguousarray(jac.cols, dtype=np.int32)
    vals = np.ascontiguousarray(jac.values, dtype=np.float64)
    _check(lib().unc_jacob_write_binary(os.fsencode(path), C.byref(h), _ptr(rows), _ptr(cols), _ptr(vals)))


class Context:
    """Owns a CUDA stream and a device workspace reused across calls."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        _check(lib().unc_context_create(device, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().unc_context_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_profiling(self, enable: bool = True):
        _check(lib().unc_context_set_profiling(self._h, int(enable)))

    def profile(self, reset: bool = True):
        """(launches, seconds, flops) of the Taylor-series products since the last reset."""
        n, s, f = C.c_longlong(), C.c_double(), C.c_double()
        _check(lib().unc_context_profile(self._h, C.byref(n), C.byref(s), C.byref(f), int(reset)))
        return n.value, s.value, f.value

    def profile_int8(self) -> float:
        """int8 multiply-adds x 2 issued by the profiled products (mixed modes), since the last reset."""
        v = C.c_double()
        _check(lib().unc_context_profile_int8(self._h, C.byref(v)))
        return v.value

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def compute_covariances(jac: Jacobian, ctx: Optional[Context] = None, algorithm: Optional[int] = None,
                        precision: str = "fp64", cam_init=None, pt_init=None, taylor: str = "powers"):
    """computeCovariances on host arrays: returns (cam (C*45,), pt (P*6,), stats dict).
    taylor: "powers" (blocked powers, the default) or "sequential" (one product
    per Taylor iteration, the reference's order)."""
    o = make_options(jac, algorithm, precision, taylor=taylor)
    cam = np.zeros(jac.num_cams * 45) if cam_init is None else np.array(cam_init, dtype=np.float64)
    pt = np.zeros(jac.num_points * 6) if pt_init is None else np.array(pt_init, dtype=np.float64)
    rows = np.ascontiguousarray(jac.rows, dtype=np.int32)
    cols = np.ascontiguousarray(jac.cols, dtype=np.int32)
    vals = np.ascontiguousarray(jac.values, dtype=np.float64)
    st = UncStatistic()
    _check(lib().unc_compute(ctx.handle if ctx else None, C.byref(o), jac.num_rows, jac.num_cols,
                             _ptr(rows), _ptr(cols), _ptr(vals), _ptr(cam), _ptr(pt), C.byref(st)))
    return cam, pt, st.as_dict()


def compute_covariances_device(ctx: Context, opts: UncOptions, num_rows: int, num_cols: int,
                               d_rows: int, d_cols: int, d_vals: int, d_cam: int, d_pt: int,
                               stream: int = 0) -> dict:
    """Device-pointer form (inputs resident in HBM); pointers are integers."""
    st = UncStatistic()
    _check(lib().unc_compute_device(ctx.handle, C.byref(opts), num_rows, num_cols, d_rows, d_cols,
                                    d_vals, d_cam, d_pt, C.byref(st), stream or None))
    return st.as_dict()


def compute_covariances_scene(scene, pts2fix, ctx: Optional[Context] = None, precision: str = "fp64",
                              algorithm: int = TAYLOR_EXPANSION, svd_remove_n: int = 7):
    """computeCovariances from a scene (cams C x 9, points P x 3, obs_cam, obs_pt):
    the Jacobian is built on the GPU. Returns (cam (C*45,), pt (P*6,), stats)."""
    cams = np.ascontiguousarray(scene.cams, dtype=np.float64)
    pts = np.ascontiguousarray(scene.points, dtype=np.float64)
    oc = np.ascontiguousarray(scene.obs_cam, dtype=np.int32)
    op = np.ascontiguousarray(scene.obs_pt, dtype=np.int32)
    o = UncOptions()
    lib().unc_options_init(C.byref(o), len(cams), 9, len(pts), len(oc))
    o.algorithm = algorithm
    o.svd_remove_n = svd_remove_n
    if pts2fix is not None:
        o.pts2fix[:] = [int(x) for x in pts2fix]
        o.has_pts2fix = 1
    o.precision = PRECISION[precision]
    cam = np.zeros(len(cams) * 45)
    pt = np.zeros(len(pts) * 6)
    st = UncStatistic()
    _check(lib().unc_compute_scene(ctx.handle if ctx else None, C.byref(o), _ptr(cams), _ptr(pts), _ptr(oc),
                                   _ptr(op), _ptr(cam), _ptr(pt), C.byref(st)))
    return cam, pt, st.as_dict()


def block_eigen(packed, block_params: int, sub_offset: int = 0, sub_dim: Optional[int] = None,
                vectors: bool = True):
    """Eigenvalues (descending) and eigenvectors of packed upper-triangle blocks on the GPU."""
    packed = np.ascontiguousarray(packed, dtype=np.float64)
    per = block_params * (block_params + 1) // 2
    nb = packed.size // per
    dim = block_params if sub_dim is None else sub_dim
    vals = np.zeros(nb * dim)
    vecs = np.zeros(nb * dim * dim) if vectors else None
    _check(lib().unc_block_eigen(_ptr(packed), nb, block_params, sub_offset, dim, _ptr(vals),
                                 _ptr(vecs) if vectors else None))
    return vals.reshape(nb, dim), (vecs.reshape(nb, dim, dim) if vectors else None)


class Server:
    """Request server on one GPU (continuous batching, admission by device bytes).

    submit() queues a reconstruction and returns its id; wait() returns
    (cam, pt, stats, latency_s, queue_s) once it has finished. The arrays of a
    request are kept alive here until its result is collected."""

    def __init__(self, device: int = 0, max_device_bytes: int = 0, max_inflight: int = 4):
        self._h = C.c_void_p()
        _check(lib().unc_server_create(device, max_device_bytes, max_inflight, C.byref(self._h)))
        self._live = {}

    def submit(self, jac: Jacobian, precision: str = "mixed", algorithm: Optional[int] = None) -> int:
        o = make_options(jac, algorithm, precision)
        rows = np.ascontiguousarray(jac.rows, dtype=np.int32)
        cols = np.ascontiguousarray(jac.cols, dtype=np.int32)
        vals = np.ascontiguousarray(jac.values, dtype=np.float64)
        cam = np.zeros(jac.num_cams * 45)
        pt = np.zeros(jac.num_points * 6)
        rid = C.c_longlong()
        _check(lib().unc_server_submit(self._h, C.byref(o), jac.num_rows, jac.num_cols, _ptr(rows), _ptr(cols),
                                       _ptr(vals), _ptr(cam), _ptr(pt), C.byref(rid)))
        self._live[rid.value] = (o, rows, cols, vals, cam, pt)
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0):
        status = C.c_int()
        st = UncStatistic()
        lat, que = C.c_double(), C.c_double()
        _check(lib().unc_server_wait(self._h, rid, timeout, C.byref(status), C.byref(st), C.byref(lat),
                                     C.byref(que)))
        _, _, _, _, cam, pt = self._live.pop(rid)
        _check(status.value)
        return cam, pt, st.as_dict(), lat.value, que.value

    def poll(self, rid: int):
        """wait() without blocking: None while request rid still runs."""
        status = C.c_int()
        st = UncStatistic()
        lat, que = C.c_double(), C.c_double()
        rc = lib().unc_server_wait(self._h, rid, 0.0, C.byref(status), C.byref(st), C.byref(lat), C.byref(que))
        if rc == UNC_ERR_TIMEOUT:
            return None
        _check(rc)
        _, _, _, _, cam, pt = self._live.pop(rid)
        _check(status.value)
        return cam, pt, st.as_dict(), lat.value, que.value

    def close(self):
        if self._h:
            lib().unc_server_destroy(self._h)
            self._h = C.c_void_p()
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many reconstructions in one grouped launch sequence (unc_batch_compute).

    compute() returns, per Jacobian, (cam, pt, stats, status) with status the
    scene's own status code (0 = UNC_OK); last_timing() the input-copy,
    device and output-copy seconds of the last call, the number of grouped
    scenes and the product tile width."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        _check(lib().unc_batch_create(device, C.byref(self._h)))

    def compute(self, jacs, precision="mixed", algorithm: Optional[int] = None, pt_init=None):
        n = len(jacs)
        precs = precision if isinstance(precision, (list, tuple)) else [precision] * n
        opts = (UncOptions * n)(*[make_options(j, algorithm, p) for j, p in zip(jacs, precs)])
        arrs = [(np.ascontiguousarray(j.rows, dtype=np.int32), np.ascontiguousarray(j.cols, dtype=np.int32),
                 np.ascontiguousarray(j.values, dtype=np.float64)) for j in jacs]
        cams = [np.zeros(j.num_cams * 45) for j in jacs]
        pts = [np.zeros(j.num_points * 6) if pt_init is None else np.array(pt_init[k], dtype=np.float64)
               for k, j in enumerate(jacs)]
        vp = C.c_void_p
        nr = (C.c_int * n)(*[j.num_rows for j in jacs])
        nc = (C.c_int * n)(*[j.num_cols for j in jacs])
        rows = (vp * n)(*[a[0].ctypes.data for a in arrs])
        cols = (vp * n)(*[a[1].ctypes.data for a in arrs])
        vals = (vp * n)(*[a[2].ctypes.data for a in arrs])
        cp = (vp * n)(*[c.ctypes.data for c in cams])
        pp = (vp * n)(*[p.ctypes.data for p in pts])
        status = (C.c_int * n)()
        stats = (UncStatistic * n)()
        _check(lib().unc_batch_compute(self._h, n, opts, nr, nc, rows, cols, vals, cp, pp, status, stats))
        return [(cams[k], pts[k], stats[k].as_dict(), status[k]) for k in range(n)]

    def last_timing(self) -> dict:
        h, d, o = C.c_double(), C.c_double(), C.c_double()
        g, t = C.c_int(), C.c_int()
        _check(lib().unc_batch_last_timing(self._h, C.byref(h), C.byref(d), C.byref(o), C.byref(g), C.byref(t)))
        return {"h2d_s": h.value, "device_s": d.value, "d2h_s": o.value, "grouped_scenes": g.value,
                "tile_n": t.value}

    def set_tile_width(self, tile_n: int):
        """5-slice product tile width: 0 = cost model, 64 or 96 forced."""
        _check(lib().unc_batch_set_tile_width(self._h, tile_n))

    def close(self):
        if self._h:
            lib().unc_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def request_bytes(jac: Jacobian, precision: str = "mixed", algorithm: Optional[int] = None) -> int:
    o = make_options(jac, algorithm, precision)
    rows = np.ascontiguousarray(jac.rows, dtype=np.int32)
    cols = np.ascontiguousarray(jac.cols, dtype=np.int32)
    return int(lib().unc_request_bytes(C.byref(o), jac.num_rows, jac.num_cols, _ptr(rows), _ptr(cols)))


def workspace_bytes(jac: Jacobian) -> int:
    o = make_options(jac)
    return int(lib().unc_workspace_bytes(C.byref(o), jac.num_rows, jac.num_cols))


def dense_inverse_device(d_ptr: int, n: int, lda: int, stream: int = 0) -> None:
    _check(lib().unc_dense_inverse_device(d_ptr, n, lda, stream or None))


def spd_inverse_tasks_bounded(d_ptr: int, n: int, lda: int, poll_limit: int, skip_task: int = -1,
                              stream: int = 0) -> None:
    """The tile-task inverse with its dependency waits limited to poll_limit
    polls, optionally with one task left out of the schedule (a test of the
    bounded waits: the call must then fail with UNC_ERR_CUDA, not hang)."""
    _check(lib().unc_spd_inverse_tasks_bounded(d_ptr, n, lda, poll_limit, skip_task, stream or None))


def dense_inverse_noalloc(d_ptr: int, n: int, lda: int, stream: int = 0) -> None:
    """In-place SPD inverse with no device allocation (static scratch, n and lda <= 512)."""
    _check(lib().unc_dense_inverse_noalloc(d_ptr, n, lda, stream or None))


SPD_TASK_KINDS = ("POTRF", "TRSM", "UPDATE", "TACC", "TFIN", "PACC")


def spd_task_list(n: int):
    """The tile-task order of the n x n SPD inverse (n <= 3584) as an int array
    of shape (tasks, 4): kind (index into SPD_TASK_KINDS), i, j, k. Host only."""
    import numpy as np
    L = lib()
    count = L.unc_spd_task_list(n, None, 0)
    if count < 0:
        _check(count)
    out = np.zeros((count, 4), dtype=np.int32)
    _check(0 if L.unc_spd_task_list(n, out.ctypes.data, count) == count else -1)
    return out


def pinv_psd_device(d_ptr: int, n: int, ld: int, remove_n: int = 7, epsilon: float = 1e-10,
                    stream: int = 0) -> None:
    """In-place pseudo-inverse of a PSD matrix without its remove_n smallest
    singular values (remove_n = -1: without those <= epsilon)."""
    _check(lib().unc_pinv_psd_device(d_ptr, n, ld, remove_n, epsilon, stream or None))


def jtj_crs(num_rows: int, num_cols: int, rows, cols, vals, num_cams: int, cam_params: int = 9):
    """GPU J^T J in the reference's CRS pattern: (rowptr, cols, vals)."""
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    nnz = C.c_longlong(0)
    L = lib()
    _check(L.unc_jtj_crs(num_rows, num_cols, _ptr(rows), _ptr(cols), _ptr(vals), num_cams, cam_params,
                         C.byref(nnz), None, None, None))
    orow = np.zeros(num_cols + 1, np.int32)
    ocol = np.zeros(nnz.value, np.int32)
    oval = np.zeros(nnz.value)
    _check(L.unc_jtj_crs(num_rows, num_cols, _ptr(rows), _ptr(cols), _ptr(vals), num_cams, cam_params,
                         C.byref(nnz), _ptr(orow), _ptr(ocol), _ptr(oval)))
    return orow, ocol, oval


def gemm_f64_device(M, N, K, alpha, d_A, lda, d_B, ldb, beta, d_C, ldc, stream: int = 0) -> None:
    """C = alpha A B + beta C (column-major device pointers) on the FP64 GEMM kernel."""
    _check(lib().unc_gemm_f64_device(M, N, K, alpha, d_A, lda, d_B, ldb, beta, d_C, ldc, stream or None))


def gemm_mixed_device(n, d_P, d_X, ld, d_C, slices=4, stream: int = 0) -> None:
    """C = P X for symmetric P, X on the int8-sliced tensor-core product."""
    _check(lib().unc_gemm_mixed_device(n, d_P, d_X, ld, d_C, slices, stream or None))


def gram_lower_mixed_device(n, d_T, ld, d_A, stream: int = 0) -> None:
    """A = T^T T for lower-triangular T on the int8-sliced tensor-core product (7 slices)."""
    _check(lib().unc_gram_lower_mixed_device(n, d_T, ld, d_A, stream or None))


def kernel_launches() -> int:
    return int(lib().unc_kernel_launches())
