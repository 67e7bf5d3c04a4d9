"""ctypes front end of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY. The oracle restates the reference's CPU algorithm
(src/uncertaintyTE/compute.cpp and the Scaled*Matrix classes) and is the
checker for the CUDA product path. Only tests/, the smoke check and the
CPU-baseline leg of bench.py may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OracleOptions(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int),
        ("epsilon", C.c_double),
        ("lam", C.c_double),
        ("num_cams", C.c_int),
        ("cam_params", C.c_int),
        ("num_points", C.c_int),
        ("num_obs", C.c_int),
        ("svd_remove_n", C.c_int),
        ("pts2fix", C.c_int * 3),
        ("has_pts2fix", C.c_int),
        ("faithful_point_scan", C.c_int),
        ("threads", C.c_int),
        ("inverse_route", C.c_int),
        ("z_perturb", C.c_double),
        ("z_perturb_terms", C.c_double),
        ("swap_products", C.c_int),
        ("skip_dense", C.c_int),
        ("offdiag_nan", C.c_int),
    ]


class OracleStats(C.Structure):
    _fields_ = [
        ("lam", C.c_double),
        ("fixed_pts", C.c_int * 3),
        ("te_iterations", C.c_int),
        ("cycle_change", C.c_double * 20),
        ("t_fix", C.c_double),
        ("t_norm", C.c_double),
        ("t_jtj", C.c_double),
        ("t_split", C.c_double),
        ("t_invv", C.c_double),
        ("t_compose_z", C.c_double),
        ("t_inv_z", C.c_double),
        ("t_te", C.c_double),
        ("t_cams", C.c_double),
        ("t_pts", C.c_double),
        ("t_all", C.c_double),
        ("lu_info", C.c_int),
    ]


def build() -> str:
    """Compile liboracle.so in place (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE, f"PY={sys.executable}"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.POINTER
        L.oracle_compute.argtypes = [P(OracleOptions), C.c_int, C.c_int, P(C.c_int), P(C.c_int),
                                     P(C.c_double), P(C.c_double), P(C.c_double), P(OracleStats),
                                     P(C.c_double), P(C.c_double), P(C.c_double)]
        L.oracle_compute.restype = C.c_int
        L.oracle_jtj.argtypes = [C.c_int, C.c_int, P(C.c_int), P(C.c_int), P(C.c_double),
                                 P(C.c_int), P(C.c_int), P(C.c_double)]
        L.oracle_jtj.restype = C.c_long
        L.oracle_dense_inv.argtypes = [C.c_int, P(C.c_double)]
        L.oracle_dense_inv.restype = C.c_int
        L.oracle_te_inverse.argtypes = [C.c_int, P(C.c_double), C.c_double, P(OracleStats)]
        L.oracle_te_inverse.restype = C.c_int
        L.oracle_te_inverse_route.argtypes = [C.c_int, P(C.c_double), C.c_double, C.c_int, P(OracleStats), C.c_int]
        L.oracle_te_inverse_route.restype = C.c_int
        L.oracle_dense_inv_cholesky.argtypes = [C.c_int, P(C.c_double)]
        L.oracle_dense_inv_cholesky.restype = C.c_int
        L.oracle_gemm.argtypes = [C.c_int, P(C.c_double), P(C.c_double), P(C.c_double)]
        L.oracle_gemm.restype = None
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_set_threads.restype = C.c_int
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def compute(jac, algorithm=2, lam=-1.0, epsilon=1e-10, svd_remove_n=-1, faithful_point_scan=False,
            threads=0, debug=False, cam_init=None, pt_init=None, route="lu", z_perturb=0.0,
            z_perturb_terms=0.0, swap_products=False, skip_dense=False, offdiag_nan=False):
    """Run the oracle on a Jacobian (uncertaintyte_b200.jacob.Jacobian-like object).

    route: "lu" (the reference's ScaledDenseMatrix::inv) or "cholesky" (the
    Jacobi-equilibrated Cholesky inverse, the CUDA path's route) for the dense
    inverse of the Taylor path. z_perturb: relative rounding-level perturbation
    of the Schur complement (see uncte_oracle.h), 0 for none; z_perturb_terms:
    the same at the size of the Schur complement's terms; swap_products: the
    Taylor products as X * add instead of add * X (same series, other
    rounding). skip_dense:
    timing samples only (the dense inverse and Taylor loop are skipped, the
    outputs are meaningless). offdiag_nan: iZ outside its camera diagonal
    blocks set to NaN before the outputs (which entries the outputs read).
    Returns dict(cam, pt, stats[, Z, iZ, d])."""
    o = OracleOptions()
    o.algorithm = algorithm
    o.epsilon = epsilon
    o.lam = lam
    o.num_cams, o.cam_params = jac.num_cams, jac.cam_params
    o.num_points, o.num_obs = jac.num_points, jac.num_obs
    o.svd_remove_n = svd_remove_n
    if jac.pts2fix is not None:
        o.pts2fix[:] = [int(x) for x in jac.pts2fix]
        o.has_pts2fix = 1
    o.faithful_point_scan = int(bool(faithful_point_scan))
    o.threads = threads
    o.inverse_route = {"lu": 0, "cholesky": 1, "recursive": 2}[route]
    o.z_perturb = z_perturb
    o.z_perturb_terms = z_perturb_terms
    o.swap_products = int(bool(swap_products))
    o.skip_dense = int(bool(skip_dense))
    o.offdiag_nan = int(bool(offdiag_nan))
    ncam = jac.num_cams * jac.cam_params * (jac.cam_params + 1) // 2
    cam = np.zeros(ncam) if cam_init is None else np.array(cam_init, dtype=np.float64)
    pt = np.zeros(jac.num_points * 6) if pt_init is None else np.array(pt_init, dtype=np.float64)
    rows = np.ascontiguousarray(jac.rows, dtype=np.int32)
    cols = np.ascontiguousarray(jac.cols, dtype=np.int32)
    vals = np.ascontiguousarray(jac.values, dtype=np.float64)
    st = OracleStats()
    N = jac.num_cams * jac.cam_params
    Z = iZ = d = None
    nullp = C.POINTER(C.c_double)()
    if debug and algorithm == 2:
        Z = np.zeros((N, N), order="F")
        iZ = np.zeros((N, N), order="F")
        d = np.zeros(N)
    rc = lib().oracle_compute(C.byref(o), jac.num_rows, jac.num_cols, _p(rows, C.c_int),
                              _p(cols, C.c_int), _p(vals, C.c_double), _p(cam, C.c_double),
                              _p(pt, C.c_double), C.byref(st),
                              _p(Z, C.c_double) if Z is not None else nullp,
                              _p(iZ, C.c_double) if iZ is not None else nullp,
                              _p(d, C.c_double) if d is not None else nullp)
    if rc != 0:
        raise ValueError(f"oracle_compute failed with status {rc}")
    out = dict(cam=cam, pt=pt, stats=st)
    if Z is not None:
        out.update(Z=Z, iZ=iZ, d=d)
    return out


def jtj(nrows, ncols, rows, cols, vals):
    """Sparse J^T J as (rowptr, cols, vals), the way the reference forms it."""
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    L = lib()
    ip = C.POINTER(C.c_int)()
    dp = C.POINTER(C.c_double)()
    nnz = L.oracle_jtj(nrows, ncols, _p(rows, C.c_int), _p(cols, C.c_int), _p(vals, C.c_double),
                       ip, ip, dp)
    orow = np.zeros(ncols + 1, np.int32)
    ocol = np.zeros(nnz, np.int32)
    oval = np.zeros(nnz)
    L.oracle_jtj(nrows, ncols, _p(rows, C.c_int), _p(cols, C.c_int), _p(vals, C.c_double),
                 _p(orow, C.c_int), _p(ocol, C.c_int), _p(oval, C.c_double))
    return orow, ocol, oval


def dense_inv(A):
    """ScaledDenseMatrix::inv restated; A is a square ndarray (any order)."""
    n = A.shape[0]
    F = np.array(A, dtype=np.float64, order="F")
    info = lib().oracle_dense_inv(n, _p(F, C.c_double))
    return F, info


def te_inverse(Z, lam, route="lu"):
    n = Z.shape[0]
    F = np.array(Z, dtype=np.float64, order="F")
    st = OracleStats()
    lib().oracle_te_inverse_route(n, _p(F, C.c_double), lam, {"lu": 0, "cholesky": 1}[route], C.byref(st), 0)
    return F, st


def dense_inv_cholesky(A):
    """The Jacobi-equilibrated Cholesky inverse (the CUDA path's route)."""
    n = A.shape[0]
    F = np.array(A, dtype=np.float64, order="F")
    info = lib().oracle_dense_inv_cholesky(n, _p(F, C.c_double))
    return F, info


def gemm(A, B):
    """One dense product of the Taylor loop (operator*=): A * B."""
    n = A.shape[0]
    Af = np.asfortranarray(A, dtype=np.float64)
    Bf = np.asfortranarray(B, dtype=np.float64)
    Cf = np.zeros((n, n), order="F")
    lib().oracle_gemm(n, _p(Af, C.c_double), _p(Bf, C.c_double), _p(Cf, C.c_double))
    return Cf


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(n)
