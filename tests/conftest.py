import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libuncte.so")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def golden_jacobian(name):
    from uncertaintyte_b200.jacob import Jacobian
    d = golden(name)
    h = d["header"]
    fix = d["pts2fix"]
    return Jacobian(int(h[1]), int(h[2]), int(h[3]), int(h[4]), int(h[5]), int(h[6]),
                    d["rows"].copy(), d["cols"].copy(), d["values"].copy(), float(h[0]),
                    fix.copy() if (fix >= 0).all() else None, algorithm=2, epsilon=1e-10,
                    svd_remove_n=7)


def _upper_weights(width):
    p = {45: 9, 6: 3}[width]
    w = []
    for i in range(p):
        for j in range(i, p):
            w.append(1.0 if i == j else 2.0)
    return np.sqrt(np.array(w))


def block_rel_err(a, b, width):
    """Max over blocks of ||a_blk - b_blk||_F / ||b_blk||_F of the full symmetric
    9x9 (width 45) or 3x3 (width 6) blocks given as packed upper triangles.
    Blocks with ||b||_F = 0 contribute their absolute error."""
    w = _upper_weights(width)
    a = np.asarray(a).reshape(-1, width) * w
    b = np.asarray(b).reshape(-1, width) * w
    num = np.linalg.norm(a - b, axis=1)
    den = np.linalg.norm(b, axis=1)
    r = np.where(den > 0, num / np.where(den > 0, den, 1), num)
    return float(r.max()) if r.size else 0.0


def fp64_floor(jac, ref_lu, threads=8, **kw):
    """How far two correct FP64 computations of this scene lie apart.

    Z + lambda*I is ill-conditioned (the gauge is fixed only by lambda), so
    FP64 results are determined only to about cond * eps. Measured on the CPU
    oracle: the Cholesky inverse route against the LU route (same Z), and the
    LU route on the Jacobian with every value moved by at most one ulp (two
    seeds): rounding-level input noise, which is what a different summation
    order in the assembly amounts to; and the LU route with the Schur
    complement Z = U - Y W^T moved by one ulp of the size of its terms (the
    rounding of another summation order of Z itself). Returns (camera floor,
    point floor, details)."""
    import copy

    import oracle
    det = {}
    chol = oracle.compute(jac, threads=threads, route="cholesky", **kw)
    det["cholesky"] = (block_rel_err(chol["cam"], ref_lu["cam"], 45), block_rel_err(chol["pt"], ref_lu["pt"], 6))
    for seed in (1, 2):
        j2 = copy.copy(jac)
        r = np.random.default_rng(seed).uniform(-1.0, 1.0, jac.values.size)
        j2.values = jac.values * (1.0 + 2.0 ** -52 * r)
        o = oracle.compute(j2, threads=threads, **kw)
        det[f"ulp{seed}"] = (block_rel_err(o["cam"], ref_lu["cam"], 45), block_rel_err(o["pt"], ref_lu["pt"], 6))
    o = oracle.compute(jac, threads=threads, z_perturb_terms=2.0 ** -52, **kw)
    det["terms"] = (block_rel_err(o["cam"], ref_lu["cam"], 45), block_rel_err(o["pt"], ref_lu["pt"], 6))
    return max(v[0] for v in det.values()), max(v[1] for v in det.values()), det, chol
