"""Sampled oracle results for the large synthetic scene (test fixture generator).

The large scene (2000 cameras on a 3-loop trajectory, 500k points,
2+Poisson(5) observations per point, N = 9C = 18000) takes the CPU oracle
about ten minutes per route on 8 cores (15 dense 18000^3 products), far too
long for a GPU test. This script runs the oracle once, on the scene the
seeded generator makes, and keeps a deterministic sample of its output:
every 10th camera block, 2000 point blocks, the Taylor-loop statistics and a
fingerprint of the scene (so that a test notices a generator change).

Both dense-inverse routes are run: "lu" (the reference's equilibrated
dgetrf/dgetri) and "cholesky" (the Jacobi-equilibrated Cholesky inverse that
the CUDA path also uses), and the LU route on the Jacobian with every value
moved by at most one ulp (two seeds, "ulp1" / "ulp2"), and the LU route with
the Schur complement moved at the size of its terms ("terms": the rounding of
Z = U - Y W^T in another summation order), the perturbations of
tests/conftest.py fp64_floor. How far these lie apart is the FP64 floor of
this ill-conditioned problem, which the GPU test uses as its bar.

The oracle's point stage runs with its per-point observation index
(faithful_point_scan=False): the reference's O(points x observations) row scan
(compute.cpp:393) would visit ~1.75e12 rows here; the index visits the same
rows of each point in the same order.

    python tests/golden/make_large_golden.py [--threads N] [--only-ulp | --only-terms]

writes tests/golden/large_sample.npz (--only-ulp, --only-terms: add those
perturbed runs to an existing file).
"""
from __future__ import annotations

import argparse
import copy
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def scene_fingerprint(jac) -> np.ndarray:
    """(number of observations, sum of |J|, a hash of the observation columns)."""
    h = hashlib.sha256(np.ascontiguousarray(jac.cols).tobytes()).digest()
    return np.array([float(jac.num_obs), float(np.abs(jac.values).sum()),
                     float(int.from_bytes(h[:6], "little"))])


def sample_indices(jac):
    cams = np.arange(0, jac.num_cams, 10)
    fixed = set(int(x) for x in jac.pts2fix)
    rng = np.random.default_rng(12345)
    pts = np.sort(rng.choice(jac.num_points, 2000, replace=False))
    pts = np.array([p for p in pts if p not in fixed])
    return cams, pts


def main():
    import oracle
    from uncertaintyte_b200 import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(HERE, "large_sample.npz"))
    ap.add_argument("--only-ulp", action="store_true")
    ap.add_argument("--only-terms", action="store_true")
    a = ap.parse_args()
    jac = scenes.synthetic_jacobian("large", seed=0)
    cams, pts = sample_indices(jac)
    out = {"fingerprint": scene_fingerprint(jac), "cams": cams, "pts": pts,
           "pts2fix": np.asarray(jac.pts2fix, dtype=np.int32)}
    runs = [("lu", "lu", None), ("cholesky", "cholesky", None), ("ulp1", "lu", 1), ("ulp2", "lu", 2),
            ("terms", "lu", "terms")]
    if a.only_ulp or a.only_terms:
        old = np.load(a.out)
        out.update({k: old[k] for k in old.files})
        runs = runs[2:4] if a.only_ulp else runs[4:]
    for name, route, seed in runs:
        t0 = time.perf_counter()
        j, zt = jac, 0.0
        if seed == "terms":  # the Schur complement moved at the size of its terms
            zt = 2.0 ** -52
        elif seed is not None:  # every value moved by at most one ulp
            j = copy.copy(jac)
            r = np.random.default_rng(seed).uniform(-1.0, 1.0, jac.values.size)
            j.values = jac.values * (1.0 + 2.0 ** -52 * r)
        r = oracle.compute(j, threads=a.threads, faithful_point_scan=False, route=route, z_perturb_terms=zt)
        st = r["stats"]
        print(f"{name}: {time.perf_counter() - t0:.1f} s, {st.te_iterations} iterations", flush=True)
        out[f"{name}_cam"] = r["cam"].reshape(-1, 45)[cams]
        out[f"{name}_pt"] = r["pt"].reshape(-1, 6)[pts]
        out[f"{name}_iters"] = np.int32(st.te_iterations)
        out[f"{name}_cycle_change"] = np.array(st.cycle_change[: st.te_iterations])
        out[f"{name}_lambda"] = np.float64(st.lam)
        out[f"{name}_fixed"] = np.array(list(st.fixed_pts), dtype=np.int32)
    np.savez_compressed(a.out, **out)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
