"""The large scene (2000 cameras, 500k points, ~3.5M observations, N = 18000)
on the GPU, against a sampled oracle result (needs a B200).

The CPU oracle takes about ten minutes per dense-inverse route on this scene,
so its output is committed as a sample (tests/golden/large_sample.npz: every
10th camera block, 2000 point blocks, the Taylor-loop statistics; made by
tests/golden/make_large_golden.py on the same seeded scene). Bars, per camera
9x9 and point 3x3 block (relative Frobenius error):
  * FP64 GPU vs the oracle's LU and Cholesky routes: max(1e-9, FLOOR_MULT x the
    floor), the floor being how far the Cholesky route, the LU route on the
    Jacobian moved by one ulp (two seeds) and the LU route with the Schur
    complement moved at the size of its terms lie from the LU route, as in
    test_gpu_parity.py;
  * mixed precision vs the FP64 oracle (sample) and vs the FP64 GPU path (all
    blocks): 1e-6, the accuracy target of the mixed path;
  * iteration count, lambda and fixed points exactly.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, block_rel_err
from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu

FP64_BAR = 1e-9
FLOOR_MULT = 4.0
MIXED_TOL = 1e-6


@pytest.fixture(scope="module")
def large():
    import sys
    sys.path.insert(0, GOLDEN)
    from make_large_golden import scene_fingerprint
    g = np.load(os.path.join(GOLDEN, "large_sample.npz"))
    jac = scenes.synthetic_jacobian("large", seed=0)
    np.testing.assert_array_equal(scene_fingerprint(jac), g["fingerprint"],
                                  err_msg="the generator no longer makes the sampled scene: rerun make_large_golden.py")
    ctx = native.Context(0)
    c64, p64, s64 = native.compute_covariances(jac, ctx, precision="fp64")
    cmx, pmx, smx = native.compute_covariances(jac, ctx, precision="mixed")
    ctx.close()
    return g, jac, (c64, p64, s64), (cmx, pmx, smx)


def _sample(cam, pt, g):
    return cam.reshape(-1, 45)[g["cams"]], pt.reshape(-1, 6)[g["pts"]]


def test_large_statistics_match_the_oracle(large):
    g, jac, (c64, p64, s64), (cmx, pmx, smx) = large
    for st in (s64, smx):
        assert st["te_iterations"] == int(g["lu_iters"]) == int(g["cholesky_iters"])
        assert st["lambda"] == float(g["lu_lambda"])
        assert st["fixed_pts"] == list(g["lu_fixed"])
        np.testing.assert_allclose(st["cycle_change"], g["lu_cycle_change"], rtol=1e-6)


def test_large_fp64_vs_oracle_sample(large):
    g, jac, (c64, p64, s64), _ = large
    # the floor: the Cholesky route and the one-ulp perturbed Jacobians against the LU route
    others = [k for k in ("cholesky", "ulp1", "ulp2", "terms") if f"{k}_cam" in g.files]
    fc = max(block_rel_err(g[f"{k}_cam"], g["lu_cam"], 45) for k in others)
    fp = max(block_rel_err(g[f"{k}_pt"], g["lu_pt"], 6) for k in others)
    bar_c, bar_p = max(FP64_BAR, FLOOR_MULT * fc), max(FP64_BAR, FLOOR_MULT * fp)
    cs, ps = _sample(c64, p64, g)
    ec, ep = block_rel_err(cs, g["lu_cam"], 45), block_rel_err(ps, g["lu_pt"], 6)
    hc, hp = block_rel_err(cs, g["cholesky_cam"], 45), block_rel_err(ps, g["cholesky_pt"], 6)
    print(f"large FP64 GPU vs LU: cams {ec:.2e} points {ep:.2e}; vs Cholesky: cams {hc:.2e} points {hp:.2e}; "
          f"floor ({', '.join(others)}) {fc:.2e} / {fp:.2e}; bar {bar_c:.2e} / {bar_p:.2e}")
    assert ec <= bar_c and ep <= bar_p
    assert hc <= bar_c and hp <= bar_p


def test_large_mixed_vs_fp64(large):
    g, jac, (c64, p64, _), (cmx, pmx, _) = large
    ec, ep = block_rel_err(cmx, c64, 45), block_rel_err(pmx, p64, 6)
    cs, ps = _sample(cmx, pmx, g)
    oc, op = block_rel_err(cs, g["lu_cam"], 45), block_rel_err(ps, g["lu_pt"], 6)
    print(f"large mixed vs FP64 GPU (all blocks): cams {ec:.2e} points {ep:.2e}; "
          f"vs FP64 oracle (sample): cams {oc:.2e} points {op:.2e}")
    assert ec < MIXED_TOL and ep < MIXED_TOL
    assert oc < MIXED_TOL and op < MIXED_TOL
    assert np.isfinite(cmx).all() and np.isfinite(pmx).all()
