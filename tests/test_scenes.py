"""Synthetic scene generator and the .jacob / .cov formats (CPU)."""
import os

import numpy as np

from uncertaintyte_b200 import scenes
from uncertaintyte_b200.jacob import load_cov, load_jacob, save_cov, save_jacob


def test_analytic_jacobian_matches_finite_differences():
    sc = scenes.make_scene("tiny", seed=3)
    Jc, Jp = scenes.observation_blocks(sc.cams, sc.points, sc.obs_cam, sc.obs_pt)
    h = 1e-6
    for j in range(9):
        cp, cm = sc.cams.copy(), sc.cams.copy()
        cp[:, j] += h
        cm[:, j] -= h
        fd = (scenes.project(cp, sc.points, sc.obs_cam, sc.obs_pt) -
              scenes.project(cm, sc.points, sc.obs_cam, sc.obs_pt)) / (2 * h)
        np.testing.assert_allclose(Jc[:, :, j], fd, rtol=2e-5, atol=1e-4 * np.abs(fd).max())
    for j in range(3):
        pp, pm = sc.points.copy(), sc.points.copy()
        pp[:, j] += h
        pm[:, j] -= h
        fd = (scenes.project(sc.cams, pp, sc.obs_cam, sc.obs_pt) -
              scenes.project(sc.cams, pm, sc.obs_cam, sc.obs_pt)) / (2 * h)
        np.testing.assert_allclose(Jp[:, :, j], fd, rtol=2e-5, atol=1e-4 * np.abs(fd).max())


def test_points_in_front_and_layout():
    sc = scenes.make_scene("small", seed=1)
    R = scenes._aa_to_rot(sc.cams[sc.obs_cam, :3])
    p = np.einsum("nij,nj->ni", R, sc.points[sc.obs_pt] - sc.cams[sc.obs_cam, 3:6])
    assert (p[:, 2] > 0).all()
    jac = scenes.scene_jacobian(sc)
    assert jac.num_rows == 2 * jac.num_obs and jac.nnz == 24 * jac.num_obs
    assert 2500 < jac.num_obs < 3500  # ~3k observations
    assert np.all(np.diff(sc.obs_pt) >= 0)  # point-major
    assert len(np.unique(sc.obs_cam)) == 10
    assert list(jac.pts2fix) == sorted(jac.pts2fix)


def test_jacob_roundtrip(tmp_path):
    jac = scenes.synthetic_jacobian("tiny", seed=2)
    p = os.path.join(tmp_path, "t.jacob")
    save_jacob(p, jac)
    j2 = load_jacob(p)
    np.testing.assert_array_equal(j2.rows, jac.rows)
    np.testing.assert_array_equal(j2.cols, jac.cols)
    np.testing.assert_array_equal(j2.values, jac.values)
    np.testing.assert_array_equal(j2.pts2fix, jac.pts2fix)
    assert j2.algorithm == 2 and j2.svd_remove_n == 7


def test_cov_roundtrip(tmp_path):
    jac = scenes.synthetic_jacobian("tiny", seed=2)
    cam = np.random.default_rng(0).standard_normal(jac.num_cams * 45)
    pt = np.random.default_rng(1).standard_normal(jac.num_points * 6)
    p = os.path.join(tmp_path, "t.cov")
    save_cov(p, jac, {"lambda": 1e-6, "fixed_pts": [1, 2, 3], "cycle_change": [3.0, 1.0]}, cam, pt)
    hdr, c, q = load_cov(p, jac.num_cams)
    assert hdr["TE number of iterations"] == "2"
    np.testing.assert_allclose(c.ravel(), cam, rtol=1e-5)
    np.testing.assert_allclose(q.ravel(), pt, rtol=1e-5)
