"""Reprojection Jacobian built on the GPU from the scene (replaces Ceres Evaluate,
JacobianComposer.cpp:123-166) against the analytic blocks of the scene
generator (numpy), and the whole solve from the scene against the CRS path."""
import numpy as np
import pytest

from conftest import block_rel_err
from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _gpu_jacobian(sc):
    import torch
    n = len(sc.obs_cam)
    dev = "cuda"
    cams = torch.from_numpy(np.ascontiguousarray(sc.cams)).to(dev)
    pts = torch.from_numpy(np.ascontiguousarray(sc.points)).to(dev)
    oc = torch.from_numpy(np.ascontiguousarray(sc.obs_cam, dtype=np.int32)).to(dev)
    op = torch.from_numpy(np.ascontiguousarray(sc.obs_pt, dtype=np.int32)).to(dev)
    rows = torch.zeros(2 * n + 1, dtype=torch.int32, device=dev)
    cols = torch.zeros(24 * n, dtype=torch.int32, device=dev)
    vals = torch.zeros(24 * n, dtype=torch.float64, device=dev)
    native._check(native.lib().unc_jacobian_device(len(sc.cams), len(sc.points), n, cams.data_ptr(),
                                                   pts.data_ptr(), oc.data_ptr(), op.data_ptr(), rows.data_ptr(),
                                                   cols.data_ptr(), vals.data_ptr(), None))
    return rows.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy()


@pytest.mark.parametrize("name", ["small", "medium"])
def test_jacobian_matches_analytic_blocks(name):
    sc = scenes.make_scene(name, 0)
    ref = scenes.scene_jacobian(sc)
    rows, cols, vals = _gpu_jacobian(sc)
    np.testing.assert_array_equal(rows, ref.rows)
    np.testing.assert_array_equal(cols, ref.cols)
    v, r = vals.reshape(-1, 12), ref.values.reshape(-1, 12)
    scale = np.abs(r).max(axis=1, keepdims=True)
    assert np.max(np.abs(v - r) / scale) < 1e-11


def test_jacobian_small_and_large_rotation_angles():
    sc = scenes.make_sized_scene(12, 40, 3, seed=4)
    sc.cams[0, 0:3] = [3e-7, -2e-7, 1e-7]   # below the first-order threshold
    sc.cams[1, 0:3] *= 1e-3
    ref = scenes.scene_jacobian(sc)
    _, _, vals = _gpu_jacobian(sc)
    v, r = vals.reshape(-1, 12), ref.values.reshape(-1, 12)
    assert np.max(np.abs(v - r) / np.abs(r).max(axis=1, keepdims=True)) < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_from_scene_matches_crs_path(precision):
    sc = scenes.make_scene("small", 3)
    jac = scenes.scene_jacobian(sc)
    c0, p0, s0 = native.compute_covariances(jac, precision=precision)
    c1, p1, s1 = native.compute_covariances_scene(sc, jac.pts2fix, precision=precision)
    assert s1["te_iterations"] == s0["te_iterations"]
    assert block_rel_err(c1, c0, 45) < 1e-7
    assert block_rel_err(p1, p0, 6) < 1e-7


def test_scene_ids_out_of_range_are_refused():
    sc = scenes.make_scene("tiny", 0)
    sc.obs_cam = sc.obs_cam.copy()
    sc.obs_cam[5] = 99
    with pytest.raises(native.UncError) as e:
        native.compute_covariances_scene(sc, scenes.farthest_triple(sc.points))
    assert e.value.status == -1
