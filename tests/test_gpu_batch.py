"""Grouped batches (unc_batch_compute) against the per-scene path (needs a B200).

A batch runs the sparse stages of its scenes as parallel branches, the dense
stage grouped across scenes (one persistent tile-task inverse over every
scene's tasks, one launch per Taylor step over all product tiles), is
captured in a CUDA graph when its shape repeats, and picks its product tile
width by a cost model. None of that may change a single bit of any scene's
result: each scene must equal unc_compute on that scene alone, bitwise, on the
first call (direct), the second (captured) and the third (replayed), and with
either tile width forced."""
import numpy as np
import pytest

from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _scenes():
    counts = [8, 30, 12, 61, 25, 95, 9, 44, 140, 16, 70, 33]
    return [scenes.scene_jacobian(scenes.make_sized_scene(C, 60, 4, seed=500 + i)) for i, C in enumerate(counts)]


def _alone(jacs, precision):
    ctx = native.Context()
    out = [native.compute_covariances(j, ctx, precision=p) for j, p in zip(jacs, precision)]
    ctx.close()
    return out


def test_batch_bitwise_equal_to_per_scene_path_over_calls_and_tile_widths():
    jacs = _scenes()
    precs = ["mixed"] * len(jacs)
    precs[3] = "mixed4"   # a second grouped slice count
    precs[5] = "fp64"     # outside the grouped path: computed per scene in the same call
    ref = _alone(jacs, precs)
    b = native.Batch()
    for call, width in enumerate([0, 0, 0, 64, 96]):
        b.set_tile_width(width)
        got = b.compute(jacs, precision=precs)
        t = b.last_timing()
        assert t["grouped_scenes"] == len(jacs) - 1
        assert t["tile_n"] in (64, 96) and (width == 0 or t["tile_n"] == width)
        for k, ((c0, p0, s0), (c1, p1, s1, status)) in enumerate(zip(ref, got)):
            assert status == 0, (call, k, status)
            np.testing.assert_array_equal(c0, c1, err_msg=f"call {call} scene {k}")
            np.testing.assert_array_equal(p0, p1, err_msg=f"call {call} scene {k}")
            assert s1["te_iterations"] == s0["te_iterations"]
            assert s1["cycle_change"] == s0["cycle_change"]
            assert s1["lambda"] == s0["lambda"] and s1["fixed_pts"] == s0["fixed_pts"]
    b.close()


def test_batch_reports_a_bad_scene_and_solves_the_rest():
    jacs = _scenes()[:5]
    bad = jacs[2]
    bad.cols = bad.cols.copy()
    bad.cols[24 * 3 + 4] += 1  # observation 3's camera columns break the layout
    ref = _alone([j for k, j in enumerate(jacs) if k != 2], ["mixed"] * 4)
    b = native.Batch()
    got = b.compute(jacs)
    b.close()
    assert got[2][3] == -2  # UNC_ERR_LAYOUT
    for (c0, p0, _), (c1, p1, _, status) in zip(ref, [g for k, g in enumerate(got) if k != 2]):
        assert status == 0
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_array_equal(p0, p1)


def test_batch_tail_rule_of_fixed_points():
    """Fixed points past 6 (P - 3) keep the caller's values, as unc_compute does."""
    sc = scenes.make_sized_scene(10, 30, 3, seed=77)
    jac = scenes.scene_jacobian(sc)
    P = jac.num_points
    jac.pts2fix = np.array([P - 3, P - 2, P - 1], dtype=np.int32)
    init = [np.full(P * 6, 7.0)]
    c0, p0, _ = native.compute_covariances(jac, precision="mixed", pt_init=init[0])
    b = native.Batch()
    (c1, p1, _, status), = b.compute([jac], pt_init=init)
    b.close()
    assert status == 0
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(c0, c1)
    assert np.all(p1.reshape(-1, 6)[-3:] == 7.0)
