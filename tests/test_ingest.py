"""`.jacob` ingest (JacobianIO.cpp:32-63) with the library's parallel parser, and
its binary form: round trips, comments, malformed files. CPU only."""
import numpy as np
import pytest

from conftest import golden_jacobian
from uncertaintyte_b200 import jacob, native, scenes


def _same(a, b):
    assert (a.num_cams, a.cam_params, a.num_points, a.num_obs, a.num_rows, a.num_cols) == \
        (b.num_cams, b.cam_params, b.num_points, b.num_obs, b.num_rows, b.num_cols)
    np.testing.assert_array_equal(a.rows, b.rows)
    np.testing.assert_array_equal(a.cols, b.cols)
    np.testing.assert_array_equal(a.values, b.values)  # %.17g text round-trips exactly
    assert (a.pts2fix is None) == (b.pts2fix is None)
    if a.pts2fix is not None:
        np.testing.assert_array_equal(a.pts2fix, b.pts2fix)


@pytest.mark.parametrize("name", ["daliborka", "cube", "toy"])
def test_text_round_trip_goldens(tmp_path, name):
    j = golden_jacobian(name)
    p = str(tmp_path / "x.jacob")
    jacob.save_jacob(p, j)
    _same(jacob.load_jacob(p), j)
    _same(jacob.load_jacob_numpy(p), j)


def test_parallel_parse_of_a_large_body(tmp_path):
    j = scenes.synthetic_jacobian("small", seed=5)  # ~70k numbers: several chunks at 1 MB of text
    reps = 20
    big = jacob.Jacobian(j.num_cams, j.cam_params, j.num_points, j.num_obs * reps, j.num_rows * reps,
                         j.num_cols, np.arange(0, 12 * j.num_rows * reps + 1, 12, dtype=np.int32),
                         np.tile(j.cols, reps), np.tile(j.values, reps), -1.0, j.pts2fix)
    p = str(tmp_path / "big.jacob")
    jacob.save_jacob(p, big)
    _same(jacob.load_jacob(p), big)


def test_binary_round_trip(tmp_path):
    j = scenes.synthetic_jacobian("small", seed=1)
    p = str(tmp_path / "x.jacobb")
    native.write_jacob_binary(p, j)
    k = jacob.load_jacob(p)
    _same(k, j)
    assert k.lam == j.lam


def test_comments_are_whitespace(tmp_path):
    p = tmp_path / "c.jacob"
    p.write_text("# a 1-camera toy\n-1 1 9 0 1 # header\n-1 -1 -1\n2 9 18\n0 9 18\n"
                 + " ".join(str(i) for i in range(9)) + " " + " ".join(str(i) for i in range(9)) + "\n"
                 + " ".join(f"{0.5 * i}" for i in range(18)) + " # values\n")
    k = jacob.load_jacob(str(p))
    assert k.num_rows == 2 and k.nnz == 18 and k.pts2fix is None
    np.testing.assert_array_equal(k.values, 0.5 * np.arange(18))


@pytest.mark.parametrize("body", ["0 9 18\n1 2 3\n", "0 9 18\n" + "1 " * 18 + "x " * 18])
def test_malformed_files_are_refused(tmp_path, body):
    p = tmp_path / "bad.jacob"
    p.write_text("-1 1 9 0 1\n-1 -1 -1\n2 9 18\n" + body)
    with pytest.raises(native.UncError) as e:
        jacob.load_jacob(str(p))
    assert e.value.status == -1


def test_header_mismatch_is_refused(tmp_path):
    j = golden_jacobian("cube")
    p = str(tmp_path / "x.jacob")
    jacob.save_jacob(p, j)
    h = native.UncJacobHeader()
    native._check(native.lib().unc_jacob_read_header(p.encode(), h))
    h.nnz += 1
    rows = np.empty(h.num_rows + 1, dtype=np.int32)
    cols = np.empty(h.nnz, dtype=np.int32)
    vals = np.empty(h.nnz)
    assert native.lib().unc_jacob_read(p.encode(), h, rows.ctypes.data, cols.ctypes.data, vals.ctypes.data) == -1
