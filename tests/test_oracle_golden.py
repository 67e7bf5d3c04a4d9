"""The CPU oracle against the reference's own golden data (no GPU).

Pins the oracle before it is trusted as the checker of the CUDA path:
  * test/EigValues/output.cov   end-to-end TAYLOR_EXPANSION on 04_Daliborka
  * test/SparseMatrix/multipl_*  J^T J pattern and values
  * test/*/inv_*_01              equilibrated LU inverse
"""
import numpy as np
import pytest

import oracle
from conftest import block_rel_err, golden, golden_jacobian


@pytest.fixture(scope="module")
def daliborka():
    jac = golden_jacobian("daliborka")
    return jac, oracle.compute(jac, threads=8), golden("daliborka")


def test_daliborka_header(daliborka):
    jac, out, g = daliborka
    st = out["stats"]
    assert list(st.fixed_pts) == list(g["gold_fixed"])
    assert abs(st.lam - g["gold_lambda"]) <= 1e-5 * g["gold_lambda"]
    # all 14 cycle-change values, including the 14th which depends on the
    # reference's 32-bit factorial wrapping at 13!
    cc = np.array(st.cycle_change[: st.te_iterations])
    assert st.te_iterations == len(g["gold_cycle_change"]) == 14
    np.testing.assert_allclose(cc, g["gold_cycle_change"], rtol=1e-5)


def test_daliborka_cameras(daliborka):
    jac, out, g = daliborka
    # the golden file prints 6 significant digits
    assert block_rel_err(out["cam"], g["gold_cam"], 45) < 1e-5


def test_daliborka_points(daliborka):
    jac, out, g = daliborka
    pt = out["pt"].reshape(-1, 6)
    gp = g["gold_pt"]
    for f in g["gold_fixed"]:
        assert np.all(pt[f] == 0) and np.all(gp[f] == 0)
    assert block_rel_err(pt, gp, 6) < 1e-5


def test_outputs_read_only_the_camera_blocks_of_iz(daliborka):
    """The reference's outputs depend on the final Taylor-series inverse iZ only
    through its 9 x 9 diagonal camera blocks (removeScaleJ4Z, compute.cpp:168-183,
    and the block-diagonal camera covariance of the point stage, compute.cpp:422-441):
    with every other entry of iZ set to NaN the outputs are bitwise the same. The
    CUDA path relies on this when it forms the last Taylor terms on those blocks only."""
    jac, out, g = daliborka
    masked = oracle.compute(jac, threads=8, offdiag_nan=True)
    np.testing.assert_array_equal(masked["cam"], out["cam"])
    np.testing.assert_array_equal(masked["pt"], out["pt"])


def test_daliborka_faithful_scan_matches_indexed(daliborka):
    jac, out, g = daliborka
    out2 = oracle.compute(jac, threads=8, faithful_point_scan=True)
    np.testing.assert_array_equal(out2["pt"], out["pt"])


def test_jtj_golden_pattern_and_values():
    d = golden("multipl_01")
    nr, nc = d["in_dims"]
    r, c, v = oracle.jtj(int(nr), int(nc), d["in_rows"], d["in_cols"], d["in_vals"])
    np.testing.assert_array_equal(r, d["out_rows"])
    np.testing.assert_array_equal(c, d["out_cols"])
    np.testing.assert_allclose(v, d["out_vals"], rtol=1e-10, atol=0)


@pytest.mark.parametrize("name", ["inv_sparse_01", "inv_dense_01"])
def test_dense_inverse_golden(name):
    d = golden(name)
    Ai, info = oracle.dense_inv(d["A"])
    assert info == 0
    # the reference's test tolerance is 1e-7 (uncTest_DenseMatrix.cpp)
    assert np.max(np.abs(Ai - d["Ainv"])) / np.max(np.abs(d["Ainv"])) < 1e-9


def test_factorial_wrap_changes_14th_term(daliborka):
    """With the true 13! the 14th change would be 2.57e-5 instead of 8.27e-5."""
    jac, out, g = daliborka
    st = out["stats"]
    ratio = 6227020800 / 1932053504  # 13! / (13! mod 2^32)
    assert abs(st.cycle_change[13] / ratio - 2.567e-5) < 2e-7


def test_oracle_rejects_missing_fixed_points():
    jac = golden_jacobian("toy")  # 03_Toy carries -1 -1 -1
    assert jac.pts2fix is None
    with pytest.raises(ValueError):
        oracle.compute(jac)


def test_oracle_svd_path_runs_on_toy():
    jac = golden_jacobian("toy")
    out = oracle.compute(jac, algorithm=0, svd_remove_n=7)
    out1 = oracle.compute(jac, algorithm=1, svd_remove_n=7)
    assert np.all(np.isfinite(out["cam"])) and np.all(np.isfinite(out["pt"]))
    # The unscaled, unfixed J^T J of 03_Toy has its 7 gauge eigenvalues and the
    # next few all at the FP64 noise floor (~1e-15 of the largest), so the two
    # LAPACK SVD drivers only agree to a few 1e-3 on the pseudo-inverse.
    assert block_rel_err(out1["cam"], out["cam"], 45) < 1e-2


def test_oracle_gemm_and_cholesky_route():
    """The dense product restated from operator*= (scaling, dgemm, unscaling) and
    the Cholesky route of the inverse agree with numpy; on Daliborka the two
    inverse routes give the same iteration count and results at the FP64 floor."""
    import oracle
    rng = np.random.default_rng(5)
    A, B = rng.standard_normal((300, 300)), rng.standard_normal((300, 300))
    C = oracle.gemm(A, B)
    assert np.max(np.abs(C - A @ B)) / np.max(np.abs(A @ B)) < 1e-13
    S = A @ A.T + 300 * np.eye(300)
    Si, info = oracle.dense_inv_cholesky(S)
    assert info == 0 and np.max(np.abs(Si - np.linalg.inv(S))) / np.max(np.abs(np.linalg.inv(S))) < 1e-13
    from conftest import block_rel_err, golden_jacobian
    jac = golden_jacobian("daliborka")
    lu = oracle.compute(jac, threads=8)
    ch = oracle.compute(jac, threads=8, route="cholesky")
    assert ch["stats"].te_iterations == lu["stats"].te_iterations == 14
    assert block_rel_err(ch["cam"], lu["cam"], 45) < 1e-8
    assert block_rel_err(ch["pt"], lu["pt"], 6) < 1e-8
