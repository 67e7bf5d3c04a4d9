"""SVD algorithms of computeCovariances (svdInverse, compute.cpp:185-249) on the GPU.

The pseudo-inverse building block is checked on synthetic PSD matrices with a
known spectrum (exact answer, tight tolerance). The full path is checked
against the oracle's LAPACK SVD on the small synthetic scene. That problem
has condition number ~1e12 (lambda_max 3.8e8, smallest kept eigenvalue
3.9e-4), so two FP64 LAPACK routes agree only to ~1e-3 (cameras) and ~1e-2
(points) per block. The test measures that floor itself (numpy's symmetric
eigensolver vs the oracle) and requires the GPU to be within twice of it.
"""
import numpy as np
import pytest

from conftest import block_rel_err, golden_jacobian
from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _psd(n, null, seed, lo=1.0, hi=1e3):
    """A PSD matrix with `null` zero eigenvalues and the rest log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.concatenate([np.zeros(null), np.exp(rng.uniform(np.log(lo), np.log(hi), n - null))])
    A = (Q * lam) @ Q.T
    return 0.5 * (A + A.T), Q, lam


def _pinv_gpu(A, remove_n, eps=1e-10):
    import torch
    n = A.shape[0]
    ld = (n + 7) & ~7
    buf = torch.zeros((n, ld), dtype=torch.float64, device="cuda")  # row i of buf = column i
    buf[:, :n] = torch.from_numpy(np.asfortranarray(A).T.copy())
    native.pinv_psd_device(buf.data_ptr(), n, ld, remove_n, eps)
    torch.cuda.synchronize()
    return buf[:, :n].cpu().numpy().T


@pytest.mark.parametrize("n,null", [(50, 7), (333, 7), (1000, 7), (129, 3)])
def test_pinv_known_spectrum(n, null):
    A, Q, lam = _psd(n, null, seed=n)
    ref = (Q[:, null:] / lam[null:]) @ Q[:, null:].T
    got = _pinv_gpu(A, null)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-10


def test_pinv_epsilon_rule():
    n = 200
    A, Q, lam = _psd(n, 0, seed=5)
    lam[:4] = [1e-14, 3e-13, 2e-12, 5e-12]  # four below epsilon = 1e-10, the rest >= 1
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    ref = (Q[:, 4:] / lam[4:]) @ Q[:, 4:].T
    got = _pinv_gpu(A, -1, 1e-10)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-9


def test_pinv_remove_none_is_inverse():
    A, _, _ = _psd(150, 0, seed=9)
    got = _pinv_gpu(A, 0)
    ref = np.linalg.inv(A)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-11


def test_pinv_rejects_extra_null_directions():
    A, _, _ = _psd(80, 9, seed=3)  # 9 null directions, only 7 removed
    with pytest.raises(native.UncError) as e:
        _pinv_gpu(A, 7)
    assert e.value.status == -6


def _eigh_outputs(jac, k=7):
    """Camera (a + b/2) and point outputs of the pseudo-inverse built from numpy's eigh."""
    import scipy.sparse as sp
    J = sp.csr_matrix((jac.values, jac.cols, jac.rows), shape=(jac.num_rows, jac.num_cols))
    M = (J.T @ J).toarray()
    w, V = np.linalg.eigh(M)
    keep = np.ones(len(w), bool)
    keep[np.argsort(np.abs(w))[:k]] = False
    P = (V[:, keep] / w[keep]) @ V[:, keep].T
    cam = []
    for c in range(jac.num_cams):
        B = P[9 * c:9 * c + 9, 9 * c:9 * c + 9]
        cam += [B[j, i] + B[i, j] / 2 for j in range(9) for i in range(j, 9)]
    b0, pt = 9 * jac.num_cams, []
    for q in range(jac.num_points):
        r = b0 + 3 * q
        pt += [P[r, r], P[r, r + 1], P[r, r + 2], P[r + 1, r + 1], P[r + 1, r + 2], P[r + 2, r + 2]]
    return np.array(cam), np.array(pt)


@pytest.mark.parametrize("algorithm", [0, 1])
def test_svd_path_small_scene_vs_oracle(algorithm):
    import oracle
    jac = scenes.synthetic_jacobian("small", seed=0)
    r = oracle.compute(jac, algorithm=algorithm, svd_remove_n=7)
    cam, pt, st = native.compute_covariances(jac, algorithm=algorithm)
    ce, pe = _eigh_outputs(jac)
    floor_c = block_rel_err(ce, r["cam"], 45)
    floor_p = block_rel_err(pe, r["pt"], 6)
    ec, ep = block_rel_err(cam, r["cam"], 45), block_rel_err(pt, r["pt"], 6)
    print(f"svd path: cams {ec:.2e} (LAPACK floor {floor_c:.2e}) points {ep:.2e} (floor {floor_p:.2e})")
    assert ec <= 2 * floor_c + 1e-9
    assert ep <= 2 * floor_p + 1e-9
    assert st["te_iterations"] > 0  # subspace iterations


def test_svd_path_daliborka_runs_and_repeats():
    """On 04_Daliborka the 7th and 8th smallest eigenvalues of J^T J are nearly
    equal (9.8e-6 vs 1.0e-5), so removing exactly 7 is ill-posed and LAPACK
    routes disagree by O(1); only completion, finiteness and determinism are
    checked here."""
    jac = golden_jacobian("daliborka")
    c1, p1, _ = native.compute_covariances(jac, algorithm=0)
    c2, p2, _ = native.compute_covariances(jac, algorithm=0)
    assert np.isfinite(c1).all() and np.isfinite(p1).all()
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(p1, p2)


def _schur_reference(jac, k=7, sample_points=None):
    """numpy restatement of the SVD on the camera Schur complement (this
    library's extension): Z = U - W V^-1 W^T of the unscaled, unfixed J^T J, its
    pseudo-inverse without the k smallest eigenvalues (eigh and SVD routes),
    camera outputs (a + b/2) and point covariances D^-1 + D^-1 (sum_o W_o^T
    Sigma_c W_o) D^-1 with the camera blocks of the pseudo-inverse."""
    import scipy.sparse as sp
    C, Pn = jac.num_cams, jac.num_points
    n = 9 * C
    J = sp.csr_matrix((jac.values, jac.cols, jac.rows), shape=(jac.num_rows, jac.num_cols))
    M = (J.T @ J).tocsr()
    U = M[:n, :n].toarray()
    W = M[:n, n:].tocsc()
    Vb = np.array([M[n + 3 * p:n + 3 * p + 3, n + 3 * p:n + 3 * p + 3].toarray() for p in range(Pn)])
    iV = np.linalg.inv(Vb)
    iVs = sp.block_diag(list(iV), format="csr")
    Z = U - (W @ iVs @ W.T).toarray()
    Z = 0.5 * (Z + Z.T)
    w, Q = np.linalg.eigh(Z)
    keep = np.ones(n, bool)
    keep[np.argsort(np.abs(w))[:k]] = False
    P_e = (Q[:, keep] / w[keep]) @ Q[:, keep].T
    Us, s, Vt = np.linalg.svd(Z)
    P_s = (Us[:, :n - k] / s[:n - k]) @ Vt[:n - k]

    def outputs(P):
        cam = []
        for c in range(C):
            B = P[9 * c:9 * c + 9, 9 * c:9 * c + 9]
            cam += [B[j, i] + B[i, j] / 2 for j in range(9) for i in range(j, 9)]
        pts = range(Pn) if sample_points is None else sample_points
        pt = np.zeros((Pn, 6))
        Wd = W.tocsc()
        for p in pts:
            Wp = Wd[:, 3 * p:3 * p + 3].toarray()  # 9C x 3
            S = np.zeros((3, 3))
            for c in np.nonzero(np.abs(Wp).sum(axis=1).reshape(C, 9).sum(axis=1))[0]:
                Wc = Wp[9 * c:9 * c + 9]
                S += Wc.T @ P[9 * c:9 * c + 9, 9 * c:9 * c + 9] @ Wc
            cov = iV[p] + iV[p] @ S @ iV[p]
            pt[p] = [cov[0, 0], cov[0, 1], cov[0, 2], cov[1, 1], cov[1, 2], cov[2, 2]]
        return np.array(cam), pt.reshape(-1)
    return outputs(P_e), outputs(P_s)


def test_svd_schur_small_scene_vs_numpy():
    jac = scenes.synthetic_jacobian("small", seed=0)
    (ce, pe), (cs, ps) = _schur_reference(jac)
    cam, pt, st = native.compute_covariances(jac, algorithm=native.SVD_SCHUR)
    floor_c, floor_p = block_rel_err(ce, cs, 45), block_rel_err(pe, ps, 6)
    ec, ep = block_rel_err(cam, ce, 45), block_rel_err(pt, pe, 6)
    print(f"svd on Z: cams {ec:.2e} (eigh vs svd {floor_c:.2e}) points {ep:.2e} (floor {floor_p:.2e})")
    assert ec <= max(4 * floor_c, 1e-9)
    assert ep <= max(4 * floor_p, 1e-9)
    assert st["te_iterations"] > 0


def test_svd_schur_medium_scene_cameras():
    """The medium scene (N = 1800), where the full-J^T J SVD would need 184 GB."""
    jac = scenes.synthetic_jacobian("medium", seed=0)
    (ce, pe), (cs, ps) = _schur_reference(jac, sample_points=range(0, jac.num_points, 997))
    cam, pt, st = native.compute_covariances(jac, algorithm=native.SVD_SCHUR)
    floor_c = block_rel_err(ce, cs, 45)
    ec = block_rel_err(cam, ce, 45)
    sel = np.zeros(jac.num_points, bool)
    sel[list(range(0, jac.num_points, 997))] = True
    ep = block_rel_err(pt.reshape(-1, 6)[sel], pe.reshape(-1, 6)[sel], 6)
    floor_p = block_rel_err(pe.reshape(-1, 6)[sel], ps.reshape(-1, 6)[sel], 6)
    print(f"svd on Z (medium): cams {ec:.2e} (floor {floor_c:.2e}) sampled points {ep:.2e} (floor {floor_p:.2e})")
    assert ec <= max(4 * floor_c, 1e-9)
    assert ep <= max(4 * floor_p, 1e-9)
