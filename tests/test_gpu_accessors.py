"""Batched eigen-decompositions behind the Uncertainty accessors
(uncertainty.cpp:74-183) against numpy's symmetric eigensolver."""
import numpy as np
import pytest

from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _packed(blocks):
    p = blocks.shape[1]
    iu = np.triu_indices(p)
    return blocks[:, iu[0], iu[1]].reshape(-1)


def _check(blocks, vals, vecs):
    ref = np.linalg.eigvalsh(blocks)[:, ::-1]
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.max(np.abs(vals - ref) / scale) < 1e-12
    if vecs is not None:
        V = np.transpose(vecs, (0, 2, 1))  # columns = eigenvectors
        res = np.einsum("bij,bjk->bik", blocks, V) - V * vals[:, None, :]
        assert np.max(np.abs(res) / scale[:, :, None]) < 1e-12
        eye = np.einsum("bji,bjk->bik", V, V)
        assert np.max(np.abs(eye - np.eye(V.shape[1]))) < 1e-12


@pytest.mark.parametrize("p,n", [(9, 1000), (3, 5000)])
def test_random_spd_blocks(p, n):
    rng = np.random.default_rng(p)
    X = rng.standard_normal((n, p, p)) * np.exp(rng.uniform(-6, 6, (n, 1, p)))
    A = np.einsum("bij,bkj->bik", X, X)
    vals, vecs = native.block_eigen(_packed(A), p)
    _check(A, vals, vecs)


def test_camera_centre_sub_blocks():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((300, 9, 9))
    A = np.einsum("bij,bkj->bik", X, X)
    vals, vecs = native.block_eigen(_packed(A), 9, sub_offset=3, sub_dim=3)
    _check(A[:, 3:6, 3:6], vals, vecs)


def test_blocks_of_a_solve():
    jac = scenes.synthetic_jacobian("small", seed=2)
    cam, pt, _ = native.compute_covariances(jac, precision="mixed")
    full = []
    for c in cam.reshape(-1, 45):
        m = np.zeros((9, 9))
        m[np.triu_indices(9)] = c
        full.append(m + np.triu(m, 1).T)
    vals, _ = native.block_eigen(cam, 9, vectors=False)
    _check(np.array(full), vals, None)
    vals, vecs = native.block_eigen(pt, 3)
    P = []
    for q in pt.reshape(-1, 6):
        m = np.zeros((3, 3))
        m[np.triu_indices(3)] = q
        P.append(m + np.triu(m, 1).T)
    keep = np.abs(pt.reshape(-1, 6)).sum(axis=1) > 0  # fixed points are zero blocks
    _check(np.array(P)[keep], vals[keep], vecs[keep])
