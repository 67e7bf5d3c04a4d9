"""Mixed-precision Taylor products (int8-sliced tcgen05 GEMMs) against the
FP64 CPU oracle, the FP64 GPU path and torch FP64 products (needs a B200).

Tolerance: the accuracy target of the mixed path is a maximum relative
Frobenius error of 1e-6 per camera 9x9 block and per point 3x3 block against
the FP64 oracle (the reference's algorithm on the CPU); MIXED_TOL below is that
bar. The mixed path is also held to it against the FP64 GPU path.
"""
import numpy as np
import pytest

import oracle
from conftest import block_rel_err, golden_jacobian
from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def _mixed_vs_fp64(jac, ctx, precision="mixed", taylor="powers"):
    c64, p64, s64 = native.compute_covariances(jac, ctx, precision="fp64", taylor=taylor)
    cmp_, pmp, smp = native.compute_covariances(jac, ctx, precision=precision, taylor=taylor)
    assert smp["te_iterations"] == s64["te_iterations"]
    # the stop-rule values come from the products' max |entry|: same ~1e-8..1e-6 agreement
    np.testing.assert_allclose(smp["cycle_change"], s64["cycle_change"], rtol=1e-5)
    ec, ep = block_rel_err(cmp_, c64, 45), block_rel_err(pmp, p64, 6)
    ref = oracle.compute(jac, threads=8)
    oc, op = block_rel_err(cmp_, ref["cam"], 45), block_rel_err(pmp, ref["pt"], 6)
    assert smp["te_iterations"] == ref["stats"].te_iterations
    print(f"{precision}: vs FP64 GPU cams {ec:.3e} points {ep:.3e}; vs FP64 oracle cams {oc:.3e} points {op:.3e}")
    assert oc < MIXED_TOL and op < MIXED_TOL
    return ec, ep


@pytest.mark.parametrize("name", ["small", "medium"])
def test_mixed_vs_fp64_synthetic(ctx, name):
    ec, ep = _mixed_vs_fp64(scenes.synthetic_jacobian(name, seed=0), ctx)
    assert ec < MIXED_TOL and ep < MIXED_TOL


@pytest.mark.parametrize("taylor", ["powers", "sequential"])
def test_mixed_vs_fp64_daliborka(ctx, taylor):
    ec, ep = _mixed_vs_fp64(golden_jacobian("daliborka"), ctx, taylor=taylor)
    assert ec < MIXED_TOL and ep < MIXED_TOL


def test_mixed4_is_faster_and_coarser(ctx):
    """4 slices: ~1e-8 per camera block on the synthetic scenes (5 slices: ~1e-10)."""
    jac = scenes.synthetic_jacobian("small", seed=1)
    e5 = _mixed_vs_fp64(jac, ctx, "mixed")
    e4 = _mixed_vs_fp64(jac, ctx, "mixed4")
    assert e5[0] < 1e-8 and e5[0] <= e4[0] and e4[0] < MIXED_TOL


@pytest.mark.parametrize("n,slices,tol", [(1, 4, 1e-6), (70, 4, 1e-5), (200, 4, 1e-5), (1800, 4, 1e-5),
                                          (1800, 5, 1e-7), (257, 3, 1e-3), (130, 5, 1e-7), (6000, 5, 1e-7)])
def test_mixed_gemm_vs_torch(n, slices, tol):
    import torch
    g = torch.Generator(device="cuda").manual_seed(n + slices)
    A = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    P, X = A + A.T, B @ B.T / n
    C = torch.zeros_like(P)
    native.gemm_mixed_device(n, P.data_ptr(), X.data_ptr(), n, C.data_ptr(), slices)
    torch.cuda.synchronize()
    ref = (P @ X).T  # column-major C read row-major by torch
    rel = ((C - ref).norm() / ref.norm()).item()
    assert rel < tol, rel


def _lower_factor_inverse(n, seed, cond):
    """T = L^-1 of a Jacobi-equilibrated SPD matrix with eigenvalues spread over `cond`."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    ev = torch.logspace(0, -float(np.log10(cond)), n, dtype=torch.float64, device="cuda")
    A = (Q * ev) @ Q.T
    d = A.diagonal().rsqrt()
    A = A * d[:, None] * d[None, :]
    L = torch.linalg.cholesky(A)
    return torch.linalg.solve_triangular(L, torch.eye(n, dtype=torch.float64, device="cuda"), upper=False)


@pytest.mark.parametrize("n,kind", [(1, "rand"), (70, "rand"), (130, "rand"), (1000, "factor"),
                                    (3701, "factor"), (4100, "rand")])
def test_mixed_gram_lower_vs_torch(n, kind):
    """A = T^T T of a lower-triangular T from 7 int8 slices (the mixed inverse's last
    product), against torch FP64. The slicing's error per term is about 2^-50 of
    the product of the two columns' maxima and zero-mean: every element within
    2e-11 of that scale, and the diagonal (sums of squares, where a dropped
    squared digit would add up with one sign over K) without a bias: the mean
    signed error of the diagonal over its scale below 1e-12."""
    import torch
    if kind == "rand":
        g = torch.Generator(device="cuda").manual_seed(n)
        T = torch.tril(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    else:
        T = _lower_factor_inverse(n, n, 1e8)
    M = T.T.contiguous()  # memory of the column-major T
    A = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    native.gram_lower_mixed_device(n, M.data_ptr(), n, A.data_ptr())
    torch.cuda.synchronize()
    ref = T.T @ T
    m = T.abs().amax(dim=0)  # column maxima of T
    scale = m[:, None] * m[None, :]
    err = ((A - ref).abs() / scale).max().item()
    bias = ((A - ref).diagonal() / scale.diagonal()).mean().item()
    assert torch.isfinite(A).all()
    assert torch.equal(A, A.T)  # both triangles written, bitwise symmetric
    assert err < 2e-11, err
    assert abs(bias) < 1e-12, bias

