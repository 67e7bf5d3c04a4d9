"""The allocation-free dense inverse (collected last on purpose).

unc_dense_inverse_noalloc serves callers that cannot let a library allocate
device memory: applications whose device memory is reserved by their own pool
allocator, and latency-critical loops where cudaMalloc / cudaFree would stall
the device. It runs the recursive inverse with a fixed static scratch array,
while unc_dense_inverse_device takes the tile-task form at these sizes, so the
two inverse routes must agree within the dense-inverse tolerance; n and lda are
limited to 512.
"""
import numpy as np
import pytest

from uncertaintyte_b200 import native

pytestmark = pytest.mark.gpu

TOL = 1e-11  # the dense-inverse tolerance of the other GPU tests


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((n, n))
    return Q @ Q.T + n * np.eye(n)


def _run(fn, A, lda):
    import torch
    n = A.shape[0]
    buf = torch.zeros((n, lda), dtype=torch.float64, device="cuda")  # row i = column i (column-major)
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T))
    fn(buf.data_ptr(), n, lda)
    torch.cuda.synchronize()
    return buf[:, :n].cpu().numpy().T


@pytest.mark.parametrize("n,lda", [(300, 304), (512, 512), (65, 72)])
def test_noalloc_matches_allocating_inverse_twice(n, lda):
    for call, seed in enumerate((n, n + 1)):  # two calls in a row share the static scratch
        A = _spd(n, seed)
        ref = _run(native.dense_inverse_device, A, lda)
        got = _run(native.dense_inverse_noalloc, A, lda)
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got - ref)) / scale < TOL, (call, n)
        assert np.max(np.abs(got @ A - np.eye(n))) < 1e-10


def test_noalloc_rejects_sizes_beyond_the_static_scratch():
    import torch
    buf = torch.zeros((513, 520), dtype=torch.float64, device="cuda")
    with pytest.raises(native.UncError) as e:
        native.dense_inverse_noalloc(buf.data_ptr(), 513, 520)
    assert e.value.status == -8  # UNC_ERR_TOO_LARGE


def test_noalloc_call_allocates_no_device_memory():
    """The property the entry point exists for: after a first call (which loads
    the kernels and looks up the array's address), a call leaves the device's
    free memory and the caching allocator's allocation count unchanged."""
    import torch
    n, lda = 300, 304
    A = _spd(n, 7)
    src = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    buf = torch.zeros((n, lda), dtype=torch.float64, device="cuda")
    buf[:, :n] = src
    native.dense_inverse_noalloc(buf.data_ptr(), n, lda)  # warm-up
    buf[:, :n] = src
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    allocs0 = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
    native.dense_inverse_noalloc(buf.data_ptr(), n, lda)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    allocs1 = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
    assert free1 == free0, (free0, free1)
    assert allocs1 == allocs0
    got = buf[:, :n].cpu().numpy().T
    assert np.max(np.abs(got @ A - np.eye(n))) < 1e-10
