"""The tile-task SPD inverse (one persistent kernel over 64 x 64 tile tasks,
used by unc_dense_inverse_device and the pipeline for n <= 3584) against
numpy: partial edge tiles, the largest task size and the first recursive size
beyond it, bitwise repeatability, and a non-SPD input that must be reported
without hanging the schedule."""
import numpy as np
import pytest

from uncertaintyte_b200 import native

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    Q = rng.standard_normal((n, n))
    return Q @ Q.T + n * np.eye(n)


def _inverse(A):
    import torch
    n = A.shape[0]
    lda = (n + 7) & ~7
    buf = torch.zeros((n, lda), dtype=torch.float64, device="cuda")  # row i of buf = column i
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T))
    native.dense_inverse_device(buf.data_ptr(), n, lda)
    torch.cuda.synchronize()
    return buf[:, :n].cpu().numpy().T


@pytest.mark.parametrize("n", [2, 63, 64, 65, 128, 129, 191, 640, 1801, 3584, 3585])
def test_task_inverse_matches_numpy(n):
    A = _spd(n, n)
    got = _inverse(A)
    ref = np.linalg.inv(A)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TOL
    assert np.max(np.abs(got - got.T)) / np.max(np.abs(ref)) < TOL  # both triangles written


def test_task_inverse_bitwise_repeatable():
    A = _spd(700, 7)
    first = _inverse(A)
    for _ in range(3):
        np.testing.assert_array_equal(_inverse(A), first)


def test_task_inverse_reports_indefinite_input():
    A = _spd(300, 3)
    w, V = np.linalg.eigh(A)
    w[5] = -abs(w[5])  # one negative eigenvalue deep inside the spectrum
    with pytest.raises(native.UncError) as e:
        _inverse((V * w) @ V.T)
    assert e.value.status == -6
    # the schedule drained: the next call on the device works
    A = _spd(200, 4)
    assert np.max(np.abs(_inverse(A) @ A - np.eye(200))) < 1e-10


def _bounded(A, poll_limit, skip_task):
    import torch
    n = A.shape[0]
    lda = (n + 7) & ~7
    buf = torch.zeros((n, lda), dtype=torch.float64, device="cuda")
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(A.T))
    native.spd_inverse_tasks_bounded(buf.data_ptr(), n, lda, poll_limit, skip_task)
    torch.cuda.synchronize()
    return buf[:, :n].cpu().numpy().T


def test_bounded_wait_runs_out_and_the_device_stays_usable():
    """A schedule with one update task left out can never publish that tile's
    counter, so the tasks after it wait on a flag that nothing sets. With the
    waits limited to a few polls the launch must drain and the call return
    UNC_ERR_CUDA (a bounded wait ran out); the next calls on the device work."""
    import ctypes
    n = 640  # 10 x 10 tiles
    cnt = native.lib().unc_spd_task_list(n, None, 0)
    tasks = (ctypes.c_int * (4 * cnt))()
    native.lib().unc_spd_task_list(n, tasks, cnt)
    kinds = np.frombuffer(tasks, dtype=np.int32).reshape(-1, 4)[:, 0]
    skip = int(np.flatnonzero(kinds == 2)[0])  # the first trailing update
    A = _spd(n, 11)
    with pytest.raises(native.UncError) as e:
        _bounded(A, 2000, skip)
    assert e.value.status == -4  # UNC_ERR_CUDA
    assert "ran out" in str(e.value)
    # the same entry point with the full schedule, then the regular inverse
    ref = np.linalg.inv(A)
    got = _bounded(A, 1 << 22, -1)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TOL
    got = _inverse(A)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TOL
