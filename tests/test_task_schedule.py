"""The task order of the tile-task SPD inverse (dag.cu), checked on the CPU:
executed one task at a time in list order, every task finds its inputs ready
(the property that lets the persistent kernel finish with any number of
resident CTAs), every tile update comes exactly once and in order, and a numpy
restatement of the tasks on small matrices gives the inverse."""
import numpy as np
import pytest

from uncertaintyte_b200 import native

TB = 64
POTRF, TRSM, UPDATE, TACC, TFIN, PACC = range(6)


def _run(tasks, n, A0=None):
    """Execute tasks in order with the kernel's wait conditions as assertions;
    with A0, also do the tile arithmetic (numpy) and return the inverse."""
    nt = (n + TB - 1) // TB
    ver, tacc, pacc = {}, {}, {}
    lrdy, trdy = set(), set()
    num = A0 is not None
    if num:
        A, T, O = A0.copy(), np.zeros((n, n)), np.full((n, n), np.nan)
    sl = lambda b: slice(TB * b, min(n, TB * (b + 1)))  # noqa: E731
    for kind, i, j, k in tasks:
        if kind == POTRF:
            if k > 0:  # its last update, from panel k-1, is applied inside the task
                assert ver.get((k, k), 0) >= k - 1 and (k, k - 1) in lrdy
                if num:
                    A[sl(k), sl(k)] -= A[sl(k), sl(k - 1)] @ A[sl(k), sl(k - 1)].T
            if num:
                L = np.linalg.cholesky(np.tril(A[sl(k), sl(k)]) + np.tril(A[sl(k), sl(k)], -1).T)
                T[sl(k), sl(k)] = np.linalg.inv(L)
            lrdy.add((k, k))
            trdy.add((k, k))
            if k + 1 < nt:  # and the next panel's first solve
                assert ver.get((k + 1, k), 0) >= k
                if num:
                    A[sl(k + 1), sl(k)] = A[sl(k + 1), sl(k)] @ T[sl(k), sl(k)].T
                lrdy.add((k + 1, k))
        elif kind == TRSM:
            assert ver.get((i, k), 0) >= k and (k, k) in lrdy and (i, k) not in lrdy
            if num:
                A[sl(i), sl(k)] = A[sl(i), sl(k)] @ T[sl(k), sl(k)].T
            lrdy.add((i, k))
        elif kind == UPDATE:
            assert k < j <= i and ver.get((i, j), 0) == k and (i, k) in lrdy and (j, k) in lrdy
            if num:
                A[sl(i), sl(j)] -= A[sl(i), sl(k)] @ A[sl(j), sl(k)].T
            ver[(i, j)] = k + 1
        elif kind == TACC:
            assert j <= k < i and tacc.get((i, j), 0) == k - j and (i, k) in lrdy and (k, j) in trdy
            if num:
                P = A[sl(i), sl(k)] @ T[sl(k), sl(j)]
                T[sl(i), sl(j)] = P if k == j else T[sl(i), sl(j)] + P
            tacc[(i, j)] = k - j + 1
        elif kind == TFIN:
            assert j < i and tacc.get((i, j), 0) == i - j and (i, i) in trdy and (i, j) not in trdy
            if num:
                T[sl(i), sl(j)] = -T[sl(i), sl(i)] @ T[sl(i), sl(j)]
            trdy.add((i, j))
        else:
            assert j <= i <= k and pacc.get((i, j), 0) == k - i and (k, i) in trdy and (k, j) in trdy
            if num:
                P = T[sl(k), sl(i)].T @ T[sl(k), sl(j)]
                O[sl(i), sl(j)] = P if k == i else O[sl(i), sl(j)] + P
                if k == nt - 1 and i > j:
                    O[sl(j), sl(i)] = O[sl(i), sl(j)].T
            pacc[(i, j)] = k - i + 1
    # every lower tile: all its updates, its L, its T and all its product terms
    for i in range(nt):
        for j in range(i + 1):
            assert (i, j) in lrdy and (i, j) in trdy
            assert pacc[(i, j)] == nt - i
            if j < i:
                assert ver.get((i, j), 0) == j and tacc[(i, j)] == i - j
            else:
                assert ver.get((i, i), 0) == max(i - 1, 0)
    return O if num else None


@pytest.mark.parametrize("n", [1, 64, 65, 200, 640])
def test_schedule_computes_the_inverse(n):
    tasks = native.spd_task_list(n)
    rng = np.random.default_rng(n)
    Q = rng.standard_normal((n, n))
    A = Q @ Q.T + n * np.eye(n)
    O = _run(tasks, n, A)
    ref = np.linalg.inv(A)
    assert np.max(np.abs(O - ref)) / np.max(np.abs(ref)) < 1e-12


@pytest.mark.parametrize("n", [1800, 3584])
def test_schedule_is_topological_at_size(n):
    tasks = native.spd_task_list(n)
    nt = (n + TB - 1) // TB
    counts = np.bincount(tasks[:, 0], minlength=6)
    assert counts[POTRF] == nt and counts[TFIN] == nt * (nt - 1) // 2
    assert counts[PACC] == nt * (nt + 1) * (nt + 2) // 6
    _run(tasks, n)


def test_schedule_rejects_sizes_outside_the_task_range():
    for n in (0, 3585):
        with pytest.raises(native.UncError) as e:
            native.spd_task_list(n)
        assert e.value.status == -1
