"""Request server: continuous batching of many reconstructions on one GPU.

Each result must be the same alone and in a mix: the server runs several
requests concurrently on separate streams, and every request's arithmetic uses
fixed reduction orders and no atomics, so the comparison is bitwise.
"""
import numpy as np
import pytest

from uncertaintyte_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _jobs():
    """Mixed sizes (8 .. 90 cameras), both precisions, one SVD request."""
    out = []
    for i, C in enumerate([8, 40, 12, 90, 25, 60, 9, 33, 70, 16]):
        jac = scenes.scene_jacobian(scenes.make_sized_scene(C, 60, 4, seed=100 + i))
        out.append((jac, "fp64" if i % 3 == 0 else "mixed", None))
    svd = scenes.scene_jacobian(scenes.make_sized_scene(10, 30, 3, seed=7))
    out.append((svd, "fp64", 0))
    return out


def _alone(jobs):
    ctx = native.Context()
    res = [native.compute_covariances(j, ctx, algorithm=a, precision=p)[:2] for j, p, a in jobs]
    ctx.close()
    return res


def test_results_identical_alone_and_in_the_mix():
    jobs = _jobs()
    ref = _alone(jobs)
    srv = native.Server(max_inflight=4)
    ids = [srv.submit(j, precision=p, algorithm=a) for j, p, a in jobs]
    got = [srv.wait(i)[:2] for i in ids]
    srv.close()
    for (c0, p0), (c1, p1) in zip(ref, got):
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_array_equal(p0, p1)


def test_tight_budget_serialises_but_completes():
    jobs = _jobs()[:6]
    need = max(native.request_bytes(j, precision=p, algorithm=a) for j, p, a in jobs)
    ref = _alone(jobs)
    srv = native.Server(max_device_bytes=int(need * 1.2), max_inflight=4)
    ids = [srv.submit(j, precision=p, algorithm=a) for j, p, a in jobs]
    out = [srv.wait(i) for i in ids]
    srv.close()
    for (c0, p0), (c1, p1, st, lat, que) in zip(ref, out):
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_array_equal(p0, p1)
        assert lat >= que >= 0.0


def test_request_above_budget_is_refused():
    jac = scenes.scene_jacobian(scenes.make_sized_scene(40, 60, 4, seed=3))
    srv = native.Server(max_device_bytes=1 << 20, max_inflight=2)
    with pytest.raises(native.UncError) as e:
        srv.submit(jac)
    assert e.value.status == -5  # UNC_ERR_OUT_OF_MEMORY
    srv.close()


def test_wait_timeout_and_single_collection():
    jac = scenes.scene_jacobian(scenes.make_sized_scene(120, 150, 4, seed=11))
    srv = native.Server(max_inflight=1)
    rid = srv.submit(jac)
    try:
        srv.wait(rid, timeout=0.0)
        finished_early = True
    except native.UncError as e:
        assert e.status == -9  # UNC_ERR_TIMEOUT: still running
        finished_early = False
    if not finished_early:
        cam, pt, st, lat, que = srv.wait(rid)
        assert np.isfinite(cam).all() and st["te_iterations"] > 0
    with pytest.raises(native.UncError):
        srv.wait(rid)  # already collected
    srv.close()


def test_waiters_survive_concurrent_submits():
    """One thread waits on a long request while the main thread submits enough
    requests to make the server's id table grow (rehash) several times; a second
    waiter on the same id fails cleanly instead of sharing the result."""
    import threading
    big = scenes.scene_jacobian(scenes.make_sized_scene(600, 100, 4, seed=21))
    tiny = scenes.scene_jacobian(scenes.make_sized_scene(8, 20, 3, seed=22))
    srv = native.Server(max_inflight=2)
    rid = srv.submit(big, precision="fp64")
    outcome = {}

    def waiter(name):
        try:
            outcome[name] = srv.wait(rid)
        except native.UncError as e:
            outcome[name] = e

    threads = [threading.Thread(target=waiter, args=(k,)) for k in ("a", "b")]
    for t in threads:
        t.start()
    ids = [srv.submit(tiny, precision="mixed") for _ in range(600)]
    for t in threads:
        t.join(timeout=600)
    got = [srv.wait(i)[:2] for i in ids]
    srv.close()
    ok = [v for v in outcome.values() if isinstance(v, tuple)]
    bad = [v for v in outcome.values() if isinstance(v, native.UncError)]
    assert len(ok) == 1 and len(bad) == 1, outcome
    assert bad[0].status == -1  # UNC_ERR_INVALID_ARG: waited for or collected by the other thread
    assert np.isfinite(ok[0][0]).all() and ok[0][2]["te_iterations"] > 0
    for c, p in got[1:]:
        np.testing.assert_array_equal(c, got[0][0])
        np.testing.assert_array_equal(p, got[0][1])


def test_worker_frees_its_other_workspace_for_room():
    """One worker and a budget that holds the large request plus half of the
    small ones: the large request grows the worker's context workspace, the
    small ones queued behind it run as one pack in the batch workspace (the
    admission counts both, so the worker frees its context workspace first),
    and the large request submitted again frees the batch workspace. Results
    equal those of the requests run alone."""
    big = scenes.scene_jacobian(scenes.make_sized_scene(400, 100, 4, seed=41))
    smalls = [scenes.scene_jacobian(scenes.make_sized_scene(C, 60, 4, seed=50 + i))
              for i, C in enumerate([10, 14, 12, 9, 11])]
    need_big = native.request_bytes(big, precision="mixed")
    need_small = sum(native.request_bytes(j, precision="mixed") for j in smalls)
    budget = need_big + need_small // 2
    ref = _alone([(j, "mixed", None) for j in [big] + smalls])
    srv = native.Server(max_device_bytes=budget, max_inflight=1)
    ids = [srv.submit(big, precision="mixed")] + [srv.submit(j, precision="mixed") for j in smalls]
    got = [srv.wait(i)[:2] for i in ids]
    got.append(srv.wait(srv.submit(big, precision="mixed"))[:2])
    srv.close()
    for (c0, p0), (c1, p1) in zip(ref + ref[:1], got):
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_array_equal(p0, p1)
