"""The C++ drop-in interface and the command-line tool, executed (needs a B200).

A small C++ program (tests/dropin_check.cpp) is compiled against
include/uncertainty.h and linked with libuncte.so, as an uncertaintyTE user
would build: it calls computeCovariances (compute.h:92-97), both
getCovariances overloads (include/uncertainty.h:55-62, uncertainty.cpp:20-30)
and the Uncertainty accessors (uncertainty.cpp:46-183). The `uncertainty`
tool is run on 04_Daliborka.jacob as main_uncertainty.cpp:66-93 is, and its
.cov is parsed back.

Bars: the reference's own goldens at their own tolerances (output.cov: 1e-5
relative per block, it prints 6 digits; the accessor test
covarianceEigenValues_test.cpp:81-136: 1e-5 absolute for the matrices, 1e-5
relative for the eigenvalues); the C++ entry points against the C ABI on the
same input bitwise (the same library call underneath).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, block_rel_err, golden, golden_jacobian
from uncertaintyte_b200 import jacob, native, scenes

pytestmark = pytest.mark.gpu

LIBDIR = os.path.join(ROOT, "uncertaintyte_b200")


@pytest.fixture(scope="module")
def prog(tmp_path_factory):
    d = tmp_path_factory.mktemp("dropin")
    exe = str(d / "dropin_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin_check.cpp"), "-o", exe, "-L" + LIBDIR, "-luncte",
                    "-Wl,-rpath," + LIBDIR], check=True)
    return exe, d


def _read(path, *sizes):
    a = np.fromfile(path, dtype=np.float64)
    assert a.size == sum(sizes), (a.size, sizes)
    out, o = [], 0
    for s in sizes:
        out.append(a[o:o + s])
        o += s
    return out


def test_cpp_entry_points_on_daliborka(prog):
    exe, d = prog
    jac = golden_jacobian("daliborka")
    g = golden("daliborka")
    path = str(d / "daliborka.jacob")
    jacob.save_jacob(path, jac)
    subprocess.run([exe, path, str(d / "dal")], check=True, timeout=300)
    C, P = jac.num_cams, jac.num_points
    cam_c, pt_c = _read(str(d / "dal.compute.bin"), 45 * C, 6 * P)
    cam_g, pt_g = _read(str(d / "dal.get5.bin"), 45 * C, 6 * P)
    stats = open(str(d / "dal.stats.txt")).read().split()
    lam, iters, fx = float(stats[0]), int(stats[1]), [int(x) for x in stats[2:5]]
    cc = [float(x) for x in stats[5:]]
    assert iters == 14 and len(cc) == 14
    assert fx == list(g["gold_fixed"])
    assert abs(lam - g["gold_lambda"]) < 1e-5 * g["gold_lambda"]
    np.testing.assert_allclose(cc, g["gold_cycle_change"], rtol=1e-5)
    for cam, pt in ((cam_c, pt_c), (cam_g, pt_g)):
        assert block_rel_err(cam, g["gold_cam"], 45) < 1e-5
        assert block_rel_err(pt, g["gold_pt"], 6) < 1e-5
    # the same library call underneath: bitwise equal to the C ABI
    c_abi, p_abi, _ = native.compute_covariances(jac)
    np.testing.assert_array_equal(cam_c, c_abi)
    np.testing.assert_array_equal(pt_c, p_abi)
    np.testing.assert_array_equal(cam_g, cam_c)
    np.testing.assert_array_equal(pt_g, pt_c)


def test_cpp_gauge_choice_and_accessors(prog):
    """getCovariances(..., points3D, Uncertainty&) picks the fixed points itself
    (deterministically here; the reference samples random triples) and fills the
    Uncertainty; its accessors decompose every block on the GPU."""
    exe, d = prog
    sc = scenes.make_scene("small", seed=3)
    jac = scenes.scene_jacobian(sc)  # the file names fixed points (the first two calls need them)
    path = str(d / "small.jacob")
    jacob.save_jacob(path, jac)
    pts = str(d / "small_pts.bin")
    np.ascontiguousarray(sc.points, dtype=np.float64).tofile(pts)
    subprocess.run([exe, path, str(d / "sm"), pts], check=True, timeout=300)
    C, P = jac.num_cams, jac.num_points
    fixed, cam, pt, cev, pev, cvec, pvec = _read(str(d / "sm.unc.bin"), 6, 45 * C, 6 * P, 9 * C, 3 * P, 9 * C,
                                                 9 * P)
    triple = scenes.farthest_triple(sc.points)
    assert list(fixed[:3].astype(int)) == list(triple) == list(fixed[3:].astype(int))
    jac.pts2fix = triple
    c_abi, p_abi, _ = native.compute_covariances(jac)
    np.testing.assert_array_equal(cam, c_abi)
    np.testing.assert_array_equal(pt, p_abi)
    iu9, iu3 = np.triu_indices(9), np.triu_indices(3)
    Bc = np.zeros((C, 9, 9))
    Bc[:, iu9[0], iu9[1]] = cam.reshape(C, 45)
    Bc = Bc + np.transpose(np.triu(Bc, 1), (0, 2, 1))
    Bp = np.zeros((P, 3, 3))
    Bp[:, iu3[0], iu3[1]] = pt.reshape(P, 6)
    Bp = Bp + np.transpose(np.triu(Bp, 1), (0, 2, 1))
    ref_c = np.linalg.eigvalsh(Bc)[:, ::-1]
    ref_p = np.linalg.eigvalsh(Bp)[:, ::-1]
    live = np.abs(ref_p).max(axis=1) > 0  # fixed points are left 0
    assert np.max(np.abs(cev.reshape(C, 9) - ref_c) / np.abs(ref_c).max(axis=1, keepdims=True)) < 1e-12
    assert np.max(np.abs(pev.reshape(P, 3)[live] - ref_p[live]) / np.abs(ref_p[live]).max(axis=1, keepdims=True)) \
        < 1e-12
    # camera-centre eigenvectors (columns, descending eigenvalues): A v = lambda v
    S = Bc[:, 3:6, 3:6]
    V = np.transpose(cvec.reshape(C, 3, 3), (0, 2, 1))
    w = np.linalg.eigvalsh(S)[:, ::-1]
    res = np.einsum("bij,bjk->bik", S, V) - V * w[:, None, :]
    assert np.max(np.abs(res) / np.abs(w).max(axis=1)[:, None, None]) < 1e-10


def test_cpp_accessors_match_the_reference_test(prog, tmp_path):
    """The expectations of covarianceEigenValues_test.cpp:81-136 on output.cov,
    through the C++ Uncertainty accessors."""
    exe, _ = prog
    g = golden("daliborka")
    e = golden("eigvalues")
    packed = str(tmp_path / "packed.bin")
    np.concatenate([g["gold_cam"].reshape(-1), g["gold_pt"].reshape(-1)]).tofile(packed)
    out = str(tmp_path / "acc.bin")
    C, P = 64, 200
    subprocess.run([exe, "--accessors", str(C), str(P), packed, out], check=True, timeout=120)
    cam5, pt143, cams, pts, cev, pev = _read(out, 81, 9, 81 * C, 9 * P, 9 * C, 3 * P)
    assert np.max(np.abs(cam5 - e["cam5"].reshape(-1))) < 1e-5
    assert np.max(np.abs(pt143 - e["pt143"].reshape(-1))) < 1e-5
    assert np.max(np.abs(cams - e["cams"].reshape(-1))) < 1e-5
    assert np.max(np.abs(pts - e["pts"].reshape(-1))) < 1e-5
    assert np.all(np.abs(cev - e["cam_eig"].reshape(-1)) <= np.abs(cev) * 1e-5)
    tol = np.maximum(np.abs(pev) * 1e-5, 1e-10)
    assert np.all(np.abs(pev - e["pt_eig"].reshape(-1)) <= tol)


def test_cli_on_daliborka(tmp_path):
    """uncertainty -in=04_Daliborka.jacob -in_form=JACOBIAN -out=X.cov
    (main_uncertainty.cpp:66-93): the .cov it writes against output.cov."""
    jac = golden_jacobian("daliborka")
    g = golden("daliborka")
    path = str(tmp_path / "daliborka.jacob")
    jacob.save_jacob(path, jac)
    out = str(tmp_path / "out.cov")
    exe = os.path.join(LIBDIR, "uncertainty")
    r = subprocess.run([exe, f"-in={path}", "-in_form=JACOBIAN", f"-out={out}"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    hdr, cam, pt = jacob.load_cov(out, jac.num_cams, jac.cam_params)
    assert hdr["Used algorithm"] == "TAYLOR_EXPANSION"
    assert [int(x) for x in hdr["Fixed points"].split(",")] == list(g["gold_fixed"])
    assert int(hdr["TE number of iterations"]) == 14
    np.testing.assert_allclose([float(x) for x in hdr["TE cycle change"].split()], g["gold_cycle_change"],
                               rtol=2e-5)
    assert abs(float(hdr["Used lambda"]) - g["gold_lambda"]) <= 1e-5 * g["gold_lambda"]
    # the file prints 6 significant digits, as the reference's does
    assert block_rel_err(cam, g["gold_cam"], 45) < 2e-5
    assert block_rel_err(pt, g["gold_pt"], 6) < 2e-5
