"""Generate the golden fixtures in this folder from the reference's own test data.

Run once with the uncertaintyTE source tree (read-only) named by the
REFERENCE_ROOT environment variable:

    REFERENCE_ROOT=<uncertaintyTE checkout> python tests/golden/make_golden.py

It converts the reference's text fixtures into compressed .npz files so the
tests do not need the reference tree at run time:

  daliborka.npz   test/input_jacobians/04_Daliborka.jacob + test/EigValues/output.cov
                  (end-to-end TAYLOR_EXPANSION golden: 64 cams, 200 points)
  cube.npz        test/input_jacobians/01_Cube.jacob (6 cams, 15 pts, fixed 11/12/14)
  toy.npz         test/input_jacobians/03_Toy.jacob (10 cams, 60 pts, no fixed points)
  multipl_01.npz  test/SparseMatrix/multipl_in_01.txt -> multipl_out_01.txt (J^T J)
  inv_sparse_01.npz, inv_dense_01.npz
                  test/{SparseMatrix,DenseMatrix}/inv_in_01.txt -> inv_out_01.txt
  eigvalues.npz   the expected arrays of src/test_eigValues/covarianceEigenValues_test.cpp
                  (Uncertainty accessors on test/EigValues/output.cov): camera #5 and point
                  #143 matrices, all camera / point matrices, all camera / point eigenvalues
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from uncertaintyte_b200.jacob import load_cov, load_jacob  # noqa: E402

REF = os.environ.get("REFERENCE_ROOT", "")


def _jac_arrays(j):
    return dict(header=np.array([j.lam, j.num_cams, j.cam_params, j.num_points, j.num_obs,
                                 j.num_rows, j.num_cols], dtype=np.float64),
                pts2fix=(j.pts2fix if j.pts2fix is not None else np.array([-1, -1, -1])).astype(np.int32),
                rows=j.rows.astype(np.int32), cols=j.cols.astype(np.int32), values=j.values)


def _crs(path):
    t = np.array(open(path).read().split(), dtype=np.float64)
    nr, nc, nnz = int(t[0]), int(t[1]), int(t[2])
    o = 3
    rows = t[o:o + nr + 1].astype(np.int32)
    o += nr + 1
    cols = t[o:o + nnz].astype(np.int32)
    o += nnz
    return np.array([nr, nc]), rows, cols, t[o:o + nnz]


def _dense(path, header):
    t = np.array(open(path).read().split(), dtype=np.float64)
    if header:
        n, m = int(t[0]), int(t[1])
        t = t[2:]
    else:
        n = m = int(round(np.sqrt(t.size)))
    # ScaledDenseMatrix(nr, nc, values) reads the file row by row (ScaledDenseMatrix.cpp:24-32)
    return t.reshape(n, m)


def _res_arrays(path):
    """The `static const double res[] = { ... };` arrays of a test source, in order."""
    import re
    txt = open(path).read()
    return [np.array([float(x) for x in body.replace("\n", " ").split(",") if x.strip()])
            for body in re.findall(r"static const double res\[\]\s*=\s*\{(.*?)\};", txt, flags=re.S)]


def main():
    if not REF:
        sys.exit("set REFERENCE_ROOT to the uncertaintyTE source tree")
    T = os.path.join(REF, "test")
    j = load_jacob(os.path.join(T, "input_jacobians/04_Daliborka.jacob"))
    hdr, cam, pt = load_cov(os.path.join(T, "EigValues/output.cov"), j.num_cams, j.cam_params)
    cc = np.array([float(x) for x in hdr["TE cycle change"].split()])
    np.savez_compressed(os.path.join(HERE, "daliborka.npz"), **_jac_arrays(j), gold_cam=cam,
                        gold_pt=pt, gold_cycle_change=cc, gold_lambda=float(hdr["Used lambda"]),
                        gold_fixed=np.array([int(x) for x in hdr["Fixed points"].split(",")]))
    for name, fn in [("cube", "01_Cube.jacob"), ("toy", "03_Toy.jacob")]:
        j = load_jacob(os.path.join(T, "input_jacobians", fn))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **_jac_arrays(j))
    dims, r, c, v = _crs(os.path.join(T, "SparseMatrix/multipl_in_01.txt"))
    odims, orr, oc, ov = _crs(os.path.join(T, "SparseMatrix/multipl_out_01.txt"))
    np.savez_compressed(os.path.join(HERE, "multipl_01.npz"), in_dims=dims, in_rows=r, in_cols=c,
                        in_vals=v, out_dims=odims, out_rows=orr, out_cols=oc, out_vals=ov)
    for name, d, h in [("inv_sparse_01", "SparseMatrix", True), ("inv_dense_01", "DenseMatrix", False)]:
        A = _dense(os.path.join(T, d, "inv_in_01.txt"), h)
        B = _dense(os.path.join(T, d, "inv_out_01.txt"), h)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), A=A, Ainv=B)
    cam5, pt143, cams, pts, cam_eig, pt_eig = _res_arrays(
        os.path.join(REF, "src", "test_eigValues", "covarianceEigenValues_test.cpp"))
    np.savez_compressed(os.path.join(HERE, "eigvalues.npz"), cam5=cam5.reshape(9, 9), pt143=pt143.reshape(3, 3),
                        cams=cams.reshape(-1, 9, 9), pts=pts.reshape(-1, 3, 3), cam_eig=cam_eig.reshape(-1, 9),
                        pt_eig=pt_eig.reshape(-1, 3))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
