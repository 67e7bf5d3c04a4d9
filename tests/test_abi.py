"""The C ABI library loads and exports every symbol include/uncte.h declares
(host-only calls; nothing here touches a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT
from uncertaintyte_b200 import native


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(unc_[a-z_0-9]+)\s*\(", txt)))


def test_header_functions_are_exported():
    names = _declared("uncte.h")
    assert "unc_compute" in names and "unc_compute_device" in names
    lib = ctypes.CDLL(native.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(native.EXPORTS) == names


def test_cpp_dropin_symbols_exported():
    out = subprocess.run(["nm", "-D", "-C", native.LIB_PATH], capture_output=True, text=True).stdout
    assert "getCovariances(cov::Options&, cov::Statistic&, ceres::CRSMatrix&, double*, double*)" in out
    assert "getCovariances(cov::Options&, cov::Statistic&, ceres::CRSMatrix&, double*, cov::Uncertainty&)" in out
    assert "computeCovariances(cov::Options&, cov::Statistic&, ceres::CRSMatrix&, double*, double*)" in out


def test_status_strings_and_defaults():
    L = native.lib()
    assert L.unc_status_string(0) == b"UNC_OK"
    assert L.unc_status_string(-2) == b"UNC_ERR_LAYOUT"
    assert L.unc_status_string(-6) == b"UNC_ERR_SINGULAR"
    o = native.UncOptions()
    L.unc_options_init(ctypes.byref(o), 10, 9, 500, 3000)
    assert o.algorithm == 2 and o.lam == -1 and o.epsilon == 1e-10
    assert o.svd_remove_n == -1 and o.max_iter_te == -1 and o.precision == 0


def test_option_validation_is_host_side():
    """Invalid options fail before any CUDA call."""
    from conftest import golden_jacobian
    jac = golden_jacobian("toy")  # no fixed points
    with pytest.raises(native.UncError) as e:
        native.compute_covariances(jac)
    assert e.value.status == -3  # UNC_ERR_NO_FIXED_POINTS
    jac = golden_jacobian("cube")
    jac.cam_params = 7
    with pytest.raises(native.UncError) as e:
        native.compute_covariances(jac)
    assert e.value.status == -7  # UNC_ERR_UNSUPPORTED


def test_svd_option_validation_is_host_side():
    """The SVD algorithms densify (9C + 3P)^2 J^T J: sizes above 46000 and more
    than 31 removed singular values are refused before any CUDA call."""
    from conftest import golden_jacobian
    jac = golden_jacobian("cube")
    jac.num_points += 20000
    jac.num_cols = 9 * jac.num_cams + 3 * jac.num_points
    with pytest.raises(native.UncError) as e:
        native.compute_covariances(jac, algorithm=0)
    assert e.value.status == -8  # UNC_ERR_TOO_LARGE
    jac = golden_jacobian("cube")
    jac.svd_remove_n = 40
    with pytest.raises(native.UncError) as e:
        native.compute_covariances(jac, algorithm=1)
    assert e.value.status == -7  # UNC_ERR_UNSUPPORTED


def test_workspace_estimate_scales_with_cameras():
    from conftest import golden_jacobian
    jac = golden_jacobian("daliborka")
    b = native.workspace_bytes(jac)
    n = 9 * jac.num_cams
    assert b > 4 * n * n * 8  # four dense N x N buffers


def test_cpp_dropin_caller_compiles_and_links(tmp_path):
    """A C++ caller of include/uncertainty.h builds against libuncte.so (the GPU
    tests run it)."""
    exe = str(tmp_path / "dropin_check")
    libdir = os.path.join(ROOT, "uncertaintyte_b200")
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin_check.cpp"), "-o", exe, "-L" + libdir, "-luncte",
                    "-Wl,-rpath," + libdir], check=True)
    assert os.path.exists(exe)
