"""uncertaintyte_b200 - B200 (sm_100a) covariance propagation for uncertaintyTE.

Host-side mirror of uncertaintyTE's `computeCovariances` / `getCovariances`
interface over the CUDA library libuncte.so (C ABI: include/uncte.h, C++
drop-in: include/uncertainty.h).

    from uncertaintyte_b200 import load_jacob, compute_covariances
    jac = load_jacob("scene.jacob")
    cam, pt, stats = compute_covariances(jac)          # 45 values/camera, 6/point
"""
from .jacob import ALGORITHMS, Jacobian, load_cov, load_jacob, save_cov, save_jacob  # noqa: F401
from .native import (Context, UncError, compute_covariances, compute_covariances_device,  # noqa: F401
                     dense_inverse_device, jtj_crs, kernel_launches, make_options, workspace_bytes)

__all__ = ["Jacobian", "load_jacob", "save_jacob", "load_cov", "save_cov", "ALGORITHMS", "Context",
           "UncError", "compute_covariances", "compute_covariances_device", "dense_inverse_device",
           "jtj_crs", "kernel_launches", "make_options", "workspace_bytes"]
