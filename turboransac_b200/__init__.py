"""B200-native absolute-pose RANSAC (P3P + truncated MSAC + LM) behind the
TurboRANSAC ``estimate_absolute_pose_cuda`` interface.

The compute path is libtbr.so (hand-written sm_100a kernels behind the C ABI in
include/tbr.h); this package is its Python host mirror.
"""
from . import build, scenes
from .api import (RESULT_DTYPE, Batch, BundleOptions_cuda, Server, Camera_cuda, CameraPose_cuda, Context, DeviceFrame,
                  RansacOptions_cuda, RansacStats_cuda, TbrError, bundle_adjust_cuda, default_context,
                  estimate_absolute_pose_cuda, estimate_batch, estimate_batch_device, estimate_batch_device_submit,
                  estimate_batch_submit,
                  BatchTicket, get_inliers_mx)

__all__ = ["RESULT_DTYPE", "Batch", "BatchTicket", "Server", "estimate_batch", "estimate_batch_device", "estimate_batch_submit", "estimate_batch_device_submit", "DeviceFrame", "BundleOptions_cuda", "Camera_cuda", "CameraPose_cuda", "Context", "RansacOptions_cuda",
           "RansacStats_cuda", "TbrError", "bundle_adjust_cuda", "default_context",
           "estimate_absolute_pose_cuda", "get_inliers_mx"]
